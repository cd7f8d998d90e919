// Cell-loop kernels for domain (material) cells: the device form of PETSc's
// DMPlexComputeResidualByKey / DMPlexComputeJacobianByKey / DMProjectFieldLocal as PyLith's
// IntegratorDomain drives them (libsrc/pylith/feassemble/IntegratorDomain.cc:422-590).
//
// One thread per cell: gather the cell's closure (corner coordinates, nodal solution),
// form geometry at each quadrature point, evaluate the solution gradient, call the
// pointwise kernels with PETSc's argument list, contract with the basis gradients
//     r_a[c] += w |J| ( f0[c] phi_a + sum_d f1[c*3+d] dphi_a/dx_d ),
// and add the element vector into the output with FP64 atomics.
#pragma once

#include "elements.cuh"
#include "pointwise.cuh"

namespace plb {

enum DomainOp { OP_RESIDUAL = 0, OP_JACOBIAN_ACTION = 1 };

struct DomainParams {
    const int32_t* cells;      // [mesh cells][nen]
    const double* coords;      // [nodes][3]
    const int32_t* cell_ids;   // integrator cell -> mesh cell (NULL: identity)
    int64_t ncells;            // integrator cells
    const double* u;           // solution (local vector)
    const double* v;           // direction for the Jacobian action
    double* out;
    const float* v32;          // FP32 Jacobian action
    float* out32;
    // aux subfields, device SoA indexed by integrator cell
    const double* mu;
    const double* K;
    const double* body_force;  // [3][ncells]
    const double* tau;         // [3][ncells]
    const double* ratio;       // [3][ncells]
    double* visc;              // [18][nq][ncells]
    double* total;             // [6][nq][ncells]
    double t, dt, s_tshift;
    int num_constants;
    double constants[8];
    unsigned int* err;
    const float* lm32;  // FP32 Jacobian action (hexahedra, tetrahedra): per-cell (lambda, mu) of the
                        // isotropic tangent at (t, dt), or NULL to evaluate the tangent per point
};

// ---- elements --------------------------------------------------------------------------
template <int CELL>
struct Elem;

template <>
struct Elem<TET4> {
    static constexpr int nen = 4, nq = 1, ngeom = 4;
    PL_D static int corner(int c) { return c; }
    PL_D static void geom(const double X[][3], int q, Geom* g) { tet_geometry(X, g); }
    PL_D static void grad(const Geom& g, int q, int n, double out[3]) { tet_grad(g, n, out); }
    PL_D static double phi(int q, int n) { return 0.25; }
    PL_D static void centre_geom(const double X[][3], Geom* g) { tet_geometry(X, g); }
    PL_D static void centre_grad(const Geom& g, int n, double out[3]) { tet_grad(g, n, out); }
};

template <>
struct Elem<HEX8> {
    static constexpr int nen = 8, nq = 8, ngeom = 8;
    PL_D static int corner(int c) { return c; }
    PL_D static void geom(const double X[][3], int q, Geom* g) {
        hex_geometry<2>(X, q & 1, (q >> 1) & 1, q >> 2, 1.0, g);
    }
    PL_D static void grad(const Geom& g, int q, int n, double out[3]) {
        double d[3];
        hex_corner_dN<2>(n, q & 1, (q >> 1) & 1, q >> 2, d);
#pragma unroll
        for (int j = 0; j < 3; ++j) out[j] = d[0] * g.inv[0][j] + d[1] * g.inv[1][j] + d[2] * g.inv[2][j];
    }
    PL_D static double phi(int q, int n) {
        return hex_corner_N(n, gauss2_x(q & 1), gauss2_x((q >> 1) & 1), gauss2_x(q >> 2));
    }
    PL_D static void centre_geom(const double X[][3], Geom* g) { hex_geometry_centre(X, g); }
    PL_D static void centre_grad(const Geom& g, int n, double out[3]) {
        const double d[3] = {lin_d(hex_cx(n)) * 0.25, lin_d(hex_cy(n)) * 0.25, lin_d(hex_cz(n)) * 0.25};
#pragma unroll
        for (int j = 0; j < 3; ++j) out[j] = d[0] * g.inv[0][j] + d[1] * g.inv[1][j] + d[2] * g.inv[2][j];
    }
};

template <>
struct Elem<HEX27> {
    static constexpr int nen = 27, nq = 27, ngeom = 8;
    PL_D static int corner(int c) { return 2 * hex_cx(c) + 6 * hex_cy(c) + 18 * hex_cz(c); }
    PL_D static void geom(const double X[][3], int q, Geom* g) {
        const int qi = q % 3, qj = (q / 3) % 3, qk = q / 9;
        hex_geometry<3>(X, qi, qj, qk, gauss3_w(qi) * gauss3_w(qj) * gauss3_w(qk), g);
    }
    PL_D static void grad(const Geom& g, int q, int n, double out[3]) {
        const double x = gauss3_x(q % 3), y = gauss3_x((q / 3) % 3), z = gauss3_x(q / 9);
        const int a = n % 3, b = (n / 3) % 3, c = n / 9;
        const double d[3] = {quad_d(a, x) * quad_v(b, y) * quad_v(c, z),
                             quad_v(a, x) * quad_d(b, y) * quad_v(c, z),
                             quad_v(a, x) * quad_v(b, y) * quad_d(c, z)};
#pragma unroll
        for (int j = 0; j < 3; ++j) out[j] = d[0] * g.inv[0][j] + d[1] * g.inv[1][j] + d[2] * g.inv[2][j];
    }
    PL_D static double phi(int q, int n) {
        const double x = gauss3_x(q % 3), y = gauss3_x((q / 3) % 3), z = gauss3_x(q / 9);
        return quad_v(n % 3, x) * quad_v((n / 3) % 3, y) * quad_v(n / 9, z);
    }
    PL_D static void centre_geom(const double X[][3], Geom* g) { hex_geometry_centre(X, g); }
    PL_D static void centre_grad(const Geom& g, int n, double out[3]) {
        const int a = n % 3, b = (n / 3) % 3, c = n / 9;
        const double d[3] = {quad_d(a, 0.0) * quad_v(b, 0.0) * quad_v(c, 0.0),
                             quad_v(a, 0.0) * quad_d(b, 0.0) * quad_v(c, 0.0),
                             quad_v(a, 0.0) * quad_v(b, 0.0) * quad_d(c, 0.0)};
#pragma unroll
        for (int j = 0; j < 3; ++j) out[j] = d[0] * g.inv[0][j] + d[1] * g.inv[1][j] + d[2] * g.inv[2][j];
    }
};

// ---- aux assembly in the reference's subfield order ----------------------------------
// Domain aux subfields: density, [body_force], shear_modulus, bulk_modulus, then for the
// generalized Maxwell model maxwell_time(3), shear_modulus_ratio(3), viscous_strain(18),
// total_strain(6) (libsrc/pylith/materials/Elasticity.cc:233-240,
// IsotropicLinearGenMaxwell.cc:94-102). Density is not read by the quasi-static kernels.
template <int RHEO, bool BF>
struct AuxLayout;

template <bool BF>
struct AuxLayout<RHEO_ILE, BF> {
    static constexpr int numA = BF ? 4 : 3;
    static constexpr int size = BF ? 6 : 3;
    PL_D static int off(int i) { return BF ? (i == 0 ? 0 : (i == 1 ? 1 : (i == 2 ? 4 : 5))) : i; }
    PL_D static void load_cell(const DomainParams& p, int64_t c, double* a) {
        a[0] = 0.0;
        if (BF) {
            a[1] = p.body_force[c];
            a[2] = p.body_force[p.ncells + c];
            a[3] = p.body_force[2 * p.ncells + c];
        }
        a[off(numA - 2)] = p.mu[c];
        a[off(numA - 1)] = p.K[c];
    }
    PL_D static void load_qp(const DomainParams&, int64_t, int, int, double*) {}
};

template <bool BF>
struct AuxLayout<RHEO_GENMAXWELL, BF> {
    static constexpr int numA = BF ? 8 : 7;
    static constexpr int base = BF ? 4 : 1;  // offset of shear_modulus
    static constexpr int size = base + 2 + 3 + 3 + 18 + 6;
    PL_D static int off(int i) {
        // density 0, [body_force 1..3], mu, K, tau(3), ratio(3), visc(18), total(6)
        if (i == 0) return 0;
        if (BF && i == 1) return 1;
        const int j = i - (BF ? 2 : 1);  // 0: mu, 1: K, 2: tau, 3: ratio, 4: visc, 5: total
        const int o[6] = {0, 1, 2, 5, 8, 26};
        return base + o[j];
    }
    PL_D static void load_cell(const DomainParams& p, int64_t c, double* a) {
        a[0] = 0.0;
        if (BF) {
            a[1] = p.body_force[c];
            a[2] = p.body_force[p.ncells + c];
            a[3] = p.body_force[2 * p.ncells + c];
        }
        a[base + 0] = p.mu[c];
        a[base + 1] = p.K[c];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            a[base + 2 + i] = p.tau[i * p.ncells + c];
            a[base + 5 + i] = p.ratio[i * p.ncells + c];
        }
    }
    PL_D static void load_qp(const DomainParams& p, int64_t c, int q, int nq, double* a) {
#pragma unroll
        for (int k = 0; k < 18; ++k) a[base + 8 + k] = p.visc[((int64_t)k * nq + q) * p.ncells + c];
#pragma unroll
        for (int k = 0; k < 6; ++k) a[base + 26 + k] = p.total[((int64_t)k * nq + q) * p.ncells + c];
    }
};

template <int RHEO, bool BF>
struct AuxOffsets {
    int v[AuxLayout<RHEO, BF>::numA];
    PL_D AuxOffsets() {
#pragma unroll
        for (int i = 0; i < AuxLayout<RHEO, BF>::numA; ++i) v[i] = AuxLayout<RHEO, BF>::off(i);
    }
};

// Pointwise dispatch for the registered rheology.
template <int RHEO>
PL_D void call_f1(int numA, const int* aOff, const double* a, const double* s, const double* s_x,
                  const DomainParams& p, const double* x, double* f1) {
    const int sOff[1] = {0}, sOff_x[1] = {0};
    if (RHEO == RHEO_ILE)
        pw::ile3d_f1v<double>(3, 1, numA, sOff, sOff_x, s, nullptr, s_x, aOff, nullptr, a, nullptr,
                              nullptr, p.t, x, p.num_constants, p.constants, f1);
    else
        pw::gm3d_f1v<double>(3, 1, numA, sOff, sOff_x, s, nullptr, s_x, aOff, nullptr, a, nullptr,
                             nullptr, p.t, x, p.num_constants, p.constants, f1);
}

template <int RHEO>
PL_D void call_jf3(int numA, const int* aOff, const double* a, const DomainParams& p,
                   const double* x, double* Jf3) {
    const int sOff[1] = {0}, sOff_x[1] = {0};
    if (RHEO == RHEO_ILE)
        pw::ile3d_Jf3vu<double>(3, 1, numA, sOff, sOff_x, nullptr, nullptr, nullptr, aOff, nullptr,
                                a, nullptr, nullptr, p.t, p.s_tshift, x, p.num_constants,
                                p.constants, Jf3);
    else
        pw::gm3d_Jf3vu<double>(3, 1, numA, sOff, sOff_x, nullptr, nullptr, nullptr, aOff, nullptr,
                               a, nullptr, nullptr, p.t, p.s_tshift, x, p.num_constants,
                               p.constants, Jf3);
}

// f1 = Jf3 : s_x for the registered tangent of either rheology on this path. Both are isotropic,
// Jf3 = -C with C = lambda d_ij d_kl + mu (d_ik d_jl + d_il d_jk) (generalized Maxwell with its
// effective shear modulus), so the tangent is evaluated by its registered function and contracted
// in closed form from its (f,g,df,dg) = (0,1,0,1) and (0,1,1,0) entries, -lambda and -mu: 12
// multiply-adds instead of 81 (the 81-entry contraction cannot drop its zero entries).
template <typename T>
PL_D void isotropic_contract(T lam, T mu, const T s_x[9], T f1[9]) {
    const T ltr = lam * (s_x[0] + s_x[4] + s_x[8]);
#pragma unroll
    for (int f = 0; f < 3; ++f)
#pragma unroll
        for (int df = 0; df < 3; ++df) f1[f * 3 + df] = -(mu * (s_x[f * 3 + df] + s_x[df * 3 + f]) + (f == df ? ltr : T(0)));
}
template <int RHEO, typename T>
PL_D void isotropic_jf3_contract(const double Jf3[81], const T s_x[9], T f1[9]) {
    static_assert(RHEO == RHEO_ILE || RHEO == RHEO_GENMAXWELL, "isotropic tangents only");
    isotropic_contract<T>((T)(-Jf3[((0 * 3 + 1) * 3 + 0) * 3 + 1]), (T)(-Jf3[((0 * 3 + 1) * 3 + 1) * 3 + 0]), s_x, f1);
}

}  // namespace plb
