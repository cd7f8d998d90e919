// Domain cell-loop kernels (thread per cell, atomic scatter) and their launchers.
#include "domain_kernels.cuh"
#include "internal.hpp"
#include "launch.hpp"

namespace plb {

// Residual (OP_RESIDUAL) or matrix-free Jacobian action (OP_JACOBIAN_ACTION) of one
// domain integrator; FP64 throughout.
template <int CELL, int RHEO, bool BF, int OP>
__global__ void __launch_bounds__(128) k_domain_apply(DomainParams p) {
    using E = Elem<CELL>;
    using L = AuxLayout<RHEO, BF>;
    const AuxOffsets<RHEO, BF> aoff;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < p.ncells;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t mc = p.cell_ids ? p.cell_ids[c] : c;
        const int32_t* cn = p.cells + mc * E::nen;
        int nodes[E::nen];
#pragma unroll
        for (int n = 0; n < E::nen; ++n) nodes[n] = cn[n];
        double X[E::ngeom][3];
#pragma unroll
        for (int k = 0; k < E::ngeom; ++k)
#pragma unroll
            for (int i = 0; i < 3; ++i) X[k][i] = p.coords[3 * (int64_t)nodes[E::corner(k)] + i];
        const double* field = OP == OP_RESIDUAL ? p.u : p.v;
        double a[L::size] = {};
        L::load_cell(p, c, a);
        double acc[E::nen * 3];
#pragma unroll
        for (int i = 0; i < E::nen * 3; ++i) acc[i] = 0.0;
#pragma unroll 1
        for (int q = 0; q < E::nq; ++q) {
            Geom g;
            E::geom(X, q, &g);
            if (!(g.detJ > 0.0)) flag_error(p.err, CHECK_NONPOSITIVE_DETJ);
            double s[3] = {0, 0, 0}, s_x[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int n = 0; n < E::nen; ++n) {
                double gr[3];
                E::grad(g, q, n, gr);
                const double* un = field + 3 * (int64_t)nodes[n];
                const double u0 = un[0], u1 = un[1], u2 = un[2];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    s_x[0 + d] += u0 * gr[d];
                    s_x[3 + d] += u1 * gr[d];
                    s_x[6 + d] += u2 * gr[d];
                }
            }
            if (OP == OP_RESIDUAL) L::load_qp(p, c, q, E::nq, a);  // the tangents read no state
            double x[3] = {0, 0, 0};
            double f0[3] = {0, 0, 0}, f1[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            if (OP == OP_RESIDUAL) {
                if (BF) {
                    const int sOff[1] = {0}, sOff_x[1] = {0};
                    pw::g0v_bodyforce<double>(3, 1, L::numA, sOff, sOff_x, s, nullptr, s_x, aoff.v,
                                              nullptr, a, nullptr, nullptr, p.t, x,
                                              p.num_constants, p.constants, f0);
                }
                call_f1<RHEO>(L::numA, aoff.v, a, s, s_x, p, x, f1);
            } else {
                double Jf3[81];
#pragma unroll
                for (int i = 0; i < 81; ++i) Jf3[i] = 0.0;
                call_jf3<RHEO>(L::numA, aoff.v, a, p, x, Jf3);
                // f1[f][df] = sum_{g,dg} Jf3[f][g][df][dg] dv_g/dx_dg
#pragma unroll
                for (int f = 0; f < 3; ++f)
#pragma unroll
                    for (int df = 0; df < 3; ++df) {
                        double acc1 = 0.0;
#pragma unroll
                        for (int gg = 0; gg < 3; ++gg)
#pragma unroll
                            for (int dg = 0; dg < 3; ++dg)
                                acc1 += Jf3[((f * 3 + gg) * 3 + df) * 3 + dg] * s_x[gg * 3 + dg];
                        f1[f * 3 + df] = acc1;
                    }
            }
#pragma unroll
            for (int n = 0; n < E::nen; ++n) {
                double gr[3];
                E::grad(g, q, n, gr);
                const double ph = BF && OP == OP_RESIDUAL ? E::phi(q, n) : 0.0;
#pragma unroll
                for (int cc = 0; cc < 3; ++cc)
                    acc[n * 3 + cc] += g.wdetJ * (f0[cc] * ph + f1[cc * 3 + 0] * gr[0] +
                                                  f1[cc * 3 + 1] * gr[1] + f1[cc * 3 + 2] * gr[2]);
            }
        }
#pragma unroll
        for (int n = 0; n < E::nen; ++n)
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) red_add(&p.out[3 * (int64_t)nodes[n] + cc], acc[n * 3 + cc]);
    }
}

// FP32 Jacobian action: FP64 geometry per cell, FP32 operand/accumulation.
template <int CELL, int RHEO>
__global__ void __launch_bounds__(128) k_domain_jv_f32(DomainParams p) {
    using E = Elem<CELL>;
    using L = AuxLayout<RHEO, false>;
    const AuxOffsets<RHEO, false> aoff;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < p.ncells;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t mc = p.cell_ids ? p.cell_ids[c] : c;
        const int32_t* cn = p.cells + mc * E::nen;
        int nodes[E::nen];
#pragma unroll
        for (int n = 0; n < E::nen; ++n) nodes[n] = cn[n];
        double X[E::ngeom][3];
#pragma unroll
        for (int k = 0; k < E::ngeom; ++k)
#pragma unroll
            for (int i = 0; i < 3; ++i) X[k][i] = p.coords[3 * (int64_t)nodes[E::corner(k)] + i];
        double a[L::size] = {};
        L::load_cell(p, c, a);
        float acc[E::nen * 3];
#pragma unroll
        for (int i = 0; i < E::nen * 3; ++i) acc[i] = 0.0f;
#pragma unroll 1
        for (int q = 0; q < E::nq; ++q) {
            Geom g;
            E::geom(X, q, &g);
            float s_x[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int n = 0; n < E::nen; ++n) {
                double grd[3];
                E::grad(g, q, n, grd);
                const float gr[3] = {(float)grd[0], (float)grd[1], (float)grd[2]};
                const float* vn = p.v32 + 3 * (int64_t)nodes[n];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    s_x[0 + d] += vn[0] * gr[d];
                    s_x[3 + d] += vn[1] * gr[d];
                    s_x[6 + d] += vn[2] * gr[d];
                }
            }
            // the tangents (Jf3vu of both rheologies) read no per-point state
            double x[3] = {0, 0, 0};
            double Jf3d[81];
#pragma unroll
            for (int i = 0; i < 81; ++i) Jf3d[i] = 0.0;
            call_jf3<RHEO>(L::numA, aoff.v, a, p, x, Jf3d);
            float f1[9];
#pragma unroll
            for (int f = 0; f < 3; ++f)
#pragma unroll
                for (int df = 0; df < 3; ++df) {
                    float acc1 = 0.0f;
#pragma unroll
                    for (int gg = 0; gg < 3; ++gg)
#pragma unroll
                        for (int dg = 0; dg < 3; ++dg)
                            acc1 += (float)Jf3d[((f * 3 + gg) * 3 + df) * 3 + dg] * s_x[gg * 3 + dg];
                    f1[f * 3 + df] = acc1;
                }
            const float w = (float)g.wdetJ;
#pragma unroll
            for (int n = 0; n < E::nen; ++n) {
                double grd[3];
                E::grad(g, q, n, grd);
#pragma unroll
                for (int cc = 0; cc < 3; ++cc)
                    acc[n * 3 + cc] += w * (f1[cc * 3 + 0] * (float)grd[0] + f1[cc * 3 + 1] * (float)grd[1] +
                                            f1[cc * 3 + 2] * (float)grd[2]);
            }
        }
#pragma unroll
        for (int n = 0; n < E::nen; ++n)
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) red_add(&p.out32[3 * (int64_t)nodes[n] + cc], acc[n * 3 + cc]);
    }
}

// Element Jacobians from the pointwise Jf3 (g3) contraction, added into a 3x3-block CSR
// matrix at precomputed block positions (DMPlexComputeJacobianByKey + MatSetClosure).
template <int CELL, int RHEO>
__global__ void __launch_bounds__(128) k_domain_jacobian(DomainParams p, const int32_t* pos,
                                                         double* vals) {
    using E = Elem<CELL>;
    using L = AuxLayout<RHEO, false>;
    const AuxOffsets<RHEO, false> aoff;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < p.ncells;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t mc = p.cell_ids ? p.cell_ids[c] : c;
        const int32_t* cn = p.cells + mc * E::nen;
        double X[E::ngeom][3];
#pragma unroll
        for (int k = 0; k < E::ngeom; ++k)
#pragma unroll
            for (int i = 0; i < 3; ++i) X[k][i] = p.coords[3 * (int64_t)cn[E::corner(k)] + i];
        double a[L::size] = {};
        L::load_cell(p, c, a);
        const int32_t* cpos = pos + mc * E::nen * E::nen;
#pragma unroll 1
        for (int q = 0; q < E::nq; ++q) {
            Geom g;
            E::geom(X, q, &g);
            if (!(g.detJ > 0.0)) flag_error(p.err, CHECK_NONPOSITIVE_DETJ);
            // the tangents (Jf3vu of both rheologies) read no per-point state
            double x[3] = {0, 0, 0};
            double Jf3[81];
#pragma unroll
            for (int i = 0; i < 81; ++i) Jf3[i] = 0.0;
            call_jf3<RHEO>(L::numA, aoff.v, a, p, x, Jf3);
#pragma unroll 1
            for (int an = 0; an < E::nen; ++an) {
                double ga[3];
                E::grad(g, q, an, ga);
                // t[g][dg] = sum_df ga[df] Jf3[f][g][df][dg], per f
#pragma unroll 1
                for (int bn = 0; bn < E::nen; ++bn) {
                    double gb[3];
                    E::grad(g, q, bn, gb);
                    double* blk = vals + 9 * (int64_t)cpos[an * E::nen + bn];
#pragma unroll
                    for (int f = 0; f < 3; ++f)
#pragma unroll
                        for (int gg = 0; gg < 3; ++gg) {
                            double v = 0.0;
#pragma unroll
                            for (int df = 0; df < 3; ++df)
#pragma unroll
                                for (int dg = 0; dg < 3; ++dg)
                                    v += ga[df] * Jf3[((f * 3 + gg) * 3 + df) * 3 + dg] * gb[dg];
                            red_add(&blk[f * 3 + gg], g.wdetJ * v);
                        }
                }
            }
        }
    }
}

// DMProjectFieldLocal at quadrature points for the generalized Maxwell state: new viscous
// strain from the previous viscous and total strain, then the new total strain; both kernels
// see the previous state (IntegratorDomain.cc:555-590), written back in place.
template <int CELL>
__global__ void __launch_bounds__(128) k_domain_update_state(DomainParams p) {
    using E = Elem<CELL>;
    using L = AuxLayout<RHEO_GENMAXWELL, false>;
    const AuxOffsets<RHEO_GENMAXWELL, false> aoff;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < p.ncells;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t mc = p.cell_ids ? p.cell_ids[c] : c;
        const int32_t* cn = p.cells + mc * E::nen;
        int nodes[E::nen];
#pragma unroll
        for (int n = 0; n < E::nen; ++n) nodes[n] = cn[n];
        double X[E::ngeom][3];
#pragma unroll
        for (int k = 0; k < E::ngeom; ++k)
#pragma unroll
            for (int i = 0; i < 3; ++i) X[k][i] = p.coords[3 * (int64_t)nodes[E::corner(k)] + i];
        double a[L::size] = {};
        L::load_cell(p, c, a);
#pragma unroll 1
        for (int q = 0; q < E::nq; ++q) {
            Geom g;
            E::geom(X, q, &g);
            double s_x[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int n = 0; n < E::nen; ++n) {
                double gr[3];
                E::grad(g, q, n, gr);
                const double* un = p.u + 3 * (int64_t)nodes[n];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    s_x[0 + d] += un[0] * gr[d];
                    s_x[3 + d] += un[1] * gr[d];
                    s_x[6 + d] += un[2] * gr[d];
                }
            }
            L::load_qp(p, c, q, E::nq, a);
            const int sOff[1] = {0}, sOff_x[1] = {0};
            double x[3] = {0, 0, 0};
            double visc[18], tot[6];
            pw::gm3d_viscous_strain<double>(3, 1, L::numA, sOff, sOff_x, nullptr, nullptr, s_x,
                                            aoff.v, nullptr, a, nullptr, nullptr, p.t, x,
                                            p.num_constants, p.constants, visc);
            pw::el3d_strain_vector<double>(3, 1, L::numA, sOff, sOff_x, nullptr, nullptr, s_x,
                                           aoff.v, nullptr, a, nullptr, nullptr, p.t, x,
                                           p.num_constants, p.constants, tot);
#pragma unroll
            for (int k = 0; k < 18; ++k) p.visc[((int64_t)k * E::nq + q) * p.ncells + c] = visc[k];
#pragma unroll
            for (int k = 0; k < 6; ++k) p.total[((int64_t)k * E::nq + q) * p.ncells + c] = tot[k];
        }
    }
}

// Derived fields of basis order 0 (IntegratorDomain::_computeDerivedField,
// IntegratorDomain.cc:596-630, with PyLith's default basis order 0 for cauchy_stress and
// cauchy_strain, DerivedSubfieldsElasticity.py:42-44): each registered project kernel evaluated
// at the cell centroid, out[c][6 * k + i] for kernel k. A generalized-Maxwell stress reads the
// state of the cell's single quadrature point (P1 tetrahedra only).
template <int CELL, int RHEO>
__global__ void __launch_bounds__(128) k_domain_derived(DomainParams p, DerivedSpec spec) {
    using E = Elem<CELL>;
    using L = AuxLayout<RHEO, false>;
    const AuxOffsets<RHEO, false> aoff;
    const int nout = 6 * spec.n;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < p.ncells;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t mc = p.cell_ids ? p.cell_ids[c] : c;
        const int32_t* cn = p.cells + mc * E::nen;
        double X[E::ngeom][3];
#pragma unroll
        for (int k = 0; k < E::ngeom; ++k)
#pragma unroll
            for (int i = 0; i < 3; ++i) X[k][i] = p.coords[3 * (int64_t)cn[E::corner(k)] + i];
        Geom g;
        E::centre_geom(X, &g);
        if (!(g.detJ > 0.0)) flag_error(p.err, CHECK_NONPOSITIVE_DETJ);
        double s_x[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int n = 0; n < E::nen; ++n) {
            double gr[3];
            E::centre_grad(g, n, gr);
            const double* un = p.u + 3 * (int64_t)cn[n];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                s_x[0 + d] += un[0] * gr[d];
                s_x[3 + d] += un[1] * gr[d];
                s_x[6 + d] += un[2] * gr[d];
            }
        }
        double a[L::size] = {};
        L::load_cell(p, c, a);
        L::load_qp(p, c, 0, E::nq, a);
        const int sOff[1] = {0}, sOff_x[1] = {0};
        double x[3] = {0, 0, 0};
        for (int k = 0; k < spec.n; ++k) {
            double o[6] = {0, 0, 0, 0, 0, 0};
            if (spec.kind[k] == K_EL_STRAIN_VECTOR)
                pw::el3d_strain_vector<double>(3, 1, L::numA, sOff, sOff_x, nullptr, nullptr, s_x, aoff.v, nullptr, a,
                                               nullptr, nullptr, p.t, x, p.num_constants, p.constants, o);
            else if (RHEO == RHEO_ILE && spec.kind[k] == K_ILE_STRESS_VECTOR)
                pw::ile3d_stress_vector<double>(3, 1, L::numA, sOff, sOff_x, nullptr, nullptr, s_x, aoff.v, nullptr, a,
                                                nullptr, nullptr, p.t, x, p.num_constants, p.constants, o);
            else if (RHEO == RHEO_GENMAXWELL && spec.kind[k] == K_GM_STRESS_VECTOR)
                pw::gm3d_stress_vector<double>(3, 1, L::numA, sOff, sOff_x, nullptr, nullptr, s_x, aoff.v, nullptr, a,
                                               nullptr, nullptr, p.t, x, p.num_constants, p.constants, o);
#pragma unroll
            for (int i = 0; i < 6; ++i) p.out[c * nout + 6 * k + i] = o[i];
        }
    }
}

static int grid_for(int64_t n, int threads) {
    const int64_t blocks = (n + threads - 1) / threads;
    return (int)(blocks < 148 * 64 ? (blocks > 0 ? blocks : 1) : 148 * 64);
}

template <int CELL, int RHEO, bool BF>
static void launch_apply_t(const DomainParams& p, int op, cudaStream_t s) {
    const int th = 128;
    if (op == OP_RESIDUAL)
        k_domain_apply<CELL, RHEO, BF, OP_RESIDUAL><<<grid_for(p.ncells, th), th, 0, s>>>(p);
    else
        k_domain_apply<CELL, RHEO, false, OP_JACOBIAN_ACTION><<<grid_for(p.ncells, th), th, 0, s>>>(p);
    count_launch();
}

template <int CELL>
static void launch_apply_cell(const DomainParams& p, int rheo, bool bf, int op, cudaStream_t s) {
    if (rheo == RHEO_ILE) {
        if (bf) launch_apply_t<CELL, RHEO_ILE, true>(p, op, s);
        else launch_apply_t<CELL, RHEO_ILE, false>(p, op, s);
    } else {
        if (bf) launch_apply_t<CELL, RHEO_GENMAXWELL, true>(p, op, s);
        else launch_apply_t<CELL, RHEO_GENMAXWELL, false>(p, op, s);
    }
}

void launch_domain_apply_atomic(const DomainParams& p, int cell, int rheo, bool bf, int op,
                                cudaStream_t s) {
    if (p.ncells == 0) return;
    if (cell == TET4) launch_apply_cell<TET4>(p, rheo, bf, op, s);
    else if (cell == HEX8) launch_apply_cell<HEX8>(p, rheo, bf, op, s);
    else launch_apply_cell<HEX27>(p, rheo, bf, op, s);
}

void launch_domain_jv_f32_atomic(const DomainParams& p, int cell, int rheo, cudaStream_t s) {
    if (p.ncells == 0) return;
    const int th = 128;
    const int gr = grid_for(p.ncells, th);
#define PLB_F32(C, R) k_domain_jv_f32<C, R><<<gr, th, 0, s>>>(p)
    if (cell == TET4) { if (rheo == RHEO_ILE) PLB_F32(TET4, RHEO_ILE); else PLB_F32(TET4, RHEO_GENMAXWELL); }
    else if (cell == HEX8) { if (rheo == RHEO_ILE) PLB_F32(HEX8, RHEO_ILE); else PLB_F32(HEX8, RHEO_GENMAXWELL); }
    else { if (rheo == RHEO_ILE) PLB_F32(HEX27, RHEO_ILE); else PLB_F32(HEX27, RHEO_GENMAXWELL); }
#undef PLB_F32
    count_launch();
}

void launch_domain_jacobian(const DomainParams& p, int cell, int rheo, const int32_t* pos,
                            double* vals, cudaStream_t s) {
    if (p.ncells == 0) return;
    const int th = 128;
    const int gr = grid_for(p.ncells, th);
#define PLB_JAC(C, R) k_domain_jacobian<C, R><<<gr, th, 0, s>>>(p, pos, vals)
    if (cell == TET4) { if (rheo == RHEO_ILE) PLB_JAC(TET4, RHEO_ILE); else PLB_JAC(TET4, RHEO_GENMAXWELL); }
    else if (cell == HEX8) { if (rheo == RHEO_ILE) PLB_JAC(HEX8, RHEO_ILE); else PLB_JAC(HEX8, RHEO_GENMAXWELL); }
    else { if (rheo == RHEO_ILE) PLB_JAC(HEX27, RHEO_ILE); else PLB_JAC(HEX27, RHEO_GENMAXWELL); }
#undef PLB_JAC
    count_launch();
}

void launch_domain_update_state(const DomainParams& p, int cell, cudaStream_t s) {
    if (p.ncells == 0) return;
    const int th = 128;
    const int gr = grid_for(p.ncells, th);
    if (cell == TET4) k_domain_update_state<TET4><<<gr, th, 0, s>>>(p);
    else if (cell == HEX8) k_domain_update_state<HEX8><<<gr, th, 0, s>>>(p);
    else k_domain_update_state<HEX27><<<gr, th, 0, s>>>(p);
    count_launch();
}

void launch_domain_derived(const DomainParams& p, int cell, int rheo, const DerivedSpec& spec, cudaStream_t s) {
    if (p.ncells == 0) return;
    const int th = 128;
    const int gr = grid_for(p.ncells, th);
    if (rheo == RHEO_GENMAXWELL) {
        if (cell == TET4) k_domain_derived<TET4, RHEO_GENMAXWELL><<<gr, th, 0, s>>>(p, spec);
        else if (cell == HEX8) k_domain_derived<HEX8, RHEO_GENMAXWELL><<<gr, th, 0, s>>>(p, spec);
        else k_domain_derived<HEX27, RHEO_GENMAXWELL><<<gr, th, 0, s>>>(p, spec);
    } else {
        if (cell == TET4) k_domain_derived<TET4, RHEO_ILE><<<gr, th, 0, s>>>(p, spec);
        else if (cell == HEX8) k_domain_derived<HEX8, RHEO_ILE><<<gr, th, 0, s>>>(p, spec);
        else k_domain_derived<HEX27, RHEO_ILE><<<gr, th, 0, s>>>(p, spec);
    }
    count_launch();
}

}  // namespace plb
