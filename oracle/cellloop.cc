// ORACLE — test infrastructure only. Nothing in the product library includes,
// links or calls this file; tests/, bench.py's CPU-baseline leg and smoke()
// use it as the oracle.
//
// CPU restatement of the PETSc finite-element cell loop that PyLith drives
// (third-party PETSc >= 3.25.4, not vendored with PyLith; call sites
// libsrc/pylith/feassemble/IntegratorDomain.cc:448 DMPlexComputeResidualByKey,
// :489 DMPlexComputeJacobianByKey, :582 DMProjectFieldLocal, and
// IntegratorInterface.cc:653,714 DMPlexCompute{Residual,Jacobian}HybridByKey).
// The published algorithm (docs/developer/implementation/petsc-fem.md:355-374):
// for each cell, gather the closure, form geometry at each quadrature point,
// evaluate the solution and its gradient, call the pointwise functions f0/f1
// (g0..g3 for Jacobians) and contract with the basis and basis gradients,
//   r_a[c] += w |J| ( f0[c] phi_a + sum_d f1[c*3+d] dphi_a/dx_d ),
// then add the element vector into the local vector (ADD_VALUES).
//
// Elements: P1 tetrahedron (1-point centroid rule), Q1 hexahedron (2x2x2 Gauss)
// and Q2 hexahedron (3x3x3 Gauss, trilinear geometry from the 8 corners).
// Cohesive cells: quadrilateral fault faces with 2x2 Gauss points.
// OpenMP over cells with one residual buffer per thread and a fixed-order
// reduction, so results are deterministic for a given thread count.
#include "pointwise.hh"

#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

using namespace oracle::pw;

namespace {

enum CellType { TET4 = 0, HEX8 = 1, HEX27 = 2 };

struct Element {
    int nen;     // field nodes per cell
    int nq;      // quadrature points
    int ngeom;   // geometry nodes (corners)
    std::vector<double> qw;        // [nq]
    std::vector<double> phi;       // [nq][nen]
    std::vector<double> dphi;      // [nq][nen][3] reference derivatives
    std::vector<double> gphi;      // [nq][ngeom] geometry basis
    std::vector<double> dgphi;     // [nq][ngeom][3]
    std::vector<int> corner;       // [ngeom] local index of each geometry node in the cell
};

// 1D Lagrange basis on nodes {-1, 1} (linear) or {-1, 0, 1} (quadratic).
void lagrange1d(int order, double x, double* v, double* d) {
    if (order == 1) {
        v[0] = 0.5 * (1.0 - x); v[1] = 0.5 * (1.0 + x);
        d[0] = -0.5; d[1] = 0.5;
    } else {
        v[0] = 0.5 * x * (x - 1.0); v[1] = 1.0 - x * x; v[2] = 0.5 * x * (x + 1.0);
        d[0] = x - 0.5; d[1] = -2.0 * x; d[2] = x + 0.5;
    }
}

void gauss1d(int n, double* x, double* w) {
    if (n == 1) {
        x[0] = 0.0; w[0] = 2.0;
    } else if (n == 2) {
        const double a = 1.0 / std::sqrt(3.0);
        x[0] = -a; x[1] = a; w[0] = w[1] = 1.0;
    } else {
        const double a = std::sqrt(3.0 / 5.0);
        x[0] = -a; x[1] = 0.0; x[2] = a;
        w[0] = 5.0 / 9.0; w[1] = 8.0 / 9.0; w[2] = 5.0 / 9.0;
    }
}

// Hexahedron corner order (0,0,0),(1,0,0),(1,1,0),(0,1,0),(0,0,1),(1,0,1),(1,1,1),(0,1,1).
const int kHexCorner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                              {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};

// centre: a single evaluation point at the cell centroid (the order-0 dual basis of derived
// fields) instead of the quadrature rule.
Element make_element(int type, bool centre = false) {
    Element e;
    if (type == TET4) {
        // Reference tetrahedron (0,0,0),(1,0,0),(0,1,0),(0,0,1); one point at the centroid.
        e.nen = 4; e.nq = 1; e.ngeom = 4;
        e.qw = {1.0 / 6.0};
        e.phi = {0.25, 0.25, 0.25, 0.25};
        e.dphi = {-1, -1, -1, 1, 0, 0, 0, 1, 0, 0, 0, 1};
        e.gphi = e.phi; e.dgphi = e.dphi;
        e.corner = {0, 1, 2, 3};
        return e;
    }
    const int order = (type == HEX8) ? 1 : 2;
    const int np1 = order + 1;          // nodes per direction
    const int nqd = centre ? 1 : ((type == HEX8) ? 2 : 3);
    e.nen = np1 * np1 * np1;
    e.nq = nqd * nqd * nqd;
    e.ngeom = 8;
    double qx[3], qwt[3];
    gauss1d(nqd, qx, qwt);
    e.qw.resize(e.nq);
    e.phi.resize(e.nq * e.nen);
    e.dphi.resize(e.nq * e.nen * 3);
    e.gphi.resize(e.nq * 8);
    e.dgphi.resize(e.nq * 8 * 3);
    for (int k = 0; k < nqd; ++k)
        for (int j = 0; j < nqd; ++j)
            for (int i = 0; i < nqd; ++i) {
                const int q = (k * nqd + j) * nqd + i;
                e.qw[q] = qwt[i] * qwt[j] * qwt[k];
                double vx[3], dx[3], vy[3], dy[3], vz[3], dz[3];
                // field basis
                lagrange1d(order, qx[i], vx, dx);
                lagrange1d(order, qx[j], vy, dy);
                lagrange1d(order, qx[k], vz, dz);
                for (int n = 0; n < e.nen; ++n) {
                    int a, b, c;
                    if (type == HEX8) {
                        a = kHexCorner[n][0]; b = kHexCorner[n][1]; c = kHexCorner[n][2];
                    } else {
                        a = n % 3; b = (n / 3) % 3; c = n / 9;  // lexicographic lattice order
                    }
                    e.phi[q * e.nen + n] = vx[a] * vy[b] * vz[c];
                    e.dphi[(q * e.nen + n) * 3 + 0] = dx[a] * vy[b] * vz[c];
                    e.dphi[(q * e.nen + n) * 3 + 1] = vx[a] * dy[b] * vz[c];
                    e.dphi[(q * e.nen + n) * 3 + 2] = vx[a] * vy[b] * dz[c];
                }
                // geometry basis: trilinear on the corners
                lagrange1d(1, qx[i], vx, dx);
                lagrange1d(1, qx[j], vy, dy);
                lagrange1d(1, qx[k], vz, dz);
                for (int n = 0; n < 8; ++n) {
                    const int a = kHexCorner[n][0], b = kHexCorner[n][1], c = kHexCorner[n][2];
                    e.gphi[q * 8 + n] = vx[a] * vy[b] * vz[c];
                    e.dgphi[(q * 8 + n) * 3 + 0] = dx[a] * vy[b] * vz[c];
                    e.dgphi[(q * 8 + n) * 3 + 1] = vx[a] * dy[b] * vz[c];
                    e.dgphi[(q * 8 + n) * 3 + 2] = vx[a] * vy[b] * dz[c];
                }
            }
    e.corner.resize(8);
    for (int n = 0; n < 8; ++n) {
        if (type == HEX8) {
            e.corner[n] = n;
        } else {
            const int a = 2 * kHexCorner[n][0], b = 2 * kHexCorner[n][1], c = 2 * kHexCorner[n][2];
            e.corner[n] = a + 3 * b + 9 * c;
        }
    }
    return e;
}

struct QPoint {
    double x[3];
    double wdetJ;
    double detJ;
    std::vector<double> gphi;  // [nen][3] physical gradients
};

// Geometry at quadrature point q of cell `cell`: J = sum_a X_a (x) dN_a, physical gradients
// dphi/dx = J^{-T} dphi/dxi.
bool eval_geometry(const Element& e, int q, const int* cellnodes, const double* coords, QPoint* p) {
    double J[3][3] = {{0}};
    p->x[0] = p->x[1] = p->x[2] = 0.0;
    for (int n = 0; n < e.ngeom; ++n) {
        const double* X = &coords[3 * (int64_t)cellnodes[e.corner[n]]];
        const double g = e.gphi[q * e.ngeom + n];
        const double* dg = &e.dgphi[(q * e.ngeom + n) * 3];
        for (int i = 0; i < 3; ++i) {
            p->x[i] += g * X[i];
            for (int j = 0; j < 3; ++j) J[i][j] += X[i] * dg[j];
        }
    }
    const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                       J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                       J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    if (!(det > 0.0)) return false;
    double inv[3][3];
    inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
    inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
    inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
    inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
    inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
    inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
    inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
    inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
    inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
    p->detJ = det;
    p->wdetJ = e.qw[q] * det;
    p->gphi.assign(e.nen * 3, 0.0);
    for (int n = 0; n < e.nen; ++n) {
        const double* d = &e.dphi[(q * e.nen + n) * 3];
        for (int j = 0; j < 3; ++j)
            p->gphi[n * 3 + j] = d[0] * inv[0][j] + d[1] * inv[1][j] + d[2] * inv[2][j];
    }
    return true;
}

// Aux field description shared by the entry points: subfield i has aux_ncomp[i] components and
// is stored per cell (kind 0: [ncells][ncomp]), per quadrature point (kind 1:
// [ncells][nq][ncomp]) or per field node (kind 2: [nnodes][ncomp], interpolated with the cell's
// field basis).
struct Aux {
    int numA;
    const int* kind;
    const int* ncomp;
    const double* const* data;
    std::vector<int> off;
    int total;
    Aux(int n, const int* k, const int* c, const double* const* d) : numA(n), kind(k), ncomp(c), data(d) {
        off.resize(n > 0 ? n : 1);
        total = 0;
        for (int i = 0; i < n; ++i) { off[i] = total; total += c[i]; }
    }
    void eval(const Element& e, int64_t cell, int q, const int* cellnodes, double* a) const {
        for (int i = 0; i < numA; ++i) {
            double* dst = a + off[i];
            const int nc = ncomp[i];
            if (kind[i] == 0) {
                for (int c = 0; c < nc; ++c) dst[c] = data[i][cell * nc + c];
            } else if (kind[i] == 1) {
                for (int c = 0; c < nc; ++c) dst[c] = data[i][(cell * e.nq + q) * nc + c];
            } else {
                for (int c = 0; c < nc; ++c) dst[c] = 0.0;
                for (int n = 0; n < e.nen; ++n) {
                    const double ph = e.phi[q * e.nen + n];
                    for (int c = 0; c < nc; ++c) dst[c] += ph * data[i][(int64_t)cellnodes[n] * nc + c];
                }
            }
        }
    }
};

// Solution value and gradient at a quadrature point for a 3-component field.
void eval_field(const Element& e, int q, const QPoint& p, const int* cellnodes, const double* u,
                double* s, double* s_x) {
    for (int i = 0; i < 3; ++i) s[i] = 0.0;
    for (int i = 0; i < 9; ++i) s_x[i] = 0.0;
    if (!u) return;
    for (int n = 0; n < e.nen; ++n) {
        const double* un = &u[3 * (int64_t)cellnodes[n]];
        const double ph = e.phi[q * e.nen + n];
        const double* g = &p.gphi[n * 3];
        for (int c = 0; c < 3; ++c) {
            s[c] += ph * un[c];
            for (int d = 0; d < 3; ++d) s_x[c * 3 + d] += un[c] * g[d];
        }
    }
}

}  // namespace

extern "C" {

int oracle_num_quadrature_points(int cell_type) { return make_element(cell_type).nq; }
int oracle_nodes_per_cell(int cell_type) { return make_element(cell_type).nen; }

// Residual: r += sum over cells of the element residual (ADD_VALUES). r has nnodes*3 entries.
// Returns 0, or -(cell+1) of the first cell with a non-positive Jacobian determinant.
int64_t oracle_residual(int cell_type, int64_t ncells, const int* cells, const double* coords,
                        int64_t nnodes, const double* u, const double* u_t, int numA,
                        const int* aux_kind, const int* aux_ncomp, const double* const* aux_data,
                        double t, int numConstants, const double* constants, PointFn f0, PointFn f1,
                        double* r, int nthreads) {
    const Element e = make_element(cell_type);
    const Aux aux(numA, aux_kind, aux_ncomp, aux_data);
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    std::vector<std::vector<double>> bufs(nthreads);
    int64_t bad = 0;
#pragma omp parallel num_threads(nthreads)
    {
        const int tid = omp_get_thread_num();
        std::vector<double>& rb = bufs[tid];
        rb.assign(nnodes * 3, 0.0);
        std::vector<double> a(aux.total > 0 ? aux.total : 1);
        std::vector<double> re(e.nen * 3);
        QPoint p;
        const int sOff[1] = {0}, sOff_x[1] = {0};
        double s[3], s_t[3], s_x[9], f0v[3], f1v[9];
#pragma omp for schedule(static)
        for (int64_t cell = 0; cell < ncells; ++cell) {
            const int* cn = &cells[cell * e.nen];
            std::fill(re.begin(), re.end(), 0.0);
            for (int q = 0; q < e.nq; ++q) {
                if (!eval_geometry(e, q, cn, coords, &p)) {
#pragma omp critical
                    { if (!bad) bad = -(cell + 1); }
                    continue;
                }
                eval_field(e, q, p, cn, u, s, s_x);
                double dummy[9];
                eval_field(e, q, p, cn, u_t, s_t, dummy);
                aux.eval(e, cell, q, cn, a.data());
                for (int i = 0; i < 3; ++i) f0v[i] = 0.0;
                for (int i = 0; i < 9; ++i) f1v[i] = 0.0;
                if (f0) f0(3, 1, numA, sOff, sOff_x, s, s_t, s_x, aux.off.data(), nullptr, a.data(),
                           nullptr, nullptr, t, p.x, numConstants, constants, f0v);
                if (f1) f1(3, 1, numA, sOff, sOff_x, s, s_t, s_x, aux.off.data(), nullptr, a.data(),
                           nullptr, nullptr, t, p.x, numConstants, constants, f1v);
                for (int n = 0; n < e.nen; ++n) {
                    const double ph = e.phi[q * e.nen + n];
                    const double* g = &p.gphi[n * 3];
                    for (int c = 0; c < 3; ++c) {
                        re[n * 3 + c] += p.wdetJ * (f0v[c] * ph + f1v[c * 3 + 0] * g[0] +
                                                    f1v[c * 3 + 1] * g[1] + f1v[c * 3 + 2] * g[2]);
                    }
                }
            }
            for (int n = 0; n < e.nen; ++n)
                for (int c = 0; c < 3; ++c) rb[3 * (int64_t)cn[n] + c] += re[n * 3 + c];
        }
    }
    for (int th = 0; th < nthreads; ++th) {
        const std::vector<double>& rb = bufs[th];
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int64_t i = 0; i < nnodes * 3; ++i) r[i] += rb[i];
    }
    return bad;
}

// Element Jacobians: Ke[cell][(a*3+fc)][(b*3+gc)] for nen field nodes, from the pointwise
// g0..g3 (layouts g0[fc*3+gc], g1[(fc*3+gc)*3+dg], g2[(fc*3+gc)*3+df],
// g3[((fc*3+gc)*3+df)*3+dg]).
int64_t oracle_jacobian_elements(int cell_type, int64_t ncells, const int* cells,
                                 const double* coords, const double* u, int numA,
                                 const int* aux_kind, const int* aux_ncomp,
                                 const double* const* aux_data, double t, double s_tshift,
                                 int numConstants, const double* constants, PointJacFn g0,
                                 PointJacFn g1, PointJacFn g2, PointJacFn g3, double* Ke,
                                 int nthreads) {
    const Element e = make_element(cell_type);
    const Aux aux(numA, aux_kind, aux_ncomp, aux_data);
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    const int nd = e.nen * 3;
    int64_t bad = 0;
#pragma omp parallel num_threads(nthreads)
    {
        std::vector<double> a(aux.total > 0 ? aux.total : 1);
        QPoint p;
        const int sOff[1] = {0}, sOff_x[1] = {0};
        double s[3], s_t[3] = {0, 0, 0}, s_x[9], G0[9], G1[27], G2[27], G3[81];
#pragma omp for schedule(static)
        for (int64_t cell = 0; cell < ncells; ++cell) {
            const int* cn = &cells[cell * e.nen];
            double* K = &Ke[cell * nd * nd];
            std::fill(K, K + nd * nd, 0.0);
            for (int q = 0; q < e.nq; ++q) {
                if (!eval_geometry(e, q, cn, coords, &p)) {
#pragma omp critical
                    { if (!bad) bad = -(cell + 1); }
                    continue;
                }
                eval_field(e, q, p, cn, u, s, s_x);
                aux.eval(e, cell, q, cn, a.data());
                std::fill(G0, G0 + 9, 0.0); std::fill(G1, G1 + 27, 0.0);
                std::fill(G2, G2 + 27, 0.0); std::fill(G3, G3 + 81, 0.0);
#define ORACLE_CALLJ(fn, out) \
    if (fn) fn(3, 1, numA, sOff, sOff_x, s, s_t, s_x, aux.off.data(), nullptr, a.data(), nullptr, \
               nullptr, t, s_tshift, p.x, numConstants, constants, out)
                ORACLE_CALLJ(g0, G0);
                ORACLE_CALLJ(g1, G1);
                ORACLE_CALLJ(g2, G2);
                ORACLE_CALLJ(g3, G3);
#undef ORACLE_CALLJ
                for (int an = 0; an < e.nen; ++an) {
                    const double pa = e.phi[q * e.nen + an];
                    const double* ga = &p.gphi[an * 3];
                    for (int bn = 0; bn < e.nen; ++bn) {
                        const double pb = e.phi[q * e.nen + bn];
                        const double* gb = &p.gphi[bn * 3];
                        for (int fc = 0; fc < 3; ++fc)
                            for (int gc = 0; gc < 3; ++gc) {
                                const int fg = fc * 3 + gc;
                                double v = G0[fg] * pa * pb;
                                for (int d = 0; d < 3; ++d) {
                                    v += G1[fg * 3 + d] * pa * gb[d];
                                    v += G2[fg * 3 + d] * ga[d] * pb;
                                }
                                for (int df = 0; df < 3; ++df)
                                    for (int dg = 0; dg < 3; ++dg)
                                        v += G3[(fg * 3 + df) * 3 + dg] * ga[df] * gb[dg];
                                K[(an * 3 + fc) * nd + (bn * 3 + gc)] += p.wdetJ * v;
                            }
                    }
                }
            }
        }
    }
    return bad;
}

// Matrix-free Jacobian action (DMPlexComputeJacobianActionByKey, called at
// libsrc/pylith/feassemble/IntegratorDomain.cc:540): jv += sum over cells of K_e v_e, with K_e
// the element Jacobian of oracle_jacobian_elements, applied at each quadrature point to the
// values and gradient of v instead of being formed: jv_a,fc += wdetJ (phi_a (G0 v + G1 grad v)
// + grad phi_a . (G2 v + G3 grad v)). The pointwise Jacobians are evaluated at u.
int64_t oracle_jacobian_action(int cell_type, int64_t ncells, const int* cells, const double* coords,
                               int64_t nnodes, const double* u, const double* v, int numA,
                               const int* aux_kind, const int* aux_ncomp, const double* const* aux_data,
                               double t, double s_tshift, int numConstants, const double* constants,
                               PointJacFn g0, PointJacFn g1, PointJacFn g2, PointJacFn g3, double* jv,
                               int nthreads) {
    const Element e = make_element(cell_type);
    const Aux aux(numA, aux_kind, aux_ncomp, aux_data);
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    std::vector<std::vector<double>> bufs(nthreads);
    int64_t bad = 0;
#pragma omp parallel num_threads(nthreads)
    {
        const int tid = omp_get_thread_num();
        std::vector<double>& rb = bufs[tid];
        rb.assign(nnodes * 3, 0.0);
        std::vector<double> a(aux.total > 0 ? aux.total : 1);
        std::vector<double> re(e.nen * 3);
        QPoint p;
        const int sOff[1] = {0}, sOff_x[1] = {0};
        double s[3], s_t[3] = {0, 0, 0}, s_x[9], w[3], w_x[9], G0[9], G1[27], G2[27], G3[81];
#pragma omp for schedule(static)
        for (int64_t cell = 0; cell < ncells; ++cell) {
            const int* cn = &cells[cell * e.nen];
            std::fill(re.begin(), re.end(), 0.0);
            for (int q = 0; q < e.nq; ++q) {
                if (!eval_geometry(e, q, cn, coords, &p)) {
#pragma omp critical
                    { if (!bad) bad = -(cell + 1); }
                    continue;
                }
                if (u) {
                    eval_field(e, q, p, cn, u, s, s_x);
                } else {
                    std::fill(s, s + 3, 0.0);
                    std::fill(s_x, s_x + 9, 0.0);
                }
                eval_field(e, q, p, cn, v, w, w_x);
                aux.eval(e, cell, q, cn, a.data());
                std::fill(G0, G0 + 9, 0.0); std::fill(G1, G1 + 27, 0.0);
                std::fill(G2, G2 + 27, 0.0); std::fill(G3, G3 + 81, 0.0);
#define ORACLE_CALLJ(fn, out) \
    if (fn) fn(3, 1, numA, sOff, sOff_x, s, s_t, s_x, aux.off.data(), nullptr, a.data(), nullptr, \
               nullptr, t, s_tshift, p.x, numConstants, constants, out)
                ORACLE_CALLJ(g0, G0);
                ORACLE_CALLJ(g1, G1);
                ORACLE_CALLJ(g2, G2);
                ORACLE_CALLJ(g3, G3);
#undef ORACLE_CALLJ
                double f0v[3], f1v[9];
                for (int fc = 0; fc < 3; ++fc) {
                    double acc0 = 0.0;
                    for (int gc = 0; gc < 3; ++gc) {
                        const int fg = fc * 3 + gc;
                        acc0 += G0[fg] * w[gc];
                        for (int dg = 0; dg < 3; ++dg) acc0 += G1[fg * 3 + dg] * w_x[gc * 3 + dg];
                    }
                    f0v[fc] = acc0;
                    for (int df = 0; df < 3; ++df) {
                        double acc1 = 0.0;
                        for (int gc = 0; gc < 3; ++gc) {
                            const int fg = fc * 3 + gc;
                            acc1 += G2[fg * 3 + df] * w[gc];
                            for (int dg = 0; dg < 3; ++dg) acc1 += G3[(fg * 3 + df) * 3 + dg] * w_x[gc * 3 + dg];
                        }
                        f1v[fc * 3 + df] = acc1;
                    }
                }
                for (int n = 0; n < e.nen; ++n) {
                    const double ph = e.phi[q * e.nen + n];
                    const double* g = &p.gphi[n * 3];
                    for (int c = 0; c < 3; ++c)
                        re[n * 3 + c] += p.wdetJ * (f0v[c] * ph + f1v[c * 3 + 0] * g[0] + f1v[c * 3 + 1] * g[1] +
                                                    f1v[c * 3 + 2] * g[2]);
                }
            }
            for (int n = 0; n < e.nen; ++n)
                for (int c = 0; c < 3; ++c) rb[3 * (int64_t)cn[n] + c] += re[n * 3 + c];
        }
    }
    for (int th = 0; th < nthreads; ++th) {
        const std::vector<double>& rb = bufs[th];
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int64_t i = 0; i < nnodes * 3; ++i) jv[i] += rb[i];
    }
    return bad;
}

// Projection of pointwise functions at quadrature points (DMProjectFieldLocal with
// point-space outputs): out_k[cell][q][ncomp_k] = fn_k(solution at q, aux at q). All functions
// see the same (previous) aux values, as the reference evaluates every kernel on the input
// auxiliary vector before replacing it (IntegratorDomain.cc:555-590).
int64_t oracle_project_qp(int cell_type, int64_t ncells, const int* cells, const double* coords,
                          const double* u, int numA, const int* aux_kind, const int* aux_ncomp,
                          const double* const* aux_data, double t, int numConstants,
                          const double* constants, int nfn, const PointFn* fns,
                          const int* out_ncomp, double* const* outs, int nthreads) {
    const Element e = make_element(cell_type);
    const Aux aux(numA, aux_kind, aux_ncomp, aux_data);
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    int64_t bad = 0;
#pragma omp parallel num_threads(nthreads)
    {
        std::vector<double> a(aux.total > 0 ? aux.total : 1);
        QPoint p;
        const int sOff[1] = {0}, sOff_x[1] = {0};
        double s[3], s_t[3] = {0, 0, 0}, s_x[9];
        std::vector<double> o(64);
#pragma omp for schedule(static)
        for (int64_t cell = 0; cell < ncells; ++cell) {
            const int* cn = &cells[cell * e.nen];
            for (int q = 0; q < e.nq; ++q) {
                if (!eval_geometry(e, q, cn, coords, &p)) {
#pragma omp critical
                    { if (!bad) bad = -(cell + 1); }
                    continue;
                }
                eval_field(e, q, p, cn, u, s, s_x);
                aux.eval(e, cell, q, cn, a.data());
                for (int k = 0; k < nfn; ++k) {
                    const int nc = out_ncomp[k];
                    std::fill(o.begin(), o.begin() + nc, 0.0);
                    fns[k](3, 1, numA, sOff, sOff_x, s, s_t, s_x, aux.off.data(), nullptr, a.data(),
                           nullptr, nullptr, t, p.x, numConstants, constants, o.data());
                    for (int c = 0; c < nc; ++c) outs[k][(cell * e.nq + q) * nc + c] = o[c];
                }
            }
        }
    }
    return bad;
}

// Derived fields of basis order 0 (IntegratorDomain::_computeDerivedField,
// IntegratorDomain.cc:596-630): each function evaluated once per cell at the centroid,
// out_k[cell][ncomp_k]. Aux subfields per quadrature point are read at point 0.
int64_t oracle_project_centroid(int cell_type, int64_t ncells, const int* cells, const double* coords,
                                const double* u, int numA, const int* aux_kind, const int* aux_ncomp,
                                const double* const* aux_data, double t, int numConstants,
                                const double* constants, int nfn, const PointFn* fns,
                                const int* out_ncomp, double* const* outs, int nthreads) {
    const Element e = make_element(cell_type, true);
    const Element eq = make_element(cell_type);
    const Aux aux(numA, aux_kind, aux_ncomp, aux_data);
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    int64_t bad = 0;
#pragma omp parallel num_threads(nthreads)
    {
        std::vector<double> a(aux.total > 0 ? aux.total : 1);
        QPoint p;
        const int sOff[1] = {0}, sOff_x[1] = {0};
        double s[3], s_t[3] = {0, 0, 0}, s_x[9];
        std::vector<double> o(64);
#pragma omp for schedule(static)
        for (int64_t cell = 0; cell < ncells; ++cell) {
            const int* cn = &cells[cell * e.nen];
            if (!eval_geometry(e, 0, cn, coords, &p)) {
#pragma omp critical
                { if (!bad) bad = -(cell + 1); }
                continue;
            }
            eval_field(e, 0, p, cn, u, s, s_x);
            aux.eval(eq, cell, 0, cn, a.data());
            for (int k = 0; k < nfn; ++k) {
                const int nc = out_ncomp[k];
                std::fill(o.begin(), o.begin() + nc, 0.0);
                fns[k](3, 1, numA, sOff, sOff_x, s, s_t, s_x, aux.off.data(), nullptr, a.data(), nullptr,
                       nullptr, t, p.x, numConstants, constants, o.data());
                for (int c = 0; c < nc; ++c) outs[k][cell * nc + c] = o[c];
            }
        }
    }
    return bad;
}

// ---------------------------------------------------------------------------------------------
// Cohesive cells (DMPlexCompute{Residual,Jacobian}HybridByKey, IntegratorInterface.cc:603-720).
// Each cohesive cell is a quadrilateral fault face: coh[c*12 + 0..3] negative-side vertices,
// [4..7] positive-side vertices (same positions), [8..11] Lagrange-multiplier nodes. The face
// normal is (dx/dxi x dx/deta)/|.| from the negative-side vertex order and points from the
// negative to the positive side. Solution at a point: s = [u-(3), u+(3), lambda(3)],
// sOff = {0, 6}; aux = slip(3) per Lagrange node (basis order 1), aOff = {0}.
// Displacement DOF of vertex v: 3*v + c; Lagrange DOF of node l: lag_offset + 3*l + c.

namespace {
struct FacePoint {
    double phi[4];
    double x[3];
    double n[3];
    double wdetJ;
};

void face_points(const int* cc, const double* coords, FacePoint fp[4]) {
    const double g = 1.0 / std::sqrt(3.0);
    const double xi[2] = {-g, g};
    const int corner[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};
    for (int qj = 0; qj < 2; ++qj)
        for (int qi = 0; qi < 2; ++qi) {
            FacePoint& p = fp[qj * 2 + qi];
            double v0[2], d0[2], v1[2], d1[2];
            lagrange1d(1, xi[qi], v0, d0);
            lagrange1d(1, xi[qj], v1, d1);
            double dxi[3] = {0, 0, 0}, deta[3] = {0, 0, 0};
            p.x[0] = p.x[1] = p.x[2] = 0.0;
            for (int a = 0; a < 4; ++a) {
                const double* X = &coords[3 * (int64_t)cc[a]];
                const int i = corner[a][0], j = corner[a][1];
                p.phi[a] = v0[i] * v1[j];
                for (int d = 0; d < 3; ++d) {
                    p.x[d] += p.phi[a] * X[d];
                    dxi[d] += d0[i] * v1[j] * X[d];
                    deta[d] += v0[i] * d1[j] * X[d];
                }
            }
            double nn[3] = {dxi[1] * deta[2] - dxi[2] * deta[1], dxi[2] * deta[0] - dxi[0] * deta[2],
                            dxi[0] * deta[1] - dxi[1] * deta[0]};
            const double area = std::sqrt(nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2]);
            for (int d = 0; d < 3; ++d) p.n[d] = nn[d] / area;
            p.wdetJ = area;  // Gauss weights are 1 for the 2-point rule
        }
}
}  // namespace

void oracle_cohesive_residual(int64_t ncoh, const int* coh, const double* coords, const double* u,
                              int64_t lag_offset, const double* slip, double t, int numConstants,
                              const double* constants, BdPointFn f0_neg, BdPointFn f0_pos,
                              BdPointFn f0_lag, double* r) {
    const int sOff[2] = {0, 6}, sOff_x[2] = {0, 0}, aOff[1] = {0};
    for (int64_t c = 0; c < ncoh; ++c) {
        const int* cc = &coh[c * 12];
        FacePoint fp[4];
        face_points(cc, coords, fp);
        double rn[12] = {0}, rp[12] = {0}, rl[12] = {0};
        for (int q = 0; q < 4; ++q) {
            const FacePoint& p = fp[q];
            double s[9] = {0}, a[3] = {0}, sx[18] = {0};
            for (int k = 0; k < 4; ++k) {
                for (int d = 0; d < 3; ++d) {
                    s[d] += p.phi[k] * u[3 * (int64_t)cc[k] + d];
                    s[3 + d] += p.phi[k] * u[3 * (int64_t)cc[4 + k] + d];
                    s[6 + d] += p.phi[k] * u[lag_offset + 3 * (int64_t)cc[8 + k] + d];
                    a[d] += p.phi[k] * slip[3 * (int64_t)cc[8 + k] + d];
                }
            }
            double fn[3] = {0}, fpv[3] = {0}, fl[3] = {0};
            if (f0_neg) f0_neg(3, 2, 1, sOff, sOff_x, s, nullptr, sx, aOff, nullptr, a, nullptr, nullptr,
                               t, p.x, p.n, numConstants, constants, fn);
            if (f0_pos) f0_pos(3, 2, 1, sOff, sOff_x, s, nullptr, sx, aOff, nullptr, a, nullptr, nullptr,
                               t, p.x, p.n, numConstants, constants, fpv);
            if (f0_lag) f0_lag(3, 2, 1, sOff, sOff_x, s, nullptr, sx, aOff, nullptr, a, nullptr, nullptr,
                               t, p.x, p.n, numConstants, constants, fl);
            for (int k = 0; k < 4; ++k)
                for (int d = 0; d < 3; ++d) {
                    rn[k * 3 + d] += p.wdetJ * p.phi[k] * fn[d];
                    rp[k * 3 + d] += p.wdetJ * p.phi[k] * fpv[d];
                    rl[k * 3 + d] += p.wdetJ * p.phi[k] * fl[d];
                }
        }
        for (int k = 0; k < 4; ++k)
            for (int d = 0; d < 3; ++d) {
                r[3 * (int64_t)cc[k] + d] += rn[k * 3 + d];
                r[3 * (int64_t)cc[4 + k] + d] += rp[k * 3 + d];
                r[lag_offset + 3 * (int64_t)cc[8 + k] + d] += rl[k * 3 + d];
            }
    }
}

// Cohesive element Jacobians over the 36 DOFs [u-(4x3), u+(4x3), lambda(4x3)]:
// Jf0ul_neg fills the (u-, lambda) block, Jf0ul_pos the (u+, lambda) block, Jf0lu the
// (lambda, u-) and (lambda, u+) blocks (two 3x3 pointwise blocks, negative side first).
void oracle_cohesive_jacobian_elements(int64_t ncoh, const int* coh, const double* coords,
                                       double t, double s_tshift, int numConstants,
                                       const double* constants, BdPointJacFn jul_neg,
                                       BdPointJacFn jul_pos, BdPointJacFn jlu, double* Ke) {
    const int sOff[2] = {0, 6}, sOff_x[2] = {0, 0}, aOff[1] = {0};
    for (int64_t c = 0; c < ncoh; ++c) {
        const int* cc = &coh[c * 12];
        FacePoint fp[4];
        face_points(cc, coords, fp);
        double* K = &Ke[c * 36 * 36];
        std::fill(K, K + 36 * 36, 0.0);
        for (int q = 0; q < 4; ++q) {
            const FacePoint& p = fp[q];
            double s[9] = {0}, a[3] = {0}, sx[18] = {0};
            double gn[9] = {0}, gp[9] = {0}, gl[18] = {0};
            if (jul_neg) jul_neg(3, 2, 1, sOff, sOff_x, s, nullptr, sx, aOff, nullptr, a, nullptr,
                                 nullptr, t, s_tshift, p.x, p.n, numConstants, constants, gn);
            if (jul_pos) jul_pos(3, 2, 1, sOff, sOff_x, s, nullptr, sx, aOff, nullptr, a, nullptr,
                                 nullptr, t, s_tshift, p.x, p.n, numConstants, constants, gp);
            if (jlu) jlu(3, 2, 1, sOff, sOff_x, s, nullptr, sx, aOff, nullptr, a, nullptr, nullptr,
                         t, s_tshift, p.x, p.n, numConstants, constants, gl);
            for (int ka = 0; ka < 4; ++ka)
                for (int kb = 0; kb < 4; ++kb) {
                    const double w = p.wdetJ * p.phi[ka] * p.phi[kb];
                    for (int fc = 0; fc < 3; ++fc)
                        for (int gc = 0; gc < 3; ++gc) {
                            // rows u-/u+ (field), cols lambda (trial)
                            K[(0 + ka * 3 + fc) * 36 + (24 + kb * 3 + gc)] += w * gn[fc * 3 + gc];
                            K[(12 + ka * 3 + fc) * 36 + (24 + kb * 3 + gc)] += w * gp[fc * 3 + gc];
                            // rows lambda, cols u- then u+
                            K[(24 + ka * 3 + fc) * 36 + (0 + kb * 3 + gc)] += w * gl[fc * 3 + gc];
                            K[(24 + ka * 3 + fc) * 36 + (12 + kb * 3 + gc)] += w * gl[9 + fc * 3 + gc];
                        }
                }
        }
    }
}

// CSR sparse matrix-vector product y = A x (the assembled-operator path PETSc's MatMult takes).
void oracle_csr_spmv(int64_t nrows, const int64_t* indptr, const int* indices, const double* data,
                     const double* x, double* y, int nthreads) {
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int64_t i = 0; i < nrows; ++i) {
        double acc = 0.0;
        for (int64_t k = indptr[i]; k < indptr[i + 1]; ++k) acc += data[k] * x[indices[k]];
        y[i] = acc;
    }
}

// Pointwise kernels of the restatement, exported for the tests and for use as the oracle
// loop's callbacks.
#define ORACLE_EXPORT_POINT(cname, fn)                                                           \
    void cname(ORACLE_POINT_ARGS, const Real x[], Int numConstants, const Real constants[],     \
               Real f[]) {                                                                      \
        fn(dim, numS, numA, sOff, sOff_x, s, s_t, s_x, aOff, aOff_x, a, a_t, a_x, t, x,         \
           numConstants, constants, f);                                                         \
    }
#define ORACLE_EXPORT_JAC(cname, fn)                                                             \
    void cname(ORACLE_POINT_ARGS, Real s_tshift, const Real x[], Int numConstants,              \
               const Real constants[], Real g[]) {                                              \
        fn(dim, numS, numA, sOff, sOff_x, s, s_t, s_x, aOff, aOff_x, a, a_t, a_x, t, s_tshift,   \
           x, numConstants, constants, g);                                                      \
    }
#define ORACLE_EXPORT_BD(cname, fn)                                                              \
    void cname(ORACLE_POINT_ARGS, const Real x[], const Real n[], Int numConstants,             \
               const Real constants[], Real f[]) {                                              \
        fn(dim, numS, numA, sOff, sOff_x, s, s_t, s_x, aOff, aOff_x, a, a_t, a_x, t, x, n,      \
           numConstants, constants, f);                                                         \
    }
#define ORACLE_EXPORT_BDJ(cname, fn)                                                             \
    void cname(ORACLE_POINT_ARGS, Real s_tshift, const Real x[], const Real n[],                \
               Int numConstants, const Real constants[], Real g[]) {                            \
        fn(dim, numS, numA, sOff, sOff_x, s, s_t, s_x, aOff, aOff_x, a, a_t, a_x, t, s_tshift,   \
           x, n, numConstants, constants, g);                                                   \
    }

ORACLE_EXPORT_POINT(oracle_g0v_bodyforce, g0v_bodyforce)
ORACLE_EXPORT_POINT(oracle_ile3d_f1v, ile3d_f1v)
ORACLE_EXPORT_JAC(oracle_ile3d_Jf3vu, ile3d_Jf3vu)
ORACLE_EXPORT_POINT(oracle_gm3d_f1v, gm3d_f1v)
ORACLE_EXPORT_JAC(oracle_gm3d_Jf3vu, gm3d_Jf3vu)
ORACLE_EXPORT_POINT(oracle_gm3d_viscous_strain, gm3d_viscous_strain)
ORACLE_EXPORT_POINT(oracle_el3d_strain_vector, el3d_strain_vector)
ORACLE_EXPORT_POINT(oracle_ile3d_stress_vector, ile3d_stress_vector)
ORACLE_EXPORT_POINT(oracle_gm3d_stress_vector, gm3d_stress_vector)
ORACLE_EXPORT_BD(oracle_fck_f0u_neg, fck_f0u_neg)
ORACLE_EXPORT_BD(oracle_fck_f0u_pos, fck_f0u_pos)
ORACLE_EXPORT_BD(oracle_fck_f0l_slip, fck_f0l_slip)
ORACLE_EXPORT_BDJ(oracle_fck_Jf0ul_neg, fck_Jf0ul_neg)
ORACLE_EXPORT_BDJ(oracle_fck_Jf0ul_pos, fck_Jf0ul_pos)
ORACLE_EXPORT_BDJ(oracle_fck_Jf0lu, fck_Jf0lu)

void oracle_tangential_directions(double t1[3], double t2[3], const double r1[3],
                                  const double r2[3], const double n[3]) {
    tangential_directions(t1, t2, r1, r2, n);
}

}  // extern "C"
