// Device Krylov solver for the quasi-static step: preconditioned conjugate gradients on
// A = -J (J = sum of the registered integrators' Jacobian actions, negative definite for the
// elasticity kernels, f1 = -sigma and Jf3 = -C), restricted to the unconstrained DOFs.
//
// Replaces the PETSc KSP the reference configures for these problems (defaults in
// libsrc/pylith/materials/Elasticity.cc:298-330, tolerances in
// libsrc/pylith/petsc/Options.cc:320-331). Preconditioner: point-block Jacobi (inverse 3x3
// node blocks of A, the "vpbjacobi" idea the reference uses on faults), optionally wrapped in
// a Chebyshev polynomial. Two precisions:
//   * FP64: every vector and reduction in FP64;
//   * FP32 refined: inner PCG in FP32 vectors and FP32 operator application with FP64 dot
//     products, inside FP64 iterative refinement (outer residual b - A x in FP64).
// Reductions are two-pass and deterministic (per-CTA partials, then one CTA in fixed order).
#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <vector>

#include "cg.cuh"
#include "domain_kernels.cuh"
#include "internal.hpp"
#include "launch.hpp"

namespace plb {

// dots (a.b, c.d) over unconstrained DOFs.
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_dot2(const T* a, const T* b, const T* c, const T* d,
                                                      const uint8_t* mask, int64_t n, double* partials) {
    double s0 = 0.0, s1 = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (mask[i]) continue;
        s0 += to_d(a[i]) * to_d(b[i]);
        if (c) s1 += to_d(c[i]) * to_d(d[i]);
    }
    block_sum2(s0, s1, partials);
}

// r := b (masked), z := P^{-1} r, p := z; partial (r.z, r.r).
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_cg_init(const T* b, const uint8_t* mask, const T* pinv, int64_t nnodes,
                                                         T* r, T* z, T* p, double* partials) {
    double rz = 0.0, rr = 0.0;
    for (int64_t nd = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; nd < nnodes; nd += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < 3; ++k) r[3 * nd + k] = mask[3 * nd + k] ? T(0) : b[3 * nd + k];
        T zz[3];
        apply_pinv(pinv, r, nd, zz);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            z[3 * nd + k] = zz[k];
            p[3 * nd + k] = zz[k];
            rz += to_d(r[3 * nd + k]) * to_d(zz[k]);
            rr += to_d(r[3 * nd + k]) * to_d(r[3 * nd + k]);
        }
    }
    block_sum2(rz, rr, partials);
}

// q holds J p (not yet negated). A p = -q on free DOFs. Partial of p.(A p).
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_cg_pq(const T* p, const T* q, const uint8_t* mask, int64_t n,
                                                       double* partials) {
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (!mask[i]) s -= to_d(p[i]) * to_d(q[i]);
    block_sum2(s, 0.0, partials);
}

// alpha = rz / pq; x += alpha p; r -= alpha A p (= r + alpha q); z = P^{-1} r; partial (r.z, r.r).
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_cg_update(T* x, T* r, const T* p, const T* q, T* z, const uint8_t* mask,
                                                           const T* pinv, int64_t nnodes, const double* scal,
                                                           double* partials) {
    // p.(A p) > 0 for the SPD operator; a search direction that has collapsed to rounding noise
    // (FP32 iterations past convergence) can give pq <= 0 or an alpha beyond T's range: no step
    const double pq = scal[S_PQ];
    const double a64 = pq > 0.0 ? scal[S_RZ] / pq : 0.0;
    const T alpha = (T)(isfinite((T)a64) ? a64 : 0.0);
    double rz = 0.0, rr = 0.0;
    for (int64_t nd = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; nd < nnodes; nd += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int64_t i = 3 * nd + k;
            if (!mask[i]) {
                x[i] += alpha * p[i];
                r[i] += alpha * q[i];
            }
        }
        T zz[3];
        apply_pinv(pinv, r, nd, zz);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            z[3 * nd + k] = zz[k];
            rz += to_d(r[3 * nd + k]) * to_d(zz[k]);
            rr += to_d(r[3 * nd + k]) * to_d(r[3 * nd + k]);
        }
    }
    block_sum2(rz, rr, partials);
}

// z = P^{-1} r; partial (r.z) (after the residual of a reliable update replaced r).
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_prec_rz(const T* r, const T* pinv, int64_t nnodes, T* z,
                                                         double* partials) {
    double rz = 0.0;
    for (int64_t nd = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; nd < nnodes; nd += (int64_t)gridDim.x * blockDim.x) {
        T zz[3];
        apply_pinv(pinv, r, nd, zz);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            z[3 * nd + k] = zz[k];
            rz += to_d(r[3 * nd + k]) * to_d(zz[k]);
        }
    }
    block_sum2(rz, 0.0, partials);
}

// beta = rz / rz_old; p = z + beta p.
template <typename T>
__global__ void k_cg_pupdate(T* p, const T* z, int64_t n, double* scal) {
    const double beta = scal[S_RZ_OLD] != 0.0 ? scal[S_RZ] / scal[S_RZ_OLD] : 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = z[i] + (T)beta * p[i];
}

__global__ void k_copy_scalar(double* scal, int from, int to) { scal[to] = scal[from]; }

// Point-block Jacobi: invert each node's 3x3 block of A = -J with constrained rows/columns
// replaced by the identity.
__global__ void k_invert_blocks(const double* __restrict__ diagJ, const uint8_t* __restrict__ mask, int64_t nnodes,
                                double* pinv, float* pinv32) {
    for (int64_t nd = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; nd < nnodes; nd += (int64_t)gridDim.x * blockDim.x) {
        double A[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                const bool ci = mask[3 * nd + i], cj = mask[3 * nd + j];
                A[i][j] = (ci || cj) ? (i == j ? 1.0 : 0.0) : -diagJ[9 * nd + 3 * i + j];
            }
        double inv[3][3];
        const double det = invert3(A, inv);
        const bool ok = det != 0.0 && isfinite(det);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                const double v = ok ? inv[i][j] : (i == j ? 1.0 : 0.0);
                pinv[9 * nd + 3 * i + j] = v;
                pinv32[9 * nd + 3 * i + j] = (float)v;
            }
    }
}

template <typename T>
__global__ void k_masked_copy(const double* src, const uint8_t* mask, int64_t n, T* dst) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = mask[i] ? T(0) : (T)src[i];
}

// r64 = b - A x = b + J x on free DOFs (q holds J x).
__global__ void k_outer_residual(const double* b, const double* Jx, const uint8_t* mask, int64_t n, double* r,
                                 float* r32, double* partials) {
    double rr = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = mask[i] ? 0.0 : b[i] + Jx[i];
        r[i] = v;
        r32[i] = (float)v;
        rr += v * v;
    }
    block_sum2(rr, 0.0, partials);
}

__global__ void k_add_correction(double* x, const float* d, const uint8_t* mask, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (!mask[i]) x[i] += (double)d[i];
}

// Diagonal 3x3 blocks of J from the registered Jf3 (thread per cell, reductions per node).
template <int CELL, int RHEO>
__global__ void __launch_bounds__(128) k_domain_diag_blocks(DomainParams p, double* diag) {
    using E = Elem<CELL>;
    using L = AuxLayout<RHEO, false>;
    const AuxOffsets<RHEO, false> aoff;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < p.ncells; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t mc = p.cell_ids ? p.cell_ids[c] : c;
        const int32_t* cn = p.cells + mc * E::nen;
        double X[E::ngeom][3];
#pragma unroll
        for (int k = 0; k < E::ngeom; ++k)
#pragma unroll
            for (int i = 0; i < 3; ++i) X[k][i] = p.coords[3 * (int64_t)cn[E::corner(k)] + i];
        double a[L::size] = {};
        L::load_cell(p, c, a);
#pragma unroll 1
        for (int q = 0; q < E::nq; ++q) {
            Geom g;
            E::geom(X, q, &g);
            // the tangents (Jf3vu of both rheologies) read no per-point state
            double x[3] = {0, 0, 0};
            double Jf3[81];
#pragma unroll
            for (int i = 0; i < 81; ++i) Jf3[i] = 0.0;
            call_jf3<RHEO>(L::numA, aoff.v, a, p, x, Jf3);
#pragma unroll 1
            for (int n = 0; n < E::nen; ++n) {
                double gr[3];
                E::grad(g, q, n, gr);
                double* blk = diag + 9 * (int64_t)cn[n];
#pragma unroll
                for (int f = 0; f < 3; ++f)
#pragma unroll
                    for (int gg = 0; gg < 3; ++gg) {
                        double v = 0.0;
#pragma unroll
                        for (int df = 0; df < 3; ++df)
#pragma unroll
                            for (int dg = 0; dg < 3; ++dg) v += gr[df] * Jf3[((f * 3 + gg) * 3 + df) * 3 + dg] * gr[dg];
                        red_add(&blk[f * 3 + gg], g.wdetJ * v);
                    }
            }
        }
    }
}

void launch_domain_diag_blocks(const DomainParams& p, int cell, int rheo, double* diag, cudaStream_t s) {
    if (p.ncells == 0) return;
    const int64_t b = (p.ncells + 127) / 128;
    const int gr = (int)std::min<int64_t>(b, 148 * 64);
#define PLB_DIAG(C, R) k_domain_diag_blocks<C, R><<<gr, 128, 0, s>>>(p, diag)
    if (cell == TET4) { if (rheo == RHEO_ILE) PLB_DIAG(TET4, RHEO_ILE); else PLB_DIAG(TET4, RHEO_GENMAXWELL); }
    else if (cell == HEX8) { if (rheo == RHEO_ILE) PLB_DIAG(HEX8, RHEO_ILE); else PLB_DIAG(HEX8, RHEO_GENMAXWELL); }
    else { if (rheo == RHEO_ILE) PLB_DIAG(HEX27, RHEO_ILE); else PLB_DIAG(HEX27, RHEO_GENMAXWELL); }
#undef PLB_DIAG
    count_launch();
}

static int vec_grid(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 148 * 8); }

// Faults are solved in the reduced space of the slip constraint u+ = u- + d: the positive-side
// DOFs of every fault node follow the negative side ("unfold"), and the equations of both sides
// are summed onto the negative side ("fold"), where the Lagrange-multiplier terms cancel
// (f0u_neg = -lambda, f0u_pos = +lambda). The reduced operator P^T (-J) P is SPD.
template <typename T>
__global__ void k_fault_unfold(T* v, const int32_t* __restrict__ neg, const int32_t* __restrict__ pos, int64_t npairs) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * npairs; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = i / 3, c = i % 3;
        v[3 * (int64_t)pos[k] + c] = v[3 * (int64_t)neg[k] + c];
    }
}

template <typename T>
__global__ void k_fault_fold(T* v, const int32_t* __restrict__ neg, const int32_t* __restrict__ pos, int64_t npairs) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * npairs; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = i / 3, c = i % 3;
        v[3 * (int64_t)neg[k] + c] += v[3 * (int64_t)pos[k] + c];
    }
}

__global__ void k_fault_fold_blocks(double* diag, const int32_t* __restrict__ neg, const int32_t* __restrict__ pos,
                                    int64_t npairs) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 9 * npairs; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = i / 9, c = i % 9;
        diag[9 * (int64_t)neg[k] + c] += diag[9 * (int64_t)pos[k] + c];
    }
}

// Dirichlet values into the solution: u[i] = values[i] at every DOF the caller constrained (not
// the DOFs the reduced fault formulation eliminates), the other entries untouched (ConstraintSpatialDB::setSolution,
// feassemble/ConstraintSpatialDB.cc:116-159, through DMPlexInsertBoundaryValuesEssentialBdField).
__global__ void k_insert_constrained(double* __restrict__ u, const double* __restrict__ values,
                                     const uint8_t* __restrict__ mask, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (mask[i]) u[i] = values[i];
}

// u+ = u- + d, d = n slip[0] + t1 slip[1] + t2 slip[2] with the fault's tangential directions
// (BoundaryDirections::tangential_directions, the same construction f0l_slip uses).
__global__ void k_fault_apply_slip(double* u, const int32_t* __restrict__ neg, const int32_t* __restrict__ pos,
                                   const double* __restrict__ normal, const double* __restrict__ slip, int64_t npairs,
                                   double r10, double r11, double r12, double r20, double r21, double r22) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < npairs; k += (int64_t)gridDim.x * blockDim.x) {
        const double n[3] = {normal[3 * k], normal[3 * k + 1], normal[3 * k + 2]};
        const double ref1[3] = {r10, r11, r12}, ref2[3] = {r20, r21, r22};
        double t1[3], t2[3];
        pw::tangential_directions(t1, t2, ref1, ref2, n);
        for (int c = 0; c < 3; ++c) {
            const double d = n[c] * slip[3 * k] + t1[c] * slip[3 * k + 1] + t2[c] * slip[3 * k + 2];
            u[3 * (int64_t)pos[k] + c] = u[3 * (int64_t)neg[k] + c] + d;
        }
    }
}

}  // namespace plb

using namespace plb;



namespace {

template <typename T>
void fault_unfold(pl_solver S, T* v) {
    if (S->npairs == 0) return;
    k_fault_unfold<T><<<vec_grid(3 * S->npairs), 256, 0, S->mesh->ctx->stream>>>(v, S->d_pair_neg, S->d_pair_pos, S->npairs);
    count_launch();
}

template <typename T>
void fault_fold(pl_solver S, T* v) {
    if (S->npairs == 0) return;
    k_fault_fold<T><<<vec_grid(3 * S->npairs), 256, 0, S->mesh->ctx->stream>>>(v, S->d_pair_neg, S->d_pair_pos, S->npairs);
    count_launch();
}

// out = P^T J P v: with S->reduced by the kernels' reduced fault space (every positive-side node
// read as, and added into, its negative-side partner), else by unfolding v in place (its
// positive-side entries are written) and folding the result.
int apply_J(pl_solver S, const double* v, double* out) {
    if (S->reduced) {
        for (size_t i = 0; i < S->ops.size(); ++i) {
            int rc = jacobian_action_reduced(S->ops[i], S->t, S->dt, v, out, i == 0 ? PL_INSERT : PL_ADD);
            if (rc) return rc;
        }
        return PL_OK;
    }
    fault_unfold(S, const_cast<double*>(v));
    for (size_t i = 0; i < S->ops.size(); ++i) {
        int rc = pl_compute_lhs_jacobian_action(S->ops[i], S->t, S->dt, 0.0, nullptr, v, out, i == 0 ? PL_INSERT : PL_ADD);
        if (rc) return rc;
    }
    fault_fold(S, out);
    return PL_OK;
}

int apply_J32(pl_solver S, const float* v, float* out) {
    if (S->reduced) {
        for (size_t i = 0; i < S->ops.size(); ++i) {
            int rc = jacobian_action_reduced_f32(S->ops[i], S->t, S->dt, v, out, i == 0 ? PL_INSERT : PL_ADD);
            if (rc) return rc;
        }
        return PL_OK;
    }
    fault_unfold(S, const_cast<float*>(v));
    for (size_t i = 0; i < S->ops.size(); ++i) {
        int rc = pl_compute_lhs_jacobian_action_f32(S->ops[i], S->t, S->dt, v, out, i == 0 ? PL_INSERT : PL_ADD);
        if (rc) return rc;
    }
    fault_fold(S, out);
    return PL_OK;
}

// One PCG iteration on the solver's private stream (capturable).
template <typename T>
int cg_iteration(pl_solver S, T* x, T* r, T* p, T* q, T* z, const T* pinv) {
    const int64_t n = S->n, nn = S->nnodes;
    double* part = S->d_partials;
    double* scal = S->d_scal;
    int rc;
    if constexpr (sizeof(T) == 8) rc = apply_J(S, (const double*)p, (double*)q);
    else rc = apply_J32(S, (const float*)p, (float*)q);
    if (rc) return rc;
    k_cg_pq<T><<<kRedBlocks, kRedThreads, 0, S->cstream>>>(p, q, S->d_mask, n, part);
    k_finish2<<<1, 1024, 0, S->cstream>>>(part, kRedBlocks, scal, S_PQ, -1);
    k_copy_scalar<<<1, 1, 0, S->cstream>>>(scal, S_RZ, S_RZ_OLD);
    k_cg_update<T><<<kRedBlocks, kRedThreads, 0, S->cstream>>>(x, r, p, q, z, S->d_mask, pinv, nn, scal, part);
    k_finish2<<<1, 1024, 0, S->cstream>>>(part, kRedBlocks, scal, S_RZ, S_RR);
    k_cg_pupdate<T><<<vec_grid(n), 256, 0, S->cstream>>>(p, z, n, scal);
    count_launch(6);
    return PL_OK;
}

// The graph of check_every iterations (index 0: FP64, 1: FP32), captured again when the
// integrators changed. The caller has switched the context to the private stream.
template <typename T>
int ensure_cg_graph(pl_solver S, T* x, T* r, T* p, T* q, T* z, const T* pinv) {
    const int gi = sizeof(T) == 8 ? 0 : 1;
    const int chunk = std::max(1, S->check_every);
    if (S->graph[gi] && S->graph_iters[gi] == chunk && S->graph_epoch[gi] == state_epoch()) return PL_OK;
    if (S->graph[gi]) cudaGraphExecDestroy(S->graph[gi]);
    S->graph[gi] = nullptr;
    int rc = PL_OK;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(S->cstream, cudaStreamCaptureModeRelaxed);
    for (int i = 0; i < chunk && rc == PL_OK && e == cudaSuccess; ++i) rc = cg_iteration<T>(S, x, r, p, q, z, pinv);
    if (e == cudaSuccess) e = cudaStreamEndCapture(S->cstream, &g);
    if (e == cudaSuccess && rc == PL_OK) e = cudaGraphInstantiate(&S->graph[gi], g, 0);
    if (g) cudaGraphDestroy(g);
    if (rc == PL_OK && e != cudaSuccess) rc = cuda_fail(e, "PCG graph capture");
    S->graph_iters[gi] = chunk;
    S->graph_epoch[gi] = state_epoch();
    return rc;
}

template <typename T>
int pcg(pl_solver S, const T* b, T* x, double rtol, double atol, int max_iter, const T* pinv, T* r, T* p, T* q, T* z,
        int* iters, double* rel) {
    cudaStream_t s = S->mesh->ctx->stream;
    const int64_t n = S->n, nn = S->nnodes;
    double* part = S->d_partials;
    double* scal = S->d_scal;
    PLB_CUDA(cudaMemsetAsync(x, 0, n * sizeof(T), s));
    k_cg_init<T><<<kRedBlocks, kRedThreads, 0, s>>>(b, S->d_mask, pinv, nn, r, z, p, part);
    k_finish2<<<1, 1024, 0, s>>>(part, kRedBlocks, scal, S_RZ, S_RR);
    count_launch(2);
    double h[S_COUNT];
    PLB_CUDA(cudaMemcpyAsync(h, scal, sizeof(h), cudaMemcpyDeviceToHost, s));
    PLB_CUDA(cudaStreamSynchronize(s));
    const double r0 = std::sqrt(h[S_RR]);
    const double stop = std::max(rtol * r0, atol);
    *iters = 0;
    *rel = r0 > 0.0 ? 1.0 : 0.0;
    if (r0 == 0.0 || r0 <= stop) return PL_OK;
    // The iterations run on the solver's private stream (capture is impossible on the legacy
    // default stream a caller may use), as a CUDA graph of check_every iterations replayed
    // between convergence checks; the graph is captured again when the integrators changed.
    pl_context c = S->mesh->ctx;
    const int gi = sizeof(T) == 8 ? 0 : 1;
    const int chunk = std::max(1, S->check_every);
    if (S->mesh->cell_type == PL_CELL_TET4)
        for (pl_integrator ig : S->ops) {
            int rcl = prepare_blocked(ig);  // allocates: outside any capture
            if (rcl) return rcl;
        }
    PLB_CUDA(cudaEventRecord(S->ev_in, s));
    PLB_CUDA(cudaStreamWaitEvent(S->cstream, S->ev_in, 0));
    c->stream = S->cstream;
    int rc = ensure_cg_graph<T>(S, x, r, p, q, z, pinv);
    for (int it = 0; rc == PL_OK && it < max_iter; it += chunk) {
        cudaError_t e = cudaGraphLaunch(S->graph[gi], S->cstream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(h, scal, sizeof(h), cudaMemcpyDeviceToHost, S->cstream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(S->cstream);
        if (e != cudaSuccess) {
            rc = cuda_fail(e, "PCG iterations");
            break;
        }
        *iters = it + chunk;
        const double rn = std::sqrt(h[S_RR]);
        *rel = rn / r0;
        if (!(rn == rn)) {
            rc = fail(PL_ERR_NOT_CONVERGED, "PCG diverged (NaN residual)");
            break;
        }
        if (rn <= stop) break;
        if (it + chunk >= max_iter) rc = fail(PL_ERR_NOT_CONVERGED, "PCG reached the iteration limit");
    }
    c->stream = s;
    cudaEventRecord(S->ev_out, S->cstream);
    cudaStreamWaitEvent(s, S->ev_out, 0);
    return rc;
}

// FP32 PCG with reliable updates (residual replacement; van der Vorst and Ye, SIAM J. Sci.
// Comput. 22 (2000); the mixed-precision CG of Clark et al., Comput. Phys. Commun. 181 (2010)):
// one FP32 PCG without restarts; whenever its iterated residual has dropped below
// reliable_delta times the last FP64 true residual, the FP32 correction is added to the FP64
// solution x, r is replaced by the FP64 true residual b - A x (and z = P r, r.z recomputed), and
// the search direction is kept. Ends when the true residual meets rtol (or atol).
int pcg32_reliable(pl_solver S, const double* b, double* x) {
    cudaStream_t s = S->mesh->ctx->stream;
    pl_context c = S->mesh->ctx;
    const int64_t n = S->n, nn = S->nnodes;
    double* scal = S->d_scal;
    double h[S_COUNT];
    if (S->mesh->cell_type == PL_CELL_TET4)
        for (pl_integrator ig : S->ops) {
            int rcl = prepare_blocked(ig);  // allocates: outside any capture
            if (rcl) return rcl;
        }
    PLB_CUDA(cudaEventRecord(S->ev_in, s));
    PLB_CUDA(cudaStreamWaitEvent(S->cstream, S->ev_in, 0));
    c->stream = S->cstream;
    cudaStream_t cs = S->cstream;
    int rc = PL_OK;
    // FP64 true residual of x into d_r (and f_r); returns |r|
    auto true_residual = [&](double* rn) -> int {
        int r2 = apply_J(S, x, S->d_q);
        if (r2) return r2;
        k_outer_residual<<<kRedBlocks, kRedThreads, 0, cs>>>(b, S->d_q, S->d_mask, n, S->d_r, S->f_r, S->d_partials);
        k_finish2<<<1, 1024, 0, cs>>>(S->d_partials, kRedBlocks, scal, S_BB, -1);
        count_launch(2);
        PLB_CUDA(cudaMemcpyAsync(h, scal, sizeof(h), cudaMemcpyDeviceToHost, cs));
        PLB_CUDA(cudaStreamSynchronize(cs));
        *rn = std::sqrt(h[S_BB]);
        return PL_OK;
    };
    double b0 = 0.0, rt = 0.0;
    int breakdowns = 0;
    do {
        if (cudaMemsetAsync(x, 0, n * sizeof(double), cs) != cudaSuccess ||
            cudaMemsetAsync(S->f_x, 0, n * sizeof(float), cs) != cudaSuccess) {
            rc = fail(PL_ERR_CUDA, "memset");
            break;
        }
        if ((rc = true_residual(&b0)) != PL_OK) break;
        rt = b0;
        const double stop = std::max(S->rtol * b0, S->atol);
        if (b0 == 0.0 || b0 <= stop) break;
        k_cg_init<float><<<kRedBlocks, kRedThreads, 0, cs>>>(S->f_r, S->d_mask, S->d_pinv32, nn, S->f_r, S->f_z, S->f_p,
                                                               S->d_partials);
        k_finish2<<<1, 1024, 0, cs>>>(S->d_partials, kRedBlocks, scal, S_RZ, S_RR);
        count_launch(2);
        if ((rc = ensure_cg_graph<float>(S, S->f_x, S->f_r, S->f_p, S->f_q, S->f_z, S->d_pinv32)) != PL_OK) break;
        const int chunk = std::max(1, S->check_every);
        double rref = b0;
        bool done = false;
        for (int it = 0; !done; it += chunk) {
            if (it >= S->max_iter) {
                rc = fail(PL_ERR_NOT_CONVERGED, "PCG reached the iteration limit");
                break;
            }
            cudaError_t e = cudaGraphLaunch(S->graph[1], cs);
            if (e == cudaSuccess) e = cudaMemcpyAsync(h, scal, sizeof(h), cudaMemcpyDeviceToHost, cs);
            if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
            if (e != cudaSuccess) {
                rc = cuda_fail(e, "PCG iterations");
                break;
            }
            S->inner_iterations += chunk;
            const double rn = std::sqrt(h[S_RR]);
            // FP32 breakdown: the iterated residual is not a number, or has grown far above the
            // last true residual (FP32 rounding of a nearly converged system can turn p.(A p) into
            // noise). The FP32 correction since the last replacement is dropped and the iteration
            // starts again from the true residual.
            const bool broke = !(rn == rn) || rn > kBreakdownGrowth * rref;
            if (!broke && rn > S->reliable_delta * rref && rn > 0.5 * stop) continue;
            if (broke && ++breakdowns > kMaxBreakdowns) {
                rc = fail(PL_ERR_NOT_CONVERGED, "FP32 PCG keeps breaking down");
                break;
            }
            if (!broke) {
                k_add_correction<<<vec_grid(n), 256, 0, cs>>>(x, S->f_x, S->d_mask, n);
                count_launch();
            }
            if (cudaMemsetAsync(S->f_x, 0, n * sizeof(float), cs) != cudaSuccess) {
                rc = fail(PL_ERR_CUDA, "memset");
                break;
            }
            if ((rc = true_residual(&rt)) != PL_OK) break;
            S->outer_iterations++;
            if (rt <= stop) {
                done = true;
                break;
            }
            rref = rt;
            k_prec_rz<float><<<kRedBlocks, kRedThreads, 0, cs>>>(S->f_r, S->d_pinv32, nn, S->f_z, S->d_partials);
            k_finish2<<<1, 1024, 0, cs>>>(S->d_partials, kRedBlocks, scal, S_RZ, -1);
            count_launch(2);
            // The FP32 iterations had run below the stopping threshold while the true residual had
            // not, or had broken down: their search direction is rounding noise, so restart it from z.
            if ((broke || rn <= 0.5 * stop) &&
                cudaMemcpyAsync(S->f_p, S->f_z, n * sizeof(float), cudaMemcpyDeviceToDevice, cs) != cudaSuccess) {
                rc = fail(PL_ERR_CUDA, "search direction restart");
                break;
            }
        }
    } while (false);
    S->rel_residual = b0 > 0.0 ? rt / b0 : 0.0;
    c->stream = s;
    cudaEventRecord(S->ev_out, cs);
    cudaStreamWaitEvent(s, S->ev_out, 0);
    fault_unfold(S, x);  // the positive side of every fault node follows its negative side
    return rc;
}

}  // namespace

namespace plb {

// Operator pieces for outside drivers (the multigrid hierarchy): q = J v with the fault's unfold
// and fold (FP64, FP32), and the unfold / fold alone.
int solver_apply_J(pl_solver S, const double* v, double* out) { return apply_J(S, v, out); }
int solver_apply_J32(pl_solver S, const float* v, float* out) { return apply_J32(S, v, out); }
void solver_unfold(pl_solver S, double* v) { fault_unfold(S, v); }
void solver_unfold32(pl_solver S, float* v) { fault_unfold(S, v); }
void solver_fold(pl_solver S, double* v) { fault_fold(S, v); }
void solver_fold32(pl_solver S, float* v) { fault_fold(S, v); }

// The reduced system's right-hand side P^T b (the two sides' equations of every fault node summed;
// the solver's d_x holds it) when the mesh has faults, else b itself.
const double* solver_reduced_rhs(pl_solver S, const double* b) {
    if (S->npairs == 0) return b;
    cudaMemcpyAsync(S->d_x, b, S->n * sizeof(double), cudaMemcpyDeviceToDevice, S->mesh->ctx->stream);
    fault_fold(S, S->d_x);
    return S->d_x;
}

// The FP32 reliable-update PCG of one solver, driven step by step by an outside loop (the ragged
// batch runs the iterations of many solvers in shared launches). Both run on the context's
// stream and synchronise it.
//
// Start: x = 0, FP64 residual r = b - A x (d_r, and f_r in FP32), z = P r, p = z, r.z and r.r in
// the solver's scalars, q = 0; *b0 = |r|.
int solver32_begin(pl_solver S, const double* b, double* x, double* b0) {
    pl_context c = S->mesh->ctx;
    cudaStream_t s = c->stream;
    const int64_t n = S->n;
    double h[S_COUNT];
    PLB_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), s));
    PLB_CUDA(cudaMemsetAsync(S->f_x, 0, n * sizeof(float), s));
    PLB_CUDA(cudaMemsetAsync(S->f_q, 0, n * sizeof(float), s));
    if (S->mesh->cell_type == PL_CELL_TET4)
        for (pl_integrator ig : S->ops) {
            int rcl = prepare_blocked(ig);
            if (rcl) return rcl;
        }
    int rc = apply_J(S, x, S->d_q);
    if (rc) return rc;
    k_outer_residual<<<kRedBlocks, kRedThreads, 0, s>>>(b, S->d_q, S->d_mask, n, S->d_r, S->f_r, S->d_partials);
    k_finish2<<<1, 1024, 0, s>>>(S->d_partials, kRedBlocks, S->d_scal, S_BB, -1);
    k_cg_init<float><<<kRedBlocks, kRedThreads, 0, s>>>(S->f_r, S->d_mask, S->d_pinv32, S->nnodes, S->f_r, S->f_z, S->f_p,
                                                         S->d_partials);
    k_finish2<<<1, 1024, 0, s>>>(S->d_partials, kRedBlocks, S->d_scal, S_RZ, S_RR);
    count_launch(4);
    PLB_CUDA(cudaMemcpyAsync(h, S->d_scal, sizeof(h), cudaMemcpyDeviceToHost, s));
    PLB_CUDA(cudaStreamSynchronize(s));
    *b0 = std::sqrt(h[S_BB]);
    return PL_OK;
}

// Residual replacement: x += f_x (unless the correction is dropped after a breakdown), f_x = 0,
// r = b - A x in FP64 (*rt = |r|), r.z for the new r (z = P r); with restart the search direction
// starts again from z; q = 0.
int solver32_replace(pl_solver S, const double* b, double* x, bool restart, bool keep_correction, double* rt) {
    pl_context c = S->mesh->ctx;
    cudaStream_t s = c->stream;
    const int64_t n = S->n;
    double h[S_COUNT];
    if (keep_correction) {
        k_add_correction<<<vec_grid(n), 256, 0, s>>>(x, S->f_x, S->d_mask, n);
        count_launch();
    }
    PLB_CUDA(cudaMemsetAsync(S->f_x, 0, n * sizeof(float), s));
    int rc = apply_J(S, x, S->d_q);
    if (rc) return rc;
    k_outer_residual<<<kRedBlocks, kRedThreads, 0, s>>>(b, S->d_q, S->d_mask, n, S->d_r, S->f_r, S->d_partials);
    k_finish2<<<1, 1024, 0, s>>>(S->d_partials, kRedBlocks, S->d_scal, S_BB, -1);
    k_prec_rz<float><<<kRedBlocks, kRedThreads, 0, s>>>(S->f_r, S->d_pinv32, S->nnodes, S->f_z, S->d_partials);
    k_finish2<<<1, 1024, 0, s>>>(S->d_partials, kRedBlocks, S->d_scal, S_RZ, -1);
    count_launch(4);
    if (restart) PLB_CUDA(cudaMemcpyAsync(S->f_p, S->f_z, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
    PLB_CUDA(cudaMemsetAsync(S->f_q, 0, n * sizeof(float), s));
    PLB_CUDA(cudaMemcpyAsync(h, S->d_scal, sizeof(h), cudaMemcpyDeviceToHost, s));
    PLB_CUDA(cudaStreamSynchronize(s));
    *rt = std::sqrt(h[S_BB]);
    return PL_OK;
}

}  // namespace plb

extern "C" {

int pl_solver_create(pl_mesh m, const uint8_t* constrained, pl_solver* out) {
    if (!m || !out) return fail(PL_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    // Fault nodes: (negative node, positive node, normal) per Lagrange node, from the cohesive cells.
    std::vector<int32_t> pneg(m->nlag, -1), ppos(m->nlag, -1);
    std::vector<double> pnrm(3 * m->nlag, 0.0);
    for (int64_t c = 0; c < m->ncoh; ++c) {
        const int32_t* cc = &m->h_coh[12 * c];
        double X[4][3];
        for (int a = 0; a < 4; ++a)
            for (int d = 0; d < 3; ++d) X[a][d] = m->h_coords[3 * (int64_t)cc[a] + d];
        double dxi[3], deta[3];
        for (int d = 0; d < 3; ++d) {
            dxi[d] = X[1][d] + X[2][d] - X[0][d] - X[3][d];
            deta[d] = X[2][d] + X[3][d] - X[0][d] - X[1][d];
        }
        double nrm[3] = {dxi[1] * deta[2] - dxi[2] * deta[1], dxi[2] * deta[0] - dxi[0] * deta[2],
                         dxi[0] * deta[1] - dxi[1] * deta[0]};
        const double mag = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
        for (int a = 0; a < 4; ++a) {
            const int32_t l = cc[8 + a];
            if (pneg[l] >= 0 && (pneg[l] != cc[a] || ppos[l] != cc[4 + a]))
                return fail(PL_ERR_INVALID_ARG, "inconsistent cohesive cells: a fault node maps to two node pairs");
            pneg[l] = cc[a];
            ppos[l] = cc[4 + a];
            for (int d = 0; d < 3; ++d) pnrm[3 * l + d] = nrm[d] / mag;
        }
    }
    for (int64_t l = 0; l < m->nlag; ++l)
        if (pneg[l] < 0) return fail(PL_ERR_INVALID_ARG, "fault node without a cohesive cell");
    pl_solver S = new pl_solver_s();
    S->mesh = m;
    mesh_retain(m);
    S->nnodes = m->nnodes + m->nlag;
    S->n = 3 * S->nnodes;
    S->npairs = m->nlag;
    PLB_CUDA(cudaSetDevice(m->ctx->device));
    const int64_t n = S->n;
    cudaError_t e = cudaSuccess;
    auto A = [&](auto** p, size_t cnt) {
        if (e == cudaSuccess) e = dev_alloc(p, cnt);
    };
    A(&S->d_mask, n);
    A(&S->d_dirichlet, n);
    A(&S->d_diag, 9 * S->nnodes);
    A(&S->d_pinv, 9 * S->nnodes);
    A(&S->d_pinv32, 9 * S->nnodes);
    A(&S->d_r, n); A(&S->d_p, n); A(&S->d_q, n); A(&S->d_z, n); A(&S->d_x, n); A(&S->d_xs, n);
    A(&S->f_r, n); A(&S->f_p, n); A(&S->f_q, n); A(&S->f_z, n); A(&S->f_x, n);
    A(&S->d_scal, S_COUNT);
    A(&S->d_partials, 2 * kRedBlocks);
    if (S->npairs > 0) {
        A(&S->d_pair_neg, S->npairs);
        A(&S->d_pair_pos, S->npairs);
        A(&S->d_pair_normal, 3 * S->npairs);
    }
    cudaStream_t s = m->ctx->stream;
    // Unknowns: DOFs not constrained by the caller, minus the positive side of fault nodes and
    // the Lagrange-multiplier DOFs (eliminated by the reduced formulation).
    std::vector<uint8_t> mask(n, 0);
    if (constrained) std::memcpy(mask.data(), constrained, n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(S->d_dirichlet, mask.data(), n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the host mask is modified below
    for (int64_t l = 0; l < S->npairs; ++l)
        for (int d = 0; d < 3; ++d) {
            mask[3 * (int64_t)ppos[l] + d] = 1;
            mask[3 * (m->nnodes + l) + d] = 1;
        }
    if (e == cudaSuccess) e = cudaMemcpyAsync(S->d_mask, mask.data(), n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && S->npairs > 0) {
        e = cudaMemcpyAsync(S->d_pair_neg, pneg.data(), pneg.size() * 4, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(S->d_pair_pos, ppos.data(), ppos.size() * 4, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(S->d_pair_normal, pnrm.data(), pnrm.size() * 8, cudaMemcpyHostToDevice, s);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(S->d_scal, 0, S_COUNT * sizeof(double), s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->cstream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S->ev_in, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S->ev_out, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        pl_solver_destroy(S);
        return cuda_fail(e, "pl_solver_create");
    }
    *out = S;
    return PL_OK;
}

int pl_solver_add_integrator(pl_solver S, pl_integrator ig) {
    if (!S || !ig || ig->mesh != S->mesh) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    if (ig->is_interface)
        return fail(PL_ERR_INVALID_ARG, "interface integrators are not part of the reduced operator; "
                                        "pass them to pl_solver_apply_fault_slip");
    if (ig->j3 == K_NONE) return fail(PL_ERR_NOT_READY, "integrator has no Jacobian kernels");
    integrator_retain(ig);  // kept alive until the solver is freed (the solver's graphs use it)
    S->ops.push_back(ig);
    S->ready = false;
    return PL_OK;
}

int pl_solver_set_tolerances(pl_solver S, double rtol, double atol, int max_iter) {
    if (!S || rtol < 0 || atol < 0 || max_iter <= 0) return fail(PL_ERR_INVALID_ARG, "bad tolerances");
    S->rtol = rtol;
    S->atol = atol;
    S->max_iter = max_iter;
    return PL_OK;
}

int pl_solver_set_reliable(pl_solver S, int enable, double delta) {
    if (!S || !(delta > 0.0 && delta < 1.0)) return fail(PL_ERR_INVALID_ARG, "delta must lie in (0, 1)");
    S->reliable = enable != 0;
    S->reliable_delta = delta;
    return PL_OK;
}

int pl_solver_set_precision(pl_solver S, int precision, double inner_rtol) {
    if (!S || (precision != PL_SOLVER_FP64 && precision != PL_SOLVER_FP32_REFINED) || !(inner_rtol > 0 && inner_rtol < 1))
        return fail(PL_ERR_INVALID_ARG, "bad precision settings");
    S->precision = precision;
    S->inner_rtol = inner_rtol;
    return PL_OK;
}

int pl_solver_setup(pl_solver S, double t, double dt) {
    if (!S || S->ops.empty()) return fail(PL_ERR_NOT_READY, "no integrators");
    pl_mesh m = S->mesh;
    cudaStream_t s = m->ctx->stream;
    PLB_CUDA(cudaSetDevice(m->ctx->device));
    S->t = t;
    S->dt = dt;
    bump_state_epoch();  // t and dt are arguments of captured kernels: re-capture
    PLB_CUDA(cudaMemsetAsync(S->d_diag, 0, 9 * S->nnodes * sizeof(double), s));
    for (pl_integrator ig : S->ops) {
        DomainParams p;
        int rc = bind_domain_jacobian(ig, &p);
        if (rc) return rc;
        p.t = t;
        p.dt = dt;
        launch_domain_diag_blocks(p, m->cell_type, ig->j3 == K_ILE_JF3VU ? RHEO_ILE : RHEO_GENMAXWELL, S->d_diag, s);
        if (S->precision != PL_SOLVER_FP64 && (rc = prepare_jv32_tangent(ig, t, dt)) != PL_OK) return rc;
    }
    if (S->npairs > 0) {
        k_fault_fold_blocks<<<vec_grid(9 * S->npairs), 256, 0, s>>>(S->d_diag, S->d_pair_neg, S->d_pair_pos, S->npairs);
        count_launch();
    }
    // the operator in the reduced fault space without unfold and fold launches, when every
    // integrator supports it (PYLITH_B200_REDUCED_KERNELS=0: always unfold and fold)
    S->reduced = false;
    if (S->npairs > 0) {
        const char* env = std::getenv("PYLITH_B200_REDUCED_KERNELS");
        bool ok = !(env && env[0] == '0');
        for (pl_integrator ig : S->ops) ok = ok && jacobian_action_reduced_supported(ig);
        S->reduced = ok;
    }
    k_invert_blocks<<<vec_grid(S->nnodes), 256, 0, s>>>(S->d_diag, S->d_mask, S->nnodes, S->d_pinv, S->d_pinv32);
    count_launch();
    PLB_CUDA(cudaGetLastError());
    if (S->mg) {
        int rc = multigrid_setup(S->mg, t, dt);
        if (rc) return rc;
    }
    S->ready = true;
    return PL_OK;
}

int pl_solver_solve(pl_solver S, const double* b, double* x) {
    if (!S || !b || !x) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    if (!S->ready) return fail(PL_ERR_NOT_READY, "call pl_solver_setup first");
    pl_mesh m = S->mesh;
    cudaStream_t s = m->ctx->stream;
    PLB_CUDA(cudaSetDevice(m->ctx->device));
    S->iterations = S->inner_iterations = S->outer_iterations = 0;
    if (S->mg) return multigrid_solve(S->mg, b, x);
    const int64_t n = S->n;
    if (S->npairs > 0) {  // right-hand side of the reduced system: P^T b
        PLB_CUDA(cudaMemcpyAsync(S->d_x, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        fault_fold(S, S->d_x);
        b = S->d_x;
    }
    if (S->precision == PL_SOLVER_FP64) {
        int it = 0;
        double rel = 0.0;
        int rc = pcg<double>(S, b, S->d_xs, S->rtol, S->atol, S->max_iter, S->d_pinv, S->d_r, S->d_p, S->d_q, S->d_z,
                             &it, &rel);
        PLB_CUDA(cudaMemcpyAsync(x, S->d_xs, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        fault_unfold(S, x);
        S->iterations = it;
        S->rel_residual = rel;
        return rc;
    }
    if (S->reliable) return pcg32_reliable(S, b, x);
    // FP64 iterative refinement around FP32 PCG (x unfolded before it is returned).
    PLB_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), s));
    double h[S_COUNT];
    double b0 = -1.0;
    for (int outer = 0; outer < 50; ++outer) {
        int rc = apply_J(S, x, S->d_q);
        if (rc) return rc;
        k_outer_residual<<<kRedBlocks, kRedThreads, 0, s>>>(b, S->d_q, S->d_mask, n, S->d_r, S->f_r, S->d_partials);
        k_finish2<<<1, 1024, 0, s>>>(S->d_partials, kRedBlocks, S->d_scal, S_BB, -1);
        count_launch(2);
        PLB_CUDA(cudaMemcpyAsync(h, S->d_scal, sizeof(h), cudaMemcpyDeviceToHost, s));
        PLB_CUDA(cudaStreamSynchronize(s));
        const double rn = std::sqrt(h[S_BB]);
        if (b0 < 0.0) b0 = rn;
        S->rel_residual = b0 > 0.0 ? rn / b0 : 0.0;
        S->outer_iterations = outer;
        if (rn <= std::max(S->rtol * b0, S->atol) || b0 == 0.0) {
            fault_unfold(S, x);
            return PL_OK;
        }
        int it = 0;
        double rel = 0.0;
        // Inner solve A d = r in FP32 (d in f_x).
        // The right-hand side f_r doubles as the inner residual vector (read before written).
        rc = pcg<float>(S, S->f_r, S->f_x, S->inner_rtol, 0.0, S->max_iter, S->d_pinv32, S->f_r, S->f_p, S->f_q, S->f_z,
                        &it, &rel);
        if (rc && rc != PL_ERR_NOT_CONVERGED) return rc;
        S->inner_iterations += it;
        k_add_correction<<<vec_grid(n), 256, 0, s>>>(x, S->f_x, S->d_mask, n);
        count_launch();
    }
    fault_unfold(S, x);
    return fail(PL_ERR_NOT_CONVERGED, "iterative refinement did not converge");
}

int pl_solver_insert_constrained(pl_solver S, const double* values, double* u) {
    if (!S || !values || !u) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    PLB_CUDA(cudaSetDevice(S->mesh->ctx->device));
    const int64_t n = S->n;
    k_insert_constrained<<<vec_grid(n), 256, 0, S->mesh->ctx->stream>>>(u, values, S->d_dirichlet, n);
    count_launch();
    PLB_CUDA(cudaGetLastError());
    return PL_OK;
}

int pl_solver_apply_fault_slip(pl_solver S, pl_integrator iface, double* u) {
    if (!S || !iface || !u || !iface->is_interface || iface->mesh != S->mesh)
        return fail(PL_ERR_INVALID_ARG, "bad arguments");
    if (S->npairs == 0) return PL_OK;
    const AuxField* slip = nullptr;
    for (const AuxField& f : iface->aux)
        if (f.name == "slip") slip = &f;
    if (!slip || slip->ncomp != 3 || slip->storage != PL_AUX_PER_FAULT_NODE)
        return fail(PL_ERR_INVALID_ARG, "interface integrator needs the slip(3) aux subfield per fault node");
    if (iface->constants.size() < 6) return fail(PL_ERR_INVALID_ARG, "interface integrator needs constants refDir1, refDir2");
    const std::vector<double>& c = iface->constants;
    PLB_CUDA(cudaSetDevice(S->mesh->ctx->device));
    k_fault_apply_slip<<<vec_grid(S->npairs), 256, 0, S->mesh->ctx->stream>>>(
        u, S->d_pair_neg, S->d_pair_pos, S->d_pair_normal, slip->d, S->npairs, c[0], c[1], c[2], c[3], c[4], c[5]);
    count_launch();
    PLB_CUDA(cudaGetLastError());
    return PL_OK;
}

int pl_solver_get_stats(pl_solver S, int* iterations, int* inner_iterations, int* outer_iterations, double* rel_residual) {
    if (!S) return fail(PL_ERR_INVALID_ARG, "null solver");
    if (iterations) *iterations = S->iterations;
    if (inner_iterations) *inner_iterations = S->inner_iterations;
    if (outer_iterations) *outer_iterations = S->outer_iterations;
    if (rel_residual) *rel_residual = S->rel_residual;
    return PL_OK;
}

}  // extern "C"

static void solver_free(pl_solver S) {
    if (S->mg) multigrid_detach(S->mg);
    cudaSetDevice(S->mesh->ctx->device);
    cudaStreamSynchronize(S->mesh->ctx->stream);
    for (cudaGraphExec_t g : S->graph)
        if (g) cudaGraphExecDestroy(g);
    if (S->cstream) cudaStreamSynchronize(S->cstream);
    if (S->ev_in) cudaEventDestroy(S->ev_in);
    if (S->ev_out) cudaEventDestroy(S->ev_out);
    if (S->cstream) cudaStreamDestroy(S->cstream);
    void* ptrs[] = {S->d_mask, S->d_dirichlet, S->d_diag, S->d_pinv, S->d_pinv32, S->d_r, S->d_p, S->d_q, S->d_z, S->d_x,
                    S->d_xs, S->f_r, S->f_p, S->f_q, S->f_z, S->f_x, S->d_scal, S->d_partials,
                    S->d_pair_neg, S->d_pair_pos, S->d_pair_normal};
    for (void* p : ptrs) dev_free(p, S->mesh->ctx->stream);
    std::vector<pl_integrator> ops;
    ops.swap(S->ops);
    pl_mesh m = S->mesh;
    delete S;
    for (pl_integrator ig : ops) integrator_release(ig);
    mesh_release(m);
}

namespace plb {
void solver_retain(pl_solver_s* S) { S->refs++; }
void solver_release(pl_solver_s* S) {
    if (--S->refs == 0 && S->destroy_requested) solver_free(S);
}
}  // namespace plb

extern "C" {

int pl_solver_destroy(pl_solver S) {
    if (!S) return PL_OK;
    if (S->refs > 0) {
        S->destroy_requested = true;
        return PL_OK;
    }
    solver_free(S);
    return PL_OK;
}

}  // extern "C"
