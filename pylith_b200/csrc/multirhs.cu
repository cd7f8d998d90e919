// Many right-hand sides at once: the batched Green's-function solve.
//
// The reference solves its Green's-function impulses one SNES/KSP solve at a time
// (libsrc/pylith/problems/GreensFns.cc:291-337, one impulse per solve, the Jacobian lagged and
// reused: SNESSetLagJacobian(-2) at :236-241). Here a tile of K right-hand sides shares every
// launch:
//   * k_tet_blocked_jv32_multi<K>: the FP32 Jacobian action of K vectors per cell block; the
//     geometry (cofactors, 1/det in FP64), the tangent and the block metadata are read and formed
//     once and applied to all K vectors, which are interleaved per DOF ([ndof][K]) so one node's
//     K values are contiguous; element contributions are summed in shared memory (native FP32
//     shared atomics) and written once per node;
//   * a batched PCG whose vector kernels update all K vectors with per-RHS step lengths and FP64
//     dot products, captured in a CUDA graph and replayed between convergence checks;
//   * FP64 iterative refinement per RHS around the FP32 tile solve (outer residual b - A x in
//     FP64 with the single-RHS FP64 action).
#include <cuda_pipeline.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "domain_kernels.cuh"
#include "internal.hpp"
#include "launch.hpp"

namespace plb {

#ifndef PLB_TET_BLOCK
#define PLB_TET_BLOCK 256
#endif
constexpr int kMultiBlockCells = PLB_TET_BLOCK;  // the cell-block layout's cells per block
constexpr uint32_t kSharedBitM = 0x80000000u;

PL_D double tet_cof_m(const double X[4][3], double cof[3][3]) {
    double J[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        J[i][0] = X[1][i] - X[0][i];
        J[i][1] = X[2][i] - X[0][i];
        J[i][2] = X[3][i] - X[0][i];
    }
    cof[0][0] = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    cof[0][1] = J[0][2] * J[2][1] - J[0][1] * J[2][2];
    cof[0][2] = J[0][1] * J[1][2] - J[0][2] * J[1][1];
    cof[1][0] = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    cof[1][1] = J[0][0] * J[2][2] - J[0][2] * J[2][0];
    cof[1][2] = J[0][2] * J[1][0] - J[0][0] * J[1][2];
    cof[2][0] = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    cof[2][1] = J[0][1] * J[2][0] - J[0][0] * J[2][1];
    cof[2][2] = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    return J[0][0] * cof[0][0] + J[0][1] * cof[1][0] + J[0][2] * cof[2][0];
}

// v, out: [ndof][K] FP32 (ndof = 3 * nodes, node-major); out must be zeroed or hold the sum to add to.
template <int K>
__global__ void __launch_bounds__(kMultiBlockCells) k_tet_blocked_jv32_multi(
    DomainParams p, const int32_t* __restrict__ slot_begin, const uint32_t* __restrict__ slot_node,
    const ushort4* __restrict__ lconn, int64_t nblocks, const float* __restrict__ v, float* out) {
    using L = AuxLayout<RHEO_ILE, false>;
    extern __shared__ __align__(16) char smem_raw[];
    const AuxOffsets<RHEO_ILE, false> aoff;
    for (int64_t b = blockIdx.x; b < nblocks; b += gridDim.x) {
        const int s0 = slot_begin[b];
        const int ns = slot_begin[b + 1] - s0;
        double* sX = reinterpret_cast<double*>(smem_raw);       // [ns][3]
        float* sV = reinterpret_cast<float*>(sX + 3 * ns);        // [ns][3][K]
        float* sR = sV + 3 * K * ns;                              // [ns][3][K]
        for (int i = threadIdx.x; i < ns; i += blockDim.x) {
            const int64_t nd = slot_node[s0 + i] & ~kSharedBitM;
#pragma unroll
            for (int d = 0; d < 3; ++d) sX[3 * i + d] = p.coords[3 * nd + d];
#pragma unroll
            for (int j = 0; j < 3 * K; ++j) {
                sV[3 * K * i + j] = v[3 * K * nd + j];
                sR[3 * K * i + j] = 0.0f;
            }
        }
        __syncthreads();
        const int64_t c = b * kMultiBlockCells + threadIdx.x;
        if (c < p.ncells) {
            const ushort4 lc = lconn[c];
            const int ln[4] = {lc.x, lc.y, lc.z, lc.w};
            double X[4][3];
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int d = 0; d < 3; ++d) X[k][d] = sX[3 * ln[k] + d];
            double cof[3][3];
            const double det = tet_cof_m(X, cof);
            if (!(det > 0.0)) flag_error(p.err, CHECK_NONPOSITIVE_DETJ);
            const double rdet = 1.0 / det;
            float inv[3][3], cf[3][3];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    inv[i][j] = (float)(cof[i][j] * rdet);
                    cf[i][j] = (float)(cof[i][j] * (1.0 / 6.0));
                }
            double a[L::size];
            L::load_cell(p, c, a);
            double x[3] = {0, 0, 0};
            double Jf3d[81];
#pragma unroll
            for (int i = 0; i < 81; ++i) Jf3d[i] = 0.0;
            call_jf3<RHEO_ILE>(L::numA, aoff.v, a, p, x, Jf3d);
#pragma unroll 1
            for (int r = 0; r < K; ++r) {
                float s_x[9];
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) {
                    const float u0 = sV[(3 * ln[0] + cc) * K + r];
                    const float g0 = sV[(3 * ln[1] + cc) * K + r] - u0;
                    const float g1 = sV[(3 * ln[2] + cc) * K + r] - u0;
                    const float g2 = sV[(3 * ln[3] + cc) * K + r] - u0;
#pragma unroll
                    for (int d = 0; d < 3; ++d) s_x[cc * 3 + d] = g0 * inv[0][d] + g1 * inv[1][d] + g2 * inv[2][d];
                }
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
                float e0[3] = {0.f, 0.f, 0.f};
#pragma unroll
                for (int k = 0; k < 3; ++k)
#pragma unroll
                    for (int cc = 0; cc < 3; ++cc) {
                        const float val = f1[cc * 3 + 0] * cf[k][0] + f1[cc * 3 + 1] * cf[k][1] + f1[cc * 3 + 2] * cf[k][2];
                        e0[cc] -= val;
                        atomicAdd(&sR[(3 * ln[k + 1] + cc) * K + r], val);
                    }
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) atomicAdd(&sR[(3 * ln[0] + cc) * K + r], e0[cc]);
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < ns; i += blockDim.x) {
            const uint32_t id = slot_node[s0 + i];
            float* o = out + 3 * K * (int64_t)(id & ~kSharedBitM);
            if (id & kSharedBitM) {
#pragma unroll
                for (int j = 0; j < 3 * K; ++j) red_add(o + j, sR[3 * K * i + j]);
            } else {
#pragma unroll
                for (int j = 0; j < 3 * K; ++j) o[j] += sR[3 * K * i + j];
            }
        }
        __syncthreads();
    }
}

// ---- batched vector kernels, layout [n][K] -------------------------------------------------
constexpr int kBThreads = 256;
constexpr int kBBlocks = 296;

// Per-block sums of K values -> partials[blk][K].
template <int K>
PL_D void block_sumK(double (&acc)[K], double* partials) {
    __shared__ double sh[K][kBThreads / 32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double a = acc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if (l == 0) sh[k][w] = a;
    }
    __syncthreads();
    if (threadIdx.x < K) {
        double s = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += sh[threadIdx.x][i];
        partials[blockIdx.x * K + threadIdx.x] = s;
    }
}

// Fixed-order final sums: out[k] = sum_blk partials[blk][k].
template <int K>
__global__ void k_b_finish(const double* __restrict__ partials, int nblk, double* out) {
    const int k = threadIdx.x;
    if (k >= K) return;
    double s = 0.0;
    for (int i = 0; i < nblk; ++i) s += partials[i * K + k];
    out[k] = s;
}

template <int K>
PL_D void pinv_apply_K(const float* __restrict__ P, const float* r, int64_t node, float z[3][K]) {
    const float* B = P + 9 * node;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const float r0 = r[(3 * node + 0) * K + k], r1 = r[(3 * node + 1) * K + k], r2 = r[(3 * node + 2) * K + k];
        z[0][k] = B[0] * r0 + B[1] * r1 + B[2] * r2;
        z[1][k] = B[3] * r0 + B[4] * r1 + B[5] * r2;
        z[2][k] = B[6] * r0 + B[7] * r1 + B[8] * r2;
    }
}

// r = b (masked); z = P r; p = z; partial (r.z)[K], (r.r)[K]
template <int K>
__global__ void __launch_bounds__(kBThreads) k_b_init(float* r, float* z, float* p, const uint8_t* mask, const float* P,
                                                      int64_t nnodes, double* part_rz, double* part_rr) {
    double rz[K], rr[K];
#pragma unroll
    for (int k = 0; k < K; ++k) rz[k] = rr[k] = 0.0;
    for (int64_t nd = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; nd < nnodes; nd += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int c = 0; c < 3; ++c)
            if (mask[3 * nd + c])
#pragma unroll
                for (int k = 0; k < K; ++k) r[(3 * nd + c) * K + k] = 0.0f;
        float zz[3][K];
        pinv_apply_K<K>(P, r, nd, zz);
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const int64_t i = (3 * nd + c) * K + k;
                z[i] = zz[c][k];
                p[i] = zz[c][k];
                rz[k] += (double)r[i] * zz[c][k];
                rr[k] += (double)r[i] * r[i];
            }
    }
    block_sumK<K>(rz, part_rz);
    __syncthreads();
    block_sumK<K>(rr, part_rr);
}

// partial p.(A p) with q = J p: -p.q over free DOFs
template <int K>
__global__ void __launch_bounds__(kBThreads) k_b_pq(const float* p, const float* q, const uint8_t* mask, int64_t n,
                                                    double* part) {
    double s[K];
#pragma unroll
    for (int k = 0; k < K; ++k) s[k] = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (mask[i]) continue;
#pragma unroll
        for (int k = 0; k < K; ++k) s[k] -= (double)p[i * K + k] * q[i * K + k];
    }
    block_sumK<K>(s, part);
}

// alpha_k = active_k ? rz_k / pq_k : 0; x += alpha p; r += alpha q; z = P r; partial rz, rr
template <int K>
__global__ void __launch_bounds__(kBThreads) k_b_update(float* x, float* r, const float* p, const float* q, float* z,
                                                        const uint8_t* mask, const float* P, int64_t nnodes,
                                                        const double* rz, const double* pq, const int* active,
                                                        double* part_rz, double* part_rr) {
    float alpha[K];
#pragma unroll
    for (int k = 0; k < K; ++k) alpha[k] = (active[k] && pq[k] != 0.0) ? (float)(rz[k] / pq[k]) : 0.0f;
    double srz[K], srr[K];
#pragma unroll
    for (int k = 0; k < K; ++k) srz[k] = srr[k] = 0.0;
    for (int64_t nd = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; nd < nnodes; nd += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (mask[3 * nd + c]) continue;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const int64_t i = (3 * nd + c) * K + k;
                x[i] += alpha[k] * p[i];
                r[i] += alpha[k] * q[i];
            }
        }
        float zz[3][K];
        pinv_apply_K<K>(P, r, nd, zz);
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const int64_t i = (3 * nd + c) * K + k;
                z[i] = zz[c][k];
                srz[k] += (double)r[i] * zz[c][k];
                srr[k] += (double)r[i] * r[i];
            }
    }
    block_sumK<K>(srz, part_rz);
    __syncthreads();
    block_sumK<K>(srr, part_rr);
}

// beta_k = rz_k / rz_old_k; p = z + beta p; then rz_old = rz
template <int K>
__global__ void k_b_pupdate(float* p, const float* z, int64_t n, const double* rz, const double* rz_old, const int* active) {
    float beta[K];
#pragma unroll
    for (int k = 0; k < K; ++k) beta[k] = (active[k] && rz_old[k] != 0.0) ? (float)(rz[k] / rz_old[k]) : 0.0f;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k) p[i * K + k] = z[i * K + k] + beta[k] * p[i * K + k];
}

template <int K>
__global__ void k_b_copyK(const double* src, double* dst) {
    if (threadIdx.x < K) dst[threadIdx.x] = src[threadIdx.x];
}

// fault unfold / fold on [n][K]
template <int K>
__global__ void k_b_unfold(float* v, const int32_t* neg, const int32_t* pos, int64_t npairs) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * K * npairs; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pr = i / (3 * K), j = i % (3 * K);
        v[3 * K * (int64_t)pos[pr] + j] = v[3 * K * (int64_t)neg[pr] + j];
    }
}
template <int K>
__global__ void k_b_fold(float* v, const int32_t* neg, const int32_t* pos, int64_t npairs) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * K * npairs; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pr = i / (3 * K), j = i % (3 * K);
        v[3 * K * (int64_t)neg[pr] + j] += v[3 * K * (int64_t)pos[pr] + j];
    }
}

// FP64 [K][n] (RHS-major) residuals -> FP32 [n][K]
__global__ void k_b_pack(const double* src, int64_t n, int K, int kk, float* dst) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i * K + kk] = (float)src[i];
}
// x64[kk] += d32[:, kk] on free DOFs
__global__ void k_b_unpack_add(const float* d, int64_t n, int K, int kk, const uint8_t* mask, double* x) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (!mask[i]) x[i] += (double)d[i * K + kk];
}

static int bgrid(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 148 * 8); }

}  // namespace plb

using namespace plb;

struct pl_batch_solver_s {
    pl_solver base = nullptr;
    int K = 0;
    int64_t n = 0, nnodes = 0;
    float *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr, *x = nullptr;
    double* scal = nullptr;   // rz[K], rz_old[K], pq[K], rr[K]
    int* active = nullptr;
    double* part_a = nullptr;
    double* part_b = nullptr;
    double* r64 = nullptr;    // single-RHS FP64 outer residual
    double* jx64 = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_iters = 0;
    // The solve runs on a private stream (graph capture is not possible on the legacy default
    // stream a caller may use), fenced against the caller's stream with events.
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    int64_t solves = 0, inner_iterations = 0, outer_iterations = 0;
    double max_rel_residual = 0.0;
};

namespace {

template <int K>
int jv32_multi(pl_batch_solver B, const float* v, float* out) {
    pl_solver S = B->base;
    pl_mesh m = S->mesh;
    cudaStream_t s = m->ctx->stream;
    if (S->npairs > 0) {
        k_b_unfold<K><<<bgrid(3 * K * S->npairs), 256, 0, s>>>(const_cast<float*>(v), S->d_pair_neg, S->d_pair_pos, S->npairs);
        count_launch();
    }
    PLB_CUDA(cudaMemsetAsync(out, 0, B->n * K * sizeof(float), s));
    for (pl_integrator ig : S->ops) {
        DomainParams pp;
        int rc = bind_domain_jacobian(ig, &pp);
        if (rc) return rc;
        pp.t = S->t;
        pp.dt = S->dt;
        if (m->cell_type != PL_CELL_TET4 || ig->j3 != K_ILE_JF3VU || ig->d_cell_ids)
            return fail(PL_ERR_UNSUPPORTED, "batched solves support P1 tetrahedra with isotropic linear elasticity");
        rc = ensure_blocked_layout(m);
        if (rc) return rc;
        const BlockedLayout& L = *m->blocked;
        if (L.num_blocks == 0) return fail(PL_ERR_UNSUPPORTED, "no cell-block layout for this mesh");
        const size_t smem = (size_t)L.max_local_nodes * (3 * sizeof(double) + 2 * 3 * K * sizeof(float));
        if (smem > 200 * 1024) return fail(PL_ERR_UNSUPPORTED, "cell blocks too large for the batched kernel");
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(k_tet_blocked_jv32_multi<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int dev = 0, nsm = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        const int grid = (int)std::min<int64_t>(L.num_blocks, (int64_t)nsm * 8);
        k_tet_blocked_jv32_multi<K><<<grid, kMultiBlockCells, smem, s>>>(
            pp, L.d_block_node_begin, L.d_slot_node, (const ushort4*)L.d_local_cells, L.num_blocks, v, out);
        count_launch();
    }
    if (S->npairs > 0) {
        k_b_fold<K><<<bgrid(3 * K * S->npairs), 256, 0, s>>>(out, S->d_pair_neg, S->d_pair_pos, S->npairs);
        count_launch();
    }
    return PL_OK;
}

// One PCG iteration for all K vectors of the tile (capturable: kernels and memsets only).
template <int K>
int pcg_iteration(pl_batch_solver B) {
    pl_solver S = B->base;
    cudaStream_t s = S->mesh->ctx->stream;
    double* rz = B->scal;
    double* rz_old = B->scal + K;
    double* pq = B->scal + 2 * K;
    double* rr = B->scal + 3 * K;
    int rc = jv32_multi<K>(B, B->p, B->q);
    if (rc) return rc;
    k_b_pq<K><<<kBBlocks, kBThreads, 0, s>>>(B->p, B->q, S->d_mask, B->n, B->part_a);
    k_b_finish<K><<<1, 32, 0, s>>>(B->part_a, kBBlocks, pq);
    k_b_copyK<K><<<1, 32, 0, s>>>(rz, rz_old);
    k_b_update<K><<<kBBlocks, kBThreads, 0, s>>>(B->x, B->r, B->p, B->q, B->z, S->d_mask, S->d_pinv32, B->nnodes, rz, pq,
                                                 B->active, B->part_a, B->part_b);
    k_b_finish<K><<<1, 32, 0, s>>>(B->part_a, kBBlocks, rz);
    k_b_finish<K><<<1, 32, 0, s>>>(B->part_b, kBBlocks, rr);
    k_b_pupdate<K><<<bgrid(B->n), 256, 0, s>>>(B->p, B->z, B->n, rz, rz_old, B->active);
    count_launch(7);
    return PL_OK;
}

// FP32 PCG on the tile: r holds the right-hand sides on entry; x returns the corrections.
template <int K>
int tile_pcg(pl_batch_solver B, int nact, double rtol, int max_iter, int* iters) {
    pl_solver S = B->base;
    cudaStream_t s = S->mesh->ctx->stream;
    PLB_CUDA(cudaMemsetAsync(B->x, 0, B->n * K * sizeof(float), s));
    k_b_init<K><<<kBBlocks, kBThreads, 0, s>>>(B->r, B->z, B->p, S->d_mask, S->d_pinv32, B->nnodes, B->part_a, B->part_b);
    k_b_finish<K><<<1, 32, 0, s>>>(B->part_a, kBBlocks, B->scal);
    k_b_finish<K><<<1, 32, 0, s>>>(B->part_b, kBBlocks, B->scal + 3 * K);
    count_launch(3);
    double h[4 * 8];
    int act[8];
    PLB_CUDA(cudaMemcpyAsync(h, B->scal, 4 * K * sizeof(double), cudaMemcpyDeviceToHost, s));
    PLB_CUDA(cudaStreamSynchronize(s));
    double r0[8];
    for (int k = 0; k < K; ++k) {
        r0[k] = std::sqrt(h[3 * K + k]);
        act[k] = (k < nact && r0[k] > 0.0) ? 1 : 0;
    }
    PLB_CUDA(cudaMemcpyAsync(B->active, act, K * sizeof(int), cudaMemcpyHostToDevice, s));
    const int chunk = S->check_every;
    // capture `chunk` iterations once per tile size, replay between checks
    if (!B->graph || B->graph_iters != chunk) {
        if (B->graph) cudaGraphExecDestroy(B->graph);
        B->graph = nullptr;
        cudaGraph_t g;
        PLB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
        int rc = PL_OK;
        for (int i = 0; i < chunk && rc == PL_OK; ++i) rc = pcg_iteration<K>(B);
        cudaError_t e = cudaStreamEndCapture(s, &g);
        if (rc) return rc;
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&B->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
        B->graph_iters = chunk;
    }
    *iters = 0;
    for (int it = 0; it < max_iter; it += chunk) {
        PLB_CUDA(cudaGraphLaunch(B->graph, s));
        *iters += chunk;
        PLB_CUDA(cudaMemcpyAsync(h, B->scal, 4 * K * sizeof(double), cudaMemcpyDeviceToHost, s));
        PLB_CUDA(cudaStreamSynchronize(s));
        bool any = false;
        for (int k = 0; k < K; ++k) {
            if (!act[k]) continue;
            const double rn = std::sqrt(h[3 * K + k]);
            if (!(rn == rn)) return fail(PL_ERR_NOT_CONVERGED, "batched PCG diverged (NaN residual)");
            if (rn <= rtol * r0[k]) act[k] = 0;
            else any = true;
        }
        if (!any) return PL_OK;
        PLB_CUDA(cudaMemcpyAsync(B->active, act, K * sizeof(int), cudaMemcpyHostToDevice, s));
    }
    return PL_ERR_NOT_CONVERGED;
}

int apply_J64(pl_solver S, const double* v, double* out) {
    for (size_t i = 0; i < S->ops.size(); ++i) {
        int rc = pl_compute_lhs_jacobian_action(S->ops[i], S->t, S->dt, 0.0, nullptr, v, out, i == 0 ? PL_INSERT : PL_ADD);
        if (rc) return rc;
    }
    return PL_OK;
}

__global__ void k_unfold64(double* v, const int32_t* neg, const int32_t* pos, int64_t npairs) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * npairs; i += (int64_t)gridDim.x * blockDim.x)
        v[3 * (int64_t)pos[i / 3] + i % 3] = v[3 * (int64_t)neg[i / 3] + i % 3];
}
__global__ void k_fold64(double* v, const int32_t* neg, const int32_t* pos, int64_t npairs) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * npairs; i += (int64_t)gridDim.x * blockDim.x)
        v[3 * (int64_t)neg[i / 3] + i % 3] += v[3 * (int64_t)pos[i / 3] + i % 3];
}
// r = P^T b + P^T J x on free DOFs (Jx already folded), returns partial |r|^2 per block
__global__ void k_outer64(const double* bf, const double* Jx, const uint8_t* mask, int64_t n, double* r, double* part) {
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = mask[i] ? 0.0 : bf[i] + Jx[i];
        r[i] = v;
        s += v * v;
    }
    double acc[1] = {s};
    block_sumK<1>(acc, part);
}

template <int K>
int solve_tile(pl_batch_solver B, int nact, const double* const* bs, double* const* xs) {
    pl_solver S = B->base;
    cudaStream_t s = S->mesh->ctx->stream;
    const int64_t n = B->n;
    double bnorm[8] = {0}, rn[8] = {0};
    for (int k = 0; k < nact; ++k) PLB_CUDA(cudaMemsetAsync(xs[k], 0, n * sizeof(double), s));
    for (int outer = 0; outer < 30; ++outer) {
        // FP64 outer residual of every RHS of the tile, packed into the FP32 tile
        PLB_CUDA(cudaMemsetAsync(B->r, 0, n * K * sizeof(float), s));
        bool done = true;
        for (int k = 0; k < nact; ++k) {
            if (S->npairs > 0) {
                k_unfold64<<<bgrid(3 * S->npairs), 256, 0, s>>>(xs[k], S->d_pair_neg, S->d_pair_pos, S->npairs);
                count_launch();
            }
            int rc = apply_J64(S, xs[k], B->jx64);
            if (rc) return rc;
            PLB_CUDA(cudaMemcpyAsync(B->r64, bs[k], n * sizeof(double), cudaMemcpyDeviceToDevice, s));
            if (S->npairs > 0) {
                k_fold64<<<bgrid(3 * S->npairs), 256, 0, s>>>(B->jx64, S->d_pair_neg, S->d_pair_pos, S->npairs);
                k_fold64<<<bgrid(3 * S->npairs), 256, 0, s>>>(B->r64, S->d_pair_neg, S->d_pair_pos, S->npairs);
                count_launch(2);
            }
            k_outer64<<<kBBlocks, kBThreads, 0, s>>>(B->r64, B->jx64, S->d_mask, n, B->r64, B->part_a);
            k_b_finish<1><<<1, 32, 0, s>>>(B->part_a, kBBlocks, B->scal);
            k_b_pack<<<bgrid(n), 256, 0, s>>>(B->r64, n, K, k, B->r);
            count_launch(3);
            double h;
            PLB_CUDA(cudaMemcpyAsync(&h, B->scal, sizeof(double), cudaMemcpyDeviceToHost, s));
            PLB_CUDA(cudaStreamSynchronize(s));
            rn[k] = std::sqrt(h);
            if (outer == 0) bnorm[k] = rn[k];
            if (rn[k] > S->rtol * bnorm[k] && bnorm[k] > 0.0) done = false;
        }
        B->outer_iterations++;
        if (done) break;
        int it = 0;
        int rc = tile_pcg<K>(B, nact, S->inner_rtol, S->max_iter, &it);
        if (rc && rc != PL_ERR_NOT_CONVERGED) return rc;
        B->inner_iterations += it;
        for (int k = 0; k < nact; ++k) {
            k_b_unpack_add<<<bgrid(n), 256, 0, s>>>(B->x, n, K, k, S->d_mask, xs[k]);
            count_launch();
        }
    }
    for (int k = 0; k < nact; ++k) {
        if (S->npairs > 0) {
            k_unfold64<<<bgrid(3 * S->npairs), 256, 0, s>>>(xs[k], S->d_pair_neg, S->d_pair_pos, S->npairs);
            count_launch();
        }
        const double rel = bnorm[k] > 0.0 ? rn[k] / bnorm[k] : 0.0;
        B->max_rel_residual = std::max(B->max_rel_residual, rel);
        if (rel > S->rtol) return fail(PL_ERR_NOT_CONVERGED, "batched refinement did not reach the tolerance");
    }
    return PL_OK;
}

}  // namespace

extern "C" {

int pl_batch_solver_create(pl_solver base, int tile, pl_batch_solver* out) {
    if (!base || !out || !(tile == 1 || tile == 2 || tile == 4 || tile == 8))
        return fail(PL_ERR_INVALID_ARG, "tile must be 1, 2, 4 or 8");
    *out = nullptr;
    pl_batch_solver B = new pl_batch_solver_s();
    B->base = base;
    B->K = tile;
    B->n = base->n;
    B->nnodes = base->nnodes;
    mesh_retain(base->mesh);
    cudaError_t e = cudaSuccess;
    auto A = [&](auto** p, size_t cnt) {
        if (e == cudaSuccess) e = cudaMalloc((void**)p, cnt * sizeof(**p));
    };
    const size_t nk = (size_t)B->n * tile;
    A(&B->r, nk); A(&B->z, nk); A(&B->p, nk); A(&B->q, nk); A(&B->x, nk);
    A(&B->scal, 4 * 8);
    A(&B->active, 8);
    A(&B->part_a, (size_t)kBBlocks * 8);
    A(&B->part_b, (size_t)kBBlocks * 8);
    A(&B->r64, B->n);
    A(&B->jx64, B->n);
    // the cell-block layout is built here, outside any stream capture
    if (e == cudaSuccess) {
        const int rc = ensure_blocked_layout(base->mesh);
        if (rc) {
            pl_batch_solver_destroy(B);
            return rc;
        }
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&B->ev_in, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&B->ev_out, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        pl_batch_solver_destroy(B);
        return cuda_fail(e, "pl_batch_solver_create");
    }
    *out = B;
    return PL_OK;
}

int pl_batch_solver_solve(pl_batch_solver B, int nrhs, const double* const* b_dev, double* const* x_dev) {
    if (!B || nrhs < 0 || (nrhs > 0 && (!b_dev || !x_dev))) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    pl_solver S = B->base;
    if (!S->ready) return fail(PL_ERR_NOT_READY, "call pl_solver_setup on the base solver first");
    pl_context c = S->mesh->ctx;
    PLB_CUDA(cudaSetDevice(c->device));
    B->solves = B->inner_iterations = B->outer_iterations = 0;
    B->max_rel_residual = 0.0;
    cudaStream_t user = c->stream;
    PLB_CUDA(cudaEventRecord(B->ev_in, user));
    PLB_CUDA(cudaStreamWaitEvent(B->stream, B->ev_in, 0));
    c->stream = B->stream;
    int rc = PL_OK;
    for (int r0 = 0; r0 < nrhs && rc == PL_OK; r0 += B->K) {
        const int nact = std::min(B->K, nrhs - r0);
        switch (B->K) {
            case 1: rc = solve_tile<1>(B, nact, b_dev + r0, x_dev + r0); break;
            case 2: rc = solve_tile<2>(B, nact, b_dev + r0, x_dev + r0); break;
            case 4: rc = solve_tile<4>(B, nact, b_dev + r0, x_dev + r0); break;
            default: rc = solve_tile<8>(B, nact, b_dev + r0, x_dev + r0); break;
        }
        if (rc == PL_OK) B->solves += nact;
    }
    c->stream = user;
    cudaEventRecord(B->ev_out, B->stream);
    cudaStreamWaitEvent(user, B->ev_out, 0);
    return rc;
}

int pl_batch_solver_get_stats(pl_batch_solver B, int64_t* solves, int64_t* inner_iterations, int64_t* outer_iterations,
                              double* max_rel_residual) {
    if (!B) return fail(PL_ERR_INVALID_ARG, "null solver");
    if (solves) *solves = B->solves;
    if (inner_iterations) *inner_iterations = B->inner_iterations;
    if (outer_iterations) *outer_iterations = B->outer_iterations;
    if (max_rel_residual) *max_rel_residual = B->max_rel_residual;
    return PL_OK;
}

int pl_batch_solver_destroy(pl_batch_solver B) {
    if (!B) return PL_OK;
    pl_mesh m = B->base->mesh;
    cudaSetDevice(m->ctx->device);
    cudaStreamSynchronize(m->ctx->stream);
    if (B->graph) cudaGraphExecDestroy(B->graph);
    if (B->stream) cudaStreamSynchronize(B->stream);
    if (B->ev_in) cudaEventDestroy(B->ev_in);
    if (B->ev_out) cudaEventDestroy(B->ev_out);
    if (B->stream) cudaStreamDestroy(B->stream);
    void* ptrs[] = {B->r, B->z, B->p, B->q, B->x, B->scal, B->active, B->part_a, B->part_b, B->r64, B->jx64};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete B;
    mesh_release(m);
    return PL_OK;
}

}  // extern "C"
