// Many right-hand sides at once: the batched Green's-function solve.
//
// The reference solves its Green's-function impulses one SNES/KSP solve at a time
// (libsrc/pylith/problems/GreensFns.cc:291-337, one impulse per solve, the Jacobian lagged and
// reused: SNESSetLagJacobian(-2) at :236-241). Here a tile of K right-hand sides shares every
// launch:
//   * k_tet_blocked_jv32_multi<K>: the FP32 Jacobian action of K vectors per cell block; the
//     geometry (cofactors, 1/det in FP64), the tangent and the block metadata are read and formed
//     once and applied to all K vectors, which are interleaved per DOF ([ndof][K]) so one node's
//     K values are contiguous; element vectors are staged in shared memory a few right-hand
//     sides at a time and summed per node over the block-local incidence list in a fixed order;
//   * a batched PCG whose vector kernels update all K vectors with per-RHS step lengths and FP64
//     dot products, captured in a CUDA graph and replayed between convergence checks;
//   * FP64 iterative refinement per RHS around the FP32 tile solve (outer residual b - A x in
//     FP64 with the single-RHS FP64 action).
#include <cuda_pipeline.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "cg.cuh"
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

// Right-hand sides handled together: their values travel as one vector (float, float2, float4)
// through shared memory and into the output.
template <int K>
struct MultiChunk {
    static constexpr int value = K < 4 ? K : 4;
    // ld_vec / st_vec / red_vec move 1, 2 or 4 floats at a time.
    static_assert(value == 1 || value == 2 || value == 4, "tile sizes are 1, 2, 4, 8 or 16");
};

// Floats per staged node row in shared memory: the 3K field values, padded so that for K a
// multiple of 4 the row is an odd number of 16-byte units; the 16-byte loads of a warp from
// random rows then reach all 8 bank groups (a 96-byte row for K = 8 reaches only 4).
template <int K>
struct MultiRow {
    static constexpr int value = (K % 4 == 0 && ((3 * K / 4) % 2 == 0)) ? 3 * K + 4 : 3 * K;
};

template <int W>
PL_D void ld_vec(const float* p, float (&v)[W]) {
    if (W == 4) {
        const float4 q = *reinterpret_cast<const float4*>(p);
        v[0] = q.x; v[1] = q.y; v[2 % W] = q.z; v[3 % W] = q.w;
    } else if (W == 2) {
        const float2 q = *reinterpret_cast<const float2*>(p);
        v[0] = q.x; v[1 % W] = q.y;
    } else {
        v[0] = p[0];
    }
}

template <int W>
PL_D void st_vec(float* p, const float (&v)[W]) {
    if (W == 4) *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1 % W], v[2 % W], v[3 % W]);
    else if (W == 2) *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1 % W]);
    else p[0] = v[0];
}

// out[0..W) += v, as one vector FP32 reduction (the address is W*4-byte aligned).
template <int W>
PL_D void red_vec(float* p, const float (&v)[W]) {
    if (W == 4)
        asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(v[0]), "f"(v[1 % W]), "f"(v[2 % W]),
                     "f"(v[3 % W])
                     : "memory");
    else if (W == 2)
        asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(v[0]), "f"(v[1 % W]) : "memory");
    else
        red_add(p, v[0]);
}

// Warp sums of the KC per-lane values e[] of right-hand-side chunk ci (right-hand sides
// ci * KC .. ci * KC + KC - 1), accumulated into one FP64 value per lane: for KC = 4 lane l
// accumulates right-hand side (l & 7) * 4 + (l >> 3) (a reduce-scatter in 6 shuffles: halves
// exchanged across lane bit 4, then bit 3, then a butterfly over bits 2..0); for KC < 4 lane l
// accumulates right-hand side l. Every lane of the warp must take part.
template <int KC>
PL_D void warp_chunk_sum(const float (&e)[KC], int ci, double& acc) {
    const int lane = threadIdx.x & 31;
    if constexpr (KC == 4) {
        const bool hi = lane & 16;
        const float a0 = (hi ? e[2] : e[0]) + __shfl_xor_sync(0xffffffffu, hi ? e[0] : e[2], 16);
        const float a1 = (hi ? e[3] : e[1]) + __shfl_xor_sync(0xffffffffu, hi ? e[1] : e[3], 16);
        const bool b3 = lane & 8;
        float c = (b3 ? a1 : a0) + __shfl_xor_sync(0xffffffffu, b3 ? a0 : a1, 8);
        c += __shfl_xor_sync(0xffffffffu, c, 4);
        c += __shfl_xor_sync(0xffffffffu, c, 2);
        c += __shfl_xor_sync(0xffffffffu, c, 1);
        if ((lane & 7) == ci) acc += c;
    } else {
#pragma unroll
        for (int rr = 0; rr < KC; ++rr) {
            float c = e[rr];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
            if (lane == ci * KC + rr) acc += c;
        }
    }
}

// The right-hand side whose sum lane l holds after warp_chunk_sum (-1: none).
template <int K>
PL_D int warp_chunk_rhs(int lane) {
    constexpr int KC = MultiChunk<K>::value;
    if constexpr (KC == 4) return (lane & 7) < K / KC ? (lane & 7) * KC + (lane >> 3) : -1;
    else return lane < K ? lane : -1;
}

// v, out: [ndof][K] FP32 (ndof = 3 * nodes, node-major); out must be zeroed or hold the sum to add to.
// Per cell block: the block's node coordinates (FP64, [3][ld]) and K field vectors (FP32, one row
// of 3K values per node as in global memory, padded to MultiRow<K>) are staged in shared memory with the block's node ids
// and incidence list, all copied asynchronously one block ahead. One thread per cell
// forms the geometry and the isotropic tangent once and then, KC right-hand sides at a time (one
// vector load per node and component), the element vectors, staged as [12][cells][KC]; then one
// work item per (node, component) sums its incident corners over the block-local incidence list
// in a fixed order, KC right-hand sides per vector, and adds the node into the output (one vector
// reduction when the node is shared with other blocks).

constexpr int kBThreads = 256;
constexpr int kBBlocks = 1184;
constexpr int kMaxTile = 16;  // right-hand sides per tile: 1, 2, 4, 8 or 16

// Final sums fused into the kernel that produced the per-block partials: the last block to finish
// (a ticket counter; the partials are fenced before the ticket is taken) sums partials[blk][K] in
// block order, like k_b_finish, into out[k] (copying the old out[k] to prev[k] first when prev is
// set). FinSpec::counter null: no fused sum (the caller launches k_b_finish).
struct FinSpec {
    unsigned int* counter = nullptr;
    double* out_a = nullptr;   // sums of the first partial array
    double* prev_a = nullptr;
    double* out_b = nullptr;   // sums of the second partial array (kernels with two)
};

PL_D bool take_last_ticket(unsigned int* counter) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
        if (last) *counter = 0u;  // every other block has taken its ticket
    }
    __syncthreads();
    if (last) __threadfence();
    return last;
}

// sh: kBThreads / 32 * K doubles of shared memory.
template <int K>
PL_D void sum_partials_last_block_in(const double* partials, double* out, double* prev, double (*sh)[K]) {
    const int k = threadIdx.x % K;
    double s = 0.0;
    for (int b = threadIdx.x / K; b < (int)gridDim.x; b += kBThreads / K) s += __ldcg(&partials[b * K + k]);
#pragma unroll
    for (int o = K; o < 32; o <<= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l < K) sh[w][l] = s;
    __syncthreads();
    if (threadIdx.x < K) {
        double t = 0.0;
#pragma unroll
        for (int i = 0; i < kBThreads / 32; ++i) t += sh[i][threadIdx.x];
        if (prev) prev[threadIdx.x] = out[threadIdx.x];
        out[threadIdx.x] = t;
    }
    __syncthreads();
}

template <int K>
PL_D void sum_partials_last_block(const double* partials, double* out, double* prev) {
    __shared__ double sh[kBThreads / 32][K];
    sum_partials_last_block_in<K>(partials, out, prev, sh);
}

// Block metadata in shared memory (two buffers: the gather reads one while the next block's is
// copied into the other): node ids [ld], incidence offsets [ld + 1], incidence list
// [4 * cells] (cell * 4 + corner).
struct MultiMeta {
    uint32_t* id;
    uint32_t* off;
    uint16_t* inc;
};

PL_HD size_t multi_r16(size_t x) { return (x + 15) & ~size_t(15); }

PL_HD size_t multi_meta_bytes(int ld) {
    return multi_r16(4 * (size_t)ld) + multi_r16(4 * ((size_t)ld + 1)) + (size_t)2 * 4 * kMultiBlockCells;
}

PL_D MultiMeta multi_meta(char* base, int ld) {
    MultiMeta m;
    m.id = reinterpret_cast<uint32_t*>(base);
    base += multi_r16(4 * (size_t)ld);
    m.off = reinterpret_cast<uint32_t*>(base);
    base += multi_r16(4 * ((size_t)ld + 1));
    m.inc = reinterpret_cast<uint16_t*>(base);
    return m;
}

// Asynchronous copies of block b's node rows (K field values per component), coordinates and
// metadata into shared memory.
template <int K>
PL_D void prefetch_multi(const DomainParams& p, const int32_t* __restrict__ slot_begin,
                         const uint32_t* __restrict__ slot_node, const uint32_t* __restrict__ inc_off,
                         const uint16_t* __restrict__ inc, const int32_t* __restrict__ pbeg,
                         const double* __restrict__ pcoords, int64_t b, int ld, const float* __restrict__ v,
                         float* sV, double* sX, const MultiMeta& mm) {
    constexpr int CB = K % 4 == 0 ? 16 : (K % 2 == 0 ? 8 : 4);  // bytes per copy; rows are 12 K bytes
    const int s0 = slot_begin[b];
    const int ns = slot_begin[b + 1] - s0;
    // coordinates: the block's [3][slots rounded up to 4] run of the padded layout, 16 bytes a copy
    const int p0 = pbeg[b], np = pbeg[b + 1] - p0, half = np >> 1;
    for (int t = threadIdx.x; t < 3 * half; t += blockDim.x) {
        const int d = t / half, j = t - d * half;
        __pipeline_memcpy_async(&sX[d * ld + 2 * j], &pcoords[3 * (int64_t)p0 + (int64_t)d * np + 2 * j], 16);
    }
    for (int i = threadIdx.x; i < ns; i += blockDim.x) {
        const uint32_t id = slot_node[s0 + i];
        const int64_t nd = id & ~kSharedBitM;
        const float* vr = v + 3 * K * nd;
        float* sr = sV + MultiRow<K>::value * i;
#pragma unroll
        for (int j = 0; j < 3 * K; j += CB / 4) __pipeline_memcpy_async(sr + j, vr + j, CB);
        mm.id[i] = id;
    }
    for (int i = threadIdx.x; i <= ns; i += blockDim.x)
        __pipeline_memcpy_async(&mm.off[i], &inc_off[s0 + b + i], sizeof(uint32_t));
    // 4 * kMultiBlockCells uint16 = kMultiBlockCells / 2 chunks of 16 bytes
    for (int i = threadIdx.x; i < kMultiBlockCells / 2; i += blockDim.x)
        __pipeline_memcpy_async(&mm.inc[8 * i], &inc[b * 4 * kMultiBlockCells + 8 * i], 16);
}

// store_owned: nodes owned by one block are stored (the output was zeroed and this is the first
// integrator); otherwise they are added.
// pq_part (optional, with fin.counter and pq_rz): the energies v.(A v) = -v.(J v) of the K
// vectors, summed from the cells: a cell's share of v.(J v) is its element vector dotted with its
// corner values, vol f1(grad v) : grad v = -vol (lambda tr(e)^2 + 2 mu e:e) with e = sym grad v, so
// the sum over cells equals the sum over DOFs of v_i (J v)_i (the fault's fold adds each
// positive-side row to its negative-side partner, whose value v carries, and constrained DOFs hold
// v = 0). FP32 squares of small gradients would underflow (a residual of 1e-11 of a unit
// right-hand side gives gradients near 1e-28), so each vector's gradient is scaled by
// s_k = 1 / sqrt(pq_rz[k]) (its current r.z, of the order of its energy) before the products and
// the FP64 sums are divided by s_k^2. Per-CTA FP64 partials [grid][K]; the last CTA forms the sums
// in CTA order into fin.out_a.
template <int K>
__global__ void __launch_bounds__(kMultiBlockCells, 3) k_tet_blocked_jv32_multi(
    DomainParams p, const int32_t* __restrict__ cell_begin, const int32_t* __restrict__ slot_begin,
    const uint32_t* __restrict__ slot_node, const ushort4* __restrict__ lconn, const uint32_t* __restrict__ inc_off,
    const uint16_t* __restrict__ inc, const int32_t* __restrict__ pbeg, const double* __restrict__ pcoords,
    int64_t nblocks, int ld, const float* __restrict__ v, float* out, bool store_owned, double* pq_part,
    const double* __restrict__ pq_rz, FinSpec fin) {
    static_assert(kMultiBlockCells == kBThreads, "the fused sums assume kBThreads threads per CTA");
    __shared__ float s_sig[K];  // energy scales (pq_part)
    if (pq_part && threadIdx.x < K) {
        const double rz = pq_rz[threadIdx.x];
        s_sig[threadIdx.x] = (rz > 0.0 && rz < 1e300) ? (float)fmin(fmax(1.0 / sqrt(rz), 1e-30), 1e30) : 1.0f;
    }
    constexpr int KC = MultiChunk<K>::value;
    using L = AuxLayout<RHEO_ILE, false>;
    extern __shared__ __align__(16) char smem_raw[];
    const AuxOffsets<RHEO_ILE, false> aoff;
    float* sE = reinterpret_cast<float*>(smem_raw);                                              // [12][cells][KC]
    float* sV = sE + 12 * kMultiBlockCells * KC;  // [ld][MultiRow<K>]
    // [3][ld], at a 16-byte boundary after sV
    double* sX = reinterpret_cast<double*>(reinterpret_cast<char*>(sV) +
                                           multi_r16((size_t)ld * MultiRow<K>::value * sizeof(float)));
    // two metadata buffers after sX
    char* metabase = reinterpret_cast<char*>(sX) + multi_r16((size_t)ld * 3 * sizeof(double));
    const size_t mb = multi_meta_bytes(ld);
    int cur = 0;
    const int tc = threadIdx.x;
    double pq_acc = 0.0;  // this lane's energy sum (warp_chunk_sum)
    if (blockIdx.x < nblocks)
        prefetch_multi<K>(p, slot_begin, slot_node, inc_off, inc, pbeg, pcoords, blockIdx.x, ld, v, sV, sX,
                          multi_meta(metabase, ld));
    __pipeline_commit();
    for (int64_t b = blockIdx.x; b < nblocks; b += gridDim.x) {
        const int ns = slot_begin[b + 1] - slot_begin[b];
        const int64_t c = cell_begin[b] + tc;
        const bool live = c < cell_begin[b + 1];
        int ln[4] = {0, 0, 0, 0};
        float inv[3][3], cf[3][3], lam = 0.f, mu = 0.f, vol = 0.f;
        // per-cell inputs from global memory first: their latency overlaps the staging copies
        if (live) {
            const ushort4 lc = lconn[c];
            ln[0] = lc.x;
            ln[1] = lc.y;
            ln[2] = lc.z;
            ln[3] = lc.w;
            // The registered tangent (Jf3vu_infinitesimalStrain) is isotropic: Jf3 = -C with
            // C = lambda d_ij d_kl + mu (d_ik d_jl + d_il d_jk); its (f,g,df,dg) = (0,1,0,1) and
            // (0,1,1,0) entries are -lambda and -mu.
            double a[L::size];
            L::load_cell(p, c, a);
            double x[3] = {0, 0, 0};
            double Jf3d[81];
#pragma unroll
            for (int i = 0; i < 81; ++i) Jf3d[i] = 0.0;
            call_jf3<RHEO_ILE>(L::numA, aoff.v, a, p, x, Jf3d);
            lam = (float)(-Jf3d[((0 * 3 + 1) * 3 + 0) * 3 + 1]);
            mu = (float)(-Jf3d[((0 * 3 + 1) * 3 + 1) * 3 + 0]);
        }
        __pipeline_wait_prior(0);
        __syncthreads();
        const MultiMeta mm = multi_meta(metabase + cur * mb, ld);
        if (live) {
            double X[4][3];
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int d = 0; d < 3; ++d) X[k][d] = sX[d * ld + ln[k]];
            double cof[3][3];
            const double det = tet_cof_m(X, cof);
            if (!(det > 0.0)) flag_error(p.err, CHECK_NONPOSITIVE_DETJ);
            const double rdet = 1.0 / det;
            vol = (float)(det * (1.0 / 6.0));
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    inv[i][j] = (float)(cof[i][j] * rdet);
                    cf[i][j] = (float)(cof[i][j] * (1.0 / 6.0));
                }
        }
#pragma unroll 1
        for (int r0 = 0; r0 < K; r0 += KC) {
            float en[KC];
#pragma unroll
            for (int rr = 0; rr < KC; ++rr) en[rr] = 0.f;
            if (live) {
                // gradient of the KC fields: G[cc][k] = v_{k+1} - v_0 per component, then s_x = G inv
                float s_x[KC][3][3];
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) {
                    float u0[KC], u1[KC], u2[KC], u3[KC];
                    ld_vec<KC>(sV + MultiRow<K>::value * ln[0] + cc * K + r0, u0);
                    ld_vec<KC>(sV + MultiRow<K>::value * ln[1] + cc * K + r0, u1);
                    ld_vec<KC>(sV + MultiRow<K>::value * ln[2] + cc * K + r0, u2);
                    ld_vec<KC>(sV + MultiRow<K>::value * ln[3] + cc * K + r0, u3);
#pragma unroll
                    for (int rr = 0; rr < KC; ++rr) {
                        const float g0 = u1[rr] - u0[rr], g1 = u2[rr] - u0[rr], g2 = u3[rr] - u0[rr];
#pragma unroll
                        for (int d = 0; d < 3; ++d) s_x[rr][cc][d] = g0 * inv[0][d] + g1 * inv[1][d] + g2 * inv[2][d];
                    }
                }
                // flux f1 = -(lambda tr(e) I + 2 mu e), in place of s_x (and, for pq_part, the
                // energy vol (lambda tr(e)^2 + 2 mu e:e) first)
#pragma unroll
                for (int rr = 0; rr < KC; ++rr) {
                    const float tr = s_x[rr][0][0] + s_x[rr][1][1] + s_x[rr][2][2];
                    const float ltr = lam * tr;
                    const float sxy = s_x[rr][0][1] + s_x[rr][1][0];
                    const float syz = s_x[rr][1][2] + s_x[rr][2][1];
                    const float sxz = s_x[rr][0][2] + s_x[rr][2][0];
                    const float xy = -mu * sxy;
                    const float yz = -mu * syz;
                    const float xz = -mu * sxz;
                    if (pq_part) {
                        // scaled gradient; every product pairs a modulus-weighted factor with a bare one
                        const float g = s_sig[r0 + rr];
                        const float t = g * tr, a = g * s_x[rr][0][0], b = g * s_x[rr][1][1], c = g * s_x[rr][2][2];
                        const float u = g * sxy, w = g * syz, z = g * sxz;
                        en[rr] = vol * ((lam * t) * t + (2.0f * mu * a) * a + (2.0f * mu * b) * b +
                                        (2.0f * mu * c) * c + (mu * u) * u + (mu * w) * w + (mu * z) * z);
                    }
                    s_x[rr][0][0] = -(2.0f * mu * s_x[rr][0][0] + ltr);
                    s_x[rr][1][1] = -(2.0f * mu * s_x[rr][1][1] + ltr);
                    s_x[rr][2][2] = -(2.0f * mu * s_x[rr][2][2] + ltr);
                    s_x[rr][0][1] = s_x[rr][1][0] = xy;
                    s_x[rr][1][2] = s_x[rr][2][1] = yz;
                    s_x[rr][0][2] = s_x[rr][2][0] = xz;
                }
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) {
                    float e0[KC];
#pragma unroll
                    for (int rr = 0; rr < KC; ++rr) e0[rr] = 0.f;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        float val[KC];
#pragma unroll
                        for (int rr = 0; rr < KC; ++rr) {
                            val[rr] = s_x[rr][cc][0] * cf[k][0] + s_x[rr][cc][1] * cf[k][1] + s_x[rr][cc][2] * cf[k][2];
                            e0[rr] -= val[rr];
                        }
                        st_vec<KC>(sE + (((k + 1) * 3 + cc) * kMultiBlockCells + tc) * KC, val);
                    }
                    st_vec<KC>(sE + ((cc)*kMultiBlockCells + tc) * KC, e0);
                }
            }
            if (pq_part) warp_chunk_sum<KC>(en, r0 / KC, pq_acc);
            __syncthreads();
            // the node rows are no longer read in this block: copy the next block's while gathering
            if (r0 + KC >= K && b + gridDim.x < nblocks)
                prefetch_multi<K>(p, slot_begin, slot_node, inc_off, inc, pbeg, pcoords, b + gridDim.x, ld, v, sV, sX,
                                  multi_meta(metabase + (cur ^ 1) * mb, ld));
            __pipeline_commit();
            // one work item per (node, component): a warp takes one component of 32 consecutive
            // nodes, the groups whose incidence order the layout spread over the banks
            const int nitems = (ns + 31) / 32 * 96;
            for (int w = tc; w < nitems; w += blockDim.x) {
                const int chunk = w >> 5, g = chunk / 3, cc = chunk - 3 * g, i = g * 32 + (w & 31);
                if (i >= ns) continue;
                const int j0 = mm.off[i], j1 = mm.off[i + 1];
                float acc[KC];
#pragma unroll
                for (int rr = 0; rr < KC; ++rr) acc[rr] = 0.f;
#pragma unroll 4
                for (int j = j0; j < j1; ++j) {
                    const int e = mm.inc[j];
                    const int cell = e >> 2, corner = e & 3;
                    float t[KC];
                    ld_vec<KC>(sE + ((corner * 3 + cc) * kMultiBlockCells + cell) * KC, t);
#pragma unroll
                    for (int rr = 0; rr < KC; ++rr) acc[rr] += t[rr];
                }
                const uint32_t id = mm.id[i];
                float* o = out + 3 * K * (int64_t)(id & ~kSharedBitM) + cc * K + r0;
                if (id & kSharedBitM) {
                    red_vec<KC>(o, acc);
                } else if (store_owned) {
                    st_vec<KC>(o, acc);
                } else {
                    float t[KC];
                    ld_vec<KC>(o, t);
#pragma unroll
                    for (int rr = 0; rr < KC; ++rr) t[rr] += acc[rr];
                    st_vec<KC>(o, t);
                }
            }
            __syncthreads();
        }
        cur ^= 1;
    }
    __pipeline_wait_prior(0);
    if (pq_part) {
        // the element-vector staging area is free after the loop's last barrier
        double* sh = reinterpret_cast<double*>(smem_raw);  // [warps][K]
        const int lane = tc & 31, wq = tc >> 5;
        const int rhs = warp_chunk_rhs<K>(lane);
        if (rhs >= 0) {
            const double g = s_sig[rhs];
            sh[wq * K + rhs] = pq_acc / (g * g);
        }
        __syncthreads();
        if (tc < K) {
            double t = 0.0;
            for (int i = 0; i < kMultiBlockCells / 32; ++i) t += sh[i * K + tc];
            pq_part[blockIdx.x * K + tc] = t;
        }
        if (fin.counter && take_last_ticket(fin.counter))
            sum_partials_last_block_in<K>(pq_part, fin.out_a, fin.prev_a,
                                          reinterpret_cast<double (*)[K]>(sh + kMultiBlockCells / 32 * K));
    }
}

template <int K>
size_t multi_smem(int ld) {
    return (size_t)12 * MultiChunk<K>::value * kMultiBlockCells * sizeof(float) +
           multi_r16((size_t)ld * MultiRow<K>::value * sizeof(float)) + multi_r16((size_t)ld * 3 * sizeof(double)) +
           2 * multi_meta_bytes(ld);
}

// ---- batched vector kernels, layout [n][K] -------------------------------------------------
// Element e of an [n][K] array is DOF e / K of right-hand side e % K; every kernel below maps
// consecutive threads to consecutive elements (thread index % K == right-hand side).

// Per-block sums of one value per thread, by right-hand side (thread index % K), in a fixed
// order -> partials[blk][K].
template <int K>
PL_D void block_sum_by_rhs(double a, double* partials) {
    __shared__ double sh[kBThreads / 32][K];
#pragma unroll
    for (int o = K; o < 32; o <<= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l < K) sh[w][l] = a;
    __syncthreads();
    if (threadIdx.x < K) {
        double s = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += sh[i][threadIdx.x];
        partials[blockIdx.x * K + threadIdx.x] = s;
    }
}

// Per-block sums of K values per thread (used by the single-RHS outer residual).
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

// Fixed-order final sums, one block per right-hand side (launch with K blocks of kBThreads):
// out[k] = sum_blk partials[blk][k]; with `prev`, the value out held before is copied there first.
template <int K>
__global__ void __launch_bounds__(kBThreads) k_b_finish(const double* __restrict__ partials, int nblk, double* out,
                                                       double* prev) {
    __shared__ double sh[kBThreads / 32];
    const int k = blockIdx.x;
    double s = 0.0;
#pragma unroll 8
    for (int i = threadIdx.x; i < nblk; i += kBThreads) s += partials[i * K + k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
#pragma unroll
        for (int i = 0; i < kBThreads / 32; ++i) t += sh[i];
        if (prev) prev[k] = out[k];
        out[k] = t;
    }
}

template <int K>
PL_D void pinv_apply(const float* __restrict__ P, const float* r, int64_t node, int k, float z[3]) {
    const float* B = P + 9 * node;
    const float r0 = r[(3 * node + 0) * K + k], r1 = r[(3 * node + 1) * K + k], r2 = r[(3 * node + 2) * K + k];
    z[0] = B[0] * r0 + B[1] * r1 + B[2] * r2;
    z[1] = B[3] * r0 + B[4] * r1 + B[5] * r2;
    z[2] = B[6] * r0 + B[7] * r1 + B[8] * r2;
}

// r = b (masked); z = P r; p = z; partial (r.z)[K], (r.r)[K]. One thread per (node, rhs).
template <int K>
__global__ void __launch_bounds__(kBThreads) k_b_init(float* r, float* z, float* p, const uint8_t* mask, const float* P,
                                                      int64_t nnodes, double* part_rz, double* part_rr) {
    double rz = 0.0, rr = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nnodes * K; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t nd = t / K;
        const int k = (int)(t % K);
#pragma unroll
        for (int c = 0; c < 3; ++c)
            if (mask[3 * nd + c]) r[(3 * nd + c) * K + k] = 0.0f;
        float zz[3];
        pinv_apply<K>(P, r, nd, k, zz);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int64_t i = (3 * nd + c) * K + k;
            const float ri = r[i];
            z[i] = zz[c];
            p[i] = zz[c];
            rz += (double)ri * zz[c];
            rr += (double)ri * ri;
        }
    }
    block_sum_by_rhs<K>(rz, part_rz);
    __syncthreads();
    block_sum_by_rhs<K>(rr, part_rr);
}

// partial p.(A p) with q = J p: -p.q over free DOFs
template <int K>
__global__ void __launch_bounds__(kBThreads) k_b_pq(const float* p, const float* q, const uint8_t* mask, int64_t n,
                                                    double* part, FinSpec fin) {
    double s = 0.0;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n * K; e += (int64_t)gridDim.x * blockDim.x)
        if (!mask[e / K]) s -= (double)p[e] * q[e];
    block_sum_by_rhs<K>(s, part);
    if (fin.counter && take_last_ticket(fin.counter)) sum_partials_last_block<K>(part, fin.out_a, fin.prev_a);
}

// alpha_k = active_k ? rz_k / pq_k : 0; r += alpha q; z = P r (stored when StoreZ); partial rz, rr
// (x is updated by k_b_pupdate). One thread per (node, rhs).
template <int K, bool StoreZ = true>
__global__ void __launch_bounds__(kBThreads) k_b_update(float* r, const float* q, float* z,
                                                        const uint8_t* mask, const float* P, int64_t nnodes,
                                                        const double* rz, const double* pq, const int* active,
                                                        double* part_rz, double* part_rr, FinSpec fin) {
    const int k = threadIdx.x % K;  // blockDim and the grid stride are multiples of K
    const float alpha = active[k] ? safe_step_f32(rz[k], pq[k]) : 0.0f;
    double srz = 0.0, srr = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nnodes * K; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t nd = t / K;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (mask[3 * nd + c]) continue;
            const int64_t i = (3 * nd + c) * K + k;
            r[i] += alpha * q[i];
        }
        float zz[3];
        pinv_apply<K>(P, r, nd, k, zz);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int64_t i = (3 * nd + c) * K + k;
            const float ri = r[i];
            if (StoreZ) z[i] = zz[c];
            srz += (double)ri * zz[c];
            srr += (double)ri * ri;
        }
    }
    block_sum_by_rhs<K>(srz, part_rz);
    __syncthreads();
    block_sum_by_rhs<K>(srr, part_rr);
    if (fin.counter && take_last_ticket(fin.counter)) {
        sum_partials_last_block<K>(part_rz, fin.out_a, fin.prev_a);
        sum_partials_last_block<K>(part_rr, fin.out_b, nullptr);
    }
}

// x += alpha p (free DOFs; alpha_k = rz_old_k / pq_k, the step of this iteration, whose r.z is
// rz_old now) and then p = z + beta p, beta_k = rz_k / rz_old_k: the solution update rides on the
// pass that reads p anyway.
template <int K>
__global__ void k_b_pupdate(float* x, float* p, const float* z, const uint8_t* mask, int64_t n, const double* rz,
                            const double* rz_old, const double* pq, const int* active, const double* zq = nullptr) {
    const int k = threadIdx.x % K;
    const float alpha = active[k] ? safe_step_f32(rz_old[k], pq[k]) : 0.0f;
    // zq (a preconditioner that is not exactly fixed, the FP32 V-cycle): the flexible step
    // beta = max(0, z.(r - r_old) / rz_old) = max(0, z.q / p.(A p)) with r - r_old = alpha q
    float beta;
    if (zq) {
        const double bz = pq[k] > 0.0 ? zq[k] / pq[k] : 0.0;
        beta = (active[k] && isfinite(bz) && bz > 0.0) ? (float)bz : 0.0f;
    } else {
        beta = (active[k] && rz_old[k] != 0.0) ? (float)(rz[k] / rz_old[k]) : 0.0f;
    }
    if (!isfinite(beta)) beta = 0.0f;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n * K; e += (int64_t)gridDim.x * blockDim.x) {
        const float pe = p[e];
        if (!mask[e / K]) x[e] += alpha * pe;
        p[e] = z[e] + beta * pe;
    }
}

// k_b_pupdate for the point-block Jacobi preconditioner, forming z = P r from r (one thread per
// (node, rhs)) instead of reading a stored z.
template <int K>
__global__ void __launch_bounds__(kBThreads) k_b_pupdate_jacobi(float* x, float* p, const float* r,
                                                                const uint8_t* mask, const float* P, int64_t nnodes,
                                                                const double* rz, const double* rz_old,
                                                                const double* pq, const int* active) {
    const int k = threadIdx.x % K;  // blockDim and the grid stride are multiples of K
    const float alpha = active[k] ? safe_step_f32(rz_old[k], pq[k]) : 0.0f;
    const float beta = (active[k] && rz_old[k] != 0.0) ? (float)(rz[k] / rz_old[k]) : 0.0f;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nnodes * K; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t nd = t / K;
        float zz[3];
        pinv_apply<K>(P, r, nd, k, zz);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int64_t i = (3 * nd + c) * K + k;
            const float pe = p[i];
            if (!mask[3 * nd + c]) x[i] += alpha * pe;
            p[i] = zz[c] + beta * pe;
        }
    }
}

// ---- Chebyshev-Jacobi preconditioner: z = q(P A) P r, with A = -J and the point-block
// Jacobi inverse P; Chebyshev iteration of a given degree for A z = r from z = 0 (Saad,
// "Iterative Methods for Sparse Linear Systems", 2nd ed., Algorithm 12.1), so the preconditioner is a
// fixed polynomial, symmetric and positive definite while the eigenvalues of P A lie below the
// upper bound. ----

PL_D void pinv_local(const float* __restrict__ P, int64_t node, const float in[3], float out[3]) {
    const float* B = P + 9 * node;
    out[0] = B[0] * in[0] + B[1] * in[1] + B[2] * in[2];
    out[1] = B[3] * in[0] + B[4] * in[1] + B[5] * in[2];
    out[2] = B[6] * in[0] + B[7] * in[1] + B[8] * in[2];
}

// r += alpha q on free DOFs; partial r.r (the preconditioner runs after; x is updated by
// k_b_pupdate).
template <int K>
__global__ void __launch_bounds__(kBThreads) k_b_update_xr(float* r, const float* q,
                                                           const uint8_t* mask, int64_t n, const double* rz,
                                                           const double* pq, const int* active, double* part_rr,
                                                           FinSpec fin) {
    const int k = threadIdx.x % K;
    const float alpha = active[k] ? safe_step_f32(rz[k], pq[k]) : 0.0f;
    double srr = 0.0;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n * K; e += (int64_t)gridDim.x * blockDim.x) {
        if (mask[e / K]) continue;
        const float ri = r[e] + alpha * q[e];
        r[e] = ri;
        srr += (double)ri * ri;
    }
    block_sum_by_rhs<K>(srr, part_rr);
    if (fin.counter && take_last_ticket(fin.counter)) sum_partials_last_block<K>(part_rr, fin.out_a, nullptr);
}

// First Chebyshev step: d = s P r, z = d (constrained DOFs zero). One thread per (node, rhs).
template <int K>
__global__ void __launch_bounds__(kBThreads) k_cheb_first(const float* r, float* d, float* z, const uint8_t* mask,
                                                          const float* P, int64_t nnodes, float s) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nnodes * K; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t nd = t / K;
        const int k = (int)(t % K);
        float zz[3];
        pinv_apply<K>(P, r, nd, k, zz);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int64_t i = (3 * nd + c) * K + k;
            const float v = mask[3 * nd + c] ? 0.0f : s * zz[c];
            d[i] = v;
            z[i] = v;
        }
    }
}

// Later steps: res = src + q (= src - A d; src is r for the first of them, res after), then
// d = c1 d + c2 P res, z += d, all on free DOFs; the last step also sums r.z per right-hand side.
template <int K, bool LAST>
__global__ void __launch_bounds__(kBThreads) k_cheb_step(const float* src, const float* q, float* res, float* d,
                                                         float* z, const float* r, const uint8_t* mask, const float* P,
                                                         int64_t nnodes, float c1, float c2, double* part_rz,
                                                         FinSpec fin) {
    double srz = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nnodes * K; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t nd = t / K;
        const int k = (int)(t % K);
        float rs[3], pr[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int64_t i = (3 * nd + c) * K + k;
            rs[c] = mask[3 * nd + c] ? 0.0f : src[i] + q[i];
            res[i] = rs[c];
        }
        pinv_local(P, nd, rs, pr);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int64_t i = (3 * nd + c) * K + k;
            const bool m = mask[3 * nd + c];
            const float dv = m ? 0.0f : c1 * d[i] + c2 * pr[c];
            const float zv = m ? 0.0f : z[i] + dv;
            d[i] = dv;
            z[i] = zv;
            if (LAST) srz += (double)r[i] * zv;
        }
    }
    if (LAST) {
        block_sum_by_rhs<K>(srz, part_rz);
        if (fin.counter && take_last_ticket(fin.counter)) sum_partials_last_block<K>(part_rz, fin.out_a, fin.prev_a);
    }
}

// Power iteration for the largest eigenvalue of P A: w = -P (J v) on free DOFs, partial |w|^2
// and |v|^2 per right-hand side.
template <int K>
__global__ void __launch_bounds__(kBThreads) k_power_step(const float* v, const float* q, float* w, const uint8_t* mask,
                                                          const float* P, int64_t nnodes, double* part_ww,
                                                          double* part_vv) {
    double sww = 0.0, svv = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nnodes * K; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t nd = t / K;
        const int k = (int)(t % K);
        float zz[3];
        pinv_apply<K>(P, q, nd, k, zz);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int64_t i = (3 * nd + c) * K + k;
            const bool m = mask[3 * nd + c];
            const float wi = m ? 0.0f : -zz[c];
            w[i] = wi;
            sww += (double)wi * wi;
            if (!m) svv += (double)v[i] * v[i];
        }
    }
    block_sum_by_rhs<K>(sww, part_ww);
    __syncthreads();
    block_sum_by_rhs<K>(svv, part_vv);
}

// v = s_k w (per right-hand side), or a deterministic pseudo-random start when w is null.
struct ColScale {
    float s[kMaxTile];
};
template <int K>
__global__ void k_power_scale(float* v, const float* w, const uint8_t* mask, int64_t n, ColScale cs) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n * K; e += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(e % K);
        float val;
        if (w) {
            val = cs.s[k] * w[e];
        } else {
            uint32_t h = (uint32_t)(e * 2654435761ull) ^ 0x9e3779b9u;
            h ^= h >> 15;
            h *= 0x85ebca6bu;
            h ^= h >> 13;
            val = (float)(h & 0xffffff) / 16777216.0f - 0.5f;
        }
        v[e] = mask[e / K] ? 0.0f : val;
    }
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

// d[:, kk] = 0
__global__ void k_b_col_zero(float* d, int64_t n, int K, int kk) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        d[i * K + kk] = 0.0f;
}

// dst[:, kk] = src[:, kk]
__global__ void k_b_col_copy(float* dst, const float* src, int64_t n, int K, int kk) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i * K + kk] = src[i * K + kk];
}

// z[:, kk] = P r[:, kk] (constrained DOFs zero); partial r.z of the column
__global__ void __launch_bounds__(kBThreads) k_b_col_prec(const float* r, float* z, const uint8_t* mask,
                                                          const float* P, int64_t nnodes, int K, int kk,
                                                          double* part) {
    double s = 0.0;
    for (int64_t nd = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; nd < nnodes; nd += (int64_t)gridDim.x * blockDim.x) {
        float in[3], out[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) in[c] = r[(3 * nd + c) * K + kk];
        pinv_local(P, nd, in, out);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float v = mask[3 * nd + c] ? 0.0f : out[c];
            z[(3 * nd + c) * K + kk] = v;
            s += (double)in[c] * v;
        }
    }
    double acc[1] = {s};
    block_sumK<1>(acc, part);
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
    unsigned int* ticket = nullptr;  // last-block counter of the fused reductions (zero between kernels)
    double* r64 = nullptr;    // single-RHS FP64 outer residual
    double* jx64 = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_iters = 0;
    unsigned long long graph_epoch = 0;
    int graph_cheb = -1;      // cheb_version the graph was captured with
    // Chebyshev-Jacobi preconditioner (degree >= 2; 0 or 1: point-block Jacobi)
    int cheb_degree = 0;
    double cheb_lower_ratio = 0.05;
    int cheb_eig_iters = 20;
    double cheb_lmax = 0.0;   // estimated largest eigenvalue of P A (before the safety factor)
    int cheb_version = 0;     // bumped when the coefficients change
    unsigned long long cheb_epoch = 0;  // state epoch of the estimate
    float cheb_s0 = 0.0f;
    float cheb_c1[8] = {}, cheb_c2[8] = {};
    float *res = nullptr, *d = nullptr;
    // Reliable updates (default): one FP32 CG per right-hand side, whose iterated residual is
    // replaced by the FP64 true residual (and the FP32 correction folded into the FP64 solution)
    // each time it has dropped by reliable_delta; off: FP64 refinement that restarts the FP32 PCG
    // from each new FP64 residual until it has dropped by the solver's inner_rtol.
    bool reliable = true;
    double reliable_delta = 0.01;
    int64_t reliable_updates = 0;
    // The solve runs on a private stream (graph capture is not possible on the legacy default
    // stream a caller may use), fenced against the caller's stream with events.
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    int64_t solves = 0, inner_iterations = 0, outer_iterations = 0;
    double max_rel_residual = 0.0;
    // Multigrid preconditioner (pl_batch_solver_set_multigrid): one V-cycle of the hierarchy on
    // the tile's K vectors per iteration, [n_l][K] work vectors per level.
    struct BmgLevel {
        float *r = nullptr, *z = nullptr, *t = nullptr, *d = nullptr, *q = nullptr, *w = nullptr;
    };
    pl_multigrid mg = nullptr;
    std::vector<BmgLevel> bmg;
    plb::MgView mgv;
};

namespace plb {
constexpr int kMaxChebDegree = 8;
}

namespace {

// Whether a PCG iteration sums p.(A p) inside the operator launch (single-integrator operators;
// PYLITH_B200_BATCH_FUSED_PQ=0 selects the separate reduction kernel instead).
// Read when an iteration is recorded (graph capture), not per replay.
bool fuses_energies(pl_batch_solver B) {
    const char* e = std::getenv("PYLITH_B200_BATCH_FUSED_PQ");
    return !(e && e[0] == '0') && B->base->ops.size() == 1;
}

// out = J v for the tile's K vectors; with pq (single-integrator operators only, see
// fuses_energies), the energies v.(A v) are summed by the same launch into pq[K] (scaled by the
// tile's current r.z, B->scal[0..K)).
template <int K>
int jv32_multi_on(pl_solver S, int64_t n, const float* v, float* out, double* pq, unsigned int* ticket, double* part,
                  const double* scal) {
    pl_mesh m = S->mesh;
    cudaStream_t s = m->ctx->stream;
    if (pq && S->ops.size() != 1) return fail(PL_ERR_UNSUPPORTED, "fused energies need a single integrator");
    // the solver's reduced fault space directly (slot ids of the reduced space: no unfold or fold)
    const bool reduced = S->npairs > 0 && S->reduced && m->blocked && m->blocked->d_slot_node_red;
    if (S->npairs > 0 && !reduced) {
        k_b_unfold<K><<<bgrid(3 * K * S->npairs), 256, 0, s>>>(const_cast<float*>(v), S->d_pair_neg, S->d_pair_pos, S->npairs);
        count_launch();
    }
    PLB_CUDA(cudaMemsetAsync(out, 0, n * K * sizeof(float), s));
    bool first = true;
    for (pl_integrator ig : S->ops) {
        DomainParams pp;
        int rc = bind_domain_jacobian(ig, &pp);
        if (rc) return rc;
        pp.t = S->t;
        pp.dt = S->dt;
        if (m->cell_type != PL_CELL_TET4 || ig->j3 != K_ILE_JF3VU || ig->subset)
            return fail(PL_ERR_UNSUPPORTED, "batched solves support P1 tetrahedra with isotropic linear elasticity");
        rc = ensure_blocked_layout(m);
        if (rc) return rc;
        const BlockedLayout& L = *m->blocked;
        if (L.num_blocks == 0) return fail(PL_ERR_UNSUPPORTED, "no cell-block layout for this mesh");
        if (L.max_local_nodes > 2 * kMultiBlockCells)
            return fail(PL_ERR_UNSUPPORTED, "cell blocks too large for the batched kernel");
        const int ld = (L.max_local_nodes + 3) & ~3;  // 16-byte rows for the coordinate runs
        const size_t smem = multi_smem<K>(ld);
        if (smem > 200 * 1024) return fail(PL_ERR_UNSUPPORTED, "cell blocks too large for the batched kernel");
        ensure_kernel_smem((const void*)k_tet_blocked_jv32_multi<K>, smem);
        static int per_sm = 0;  // occupancy of this instantiation for its shared memory
        static size_t per_sm_smem = 0;
        if (per_sm_smem != smem) {
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tet_blocked_jv32_multi<K>, kMultiBlockCells, smem);
            per_sm = std::max(per_sm, 1);
            per_sm_smem = smem;
        }
        const int grid = (int)std::min<int64_t>(L.num_blocks, (int64_t)sm_count() * per_sm);
        FinSpec fin;
        if (pq) {
            fin.counter = ticket;
            fin.out_a = pq;
        }
        k_tet_blocked_jv32_multi<K><<<grid, kMultiBlockCells, smem, s>>>(
            pp, L.d_cell_begin, L.d_block_node_begin, reduced ? L.d_slot_node_red : L.d_slot_node,
            (const ushort4*)L.d_local_cells, L.d_inc_off, L.d_inc,
            L.d_pipe_begin, L.d_pipe_coords, L.num_blocks, ld, v, out, first, pq ? part : nullptr, scal, fin);
        first = false;
        count_launch();
    }
    if (S->npairs > 0 && !reduced) {
        k_b_fold<K><<<bgrid(3 * K * S->npairs), 256, 0, s>>>(out, S->d_pair_neg, S->d_pair_pos, S->npairs);
        count_launch();
    }
    return PL_OK;
}

template <int K>
int jv32_multi(pl_batch_solver B, const float* v, float* out, double* pq = nullptr) {
    return jv32_multi_on<K>(B->base, B->n, v, out, pq, B->ticket, B->part_a, B->scal);
}

// z = q(P A) P r with the Chebyshev coefficients of the solver; partial r.z into part_a (and,
// with fin.counter, the final r.z into fin.out_a, the old value into fin.prev_a).
template <int K>
int cheb_apply(pl_batch_solver B, FinSpec fin = FinSpec()) {
    pl_solver S = B->base;
    cudaStream_t s = S->mesh->ctx->stream;
    k_cheb_first<K><<<kBBlocks, kBThreads, 0, s>>>(B->r, B->d, B->z, S->d_mask, S->d_pinv32, B->nnodes, B->cheb_s0);
    count_launch();
    for (int i = 1; i < B->cheb_degree; ++i) {
        int rc = jv32_multi<K>(B, B->d, B->q);
        if (rc) return rc;
        const float* src = i == 1 ? B->r : B->res;
        if (i == B->cheb_degree - 1)
            k_cheb_step<K, true><<<kBBlocks, kBThreads, 0, s>>>(src, B->q, B->res, B->d, B->z, B->r, S->d_mask,
                                                                S->d_pinv32, B->nnodes, B->cheb_c1[i], B->cheb_c2[i],
                                                                B->part_a, fin);
        else
            k_cheb_step<K, false><<<kBBlocks, kBThreads, 0, s>>>(src, B->q, B->res, B->d, B->z, B->r, S->d_mask,
                                                                 S->d_pinv32, B->nnodes, B->cheb_c1[i], B->cheb_c2[i],
                                                                 nullptr, FinSpec());
        count_launch();
    }
    return PL_OK;
}

// ---- multigrid V-cycles on the tile's K vectors ([n][K], one thread per (DOF or node, rhs)) ----
// The same cycle as the single-vector multigrid (csrc/multigrid.cu): Chebyshev-Jacobi pre- and
// post-smoothing, restriction and prolongation in the coarse levels' reduced fault spaces, the
// coarsest level by its dense inverse; the level operators are the batched cell-block kernel.

// out = D^{-1} in / theta; d = out
template <int K>
__global__ void __launch_bounds__(kBThreads) k_bmg_cheb_first(const float* __restrict__ in, const float* __restrict__ P,
                                                              int64_t nnodes, float inv_theta, float* __restrict__ d,
                                                              float* __restrict__ out) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nnodes * K; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t nd = t / K;
        const int k = (int)(t % K);
        float z[3];
        pinv_apply<K>(P, in, nd, k, z);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int64_t i = (3 * nd + c) * K + k;
            const float v = z[c] * inv_theta;
            d[i] = v;
            out[i] = v;
        }
    }
}

// res = in - A out (= in + q on free DOFs), d = c1 d + c2 D^{-1} res, out += d
template <int K>
__global__ void __launch_bounds__(kBThreads) k_bmg_cheb_next(const float* __restrict__ in, const float* __restrict__ q,
                                                             const float* __restrict__ P, const uint8_t* __restrict__ mask,
                                                             int64_t nnodes, float c1, float c2, float* __restrict__ d,
                                                             float* __restrict__ out) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nnodes * K; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t nd = t / K;
        const int k = (int)(t % K);
        float res[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int64_t i = (3 * nd + c) * K + k;
            res[c] = mask[3 * nd + c] ? 0.0f : in[i] + q[i];
        }
        const float* Bk = P + 9 * nd;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int64_t i = (3 * nd + c) * K + k;
            const float zr = Bk[3 * c] * res[0] + Bk[3 * c + 1] * res[1] + Bk[3 * c + 2] * res[2];
            const float dv = c1 * d[i] + c2 * zr;
            d[i] = dv;
            out[i] += dv;
        }
    }
}

// t = in + q on free DOFs (in - A z), 0 elsewhere
template <int K>
__global__ void __launch_bounds__(kBThreads) k_bmg_residual(const float* __restrict__ in, const float* __restrict__ q,
                                                            const uint8_t* __restrict__ mask, int64_t n,
                                                            float* __restrict__ t) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n * K; e += (int64_t)gridDim.x * blockDim.x)
        t[e] = mask[e / K] ? 0.0f : in[e] + q[e];
}

template <int K>
__global__ void __launch_bounds__(kBThreads) k_bmg_axpy(float* __restrict__ y, const float* __restrict__ x, int64_t n) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n * K; e += (int64_t)gridDim.x * blockDim.x)
        y[e] += x[e];
}

// coarse[(3c + comp)][k] = sum_j R[c][j] fine[(3 col_j + comp)][k], 0 on the coarse level's masked
// DOFs (R = P^T in coarse rows, in the coarse reduced space): one warp per coarse node, its lanes
// (32 / K row entries at a time) x (K right-hand sides); the entry groups' sums meet in a fixed
// shuffle tree.
template <int K>
__global__ void __launch_bounds__(kBThreads) k_bmg_restrict(const float* __restrict__ fine, const int32_t* __restrict__ row,
                                                            const int32_t* __restrict__ col, const double* __restrict__ val,
                                                            const uint8_t* __restrict__ cmask, int64_t nc,
                                                            float* __restrict__ coarse) {
    constexpr int G = 32 / K;  // entries per step
    const int lane = threadIdx.x & 31, k = lane % K, g = lane / K;
    for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < nc;
         c += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        for (int32_t j = row[c] + g; j < row[c + 1]; j += G) {
            const double w = val[j];
            const float* f = fine + 3 * (int64_t)col[j] * K + k;
            s0 += w * (double)f[0];
            s1 += w * (double)f[K];
            s2 += w * (double)f[2 * K];
        }
#pragma unroll
        for (int o = K; o < 32; o <<= 1) {
            s0 += __shfl_xor_sync(0xffffffffu, s0, o);
            s1 += __shfl_xor_sync(0xffffffffu, s1, o);
            s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        }
        if (g == 0) {
            coarse[(3 * c + 0) * K + k] = cmask[3 * c + 0] ? 0.0f : (float)s0;
            coarse[(3 * c + 1) * K + k] = cmask[3 * c + 1] ? 0.0f : (float)s1;
            coarse[(3 * c + 2) * K + k] = cmask[3 * c + 2] ? 0.0f : (float)s2;
        }
    }
}

// fine[(3f + comp)][k] += sum_j P[f][j] coarse[(3 col_j + comp)][k] on free fine DOFs
template <int K>
__global__ void __launch_bounds__(kBThreads) k_bmg_prolong_add(const float* __restrict__ coarse, const int32_t* __restrict__ row,
                                                               const int32_t* __restrict__ col, const double* __restrict__ val,
                                                               const uint8_t* __restrict__ mask, int64_t nf,
                                                               float* __restrict__ fine) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 3 * nf * K; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t fk = t / K;
        if (mask[fk]) continue;
        const int k = (int)(t % K);
        const int64_t f = fk / 3;
        const int comp = (int)(fk % 3);
        double sum = 0.0;
        for (int32_t j = row[f]; j < row[f + 1]; ++j) sum += val[j] * (double)coarse[(3 * (int64_t)col[j] + comp) * K + k];
        fine[t] += (float)sum;
    }
}

// z[idx[i]][k] = sum_j inv[i][j] r[idx[j]][k] (z zeroed before): each block stages the gathered
// right-hand sides ([n][K] floats of dynamic shared memory); one warp per row, its lanes over the
// row's columns with K sums each, reduced across the warp.
template <int K>
__global__ void __launch_bounds__(kBThreads) k_bmg_dense(const float* __restrict__ inv, const int32_t* __restrict__ idx, int n,
                                                         const float* __restrict__ r, float* __restrict__ z) {
    extern __shared__ float sr[];
    for (int t = threadIdx.x; t < n * K; t += blockDim.x) sr[t] = r[(int64_t)idx[t / K] * K + t % K];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    for (int i = blockIdx.x * (kBThreads / 32) + (threadIdx.x >> 5); i < n; i += gridDim.x * (kBThreads / 32)) {
        const float* row = inv + (int64_t)i * n;
        float acc[K];
#pragma unroll
        for (int k = 0; k < K; ++k) acc[k] = 0.0f;
        for (int j = lane; j < n; j += 32) {
            const float a = row[j];
#pragma unroll
            for (int k = 0; k < K; ++k) acc[k] += a * sr[j * K + k];
        }
#pragma unroll
        for (int k = 0; k < K; ++k)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
        if (lane < K) {
            float v = acc[0];
#pragma unroll
            for (int k = 1; k < K; ++k)
                if (lane == k) v = acc[k];
            z[(int64_t)idx[i] * K + lane] = v;
        }
    }
}

// partials of r.z (part) and, with q, of z.q (part_q) over free DOFs by right-hand side (and, with
// fin.counter, the final sums: r.z into fin.out_a, z.q into fin.out_b)
template <int K>
__global__ void __launch_bounds__(kBThreads) k_b_rz(const float* __restrict__ r, const float* __restrict__ z,
                                                    const float* __restrict__ q, const uint8_t* __restrict__ mask,
                                                    int64_t n, double* part, double* part_q, FinSpec fin) {
    double acc = 0.0, accq = 0.0;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n * K; e += (int64_t)gridDim.x * blockDim.x)
        if (!mask[e / K]) {
            acc += (double)r[e] * z[e];
            if (q) accq += (double)z[e] * q[e];
        }
    block_sum_by_rhs<K>(acc, part);
    if (q) {
        __syncthreads();
        block_sum_by_rhs<K>(accq, part_q);
    }
    if (fin.counter && take_last_ticket(fin.counter)) {
        sum_partials_last_block<K>(part, fin.out_a, fin.prev_a);
        if (q && fin.out_b) sum_partials_last_block<K>(part_q, fin.out_b, nullptr);
    }
}

// Level l's operator on K vectors: the batched cell-block kernel of its solver (level 0: the
// tile's own solver) with its faults' unfold and fold.
template <int K>
int bmg_jv(pl_batch_solver B, int l, const float* v, float* out) {
    pl_solver S = l == 0 ? B->base : B->mgv.levels[l].S;
    return jv32_multi_on<K>(S, S->n, v, out, nullptr, B->ticket, B->part_a, B->scal);
}

// Chebyshev-Jacobi polynomial of level l on K vectors from a zero guess (as the single-vector
// multigrid's cheb()).
template <int K>
int bmg_cheb(pl_batch_solver B, int l, const float* in, float* out, int degree, double lower) {
    const MgLevelView& L = B->mgv.levels[l];
    pl_solver S = l == 0 ? B->base : L.S;
    const pl_batch_solver_s::BmgLevel& W = B->bmg[l];
    cudaStream_t s = S->mesh->ctx->stream;
    const double b = 1.1 * L.lmax, a = lower * b;
    const double theta = 0.5 * (b + a), delta = 0.5 * (b - a), sigma = theta / delta;
    k_bmg_cheb_first<K><<<kBBlocks, kBThreads, 0, s>>>(in, S->d_pinv32, S->nnodes, (float)(1.0 / theta), W.d, out);
    count_launch();
    double rho_old = 1.0 / sigma;
    for (int i = 1; i < degree; ++i) {
        int rc = bmg_jv<K>(B, l, out, W.q);
        if (rc) return rc;
        const double rho = 1.0 / (2.0 * sigma - rho_old);
        k_bmg_cheb_next<K><<<kBBlocks, kBThreads, 0, s>>>(in, W.q, S->d_pinv32, S->d_mask, S->nnodes, (float)(rho * rho_old),
                                                          (float)(2.0 * rho / delta), W.d, out);
        count_launch();
        rho_old = rho;
    }
    return PL_OK;
}

// z = V(r) on level l (K vectors)
template <int K>
int bmg_vcycle(pl_batch_solver B, int l, const float* r, float* z) {
    const MgView& V = B->mgv;
    const MgLevelView& L = V.levels[l];
    pl_solver S = l == 0 ? B->base : L.S;
    const pl_batch_solver_s::BmgLevel& W = B->bmg[l];
    cudaStream_t s = S->mesh->ctx->stream;
    const int last = (int)V.levels.size() - 1;
    if (l == last) {
        if (V.dense_n > 0) {
            PLB_CUDA(cudaMemsetAsync(z, 0, S->n * K * sizeof(float), s));
            const size_t smem = (size_t)V.dense_n * K * sizeof(float);
            ensure_kernel_smem((const void*)k_bmg_dense<K>, smem);
            const int grid = std::max(1, std::min((V.dense_n + kBThreads / 32 - 1) / (kBThreads / 32), 4 * 148));
            k_bmg_dense<K><<<grid, kBThreads, smem, s>>>(V.dense_inv32, V.dense_idx, V.dense_n, r, z);
            count_launch();
            return PL_OK;
        }
        return bmg_cheb<K>(B, l, r, z, V.coarse_degree, V.coarse_lower);
    }
    int rc = PL_OK;
    const float* tr = r;  // the residual to restrict
    if (V.pre_smooth) {
        if ((rc = bmg_cheb<K>(B, l, r, z, V.degree, V.lower))) return rc;
        if ((rc = bmg_jv<K>(B, l, z, W.q))) return rc;
        k_bmg_residual<K><<<kBBlocks, kBThreads, 0, s>>>(r, W.q, S->d_mask, S->n, W.t);
        count_launch();
        tr = W.t;
    } else {
        PLB_CUDA(cudaMemsetAsync(z, 0, S->n * K * sizeof(float), s));
    }
    const MgLevelView& C = V.levels[l + 1];
    const pl_batch_solver_s::BmgLevel& Wc = B->bmg[l + 1];
    if (C.n > 3 * C.nmesh) PLB_CUDA(cudaMemsetAsync(Wc.r + 3 * C.nmesh * K, 0, (C.n - 3 * C.nmesh) * K * sizeof(float), s));
    k_bmg_restrict<K><<<(int)std::max<int64_t>(1, std::min<int64_t>((C.nmesh + 7) / 8, kBBlocks)), kBThreads, 0, s>>>(
        tr, L.r_row, L.r_col, L.r_val, C.S->d_mask, C.nmesh, Wc.r);
    count_launch();
    if ((rc = bmg_vcycle<K>(B, l + 1, Wc.r, Wc.z))) return rc;
    k_bmg_prolong_add<K><<<kBBlocks, kBThreads, 0, s>>>(Wc.z, L.p_row, L.p_col, L.p_val, S->d_mask, L.nmesh, z);
    count_launch();
    if (!V.post_smooth) return PL_OK;
    if ((rc = bmg_jv<K>(B, l, z, W.q))) return rc;
    k_bmg_residual<K><<<kBBlocks, kBThreads, 0, s>>>(r, W.q, S->d_mask, S->n, W.t);
    count_launch();
    if ((rc = bmg_cheb<K>(B, l, W.t, W.w, V.degree, V.lower))) return rc;
    k_bmg_axpy<K><<<kBBlocks, kBThreads, 0, s>>>(z, W.w, S->n);
    count_launch();
    return PL_OK;
}

// z = V(r) for the tile; partial r.z into part_a (and with fin.counter the final sums).
template <int K>
int bmg_apply(pl_batch_solver B, FinSpec fin = FinSpec()) {
    pl_solver S = B->base;
    cudaStream_t s = S->mesh->ctx->stream;
    int rc = bmg_vcycle<K>(B, 0, B->r, B->z);
    if (rc) return rc;
    // inside an iteration (fin.out_b set) also z.q for the flexible step (q = J p of this iteration)
    k_b_rz<K><<<kBBlocks, kBThreads, 0, s>>>(B->r, B->z, fin.out_b ? B->q : nullptr, S->d_mask, B->n, B->part_a,
                                             B->part_b, fin);
    count_launch();
    return PL_OK;
}

// The polynomial or multigrid preconditioner of the tile (point-block Jacobi runs inside the
// update kernels instead).
bool tile_preconditioned(pl_batch_solver B) { return B->mg || B->cheb_degree >= 2; }

template <int K>
int precond_apply(pl_batch_solver B, FinSpec fin = FinSpec()) {
    return B->mg ? bmg_apply<K>(B, fin) : cheb_apply<K>(B, fin);
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
    // the final sums are formed by the last block of each reduction kernel (no k_b_finish launches)
    const bool fused = fuses_energies(B);
    int rc = jv32_multi<K>(B, B->p, B->q, fused ? pq : nullptr);
    if (rc) return rc;
    if (!fused) {
        FinSpec fpq;
        fpq.counter = B->ticket;
        fpq.out_a = pq;
        k_b_pq<K><<<kBBlocks, kBThreads, 0, s>>>(B->p, B->q, S->d_mask, B->n, B->part_a, fpq);
        count_launch();
    }
    if (tile_preconditioned(B)) {
        FinSpec frr;
        frr.counter = B->ticket;
        frr.out_a = rr;
        k_b_update_xr<K><<<kBBlocks, kBThreads, 0, s>>>(B->r, B->q, S->d_mask, B->n, rz, pq, B->active, B->part_b,
                                                        frr);
        count_launch();
        FinSpec frz;
        frz.counter = B->ticket;
        frz.out_a = rz;
        frz.prev_a = rz_old;
        if (B->mg) frz.out_b = B->scal + 5 * kMaxTile;  // z.q of the flexible step
        rc = precond_apply<K>(B, frz);
        if (rc) return rc;
    } else {
        FinSpec fu;
        fu.counter = B->ticket;
        fu.out_a = rz;
        fu.prev_a = rz_old;
        fu.out_b = rr;
        // z = P r is not stored: k_b_pupdate_jacobi forms it again from r
        k_b_update<K, false><<<kBBlocks, kBThreads, 0, s>>>(B->r, B->q, nullptr, S->d_mask, S->d_pinv32, B->nnodes, rz,
                                                            pq, B->active, B->part_a, B->part_b, fu);
        count_launch();
        k_b_pupdate_jacobi<K><<<kBBlocks, kBThreads, 0, s>>>(B->x, B->p, B->r, S->d_mask, S->d_pinv32, B->nnodes, rz,
                                                             rz_old, pq, B->active);
        count_launch();
        return PL_OK;
    }
    k_b_pupdate<K><<<kBBlocks, kBThreads, 0, s>>>(B->x, B->p, B->z, S->d_mask, B->n, rz, rz_old, pq, B->active,
                                                  B->mg ? B->scal + 5 * kMaxTile : nullptr);
    count_launch();
    return PL_OK;
}

// Largest eigenvalue of P A by power iteration on the tile's K vectors (deterministic start);
// sets the Chebyshev coefficients for the interval [lower_ratio b, b], b = 1.1 lambda_max.
template <int K>
int cheb_setup(pl_batch_solver B) {
    pl_solver S = B->base;
    cudaStream_t s = S->mesh->ctx->stream;
    const int64_t n = B->n;
    ColScale cs{};
    k_power_scale<K><<<kBBlocks, kBThreads, 0, s>>>(B->p, nullptr, S->d_mask, n, cs);
    count_launch();
    double lam = 0.0;
    double h[2 * kMaxTile];
    for (int it = 0; it < B->cheb_eig_iters; ++it) {
        int rc = jv32_multi<K>(B, B->p, B->q);
        if (rc) return rc;
        k_power_step<K><<<kBBlocks, kBThreads, 0, s>>>(B->p, B->q, B->z, S->d_mask, S->d_pinv32, B->nnodes, B->part_a,
                                                       B->part_b);
        k_b_finish<K><<<K, kBThreads, 0, s>>>(B->part_a, kBBlocks, B->scal, nullptr);
        k_b_finish<K><<<K, kBThreads, 0, s>>>(B->part_b, kBBlocks, B->scal + K, nullptr);
        count_launch(3);
        PLB_CUDA(cudaMemcpyAsync(h, B->scal, 2 * K * sizeof(double), cudaMemcpyDeviceToHost, s));
        PLB_CUDA(cudaStreamSynchronize(s));
        lam = 0.0;
        for (int k = 0; k < K; ++k) {
            const double ww = h[k], vv = h[K + k];
            if (vv > 0.0 && ww > 0.0) lam = std::max(lam, std::sqrt(ww / vv));
            cs.s[k] = ww > 0.0 ? (float)(1.0 / std::sqrt(ww)) : 0.0f;
        }
        if (!(lam > 0.0) || !std::isfinite(lam)) return fail(PL_ERR_NOT_CONVERGED, "eigenvalue estimate failed");
        k_power_scale<K><<<kBBlocks, kBThreads, 0, s>>>(B->p, B->z, S->d_mask, n, cs);
        count_launch();
    }
    B->cheb_lmax = lam;
    const double b = 1.1 * lam, a = B->cheb_lower_ratio * b;
    const double theta = 0.5 * (b + a), delta = 0.5 * (b - a), sigma = theta / delta;
    double rho = 1.0 / sigma;
    B->cheb_s0 = (float)(1.0 / theta);
    for (int i = 1; i < B->cheb_degree; ++i) {
        const double rho_new = 1.0 / (2.0 * sigma - rho);
        B->cheb_c1[i] = (float)(rho_new * rho);
        B->cheb_c2[i] = (float)(2.0 * rho_new / delta);
        rho = rho_new;
    }
    B->cheb_version++;
    B->cheb_epoch = state_epoch();
    return PL_OK;
}

// Captures (once per tile size, state epoch and preconditioner) the graph of check_every PCG
// iterations.
template <int K>
int ensure_pcg_graph(pl_batch_solver B) {
    pl_solver S = B->base;
    cudaStream_t s = S->mesh->ctx->stream;
    const int chunk = S->check_every;
    if (B->graph && B->graph_iters == chunk && B->graph_epoch == state_epoch() && B->graph_cheb == B->cheb_version)
        return PL_OK;
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
    B->graph_epoch = state_epoch();
    B->graph_cheb = B->cheb_version;
    return PL_OK;
}

// FP32 PCG on the tile: r holds the right-hand sides on entry; x returns the corrections.
template <int K>
int tile_pcg(pl_batch_solver B, int nact, double rtol, int max_iter, int* iters) {
    pl_solver S = B->base;
    cudaStream_t s = S->mesh->ctx->stream;
    PLB_CUDA(cudaMemsetAsync(B->x, 0, B->n * K * sizeof(float), s));
    k_b_init<K><<<kBBlocks, kBThreads, 0, s>>>(B->r, B->z, B->p, S->d_mask, S->d_pinv32, B->nnodes, B->part_a, B->part_b);
    k_b_finish<K><<<K, kBThreads, 0, s>>>(B->part_a, kBBlocks, B->scal, nullptr);
    k_b_finish<K><<<K, kBThreads, 0, s>>>(B->part_b, kBBlocks, B->scal + 3 * K, nullptr);
    count_launch(3);
    double h[4 * kMaxTile];
    int act[kMaxTile];
    if (tile_preconditioned(B)) {
        // z = q(P A) P r or V(r), p = z, rz = r.z
        int rc = precond_apply<K>(B);
        if (rc) return rc;
        k_b_finish<K><<<K, kBThreads, 0, s>>>(B->part_a, kBBlocks, B->scal, nullptr);
        count_launch();
        PLB_CUDA(cudaMemcpyAsync(B->p, B->z, B->n * K * sizeof(float), cudaMemcpyDeviceToDevice, s));
    }
    PLB_CUDA(cudaMemcpyAsync(h, B->scal, 4 * K * sizeof(double), cudaMemcpyDeviceToHost, s));
    PLB_CUDA(cudaStreamSynchronize(s));
    double r0[kMaxTile];
    for (int k = 0; k < K; ++k) {
        r0[k] = std::sqrt(h[3 * K + k]);
        act[k] = (k < nact && r0[k] > 0.0) ? 1 : 0;
    }
    PLB_CUDA(cudaMemcpyAsync(B->active, act, K * sizeof(int), cudaMemcpyHostToDevice, s));
    const int chunk = S->check_every;
    int rc = ensure_pcg_graph<K>(B);
    if (rc) return rc;
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

// FP64 true residual of right-hand side kk, r = P^T (b + J x) on free DOFs (x unfolded first for
// faults), packed into column kk of the FP32 tile residual; returns |r|.
int col_true_residual(pl_batch_solver B, int K, int kk, const double* b, double* x, double* rnorm) {
    pl_solver S = B->base;
    cudaStream_t s = S->mesh->ctx->stream;
    const int64_t n = B->n;
    if (S->npairs > 0) {
        k_unfold64<<<bgrid(3 * S->npairs), 256, 0, s>>>(x, S->d_pair_neg, S->d_pair_pos, S->npairs);
        count_launch();
    }
    int rc = apply_J64(S, x, B->jx64);
    if (rc) return rc;
    PLB_CUDA(cudaMemcpyAsync(B->r64, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if (S->npairs > 0) {
        k_fold64<<<bgrid(3 * S->npairs), 256, 0, s>>>(B->jx64, S->d_pair_neg, S->d_pair_pos, S->npairs);
        k_fold64<<<bgrid(3 * S->npairs), 256, 0, s>>>(B->r64, S->d_pair_neg, S->d_pair_pos, S->npairs);
        count_launch(2);
    }
    k_outer64<<<kBBlocks, kBThreads, 0, s>>>(B->r64, B->jx64, S->d_mask, n, B->r64, B->part_a);
    k_b_finish<1><<<1, kBThreads, 0, s>>>(B->part_a, kBBlocks, B->scal + 4 * kMaxTile, nullptr);
    k_b_pack<<<bgrid(n), 256, 0, s>>>(B->r64, n, K, kk, B->r);
    count_launch(3);
    double h;
    PLB_CUDA(cudaMemcpyAsync(&h, B->scal + 4 * kMaxTile, sizeof(double), cudaMemcpyDeviceToHost, s));
    PLB_CUDA(cudaStreamSynchronize(s));
    *rnorm = std::sqrt(h);
    return PL_OK;
}

// All right-hand sides with reliable updates (van der Vorst and Ye, "Residual replacement
// strategies for Krylov subspace iterative methods for the convergence of true residuals", SIAM J.
// Sci. Comput. 22 (2000); as in the mixed-precision CG of Clark et al., Comput. Phys. Commun. 181
// (2010)). Each of the K columns of the tile runs the FP32 PCG of one right-hand side without
// restarts. At a convergence check, a column whose iterated residual has dropped below
// reliable_delta times its last true residual adds its FP32 correction to the FP64 solution and
// gets the FP64 true residual (with z = M r and r.z) in place of the iterated one, keeping its
// search direction. A right-hand side is done when its true residual meets rtol; its column then
// starts the next pending right-hand side (r = b, z = M r, p = z), so no column idles while
// right-hand sides remain.
template <int K>
int solve_reliable(pl_batch_solver B, int nrhs, const double* const* bs, double* const* xs) {
    pl_solver S = B->base;
    cudaStream_t s = S->mesh->ctx->stream;
    const int64_t n = B->n;
    double bnorm[kMaxTile] = {0}, rref[kMaxTile] = {0};
    int act[kMaxTile] = {0}, slot[kMaxTile], iters[kMaxTile] = {0}, breakdowns[kMaxTile] = {0};
    bool fresh[kMaxTile] = {false}, replaced[kMaxTile] = {false};
    for (int k = 0; k < K; ++k) slot[k] = -1;
    int next = 0;
    int rc = PL_OK;
    PLB_CUDA(cudaMemsetAsync(B->r, 0, n * K * sizeof(float), s));
    PLB_CUDA(cudaMemsetAsync(B->x, 0, n * K * sizeof(float), s));
    // final FP64 solution of right-hand side j (faults: the positive side follows the negative)
    auto finish_rhs = [&](int j) {
        if (S->npairs > 0) {
            k_unfold64<<<bgrid(3 * S->npairs), 256, 0, s>>>(xs[j], S->d_pair_neg, S->d_pair_pos, S->npairs);
            count_launch();
        }
    };
    // column k takes the next pending right-hand side with a nonzero residual (r = b, x = 0)
    auto assign = [&](int k) -> int {
        slot[k] = -1;
        act[k] = 0;
        while (next < nrhs) {
            const int j = next++;
            PLB_CUDA(cudaMemsetAsync(xs[j], 0, n * sizeof(double), s));
            double bn = 0.0;
            int r2 = col_true_residual(B, K, k, bs[j], xs[j], &bn);
            if (r2) return r2;
            B->outer_iterations++;
            if (bn > 0.0) {
                slot[k] = j;
                act[k] = 1;
                bnorm[k] = rref[k] = bn;
                iters[k] = 0;
                return PL_OK;
            }
            finish_rhs(j);
        }
        // no right-hand side left: the column's residual is cleared (it stays inactive)
        k_b_col_zero<<<bgrid(n), 256, 0, s>>>(B->r, n, K, k);
        count_launch();
        return PL_OK;
    };
    for (int k = 0; k < K; ++k)
        if ((rc = assign(k)) != PL_OK) return rc;
    k_b_init<K><<<kBBlocks, kBThreads, 0, s>>>(B->r, B->z, B->p, S->d_mask, S->d_pinv32, B->nnodes, B->part_a, B->part_b);
    k_b_finish<K><<<K, kBThreads, 0, s>>>(B->part_a, kBBlocks, B->scal, nullptr);
    k_b_finish<K><<<K, kBThreads, 0, s>>>(B->part_b, kBBlocks, B->scal + 3 * K, nullptr);
    count_launch(3);
    if (tile_preconditioned(B)) {
        if ((rc = precond_apply<K>(B)) != PL_OK) return rc;
        k_b_finish<K><<<K, kBThreads, 0, s>>>(B->part_a, kBBlocks, B->scal, nullptr);
        count_launch();
        PLB_CUDA(cudaMemcpyAsync(B->p, B->z, n * K * sizeof(float), cudaMemcpyDeviceToDevice, s));
    }
    PLB_CUDA(cudaMemcpyAsync(B->active, act, K * sizeof(int), cudaMemcpyHostToDevice, s));
    if ((rc = ensure_pcg_graph<K>(B)) != PL_OK) return rc;
    const int chunk = S->check_every;
    double h[4 * kMaxTile];
    bool any = false;
    for (int k = 0; k < K; ++k) any = any || act[k];
    while (any) {
        PLB_CUDA(cudaGraphLaunch(B->graph, s));
        B->inner_iterations += chunk;
        PLB_CUDA(cudaMemcpyAsync(h, B->scal, 4 * K * sizeof(double), cudaMemcpyDeviceToHost, s));
        PLB_CUDA(cudaStreamSynchronize(s));
        bool changed = false, update_z = false;
        for (int k = 0; k < K; ++k) {
            fresh[k] = replaced[k] = false;
            if (!act[k]) continue;
            iters[k] += chunk;
            if (iters[k] > S->max_iter) return fail(PL_ERR_NOT_CONVERGED, "batched PCG reached the iteration limit");
            const double rn = std::sqrt(h[3 * K + k]);
            // FP32 breakdown (the iterated residual not a number or far above the last true one):
            // drop the column's FP32 correction and restart it from its FP64 true residual
            const bool broke = !(rn == rn) || rn > kBreakdownGrowth * rref[k];
            if (broke) {
                if (++breakdowns[k] > kMaxBreakdowns)
                    return fail(PL_ERR_NOT_CONVERGED, "batched PCG broke down repeatedly");
                k_b_col_zero<<<bgrid(n), 256, 0, s>>>(B->x, n, K, k);
                count_launch();
                double rt = 0.0;
                if ((rc = col_true_residual(B, K, k, bs[slot[k]], xs[slot[k]], &rt)) != PL_OK) return rc;
                B->outer_iterations++;
                rref[k] = rt;
                fresh[k] = update_z = true;  // p = z again
                continue;
            }
            if (rn > B->reliable_delta * rref[k] && rn > 0.5 * S->rtol * bnorm[k]) continue;
            const int j = slot[k];
            k_b_unpack_add<<<bgrid(n), 256, 0, s>>>(B->x, n, K, k, S->d_mask, xs[j]);
            k_b_col_zero<<<bgrid(n), 256, 0, s>>>(B->x, n, K, k);
            count_launch(2);
            double rt = 0.0;
            if ((rc = col_true_residual(B, K, k, bs[j], xs[j], &rt)) != PL_OK) return rc;
            B->reliable_updates++;
            B->outer_iterations++;
            if (rt <= S->rtol * bnorm[k]) {
                B->max_rel_residual = std::max(B->max_rel_residual, rt / bnorm[k]);
                finish_rhs(j);
                if ((rc = assign(k)) != PL_OK) return rc;
                changed = true;
                if (act[k]) fresh[k] = update_z = true;
                continue;
            }
            rref[k] = rt;
            replaced[k] = update_z = true;
        }
        if (update_z && B->mg) {
            // multigrid (flexible steps): no V-cycle of the whole tile here, which would cost as
            // much as an iteration. A replaced residual keeps its column's z, the V-cycle of the
            // residual it replaces (they differ by the FP32 drift, which the flexible step
            // absorbs); a new (or restarted) column starts from point-block Jacobi, z = P r, and
            // meets the V-cycle at its next iteration. Then r.z of every column again.
            for (int k = 0; k < K; ++k)
                if (fresh[k]) {
                    k_b_col_prec<<<kBBlocks, kBThreads, 0, s>>>(B->r, B->z, S->d_mask, S->d_pinv32, B->nnodes, K, k,
                                                                B->part_a);
                    k_b_col_copy<<<bgrid(n), 256, 0, s>>>(B->p, B->z, n, K, k);
                    count_launch(2);
                }
            k_b_rz<K><<<kBBlocks, kBThreads, 0, s>>>(B->r, B->z, nullptr, S->d_mask, B->n, B->part_a, B->part_b, FinSpec());
            k_b_finish<K><<<K, kBThreads, 0, s>>>(B->part_a, kBBlocks, B->scal, nullptr);
            count_launch(2);
        } else if (update_z) {
            if (tile_preconditioned(B)) {
                // z = q(P A) P r (or V(r)) with the same operator for the whole tile (the other
                // columns get their own z and r.z again), so the preconditioner stays fixed
                if ((rc = precond_apply<K>(B)) != PL_OK) return rc;
                k_b_finish<K><<<K, kBThreads, 0, s>>>(B->part_a, kBBlocks, B->scal, nullptr);
                count_launch();
            } else {
                for (int k = 0; k < K; ++k) {
                    if (!fresh[k] && !replaced[k]) continue;
                    k_b_col_prec<<<kBBlocks, kBThreads, 0, s>>>(B->r, B->z, S->d_mask, S->d_pinv32, B->nnodes, K, k,
                                                                B->part_a);
                    k_b_finish<1><<<1, kBThreads, 0, s>>>(B->part_a, kBBlocks, B->scal + k, nullptr);
                    count_launch(2);
                }
            }
            // a new right-hand side starts from p = z
            for (int k = 0; k < K; ++k)
                if (fresh[k]) {
                    k_b_col_copy<<<bgrid(n), 256, 0, s>>>(B->p, B->z, n, K, k);
                    count_launch();
                }
        }
        if (changed) PLB_CUDA(cudaMemcpyAsync(B->active, act, K * sizeof(int), cudaMemcpyHostToDevice, s));
        any = false;
        for (int k = 0; k < K; ++k) any = any || act[k];
    }
    B->solves += nrhs;
    return PL_OK;
}

template <int K>
int solve_tile(pl_batch_solver B, int nact, const double* const* bs, double* const* xs) {
    pl_solver S = B->base;
    cudaStream_t s = S->mesh->ctx->stream;
    const int64_t n = B->n;
    double bnorm[kMaxTile] = {0}, rn[kMaxTile] = {0};
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
            k_b_finish<1><<<1, kBThreads, 0, s>>>(B->part_a, kBBlocks, B->scal, nullptr);
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
    if (!base || !out || !(tile == 1 || tile == 2 || tile == 4 || tile == 8 || tile == 16))
        return fail(PL_ERR_INVALID_ARG, "tile must be 1, 2, 4, 8 or 16");
    *out = nullptr;
    pl_batch_solver B = new pl_batch_solver_s();
    B->base = base;
    B->K = tile;
    B->n = base->n;
    B->nnodes = base->nnodes;
    mesh_retain(base->mesh);
    solver_retain(base);
    cudaError_t e = cudaSuccess;
    auto A = [&](auto** p, size_t cnt) {
        if (e == cudaSuccess) e = dev_alloc(p, cnt);
    };
    const size_t nk = (size_t)B->n * tile;
    A(&B->r, nk); A(&B->z, nk); A(&B->p, nk); A(&B->q, nk); A(&B->x, nk);
    A(&B->scal, 6 * kMaxTile);  // rz, rz_old, pq, rr; the outer residual; z.q (flexible step)
    A(&B->active, kMaxTile);
    A(&B->part_a, (size_t)kBBlocks * kMaxTile);
    A(&B->part_b, (size_t)kBBlocks * kMaxTile);
    A(&B->ticket, 1);
    if (e == cudaSuccess) e = cudaMemset(B->ticket, 0, sizeof(unsigned int));
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
    if (nrhs > 0 && B->mg) {
        // the hierarchy's eigenvalue estimates and dense coarsest inverse (made by its first solve
        // after a setup, or here)
        rc = multigrid_prepare(B->mg);
        if (rc == PL_OK) {
            const MgView v = multigrid_view(B->mg);
            bool changed = v.levels.size() != B->mgv.levels.size() || v.dense_inv32 != B->mgv.dense_inv32 ||
                           v.degree != B->mgv.degree || v.lower != B->mgv.lower ||
                           v.pre_smooth != B->mgv.pre_smooth || v.post_smooth != B->mgv.post_smooth;
            for (size_t l = 0; !changed && l < v.levels.size(); ++l) changed = v.levels[l].lmax != B->mgv.levels[l].lmax;
            B->mgv = v;
            if (changed) B->cheb_version++;  // the captured iterations hold the coefficients
        }
    }
    if (rc == PL_OK && nrhs > 0 && !B->mg && B->cheb_degree >= 2 &&
        (B->cheb_version == 0 || B->cheb_epoch != state_epoch())) {
        switch (B->K) {
            case 1: rc = cheb_setup<1>(B); break;
            case 2: rc = cheb_setup<2>(B); break;
            case 4: rc = cheb_setup<4>(B); break;
            case 8: rc = cheb_setup<8>(B); break;
            default: rc = cheb_setup<16>(B); break;
        }
    }
    if (rc == PL_OK && B->reliable && nrhs > 0) {
        switch (B->K) {
            case 1: rc = solve_reliable<1>(B, nrhs, b_dev, x_dev); break;
            case 2: rc = solve_reliable<2>(B, nrhs, b_dev, x_dev); break;
            case 4: rc = solve_reliable<4>(B, nrhs, b_dev, x_dev); break;
            case 8: rc = solve_reliable<8>(B, nrhs, b_dev, x_dev); break;
            default: rc = solve_reliable<16>(B, nrhs, b_dev, x_dev); break;
        }
    }
    for (int r0 = 0; !B->reliable && r0 < nrhs && rc == PL_OK; r0 += B->K) {
        const int nact = std::min(B->K, nrhs - r0);
        switch (B->K) {
            case 1: rc = solve_tile<1>(B, nact, b_dev + r0, x_dev + r0); break;
            case 2: rc = solve_tile<2>(B, nact, b_dev + r0, x_dev + r0); break;
            case 4: rc = solve_tile<4>(B, nact, b_dev + r0, x_dev + r0); break;
            case 8: rc = solve_tile<8>(B, nact, b_dev + r0, x_dev + r0); break;
            default: rc = solve_tile<16>(B, nact, b_dev + r0, x_dev + r0); break;
        }
        if (rc == PL_OK) B->solves += nact;
    }
    c->stream = user;
    cudaEventRecord(B->ev_out, B->stream);
    cudaStreamWaitEvent(user, B->ev_out, 0);
    return rc;
}

int pl_batch_solver_set_chebyshev(pl_batch_solver B, int degree, double lower_ratio, int eig_iters) {
    if (!B || degree < 0 || degree > kMaxChebDegree || !(lower_ratio > 0.0 && lower_ratio < 1.0) || eig_iters < 1 ||
        eig_iters > 1000)
        return fail(PL_ERR_INVALID_ARG, "degree 0-8, lower_ratio in (0, 1), eig_iters 1-1000");
    PLB_CUDA(cudaSetDevice(B->base->mesh->ctx->device));
    if (degree >= 2 && !B->res) {
        const size_t nk = (size_t)B->n * B->K;
        PLB_CUDA(dev_alloc(&B->res, nk));
        cudaError_t e = dev_alloc(&B->d, nk);
        if (e != cudaSuccess) {
            dev_free(B->res, nullptr);
            B->res = nullptr;
            return cuda_fail(e, "pl_batch_solver_set_chebyshev");
        }
    }
    B->cheb_degree = degree;
    B->cheb_lower_ratio = lower_ratio;
    B->cheb_eig_iters = eig_iters;
    B->cheb_version = 0;  // estimate again at the next solve
    B->cheb_lmax = 0.0;
    B->graph_cheb = -1;
    return PL_OK;
}

int pl_batch_solver_set_reliable(pl_batch_solver B, int enable, double delta) {
    if (!B || !(delta > 0.0 && delta < 1.0)) return fail(PL_ERR_INVALID_ARG, "delta must lie in (0, 1)");
    B->reliable = enable != 0;
    B->reliable_delta = delta;
    return PL_OK;
}

int pl_batch_solver_get_chebyshev(pl_batch_solver B, double* lambda_max) {
    if (!B || !lambda_max) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    *lambda_max = B->cheb_lmax;
    return PL_OK;
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

static void bmg_release(pl_batch_solver B) {
    cudaStream_t s = B->base->mesh->ctx->stream;
    for (auto& W : B->bmg)
        for (float* p : {W.r, W.z, W.t, W.d, W.q, W.w}) dev_free(p, s);
    B->bmg.clear();
    if (B->mg) multigrid_batch_use(B->mg, -1);
    B->mg = nullptr;
    B->mgv = MgView();
}

int pl_batch_solver_set_multigrid(pl_batch_solver B, pl_multigrid mg) {
    if (!B) return fail(PL_ERR_INVALID_ARG, "null batched solver");
    pl_solver S = B->base;
    PLB_CUDA(cudaSetDevice(S->mesh->ctx->device));
    PLB_CUDA(cudaStreamSynchronize(S->mesh->ctx->stream));
    if (B->stream) PLB_CUDA(cudaStreamSynchronize(B->stream));
    bmg_release(B);
    B->cheb_version++;  // the captured iterations change
    if (!mg) return PL_OK;
    const MgView v = multigrid_view(mg);
    if (v.levels.empty() || v.levels[0].S->mesh != S->mesh || v.levels[0].n != S->n)
        return fail(PL_ERR_INVALID_ARG, "the hierarchy's fine level is not the batched solver's mesh");
    if (B->K > 8) return fail(PL_ERR_UNSUPPORTED, "multigrid tiles of at most 8 right-hand sides");
    // every level's operator is the batched cell-block kernel: its layout is built now, outside
    // any stream capture
    for (const MgLevelView& L : v.levels) {
        pl_mesh lm = L.S->mesh;
        if (lm->cell_type != PL_CELL_TET4) return fail(PL_ERR_UNSUPPORTED, "batched multigrid needs P1 tetrahedral levels");
        int rc = ensure_blocked_layout(lm);
        if (rc) return rc;
    }
    B->bmg.resize(v.levels.size());
    cudaError_t e = cudaSuccess;
    for (size_t l = 0; l < v.levels.size() && e == cudaSuccess; ++l) {
        const size_t nk = (size_t)v.levels[l].n * B->K;
        auto& W = B->bmg[l];
        for (float** p : {&W.r, &W.z, &W.t, &W.d, &W.q, &W.w})
            if (e == cudaSuccess) e = dev_alloc(p, nk);
        if (e == cudaSuccess) e = cudaMemsetAsync(W.r, 0, nk * sizeof(float), S->mesh->ctx->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(S->mesh->ctx->stream);
    if (e != cudaSuccess) {
        bmg_release(B);
        return cuda_fail(e, "pl_batch_solver_set_multigrid");
    }
    B->mg = mg;
    multigrid_batch_use(mg, +1);
    B->mgv = v;
    return PL_OK;
}

int pl_batch_solver_destroy(pl_batch_solver B) {
    if (!B) return PL_OK;
    pl_mesh m = B->base->mesh;
    cudaSetDevice(m->ctx->device);
    cudaStreamSynchronize(m->ctx->stream);
    bmg_release(B);
    if (B->graph) cudaGraphExecDestroy(B->graph);
    if (B->stream) cudaStreamSynchronize(B->stream);
    if (B->ev_in) cudaEventDestroy(B->ev_in);
    if (B->ev_out) cudaEventDestroy(B->ev_out);
    if (B->stream) cudaStreamDestroy(B->stream);
    void* ptrs[] = {B->r, B->z, B->p, B->q, B->x, B->scal, B->active, B->part_a, B->part_b, B->r64, B->jx64, B->res, B->d, B->ticket};
    for (void* p : ptrs) dev_free(p, m->ctx->stream);
    pl_solver base = B->base;
    delete B;
    mesh_release(m);
    solver_release(base);
    return PL_OK;
}

}  // extern "C"
