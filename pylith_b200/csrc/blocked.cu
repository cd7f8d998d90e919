// Cell-block kernels for P1 tetrahedra: the hot path of the residual and Jacobian action.
//
// Cells are processed in blocks of kTetBlockCells consecutive cells (meshes are ordered along
// a Morton curve, so a block is a compact patch). Persistent CTAs walk every gridDim.x-th block.
// For each block the CTA
//   1. has the block's nodes (coordinates and input field), node ids and incidence list in
//      shared memory: they were copied asynchronously (cp.async) into a second buffer while the
//      previous block computed, so a node is read from global memory once per block instead of
//      once per incident cell;
//   2. forms, one thread per cell, the affine geometry and the solution gradient, calls the
//      pointwise kernel and stages the 12-entry element vector in shared memory;
//   3. sums, one thread per node, the staged entries of the node's incident corners in a fixed
//      order (the precomputed block-local incidence list) and writes the node: a plain store for
//      nodes whose cells all lie in the block, one FP64 reduction into global memory for nodes
//      shared with other blocks.
// Geometry in cofactor form: with C = det(J) J^{-1}, grad(u) = (G C) / det(J) for the edge
// differences G, and the element vector of corner a (a = 1..3) is f1 C_{a-1}^T / 6, so the
// Jacobian determinant enters through one reciprocal.
#include <cuda_pipeline.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "domain_kernels.cuh"
#include "internal.hpp"
#include "launch.hpp"

namespace plb {

#ifndef PLB_TET_BLOCK
#define PLB_TET_BLOCK 256
#endif
#ifndef PLB_TET_CPT
#define PLB_TET_CPT 1
#endif
constexpr int kTetBlockCells = PLB_TET_BLOCK;
// cells per thread of the FP64 cell-block kernel (two independent cells per thread give the
// scheduler more independent instructions per warp)
constexpr int kTetCellsPerThread = PLB_TET_CPT;
constexpr int kTetThreads = kTetBlockCells / kTetCellsPerThread;
constexpr int kMaxSlotsPerThread = 512 / kTetThreads;  // blocks touching more than 512 nodes use the atomic kernel
constexpr uint32_t kSharedBit = 0x80000000u;

// cof[i][j] = det(J) (J^{-1})[i][j] with J = [X1-X0, X2-X0, X3-X0] (columns); returns det(J).
PL_D double tet_cofactors(const double X[4][3], double cof[3][3]) {
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

struct BlockArrays {
    const int32_t* cell_begin;  // [nblocks + 1] first cell of each block (at most kTetBlockCells each)
    const int32_t* slot_begin;  // [nblocks + 1]
    const uint32_t* slot_node;  // node id | kSharedBit if other blocks touch the node
    const ushort4* lconn;       // [ncells] block-local slots of the 4 corners
    const uint32_t* inc_off;    // per block ns+1 offsets (block b starts at slot_begin[b] + b)
    const uint16_t* inc;        // [nblocks][4 * kTetBlockCells] cell * 4 + corner
    double* partial;            // [slots][3] sums of shared nodes, per block (FP64 kernels)
    int64_t nblocks;
    int max_local_nodes;
};

// Shared-memory buffer of one block: node data, 6 doubles per node (x, y, z, u0, u1, u2; see
// node_index), node ids [maxloc], incidence offsets [maxloc + 1], incidence list
// [4 * kTetBlockCells].
struct SmemBuf {
    double* node;
    uint32_t* id;
    uint32_t* off;
    uint16_t* inc;
    int ld;  // leading dimension of the node arrays
};

// Word index of component d (0-2 coordinates, 3-5 field) of block-local node i. Component-major
// storage makes consecutive nodes fall in consecutive bank pairs, so the random node reads of a
// warp spread over all 16 bank pairs (a 6-double record per node reaches only 8 of them).
PL_D int node_index(const SmemBuf& s, int i, int d) { return d * s.ld + i; }

PL_HD size_t round16(size_t x) { return (x + 15) & ~size_t(15); }

PL_HD size_t buf_bytes(int maxloc) {
    return round16(48 * (size_t)maxloc) + round16(4 * (size_t)maxloc) + round16(4 * ((size_t)maxloc + 1)) +
           round16(2 * 4 * (size_t)kTetBlockCells);
}

PL_D SmemBuf make_buf(char* base, int maxloc) {
    SmemBuf s;
    s.ld = maxloc;
    s.node = reinterpret_cast<double*>(base);
    base += round16(48 * (size_t)maxloc);
    s.id = reinterpret_cast<uint32_t*>(base);
    base += round16(4 * (size_t)maxloc);
    s.off = reinterpret_cast<uint32_t*>(base);
    base += round16(4 * ((size_t)maxloc + 1));
    s.inc = reinterpret_cast<uint16_t*>(base);
    return s;
}

// Asynchronous copies of block b into buffer s; nd[k] holds slot_node of slots tid + k*blockDim
// (read one block earlier, so no global latency is exposed here).
PL_D void prefetch_block(const DomainParams& p, const double* __restrict__ field, const BlockArrays& A, int64_t b,
                         const uint32_t nd[kMaxSlotsPerThread], const SmemBuf& s) {
    const int s0 = A.slot_begin[b];
    const int ns = A.slot_begin[b + 1] - s0;
#pragma unroll
    for (int k = 0; k < kMaxSlotsPerThread; ++k) {
        const int i = threadIdx.x + k * blockDim.x;
        if (i < ns) {
            const int64_t node = nd[k] & ~kSharedBit;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                __pipeline_memcpy_async(&s.node[node_index(s, i, d)], &p.coords[3 * node + d], sizeof(double));
                __pipeline_memcpy_async(&s.node[node_index(s, i, 3 + d)], &field[3 * node + d], sizeof(double));
            }
            s.id[i] = nd[k];
        }
    }
    for (int i = threadIdx.x; i <= ns; i += blockDim.x)
        __pipeline_memcpy_async(&s.off[i], &A.inc_off[s0 + b + i], sizeof(uint32_t));
    // 4 * kTetBlockCells uint16 = kTetBlockCells / 2 chunks of 16 bytes
    for (int i = threadIdx.x; i < kTetBlockCells / 2; i += blockDim.x)
        __pipeline_memcpy_async(&s.inc[8 * i], &A.inc[b * 4 * kTetBlockCells + 8 * i], 16);
}

PL_D void load_slot_ids(const BlockArrays& A, int64_t b, uint32_t nd[kMaxSlotsPerThread]) {
    if (b >= A.nblocks) return;
    const int s0 = A.slot_begin[b];
    const int ns = A.slot_begin[b + 1] - s0;
#pragma unroll
    for (int k = 0; k < kMaxSlotsPerThread; ++k) {
        const int i = threadIdx.x + k * blockDim.x;
        nd[k] = i < ns ? A.slot_node[s0 + i] : 0u;
    }
}

#ifndef PLB_PREFETCH_CELLS
#define PLB_PREFETCH_CELLS 1
#endif

PL_D void prefetch_l2(const void* ptr) { asm volatile("prefetch.global.L2 [%0];" ::"l"(ptr)); }

#ifndef PLB_TET_MIN_BLOCKS
#define PLB_TET_MIN_BLOCKS 4
#endif

// Element vector of one cell (block slot `slot`) into the staging array sE.
template <int RHEO, bool BF, int OP>
PL_D void tet_cell_element(const DomainParams& p, const int* aoff, const double* a, ushort4 lc, const SmemBuf& S,
                           double* sE, int slot) {
    using L = AuxLayout<RHEO, BF>;
    const int ln[4] = {lc.x, lc.y, lc.z, lc.w};
    double X[4][3], U[4][3];
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            X[k][d] = S.node[node_index(S, ln[k], d)];
            U[k][d] = S.node[node_index(S, ln[k], 3 + d)];
        }
    double cof[3][3];
    const double det = tet_cofactors(X, cof);
    if (!(det > 0.0)) flag_error(p.err, CHECK_NONPOSITIVE_DETJ);
    const double rdet = 1.0 / det;
    // G[c][k] = u_{k+1}[c] - u_0[c]; s_x = G cof / det
    double Gm[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) Gm[cc][k] = U[k + 1][cc] - U[0][cc];
    double s_x[9];
#pragma unroll
    for (int cc = 0; cc < 3; ++cc)
#pragma unroll
        for (int d = 0; d < 3; ++d)
            s_x[cc * 3 + d] = (Gm[cc][0] * cof[0][d] + Gm[cc][1] * cof[1][d] + Gm[cc][2] * cof[2][d]) * rdet;
    double x[3] = {0, 0, 0}, s[3] = {0, 0, 0};
    double f0[3] = {0, 0, 0}, f1[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (OP == OP_RESIDUAL) {
        if (BF) {
            const int sOff[1] = {0}, sOff_x[1] = {0};
            pw::g0v_bodyforce<double>(3, 1, L::numA, sOff, sOff_x, s, nullptr, s_x, aoff, nullptr, a, nullptr,
                                      nullptr, p.t, x, p.num_constants, p.constants, f0);
        }
        call_f1<RHEO>(L::numA, aoff, a, s, s_x, p, x, f1);
    } else {
        double Jf3[81];
#pragma unroll
        for (int i = 0; i < 81; ++i) Jf3[i] = 0.0;
        call_jf3<RHEO>(L::numA, aoff, a, p, x, Jf3);
        isotropic_jf3_contract<RHEO>(Jf3, s_x, f1);
    }
    // corners 1..3: |J|/6 * f1 . grad(phi_a) = f1 . cof_{a-1} / 6; corner 0: minus their sum,
    // plus the body-force term |J|/6 * f0 / 4 at every corner.
    const double sixth = 1.0 / 6.0;
    const double bfw = BF && OP == OP_RESIDUAL ? det * sixth * 0.25 : 0.0;
    double e0[3] = {0, 0, 0};
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
            const double v = (f1[cc * 3 + 0] * cof[k][0] + f1[cc * 3 + 1] * cof[k][1] + f1[cc * 3 + 2] * cof[k][2]) * sixth;
            e0[cc] -= v;
            sE[((k + 1) * 3 + cc) * kTetBlockCells + slot] = v + bfw * f0[cc];
        }
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) sE[cc * kTetBlockCells + slot] = e0[cc] + bfw * f0[cc];
}

// DET: a shared node's block sum goes to the partial-sum buffer for the fixup pass (bit-identical
// results run to run); otherwise it is added into the output with an FP64 reduction (the output
// was zeroed first for INSERT).
template <int RHEO, bool BF, int OP, bool INSERT, bool DET>
__global__ void __launch_bounds__(kTetThreads, PLB_TET_MIN_BLOCKS) k_tet_blocked(DomainParams p, BlockArrays A) {
    using L = AuxLayout<RHEO, BF>;
    extern __shared__ __align__(16) char smem_raw[];
    const AuxOffsets<RHEO, BF> aoff;
    const double* __restrict__ field = OP == OP_RESIDUAL ? p.u : p.v;
    double* sE = reinterpret_cast<double*>(smem_raw);  // [12][kTetBlockCells]
    char* bufbase = smem_raw + 12 * kTetBlockCells * sizeof(double);
    const size_t bb = buf_bytes(A.max_local_nodes);
    const int64_t G = gridDim.x;
    int64_t b = blockIdx.x;
    uint32_t nd_next[kMaxSlotsPerThread] = {};
    {
        uint32_t nd0[kMaxSlotsPerThread] = {};
        load_slot_ids(A, b, nd0);
        if (b < A.nblocks) prefetch_block(p, field, A, b, nd0, make_buf(bufbase, A.max_local_nodes));
        __pipeline_commit();
        load_slot_ids(A, b + G, nd_next);
    }
    int cur = 0;
    for (; b < A.nblocks; b += G) {
        const int s0 = A.slot_begin[b];
        const int ns = A.slot_begin[b + 1] - s0;
        const int tc = threadIdx.x;
        // per-cell inputs and the slot ids two blocks ahead: issued before the wait
        ushort4 lc[kTetCellsPerThread];
        double a[kTetCellsPerThread][L::size];
        const int64_t cb0 = A.cell_begin[b], cb1 = A.cell_begin[b + 1];
#pragma unroll
        for (int j = 0; j < kTetCellsPerThread; ++j) {
            const int64_t c = cb0 + tc + j * kTetThreads;
            lc[j] = make_ushort4(0, 0, 0, 0);
            if (c < cb1) {
                lc[j] = A.lconn[c];
                L::load_cell(p, c, a[j]);
            }
        }
        uint32_t nd_after[kMaxSlotsPerThread] = {};
        load_slot_ids(A, b + 2 * G, nd_after);
        __pipeline_wait_prior(0);
        __syncthreads();
        if (b + G < A.nblocks) {
            prefetch_block(p, field, A, b + G, nd_next, make_buf(bufbase + (cur ^ 1) * bb, A.max_local_nodes));
#if PLB_PREFETCH_CELLS
            // the next block's per-cell inputs, streamed once: start their trip to L2 now
#pragma unroll
            for (int j = 0; j < kTetCellsPerThread; ++j) {
                const int64_t cn = A.cell_begin[b + G] + tc + j * kTetThreads;
                if (cn < A.cell_begin[b + G + 1]) {
                    prefetch_l2(&A.lconn[cn]);
                    prefetch_l2(&p.mu[cn]);
                    prefetch_l2(&p.K[cn]);
                    if (BF)
#pragma unroll
                        for (int d = 0; d < 3; ++d) prefetch_l2(&p.body_force[d * p.ncells + cn]);
                }
            }
#endif
        }
        __pipeline_commit();
#pragma unroll
        for (int k = 0; k < kMaxSlotsPerThread; ++k) nd_next[k] = nd_after[k];
        const SmemBuf S = make_buf(bufbase + cur * bb, A.max_local_nodes);
#pragma unroll
        for (int j = 0; j < kTetCellsPerThread; ++j)
            if (cb0 + tc + j * kTetThreads < cb1)
                tet_cell_element<RHEO, BF, OP>(p, aoff.v, a[j], lc[j], S, sE, tc + j * kTetThreads);
        __syncthreads();
        for (int i = threadIdx.x; i < ns; i += blockDim.x) {
            const int j0 = S.off[i], j1 = S.off[i + 1];
            double r0 = 0.0, r1 = 0.0, r2 = 0.0;
#pragma unroll 4
            for (int j = j0; j < j1; ++j) {
                const int e = S.inc[j];
                const int cell = e >> 2, corner = e & 3;
                r0 += sE[(corner * 3 + 0) * kTetBlockCells + cell];
                r1 += sE[(corner * 3 + 1) * kTetBlockCells + cell];
                r2 += sE[(corner * 3 + 2) * kTetBlockCells + cell];
            }
            const uint32_t id = S.id[i];
            double* o = p.out + 3 * (int64_t)(id & ~kSharedBit);
            if ((id & kSharedBit) && DET) {
                // this block's part of a shared node: summed over blocks by the fixup pass
                double* pp = A.partial + 3 * (int64_t)(s0 + i);
                pp[0] = r0;
                pp[1] = r1;
                pp[2] = r2;
            } else if (id & kSharedBit) {
                red_add(o, r0);
                red_add(o + 1, r1);
                red_add(o + 2, r2);
            } else if (INSERT) {
                o[0] = r0;
                o[1] = r1;
                o[2] = r2;
            } else {
                o[0] += r0;
                o[1] += r1;
                o[2] += r2;
            }
        }
        // No barrier here: the next iteration writes shared memory (sE, and the prefetch into
        // this block's buffer) only after its own barrier, which every thread reaches after
        // finishing this gather.
        cur ^= 1;
    }
    __pipeline_wait_prior(0);
}

// ---- cell-block kernels over the padded layout ---------------------------------------------------
// The same cell blocks, staged from padded per-block arrays (built with the layout): per block the
// CTA copies, one block ahead, its coordinates, node ids, incidence offsets and incidence list as
// 16-byte cp.async runs, and gathers the input field of its nodes with 8-byte cp.async; the
// incidence list holds staging offsets (corner * 3 * cells + cell), so the node sums do no index
// arithmetic. Two schedules:
//  * PIPE: one barrier per block: iteration i computes the element vectors of block b_i into one
//    staging buffer while the node sums of block b_{i-1} read the other (element vectors x2, node
//    data x2, block metadata x3; 3 CTAs per SM);
//  * two barriers per block (element vectors, then node sums of the same block; element vectors
//    x1, node data x2, metadata x2; 4 CTAs per SM).
#ifndef PLB_PIPE_MIN_BLOCKS
#define PLB_PIPE_MIN_BLOCKS 3
#endif
#ifndef PLB_PAD2_MIN_BLOCKS
#define PLB_PAD2_MIN_BLOCKS 4
#endif

struct PipeArrays {
    const int32_t* cell_begin;  // [nblocks + 1] first cell of each block (at most kTetBlockCells each)
    const int32_t* slot_begin;  // [nblocks + 1] unpadded slots (slot counts, deterministic partials)
    const int32_t* pbeg;        // [nblocks + 1] padded slot starts (multiples of 4)
    const uint32_t* ids;        // per padded slot: node id | kSharedBit
    const double* coords;       // per block [3][padded slots]
    const uint32_t* off;        // per block at pbeg[b] + 4 b: ns + 1 incidence offsets
    const uint16_t* inc;        // [nblocks][4 * kTetBlockCells] staging offsets
    const ushort4* lconn;       // [ncells] block-local slots of the 4 corners
    double* partial;            // [slots][3] deterministic partial sums (unpadded slot index)
    int64_t nblocks;
    int ld;                     // padded slots of the largest block (multiple of 4)
};

PL_HD size_t pipe_meta_bytes(int ld) {
    return round16(4 * (size_t)ld) + round16(4 * ((size_t)ld + 4)) + round16(2 * 4 * (size_t)kTetBlockCells);
}

PL_HD size_t pipe_smem_bytes(int ld) {
    return 2 * 12 * (size_t)kTetBlockCells * sizeof(double) + 2 * 6 * (size_t)ld * sizeof(double) + 3 * pipe_meta_bytes(ld);
}

PL_HD size_t pad2_smem_bytes(int ld) {
    return 12 * (size_t)kTetBlockCells * sizeof(double) + 2 * 6 * (size_t)ld * sizeof(double) + 2 * pipe_meta_bytes(ld);
}

struct PipeMeta {
    uint32_t* ids;
    uint32_t* off;
    uint16_t* inc;
};

PL_D PipeMeta pipe_meta(char* base, int ld) {
    PipeMeta m;
    m.ids = reinterpret_cast<uint32_t*>(base);
    base += round16(4 * (size_t)ld);
    m.off = reinterpret_cast<uint32_t*>(base);
    base += round16(4 * ((size_t)ld + 4));
    m.inc = reinterpret_cast<uint16_t*>(base);
    return m;
}

PL_D void pipe_load_ids(const PipeArrays& A, int64_t b, uint32_t nd[kMaxSlotsPerThread]) {
#pragma unroll
    for (int k = 0; k < kMaxSlotsPerThread; ++k) nd[k] = 0u;
    if (b >= A.nblocks) return;
    const int p0 = A.pbeg[b];
    const int ns = A.slot_begin[b + 1] - A.slot_begin[b];
#pragma unroll
    for (int k = 0; k < kMaxSlotsPerThread; ++k) {
        const int i = threadIdx.x + k * blockDim.x;
        if (i < ns) nd[k] = A.ids[p0 + i];
    }
}

// Asynchronous copies of block b: coordinates, ids, offsets and incidences as aligned 16-byte
// runs, the field of its nodes (ids in nd, read one block earlier) as 8-byte gathers.
PL_D void pipe_stage(const double* __restrict__ field, const PipeArrays& A, int64_t b,
                     const uint32_t nd[kMaxSlotsPerThread], double* node, const PipeMeta& M, int ld) {
    const int p0 = A.pbeg[b];
    const int np = A.pbeg[b + 1] - p0;
    const int ns = A.slot_begin[b + 1] - A.slot_begin[b];
    const int half = np >> 1;  // 16-byte chunks per coordinate component
    for (int t = threadIdx.x; t < 3 * half; t += blockDim.x) {
        const int d = t / half, j = t - d * half;
        __pipeline_memcpy_async(&node[d * ld + 2 * j], &A.coords[3 * (int64_t)p0 + (int64_t)d * np + 2 * j], 16);
    }
#pragma unroll
    for (int k = 0; k < kMaxSlotsPerThread; ++k) {
        const int i = threadIdx.x + k * blockDim.x;
        if (i < ns) {
            const int64_t n = nd[k] & ~kSharedBit;
#pragma unroll
            for (int d = 0; d < 3; ++d) __pipeline_memcpy_async(&node[(3 + d) * ld + i], &field[3 * n + d], sizeof(double));
        }
    }
    const int q = np >> 2;  // 16-byte chunks of ids; offsets take one more
    for (int t = threadIdx.x; t < q; t += blockDim.x) __pipeline_memcpy_async(&M.ids[4 * t], &A.ids[p0 + 4 * t], 16);
    for (int t = threadIdx.x; t <= q; t += blockDim.x)
        __pipeline_memcpy_async(&M.off[4 * t], &A.off[(int64_t)p0 + 4 * b + 4 * t], 16);
    for (int t = threadIdx.x; t < kTetBlockCells / 2; t += blockDim.x)
        __pipeline_memcpy_async(&M.inc[8 * t], &A.inc[b * 4 * kTetBlockCells + 8 * t], 16);
}

// Node sums of block b (element vectors in sE, metadata in M): one thread per node.
template <bool INSERT, bool DET>
PL_D void pipe_node_sums(const DomainParams& p, const PipeArrays& A, int64_t b, const double* sE, const PipeMeta& M) {
    const int s0 = A.slot_begin[b];
    const int ns = A.slot_begin[b + 1] - s0;
    for (int k = threadIdx.x; k < ns; k += blockDim.x) {
        const int j0 = M.off[k], j1 = M.off[k + 1];
        double r0 = 0.0, r1 = 0.0, r2 = 0.0;
#pragma unroll 4
        for (int j = j0; j < j1; ++j) {
            const int e = M.inc[j];
            r0 += sE[e];
            r1 += sE[e + kTetBlockCells];
            r2 += sE[e + 2 * kTetBlockCells];
        }
        const uint32_t id = M.ids[k];
        double* o = p.out + 3 * (int64_t)(id & ~kSharedBit);
        if ((id & kSharedBit) && DET) {
            double* pp = A.partial + 3 * (int64_t)(s0 + k);
            pp[0] = r0;
            pp[1] = r1;
            pp[2] = r2;
        } else if (id & kSharedBit) {
            red_add(o, r0);
            red_add(o + 1, r1);
            red_add(o + 2, r2);
        } else if (INSERT) {
            o[0] = r0;
            o[1] = r1;
            o[2] = r2;
        } else {
            o[0] += r0;
            o[1] += r1;
            o[2] += r2;
        }
    }
}

template <int RHEO, bool BF, int OP, bool INSERT, bool DET>
__global__ void __launch_bounds__(kTetBlockCells, PLB_PIPE_MIN_BLOCKS) k_tet_pipe(DomainParams p, PipeArrays A) {
    using L = AuxLayout<RHEO, BF>;
    extern __shared__ __align__(16) char smem_raw[];
    const AuxOffsets<RHEO, BF> aoff;
    const double* __restrict__ field = OP == OP_RESIDUAL ? p.u : p.v;
    const int ld = A.ld;
    double* sEb = reinterpret_cast<double*>(smem_raw);            // [2][12][kTetBlockCells]
    double* nodeb = sEb + 2 * 12 * kTetBlockCells;                // [2][6][ld]
    char* metab = reinterpret_cast<char*>(nodeb + 2 * 6 * ld);   // [3][pipe_meta_bytes]
    const size_t mb = pipe_meta_bytes(ld);
    const int64_t G = gridDim.x;
    const int tc = threadIdx.x;
    int64_t b = blockIdx.x;
    if (b >= A.nblocks) return;
    uint32_t nd_next[kMaxSlotsPerThread];
    {
        uint32_t nd0[kMaxSlotsPerThread];
        pipe_load_ids(A, b, nd0);
        pipe_stage(field, A, b, nd0, nodeb, pipe_meta(metab, ld), ld);
        __pipeline_commit();
        pipe_load_ids(A, b + G, nd_next);
    }
    int it = 0;
    int64_t bprev = -1;
    for (; b < A.nblocks; b += G, ++it) {
        // this block's per-cell inputs and the slot ids two blocks ahead: issued before the wait
        const int64_t c = A.cell_begin[b] + tc;
        const bool live = c < A.cell_begin[b + 1];
        ushort4 lc = make_ushort4(0, 0, 0, 0);
        double a[L::size];
        if (live) {
            lc = A.lconn[c];
            L::load_cell(p, c, a);
        }
        uint32_t nd_after[kMaxSlotsPerThread];
        pipe_load_ids(A, b + 2 * G, nd_after);
        __pipeline_wait_prior(0);
        // block b's copies have landed, and every thread has finished iteration it - 1 (its
        // element vectors are complete; the buffers staged below are no longer read)
        __syncthreads();
        if (b + G < A.nblocks) {
            pipe_stage(field, A, b + G, nd_next, nodeb + ((it + 1) & 1) * 6 * ld, pipe_meta(metab + ((it + 1) % 3) * mb, ld), ld);
            const int64_t cn = A.cell_begin[b + G] + tc;
            if (cn < A.cell_begin[b + G + 1]) {
                prefetch_l2(&A.lconn[cn]);
                prefetch_l2(&p.mu[cn]);
                prefetch_l2(&p.K[cn]);
                if (BF)
#pragma unroll
                    for (int d = 0; d < 3; ++d) prefetch_l2(&p.body_force[d * p.ncells + cn]);
            }
        }
        __pipeline_commit();
#pragma unroll
        for (int k = 0; k < kMaxSlotsPerThread; ++k) nd_next[k] = nd_after[k];
        SmemBuf S;
        S.node = nodeb + (it & 1) * 6 * ld;
        S.ld = ld;
        double* sE = sEb + (it & 1) * 12 * kTetBlockCells;
        if (live) tet_cell_element<RHEO, BF, OP>(p, aoff.v, a, lc, S, sE, tc);
        if (bprev >= 0)
            pipe_node_sums<INSERT, DET>(p, A, bprev, sEb + ((it + 1) & 1) * 12 * kTetBlockCells,
                                        pipe_meta(metab + ((it + 2) % 3) * mb, ld));
        bprev = b;
    }
    __syncthreads();
    pipe_node_sums<INSERT, DET>(p, A, bprev, sEb + ((it + 1) & 1) * 12 * kTetBlockCells,
                                pipe_meta(metab + ((it + 2) % 3) * mb, ld));
    __pipeline_wait_prior(0);
}

template <int RHEO, bool BF, int OP, bool INSERT, bool DET>
__global__ void __launch_bounds__(kTetBlockCells, PLB_PAD2_MIN_BLOCKS) k_tet_pad2(DomainParams p, PipeArrays A) {
    using L = AuxLayout<RHEO, BF>;
    extern __shared__ __align__(16) char smem_raw[];
    const AuxOffsets<RHEO, BF> aoff;
    const double* __restrict__ field = OP == OP_RESIDUAL ? p.u : p.v;
    const int ld = A.ld;
    double* sE = reinterpret_cast<double*>(smem_raw);             // [12][kTetBlockCells]
    double* nodeb = sE + 12 * kTetBlockCells;                      // [2][6][ld]
    char* metab = reinterpret_cast<char*>(nodeb + 2 * 6 * ld);    // [2][pipe_meta_bytes]
    const size_t mb = pipe_meta_bytes(ld);
    const int64_t G = gridDim.x;
    const int tc = threadIdx.x;
    int64_t b = blockIdx.x;
    if (b >= A.nblocks) return;
    uint32_t nd_next[kMaxSlotsPerThread];
    {
        uint32_t nd0[kMaxSlotsPerThread];
        pipe_load_ids(A, b, nd0);
        pipe_stage(field, A, b, nd0, nodeb, pipe_meta(metab, ld), ld);
        __pipeline_commit();
        pipe_load_ids(A, b + G, nd_next);
    }
    for (int it = 0; b < A.nblocks; b += G, ++it) {
        const int64_t c = A.cell_begin[b] + tc;
        const bool live = c < A.cell_begin[b + 1];
        ushort4 lc = make_ushort4(0, 0, 0, 0);
        double a[L::size];
        if (live) {
            lc = A.lconn[c];
            L::load_cell(p, c, a);
        }
        uint32_t nd_after[kMaxSlotsPerThread];
        pipe_load_ids(A, b + 2 * G, nd_after);
        __pipeline_wait_prior(0);
        // block b's copies have landed; every thread has finished the node sums of the previous
        // block (its buffers are free for block b + G)
        __syncthreads();
        if (b + G < A.nblocks) {
            pipe_stage(field, A, b + G, nd_next, nodeb + ((it + 1) & 1) * 6 * ld, pipe_meta(metab + ((it + 1) & 1) * mb, ld), ld);
            const int64_t cn = A.cell_begin[b + G] + tc;
            if (cn < A.cell_begin[b + G + 1]) {
                prefetch_l2(&A.lconn[cn]);
                prefetch_l2(&p.mu[cn]);
                prefetch_l2(&p.K[cn]);
                if (BF)
#pragma unroll
                    for (int d = 0; d < 3; ++d) prefetch_l2(&p.body_force[d * p.ncells + cn]);
            }
        }
        __pipeline_commit();
#pragma unroll
        for (int k = 0; k < kMaxSlotsPerThread; ++k) nd_next[k] = nd_after[k];
        SmemBuf S;
        S.node = nodeb + (it & 1) * 6 * ld;
        S.ld = ld;
        if (live) tet_cell_element<RHEO, BF, OP>(p, aoff.v, a, lc, S, sE, tc);
        __syncthreads();
        pipe_node_sums<INSERT, DET>(p, A, b, sE, pipe_meta(metab + (it & 1) * mb, ld));
    }
    __pipeline_wait_prior(0);
}

// ---- FP32 Jacobian action over the padded layout ---------------------------------------------
// Shared memory of k_tet_pad_jv32: element vectors (FP32) [12][kTetBlockCells], then two node
// buffers of [3][ld] FP64 coordinates and [3][ld] FP32 field values, then two metadata buffers.
PL_HD size_t padjv_node_bytes(int ld) { return round16(3 * (size_t)ld * sizeof(double) + 3 * (size_t)ld * sizeof(float)); }

PL_HD size_t padjv_smem_bytes(int ld) {
    return 12 * (size_t)kTetBlockCells * sizeof(float) + 2 * padjv_node_bytes(ld) + 2 * pipe_meta_bytes(ld);
}

// Asynchronous copies of block b for k_tet_pad_jv32: coordinates, ids, offsets and incidences as
// 16-byte runs (as pipe_stage), the FP32 field of its nodes as 4-byte gathers.
PL_D void padjv_stage(const float* __restrict__ v32, const PipeArrays& A, int64_t b,
                      const uint32_t nd[kMaxSlotsPerThread], char* buf, const PipeMeta& M, int ld) {
    double* X = reinterpret_cast<double*>(buf);
    float* V = reinterpret_cast<float*>(buf + 3 * (size_t)ld * sizeof(double));
    const int p0 = A.pbeg[b];
    const int np = A.pbeg[b + 1] - p0;
    const int ns = A.slot_begin[b + 1] - A.slot_begin[b];
    const int half = np >> 1;
    for (int t = threadIdx.x; t < 3 * half; t += blockDim.x) {
        const int d = t / half, j = t - d * half;
        __pipeline_memcpy_async(&X[d * ld + 2 * j], &A.coords[3 * (int64_t)p0 + (int64_t)d * np + 2 * j], 16);
    }
#pragma unroll
    for (int k = 0; k < kMaxSlotsPerThread; ++k) {
        const int i = threadIdx.x + k * blockDim.x;
        if (i < ns) {
            const int64_t n = nd[k] & ~kSharedBit;
#pragma unroll
            for (int d = 0; d < 3; ++d) __pipeline_memcpy_async(&V[d * ld + i], &v32[3 * n + d], sizeof(float));
        }
    }
    const int q = np >> 2;
    for (int t = threadIdx.x; t < q; t += blockDim.x) __pipeline_memcpy_async(&M.ids[4 * t], &A.ids[p0 + 4 * t], 16);
    for (int t = threadIdx.x; t <= q; t += blockDim.x)
        __pipeline_memcpy_async(&M.off[4 * t], &A.off[(int64_t)p0 + 4 * b + 4 * t], 16);
    for (int t = threadIdx.x; t < kTetBlockCells / 2; t += blockDim.x)
        __pipeline_memcpy_async(&M.inc[8 * t], &A.inc[b * 4 * kTetBlockCells + 8 * t], 16);
}

// One cell of the FP32 Jacobian action over the padded layout: FP64 geometry (cofactors, 1/det)
// from the staged coordinates X [3][ld], gradient and flux of the FP32 field V [3][ld] with the
// isotropic tangent (lam, mu), and the element vector into column tc of sE [12][kTetBlockCells].
PL_D void padjv_cell(const DomainParams& p, ushort4 lc, float lam, float mu, const double* X, const float* V, int ld,
                     float* sE, int tc) {
    const int ln[4] = {lc.x, lc.y, lc.z, lc.w};
    double Xc[4][3];
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int d = 0; d < 3; ++d) Xc[k][d] = X[d * ld + ln[k]];
    double cof[3][3];
    const double det = tet_cofactors(Xc, cof);
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
    float s[3][3];
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) {
        const float v0 = V[cc * ld + ln[0]];
        const float g0 = V[cc * ld + ln[1]] - v0, g1 = V[cc * ld + ln[2]] - v0, g2 = V[cc * ld + ln[3]] - v0;
#pragma unroll
        for (int d = 0; d < 3; ++d) s[cc][d] = g0 * inv[0][d] + g1 * inv[1][d] + g2 * inv[2][d];
    }
    // flux f1 = -(lambda tr(e) I + 2 mu e), e = sym grad v
    const float ltr = lam * (s[0][0] + s[1][1] + s[2][2]);
    const float xy = -mu * (s[0][1] + s[1][0]), yz = -mu * (s[1][2] + s[2][1]), xz = -mu * (s[0][2] + s[2][0]);
    const float f[3][3] = {{-(2.0f * mu * s[0][0] + ltr), xy, xz},
                           {xy, -(2.0f * mu * s[1][1] + ltr), yz},
                           {xz, yz, -(2.0f * mu * s[2][2] + ltr)}};
    float e0[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
            const float v = f[cc][0] * cf[k][0] + f[cc][1] * cf[k][1] + f[cc][2] * cf[k][2];
            e0[cc] -= v;
            sE[((k + 1) * 3 + cc) * kTetBlockCells + tc] = v;
        }
#pragma unroll
    for (int cc = 0; cc < 3; ++cc) sE[cc * kTetBlockCells + tc] = e0[cc];
}

// Node sums of block b from its element vectors sE and metadata M: owned nodes added, shared
// nodes reduced into p.out32.
PL_D void padjv_node_sums(const DomainParams& p, const PipeArrays& A, int64_t b, const float* sE, const PipeMeta& M) {
    const int ns = A.slot_begin[b + 1] - A.slot_begin[b];
    for (int k = threadIdx.x; k < ns; k += blockDim.x) {
        const int j0 = M.off[k], j1 = M.off[k + 1];
        float r0 = 0.f, r1 = 0.f, r2 = 0.f;
#pragma unroll 4
        for (int j = j0; j < j1; ++j) {
            const int e = M.inc[j];
            r0 += sE[e];
            r1 += sE[e + kTetBlockCells];
            r2 += sE[e + 2 * kTetBlockCells];
        }
        const uint32_t id = M.ids[k];
        float* o = p.out32 + 3 * (int64_t)(id & ~kSharedBit);
        if (id & kSharedBit) {
            red_add(o, r0);
            red_add(o + 1, r1);
            red_add(o + 2, r2);
        } else {
            o[0] += r0;
            o[1] += r1;
            o[2] += r2;
        }
    }
}

// FP32 Jacobian action of an isotropic tangent on the padded cell-block layout, in the shape of
// k_tet_pad2: block b + G is staged with cp.async while block b is computed, geometry (cofactors,
// 1/det) in FP64 per cell, field, gradient, flux, element vectors and node sums in FP32. The
// tangent's (lambda, mu) per cell come from the solver's cache (p.lm32; CACHED) or from the
// registered Jacobian kernel. The output holds zero (INSERT) or the sum to add to: owned nodes are
// added, shared ones reduced.
template <bool CACHED>
__global__ void __launch_bounds__(kTetBlockCells, 4) k_tet_pad_jv32(DomainParams p, PipeArrays A) {
    using L = AuxLayout<RHEO_ILE, false>;
    extern __shared__ __align__(16) char smem_raw[];
    const AuxOffsets<RHEO_ILE, false> aoff;
    const int ld = A.ld;
    float* sE = reinterpret_cast<float*>(smem_raw);  // [12][kTetBlockCells]
    char* nodeb = smem_raw + 12 * kTetBlockCells * sizeof(float);
    const size_t nbytes = padjv_node_bytes(ld);
    char* metab = nodeb + 2 * nbytes;
    const size_t mb = pipe_meta_bytes(ld);
    const int64_t G = gridDim.x;
    const int tc = threadIdx.x;
    int64_t b = blockIdx.x;
    if (b >= A.nblocks) return;
    uint32_t nd_next[kMaxSlotsPerThread];
    {
        uint32_t nd0[kMaxSlotsPerThread];
        pipe_load_ids(A, b, nd0);
        padjv_stage(p.v32, A, b, nd0, nodeb, pipe_meta(metab, ld), ld);
        __pipeline_commit();
        pipe_load_ids(A, b + G, nd_next);
    }
    for (int it = 0; b < A.nblocks; b += G, ++it) {
        const int64_t c = A.cell_begin[b] + tc;
        const bool live = c < A.cell_begin[b + 1];
        ushort4 lc = make_ushort4(0, 0, 0, 0);
        float lam = 0.f, mu = 0.f;
        if (live) {
            lc = A.lconn[c];
            if (CACHED) {
                const float2 lm = reinterpret_cast<const float2*>(p.lm32)[c];
                lam = lm.x;
                mu = lm.y;
            } else {
                double a[L::size];
                L::load_cell(p, c, a);
                double x[3] = {0, 0, 0}, Jf3[81];
#pragma unroll
                for (int i = 0; i < 81; ++i) Jf3[i] = 0.0;
                call_jf3<RHEO_ILE>(L::numA, aoff.v, a, p, x, Jf3);
                lam = (float)(-Jf3[((0 * 3 + 1) * 3 + 0) * 3 + 1]);
                mu = (float)(-Jf3[((0 * 3 + 1) * 3 + 1) * 3 + 0]);
            }
        }
        uint32_t nd_after[kMaxSlotsPerThread];
        pipe_load_ids(A, b + 2 * G, nd_after);
        __pipeline_wait_prior(0);
        // block b's copies have landed; every thread has finished the node sums of the previous
        // block (its buffers are free for block b + G)
        __syncthreads();
        if (b + G < A.nblocks) {
            padjv_stage(p.v32, A, b + G, nd_next, nodeb + ((it + 1) & 1) * nbytes, pipe_meta(metab + ((it + 1) & 1) * mb, ld),
                        ld);
            const int64_t cn = A.cell_begin[b + G] + tc;
            if (cn < A.cell_begin[b + G + 1]) {
                prefetch_l2(&A.lconn[cn]);
                if (CACHED) prefetch_l2(&p.lm32[2 * cn]);
            }
        }
        __pipeline_commit();
#pragma unroll
        for (int k = 0; k < kMaxSlotsPerThread; ++k) nd_next[k] = nd_after[k];
        const double* X = reinterpret_cast<const double*>(nodeb + (it & 1) * nbytes);
        const float* V = reinterpret_cast<const float*>(nodeb + (it & 1) * nbytes + 3 * (size_t)ld * sizeof(double));
        if (live) padjv_cell(p, lc, lam, mu, X, V, ld, sE, tc);
        __syncthreads();
        padjv_node_sums(p, A, b, sE, pipe_meta(metab + (it & 1) * mb, ld));
    }
    __pipeline_wait_prior(0);
}


// FP32 Jacobian action of isotropic linear elasticity on the cell blocks: geometry (cofactors,
// 1/det) and the elastic tangent in FP64 per cell, the field, gradient, flux and element vectors
// in FP32. Used by the inner iterations of the mixed-precision solver.
__global__ void __launch_bounds__(kTetBlockCells, 4) k_tet_blocked_jv32(DomainParams p, BlockArrays A) {
    using L = AuxLayout<RHEO_ILE, false>;
    extern __shared__ __align__(16) char smem_raw[];
    const AuxOffsets<RHEO_ILE, false> aoff;
    float* sE = reinterpret_cast<float*>(smem_raw);                                          // [12][kTetBlockCells]
    double* sX = reinterpret_cast<double*>(smem_raw + 12 * kTetBlockCells * sizeof(float));  // [ns][3]
    for (int64_t b = blockIdx.x; b < A.nblocks; b += gridDim.x) {
        const int s0 = A.slot_begin[b];
        const int ns = A.slot_begin[b + 1] - s0;
        float* sV = reinterpret_cast<float*>(sX + 3 * ns);  // [ns][3] field
        for (int i = threadIdx.x; i < ns; i += blockDim.x) {
            const int64_t nd = A.slot_node[s0 + i] & ~kSharedBit;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                sX[3 * i + d] = p.coords[3 * nd + d];
                sV[3 * i + d] = p.v32[3 * nd + d];
            }
        }
        __syncthreads();
        const int tc = threadIdx.x;
        const int64_t c = A.cell_begin[b] + tc;
        if (c < A.cell_begin[b + 1]) {
            const ushort4 lc = A.lconn[c];
            const int ln[4] = {lc.x, lc.y, lc.z, lc.w};
            double X[4][3];
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int d = 0; d < 3; ++d) X[k][d] = sX[3 * ln[k] + d];
            double cof[3][3];
            const double det = tet_cofactors(X, cof);
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
            float s_x[9];
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
                const float g0 = sV[3 * ln[1] + cc] - sV[3 * ln[0] + cc];
                const float g1 = sV[3 * ln[2] + cc] - sV[3 * ln[0] + cc];
                const float g2 = sV[3 * ln[3] + cc] - sV[3 * ln[0] + cc];
#pragma unroll
                for (int d = 0; d < 3; ++d) s_x[cc * 3 + d] = g0 * inv[0][d] + g1 * inv[1][d] + g2 * inv[2][d];
            }
            float f1[9];
            isotropic_jf3_contract<RHEO_ILE>(Jf3d, s_x, f1);
            float e0[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) {
                    const float v = f1[cc * 3 + 0] * cf[k][0] + f1[cc * 3 + 1] * cf[k][1] + f1[cc * 3 + 2] * cf[k][2];
                    e0[cc] -= v;
                    sE[((k + 1) * 3 + cc) * kTetBlockCells + tc] = v;
                }
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) sE[cc * kTetBlockCells + tc] = e0[cc];
        }
        __syncthreads();
        for (int i = threadIdx.x; i < ns; i += blockDim.x) {
            const int j0 = A.inc_off[s0 + b + i], j1 = A.inc_off[s0 + b + i + 1];
            const uint16_t* lst = A.inc + b * 4 * kTetBlockCells;
            float r0 = 0.f, r1 = 0.f, r2 = 0.f;
            for (int j = j0; j < j1; ++j) {
                const int e = lst[j];
                const int cell = e >> 2, corner = e & 3;
                r0 += sE[(corner * 3 + 0) * kTetBlockCells + cell];
                r1 += sE[(corner * 3 + 1) * kTetBlockCells + cell];
                r2 += sE[(corner * 3 + 2) * kTetBlockCells + cell];
            }
            const uint32_t id = A.slot_node[s0 + i];
            float* o = p.out32 + 3 * (int64_t)(id & ~kSharedBit);
            if (id & kSharedBit) {
                red_add(o, r0);
                red_add(o + 1, r1);
                red_add(o + 2, r2);
            } else {
                o[0] += r0;
                o[1] += r1;
                o[2] += r2;
            }
        }
        __syncthreads();
    }
}

// Second pass of the FP64 cell-block kernels: every node that is not owned by exactly one block
// gets the sum of its blocks' partial sums, in block order (nodes in no cell get zero).
template <bool INSERT>
__global__ void k_blocked_fixup(double* __restrict__ out, const double* __restrict__ partial,
                                const int32_t* __restrict__ fix_node, const int32_t* __restrict__ fix_off,
                                const int32_t* __restrict__ fix_slot, int64_t nfix) {
    for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < nfix; f += (int64_t)gridDim.x * blockDim.x) {
        double r0 = 0.0, r1 = 0.0, r2 = 0.0;
        for (int j = fix_off[f]; j < fix_off[f + 1]; ++j) {
            const double* pp = partial + 3 * (int64_t)fix_slot[j];
            r0 += pp[0];
            r1 += pp[1];
            r2 += pp[2];
        }
        double* o = out + 3 * (int64_t)fix_node[f];
        if (INSERT) {
            o[0] = r0;
            o[1] = r1;
            o[2] = r2;
        } else {
            o[0] += r0;
            o[1] += r1;
            o[2] += r2;
        }
    }
}

static BlockArrays arrays_of(const BlockedLayout& b, double* partial = nullptr) {
    BlockArrays A;
    A.partial = partial;
    A.cell_begin = b.d_cell_begin;
    A.slot_begin = b.d_block_node_begin;
    A.slot_node = b.d_slot_node;
    A.lconn = (const ushort4*)b.d_local_cells;
    A.inc_off = b.d_inc_off;
    A.inc = b.d_inc;
    A.nblocks = b.num_blocks;
    A.max_local_nodes = b.max_local_nodes;
    return A;
}

static size_t blocked_smem(const BlockedLayout& b) {
    return (size_t)12 * kTetBlockCells * sizeof(double) + 2 * buf_bytes(b.max_local_nodes);
}

static int persistent_grid(int64_t nblocks) { return (int)std::min<int64_t>(nblocks, (int64_t)sm_count() * PLB_TET_MIN_BLOCKS); }

template <int RHEO, bool BF, int OP, bool INSERT, bool DET>
static void launch_one(const DomainParams& p, const BlockArrays& A, size_t smem, int grid, cudaStream_t s) {
    auto kern = k_tet_blocked<RHEO, BF, OP, INSERT, DET>;
    ensure_kernel_smem((const void*)kern, smem);
    kern<<<grid, kTetThreads, smem, s>>>(p, A);
    count_launch();
}

template <int RHEO, bool BF, int OP>
static void launch_t(const DomainParams& p, const BlockedLayout& b, bool insert, double* partial, cudaStream_t s) {
    const size_t smem = blocked_smem(b);
    const int grid = persistent_grid(b.num_blocks);
    const BlockArrays A = arrays_of(b, partial);
    const bool det = partial != nullptr;
    if (insert && det) launch_one<RHEO, BF, OP, true, true>(p, A, smem, grid, s);
    else if (insert) launch_one<RHEO, BF, OP, true, false>(p, A, smem, grid, s);
    else if (det) launch_one<RHEO, BF, OP, false, true>(p, A, smem, grid, s);
    else launch_one<RHEO, BF, OP, false, false>(p, A, smem, grid, s);
    if (det && b.num_fix > 0) {
        const int fg = (int)std::min<int64_t>((b.num_fix + 255) / 256, 148 * 8);
        if (insert) k_blocked_fixup<true><<<fg, 256, 0, s>>>(p.out, partial, b.d_fix_node, b.d_fix_off, b.d_fix_slot, b.num_fix);
        else k_blocked_fixup<false><<<fg, 256, 0, s>>>(p.out, partial, b.d_fix_node, b.d_fix_off, b.d_fix_slot, b.num_fix);
        count_launch();
    }
}

static PipeArrays pipe_arrays_of(const BlockedLayout& b, double* partial, bool reduced = false) {
    PipeArrays A;
    A.cell_begin = b.d_cell_begin;
    A.slot_begin = b.d_block_node_begin;
    A.pbeg = b.d_pipe_begin;
    A.ids = reduced ? b.d_pipe_ids_red : b.d_pipe_ids;
    A.coords = b.d_pipe_coords;
    A.off = b.d_pipe_off;
    A.inc = b.d_pipe_inc;
    A.lconn = (const ushort4*)b.d_local_cells;
    A.partial = partial;
    A.nblocks = b.num_blocks;
    A.ld = (b.max_local_nodes + 3) & ~3;
    return A;
}

template <bool PIPE, int RHEO, bool BF, int OP, bool INSERT, bool DET>
static void launch_pipe_one(const DomainParams& p, const PipeArrays& A, size_t smem, int grid, cudaStream_t s) {
    auto kern = PIPE ? k_tet_pipe<RHEO, BF, OP, INSERT, DET> : k_tet_pad2<RHEO, BF, OP, INSERT, DET>;
    ensure_kernel_smem((const void*)kern, smem);
    kern<<<grid, kTetBlockCells, smem, s>>>(p, A);
    count_launch();
}

template <bool PIPE, int RHEO, bool BF, int OP>
static void launch_pipe_t(const DomainParams& p, const BlockedLayout& b, bool insert, double* partial, cudaStream_t s,
                          bool reduced = false) {
    const PipeArrays A = pipe_arrays_of(b, partial, reduced);
    const size_t smem = PIPE ? pipe_smem_bytes(A.ld) : pad2_smem_bytes(A.ld);
    const int grid = (int)std::min<int64_t>(b.num_blocks, (int64_t)sm_count() * (PIPE ? PLB_PIPE_MIN_BLOCKS : PLB_PAD2_MIN_BLOCKS));
    const bool det = partial != nullptr;
    if (insert && det) launch_pipe_one<PIPE, RHEO, BF, OP, true, true>(p, A, smem, grid, s);
    else if (insert) launch_pipe_one<PIPE, RHEO, BF, OP, true, false>(p, A, smem, grid, s);
    else if (det) launch_pipe_one<PIPE, RHEO, BF, OP, false, true>(p, A, smem, grid, s);
    else launch_pipe_one<PIPE, RHEO, BF, OP, false, false>(p, A, smem, grid, s);
    if (det && b.num_fix > 0) {
        const int fg = (int)std::min<int64_t>((b.num_fix + 255) / 256, 148 * 8);
        if (insert) k_blocked_fixup<true><<<fg, 256, 0, s>>>(p.out, partial, b.d_fix_node, b.d_fix_off, b.d_fix_slot, b.num_fix);
        else k_blocked_fixup<false><<<fg, 256, 0, s>>>(p.out, partial, b.d_fix_node, b.d_fix_off, b.d_fix_slot, b.num_fix);
        count_launch();
    }
}

// Which FP64 cell-block kernel runs, read once per process from PYLITH_B200_TET_KERNEL: "pad2" (the
// default: two barriers per block over the padded layout), "pipe" (one barrier per block over the
// padded layout) or "twophase" (two barriers per block, per-thread 8-byte gathers of all node data).
enum TetKernel { TK_PAD2, TK_PIPE, TK_TWOPHASE };
static TetKernel tet_kernel_choice() {
    static const TetKernel k = [] {
        const char* v = std::getenv("PYLITH_B200_TET_KERNEL");
        if (v && std::strcmp(v, "pipe") == 0) return TK_PIPE;
        if (v && std::strcmp(v, "twophase") == 0) return TK_TWOPHASE;
        return TK_PAD2;
    }();
    return k;
}

static bool blocked_usable(const BlockedLayout& b) {
    return b.num_blocks > 0 && b.max_local_nodes <= kMaxSlotsPerThread * kTetThreads &&
           blocked_smem(b) <= 200 * 1024;
}

bool launch_domain_apply_blocked(const DomainParams& p, const BlockedLayout& b, int cell, int rheo, bool bf,
                                 int op, bool insert, int64_t nnodes, double* partial, cudaStream_t s, bool reduced) {
    if (cell != TET4 || rheo != RHEO_ILE || !blocked_usable(b)) return false;
    if (reduced) {
        // padded-layout kernels with the reduced slot ids; the caller zeroed the output
        const int ld = (b.max_local_nodes + 3) & ~3;
        const TetKernel kr = tet_kernel_choice();
        if (partial || insert || !b.d_pipe_ids_red || kr == TK_TWOPHASE ||
            (kr == TK_PIPE && pipe_smem_bytes(ld) > 75 * 1024) || (kr == TK_PAD2 && pad2_smem_bytes(ld) > 56 * 1024))
            return false;
        const bool pipe = kr == TK_PIPE;
        if (op == OP_RESIDUAL) {
            if (pipe && bf) launch_pipe_t<true, RHEO_ILE, true, OP_RESIDUAL>(p, b, false, nullptr, s, true);
            else if (pipe) launch_pipe_t<true, RHEO_ILE, false, OP_RESIDUAL>(p, b, false, nullptr, s, true);
            else if (bf) launch_pipe_t<false, RHEO_ILE, true, OP_RESIDUAL>(p, b, false, nullptr, s, true);
            else launch_pipe_t<false, RHEO_ILE, false, OP_RESIDUAL>(p, b, false, nullptr, s, true);
        } else if (pipe) {
            launch_pipe_t<true, RHEO_ILE, false, OP_JACOBIAN_ACTION>(p, b, false, nullptr, s, true);
        } else {
            launch_pipe_t<false, RHEO_ILE, false, OP_JACOBIAN_ACTION>(p, b, false, nullptr, s, true);
        }
        return true;
    }
    // Nodes owned by one block are stored (INSERT) or added (ADD) by their block. With a
    // partial-sum buffer (deterministic mode) the fixup pass then writes or adds every other
    // node, so no output zeroing and no atomics are needed and the sums are the same every run.
    // Without one, shared nodes get FP64 reductions, and for INSERT the output starts from zero.
    if (!partial && insert && (b.num_shared_nodes > 0 || b.num_untouched > 0))
        if (cudaMemsetAsync(p.out, 0, 3 * nnodes * sizeof(double), s) != cudaSuccess) return false;
    const int ld = (b.max_local_nodes + 3) & ~3;
    TetKernel k = tet_kernel_choice();
    if (!b.d_pipe_begin || (k == TK_PIPE && pipe_smem_bytes(ld) > 75 * 1024) || (k == TK_PAD2 && pad2_smem_bytes(ld) > 56 * 1024))
        k = TK_TWOPHASE;
    if (op == OP_RESIDUAL) {
        if (k == TK_PIPE && bf) launch_pipe_t<true, RHEO_ILE, true, OP_RESIDUAL>(p, b, insert, partial, s);
        else if (k == TK_PIPE) launch_pipe_t<true, RHEO_ILE, false, OP_RESIDUAL>(p, b, insert, partial, s);
        else if (k == TK_PAD2 && bf) launch_pipe_t<false, RHEO_ILE, true, OP_RESIDUAL>(p, b, insert, partial, s);
        else if (k == TK_PAD2) launch_pipe_t<false, RHEO_ILE, false, OP_RESIDUAL>(p, b, insert, partial, s);
        else if (bf) launch_t<RHEO_ILE, true, OP_RESIDUAL>(p, b, insert, partial, s);
        else launch_t<RHEO_ILE, false, OP_RESIDUAL>(p, b, insert, partial, s);
    } else {
        if (k == TK_PIPE) launch_pipe_t<true, RHEO_ILE, false, OP_JACOBIAN_ACTION>(p, b, insert, partial, s);
        else if (k == TK_PAD2) launch_pipe_t<false, RHEO_ILE, false, OP_JACOBIAN_ACTION>(p, b, insert, partial, s);
        else launch_t<RHEO_ILE, false, OP_JACOBIAN_ACTION>(p, b, insert, partial, s);
    }
    return true;
}

bool launch_domain_jv32_blocked(const DomainParams& p, const BlockedLayout& b, int cell, int rheo, int64_t nnodes,
                                cudaStream_t s, bool reduced) {
    if (cell != TET4 || !blocked_usable(b)) return false;
    if (reduced && !b.d_pipe_ids_red) return false;
    // the padded-layout kernel (default); with the solver's cached tangent any isotropic rheology
    const int ld = (b.max_local_nodes + 3) & ~3;
    if (tet_kernel_choice() != TK_TWOPHASE && b.d_pipe_begin && padjv_smem_bytes(ld) <= 48 * 1024 &&
        (p.lm32 || rheo == RHEO_ILE)) {
        const size_t smem = padjv_smem_bytes(ld);
        const void* kern = p.lm32 ? (const void*)k_tet_pad_jv32<true> : (const void*)k_tet_pad_jv32<false>;
        ensure_kernel_smem(kern, smem);
        const int grid = (int)std::min<int64_t>(b.num_blocks, (int64_t)sm_count() * 4);
        if (p.lm32) k_tet_pad_jv32<true><<<grid, kTetBlockCells, smem, s>>>(p, pipe_arrays_of(b, nullptr, reduced));
        else k_tet_pad_jv32<false><<<grid, kTetBlockCells, smem, s>>>(p, pipe_arrays_of(b, nullptr, reduced));
        count_launch();
        return true;
    }
    if (rheo != RHEO_ILE || reduced) return false;
    const size_t smem = (size_t)12 * kTetBlockCells * sizeof(float) +
                        (size_t)b.max_local_nodes * (3 * sizeof(double) + 3 * sizeof(float));
    if (smem > 200 * 1024) return false;
    ensure_kernel_smem((const void*)k_tet_blocked_jv32, smem);
    // the output was zeroed by the caller (INSERT) or holds the partial sum (ADD)
    k_tet_blocked_jv32<<<persistent_grid(b.num_blocks), kTetBlockCells, smem, s>>>(p, arrays_of(b));
    count_launch();
    return true;
}

// Host: bank-aware numbering of one block's local nodes and order of their incidence sums.
//
// The kernels keep node values component-major in shared memory, so the bank pair of node i in
// an FP64 array is i mod 16 (and the 16-byte bank group of an FP32 row of 28 floats is 7 i mod 8):
// the 32 reads of one corner by a warp's 32 cells conflict when distinct nodes share an index
// residue. Starting from the nodes sorted by global id, a local search over swaps of two nodes'
// indices (deterministic, seeded by the block index) lowers the sum over (warp, corner) of the
// largest number of distinct nodes on one residue. Within each residue class the nodes are then
// placed by decreasing incidence count, so each warp of the per-node sums gets nodes of similar
// counts and runs fewer steps. Finally each node's incidences are ordered, warp by warp and step
// by step, so that the staged element entries read in one step (bank pair = cell mod 16) spread
// over the banks. Any fixed order keeps the sums identical from run to run.
#ifndef PLB_PLAN_ITERS
#define PLB_PLAN_ITERS 12000
#endif
struct BlockPlan {
    std::vector<int32_t> loc;       // global ids of the local nodes, sorted
    std::vector<int32_t> newidx;    // local index of loc[l]
    std::vector<uint16_t> inc;      // incidence entries (cell * 4 + corner) by local index
    std::vector<uint32_t> off;      // [nloc + 1] offsets into inc
    std::vector<uint16_t> inc_pipe; // the same incidences in the same order, as staging offsets
                                    // corner * 3 * kTetBlockCells + cell (padded-layout kernels)
};

// Orders each node's incidences (lists[k], entries cell * 4 + corner) so that the entries that
// the lanes of one warp read in one step (bank pair = cell mod 16) spread over the banks; the
// warp of node k is group(k) and its lanes run the group's nodes in increasing k. Returns the
// per-node ordered lists.
template <typename Group>
static std::vector<std::vector<int>> order_for_banks(std::vector<std::vector<int>> lists, int ngroups, Group group) {
    constexpr int R = 16;
    const int nloc = (int)lists.size();
    std::vector<std::vector<int>> members(ngroups), ordered(nloc);
    for (int k = 0; k < nloc; ++k) members[group(k)].push_back(k);
    for (const std::vector<int>& mem : members) {
        const int nl = (int)mem.size();
        if (nl == 0) continue;
        std::vector<int> lanes(nl);
        int depth = 0;
        for (int k : mem) depth = std::max(depth, (int)lists[k].size());
        for (int j = 0; j < depth; ++j) {
            int c16[R] = {0};
            for (int i = 0; i < nl; ++i) lanes[i] = i;
            std::stable_sort(lanes.begin(), lanes.end(),
                             [&](int x, int y) { return lists[mem[x]].size() > lists[mem[y]].size(); });
            for (int i : lanes) {
                std::vector<int>& L = lists[mem[i]];
                if (L.empty()) continue;
                size_t best = 0;
                for (size_t t = 1; t < L.size(); ++t)
                    if (c16[(L[t] >> 2) & (R - 1)] < c16[(L[best] >> 2) & (R - 1)]) best = t;
                c16[(L[best] >> 2) & (R - 1)]++;
                ordered[mem[i]].push_back(L[best]);
                L.erase(L.begin() + best);
            }
        }
    }
    return ordered;
}

static uint64_t splitmix64(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static void plan_block(const int32_t* bc, int ncell, uint64_t seed, BlockPlan& P) {
    constexpr int R = 16, W = 32, kIters = PLB_PLAN_ITERS;
    P.loc.assign(bc, bc + 4 * (size_t)ncell);
    std::sort(P.loc.begin(), P.loc.end());
    P.loc.erase(std::unique(P.loc.begin(), P.loc.end()), P.loc.end());
    const int nloc = (int)P.loc.size();
    std::vector<int> lcs(4 * (size_t)ncell);
    for (int i = 0; i < 4 * ncell; ++i)
        lcs[i] = (int)(std::lower_bound(P.loc.begin(), P.loc.end(), bc[i]) - P.loc.begin());
    // groups: (warp of cells, corner) -> distinct nodes; each node's groups
    const int ng = (ncell + W - 1) / W * 4;
    std::vector<std::vector<int>> node_groups(nloc);
    std::vector<int> stamp(nloc, -1);
    for (int g = 0; g < ng; ++g) {
        const int w = g / 4, k = g % 4;
        for (int c = w * W; c < std::min(ncell, (w + 1) * W); ++c) {
            const int l = lcs[4 * c + k];
            if (stamp[l] != g) {
                stamp[l] = g;
                node_groups[l].push_back(g);
            }
        }
    }
    std::vector<int>& perm = P.newidx;
    perm.resize(nloc);
    for (int l = 0; l < nloc; ++l) perm[l] = l;
    std::vector<int> cnt((size_t)ng * R, 0);
    for (int l = 0; l < nloc; ++l)
        for (int g : node_groups[l]) cnt[(size_t)g * R + (perm[l] & (R - 1))]++;
    auto gmax = [&](int g) {
        int m = 0;
        for (int r = 0; r < R; ++r) m = std::max(m, cnt[(size_t)g * R + r]);
        return m;
    };
    auto move = [&](int l, int from, int to) {
        for (int g : node_groups[l]) {
            cnt[(size_t)g * R + from]--;
            cnt[(size_t)g * R + to]++;
        }
    };
    std::vector<int> mark(ng, -1), aff;
    uint64_t rs = seed;
    for (int it = 0; it < kIters && nloc > 1; ++it) {
        const int a = (int)(splitmix64(rs) % (uint64_t)nloc), b = (int)(splitmix64(rs) % (uint64_t)nloc);
        const int ra = perm[a] & (R - 1), rb = perm[b] & (R - 1);
        if (ra == rb) continue;
        aff.clear();
        for (int g : node_groups[a])
            if (mark[g] != it) mark[g] = it, aff.push_back(g);
        for (int g : node_groups[b])
            if (mark[g] != it) mark[g] = it, aff.push_back(g);
        int before = 0, after = 0;
        for (int g : aff) before += gmax(g);
        move(a, ra, rb);
        move(b, rb, ra);
        for (int g : aff) after += gmax(g);
        if (after <= before) {
            std::swap(perm[a], perm[b]);
        } else {
            move(a, rb, ra);
            move(b, ra, rb);
        }
    }
    // within each residue class: decreasing incidence count
    std::vector<int> deg(nloc, 0);
    for (int i = 0; i < 4 * ncell; ++i) deg[lcs[i]]++;
    for (int r = 0; r < R; ++r) {
        std::vector<int> nodes, slots;
        for (int l = 0; l < nloc; ++l)
            if ((perm[l] & (R - 1)) == r) nodes.push_back(l), slots.push_back(perm[l]);
        std::sort(slots.begin(), slots.end());
        std::stable_sort(nodes.begin(), nodes.end(), [&](int x, int y) { return deg[x] > deg[y]; });
        for (size_t i = 0; i < nodes.size(); ++i) perm[nodes[i]] = slots[i];
    }
    // incidences by new index, in (cell, corner) order, then ordered for the banks (the warps of
    // the node sums take 32 consecutive nodes)
    std::vector<std::vector<int>> lists(nloc);
    for (int c = 0; c < ncell; ++c)
        for (int k = 0; k < 4; ++k) lists[perm[lcs[4 * c + k]]].push_back(4 * c + k);
    const std::vector<std::vector<int>> by_warp = order_for_banks(lists, (nloc + W - 1) / W, [](int k) { return k / W; });
    P.off.assign(nloc + 1, 0);
    P.inc.clear();
    P.inc.reserve(4 * (size_t)ncell);
    P.inc_pipe.clear();
    P.inc_pipe.reserve(4 * (size_t)ncell);
    for (int k = 0; k < nloc; ++k) {
        for (int e : by_warp[k]) P.inc.push_back((uint16_t)e);
        for (int e : by_warp[k]) P.inc_pipe.push_back((uint16_t)((e & 3) * 3 * kTetBlockCells + (e >> 2)));
        P.off[k + 1] = (uint32_t)P.inc.size();
    }
}

// Host: block layout from the cell connectivity (cells should be in a locality-preserving order).
static int build_blocked_layout(pl_mesh_s* m) {
    if (m->blocked) return PL_OK;
    if (m->cell_type != PL_CELL_TET4 || m->nnodes >= (int64_t)kSharedBit) {
        m->blocked = new BlockedLayout();  // empty: not supported for this mesh
        return PL_OK;
    }
    const int B = kTetBlockCells;
    const int64_t nc = m->ncells;
    // Blocks of at most B consecutive cells, as even as the count allows. (Rounding the count up
    // to whole waves of the persistent grid, 5,328 blocks of 229 cells instead of 4,761 of 256 on
    // the 1.2 M-cell mesh, measured slower: 60.6 against 58.8 us per residual. The per-block cost
    // does not shrink with the cells, and the CTAs still running in a last partial wave have
    // their SMs to themselves.)
    const int64_t nb = (nc + B - 1) / B;
    std::vector<int32_t> cell_begin(nb + 1);
    for (int64_t b = 0; b <= nb; ++b) cell_begin[b] = (int32_t)(b * nc / nb);
    std::vector<int32_t> begin(nb + 1, 0);
    std::vector<uint32_t> node_ids;
    std::vector<uint16_t> lconn((size_t)nc * 4);
    std::vector<uint16_t> inc((size_t)nb * 4 * B, 0);
    std::vector<uint32_t> inc_off;
    std::vector<int32_t> nblocks_of(m->nnodes, 0);
    node_ids.reserve((size_t)nc);
    inc_off.reserve((size_t)nc + nb);
    int maxloc = 0;
    // the blocks' numberings and incidence orders, planned in parallel (a block's plan depends
    // only on its cells and index; the calling thread takes blocks too, so the layout is complete
    // even where no helper thread can be started)
    std::vector<BlockPlan> plans(nb);
    {
        std::atomic<int64_t> next{0};
        std::atomic<bool> failed{false};
        // an exception (bad_alloc in a plan) must not leave a thread: it stops the block loop of
        // every thread, and the layout reports the failure after all threads are joined
        auto work = [&]() noexcept {
            try {
                for (int64_t b; !failed.load() && (b = next.fetch_add(1)) < nb;) {
                    const int64_t c0 = cell_begin[b], c1 = cell_begin[b + 1];
                    plan_block(m->h_cells.data() + c0 * 4, (int)(c1 - c0), (uint64_t)b, plans[b]);
                }
            } catch (...) {
                failed.store(true);
            }
        };
        const int nth = (int)std::min(15u, std::thread::hardware_concurrency());
        std::vector<std::thread> th;
        try {
            for (int t = 1; t < nth; ++t) th.emplace_back(work);
        } catch (...) {
        }
        work();
        for (std::thread& x : th) x.join();
        if (failed.load()) return fail(PL_ERR_OUT_OF_MEMORY, "cell-block layout planning ran out of host memory");
    }
    // padded per-block regions of the pipelined kernel: block b's slots start at pbeg[b], a
    // multiple of 4, so that its node ids, coordinates ([3][ns rounded up to 4]) and incidence
    // offsets are 16-byte aligned runs that the kernel copies with 16-byte cp.async
    std::vector<int32_t> pbeg(nb + 1, 0);
    std::vector<uint32_t> pids;
    std::vector<double> pcoords;
    std::vector<uint32_t> poff;
    std::vector<uint16_t> pinc((size_t)nb * 4 * B, 0);
    for (int64_t b = 0; b < nb; ++b) {
        BlockPlan& P = plans[b];
        const int64_t c0 = cell_begin[b], c1 = cell_begin[b + 1];
        const int nloc = (int)P.loc.size();
        maxloc = std::max(maxloc, nloc);
        begin[b] = (int32_t)node_ids.size();
        node_ids.resize(node_ids.size() + nloc);
        for (int l = 0; l < nloc; ++l) {
            node_ids[begin[b] + P.newidx[l]] = (uint32_t)P.loc[l];
            nblocks_of[P.loc[l]]++;
        }
        const int npad = (nloc + 3) & ~3;
        pbeg[b + 1] = pbeg[b] + npad;
        pids.resize(pbeg[b + 1], 0u);
        pcoords.resize(3 * (size_t)pbeg[b + 1], 0.0);
        for (int l = 0; l < nloc; ++l) {
            const int i = P.newidx[l];
            pids[pbeg[b] + i] = (uint32_t)P.loc[l];
            for (int d = 0; d < 3; ++d) pcoords[3 * (size_t)pbeg[b] + (size_t)d * npad + i] = m->h_coords[3 * (size_t)P.loc[l] + d];
        }
        poff.resize((size_t)pbeg[b + 1] + 4 * (b + 1), 0u);
        for (int i = 0; i <= nloc; ++i) poff[(size_t)pbeg[b] + 4 * b + i] = P.off[i];
        std::copy(P.inc_pipe.begin(), P.inc_pipe.end(), pinc.begin() + (size_t)b * 4 * B);
        for (int64_t c = c0; c < c1; ++c)
            for (int k = 0; k < 4; ++k) {
                const int32_t nd = m->h_cells[c * 4 + k];
                const int l = (int)(std::lower_bound(P.loc.begin(), P.loc.end(), nd) - P.loc.begin());
                lconn[c * 4 + k] = (uint16_t)P.newidx[l];
            }
        for (int i = 0; i <= nloc; ++i) inc_off.push_back(P.off[i]);
        std::copy(P.inc.begin(), P.inc.end(), inc.begin() + (size_t)b * 4 * B);
        P = BlockPlan();
    }
    begin[nb] = (int32_t)node_ids.size();
    for (uint32_t& id : node_ids)
        if (nblocks_of[id] > 1) id |= kSharedBit;
    for (int64_t b = 0; b < nb; ++b)
        for (int i = 0; i < begin[b + 1] - begin[b]; ++i)
            if (nblocks_of[pids[pbeg[b] + i]] > 1) pids[pbeg[b] + i] |= kSharedBit;
    int64_t nshared = 0, nuntouched = 0;
    for (int64_t nd = 0; nd < m->nnodes; ++nd) {
        nshared += nblocks_of[nd] > 1;
        nuntouched += nblocks_of[nd] == 0;
    }
    // fixup lists: nodes not owned by exactly one block, with their slots in block order
    std::vector<int32_t> fix_node, fix_off(1, 0), fix_slot;
    {
        std::vector<int32_t> first(m->nnodes + 1, 0);
        for (size_t gs = 0; gs < node_ids.size(); ++gs) {
            const uint32_t nd = node_ids[gs] & ~kSharedBit;
            if (nblocks_of[nd] > 1) first[nd + 1]++;
        }
        for (int64_t nd = 0; nd < m->nnodes; ++nd) first[nd + 1] += first[nd];
        std::vector<int32_t> slots(first[m->nnodes]);
        std::vector<int32_t> pos(first.begin(), first.end() - 1);
        for (size_t gs = 0; gs < node_ids.size(); ++gs) {
            const uint32_t nd = node_ids[gs] & ~kSharedBit;
            if (nblocks_of[nd] > 1) slots[pos[nd]++] = (int32_t)gs;
        }
        for (int64_t nd = 0; nd < m->nnodes; ++nd) {
            if (nblocks_of[nd] == 1) continue;
            fix_node.push_back((int32_t)nd);
            for (int32_t j = first[nd]; j < first[nd + 1]; ++j) fix_slot.push_back(slots[j]);
            fix_off.push_back((int32_t)fix_slot.size());
        }
    }
    BlockedLayout* L = new BlockedLayout();
    L->num_slots = (int64_t)node_ids.size();
    L->num_fix = (int64_t)fix_node.size();
    L->cells_per_block = B;
    L->num_blocks = nb;
    L->max_local_nodes = maxloc;
    L->num_shared_nodes = nshared;
    L->num_untouched = nuntouched;
    cudaStream_t s = m->ctx->stream;
    cudaError_t e = cudaSuccess;
    auto up = [&](auto** dst, const auto& v) {
        if (e != cudaSuccess || v.empty()) return;
        const size_t bytes = v.size() * sizeof(v[0]);
        e = dev_alloc((void**)dst, bytes);
        if (e == cudaSuccess) e = cudaMemcpyAsync(*dst, v.data(), bytes, cudaMemcpyHostToDevice, s);
        L->device_bytes += bytes;
    };
    up(&L->d_cell_begin, cell_begin);
    up(&L->d_block_node_begin, begin);
    up(&L->d_slot_node, node_ids);
    up(&L->d_local_cells, lconn);
    up(&L->d_inc_off, inc_off);
    up(&L->d_inc, inc);
    up(&L->d_fix_node, fix_node);
    up(&L->d_fix_off, fix_off);
    up(&L->d_fix_slot, fix_slot);
    up(&L->d_pipe_begin, pbeg);
    up(&L->d_pipe_ids, pids);
    L->h_pipe_ids = pids;
    L->h_pipe_begin = pbeg;
    L->h_block_node_begin = begin;
    up(&L->d_pipe_coords, pcoords);
    up(&L->d_pipe_off, poff);
    up(&L->d_pipe_inc, pinc);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        free_blocked_layout(L, s);
        return cuda_fail(e, "blocked layout upload");
    }
    m->blocked = L;
    return PL_OK;
}

int ensure_blocked_layout(pl_mesh_s* m) {
    try {
        return build_blocked_layout(m);
    } catch (const std::bad_alloc&) {
        return fail(PL_ERR_OUT_OF_MEMORY, "cell-block layout: out of host memory");
    } catch (...) {
        return fail(PL_ERR_INVALID_ARG, "cell-block layout failed");
    }
}

int ensure_reduced_ids(pl_mesh_s* m) {
    BlockedLayout* L = m->blocked;
    if (!L || L->num_blocks == 0) return fail(PL_ERR_UNSUPPORTED, "no cell-block layout");
    if (L->d_pipe_ids_red) return PL_OK;
    if (m->h_node_red.size() != (size_t)m->nnodes) return fail(PL_ERR_UNSUPPORTED, "no reduced fault space");
    // a node of the reduced space is owned by its block only if it has one slot in all blocks
    std::vector<uint32_t> ids(L->h_pipe_ids.size(), 0u);
    std::vector<int32_t> slots(m->nnodes, 0);
    for (int64_t b = 0; b < L->num_blocks; ++b) {
        const int p0 = L->h_pipe_begin[b], ns = L->h_block_node_begin[b + 1] - L->h_block_node_begin[b];
        for (int i = 0; i < ns; ++i) {
            const uint32_t r = (uint32_t)m->h_node_red[L->h_pipe_ids[p0 + i] & ~kSharedBit];
            ids[p0 + i] = r;
            slots[r]++;
        }
    }
    for (int64_t b = 0; b < L->num_blocks; ++b) {
        const int p0 = L->h_pipe_begin[b], ns = L->h_block_node_begin[b + 1] - L->h_block_node_begin[b];
        for (int i = 0; i < ns; ++i)
            if (slots[ids[p0 + i]] > 1) ids[p0 + i] |= kSharedBit;
    }
    // the same ids without the padding, for the batched kernel's slot order
    std::vector<uint32_t> slot_ids((size_t)L->h_block_node_begin[L->num_blocks], 0u);
    for (int64_t b = 0; b < L->num_blocks; ++b) {
        const int p0 = L->h_pipe_begin[b], s0 = L->h_block_node_begin[b], ns = L->h_block_node_begin[b + 1] - s0;
        for (int i = 0; i < ns; ++i) slot_ids[s0 + i] = ids[p0 + i];
    }
    uint32_t *d = nullptr, *d2 = nullptr;
    PLB_CUDA(dev_alloc(&d, ids.size()));
    cudaError_t e = dev_alloc(&d2, slot_ids.size());
    if (e != cudaSuccess) {
        dev_free(d, nullptr);
        return cuda_fail(e, "reduced slot ids");
    }
    PLB_CUDA(cudaMemcpyAsync(d, ids.data(), ids.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, m->ctx->stream));
    PLB_CUDA(cudaMemcpyAsync(d2, slot_ids.data(), slot_ids.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                             m->ctx->stream));
    PLB_CUDA(cudaStreamSynchronize(m->ctx->stream));
    L->d_pipe_ids_red = d;
    L->d_slot_node_red = d2;
    return PL_OK;
}

void free_blocked_layout(BlockedLayout* b, cudaStream_t after) {
    if (!b) return;
    dev_free(b->d_pipe_ids_red, after);
    dev_free(b->d_slot_node_red, after);
    void* ptrs[] = {b->d_cell_begin, b->d_block_node_begin, b->d_slot_node, b->d_local_cells, b->d_inc_off, b->d_inc,
                    b->d_fix_node, b->d_fix_off, b->d_fix_slot, b->d_pipe_begin, b->d_pipe_ids,
                    b->d_pipe_coords, b->d_pipe_off, b->d_pipe_inc};
    for (void* p : ptrs) dev_free(p, after);
    delete b;
}

}  // namespace plb
