// Pieces of the conjugate-gradient kernels shared by the single-solver PCG (solver.cu) and the
// ragged batch of solvers (ragged.cu): the scalar slots, deterministic block sums and the
// point-block Jacobi preconditioner.
#pragma once

#include "common.cuh"

namespace plb {

constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 296;  // 2 per SM

// FP32 reliable-update PCG: an iterated residual this many times the last true residual counts
// as a breakdown (the FP32 correction is dropped and the iteration restarts from the true
// residual); a solve gives up after kMaxBreakdowns of them.
constexpr double kBreakdownGrowth = 100.0;
constexpr int kMaxBreakdowns = 20;

enum Scalar { S_RZ = 0, S_RZ_OLD, S_PQ, S_RR, S_ALPHA, S_BETA, S_BB, S_COUNT };

template <typename T>
PL_D double to_d(T v) { return (double)v; }

// Block-level sum of up to 2 values; thread 0 of each block writes partials[blk*2 + k].
PL_D void block_sum2(double a, double b, double* partials) {
    __shared__ double sa[kRedThreads / 32], sb[kRedThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        sa[w] = a;
        sb[w] = b;
    }
    __syncthreads();
    if (w == 0) {
        a = l < (int)(blockDim.x >> 5) ? sa[l] : 0.0;
        b = l < (int)(blockDim.x >> 5) ? sb[l] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
        if (l == 0) {
            partials[2 * blockIdx.x] = a;
            partials[2 * blockIdx.x + 1] = b;
        }
    }
}

// Sum the partials of the previous pass in a fixed order into scal[i0], scal[i1].
static __global__ void k_finish2(const double* __restrict__ partials, int nblk, double* scal, int i0, int i1) {
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) {
        a += partials[2 * i];
        b += partials[2 * i + 1];
    }
    __shared__ double sa[32], sb[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        sa[w] = a;
        sb[w] = b;
    }
    __syncthreads();
    if (w == 0) {
        a = l < (int)(blockDim.x >> 5) ? sa[l] : 0.0;
        b = l < (int)(blockDim.x >> 5) ? sb[l] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
        if (l == 0) {
            if (i0 >= 0) scal[i0] = a;
            if (i1 >= 0) scal[i1] = b;
        }
    }
}

// z = P^{-1} r with point blocks; constrained entries of r are zero and P^{-1} is the identity
// on them, so z stays zero there.
template <typename T>
PL_D void apply_pinv(const T* pinv, const T* r, int64_t node, T out[3]) {
    const T* B = pinv + 9 * node;
    const T r0 = r[3 * node], r1 = r[3 * node + 1], r2 = r[3 * node + 2];
    out[0] = B[0] * r0 + B[1] * r1 + B[2] * r2;
    out[1] = B[3] * r0 + B[4] * r1 + B[5] * r2;
    out[2] = B[6] * r0 + B[7] * r1 + B[8] * r2;
}

}  // namespace plb
