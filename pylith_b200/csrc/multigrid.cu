// Geometric multigrid preconditioner for the device solver: V-cycles over a hierarchy of solvers
// (one per level: operator, constraint mask, point-block Jacobi, fault pairs), tied by
// caller-built prolongations, inside flexible conjugate gradients.
//
// The reference preconditions these solves with PETSc's algebraic multigrid (GAMG with a
// point-block Jacobi fine smoother on faults, libsrc/pylith/materials/Elasticity.cc:298-330). Here
// each level smooths with a Chebyshev polynomial of point-block Jacobi (degree `degree`, interval
// [lower b, b] with b = 1.1 lambda_max(D^-1 A) from power iterations at setup), the coarsest level
// is solved exactly with the inverse of its reduced matrix when it has at most kDenseMax unknowns
// (assembled from the level's element Jacobians and inverted by Gauss-Jordan elimination on the
// device at setup; one matrix-vector launch per V-cycle), else approximated by a higher-degree
// Chebyshev polynomial over a wider interval, restriction is
// the transpose of the prolongation (coarse vectors are unfolded before prolongation and the
// restricted ones folded, so that both act in the solvers' reduced fault spaces), and the V-cycle
// runs in FP64 or FP32 (FP32 operators with the cached per-cell tangent and FP32 vectors) while
// the outer conjugate gradients stay in FP64: a flexible (Polak-Ribiere) step length absorbs the
// rounding of an FP32 preconditioner. Everything a PCG iteration launches is captured as one CUDA
// graph per chunk of iterations.
#include <algorithm>
#include <cmath>
#include <vector>

#include "cg.cuh"
#include "domain_kernels.cuh"
#include "internal.hpp"
#include "launch.hpp"

namespace plb {

namespace {

constexpr int kMgRedBlocks = 296;

enum MgScalar { M_RZ = 0, M_RZ_OLD, M_PQ, M_RR, M_ZROLD, M_COUNT };

// Coarsest levels with at most this many unknowns are solved with their dense inverse.
constexpr int kDenseMax = 1536;

// dense[map[row dof]][map[col dof]] -= J block entry (A = -J; a fault node's two sides both land
// on its negative-side unknown); one warp per block row of the mesh nodes (Lagrange rows are not
// read), the entries' 9 components over the lanes.
__global__ void k_dense_scatter(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                const double* __restrict__ val, int64_t nmesh, const int32_t* __restrict__ map, int n,
                                double* dense) {
    const int lane = threadIdx.x & 31;
    for (int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; r < nmesh;
         r += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int64_t k0 = rp[r], k1 = rp[r + 1];
        for (int64_t e = k0 * 9 + lane; e < k1 * 9; e += 32) {
            const int64_t k = e / 9;
            const int ab = (int)(e - 9 * k), a = ab / 3, b = ab - 3 * a;
            const int64_t c = ci[k];
            if (c >= nmesh) continue;
            const int fi = map[3 * r + a], fj = map[3 * c + b];
            if (fi >= 0 && fj >= 0) atomicAdd(&dense[(int64_t)fi * n + fj], -val[e]);
        }
    }
}

// Gauss-Jordan step k, part 1: row k and column k of the current matrix into row[], col[]; a
// non-positive pivot (the reduced matrix is symmetric positive definite) sets *flag.
__global__ void k_gj_take(const double* __restrict__ a, int n, int k, double* row, double* col, unsigned int* flag) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        row[i] = a[(int64_t)k * n + i];
        col[i] = a[(int64_t)i * n + k];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && !(a[(int64_t)k * n + k] > 0.0)) atomicOr(flag, 1u);
}

// Gauss-Jordan step k, part 2 (in place, no pivoting): with p = a_kk, row k becomes row/p (its
// diagonal 1/p) and every other row i becomes a_ij - a_ik a_kj / p (its column-k entry -a_ik / p).
__global__ void k_gj_update(double* a, int n, int k, const double* __restrict__ row, const double* __restrict__ col) {
    const double p = row[k];
    const double inv = p != 0.0 ? 1.0 / p : 0.0;
    const int64_t nn = (int64_t)n * n;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nn; e += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(e / n), j = (int)(e - (int64_t)i * n);
        const double rk = j == k ? 1.0 : row[j];
        if (i == k) a[e] = rk * inv;
        else a[e] = (j == k ? 0.0 : a[e]) - col[i] * rk * inv;
    }
}

__global__ void k_dense_to_f32(const double* __restrict__ a, int64_t nn, float* out) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nn; e += (int64_t)gridDim.x * blockDim.x)
        out[e] = (float)a[e];
}

// z[idx[i]] = sum_j inv[i][j] r[idx[j]] (z zeroed before): each block stages the gathered right-
// hand side in shared memory, one warp per row.
template <typename T>
__global__ void __launch_bounds__(256) k_dense_apply(const T* __restrict__ inv, const int32_t* __restrict__ idx, int n,
                                                     const T* __restrict__ r, T* __restrict__ z) {
    __shared__ T sr[kDenseMax];
    for (int j = threadIdx.x; j < n; j += blockDim.x) sr[j] = r[idx[j]];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    for (int i = blockIdx.x * 8 + (threadIdx.x >> 5); i < n; i += gridDim.x * 8) {
        const T* row = inv + (int64_t)i * n;
        T acc = T(0);
        for (int j = lane; j < n; j += 32) acc += row[j] * sr[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (lane == 0) z[idx[i]] = acc;
    }
}

int mg_grid(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8)); }

// out = D^{-1} in / theta; d = out (first Chebyshev step from a zero guess).
template <typename T>
__global__ void k_mg_cheb_first(const T* __restrict__ in, const T* __restrict__ pinv, int64_t nn, double inv_theta,
                                T* __restrict__ d, T* __restrict__ out) {
    for (int64_t nd = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; nd < nn; nd += (int64_t)gridDim.x * blockDim.x) {
        T z[3];
        apply_pinv(pinv, in, nd, z);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const T v = (T)(z[k] * inv_theta);
            d[3 * nd + k] = v;
            out[3 * nd + k] = v;
        }
    }
}

// Chebyshev step: res = in - A out (= in + q on free DOFs, q = J out), d = c1 d + c2 D^{-1} res,
// out += d.
template <typename T>
__global__ void k_mg_cheb_next(const T* __restrict__ in, const T* __restrict__ q, const T* __restrict__ pinv,
                               const uint8_t* __restrict__ mask, int64_t nn, double c1, double c2, T* __restrict__ d,
                               T* __restrict__ out) {
    for (int64_t nd = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; nd < nn; nd += (int64_t)gridDim.x * blockDim.x) {
        T res[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) res[k] = mask[3 * nd + k] ? T(0) : (T)(in[3 * nd + k] + q[3 * nd + k]);
        const T* B = pinv + 9 * nd;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const T zr = B[3 * k] * res[0] + B[3 * k + 1] * res[1] + B[3 * k + 2] * res[2];
            const T dv = (T)(c1 * d[3 * nd + k] + c2 * zr);
            d[3 * nd + k] = dv;
            out[3 * nd + k] += dv;
        }
    }
}

// t = in - A z = in + q on free DOFs, 0 elsewhere.
template <typename T>
__global__ void k_mg_residual(const T* __restrict__ in, const T* __restrict__ q, const uint8_t* __restrict__ mask,
                              int64_t n, T* __restrict__ t) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        t[i] = mask[i] ? T(0) : (T)(in[i] + q[i]);
}

// coarse[c] = sum_j R[c][j] fine[col_j] (R = P^T in coarse rows) for the 3 components, 0 on the
// coarse level's masked DOFs: one warp per coarse node, its lanes over the row's entries, a fixed
// shuffle tree for the sums.
template <typename T>
__global__ void k_mg_restrict(const T* __restrict__ fine, const int32_t* __restrict__ row, const int32_t* __restrict__ col,
                              const double* __restrict__ val, const uint8_t* __restrict__ cmask, int64_t nc,
                              T* __restrict__ coarse) {
    const int lane = threadIdx.x & 31;
    for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < nc;
         c += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        for (int32_t j = row[c] + lane; j < row[c + 1]; j += 32) {
            const double w = val[j];
            const int64_t f = 3 * (int64_t)col[j];
            s0 += w * (double)fine[f];
            s1 += w * (double)fine[f + 1];
            s2 += w * (double)fine[f + 2];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s0 += __shfl_xor_sync(0xffffffffu, s0, o);
            s1 += __shfl_xor_sync(0xffffffffu, s1, o);
            s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        }
        if (lane < 3) {
            const int64_t i = 3 * c + lane;
            coarse[i] = cmask[i] ? T(0) : (T)(lane == 0 ? s0 : (lane == 1 ? s1 : s2));
        }
    }
}

// Prolongation columns in the coarse level's reduced space: a positive-side fault node's column
// becomes its negative-side partner's (map: node -> node of the reduced space).
__global__ void k_mg_map_cols(int32_t* col, int64_t nnz, const int32_t* __restrict__ map) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nnz; j += (int64_t)gridDim.x * blockDim.x)
        col[j] = map[col[j]];
}

__global__ void k_mg_iota(int32_t* map, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        map[i] = (int32_t)i;
}

__global__ void k_mg_pair_map2(int32_t* map, const int32_t* __restrict__ neg, const int32_t* __restrict__ pos,
                               int64_t npairs) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < npairs; k += (int64_t)gridDim.x * blockDim.x)
        map[pos[k]] = neg[k];
}

// fine[f] += sum_j P[f][j] coarse[col_j] on free DOFs (P in fine rows).
template <typename T>
__global__ void k_mg_prolong_add(const T* __restrict__ coarse, const int32_t* __restrict__ row,
                                 const int32_t* __restrict__ col, const double* __restrict__ val,
                                 const uint8_t* __restrict__ mask, int64_t nf, T* __restrict__ fine) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * nf; i += (int64_t)gridDim.x * blockDim.x) {
        if (mask[i]) continue;
        const int64_t f = i / 3;
        const int k = (int)(i % 3);
        double s = 0.0;
        for (int32_t j = row[f]; j < row[f + 1]; ++j) s += val[j] * (double)coarse[3 * (int64_t)col[j] + k];
        fine[i] += (T)s;
    }
}

template <typename T>
__global__ void k_mg_mask(T* __restrict__ v, const uint8_t* __restrict__ mask, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (mask[i]) v[i] = T(0);
}

template <typename T>
__global__ void k_mg_axpy(T* __restrict__ y, const T* __restrict__ x, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) y[i] += x[i];
}

template <typename A, typename B>
__global__ void k_mg_convert(const A* __restrict__ in, B* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (B)in[i];
}

// power iteration for lambda_max(D^{-1} A): w = D^{-1} (-J v) on free DOFs, partial w.w and v.v
__global__ void k_mg_power(const double* __restrict__ q, const double* __restrict__ pinv, const uint8_t* __restrict__ mask,
                           int64_t nn, double* __restrict__ w, double* partials) {
    double ww = 0.0;
    for (int64_t nd = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; nd < nn; nd += (int64_t)gridDim.x * blockDim.x) {
        double a[3], z[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) a[k] = mask[3 * nd + k] ? 0.0 : -q[3 * nd + k];
        const double* B = pinv + 9 * nd;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            z[k] = B[3 * k] * a[0] + B[3 * k + 1] * a[1] + B[3 * k + 2] * a[2];
            w[3 * nd + k] = z[k];
            ww += z[k] * z[k];
        }
    }
    block_sum2(ww, 0.0, partials);
}

// a fixed pseudo-random start vector on the free DOFs, and its partial squared norm
__global__ void __launch_bounds__(kRedThreads) k_mg_seed(double* __restrict__ v, const uint8_t* __restrict__ mask, int64_t n,
                                                         double* partials) {
    double vv = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t h = (uint64_t)i * 0x9E3779B97F4A7C15ull;
        h ^= h >> 29;
        h *= 0xBF58476D1CE4E5B9ull;
        h ^= h >> 32;
        const double x = mask[i] ? 0.0 : (double)(h >> 11) * (1.0 / 9007199254740992.0) - 0.5;
        v[i] = x;
        vv += x * x;
    }
    block_sum2(vv, 0.0, partials);
}

// v = w / |w| with |w|^2 in scal[slot] (on the device: no host round trip per power iteration)
__global__ void k_mg_normalize(double* __restrict__ v, const double* __restrict__ w, int64_t n, const double* scal, int slot) {
    const double nrm = sqrt(scal[slot]);
    const double s = nrm > 0.0 ? 1.0 / nrm : 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) v[i] = w[i] * s;
}

// ---- outer flexible PCG (FP64) ----------------------------------------------------------------
// partials of r.z and z.r_old (flexible beta) and r.r
__global__ void __launch_bounds__(kRedThreads) k_mg_dots(const double* __restrict__ r, const double* __restrict__ z,
                                                         const double* __restrict__ r_old, const uint8_t* __restrict__ mask,
                                                         int64_t n, double* partials) {
    double rz = 0.0, zro = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (mask[i]) continue;
        rz += r[i] * z[i];
        zro += z[i] * r_old[i];
    }
    block_sum2(rz, zro, partials);
}

__global__ void __launch_bounds__(kRedThreads) k_mg_pq(const double* __restrict__ p, const double* __restrict__ q,
                                                       const uint8_t* __restrict__ mask, int64_t n, double* partials) {
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (!mask[i]) s -= p[i] * q[i];
    block_sum2(s, 0.0, partials);
}

// x += alpha p, r_old = r, r += alpha q (free DOFs); partial r.r
__global__ void __launch_bounds__(kRedThreads) k_mg_update(double* __restrict__ x, double* __restrict__ r,
                                                           double* __restrict__ r_old, const double* __restrict__ p,
                                                           const double* __restrict__ q, const uint8_t* __restrict__ mask,
                                                           int64_t n, const double* __restrict__ scal, double* partials) {
    const double pq = scal[M_PQ];
    const double alpha = pq > 0.0 ? scal[M_RZ] / pq : 0.0;
    double rr = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        r_old[i] = r[i];
        if (!mask[i]) {
            x[i] += alpha * p[i];
            r[i] += alpha * q[i];
        }
        rr += r[i] * r[i];
    }
    block_sum2(rr, 0.0, partials);
}

// beta = (r.z - z.r_old) / rz_old (Polak-Ribiere, for a preconditioner that may vary), p = z + beta p
__global__ void k_mg_pupdate(double* __restrict__ p, const double* __restrict__ z, int64_t n, double* scal) {
    const double ro = scal[M_RZ_OLD];
    const double beta = ro != 0.0 ? std::max(0.0, (scal[M_RZ] - scal[M_ZROLD]) / ro) : 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = z[i] + beta * p[i];
}

__global__ void k_mg_copy_scalar(double* scal, int from, int to) { scal[to] = scal[from]; }

// ---- restriction = transpose of the prolongation, built on the device -------------------------
// Entries per coarse node (cnt zeroed before).
__global__ void k_tr_count(const int32_t* __restrict__ col, int64_t nnz, int32_t* cnt) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nnz; j += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&cnt[col[j]], 1);
}

// out[0] = 0, out[i + 1] = cnt[0] + .. + cnt[i] (one block of 1024 threads, each summing a
// contiguous run).
__global__ void __launch_bounds__(1024) k_tr_scan(const int32_t* __restrict__ cnt, int64_t n, int32_t* out) {
    __shared__ int32_t part[1024];
    const int t = threadIdx.x;
    const int64_t per = (n + 1023) / 1024, a = t * per, b = std::min<int64_t>(n, a + per);
    int32_t sum = 0;
    for (int64_t i = a; i < b; ++i) sum += cnt[i];
    part[t] = sum;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int32_t v = t >= off ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int32_t run = t > 0 ? part[t - 1] : 0;
    if (t == 0) out[0] = 0;
    for (int64_t i = a; i < b; ++i) {
        run += cnt[i];
        out[i + 1] = run;
    }
}

// Scatter of every prolongation entry (fine row f, coarse col c) into coarse row c (fill zeroed).
__global__ void k_tr_fill(const int32_t* __restrict__ rp, const int32_t* __restrict__ col, const double* __restrict__ val,
                          int64_t nf, const int32_t* __restrict__ rrow, int32_t* fill, int32_t* rcol, double* rval) {
    for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < nf; f += (int64_t)gridDim.x * blockDim.x)
        for (int32_t j = rp[f]; j < rp[f + 1]; ++j) {
            const int32_t c = col[j];
            const int32_t pos = rrow[c] + atomicAdd(&fill[c], 1);
            rcol[pos] = (int32_t)f;
            rval[pos] = val[j];
        }
}

// Each coarse row's entries in increasing fine row (the order the atomics left is arbitrary).
__global__ void k_tr_sort(const int32_t* __restrict__ rrow, int64_t nc, int32_t* rcol, double* rval) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
        const int32_t a = rrow[c], b = rrow[c + 1];
        for (int32_t i = a + 1; i < b; ++i) {
            const int32_t k = rcol[i];
            const double v = rval[i];
            int32_t j = i - 1;
            while (j >= a && rcol[j] > k) {
                rcol[j + 1] = rcol[j];
                rval[j + 1] = rval[j];
                --j;
            }
            rcol[j + 1] = k;
            rval[j + 1] = v;
        }
    }
}

}  // namespace
}  // namespace plb

using namespace plb;

struct MgLevel {
    pl_solver S = nullptr;
    int64_t n = 0, nn = 0;  // DOFs and node rows of the solver (mesh nodes, then Lagrange nodes)
    int64_t nmesh = 0;      // mesh nodes: the rows and columns of the prolongations
    // prolongation from the next coarser level into this one: fine-row CSR and its transpose
    int32_t *p_row = nullptr, *p_col = nullptr, *r_row = nullptr, *r_col = nullptr;
    double *p_val = nullptr, *r_val = nullptr;
    double lmax = 0.0;
    // work vectors of the V-cycle (FP64 and FP32)
    double *r = nullptr, *z = nullptr, *t = nullptr, *d = nullptr, *w = nullptr, *q = nullptr;
    float *r32 = nullptr, *z32 = nullptr, *t32 = nullptr, *d32 = nullptr, *w32 = nullptr, *q32 = nullptr;
};

struct pl_multigrid_s {
    pl_context ctx = nullptr;  // retained: the levels' context (the fine solver may go first)
    std::vector<MgLevel> lv;
    int degree = 2, coarse_degree = 40;
    bool pre_smooth = true, post_smooth = true;  // pl_multigrid_set_cycle
    double lower = 0.1, coarse_lower = 0.01;
    bool fp32 = false;
    bool eig_valid = false;
    pl_solver attached = nullptr;
    int batch_users = 0;  // batched solvers preconditioned by this hierarchy
    // outer PCG state
    double *x = nullptr, *r = nullptr, *r_old = nullptr, *p = nullptr, *q = nullptr, *z = nullptr;
    double* scal = nullptr;
    double* partials = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_iters = 0;
    unsigned long long graph_epoch = 0;
    // dense solve of the coarsest level (dense_n: -1 not examined yet, 0 too large)
    int dense_n = -1;
    bool dense_ok = false;
    int32_t* d_dense_idx = nullptr;  // [dense_n] DOF of each unknown
    int32_t* d_dense_map = nullptr;  // [3 nmesh] unknown of each mesh DOF (-1: constrained)
    double* d_dense = nullptr;       // [dense_n^2] matrix, inverted in place
    float* d_dense32 = nullptr;
    double* d_gj = nullptr;          // [2 dense_n] Gauss-Jordan row and column
    unsigned int* d_flag = nullptr;
    pl_matrix dense_A = nullptr;     // the coarsest level's assembled Jacobian
};

namespace {

cudaStream_t mg_stream(pl_multigrid mg) { return mg->lv[0].S->mesh->ctx->stream; }

// Chebyshev polynomial of point-block Jacobi on level l: out = p(D^-1 A) D^-1 in, from zero.
template <typename T>
int cheb(pl_multigrid mg, int l, const T* in, T* out, int degree, double lower) {
    MgLevel& L = mg->lv[l];
    cudaStream_t s = mg_stream(mg);
    const double b = 1.1 * L.lmax, a = lower * b;
    const double theta = 0.5 * (b + a), delta = 0.5 * (b - a), sigma = theta / delta;
    T* d = sizeof(T) == 8 ? (T*)L.d : (T*)L.d32;
    T* q = sizeof(T) == 8 ? (T*)L.q : (T*)L.q32;
    const T* pinv = sizeof(T) == 8 ? (const T*)L.S->d_pinv : (const T*)L.S->d_pinv32;
    k_mg_cheb_first<T><<<mg_grid(L.nn), 256, 0, s>>>(in, pinv, L.nn, 1.0 / theta, d, out);
    count_launch();
    double rho_old = 1.0 / sigma;
    for (int k = 1; k < degree; ++k) {
        int rc = sizeof(T) == 8 ? solver_apply_J(L.S, (const double*)out, (double*)q)
                                : solver_apply_J32(L.S, (const float*)out, (float*)q);
        if (rc) return rc;
        const double rho = 1.0 / (2.0 * sigma - rho_old);
        k_mg_cheb_next<T><<<mg_grid(L.nn), 256, 0, s>>>(in, q, pinv, L.S->d_mask, L.nn, rho * rho_old, 2.0 * rho / delta,
                                                        d, out);
        count_launch();
        rho_old = rho;
    }
    return PL_OK;
}

// z_l = V(r_l) on level l (vectors of the level's work set in precision T).
template <typename T>
int vcycle(pl_multigrid mg, int l) {
    MgLevel& L = mg->lv[l];
    cudaStream_t s = mg_stream(mg);
    const bool f32 = sizeof(T) == 4;
    T* r = f32 ? (T*)L.r32 : (T*)L.r;
    T* z = f32 ? (T*)L.z32 : (T*)L.z;
    T* t = f32 ? (T*)L.t32 : (T*)L.t;
    T* w = f32 ? (T*)L.w32 : (T*)L.w;
    T* q = f32 ? (T*)L.q32 : (T*)L.q;
    const int last = (int)mg->lv.size() - 1;
    if (l == last) {
        if (!mg->dense_ok) return cheb<T>(mg, l, r, z, mg->coarse_degree, mg->coarse_lower);
        PLB_CUDA(cudaMemsetAsync(z, 0, L.n * sizeof(T), s));
        const T* inv = f32 ? (const T*)mg->d_dense32 : (const T*)mg->d_dense;
        k_dense_apply<T><<<std::max(1, std::min((mg->dense_n + 7) / 8, 148)), 256, 0, s>>>(inv, mg->d_dense_idx,
                                                                                             mg->dense_n, r, z);
        count_launch();
        return PL_OK;
    }
    auto apply = [&](T* v) { return f32 ? solver_apply_J32(L.S, (const float*)v, (float*)q) : solver_apply_J(L.S, (const double*)v, (double*)q); };
    int rc = PL_OK;
    const T* tr = r;  // the residual to restrict
    if (mg->pre_smooth) {
        if ((rc = cheb<T>(mg, l, r, z, mg->degree, mg->lower))) return rc;
        if ((rc = apply(z))) return rc;
        k_mg_residual<T><<<mg_grid(L.n), 256, 0, s>>>(r, q, L.S->d_mask, L.n, t);
        tr = t;
    } else {
        PLB_CUDA(cudaMemsetAsync(z, 0, L.n * sizeof(T), s));
    }
    // restriction into the coarse level's r, folded and masked
    MgLevel& C = mg->lv[l + 1];
    T* rc_ = f32 ? (T*)C.r32 : (T*)C.r;
    T* zc = f32 ? (T*)C.z32 : (T*)C.z;
    // the restriction's rows are the coarse level's reduced space (its prolongation columns were
    // mapped onto it): no fold; the Lagrange rows of the coarse vector stay zero
    if (C.n > 3 * C.nmesh) PLB_CUDA(cudaMemsetAsync(rc_ + 3 * C.nmesh, 0, (C.n - 3 * C.nmesh) * sizeof(T), s));
    k_mg_restrict<T><<<mg_grid(32 * C.nmesh), 256, 0, s>>>(tr, L.r_row, L.r_col, L.r_val, C.S->d_mask, C.nmesh, rc_);
    count_launch(2);
    if ((rc = vcycle<T>(mg, l + 1))) return rc;
    // ... and the prolongation reads the coarse correction there: no unfold
    k_mg_prolong_add<T><<<mg_grid(3 * L.nmesh), 256, 0, s>>>(zc, L.p_row, L.p_col, L.p_val, L.S->d_mask, L.nmesh, z);
    count_launch();
    // post-smoothing on the new residual
    if (!mg->post_smooth) return PL_OK;
    if ((rc = apply(z))) return rc;
    k_mg_residual<T><<<mg_grid(L.n), 256, 0, s>>>(r, q, L.S->d_mask, L.n, t);
    count_launch();
    if ((rc = cheb<T>(mg, l, t, w, mg->degree, mg->lower))) return rc;
    k_mg_axpy<T><<<mg_grid(L.n), 256, 0, s>>>(z, w, L.n);
    count_launch();
    return PL_OK;
}

// z = M r on the fine level (FP64 vectors in and out; an FP32 V-cycle converts at the ends).
int precondition(pl_multigrid mg, const double* r, double* z) {
    MgLevel& L = mg->lv[0];
    cudaStream_t s = mg_stream(mg);
    int rc;
    if (mg->fp32) {
        k_mg_convert<double, float><<<mg_grid(L.n), 256, 0, s>>>(r, L.r32, L.n);
        count_launch();
        if ((rc = vcycle<float>(mg, 0))) return rc;
        k_mg_convert<float, double><<<mg_grid(L.n), 256, 0, s>>>(L.z32, z, L.n);
        count_launch();
    } else {
        PLB_CUDA(cudaMemcpyAsync(L.r, r, L.n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        if ((rc = vcycle<double>(mg, 0))) return rc;
        PLB_CUDA(cudaMemcpyAsync(z, L.z, L.n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    return PL_OK;
}

// lambda_max(D^{-1} A) of every level by power iteration (FP64), after the levels' setup: the
// iterates are normalised on the device and the host reads one number per level.
int estimate_eigenvalues(pl_multigrid mg, int iters = 12) {
    cudaStream_t s = mg_stream(mg);
    for (size_t l = 0; l < mg->lv.size(); ++l) {
        MgLevel& L = mg->lv[l];
        if (l + 1 == mg->lv.size() && mg->dense_ok) break;  // solved exactly: no smoother
        k_mg_seed<<<kMgRedBlocks, kRedThreads, 0, s>>>(L.t, L.S->d_mask, L.n, mg->partials);
        k_finish2<<<1, 1024, 0, s>>>(mg->partials, kMgRedBlocks, mg->scal, M_RR, -1);
        k_mg_normalize<<<mg_grid(L.n), 256, 0, s>>>(L.t, L.t, L.n, mg->scal, M_RR);
        count_launch(3);
        for (int it = 0; it < iters; ++it) {
            int rc = solver_apply_J(L.S, L.t, L.q);
            if (rc) return rc;
            k_mg_power<<<kMgRedBlocks, kRedThreads, 0, s>>>(L.q, L.S->d_pinv, L.S->d_mask, L.nn, L.w, mg->partials);
            k_finish2<<<1, 1024, 0, s>>>(mg->partials, kMgRedBlocks, mg->scal, M_RR, -1);
            k_mg_normalize<<<mg_grid(L.n), 256, 0, s>>>(L.t, L.w, L.n, mg->scal, M_RR);
            count_launch(3);
        }
        double h[M_COUNT];
        PLB_CUDA(cudaMemcpyAsync(h, mg->scal, sizeof(h), cudaMemcpyDeviceToHost, s));
        PLB_CUDA(cudaStreamSynchronize(s));
        const double lam = std::sqrt(h[M_RR]);  // |D^-1 A v| for the unit iterate v
        if (!(lam > 0.0) || !std::isfinite(lam)) return fail(PL_ERR_NOT_CONVERGED, "multigrid: no eigenvalue estimate");
        L.lmax = lam;
    }
    mg->eig_valid = true;
    return PL_OK;
}

// The coarsest level's dense inverse (after each setup): the unknowns' maps on first use, then the
// reduced matrix from the level's assembled Jacobian and its Gauss-Jordan inverse. Levels with more
// than kDenseMax unknowns, or a matrix that is not positive definite, keep the Chebyshev solve.
int prepare_dense(pl_multigrid mg) {
    MgLevel& L = mg->lv.back();
    pl_solver S = L.S;
    cudaStream_t s = mg_stream(mg);
    mg->dense_ok = false;
    if (mg->dense_n < 0) {
        std::vector<uint8_t> mask(L.n);
        std::vector<int32_t> pneg(S->npairs), ppos(S->npairs);
        PLB_CUDA(cudaMemcpyAsync(mask.data(), S->d_mask, L.n, cudaMemcpyDeviceToHost, s));
        if (S->npairs) {
            PLB_CUDA(cudaMemcpyAsync(pneg.data(), S->d_pair_neg, S->npairs * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
            PLB_CUDA(cudaMemcpyAsync(ppos.data(), S->d_pair_pos, S->npairs * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        }
        PLB_CUDA(cudaStreamSynchronize(s));
        std::vector<int32_t> fidx(L.n, -1), idx;
        for (int64_t i = 0; i < L.n; ++i)
            if (!mask[i]) {
                fidx[i] = (int32_t)idx.size();
                idx.push_back((int32_t)i);
            }
        if (idx.empty() || idx.size() > (size_t)kDenseMax) {
            mg->dense_n = 0;
            return PL_OK;
        }
        std::vector<int64_t> node_of(L.nmesh);
        for (int64_t v = 0; v < L.nmesh; ++v) node_of[v] = v;
        for (int64_t k = 0; k < S->npairs; ++k) node_of[ppos[k]] = pneg[k];
        std::vector<int32_t> map(3 * L.nmesh);
        for (int64_t i = 0; i < 3 * L.nmesh; ++i) map[i] = fidx[3 * node_of[i / 3] + i % 3];
        const int n = (int)idx.size();
        cudaError_t e = dev_alloc(&mg->d_dense_idx, n);
        if (e == cudaSuccess) e = dev_alloc(&mg->d_dense_map, map.size());
        if (e == cudaSuccess) e = dev_alloc(&mg->d_dense, (size_t)n * n);
        if (e == cudaSuccess) e = dev_alloc(&mg->d_dense32, (size_t)n * n);
        if (e == cudaSuccess) e = dev_alloc(&mg->d_gj, 2 * (size_t)n);
        if (e == cudaSuccess) e = dev_alloc(&mg->d_flag, 1);
        if (e == cudaSuccess) e = cudaMemcpyAsync(mg->d_dense_idx, idx.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(mg->d_dense_map, map.data(), map.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return cuda_fail(e, "multigrid dense coarse solve");
        int rc = pl_matrix_create(S->mesh, &mg->dense_A);
        if (rc) return rc;
        mg->dense_n = n;
    }
    if (mg->dense_n == 0) return PL_OK;
    const int n = mg->dense_n;
    int rc = pl_matrix_zero(mg->dense_A);
    if (rc) return rc;
    PLB_CUDA(cudaMemsetAsync(L.t, 0, L.n * sizeof(double), s));  // the state the Jacobian kernels read
    for (pl_integrator ig : S->ops)
        if ((rc = pl_compute_lhs_jacobian(ig, S->t, S->dt, 0.0, L.t, mg->dense_A)) != PL_OK) return rc;
    PLB_CUDA(cudaMemsetAsync(mg->d_dense, 0, (size_t)n * n * sizeof(double), s));
    PLB_CUDA(cudaMemsetAsync(mg->d_flag, 0, sizeof(unsigned int), s));
    const pl_matrix_s& A = *mg->dense_A;
    k_dense_scatter<<<mg_grid(32 * L.nmesh), 256, 0, s>>>(A.d_row_ptr, A.d_col, A.d_val, L.nmesh, mg->d_dense_map, n,
                                                          mg->d_dense);
    count_launch();
    double* row = mg->d_gj;
    double* col = mg->d_gj + n;
    const int gt = std::max(1, std::min((n + 255) / 256, 8));
    const int gu = mg_grid((int64_t)n * n);
    for (int k = 0; k < n; ++k) {
        k_gj_take<<<gt, 256, 0, s>>>(mg->d_dense, n, k, row, col, mg->d_flag);
        k_gj_update<<<gu, 256, 0, s>>>(mg->d_dense, n, k, row, col);
    }
    count_launch(2 * n);
    k_dense_to_f32<<<mg_grid((int64_t)n * n), 256, 0, s>>>(mg->d_dense, (int64_t)n * n, mg->d_dense32);
    count_launch();
    unsigned int flag = 0;
    PLB_CUDA(cudaMemcpyAsync(&flag, mg->d_flag, sizeof(flag), cudaMemcpyDeviceToHost, s));
    PLB_CUDA(cudaStreamSynchronize(s));
    mg->dense_ok = flag == 0;
    return PL_OK;
}

// One flexible PCG iteration (capturable).
int mg_iteration(pl_multigrid mg) {
    pl_solver S = mg->lv[0].S;
    cudaStream_t s = mg_stream(mg);
    const int64_t n = S->n;
    int rc = solver_apply_J(S, mg->p, mg->q);
    if (rc) return rc;
    k_mg_pq<<<kMgRedBlocks, kRedThreads, 0, s>>>(mg->p, mg->q, S->d_mask, n, mg->partials);
    k_finish2<<<1, 1024, 0, s>>>(mg->partials, kMgRedBlocks, mg->scal, M_PQ, -1);
    k_mg_copy_scalar<<<1, 1, 0, s>>>(mg->scal, M_RZ, M_RZ_OLD);
    k_mg_update<<<kMgRedBlocks, kRedThreads, 0, s>>>(mg->x, mg->r, mg->r_old, mg->p, mg->q, S->d_mask, n, mg->scal,
                                                       mg->partials);
    k_finish2<<<1, 1024, 0, s>>>(mg->partials, kMgRedBlocks, mg->scal, M_RR, -1);
    count_launch(5);
    if ((rc = precondition(mg, mg->r, mg->z))) return rc;
    k_mg_mask<double><<<mg_grid(n), 256, 0, s>>>(mg->z, S->d_mask, n);
    k_mg_dots<<<kMgRedBlocks, kRedThreads, 0, s>>>(mg->r, mg->z, mg->r_old, S->d_mask, n, mg->partials);
    k_finish2<<<1, 1024, 0, s>>>(mg->partials, kMgRedBlocks, mg->scal, M_RZ, M_ZROLD);
    k_mg_pupdate<<<mg_grid(n), 256, 0, s>>>(mg->p, mg->z, n, mg->scal);
    count_launch(4);
    return PL_OK;
}

}  // namespace

namespace plb {

// Called by pl_solver_setup of the fine solver: the coarse levels' setup at the same (t, dt)
// and, lazily at the next solve, their eigenvalue estimates.
int multigrid_setup(pl_multigrid mg, double t, double dt) {
    for (size_t l = 1; l < mg->lv.size(); ++l) {
        int rc = pl_solver_setup(mg->lv[l].S, t, dt);
        if (rc) return rc;
    }
    mg->eig_valid = false;
    return PL_OK;
}

// Multigrid-preconditioned flexible CG in FP64 for pl_solver_solve.
int multigrid_solve(pl_multigrid mg, const double* b, double* x) {
    pl_solver S = mg->lv[0].S;
    pl_context c = S->mesh->ctx;
    cudaStream_t s0 = c->stream;
    const int64_t n = S->n;
    int rc;
    if (!mg->eig_valid && ((rc = prepare_dense(mg)) != PL_OK || (rc = estimate_eigenvalues(mg)) != PL_OK)) return rc;
    for (const MgLevel& L : mg->lv)
        for (pl_integrator ig : L.S->ops)
            if ((rc = prepare_jv32_tangent(ig, L.S->t, L.S->dt)) != PL_OK) return rc;
    // the fine solver's private stream carries the iterations (and their graph)
    PLB_CUDA(cudaEventRecord(S->ev_in, s0));
    PLB_CUDA(cudaStreamWaitEvent(S->cstream, S->ev_in, 0));
    c->stream = S->cstream;
    cudaStream_t s = S->cstream;
    double h[M_COUNT];
    rc = PL_OK;
    double r0 = 0.0;
    do {
        const double* bb = solver_reduced_rhs(S, b);
        if (cudaMemsetAsync(mg->x, 0, n * sizeof(double), s) != cudaSuccess ||
            cudaMemcpyAsync(mg->r, bb, n * sizeof(double), cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
            rc = fail(PL_ERR_CUDA, "multigrid start");
            break;
        }
        k_mg_mask<double><<<mg_grid(n), 256, 0, s>>>(mg->r, S->d_mask, n);
        k_mg_pq<<<kMgRedBlocks, kRedThreads, 0, s>>>(mg->r, mg->r, S->d_mask, n, mg->partials);  // -r.r
        k_finish2<<<1, 1024, 0, s>>>(mg->partials, kMgRedBlocks, mg->scal, M_RR, -1);
        count_launch(3);
        if ((rc = precondition(mg, mg->r, mg->z)) != PL_OK) break;
        k_mg_mask<double><<<mg_grid(n), 256, 0, s>>>(mg->z, S->d_mask, n);
        k_mg_dots<<<kMgRedBlocks, kRedThreads, 0, s>>>(mg->r, mg->z, mg->z, S->d_mask, n, mg->partials);
        k_finish2<<<1, 1024, 0, s>>>(mg->partials, kMgRedBlocks, mg->scal, M_RZ, -1);
        count_launch(3);
        if (cudaMemcpyAsync(mg->p, mg->z, n * sizeof(double), cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
            cudaMemcpyAsync(h, mg->scal, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            rc = fail(PL_ERR_CUDA, "multigrid start");
            break;
        }
        r0 = std::sqrt(std::fabs(h[M_RR]));
        const double stop = std::max(S->rtol * r0, S->atol);
        S->iterations = 0;
        S->rel_residual = r0 > 0.0 ? 1.0 : 0.0;
        if (r0 == 0.0 || r0 <= stop) break;
        const int chunk = std::max(1, std::min(S->check_every, 5));
        if (!mg->graph || mg->graph_iters != chunk || mg->graph_epoch != state_epoch()) {
            if (mg->graph) cudaGraphExecDestroy(mg->graph);
            mg->graph = nullptr;
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed);
            for (int i = 0; i < chunk && rc == PL_OK && e == cudaSuccess; ++i) rc = mg_iteration(mg);
            if (e == cudaSuccess) e = cudaStreamEndCapture(s, &g);
            if (e == cudaSuccess && rc == PL_OK) e = cudaGraphInstantiate(&mg->graph, g, 0);
            if (g) cudaGraphDestroy(g);
            if (rc == PL_OK && e != cudaSuccess) rc = cuda_fail(e, "multigrid graph capture");
            if (rc) break;
            mg->graph_iters = chunk;
            mg->graph_epoch = state_epoch();
        }
        for (int it = 0; it < S->max_iter; it += chunk) {
            cudaError_t e = cudaGraphLaunch(mg->graph, s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(h, mg->scal, sizeof(h), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) {
                rc = cuda_fail(e, "multigrid PCG");
                break;
            }
            S->iterations = it + chunk;
            const double rn = std::sqrt(h[M_RR]);
            S->rel_residual = rn / r0;
            if (!(rn == rn)) {
                rc = fail(PL_ERR_NOT_CONVERGED, "multigrid PCG diverged (NaN residual)");
                break;
            }
            if (rn <= stop) break;
            if (it + chunk >= S->max_iter) rc = fail(PL_ERR_NOT_CONVERGED, "multigrid PCG reached the iteration limit");
        }
    } while (false);
    if (rc == PL_OK) {
        if (cudaMemcpyAsync(x, mg->x, n * sizeof(double), cudaMemcpyDeviceToDevice, s) != cudaSuccess) rc = fail(PL_ERR_CUDA, "copy");
        else solver_unfold(S, x);
    }
    c->stream = s0;
    cudaEventRecord(S->ev_out, s);
    cudaStreamWaitEvent(s0, S->ev_out, 0);
    return rc;
}

void multigrid_detach(pl_multigrid mg) { mg->attached = nullptr; }

int multigrid_prepare(pl_multigrid mg) {
    if (mg->eig_valid) return PL_OK;
    int rc = prepare_dense(mg);
    if (rc == PL_OK) rc = estimate_eigenvalues(mg);
    return rc;
}

MgView multigrid_view(const pl_multigrid_s* mg) {
    MgView v;
    for (const MgLevel& L : mg->lv)
        v.levels.push_back({L.S, L.n, L.nn, L.nmesh, L.p_row, L.p_col, L.r_row, L.r_col, L.p_val, L.r_val, L.lmax});
    v.degree = mg->degree;
    v.lower = mg->lower;
    v.coarse_degree = mg->coarse_degree;
    v.pre_smooth = mg->pre_smooth;
    v.post_smooth = mg->post_smooth;
    v.coarse_lower = mg->coarse_lower;
    v.dense_inv32 = mg->dense_ok ? mg->d_dense32 : nullptr;
    v.dense_idx = mg->dense_ok ? mg->d_dense_idx : nullptr;
    v.dense_n = mg->dense_ok ? mg->dense_n : 0;
    return v;
}

void multigrid_batch_use(pl_multigrid mg, int delta) { mg->batch_users += delta; }

}  // namespace plb

extern "C" {

int pl_multigrid_create(pl_solver fine, int num_coarse, const pl_solver* coarse, const int32_t* const* prolong_row_ptr,
                        const int32_t* const* prolong_col, const double* const* prolong_val, pl_multigrid* out) {
    if (!fine || !out || num_coarse < 1 || !coarse || !prolong_row_ptr || !prolong_col || !prolong_val)
        return fail(PL_ERR_INVALID_ARG, "bad arguments");
    *out = nullptr;
    std::vector<pl_solver> levels{fine};
    for (int i = 0; i < num_coarse; ++i) {
        if (!coarse[i]) return fail(PL_ERR_INVALID_ARG, "null coarse solver");
        if (coarse[i]->mesh->ctx != fine->mesh->ctx) return fail(PL_ERR_INVALID_ARG, "levels must share one context");
        if (coarse[i]->ops.empty()) return fail(PL_ERR_NOT_READY, "a coarse level has no integrators");
        levels.push_back(coarse[i]);
    }
    PLB_CUDA(cudaSetDevice(fine->mesh->ctx->device));
    pl_multigrid mg = new pl_multigrid_s();
    cudaError_t e = cudaSuccess;
    auto A = [&](auto** p, size_t cnt) {
        if (e == cudaSuccess && cnt) e = dev_alloc(p, cnt);
    };
    auto up = [&](auto** p, const auto* src, size_t cnt) {
        A(p, cnt);
        if (e == cudaSuccess && cnt)
            e = cudaMemcpyAsync(*p, src, cnt * sizeof(*src), cudaMemcpyHostToDevice, fine->mesh->ctx->stream);
    };
    for (size_t l = 0; l < levels.size(); ++l) {
        MgLevel L;
        L.S = levels[l];
        L.n = L.S->n;
        L.nn = L.S->nnodes;
        L.nmesh = L.S->mesh->nnodes;
        A(&L.r, L.n); A(&L.z, L.n); A(&L.t, L.n); A(&L.d, L.n); A(&L.w, L.n); A(&L.q, L.n);
        A(&L.r32, L.n); A(&L.z32, L.n); A(&L.t32, L.n); A(&L.d32, L.n); A(&L.w32, L.n); A(&L.q32, L.n);
        mg->lv.push_back(L);
    }
    cudaStream_t s = fine->mesh->ctx->stream;
    int32_t* d_tmp = nullptr;  // per coarse node: counts, then fill positions
    for (int l = 0; l < num_coarse && e == cudaSuccess; ++l) {
        MgLevel& F = mg->lv[l];
        const MgLevel& C = mg->lv[l + 1];
        const int32_t* rp = prolong_row_ptr[l];
        const int64_t nf = F.nmesh, nc = C.nmesh;
        const int64_t nnz = rp[nf];
        bool ok = rp[0] == 0 && nnz >= 0;
        for (int64_t f = 0; f < nf && ok; ++f) ok = rp[f + 1] >= rp[f];
        for (int64_t j = 0; j < nnz && ok; ++j) ok = prolong_col[l][j] >= 0 && prolong_col[l][j] < nc;
        if (!ok) {
            for (MgLevel& L : mg->lv) {
                void* ptrs[] = {L.r, L.z, L.t, L.d, L.w, L.q, L.r32, L.z32, L.t32, L.d32, L.w32, L.q32, L.p_row, L.p_col, L.p_val,
                                L.r_row, L.r_col, L.r_val};
                for (void* p : ptrs) dev_free(p, nullptr);
            }
            delete mg;
            return fail(PL_ERR_INVALID_ARG, "prolongation column outside the coarse level");
        }
        up(&F.p_row, rp, (size_t)nf + 1);
        up(&F.p_col, prolong_col[l], (size_t)nnz);
        up(&F.p_val, prolong_val[l], (size_t)nnz);
        if (e == cudaSuccess && C.S->npairs > 0 && nnz > 0) {
            int32_t* d_map = nullptr;
            e = dev_alloc(&d_map, (size_t)nc);
            if (e == cudaSuccess) {
                k_mg_iota<<<mg_grid(nc), 256, 0, s>>>(d_map, nc);
                k_mg_pair_map2<<<mg_grid(C.S->npairs), 256, 0, s>>>(d_map, C.S->d_pair_neg, C.S->d_pair_pos, C.S->npairs);
                k_mg_map_cols<<<mg_grid(nnz), 256, 0, s>>>(F.p_col, nnz, d_map);
                count_launch(3);
                dev_free(d_map, s);
            }
        }
        // the restriction P^T, its rows in increasing fine index
        A(&F.r_row, (size_t)nc + 1);
        A(&F.r_col, (size_t)nnz);
        A(&F.r_val, (size_t)nnz);
        if (e == cudaSuccess) e = dev_alloc(&d_tmp, (size_t)nc);
        if (e == cudaSuccess) e = cudaMemsetAsync(d_tmp, 0, nc * sizeof(int32_t), s);
        if (e == cudaSuccess && nnz > 0) {
            k_tr_count<<<mg_grid(nnz), 256, 0, s>>>(F.p_col, nnz, d_tmp);
            k_tr_scan<<<1, 1024, 0, s>>>(d_tmp, nc, F.r_row);
            e = cudaMemsetAsync(d_tmp, 0, nc * sizeof(int32_t), s);
            k_tr_fill<<<mg_grid(nf), 256, 0, s>>>(F.p_row, F.p_col, F.p_val, nf, F.r_row, d_tmp, F.r_col, F.r_val);
            k_tr_sort<<<mg_grid(nc), 256, 0, s>>>(F.r_row, nc, F.r_col, F.r_val);
            count_launch(4);
        } else if (e == cudaSuccess) {
            e = cudaMemsetAsync(F.r_row, 0, (nc + 1) * sizeof(int32_t), s);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        dev_free(d_tmp, s);
        d_tmp = nullptr;
    }
    const int64_t n = fine->n;
    A(&mg->x, n); A(&mg->r, n); A(&mg->r_old, n); A(&mg->p, n); A(&mg->q, n); A(&mg->z, n);
    A(&mg->scal, M_COUNT);
    A(&mg->partials, 2 * kMgRedBlocks);
    if (e != cudaSuccess) {
        for (MgLevel& L : mg->lv) {
            void* ptrs[] = {L.r, L.z, L.t, L.d, L.w, L.q, L.r32, L.z32, L.t32, L.d32, L.w32, L.q32, L.p_row, L.p_col, L.p_val,
                            L.r_row, L.r_col, L.r_val};
            for (void* p : ptrs) dev_free(p, s);
        }
        void* ptrs[] = {mg->x, mg->r, mg->r_old, mg->p, mg->q, mg->z, mg->scal, mg->partials};
        for (void* p : ptrs) dev_free(p, s);
        delete mg;
        return cuda_fail(e, "pl_multigrid_create");
    }
    // the coarse solvers belong to the hierarchy; the fine solver holds the hierarchy instead
    for (size_t l = 1; l < levels.size(); ++l) solver_retain(levels[l]);
    mg->ctx = fine->mesh->ctx;
    context_retain(mg->ctx);
    *out = mg;
    return PL_OK;
}

int pl_multigrid_set_smoother(pl_multigrid mg, int degree, double lower_ratio, int coarse_degree, double coarse_lower_ratio,
                              int precision) {
    if (!mg || degree < 1 || degree > 16 || coarse_degree < 1 || coarse_degree > 200 || !(lower_ratio > 0 && lower_ratio < 1) ||
        !(coarse_lower_ratio > 0 && coarse_lower_ratio < 1) || (precision != PL_SOLVER_FP64 && precision != PL_SOLVER_FP32_REFINED))
        return fail(PL_ERR_INVALID_ARG, "bad smoother settings");
    mg->degree = degree;
    mg->lower = lower_ratio;
    mg->coarse_degree = coarse_degree;
    mg->coarse_lower = coarse_lower_ratio;
    mg->fp32 = precision == PL_SOLVER_FP32_REFINED;
    if (mg->graph) cudaGraphExecDestroy(mg->graph);
    mg->graph = nullptr;
    return PL_OK;
}

int pl_solver_set_multigrid(pl_solver S, pl_multigrid mg) {
    if (!S) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    if (mg && mg->lv[0].S != S) return fail(PL_ERR_INVALID_ARG, "the hierarchy was built on another fine solver");
    if (S->mg) multigrid_detach(S->mg);
    S->mg = mg;
    if (mg) mg->attached = S;
    S->ready = false;  // the coarse levels are set up with the next pl_solver_setup
    return PL_OK;
}

int pl_multigrid_set_cycle(pl_multigrid mg, int pre_smooth, int post_smooth) {
    if (!mg || (!pre_smooth && !post_smooth)) return fail(PL_ERR_INVALID_ARG, "a V-cycle smooths at least once");
    mg->pre_smooth = pre_smooth != 0;
    mg->post_smooth = post_smooth != 0;
    if (mg->graph) cudaGraphExecDestroy(mg->graph);
    mg->graph = nullptr;
    return PL_OK;
}

int pl_multigrid_get_levels(pl_multigrid mg, int* num_levels, double* lambda_max) {
    if (!mg) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    if (num_levels) *num_levels = (int)mg->lv.size();
    if (lambda_max)
        for (size_t l = 0; l < mg->lv.size(); ++l) lambda_max[l] = mg->lv[l].lmax;
    return PL_OK;
}

int pl_multigrid_destroy(pl_multigrid mg) {
    if (!mg) return PL_OK;
    if (mg->attached) return fail(PL_ERR_INVALID_ARG, "the hierarchy is still attached to its solver");
    if (mg->batch_users > 0) return fail(PL_ERR_INVALID_ARG, "the hierarchy still preconditions a batched solver");
    if (mg->ctx) {
        cudaSetDevice(mg->ctx->device);
        cudaStreamSynchronize(mg->ctx->stream);
    }
    if (mg->graph) cudaGraphExecDestroy(mg->graph);
    for (MgLevel& L : mg->lv) {
        void* ptrs[] = {L.r, L.z, L.t, L.d, L.w, L.q, L.r32, L.z32, L.t32, L.d32, L.w32, L.q32, L.p_row, L.p_col, L.p_val,
                        L.r_row, L.r_col, L.r_val};
        for (void* p : ptrs) dev_free(p, mg->ctx ? mg->ctx->stream : nullptr);
    }
    void* ptrs[] = {mg->x, mg->r, mg->r_old, mg->p, mg->q, mg->z, mg->scal, mg->partials,
                    mg->d_dense_idx, mg->d_dense_map, mg->d_dense, mg->d_dense32, mg->d_gj, mg->d_flag};
    for (void* p : ptrs) dev_free(p, mg->ctx ? mg->ctx->stream : nullptr);
    if (mg->dense_A) pl_matrix_destroy(mg->dense_A);
    std::vector<pl_solver> coarse;
    for (size_t l = 1; l < mg->lv.size(); ++l) coarse.push_back(mg->lv[l].S);
    pl_context c = mg->ctx;
    delete mg;
    for (pl_solver S : coarse) solver_release(S);
    if (c) context_release(c);
    return PL_OK;
}

}  // extern "C"
