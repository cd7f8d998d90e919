// Hexahedral cells with a group of lanes per cell: the residual and Jacobian action of Q1 (8
// quadrature points) and Q2 (27 quadrature points) hexahedra.
//
// The thread-per-cell kernel (domain.cu) keeps a whole Q2 cell in one thread (81 accumulators,
// 27 quadrature points in a loop) and spills. Here a group of lanes shares one cell: a full warp
// for Q2 (27 lanes busy), 8 lanes for Q1 (four cells per warp). Lane q owns quadrature point q:
// it forms the trilinear geometry, the solution gradient from the cell's node values staged in
// shared memory, calls the registered pointwise kernel and stages its test-function weights
// wdetJ f1 J^{-T} (and wdetJ f0). Lane n then owns node n: it contracts the staged weights with
// the reference basis gradients of node n over all quadrature points and adds the result into
// the output (FP64 reductions; nodes are shared with neighbouring cells). The reference basis
// tables (gradients and values at the quadrature points, and the trilinear geometry gradients)
// are built once per block in shared memory. The FP32 variant (inner iterations of the refined
// solver) keeps the geometry and the tangent in FP64 and stages the field, the weights and the
// sums in FP32.
#include "domain_kernels.cuh"
#include "internal.hpp"
#include "launch.hpp"

namespace plb {

template <int CELL, typename T = double>
struct HexGroup {
    using E = Elem<CELL>;
    static constexpr int NEN = E::nen;
    static constexpr int NQ = E::nq;
    static constexpr int G = CELL == HEX27 ? 32 : 8;   // lanes per cell
    static constexpr int CPW = 32 / G;                 // cells per warp
    static constexpr int LDB = (NEN * 3) | 1;          // odd row stride: lanes q spread over banks
    static constexpr int WARPS = 8;
    // FP64 tables (bytes from the start): geometry gradients [NQ][25], weights [NQ]
    static constexpr int T_W = NQ * 25;
    static constexpr int T_END64 = T_W + NQ;
    // T tables after them: field-basis gradients [NQ][LDB], basis values [NQ][NEN]
    static constexpr int T_PHI = NQ * LDB;
    static constexpr int T_ENDT = T_PHI + NQ * NEN;
    // per-group staging: corner coordinates [8][3] FP64; node field [NEN][3], test-function
    // weights [NQ][9] and body-force weights [NQ][3] in T; odd stride between groups
    static constexpr int OFF_F = NEN * 3;
    static constexpr int OFF_F0 = OFF_F + NQ * 9;
    static constexpr int PER_GROUP_T = (OFF_F0 + NQ * 3) | 1;
    static constexpr int PER_GROUP_X = 25;
    static constexpr int GROUPS = WARPS * CPW;
    static constexpr size_t bytes64() { return sizeof(double) * ((size_t)T_END64 + (size_t)GROUPS * PER_GROUP_X); }
    static constexpr size_t smem_bytes() {
        return bytes64() + sizeof(T) * ((size_t)T_ENDT + (size_t)GROUPS * PER_GROUP_T);
    }
};

template <int CELL, typename T>
PL_D void fill_tables(double* t64, T* tt) {
    using H = HexGroup<CELL, T>;
    for (int i = threadIdx.x; i < H::NQ * H::NEN; i += blockDim.x) {
        const int q = i / H::NEN, n = i % H::NEN;
        double d[3];
        if (CELL == HEX8) {
            hex_corner_dN<2>(n, q & 1, (q >> 1) & 1, q >> 2, d);
        } else {
            const double x = gauss3_x(q % 3), y = gauss3_x((q / 3) % 3), z = gauss3_x(q / 9);
            const int a = n % 3, b = (n / 3) % 3, c = n / 9;
            d[0] = quad_d(a, x) * quad_v(b, y) * quad_v(c, z);
            d[1] = quad_v(a, x) * quad_d(b, y) * quad_v(c, z);
            d[2] = quad_v(a, x) * quad_v(b, y) * quad_d(c, z);
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) tt[q * H::LDB + n * 3 + k] = (T)d[k];
        tt[H::T_PHI + q * H::NEN + n] = (T)Elem<CELL>::phi(q, n);
    }
    for (int i = threadIdx.x; i < H::NQ * 8; i += blockDim.x) {
        const int q = i / 8, c = i % 8;
        double d[3];
        if (CELL == HEX8) hex_corner_dN<2>(c, q & 1, (q >> 1) & 1, q >> 2, d);
        else hex_corner_dN<3>(c, q % 3, (q / 3) % 3, q / 9, d);
#pragma unroll
        for (int k = 0; k < 3; ++k) t64[q * 25 + c * 3 + k] = d[k];
    }
    for (int q = threadIdx.x; q < H::NQ; q += blockDim.x)
        t64[H::T_W + q] = CELL == HEX8 ? 1.0 : gauss3_w(q % 3) * gauss3_w((q / 3) % 3) * gauss3_w(q / 9);
}

// Per-block tables and per-group staging of the group-of-lanes hexahedral kernels.
template <int CELL, typename T>
struct HexGroupSmem {
    const double* tN;  // geometry gradients [NQ][25]
    const double* tW;  // quadrature weights
    const T* tB;       // field-basis gradients [NQ][LDB]
    const T* tPhi;     // basis values [NQ][NEN]
    double* sX;        // this group's corner coordinates
    T* su;             // this group's node field
    T* sF;             // test-function weights
    T* sF0;            // body-force weights
    int grp, l;        // group of this lane within its warp, lane within the group
};

template <int CELL, typename T>
PL_D HexGroupSmem<CELL, T> hex_group_smem(double* hsm) {
    using H = HexGroup<CELL, T>;
    HexGroupSmem<CELL, T> g;
    double* t64 = hsm;
    T* tt = reinterpret_cast<T*>(hsm + H::T_END64 + H::GROUPS * H::PER_GROUP_X);
    g.tN = t64;
    g.tW = t64 + H::T_W;
    g.tB = tt;
    g.tPhi = tt + H::T_PHI;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    g.grp = lane / H::G;
    g.l = lane % H::G;
    const int gid = warp * H::CPW + g.grp;
    g.sX = hsm + H::T_END64 + gid * H::PER_GROUP_X;
    T* sg = tt + H::T_ENDT + gid * H::PER_GROUP_T;
    g.su = sg;
    g.sF = sg + H::OFF_F;
    g.sF0 = sg + H::OFF_F0;
    return g;
}

// The CPW cells base .. base + CPW - 1 of p, one per group of lanes of the calling warp (every
// lane of the warp calls it: it synchronises the warp).
template <int CELL, int RHEO, bool BF, int OP, typename T>
PL_D void hex_group_cells(const DomainParams& p, int64_t base, const HexGroupSmem<CELL, T>& g) {
    using H = HexGroup<CELL, T>;
    using L = AuxLayout<RHEO, BF>;
    const AuxOffsets<RHEO, BF> aoff;
    const double* tN = g.tN;
    const double* tW = g.tW;
    const T* tB = g.tB;
    const T* tPhi = g.tPhi;
    double* sX = g.sX;
    T* su = g.su;
    T* sF = g.sF;
    T* sF0 = g.sF0;
    const int grp = g.grp, l = g.l;
    const bool f32 = sizeof(T) == 4;
    {
        const int64_t c = base + grp;
        const bool live = c < p.ncells;
        const int64_t mc = live ? (p.cell_ids ? p.cell_ids[c] : c) : 0;
        int node = 0;
        if (live && l < H::NEN) {
            node = p.cells[mc * H::NEN + l];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (f32) su[l * 3 + k] = (T)p.v32[3 * (int64_t)node + k];
                else su[l * 3 + k] = (T)(OP == OP_RESIDUAL ? p.u : p.v)[3 * (int64_t)node + k];
            }
        }
        if (live && l < 8) {
            const int cn = p.cells[mc * H::NEN + Elem<CELL>::corner(l)];
#pragma unroll
            for (int k = 0; k < 3; ++k) sX[l * 3 + k] = p.coords[3 * (int64_t)cn + k];
        }
        __syncwarp();
        if (live && l < H::NQ) {
            const int q = l;
            T inv[3][3];
            T wdetJ;
            if constexpr (sizeof(T) == 4 && CELL == HEX8) {
                // FP32 Jacobian action: FP32 geometry from the corners relative to corner 0 (the
                // basis gradients sum to zero, so J is unchanged and no large coordinates cancel),
                // with the field-basis gradient table (the Q1 field basis is the geometry basis)
                float J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
                for (int k = 1; k < 8; ++k)
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        const float dx = (float)(sX[k * 3 + i] - sX[i]);
#pragma unroll
                        for (int j = 0; j < 3; ++j) J[i][j] += dx * tB[q * H::LDB + k * 3 + j];
                    }
                const float detJ = invert3(J, inv);
                if (!(detJ > 0.f)) flag_error(p.err, CHECK_NONPOSITIVE_DETJ);
                wdetJ = (float)tW[q] * detJ;
            } else {
                double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
                for (int k = 0; k < 8; ++k)
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int j = 0; j < 3; ++j) J[i][j] += sX[k * 3 + i] * tN[q * 25 + k * 3 + j];
                double inv64[3][3];
                const double detJ = invert3(J, inv64);
                if (!(detJ > 0.0)) flag_error(p.err, CHECK_NONPOSITIVE_DETJ);
                wdetJ = (T)(tW[q] * detJ);
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) inv[i][j] = (T)inv64[i][j];
            }
            // reference gradient of the field, then s_x = Gref J^{-1}
            T Gr[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll 9
            for (int n = 0; n < H::NEN; ++n) {
                const T b0 = tB[q * H::LDB + n * 3], b1 = tB[q * H::LDB + n * 3 + 1], b2 = tB[q * H::LDB + n * 3 + 2];
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) {
                    const T un = su[n * 3 + cc];
                    Gr[cc][0] += un * b0;
                    Gr[cc][1] += un * b1;
                    Gr[cc][2] += un * b2;
                }
            }
            T s_x[9];
#pragma unroll
            for (int cc = 0; cc < 3; ++cc)
#pragma unroll
                for (int e = 0; e < 3; ++e)
                    s_x[cc * 3 + e] = Gr[cc][0] * inv[0][e] + Gr[cc][1] * inv[1][e] + Gr[cc][2] * inv[2][e];
            double a[L::size] = {};
            const bool cached = f32 && OP == OP_JACOBIAN_ACTION && p.lm32;
            if (!cached) L::load_cell(p, c, a);
            if (OP == OP_RESIDUAL) L::load_qp(p, c, q, H::NQ, a);  // the tangents read no state
            double x[3] = {0, 0, 0}, s[3] = {0, 0, 0};
            double f0[3] = {0, 0, 0};
            T f1[9];
            if (cached) {
                isotropic_contract<T>((T)p.lm32[2 * c], (T)p.lm32[2 * c + 1], s_x, f1);
            } else if (OP == OP_RESIDUAL) {
                double s_x64[9], f164[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
                for (int i = 0; i < 9; ++i) s_x64[i] = (double)s_x[i];
                if (BF) {
                    const int sOff[1] = {0}, sOff_x[1] = {0};
                    pw::g0v_bodyforce<double>(3, 1, L::numA, sOff, sOff_x, s, nullptr, s_x64, aoff.v, nullptr, a,
                                              nullptr, nullptr, p.t, x, p.num_constants, p.constants, f0);
                }
                call_f1<RHEO>(L::numA, aoff.v, a, s, s_x64, p, x, f164);
#pragma unroll
                for (int i = 0; i < 9; ++i) f1[i] = (T)f164[i];
            } else {
                double Jf3[81];
#pragma unroll
                for (int i = 0; i < 81; ++i) Jf3[i] = 0.0;
                call_jf3<RHEO>(L::numA, aoff.v, a, p, x, Jf3);
                isotropic_jf3_contract<RHEO>(Jf3, s_x, f1);
            }
            // test-function weights: grad(phi_n) . f1 = tB_n . (J^{-1} f1^T), so stage
            // W[cc][d] = wdetJ sum_e inv[d][e] f1[cc][e]
#pragma unroll
            for (int cc = 0; cc < 3; ++cc)
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    sF[q * 9 + cc * 3 + d] =
                        wdetJ * (inv[d][0] * f1[cc * 3 + 0] + inv[d][1] * f1[cc * 3 + 1] + inv[d][2] * f1[cc * 3 + 2]);
            if (BF && OP == OP_RESIDUAL)
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) sF0[q * 3 + cc] = wdetJ * (T)f0[cc];
        }
        __syncwarp();
        if (live && l < H::NEN) {
            const int n = l;
            T r0 = 0, r1 = 0, r2 = 0;
#pragma unroll 9
            for (int q = 0; q < H::NQ; ++q) {
                const T b0 = tB[q * H::LDB + n * 3], b1 = tB[q * H::LDB + n * 3 + 1], b2 = tB[q * H::LDB + n * 3 + 2];
                const T* w = sF + q * 9;
                r0 += b0 * w[0] + b1 * w[1] + b2 * w[2];
                r1 += b0 * w[3] + b1 * w[4] + b2 * w[5];
                r2 += b0 * w[6] + b1 * w[7] + b2 * w[8];
                if (BF && OP == OP_RESIDUAL) {
                    const T ph = tPhi[q * H::NEN + n];
                    r0 += ph * sF0[q * 3 + 0];
                    r1 += ph * sF0[q * 3 + 1];
                    r2 += ph * sF0[q * 3 + 2];
                }
            }
            if (f32) {
                float* o = p.out32 + 3 * (int64_t)node;
                red_add(o, (float)r0);
                red_add(o + 1, (float)r1);
                red_add(o + 2, (float)r2);
            } else {
                double* o = p.out + 3 * (int64_t)node;
                red_add(o, (double)r0);
                red_add(o + 1, (double)r1);
                red_add(o + 2, (double)r2);
            }
        }
        __syncwarp();
    }
}

// T = double: residual (OP_RESIDUAL) or Jacobian action into p.out from p.u / p.v;
// T = float: Jacobian action into p.out32 from p.v32.
template <int CELL, int RHEO, bool BF, int OP, typename T>
__global__ void __launch_bounds__(HexGroup<CELL, T>::WARPS * 32) k_hex_group(DomainParams p) {
    using H = HexGroup<CELL, T>;
    extern __shared__ __align__(16) double hsm[];
    fill_tables<CELL, T>(hsm, reinterpret_cast<T*>(hsm + H::T_END64 + H::GROUPS * H::PER_GROUP_X));
    __syncthreads();
    const HexGroupSmem<CELL, T> g = hex_group_smem<CELL, T>(hsm);
    const int warp = threadIdx.x >> 5;
    const int64_t cells_per_pass = (int64_t)gridDim.x * H::WARPS * H::CPW;
    // every lane of a warp runs the same number of passes (the __syncwarp calls need them all)
    for (int64_t base = ((int64_t)blockIdx.x * H::WARPS + warp) * H::CPW; base < p.ncells; base += cells_per_pass)
        hex_group_cells<CELL, RHEO, BF, OP, T>(p, base, g);
}

// FP32 Jacobian action of Q1 hexahedra over the cells of many meshes in one launch (the ragged
// batch of solvers, ragged.cu): member m's cells form warp chunks chunk0[m] .. chunk0[m + 1] - 1
// of one index space (4 cells per chunk), so a warp never mixes members; ops[m] holds member m's
// operator arguments (its own cells, coordinates, cached per-cell tangent, input and output).
// Members must have the cached isotropic tangent (lm32).
__global__ void __launch_bounds__(HexGroup<HEX8, float>::WARPS * 32)
    k_hex8_jv32_ragged(const DomainParams* __restrict__ ops, const int64_t* __restrict__ chunk0,
                       const int* __restrict__ active, const int* __restrict__ nmembers) {
    using H = HexGroup<HEX8, float>;
    extern __shared__ __align__(16) double hsm[];
    fill_tables<HEX8, float>(hsm, reinterpret_cast<float*>(hsm + H::T_END64 + H::GROUPS * H::PER_GROUP_X));
    __syncthreads();
    const HexGroupSmem<HEX8, float> g = hex_group_smem<HEX8, float>(hsm);
    const int M = *nmembers;
    const int64_t total = chunk0[M];
    const int warp = threadIdx.x >> 5;
    for (int64_t w = (int64_t)blockIdx.x * H::WARPS + warp; w < total; w += (int64_t)gridDim.x * H::WARPS) {
        int lo = 0, hi = M;  // the member of chunk w: largest m with chunk0[m] <= w
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (chunk0[mid] <= w) lo = mid;
            else hi = mid;
        }
        if (!active[lo]) continue;  // the whole warp shares w
        hex_group_cells<HEX8, RHEO_ILE, false, OP_JACOBIAN_ACTION, float>(ops[lo], (w - chunk0[lo]) * H::CPW, g);
    }
}

void launch_hex8_jv32_ragged(const DomainParams* ops, const int64_t* chunk0, const int* active, const int* nmembers,
                             cudaStream_t s) {
    using H = HexGroup<HEX8, float>;
    const size_t smem = H::smem_bytes();
    static int per_sm = 0, nsm = 0;
    if (!per_sm) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        ensure_kernel_smem((const void*)k_hex8_jv32_ragged, smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_hex8_jv32_ragged, H::WARPS * 32, smem);
        per_sm = std::max(per_sm, 1);
    }
    k_hex8_jv32_ragged<<<nsm * per_sm, H::WARPS * 32, smem, s>>>(ops, chunk0, active, nmembers);
}

// ---- Q2 hexahedra by sum factorisation --------------------------------------------------------
// One warp per cell, lane l = i + 3 j + 9 k (27 lanes). The Q2 basis is a tensor product of the
// 1-D quadratic basis, so the reference gradient of the field at the 27 Gauss points is three
// 1-D contractions (x, then y, then z) with the 3×3 value (B) and derivative (D) matrices, one
// lane per output entry, staged through shared memory; the test-function contraction runs the
// same stages in reverse. Per lane this is ~145 multiply-adds for the two contractions instead
// of ~490 with the full 27×27 tables, and as many fewer shared-memory reads.
struct SumFact {
    static constexpr int WARPS = 4;
    // block tables (doubles): B[3][3], D[3][3] (point i, node a), geometry gradients [27][25],
    // weights [27]
    static constexpr int T_D = 9, T_N = 18, T_W = T_N + 27 * 25, T_END = T_W + 27;
    // per warp (doubles): su[3][27] field, S[9][27] stage buffer, R[9][27] stage buffer,
    // W[12][27] test weights (9 gradient + 3 value), X[8][3]; odd stride
    static constexpr int O_S = 81, O_R = O_S + 243, O_W = O_R + 243, O_X = O_W + 324;
    static constexpr int PER_WARP = (O_X + 24) | 1;
    static constexpr size_t smem_bytes() { return sizeof(double) * ((size_t)T_END + (size_t)WARPS * PER_WARP); }
};

template <int RHEO, bool BF, int OP, typename T>
__global__ void __launch_bounds__(SumFact::WARPS * 32) k_hex27_sumfact(DomainParams p) {
    using SF = SumFact;
    using L = AuxLayout<RHEO, BF>;
    const AuxOffsets<RHEO, BF> aoff;
    extern __shared__ __align__(16) double fsm[];
    double* tB = fsm;
    double* tD = fsm + SF::T_D;
    double* tN = fsm + SF::T_N;
    double* tW = fsm + SF::T_W;
    for (int i = threadIdx.x; i < 9; i += blockDim.x) {
        const double x = gauss3_x(i / 3);
        tB[i] = quad_v(i % 3, x);
        tD[i] = quad_d(i % 3, x);
    }
    for (int i = threadIdx.x; i < 27 * 8; i += blockDim.x) {
        const int q = i / 8, c = i % 8;
        double d[3];
        hex_corner_dN<3>(c, q % 3, (q / 3) % 3, q / 9, d);
#pragma unroll
        for (int k = 0; k < 3; ++k) tN[q * 25 + c * 3 + k] = d[k];
    }
    for (int q = threadIdx.x; q < 27; q += blockDim.x) tW[q] = gauss3_w(q % 3) * gauss3_w((q / 3) % 3) * gauss3_w(q / 9);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double* wb = fsm + SF::T_END + warp * SF::PER_WARP;
    double* su = wb;            // [c][27] node values
    double* S = wb + SF::O_S;   // stage buffer [9][27]
    double* R = wb + SF::O_R;   // stage buffer [9][27]
    double* W = wb + SF::O_W;   // [12][27]: test weights per point, gradient part [c*3+d], value part [9+c]
    double* sX = wb + SF::O_X;
    const bool act = lane < 27;
    const int i0 = lane % 3, i1 = (lane / 3) % 3, i2 = lane / 9;  // this lane's (x, y, z) index
    const bool f32 = sizeof(T) == 4;
    for (int64_t c = (int64_t)blockIdx.x * SF::WARPS + warp; c < p.ncells; c += (int64_t)gridDim.x * SF::WARPS) {
        const int64_t mc = p.cell_ids ? p.cell_ids[c] : c;
        int node = 0;
        if (act) {
            node = p.cells[mc * 27 + lane];
#pragma unroll
            for (int k = 0; k < 3; ++k)
                su[k * 27 + lane] = f32 ? (double)p.v32[3 * (int64_t)node + k]
                                        : (OP == OP_RESIDUAL ? p.u : p.v)[3 * (int64_t)node + k];
        }
        if (lane < 8) {
            const int cn = p.cells[mc * 27 + Elem<HEX27>::corner(lane)];
#pragma unroll
            for (int k = 0; k < 3; ++k) sX[lane * 3 + k] = p.coords[3 * (int64_t)cn + k];
        }
        __syncwarp();
        // stage 1 (x): lane (i, b, c3): U_B, U_D [comp][lane]
        if (act) {
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
                const double* u = su + cc * 27 + 3 * i1 + 9 * i2;
                double vb = 0.0, vd = 0.0;
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    vb += tB[i0 * 3 + a] * u[a];
                    vd += tD[i0 * 3 + a] * u[a];
                }
                S[cc * 27 + lane] = vb;        // B in x
                S[(3 + cc) * 27 + lane] = vd;  // D in x
            }
        }
        __syncwarp();
        // stage 2 (y): lane (i, j, c3): BB, BD (y derivative), DB (x derivative)
        if (act) {
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
                const double* ub = S + cc * 27 + i0 + 9 * i2;
                const double* ud = S + (3 + cc) * 27 + i0 + 9 * i2;
                double bb = 0.0, bd = 0.0, db = 0.0;
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    bb += tB[i1 * 3 + b] * ub[3 * b];
                    bd += tD[i1 * 3 + b] * ub[3 * b];
                    db += tB[i1 * 3 + b] * ud[3 * b];
                }
                R[cc * 27 + lane] = bb;
                R[(3 + cc) * 27 + lane] = bd;
                R[(6 + cc) * 27 + lane] = db;
            }
        }
        __syncwarp();
        if (act) {
            const int q = lane;
            // stage 3 (z): reference gradient at point (i, j, k)
            double Gr[3][3];
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
                const double* bb = R + cc * 27 + i0 + 3 * i1;
                const double* bd = R + (3 + cc) * 27 + i0 + 3 * i1;
                const double* db = R + (6 + cc) * 27 + i0 + 3 * i1;
                double gx = 0.0, gy = 0.0, gz = 0.0;
#pragma unroll
                for (int c3 = 0; c3 < 3; ++c3) {
                    gx += tB[i2 * 3 + c3] * db[9 * c3];
                    gy += tB[i2 * 3 + c3] * bd[9 * c3];
                    gz += tD[i2 * 3 + c3] * bb[9 * c3];
                }
                Gr[cc][0] = gx;
                Gr[cc][1] = gy;
                Gr[cc][2] = gz;
            }
            double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
            for (int k = 0; k < 8; ++k)
#pragma unroll
                for (int ii = 0; ii < 3; ++ii)
#pragma unroll
                    for (int jj = 0; jj < 3; ++jj) J[ii][jj] += sX[k * 3 + ii] * tN[q * 25 + k * 3 + jj];
            double inv[3][3];
            const double detJ = invert3(J, inv);
            if (!(detJ > 0.0)) flag_error(p.err, CHECK_NONPOSITIVE_DETJ);
            const double wdetJ = tW[q] * detJ;
            double s_x[9];
#pragma unroll
            for (int cc = 0; cc < 3; ++cc)
#pragma unroll
                for (int e = 0; e < 3; ++e)
                    s_x[cc * 3 + e] = Gr[cc][0] * inv[0][e] + Gr[cc][1] * inv[1][e] + Gr[cc][2] * inv[2][e];
            if (f32)
#pragma unroll
                for (int e = 0; e < 9; ++e) s_x[e] = (double)(float)s_x[e];
            double a[L::size] = {};
            L::load_cell(p, c, a);
            if (OP == OP_RESIDUAL) L::load_qp(p, c, q, 27, a);  // the tangents read no state
            double x[3] = {0, 0, 0}, s3[3] = {0, 0, 0};
            double f0[3] = {0, 0, 0}, f1[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            if (OP == OP_RESIDUAL) {
                if (BF) {
                    const int sOff[1] = {0}, sOff_x[1] = {0};
                    pw::g0v_bodyforce<double>(3, 1, L::numA, sOff, sOff_x, s3, nullptr, s_x, aoff.v, nullptr, a,
                                              nullptr, nullptr, p.t, x, p.num_constants, p.constants, f0);
                }
                call_f1<RHEO>(L::numA, aoff.v, a, s3, s_x, p, x, f1);
            } else {
                double Jf3[81];
#pragma unroll
                for (int ii = 0; ii < 81; ++ii) Jf3[ii] = 0.0;
                call_jf3<RHEO>(L::numA, aoff.v, a, p, x, Jf3);
                isotropic_jf3_contract<RHEO>(Jf3, s_x, f1);
            }
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    W[(cc * 3 + d) * 27 + q] =
                        wdetJ * (inv[d][0] * f1[cc * 3 + 0] + inv[d][1] * f1[cc * 3 + 1] + inv[d][2] * f1[cc * 3 + 2]);
                W[(9 + cc) * 27 + q] = (BF && OP == OP_RESIDUAL) ? wdetJ * f0[cc] : 0.0;
            }
        }
        __syncwarp();
        // reverse stage 3 (over k): lane (i, j, c3): Tx, Ty, Tz, T0 [comp]
        if (act) {
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
                const double* wx = W + (cc * 3 + 0) * 27 + i0 + 3 * i1;
                const double* wy = W + (cc * 3 + 1) * 27 + i0 + 3 * i1;
                const double* wz = W + (cc * 3 + 2) * 27 + i0 + 3 * i1;
                const double* w0 = W + (9 + cc) * 27 + i0 + 3 * i1;
                double tx = 0.0, ty = 0.0, tz = 0.0, t0 = 0.0;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const double bk = tB[k * 3 + i2], dk = tD[k * 3 + i2];
                    tx += bk * wx[9 * k];
                    ty += bk * wy[9 * k];
                    tz += dk * wz[9 * k];
                    if (BF && OP == OP_RESIDUAL) t0 += bk * w0[9 * k];
                }
                S[cc * 27 + lane] = tx;
                S[(3 + cc) * 27 + lane] = ty;
                S[(6 + cc) * 27 + lane] = tz;
                if (BF && OP == OP_RESIDUAL) R[cc * 27 + lane] = t0;
            }
        }
        __syncwarp();
        // reverse stage 2 (over j): lane (i, b, c3): QD (x-derivative channel), QB (the others)
        double qd[3], qb[3];
        if (act) {
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
                const double* tx = S + cc * 27 + i0 + 9 * i2;
                const double* ty = S + (3 + cc) * 27 + i0 + 9 * i2;
                const double* tz = S + (6 + cc) * 27 + i0 + 9 * i2;
                const double* t0 = R + cc * 27 + i0 + 9 * i2;
                double px = 0.0, py = 0.0, pz = 0.0;
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const double bj = tB[j * 3 + i1], dj = tD[j * 3 + i1];
                    px += bj * tx[3 * j];
                    py += dj * ty[3 * j];
                    pz += bj * tz[3 * j];
                    if (BF && OP == OP_RESIDUAL) pz += bj * t0[3 * j];
                }
                qd[cc] = px;
                qb[cc] = py + pz;
            }
        }
        __syncwarp();
        if (act)
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
                S[cc * 27 + lane] = qd[cc];
                S[(3 + cc) * 27 + lane] = qb[cc];
            }
        __syncwarp();
        // reverse stage 1 (over i): lane = node (a, b, c3)
        if (act) {
            double r[3];
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
                const double* pd = S + cc * 27 + 3 * i1 + 9 * i2;
                const double* pb = S + (3 + cc) * 27 + 3 * i1 + 9 * i2;
                double acc = 0.0;
#pragma unroll
                for (int ii = 0; ii < 3; ++ii) acc += tD[ii * 3 + i0] * pd[ii] + tB[ii * 3 + i0] * pb[ii];
                r[cc] = acc;
            }
            if (f32) {
                float* o = p.out32 + 3 * (int64_t)node;
                red_add(o, (float)r[0]);
                red_add(o + 1, (float)r[1]);
                red_add(o + 2, (float)r[2]);
            } else {
                double* o = p.out + 3 * (int64_t)node;
                red_add(o, r[0]);
                red_add(o + 1, r[1]);
                red_add(o + 2, r[2]);
            }
        }
        __syncwarp();
    }
}

// Q2 hexahedra by sum factorisation with one 1-D line of 3 points per lane: a warp holds 3
// cells, 9 lanes each. A 1-D pass along a line runs in the lane's registers; the values move
// through shared memory only when the pass direction changes (x-lines, y-lines, z-lines: lane l
// of a cell owns the line with fixed indices (l % 3, l / 3) in the other two directions). The
// pointwise stage runs on the z-lines, each lane evaluating its line's 3 Gauss points one after
// the other. Compared with one point per lane (k_hex27_sumfact, where every pass reads three
// neighbours from a stage buffer and writes one value), this moves each staged value through
// shared memory once per direction change instead of once per pass.
struct Lines {
    static constexpr int WARPS = 2;
    static constexpr int T_D = 9, T_W = 18, T_END = 18 + 27;  // B[3][3], D[3][3] (point i, node a), weights[27]
    // per cell: A and Bf stage buffers [12][27] each, corner coordinates [8][3]. The cell stride,
    // 11 modulo the 16 eight-byte bank pairs, staggers the three cells of a warp; with the point
    // orders of the kernel a warp's line accesses take 2 or 3 shared-memory wavefronts (2 is the
    // least for 27 eight-byte accesses).
    static constexpr int O_B = 12 * 27, O_X = 24 * 27, CS = 683;
    static_assert(CS >= O_X + 24 && CS % 16 == 11, "cell stride");
    static constexpr size_t smem_bytes() { return sizeof(double) * ((size_t)T_END + (size_t)WARPS * 3 * CS); }
};

template <int RHEO, bool BF, int OP>
__global__ void __launch_bounds__(Lines::WARPS * 32) k_hex27_lines(DomainParams p) {
    using LN = Lines;
    using L = AuxLayout<RHEO, BF>;
    const AuxOffsets<RHEO, BF> aoff;
    extern __shared__ __align__(16) double lsm[];
    double* tB = lsm;
    double* tD = lsm + LN::T_D;
    double* tW = lsm + LN::T_W;
    for (int i = threadIdx.x; i < 9; i += blockDim.x) {
        const double x = gauss3_x(i / 3);
        tB[i] = quad_v(i % 3, x);
        tD[i] = quad_d(i % 3, x);
    }
    for (int q = threadIdx.x; q < 27; q += blockDim.x) tW[q] = gauss3_w(q % 3) * gauss3_w((q / 3) % 3) * gauss3_w(q / 9);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool inwarp = lane < 27;
    const int g = inwarp ? lane / 9 : 0, l = inwarp ? lane - 9 * (lane / 9) : 0;
    const int la = l % 3, lb = l / 3;
    double* cb = lsm + LN::T_END + (warp * 3 + g) * LN::CS;
    double* A = cb;
    double* Bf = cb + LN::O_B;
    double* sX = cb + LN::O_X;
    const double* __restrict__ field = OP == OP_RESIDUAL ? p.u : p.v;
    // Position of point (i0, i1, i2) in a stage buffer: two orders, each keeping both the
    // writing and the reading lines of its transposes on distinct banks within a cell
    // (i0 + 3 i1 + 9 i2 would put a y-line's 9 lanes on 7 bank pairs).
    auto iy = [](int a0, int a1, int a2) { return a0 + 9 * a1 + 3 * a2; };  // x <-> y transposes
    auto iz = [](int a0, int a1, int a2) { return 3 * a0 + a1 + 9 * a2; };  // y <-> z and the z stage
    const int64_t stride = (int64_t)gridDim.x * LN::WARPS * 3;
    // every lane of a warp runs the same number of passes (the __syncwarp calls need them all)
    for (int64_t c0 = ((int64_t)blockIdx.x * LN::WARPS + warp) * 3; c0 < p.ncells; c0 += stride) {
        const int64_t c = c0 + g;
        const bool live = inwarp && c < p.ncells;
        const int64_t mc = live ? (p.cell_ids ? p.cell_ids[c] : c) : 0;
        // x-line (i1, i2) = (la, lb): the nodes a + 3 la + 9 lb
        int nodes[3] = {0, 0, 0};
        double u[3][3];
        if (live) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                nodes[a] = p.cells[mc * 27 + a + 3 * la + 9 * lb];
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) u[a][cc] = field[3 * (int64_t)nodes[a] + cc];
            }
            if (l < 8) {
                const int cn = p.cells[mc * 27 + Elem<HEX27>::corner(l)];
#pragma unroll
                for (int k = 0; k < 3; ++k) sX[l * 3 + k] = p.coords[3 * (int64_t)cn + k];
            }
            // forward x: B u and D u along the line
#pragma unroll
            for (int cc = 0; cc < 3; ++cc)
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    double vb = 0.0, vd = 0.0;
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        vb += tB[i * 3 + a] * u[a][cc];
                        vd += tD[i * 3 + a] * u[a][cc];
                    }
                    A[cc * 27 + iy(i, la, lb)] = vb;
                    A[(3 + cc) * 27 + iy(i, la, lb)] = vd;
                }
        }
        __syncwarp();
        // forward y on y-lines (i0, i2) = (la, lb): BB, BD (y derivative), DB (x derivative)
        if (live) {
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
                double bx[3], dx[3];
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    bx[b] = A[cc * 27 + iy(la, b, lb)];
                    dx[b] = A[(3 + cc) * 27 + iy(la, b, lb)];
                }
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    double bb = 0.0, bd = 0.0, db = 0.0;
#pragma unroll
                    for (int b = 0; b < 3; ++b) {
                        bb += tB[j * 3 + b] * bx[b];
                        bd += tD[j * 3 + b] * bx[b];
                        db += tB[j * 3 + b] * dx[b];
                    }
                    Bf[cc * 27 + iz(la, j, lb)] = bb;
                    Bf[(3 + cc) * 27 + iz(la, j, lb)] = bd;
                    Bf[(6 + cc) * 27 + iz(la, j, lb)] = db;
                }
            }
        }
        __syncwarp();
        // z-lines (i0, i1) = (la, lb): forward z, geometry and the pointwise function at the
        // line's 3 Gauss points; the test-function weights go to A at the points' positions
        if (live) {
            double a[L::size] = {};
            L::load_cell(p, c, a);
#pragma unroll 1
            for (int k = 0; k < 3; ++k) {
                const int q = la + 3 * lb + 9 * k;
                double Gr[3][3];
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) {
                    double gx = 0.0, gy = 0.0, gz = 0.0;
#pragma unroll
                    for (int c3 = 0; c3 < 3; ++c3) {
                        const int pt = iz(la, lb, c3);
                        gx += tB[k * 3 + c3] * Bf[(6 + cc) * 27 + pt];
                        gy += tB[k * 3 + c3] * Bf[(3 + cc) * 27 + pt];
                        gz += tD[k * 3 + c3] * Bf[cc * 27 + pt];
                    }
                    Gr[cc][0] = gx;
                    Gr[cc][1] = gy;
                    Gr[cc][2] = gz;
                }
                double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
                for (int cr = 0; cr < 8; ++cr) {
                    double d[3];
                    hex_corner_dN<3>(cr, la, lb, k, d);
#pragma unroll
                    for (int ii = 0; ii < 3; ++ii)
#pragma unroll
                        for (int jj = 0; jj < 3; ++jj) J[ii][jj] += sX[cr * 3 + ii] * d[jj];
                }
                double inv[3][3];
                const double detJ = invert3(J, inv);
                if (!(detJ > 0.0)) flag_error(p.err, CHECK_NONPOSITIVE_DETJ);
                const double wdetJ = tW[q] * detJ;
                double s_x[9];
#pragma unroll
                for (int cc = 0; cc < 3; ++cc)
#pragma unroll
                    for (int e = 0; e < 3; ++e)
                        s_x[cc * 3 + e] = Gr[cc][0] * inv[0][e] + Gr[cc][1] * inv[1][e] + Gr[cc][2] * inv[2][e];
                if (OP == OP_RESIDUAL) L::load_qp(p, c, q, 27, a);  // the tangents read no state
                double x[3] = {0, 0, 0}, s3[3] = {0, 0, 0};
                double f0[3] = {0, 0, 0}, f1[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
                if (OP == OP_RESIDUAL) {
                    if (BF) {
                        const int sOff[1] = {0}, sOff_x[1] = {0};
                        pw::g0v_bodyforce<double>(3, 1, L::numA, sOff, sOff_x, s3, nullptr, s_x, aoff.v, nullptr, a,
                                                  nullptr, nullptr, p.t, x, p.num_constants, p.constants, f0);
                    }
                    call_f1<RHEO>(L::numA, aoff.v, a, s3, s_x, p, x, f1);
                } else {
                    double Jf3[81];
#pragma unroll
                    for (int ii = 0; ii < 81; ++ii) Jf3[ii] = 0.0;
                    call_jf3<RHEO>(L::numA, aoff.v, a, p, x, Jf3);
                    isotropic_jf3_contract<RHEO>(Jf3, s_x, f1);
                }
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) {
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        A[(cc * 3 + d) * 27 + iz(la, lb, k)] =
                            wdetJ * (inv[d][0] * f1[cc * 3 + 0] + inv[d][1] * f1[cc * 3 + 1] + inv[d][2] * f1[cc * 3 + 2]);
                    if (BF && OP == OP_RESIDUAL) A[(9 + cc) * 27 + iz(la, lb, k)] = wdetJ * f0[cc];
                }
            }
            // reverse z on the same line (this lane's own points): Tx, Ty, Tz, T0 into Bf
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
                double wx[3], wy[3], wz[3], w0[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const int pt = iz(la, lb, k);
                    wx[k] = A[(cc * 3 + 0) * 27 + pt];
                    wy[k] = A[(cc * 3 + 1) * 27 + pt];
                    wz[k] = A[(cc * 3 + 2) * 27 + pt];
                    w0[k] = (BF && OP == OP_RESIDUAL) ? A[(9 + cc) * 27 + pt] : 0.0;
                }
#pragma unroll
                for (int c3 = 0; c3 < 3; ++c3) {
                    double tx = 0.0, ty = 0.0, tz = 0.0, t0 = 0.0;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const double bk = tB[k * 3 + c3], dk = tD[k * 3 + c3];
                        tx += bk * wx[k];
                        ty += bk * wy[k];
                        tz += dk * wz[k];
                        if (BF && OP == OP_RESIDUAL) t0 += bk * w0[k];
                    }
                    const int pt = iz(la, lb, c3);
                    Bf[cc * 27 + pt] = tx;
                    Bf[(3 + cc) * 27 + pt] = ty;
                    Bf[(6 + cc) * 27 + pt] = tz + t0;
                }
            }
        }
        __syncwarp();
        // reverse y on y-lines (i0, i2) = (la, lb): QD (x-derivative channel), QB (the others)
        if (live) {
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
                double tx[3], ty[3], tz[3];
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const int pt = iz(la, j, lb);
                    tx[j] = Bf[cc * 27 + pt];
                    ty[j] = Bf[(3 + cc) * 27 + pt];
                    tz[j] = Bf[(6 + cc) * 27 + pt];
                }
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    double px = 0.0, py = 0.0, pz = 0.0;
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        const double bj = tB[j * 3 + b], dj = tD[j * 3 + b];
                        px += bj * tx[j];
                        py += dj * ty[j];
                        pz += bj * tz[j];
                    }
                    const int pt = iy(la, b, lb);
                    A[cc * 27 + pt] = px;
                    A[(3 + cc) * 27 + pt] = py + pz;
                }
            }
        }
        __syncwarp();
        // reverse x on x-lines (i1, i2) = (la, lb): node values, added into the output
        if (live) {
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
                double qd[3], qb[3];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    qd[i] = A[cc * 27 + iy(i, la, lb)];
                    qb[i] = A[(3 + cc) * 27 + iy(i, la, lb)];
                }
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    double r = 0.0;
#pragma unroll
                    for (int i = 0; i < 3; ++i) r += tD[i * 3 + a] * qd[i] + tB[i * 3 + a] * qb[i];
                    red_add(p.out + 3 * (int64_t)nodes[a] + cc, r);
                }
            }
        }
        __syncwarp();
    }
}

template <int RHEO, bool BF, int OP>
static void launch_lines_t(const DomainParams& p, cudaStream_t s) {
    auto kern = k_hex27_lines<RHEO, BF, OP>;
    const size_t smem = Lines::smem_bytes();
    ensure_kernel_smem((const void*)kern, smem);
    const int nsm = sm_count();
    static int per_sm = 0;  // occupancy of this instantiation (the same on every B200)
    if (!per_sm) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Lines::WARPS * 32, smem);
        per_sm = std::max(per_sm, 1);
    }
    const int64_t blocks = (p.ncells + 3 * Lines::WARPS - 1) / (3 * Lines::WARPS);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(blocks, (int64_t)nsm * std::max(per_sm, 1)));
    kern<<<grid, Lines::WARPS * 32, smem, s>>>(p);
    count_launch();
}

#ifndef PLB_Q2_LINES
#define PLB_Q2_LINES 1
#endif

static void launch_lines(const DomainParams& p, int rheo, bool bf, int op, cudaStream_t s) {
    if (op == OP_RESIDUAL) {
        if (rheo == RHEO_ILE) {
            if (bf) launch_lines_t<RHEO_ILE, true, OP_RESIDUAL>(p, s);
            else launch_lines_t<RHEO_ILE, false, OP_RESIDUAL>(p, s);
        } else {
            if (bf) launch_lines_t<RHEO_GENMAXWELL, true, OP_RESIDUAL>(p, s);
            else launch_lines_t<RHEO_GENMAXWELL, false, OP_RESIDUAL>(p, s);
        }
    } else {
        if (rheo == RHEO_ILE) launch_lines_t<RHEO_ILE, false, OP_JACOBIAN_ACTION>(p, s);
        else launch_lines_t<RHEO_GENMAXWELL, false, OP_JACOBIAN_ACTION>(p, s);
    }
}

template <int RHEO, bool BF, int OP, typename T = double>
static void launch_sumfact_t(const DomainParams& p, cudaStream_t s) {
    auto kern = k_hex27_sumfact<RHEO, BF, OP, T>;
    const size_t smem = SumFact::smem_bytes();
    ensure_kernel_smem((const void*)kern, smem);
    const int nsm = sm_count();
    static int per_sm = 0;  // occupancy of this instantiation (the same on every B200)
    if (!per_sm) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, SumFact::WARPS * 32, smem);
        per_sm = std::max(per_sm, 1);
    }
    const int64_t blocks = (p.ncells + SumFact::WARPS - 1) / SumFact::WARPS;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(blocks, (int64_t)nsm * std::max(per_sm, 1)));
    kern<<<grid, SumFact::WARPS * 32, smem, s>>>(p);
    count_launch();
}

template <int CELL, int RHEO, bool BF, int OP, typename T = double>
static void launch_group_t(const DomainParams& p, cudaStream_t s) {
    using H = HexGroup<CELL, T>;
    auto kern = k_hex_group<CELL, RHEO, BF, OP, T>;
    const size_t smem = H::smem_bytes();
    ensure_kernel_smem((const void*)kern, smem);
    const int nsm = sm_count();
    static int per_sm = 0;  // occupancy of this instantiation (the same on every B200)
    if (!per_sm) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, H::WARPS * 32, smem);
        per_sm = std::max(per_sm, 1);
    }
    const int64_t groups = (p.ncells + H::WARPS * H::CPW - 1) / (H::WARPS * H::CPW);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(groups, (int64_t)nsm * std::max(per_sm, 1)));
    kern<<<grid, H::WARPS * 32, smem, s>>>(p);
    count_launch();
}

template <int CELL>
static void launch_group_cell(const DomainParams& p, int rheo, bool bf, int op, cudaStream_t s) {
    if (op == OP_RESIDUAL) {
        if (rheo == RHEO_ILE) {
            if (bf) launch_group_t<CELL, RHEO_ILE, true, OP_RESIDUAL>(p, s);
            else launch_group_t<CELL, RHEO_ILE, false, OP_RESIDUAL>(p, s);
        } else {
            if (bf) launch_group_t<CELL, RHEO_GENMAXWELL, true, OP_RESIDUAL>(p, s);
            else launch_group_t<CELL, RHEO_GENMAXWELL, false, OP_RESIDUAL>(p, s);
        }
    } else {
        if (rheo == RHEO_ILE) launch_group_t<CELL, RHEO_ILE, false, OP_JACOBIAN_ACTION>(p, s);
        else launch_group_t<CELL, RHEO_GENMAXWELL, false, OP_JACOBIAN_ACTION>(p, s);
    }
}

#ifndef PLB_Q2_SUMFACT
#define PLB_Q2_SUMFACT 1
#endif

static void launch_sumfact(const DomainParams& p, int rheo, bool bf, int op, cudaStream_t s) {
    if (op == OP_RESIDUAL) {
        if (rheo == RHEO_ILE) {
            if (bf) launch_sumfact_t<RHEO_ILE, true, OP_RESIDUAL>(p, s);
            else launch_sumfact_t<RHEO_ILE, false, OP_RESIDUAL>(p, s);
        } else {
            if (bf) launch_sumfact_t<RHEO_GENMAXWELL, true, OP_RESIDUAL>(p, s);
            else launch_sumfact_t<RHEO_GENMAXWELL, false, OP_RESIDUAL>(p, s);
        }
    } else {
        if (rheo == RHEO_ILE) launch_sumfact_t<RHEO_ILE, false, OP_JACOBIAN_ACTION>(p, s);
        else launch_sumfact_t<RHEO_GENMAXWELL, false, OP_JACOBIAN_ACTION>(p, s);
    }
}

bool launch_domain_apply_hexgroup(const DomainParams& p, int cell, int rheo, bool bf, int op, cudaStream_t s) {
    if (p.ncells == 0) return true;
    if (cell == HEX8) launch_group_cell<HEX8>(p, rheo, bf, op, s);
    else if (cell == HEX27 && PLB_Q2_LINES) launch_lines(p, rheo, bf, op, s);
    else if (cell == HEX27 && PLB_Q2_SUMFACT) launch_sumfact(p, rheo, bf, op, s);
    else if (cell == HEX27) launch_group_cell<HEX27>(p, rheo, bf, op, s);
    else return false;
    return true;
}

// (lambda, mu) of the isotropic tangent per integrator cell at p.t, p.dt, from the registered
// Jacobian kernel: the FP32 Jacobian action of hexahedra reads them instead of evaluating the
// tangent (for generalized Maxwell, three exponentials in FP64) at each quadrature point.
template <int RHEO>
__global__ void k_tangent_lm32(DomainParams p, float* __restrict__ out) {
    using L = AuxLayout<RHEO, false>;
    const AuxOffsets<RHEO, false> aoff;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < p.ncells; c += (int64_t)gridDim.x * blockDim.x) {
        double a[L::size] = {};
        L::load_cell(p, c, a);
        double x[3] = {0, 0, 0}, Jf3[81];
#pragma unroll
        for (int i = 0; i < 81; ++i) Jf3[i] = 0.0;
        call_jf3<RHEO>(L::numA, aoff.v, a, p, x, Jf3);
        out[2 * c] = (float)(-Jf3[((0 * 3 + 1) * 3 + 0) * 3 + 1]);
        out[2 * c + 1] = (float)(-Jf3[((0 * 3 + 1) * 3 + 1) * 3 + 0]);
    }
}

bool launch_tangent_lm32(const DomainParams& p, int rheo, float* out, cudaStream_t s) {
    if (rheo != RHEO_ILE && rheo != RHEO_GENMAXWELL) return false;
    if (p.ncells == 0) return true;
    const int grid = (int)std::min<int64_t>((p.ncells + 255) / 256, 148 * 16);
    if (rheo == RHEO_GENMAXWELL) k_tangent_lm32<RHEO_GENMAXWELL><<<grid, 256, 0, s>>>(p, out);
    else k_tangent_lm32<RHEO_ILE><<<grid, 256, 0, s>>>(p, out);
    count_launch();
    return true;
}

bool launch_domain_jv32_hexgroup(const DomainParams& p, int cell, int rheo, cudaStream_t s) {
    if (p.ncells == 0) return true;
    const bool gm = rheo == RHEO_GENMAXWELL;
    if (cell == HEX8) {
        if (gm) launch_group_t<HEX8, RHEO_GENMAXWELL, false, OP_JACOBIAN_ACTION, float>(p, s);
        else launch_group_t<HEX8, RHEO_ILE, false, OP_JACOBIAN_ACTION, float>(p, s);
    } else if (cell == HEX27) {
        if (gm) launch_group_t<HEX27, RHEO_GENMAXWELL, false, OP_JACOBIAN_ACTION, float>(p, s);
        else launch_group_t<HEX27, RHEO_ILE, false, OP_JACOBIAN_ACTION, float>(p, s);
    } else {
        return false;
    }
    return true;
}

}  // namespace plb
