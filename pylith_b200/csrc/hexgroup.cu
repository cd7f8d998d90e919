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

// T = double: residual (OP_RESIDUAL) or Jacobian action into p.out from p.u / p.v;
// T = float: Jacobian action into p.out32 from p.v32.
template <int CELL, int RHEO, bool BF, int OP, typename T>
__global__ void __launch_bounds__(HexGroup<CELL, T>::WARPS * 32) k_hex_group(DomainParams p) {
    using H = HexGroup<CELL, T>;
    using L = AuxLayout<RHEO, BF>;
    const AuxOffsets<RHEO, BF> aoff;
    extern __shared__ __align__(16) double hsm[];
    double* t64 = hsm;
    T* tt = reinterpret_cast<T*>(hsm + H::T_END64 + H::GROUPS * H::PER_GROUP_X);
    fill_tables<CELL, T>(t64, tt);
    __syncthreads();
    const double* tN = t64;
    const double* tW = t64 + H::T_W;
    const T* tB = tt;
    const T* tPhi = tt + H::T_PHI;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int grp = lane / H::G, l = lane % H::G;
    const int gid = warp * H::CPW + grp;
    double* sX = hsm + H::T_END64 + gid * H::PER_GROUP_X;
    T* sg = tt + H::T_ENDT + gid * H::PER_GROUP_T;
    T* su = sg;
    T* sF = sg + H::OFF_F;
    T* sF0 = sg + H::OFF_F0;
    const bool f32 = sizeof(T) == 4;
    const int64_t cells_per_pass = (int64_t)gridDim.x * H::WARPS * H::CPW;
    // every lane of a warp runs the same number of passes (the __syncwarp calls need them all)
    for (int64_t base = ((int64_t)blockIdx.x * H::WARPS + warp) * H::CPW; base < p.ncells; base += cells_per_pass) {
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
            const T wdetJ = (T)(tW[q] * detJ);
            T inv[3][3];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) inv[i][j] = (T)inv64[i][j];
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
            L::load_cell(p, c, a);
            if (OP == OP_RESIDUAL) L::load_qp(p, c, q, H::NQ, a);  // the tangents read no state
            double x[3] = {0, 0, 0}, s[3] = {0, 0, 0};
            double f0[3] = {0, 0, 0};
            T f1[9];
            if (OP == OP_RESIDUAL) {
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
#pragma unroll
                for (int f = 0; f < 3; ++f)
#pragma unroll
                    for (int df = 0; df < 3; ++df) {
                        T acc1 = 0;
#pragma unroll
                        for (int gg = 0; gg < 3; ++gg)
#pragma unroll
                            for (int dg = 0; dg < 3; ++dg)
                                acc1 += (T)Jf3[((f * 3 + gg) * 3 + df) * 3 + dg] * s_x[gg * 3 + dg];
                        f1[f * 3 + df] = acc1;
                    }
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

template <int CELL, int RHEO, bool BF, int OP, typename T = double>
static void launch_group_t(const DomainParams& p, cudaStream_t s) {
    using H = HexGroup<CELL, T>;
    auto kern = k_hex_group<CELL, RHEO, BF, OP, T>;
    const size_t smem = H::smem_bytes();
    if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int dev = 0, nsm = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, H::WARPS * 32, smem);
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

bool launch_domain_apply_hexgroup(const DomainParams& p, int cell, int rheo, bool bf, int op, cudaStream_t s) {
    if (p.ncells == 0) return true;
    if (cell == HEX8) launch_group_cell<HEX8>(p, rheo, bf, op, s);
    else if (cell == HEX27) launch_group_cell<HEX27>(p, rheo, bf, op, s);
    else return false;
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
