// Cell-block kernels for P1 tetrahedra: the hot path of the residual and Jacobian action.
//
// Cells are processed in blocks of kTetBlockCells consecutive cells (meshes are ordered along
// a Morton curve, so a block is a compact patch). One CTA per block:
//   1. gathers the block's nodes (coordinates and the input field) into shared memory once,
//      instead of once per incident cell;
//   2. one thread per cell forms the affine geometry, the solution gradient, calls the
//      pointwise kernel and stages its 12-entry element vector in shared memory;
//   3. one thread per node sums the staged entries of its incident corners in a fixed order
//      (a precomputed block-local incidence list) and writes the node's value: a plain store
//      for nodes whose cells all lie in the block, one FP64 reduction into global memory for
//      nodes shared with other blocks.
// Geometry in cofactor form: with C = det(J) J^{-1}, grad(u) = (G C) / det(J) for the edge
// differences G, and the element vector of corner a (a = 1..3) is f1 C_{a-1}^T / 6, so the
// Jacobian determinant only enters through one reciprocal.
#include <algorithm>
#include <vector>

#include "domain_kernels.cuh"
#include "internal.hpp"
#include "launch.hpp"

namespace plb {

constexpr int kTetBlockCells = 256;

// Cofactor matrix C = adj(J)^T with J = [X1-X0, X2-X0, X3-X0] (columns), so that
// J^{-1} = C^T / det ... stored here directly as cof[i][j] = (J^{-1})[i][j] * det.
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

template <int RHEO, bool BF, int OP, bool INSERT>
__global__ void __launch_bounds__(kTetBlockCells, 4)
    k_tet_blocked(DomainParams p, const int32_t* __restrict__ slot_begin, const int32_t* __restrict__ slot_node,
                  const uint8_t* __restrict__ slot_shared, const ushort4* __restrict__ lconn,
                  const uint16_t* __restrict__ inc_off, const uint16_t* __restrict__ inc, int64_t nblocks) {
    using L = AuxLayout<RHEO, BF>;
    extern __shared__ double smem[];
    const AuxOffsets<RHEO, BF> aoff;
    const double* __restrict__ field = OP == OP_RESIDUAL ? p.u : p.v;
    double* sE = smem;                          // [12][kTetBlockCells] staged element vectors
    double* sN = smem + 12 * kTetBlockCells;    // [ns][6]: coordinates, field
    for (int64_t b = blockIdx.x; b < nblocks; b += gridDim.x) {
        const int s0 = slot_begin[b];
        const int ns = slot_begin[b + 1] - s0;
        for (int i = threadIdx.x; i < ns; i += blockDim.x) {
            const int64_t nd = slot_node[s0 + i];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                sN[6 * i + d] = p.coords[3 * nd + d];
                sN[6 * i + 3 + d] = field[3 * nd + d];
            }
        }
        __syncthreads();
        const int tc = threadIdx.x;
        const int64_t c = b * kTetBlockCells + tc;
        if (c < p.ncells) {
            const ushort4 lc = lconn[c];
            const int ln[4] = {lc.x, lc.y, lc.z, lc.w};
            double X[4][3];
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int d = 0; d < 3; ++d) X[k][d] = sN[6 * ln[k] + d];
            double cof[3][3];
            const double det = tet_cofactors(X, cof);
            if (!(det > 0.0)) flag_error(p.err, CHECK_NONPOSITIVE_DETJ);
            const double rdet = 1.0 / det;
            // G[c][k] = u_{k+1}[c] - u_0[c]; s_x = G cof / det
            double G[3][3];
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) G[cc][k] = sN[6 * ln[k + 1] + 3 + cc] - sN[6 * ln[0] + 3 + cc];
            double s_x[9];
#pragma unroll
            for (int cc = 0; cc < 3; ++cc)
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    s_x[cc * 3 + d] = (G[cc][0] * cof[0][d] + G[cc][1] * cof[1][d] + G[cc][2] * cof[2][d]) * rdet;
            double a[L::size];
            L::load_cell(p, c, a);
            double x[3] = {0, 0, 0}, s[3] = {0, 0, 0};
            double f0[3] = {0, 0, 0}, f1[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            if (OP == OP_RESIDUAL) {
                if (BF) {
                    const int sOff[1] = {0}, sOff_x[1] = {0};
                    pw::g0v_bodyforce<double>(3, 1, L::numA, sOff, sOff_x, s, nullptr, s_x, aoff.v, nullptr, a,
                                              nullptr, nullptr, p.t, x, p.num_constants, p.constants, f0);
                }
                call_f1<RHEO>(L::numA, aoff.v, a, s, s_x, p, x, f1);
            } else {
                double Jf3[81];
#pragma unroll
                for (int i = 0; i < 81; ++i) Jf3[i] = 0.0;
                call_jf3<RHEO>(L::numA, aoff.v, a, p, x, Jf3);
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
            // corners 1..3: |J|/6 * f1 . grad(phi_a) = f1 . cof_{a-1} / 6; corner 0: minus their sum,
            // plus the body-force term |J|/6 * f0 / 4 at every corner.
            const double sixth = 1.0 / 6.0;
            const double bfw = BF && OP == OP_RESIDUAL ? det * sixth * 0.25 : 0.0;
            double e0[3] = {0, 0, 0};
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) {
                    const double v =
                        (f1[cc * 3 + 0] * cof[k][0] + f1[cc * 3 + 1] * cof[k][1] + f1[cc * 3 + 2] * cof[k][2]) * sixth;
                    e0[cc] -= v;
                    sE[((k + 1) * 3 + cc) * kTetBlockCells + tc] = v + bfw * f0[cc];
                }
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) sE[cc * kTetBlockCells + tc] = e0[cc] + bfw * f0[cc];
        }
        __syncthreads();
        for (int i = threadIdx.x; i < ns; i += blockDim.x) {
            const int j0 = inc_off[s0 + b + i], j1 = inc_off[s0 + b + i + 1];
            const uint16_t* lst = inc + b * 4 * kTetBlockCells;
            double r0 = 0.0, r1 = 0.0, r2 = 0.0;
            for (int j = j0; j < j1; ++j) {
                const int e = lst[j];
                const int cell = e >> 2, corner = e & 3;
                r0 += sE[(corner * 3 + 0) * kTetBlockCells + cell];
                r1 += sE[(corner * 3 + 1) * kTetBlockCells + cell];
                r2 += sE[(corner * 3 + 2) * kTetBlockCells + cell];
            }
            const int64_t nd = slot_node[s0 + i];
            double* o = p.out + 3 * nd;
            if (slot_shared[s0 + i]) {
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
        __syncthreads();
    }
}

template <int RHEO, bool BF, int OP>
static void launch_t(const DomainParams& p, const BlockedLayout& b, bool insert, cudaStream_t s) {
    const size_t smem = (size_t)(12 * kTetBlockCells + 6 * b.max_local_nodes) * sizeof(double);
    const int grid = (int)b.num_blocks;
#define PLB_ARGS p, b.d_block_node_begin, b.d_node_ids, b.d_slot_shared, (const ushort4*)b.d_local_cells, b.d_inc_off, b.d_inc, b.num_blocks
    if (insert) k_tet_blocked<RHEO, BF, OP, true><<<grid, kTetBlockCells, smem, s>>>(PLB_ARGS);
    else k_tet_blocked<RHEO, BF, OP, false><<<grid, kTetBlockCells, smem, s>>>(PLB_ARGS);
#undef PLB_ARGS
    count_launch();
}

bool launch_domain_apply_blocked(const DomainParams& p, const BlockedLayout& b, int cell, int rheo, bool bf,
                                 int op, bool insert, int64_t nnodes, cudaStream_t s) {
    if (cell != TET4 || rheo != RHEO_ILE || b.num_blocks == 0) return false;
    if ((size_t)(12 * kTetBlockCells + 6 * b.max_local_nodes) * sizeof(double) > 200 * 1024) return false;
    // INSERT: shared nodes receive reductions from several blocks, untouched nodes none, so the
    // output starts from zero; nodes owned by one block are then stored directly.
    if (insert && (b.num_shared_nodes > 0 || b.num_untouched > 0))
        if (cudaMemsetAsync(p.out, 0, 3 * nnodes * sizeof(double), s) != cudaSuccess) return false;
    if (op == OP_RESIDUAL) {
        if (bf) launch_t<RHEO_ILE, true, OP_RESIDUAL>(p, b, insert, s);
        else launch_t<RHEO_ILE, false, OP_RESIDUAL>(p, b, insert, s);
    } else {
        launch_t<RHEO_ILE, false, OP_JACOBIAN_ACTION>(p, b, insert, s);
    }
    return true;
}

// Host: block layout from the cell connectivity (cells should be in a locality-preserving order).
int ensure_blocked_layout(pl_mesh_s* m) {
    if (m->blocked) return PL_OK;
    if (m->cell_type != PL_CELL_TET4) {
        m->blocked = new BlockedLayout();  // empty: not supported for this cell type
        return PL_OK;
    }
    const int B = kTetBlockCells;
    const int64_t nc = m->ncells;
    const int64_t nb = (nc + B - 1) / B;
    std::vector<int32_t> begin(nb + 1, 0);
    std::vector<int32_t> node_ids;
    std::vector<uint16_t> lconn((size_t)nc * 4);
    std::vector<uint16_t> inc((size_t)nb * 4 * B, 0);
    std::vector<uint16_t> inc_off;
    std::vector<int32_t> nblocks_of(m->nnodes, 0);
    node_ids.reserve((size_t)nc);
    inc_off.reserve((size_t)nc + nb);
    int maxloc = 0;
    std::vector<int32_t> loc;
    std::vector<int> count;
    for (int64_t b = 0; b < nb; ++b) {
        const int64_t c0 = b * B, c1 = std::min<int64_t>(nc, c0 + B);
        loc.assign(m->h_cells.begin() + c0 * 4, m->h_cells.begin() + c1 * 4);
        std::sort(loc.begin(), loc.end());
        loc.erase(std::unique(loc.begin(), loc.end()), loc.end());
        maxloc = std::max<int>(maxloc, (int)loc.size());
        begin[b] = (int32_t)node_ids.size();
        for (int32_t nd : loc) {
            node_ids.push_back(nd);
            nblocks_of[nd]++;
        }
        count.assign(loc.size() + 1, 0);
        for (int64_t c = c0; c < c1; ++c)
            for (int k = 0; k < 4; ++k) {
                const int32_t nd = m->h_cells[c * 4 + k];
                const int l = (int)(std::lower_bound(loc.begin(), loc.end(), nd) - loc.begin());
                lconn[c * 4 + k] = (uint16_t)l;
                count[l + 1]++;
            }
        for (size_t i = 0; i < loc.size(); ++i) count[i + 1] += count[i];
        for (size_t i = 0; i <= loc.size(); ++i) inc_off.push_back((uint16_t)count[i]);
        // incidence entries in (cell, corner) order for every node: fixed summation order
        std::vector<int> fill(count.begin(), count.end() - 1);
        for (int64_t c = c0; c < c1; ++c)
            for (int k = 0; k < 4; ++k) {
                const int l = lconn[c * 4 + k];
                inc[(size_t)b * 4 * B + fill[l]++] = (uint16_t)((c - c0) * 4 + k);
            }
    }
    begin[nb] = (int32_t)node_ids.size();
    std::vector<uint8_t> shared(node_ids.size());
    for (size_t i = 0; i < node_ids.size(); ++i) shared[i] = nblocks_of[node_ids[i]] > 1 ? 1 : 0;
    int64_t nshared = 0, nuntouched = 0;
    for (int64_t nd = 0; nd < m->nnodes; ++nd) {
        nshared += nblocks_of[nd] > 1;
        nuntouched += nblocks_of[nd] == 0;
    }
    BlockedLayout* L = new BlockedLayout();
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
        e = cudaMalloc((void**)dst, bytes);
        if (e == cudaSuccess) e = cudaMemcpyAsync(*dst, v.data(), bytes, cudaMemcpyHostToDevice, s);
        L->device_bytes += bytes;
    };
    up(&L->d_block_node_begin, begin);
    up(&L->d_node_ids, node_ids);
    up(&L->d_local_cells, lconn);
    up(&L->d_slot_shared, shared);
    up(&L->d_inc_off, inc_off);
    up(&L->d_inc, inc);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        free_blocked_layout(L);
        return cuda_fail(e, "blocked layout upload");
    }
    m->blocked = L;
    return PL_OK;
}

void free_blocked_layout(BlockedLayout* b) {
    if (!b) return;
    cudaFree(b->d_block_node_begin);
    cudaFree(b->d_node_ids);
    cudaFree(b->d_local_cells);
    cudaFree(b->d_slot_shared);
    cudaFree(b->d_inc_off);
    cudaFree(b->d_inc);
    delete b;
}

}  // namespace plb
