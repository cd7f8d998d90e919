// Cell-block kernels for P1 tetrahedra: the hot path of the residual and Jacobian action.
//
// Cells are processed in blocks of consecutive cells (the mesh is ordered along a Morton curve,
// so a block is a compact patch). One CTA per block:
//   1. gathers the block's nodes (coordinates and the input field) into shared memory once,
//      instead of once per incident cell;
//   2. one thread per cell forms geometry, the solution gradient, calls the pointwise kernel
//      and adds its element vector into per-node shared-memory accumulators;
//   3. writes each node's sum: a plain store (or add) for nodes whose cells all lie in the block,
//      one FP64 reduction into global memory for nodes shared with other blocks.
// Per cell the CTA reads 8 bytes of block-local connectivity (uint16) and the material; per node
// it reads the coordinates and field once and writes the result once (shared nodes: one L2
// reduction per block that touches them).
#include <algorithm>
#include <vector>

#include "domain_kernels.cuh"
#include "internal.hpp"
#include "launch.hpp"

namespace plb {

constexpr int kTetBlockCells = 256;

template <int RHEO, bool BF, int OP, bool INSERT>
__global__ void __launch_bounds__(kTetBlockCells) k_tet_blocked(DomainParams p, const int32_t* __restrict__ slot_begin,
                                                                const int32_t* __restrict__ slot_node,
                                                                const uint8_t* __restrict__ slot_shared,
                                                                const ushort4* __restrict__ lconn, int64_t nblocks) {
    using L = AuxLayout<RHEO, BF>;
    extern __shared__ double smem[];
    const AuxOffsets<RHEO, BF> aoff;
    const double* __restrict__ field = OP == OP_RESIDUAL ? p.u : p.v;
    for (int64_t b = blockIdx.x; b < nblocks; b += gridDim.x) {
        const int s0 = slot_begin[b];
        const int ns = slot_begin[b + 1] - s0;
        double* sX = smem;             // [ns][3]
        double* sU = smem + 3 * ns;    // [ns][3]
        double* sR = smem + 6 * ns;    // [ns][3]
        for (int i = threadIdx.x; i < ns; i += blockDim.x) {
            const int64_t nd = slot_node[s0 + i];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                sX[3 * i + d] = p.coords[3 * nd + d];
                sU[3 * i + d] = field[3 * nd + d];
                sR[3 * i + d] = 0.0;
            }
        }
        __syncthreads();
        const int64_t c = b * kTetBlockCells + threadIdx.x;
        if (c < p.ncells) {
            const ushort4 lc = lconn[c];
            const int ln[4] = {lc.x, lc.y, lc.z, lc.w};
            double X[4][3];
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int d = 0; d < 3; ++d) X[k][d] = sX[3 * ln[k] + d];
            Geom g;
            tet_geometry(X, &g);
            if (!(g.detJ > 0.0)) flag_error(p.err, CHECK_NONPOSITIVE_DETJ);
            double gr[4][3];
#pragma unroll
            for (int n = 0; n < 4; ++n) tet_grad(g, n, gr[n]);
            double s[3] = {0, 0, 0}, s_x[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
            for (int n = 0; n < 4; ++n) {
                const double u0 = sU[3 * ln[n]], u1 = sU[3 * ln[n] + 1], u2 = sU[3 * ln[n] + 2];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    s_x[0 + d] += u0 * gr[n][d];
                    s_x[3 + d] += u1 * gr[n][d];
                    s_x[6 + d] += u2 * gr[n][d];
                }
            }
            double a[L::size];
            L::load_cell(p, c, a);
            double x[3] = {0, 0, 0};
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
#pragma unroll
            for (int n = 0; n < 4; ++n)
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) {
                    const double v = g.wdetJ * (f0[cc] * 0.25 + f1[cc * 3 + 0] * gr[n][0] + f1[cc * 3 + 1] * gr[n][1] +
                                                f1[cc * 3 + 2] * gr[n][2]);
                    atomicAdd(&sR[3 * ln[n] + cc], v);
                }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < ns; i += blockDim.x) {
            const int64_t nd = slot_node[s0 + i];
            const bool shared = slot_shared[s0 + i] != 0;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                double* o = p.out + 3 * nd + d;
                if (shared) red_add(o, sR[3 * i + d]);
                else if (INSERT) *o = sR[3 * i + d];
                else *o += sR[3 * i + d];
            }
        }
        __syncthreads();
    }
}

// Zero the nodes that several blocks add into (INSERT mode) and the nodes no cell touches.
__global__ void k_zero_nodes(const int32_t* __restrict__ nodes, int64_t n, double* out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t nd = nodes[i];
        out[3 * nd] = 0.0;
        out[3 * nd + 1] = 0.0;
        out[3 * nd + 2] = 0.0;
    }
}

template <int RHEO, bool BF, int OP>
static void launch_t(const DomainParams& p, const BlockedLayout& b, bool insert, cudaStream_t s) {
    const size_t smem = (size_t)9 * b.max_local_nodes * sizeof(double);
    const int grid = (int)b.num_blocks;
    if (insert)
        k_tet_blocked<RHEO, BF, OP, true><<<grid, kTetBlockCells, smem, s>>>(
            p, b.d_block_node_begin, b.d_node_ids, b.d_slot_shared, (const ushort4*)b.d_local_cells, b.num_blocks);
    else
        k_tet_blocked<RHEO, BF, OP, false><<<grid, kTetBlockCells, smem, s>>>(
            p, b.d_block_node_begin, b.d_node_ids, b.d_slot_shared, (const ushort4*)b.d_local_cells, b.num_blocks);
    count_launch();
}

bool launch_domain_apply_blocked(const DomainParams& p, const BlockedLayout& b, int cell, int rheo, bool bf,
                                 int op, bool insert, int64_t nnodes, cudaStream_t s) {
    if (cell != TET4 || rheo != RHEO_ILE || b.num_blocks == 0) return false;
    if ((size_t)9 * b.max_local_nodes * sizeof(double) > 200 * 1024) return false;
    if (insert && b.num_shared_nodes > 0) {
        const int64_t n = b.num_shared_nodes;
        k_zero_nodes<<<(int)std::min<int64_t>((n + 255) / 256, 148 * 16), 256, 0, s>>>(b.d_shared_node, n, p.out);
        count_launch();
    }
    if (insert && b.num_untouched > 0) {
        k_zero_nodes<<<(int)std::min<int64_t>((b.num_untouched + 255) / 256, 148 * 16), 256, 0, s>>>(
            b.d_untouched, b.num_untouched, p.out);
        count_launch();
    }
    if (op == OP_RESIDUAL) {
        if (bf) launch_t<RHEO_ILE, true, OP_RESIDUAL>(p, b, insert, s);
        else launch_t<RHEO_ILE, false, OP_RESIDUAL>(p, b, insert, s);
    } else {
        launch_t<RHEO_ILE, false, OP_JACOBIAN_ACTION>(p, b, insert, s);
    }
    return true;
}

// Host: block layout from the cell connectivity (cells must be in a locality-preserving order).
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
    std::vector<int32_t> nblocks_of(m->nnodes, 0);
    node_ids.reserve((size_t)nc);
    int maxloc = 0;
    std::vector<int32_t> loc;
    for (int64_t b = 0; b < nb; ++b) {
        const int64_t c0 = b * B, c1 = std::min<int64_t>(nc, c0 + B);
        loc.assign(m->h_cells.begin() + c0 * 4, m->h_cells.begin() + c1 * 4);
        std::sort(loc.begin(), loc.end());
        loc.erase(std::unique(loc.begin(), loc.end()), loc.end());
        if (loc.size() > 65535) return fail(PL_ERR_UNSUPPORTED, "cell block touches too many nodes");
        maxloc = std::max<int>(maxloc, (int)loc.size());
        begin[b] = (int32_t)node_ids.size();
        for (int32_t nd : loc) {
            node_ids.push_back(nd);
            nblocks_of[nd]++;
        }
        for (int64_t c = c0; c < c1; ++c)
            for (int k = 0; k < 4; ++k) {
                const int32_t nd = m->h_cells[c * 4 + k];
                lconn[c * 4 + k] = (uint16_t)(std::lower_bound(loc.begin(), loc.end(), nd) - loc.begin());
            }
    }
    begin[nb] = (int32_t)node_ids.size();
    std::vector<uint8_t> shared(node_ids.size());
    for (size_t i = 0; i < node_ids.size(); ++i) shared[i] = nblocks_of[node_ids[i]] > 1 ? 1 : 0;
    std::vector<int32_t> shared_nodes, untouched;
    for (int64_t nd = 0; nd < m->nnodes; ++nd) {
        if (nblocks_of[nd] > 1) shared_nodes.push_back((int32_t)nd);
        if (nblocks_of[nd] == 0) untouched.push_back((int32_t)nd);
    }
    BlockedLayout* L = new BlockedLayout();
    L->cells_per_block = B;
    L->num_blocks = nb;
    L->max_local_nodes = maxloc;
    L->num_shared_nodes = (int64_t)shared_nodes.size();
    L->num_untouched = (int64_t)untouched.size();
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
    up(&L->d_shared_node, shared_nodes);
    up(&L->d_untouched, untouched);
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
    cudaFree(b->d_shared_node);
    cudaFree(b->d_untouched);
    delete b;
}

}  // namespace plb
