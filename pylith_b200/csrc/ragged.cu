// Ragged batch of quasi-static solves: many meshes of uneven size, each with its own solver, in
// shared launches.
//
// The reference solves one problem at a time (one SNES/KSP solve per Green's-function impulse,
// libsrc/pylith/problems/GreensFns.cc:291-337, and one PyLith process per forward problem). A
// serving loop on one GPU has many small problems at once, each too small to fill the device:
// here every PCG iteration of every active problem runs in the same eight launches -- fault
// unfold, the FP32 Q1 Jacobian action over all members' cells (k_hex8_jv32_ragged, hexgroup.cu),
// fault fold, p.Ap, its per-member sum, the x/r/z update with its r.z and r.r, their per-member
// sums, and the search-direction update -- with every dot product and step length kept per member
// (each member runs exactly its own PCG). Members join and leave between iterations; the
// launches read the member tables from device memory, so one captured graph of a chunk of
// iterations serves any membership. Each member reaches FP64 accuracy by reliable updates
// (residual replacement in FP64 with its own launches, solver32_replace) exactly as
// pl_solver_solve does for one solver.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "cg.cuh"
#include "domain_kernels.cuh"
#include "internal.hpp"
#include "launch.hpp"

namespace plb {

constexpr int kRgChunk = 256;     // nodes per CTA chunk of the vector kernels
constexpr int kRgGrid = 148 * 4;  // persistent grid of the vector kernels

// Per-member vectors and scalars of the FP32 PCG (device table).
struct RgVec {
    float *x, *r, *p, *q, *z;
    const float* pinv;
    const uint8_t* mask;
    const int32_t* pneg;
    const int32_t* ppos;
    int64_t nnodes;
    int64_t npairs;
    double* scal;  // the member solver's scalar slots
};

// Shared tables: member count, prefix sums of node chunks and fault pairs, active flags.
struct RgTables {
    const RgVec* vec;
    const int64_t* node_chunk0;  // [M + 1] chunks of kRgChunk nodes
    const int64_t* pair0;        // [M + 1] fault pairs
    const int* active;           // [M]
    const int* nmembers;
    double* partials;            // [2 * total chunks]
    double* rr_out;              // [M] r.r of each member (read by the host between chunks)
};

PL_D int rg_find(const int64_t* prefix, int M, int64_t w) {
    int lo = 0, hi = M;  // largest m with prefix[m] <= w
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (prefix[mid] <= w) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void k_rg_unfold(RgTables T) {
    const int M = *T.nmembers;
    const int64_t total = T.pair0[M];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = i / 3;
        const int m = rg_find(T.pair0, M, k);
        if (!T.active[m]) continue;
        const RgVec& v = T.vec[m];
        const int64_t j = k - T.pair0[m];
        const int c = (int)(i % 3);
        v.p[3 * (int64_t)v.ppos[j] + c] = v.p[3 * (int64_t)v.pneg[j] + c];
    }
}

__global__ void k_rg_fold(RgTables T) {
    const int M = *T.nmembers;
    const int64_t total = T.pair0[M];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = i / 3;
        const int m = rg_find(T.pair0, M, k);
        if (!T.active[m]) continue;
        const RgVec& v = T.vec[m];
        const int64_t j = k - T.pair0[m];
        const int c = (int)(i % 3);
        v.q[3 * (int64_t)v.pneg[j] + c] += v.q[3 * (int64_t)v.ppos[j] + c];
    }
}

// Per chunk of a member's nodes: partial of p.(A p) = -p.q over free DOFs.
__global__ void __launch_bounds__(kRgChunk) k_rg_pq(RgTables T) {
    const int M = *T.nmembers;
    const int64_t total = T.node_chunk0[M];
    for (int64_t ch = blockIdx.x; ch < total; ch += gridDim.x) {
        const int m = rg_find(T.node_chunk0, M, ch);
        double s = 0.0;
        if (T.active[m]) {
            const RgVec& v = T.vec[m];
            const int64_t nd = (ch - T.node_chunk0[m]) * kRgChunk + threadIdx.x;
            if (nd < v.nnodes)
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const int64_t i = 3 * nd + k;
                    if (!v.mask[i]) s -= (double)v.p[i] * (double)v.q[i];
                }
        }
        block_sum2(s, 0.0, T.partials + 2 * ch - 2 * (int64_t)blockIdx.x);
        __syncthreads();
    }
}

// x += alpha p, r += alpha q (free DOFs), z = P r; per-chunk partials of r.z and r.r.
__global__ void __launch_bounds__(kRgChunk) k_rg_update(RgTables T) {
    const int M = *T.nmembers;
    const int64_t total = T.node_chunk0[M];
    for (int64_t ch = blockIdx.x; ch < total; ch += gridDim.x) {
        const int m = rg_find(T.node_chunk0, M, ch);
        double rz = 0.0, rr = 0.0;
        if (T.active[m]) {
            const RgVec& v = T.vec[m];
            const float alpha = safe_step_f32(v.scal[S_RZ], v.scal[S_PQ]);
            const int64_t nd = (ch - T.node_chunk0[m]) * kRgChunk + threadIdx.x;
            if (nd < v.nnodes) {
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const int64_t i = 3 * nd + k;
                    if (!v.mask[i]) {
                        v.x[i] += alpha * v.p[i];
                        v.r[i] += alpha * v.q[i];
                    }
                }
                float zz[3];
                apply_pinv(v.pinv, v.r, nd, zz);
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    v.z[3 * nd + k] = zz[k];
                    rz += (double)v.r[3 * nd + k] * (double)zz[k];
                    rr += (double)v.r[3 * nd + k] * (double)v.r[3 * nd + k];
                }
            }
        }
        block_sum2(rz, rr, T.partials + 2 * ch - 2 * (int64_t)blockIdx.x);
        __syncthreads();
    }
}

// p = z + beta p with beta = rz / rz_old; q = 0 for the next operator application.
__global__ void k_rg_pupdate(RgTables T) {
    const int M = *T.nmembers;
    const int64_t total = T.node_chunk0[M];
    for (int64_t ch = blockIdx.x; ch < total; ch += gridDim.x) {
        const int m = rg_find(T.node_chunk0, M, ch);
        if (!T.active[m]) continue;
        const RgVec& v = T.vec[m];
        const double ro = v.scal[S_RZ_OLD];
        const float beta = ro != 0.0 ? (float)(v.scal[S_RZ] / ro) : 0.0f;
        const int64_t nd = (ch - T.node_chunk0[m]) * kRgChunk + threadIdx.x;
        if (nd < v.nnodes)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int64_t i = 3 * nd + k;
                v.p[i] = v.z[i] + (isfinite(beta) ? beta : 0.0f) * v.p[i];
                v.q[i] = 0.0f;
            }
    }
}

// Per member (one warp each): sum its chunks' partials in chunk order into its scalars. mode 0:
// p.Ap into S_PQ (and r.z into S_RZ_OLD); mode 1: r.z into S_RZ and r.r into S_RR and rr_out.
__global__ void k_rg_finish(RgTables T, int mode) {
    const int M = *T.nmembers;
    const int lane = threadIdx.x & 31;
    for (int m = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); m < M; m += gridDim.x * (blockDim.x >> 5)) {
        if (!T.active[m]) continue;
        double a = 0.0, b = 0.0;
        for (int64_t ch = T.node_chunk0[m] + lane; ch < T.node_chunk0[m + 1]; ch += 32) {
            a += T.partials[2 * ch];
            b += T.partials[2 * ch + 1];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
        if (lane == 0) {
            double* sc = T.vec[m].scal;
            if (mode == 0) {
                sc[S_PQ] = a;
                sc[S_RZ_OLD] = sc[S_RZ];
            } else {
                sc[S_RZ] = a;
                sc[S_RR] = b;
                T.rr_out[m] = b;
            }
        }
    }
}

}  // namespace plb

using namespace plb;

namespace {

struct Member {
    pl_solver S = nullptr;
    const double* b = nullptr;
    double* x = nullptr;
    bool active = false;
    int status = PL_ERR_NOT_READY;  // PL_OK when converged, an error code on failure
    double b0 = 0.0, rref = 0.0, rt = 0.0, stop = 0.0;
    int iterations = 0, replacements = 0, breakdowns = 0;
};

}  // namespace

struct pl_ragged_s {
    pl_context ctx = nullptr;
    int capacity = 0;
    int chunk = 10;  // PCG iterations per graph launch between convergence checks
    std::vector<Member> members;
    bool dirty = true;
    // device tables
    DomainParams* d_ops = nullptr;
    int64_t* d_cell_chunk0 = nullptr;
    RgVec* d_vec = nullptr;
    int64_t* d_node_chunk0 = nullptr;
    int64_t* d_pair0 = nullptr;
    int* d_active = nullptr;
    int* d_nmembers = nullptr;
    double* d_partials = nullptr;
    int64_t partials_cap = 0;
    double* d_rr = nullptr;
    // iteration graph on a private stream
    cudaStream_t cs = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_chunk = 0;
    int64_t launches_per_iteration = 8;
};

namespace {

int upload_tables(pl_ragged R) {
    const int M = (int)R->members.size();
    std::vector<DomainParams> ops(M);
    std::vector<RgVec> vec(M);
    std::vector<int64_t> cell0(M + 1, 0), node0(M + 1, 0), pair0(M + 1, 0);
    std::vector<int> active(M, 0);
    for (int i = 0; i < M; ++i) {
        Member& mb = R->members[i];
        pl_solver S = mb.S;
        if (!S) {  // a free slot: no cells, nodes or pairs
            std::memset(&ops[i], 0, sizeof(DomainParams));
            std::memset(&vec[i], 0, sizeof(RgVec));
            cell0[i + 1] = cell0[i];
            node0[i + 1] = node0[i];
            pair0[i + 1] = pair0[i];
            continue;
        }
        pl_integrator ig = S->ops[0];
        DomainParams p;
        int rc = bind_domain_jacobian(ig, &p);
        if (rc) return rc;
        p.t = S->t;
        p.dt = S->dt;
        p.v32 = S->f_p;
        p.out32 = S->f_q;
        p.lm32 = ig->d_lm32;
        ops[i] = p;
        vec[i] = RgVec{S->f_x, S->f_r, S->f_p, S->f_q, S->f_z, S->d_pinv32, S->d_mask, S->d_pair_neg, S->d_pair_pos,
                       S->nnodes, S->npairs, S->d_scal};
        cell0[i + 1] = cell0[i] + (ig->ncells + 3) / 4;  // warp chunks of 4 Q1 cells
        node0[i + 1] = node0[i] + (S->nnodes + kRgChunk - 1) / kRgChunk;
        pair0[i + 1] = pair0[i] + S->npairs;
        active[i] = mb.active ? 1 : 0;
    }
    cudaStream_t s = R->ctx->stream;
    if (node0[M] > R->partials_cap) {
        dev_free(R->d_partials, R->cs);
        R->d_partials = nullptr;
        R->partials_cap = std::max<int64_t>(node0[M], 2 * R->partials_cap);
        PLB_CUDA(dev_alloc(&R->d_partials, 2 * R->partials_cap));
        // the captured graph holds the old partials buffer
        if (R->graph) cudaGraphExecDestroy(R->graph);
        R->graph = nullptr;
    }
    if (M > 0) {
        PLB_CUDA(cudaMemcpyAsync(R->d_ops, ops.data(), M * sizeof(DomainParams), cudaMemcpyHostToDevice, s));
        PLB_CUDA(cudaMemcpyAsync(R->d_vec, vec.data(), M * sizeof(RgVec), cudaMemcpyHostToDevice, s));
        PLB_CUDA(cudaMemcpyAsync(R->d_active, active.data(), M * sizeof(int), cudaMemcpyHostToDevice, s));
    }
    PLB_CUDA(cudaMemcpyAsync(R->d_cell_chunk0, cell0.data(), (M + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    PLB_CUDA(cudaMemcpyAsync(R->d_node_chunk0, node0.data(), (M + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    PLB_CUDA(cudaMemcpyAsync(R->d_pair0, pair0.data(), (M + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    PLB_CUDA(cudaMemcpyAsync(R->d_nmembers, &M, sizeof(int), cudaMemcpyHostToDevice, s));
    // the host vectors above go out of scope: wait for the copies
    PLB_CUDA(cudaStreamSynchronize(s));
    R->dirty = false;
    return PL_OK;
}

RgTables tables_of(pl_ragged R) {
    return RgTables{R->d_vec, R->d_node_chunk0, R->d_pair0, R->d_active, R->d_nmembers, R->d_partials, R->d_rr};
}

void rg_iteration(pl_ragged R) {
    const RgTables T = tables_of(R);
    cudaStream_t cs = R->cs;
    k_rg_unfold<<<kRgGrid, 256, 0, cs>>>(T);
    launch_hex8_jv32_ragged(R->d_ops, R->d_cell_chunk0, R->d_active, R->d_nmembers, cs);
    k_rg_fold<<<kRgGrid, 256, 0, cs>>>(T);
    k_rg_pq<<<kRgGrid, kRgChunk, 0, cs>>>(T);
    k_rg_finish<<<16, 256, 0, cs>>>(T, 0);
    k_rg_update<<<kRgGrid, kRgChunk, 0, cs>>>(T);
    k_rg_finish<<<16, 256, 0, cs>>>(T, 1);
    k_rg_pupdate<<<kRgGrid, kRgChunk, 0, cs>>>(T);
}

int ensure_graph(pl_ragged R) {
    if (R->graph && R->graph_chunk == R->chunk) return PL_OK;
    if (R->graph) cudaGraphExecDestroy(R->graph);
    R->graph = nullptr;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(R->cs, cudaStreamCaptureModeRelaxed);
    for (int i = 0; i < R->chunk && e == cudaSuccess; ++i) rg_iteration(R);
    if (e == cudaSuccess) e = cudaStreamEndCapture(R->cs, &g);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&R->graph, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "ragged PCG graph");
    R->graph_chunk = R->chunk;
    return PL_OK;
}

void finish_member(pl_ragged R, Member& mb, int status) {
    mb.active = false;
    mb.status = status;
    R->dirty = true;
    if (mb.S && mb.x) solver_unfold(mb.S, mb.x);  // the positive side of every fault node follows its negative side
}

}  // namespace

extern "C" {

int pl_ragged_create(pl_context ctx, int capacity, pl_ragged* out) {
    if (!ctx || !out || capacity <= 0 || capacity > 4096) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    *out = nullptr;
    PLB_CUDA(cudaSetDevice(ctx->device));
    pl_ragged R = new pl_ragged_s();
    R->ctx = ctx;
    R->capacity = capacity;
    cudaError_t e = cudaSuccess;
    auto A = [&](auto** p, size_t cnt) {
        if (e == cudaSuccess) e = dev_alloc(p, cnt);
    };
    A(&R->d_ops, capacity);
    A(&R->d_cell_chunk0, capacity + 1);
    A(&R->d_vec, capacity);
    A(&R->d_node_chunk0, capacity + 1);
    A(&R->d_pair0, capacity + 1);
    A(&R->d_active, capacity);
    A(&R->d_nmembers, 1);
    A(&R->d_rr, capacity);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&R->cs, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&R->ev_in, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&R->ev_out, cudaEventDisableTiming);
    context_retain(ctx);
    if (e != cudaSuccess) {
        pl_ragged_destroy(R);
        return cuda_fail(e, "pl_ragged_create");
    }
    *out = R;
    return PL_OK;
}

int pl_ragged_add(pl_ragged R, pl_solver S, const double* b_dev, double* x_dev, int* member) {
    if (!R || !S || !b_dev || !x_dev || !member) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    if (S->mesh->ctx != R->ctx) return fail(PL_ERR_INVALID_ARG, "the solver belongs to another context");
    if (!S->ready || S->precision != PL_SOLVER_FP32_REFINED)
        return fail(PL_ERR_NOT_READY, "the solver must be set up with PL_SOLVER_FP32_REFINED");
    if (S->mesh->cell_type != PL_CELL_HEX8 || S->ops.size() != 1)
        return fail(PL_ERR_UNSUPPORTED, "ragged batches take Q1 hexahedral solvers with one domain integrator");
    pl_integrator ig = S->ops[0];
    if (!ig->lm32_valid || ig->lm32_t != S->t || ig->lm32_dt != S->dt || !ig->d_lm32)
        return fail(PL_ERR_NOT_READY, "the integrator's FP32 tangent is stale: call pl_solver_setup again");
    for (const Member& mb : R->members)
        if (mb.S == S) return fail(PL_ERR_INVALID_ARG, "the solver is already a member");
    PLB_CUDA(cudaSetDevice(R->ctx->device));
    Member mb;
    mb.S = S;
    mb.b = solver_reduced_rhs(S, b_dev);  // with faults: P^T b in the solver's scratch vector
    mb.x = x_dev;
    int rc = solver32_begin(S, mb.b, x_dev, &mb.b0);
    if (rc) return rc;
    mb.rref = mb.rt = mb.b0;
    mb.stop = std::max(S->rtol * mb.b0, S->atol);
    if (mb.b0 == 0.0 || mb.b0 <= mb.stop) {
        mb.status = PL_OK;  // x = 0 solves it
    } else {
        mb.active = true;
        mb.status = PL_ERR_NOT_READY;
    }
    // a free slot (a removed member's) or a new one
    int slot = -1;
    for (int i = 0; i < (int)R->members.size() && slot < 0; ++i)
        if (!R->members[i].S) slot = i;
    if (slot < 0) {
        if ((int)R->members.size() >= R->capacity) return fail(PL_ERR_OUT_OF_MEMORY, "ragged batch is full");
        R->members.emplace_back();
        slot = (int)R->members.size() - 1;
    }
    solver_retain(S);
    R->members[slot] = mb;
    R->dirty = true;
    *member = slot;
    return PL_OK;
}

int pl_ragged_iterate(pl_ragged R, int* active_left) {
    if (!R) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    PLB_CUDA(cudaSetDevice(R->ctx->device));
    int left = 0;
    for (const Member& mb : R->members) left += mb.active;
    if (left > 0) {
        int rc;
        if (R->dirty && (rc = upload_tables(R)) != PL_OK) return rc;
        if ((rc = ensure_graph(R)) != PL_OK) return rc;
        cudaStream_t s = R->ctx->stream;
        PLB_CUDA(cudaEventRecord(R->ev_in, s));
        PLB_CUDA(cudaStreamWaitEvent(R->cs, R->ev_in, 0));
        PLB_CUDA(cudaGraphLaunch(R->graph, R->cs));
        count_launch(8 * R->chunk);  // the graph's launches
        const int M = (int)R->members.size();
        std::vector<double> rr(M);
        PLB_CUDA(cudaMemcpyAsync(rr.data(), R->d_rr, M * sizeof(double), cudaMemcpyDeviceToHost, R->cs));
        PLB_CUDA(cudaEventRecord(R->ev_out, R->cs));
        PLB_CUDA(cudaStreamWaitEvent(s, R->ev_out, 0));
        PLB_CUDA(cudaStreamSynchronize(s));
        for (int i = 0; i < M; ++i) {
            Member& mb = R->members[i];
            if (!mb.active) continue;
            pl_solver S = mb.S;
            mb.iterations += R->chunk;
            S->inner_iterations = mb.iterations;
            const double rn = std::sqrt(rr[i]);
            // FP32 breakdown (see pcg32_reliable): drop the correction, restart from the true residual
            const bool broke = !(rn == rn) || rn > kBreakdownGrowth * mb.rref;
            if (!broke && rn > S->reliable_delta * mb.rref && rn > 0.5 * mb.stop) {
                if (mb.iterations >= S->max_iter) finish_member(R, mb, PL_ERR_NOT_CONVERGED);
                continue;
            }
            if (broke && ++mb.breakdowns > kMaxBreakdowns) {
                finish_member(R, mb, PL_ERR_NOT_CONVERGED);
                continue;
            }
            // residual replacement with this member's own FP64 launches
            double rt = 0.0;
            if ((rc = solver32_replace(S, mb.b, mb.x, broke || rn <= 0.5 * mb.stop, !broke, &rt)) != PL_OK) return rc;
            mb.replacements++;
            mb.rt = rt;
            S->outer_iterations = mb.replacements;
            S->rel_residual = mb.b0 > 0.0 ? rt / mb.b0 : 0.0;
            if (rt <= mb.stop) finish_member(R, mb, PL_OK);
            else if (mb.iterations >= S->max_iter) finish_member(R, mb, PL_ERR_NOT_CONVERGED);
            else mb.rref = rt;
        }
    }
    left = 0;
    for (const Member& mb : R->members) left += mb.active;
    if (active_left) *active_left = left;
    return PL_OK;
}

int pl_ragged_member_status(pl_ragged R, int member, int* status, int* iterations, double* rel_residual) {
    if (!R || member < 0 || member >= (int)R->members.size()) return fail(PL_ERR_INVALID_ARG, "bad member");
    const Member& mb = R->members[member];
    if (status) *status = mb.active ? PL_ERR_NOT_READY : mb.status;
    if (iterations) *iterations = mb.iterations;
    if (rel_residual) *rel_residual = mb.b0 > 0.0 ? mb.rt / mb.b0 : 0.0;
    return PL_OK;
}

int pl_ragged_remove(pl_ragged R, int member) {
    if (!R || member < 0 || member >= (int)R->members.size()) return fail(PL_ERR_INVALID_ARG, "bad member");
    Member& mb = R->members[member];
    if (!mb.S) return PL_OK;
    pl_solver S = mb.S;
    if (mb.active) finish_member(R, mb, PL_ERR_NOT_CONVERGED);
    mb = Member();  // the slot is free for the next pl_ragged_add; the other members keep theirs
    R->dirty = true;
    // the tables still point into S until they are uploaded again: wait for the batch's work
    cudaStreamSynchronize(R->cs);
    solver_release(S);
    return PL_OK;
}

int pl_ragged_set_chunk(pl_ragged R, int iterations) {
    if (!R || iterations <= 0 || iterations > 1000) return fail(PL_ERR_INVALID_ARG, "bad chunk");
    R->chunk = iterations;
    return PL_OK;
}

int pl_ragged_destroy(pl_ragged R) {
    if (!R) return PL_OK;
    cudaSetDevice(R->ctx->device);
    if (R->cs) cudaStreamSynchronize(R->cs);
    for (Member& mb : R->members)
        if (mb.S) solver_release(mb.S);
    if (R->graph) cudaGraphExecDestroy(R->graph);
    if (R->ev_in) cudaEventDestroy(R->ev_in);
    if (R->ev_out) cudaEventDestroy(R->ev_out);
    if (R->cs) cudaStreamDestroy(R->cs);
    void* ptrs[] = {R->d_ops, R->d_cell_chunk0, R->d_vec, R->d_node_chunk0, R->d_pair0, R->d_active, R->d_nmembers,
                    R->d_partials, R->d_rr};
    for (void* p : ptrs) dev_free(p, R->ctx->stream);
    pl_context c = R->ctx;
    delete R;
    context_release(c);
    return PL_OK;
}

}  // extern "C"
