// Shared-node exchange of a partitioned residual: the pack and add steps around the point-to-point
// transfers that replace DMLocalToGlobal(ADD_VALUES) over the PetscSF
// (libsrc/pylith/topology/Field.cc:394-402, called from TimeDependent.cc:667).
//
// A partition's shared nodes are listed per neighbouring partition, in an order both sides agree
// on (global node id). pl_halo_pack copies the three values of every listed node, neighbour after
// neighbour, into one contiguous send buffer (one launch); the caller moves each neighbour's slice
// (NCCL send/recv, or a copy inside one process); pl_halo_unpack_add adds what came back. A node
// shared with several neighbours gets their values summed in neighbour order by one thread and
// added once, so the result needs no atomics and is the same every run.
#include <algorithm>
#include <vector>

#include "internal.hpp"
#include "launch.hpp"

struct pl_halo_s {
    pl_context ctx = nullptr;
    int npeers = 0;
    int64_t total = 0;             // listed entries over all neighbours
    int64_t nunique = 0;           // distinct shared nodes
    std::vector<int64_t> counts;   // entries per neighbour
    int32_t* d_nodes = nullptr;    // [total] local node of each entry, neighbour after neighbour
    int32_t* d_unique = nullptr;   // [nunique] distinct shared nodes
    int32_t* d_off = nullptr;      // [nunique + 1] offsets into d_pos
    int32_t* d_pos = nullptr;      // [total] entries of each distinct node, in neighbour order
};

namespace plb {

template <typename T>
__global__ void k_halo_pack(const T* __restrict__ r, const int32_t* __restrict__ nodes, int64_t total,
                            T* __restrict__ send) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * total; i += (int64_t)gridDim.x * blockDim.x)
        send[i] = r[3 * (int64_t)nodes[i / 3] + i % 3];
}

template <typename T>
__global__ void k_halo_unpack_add(const T* __restrict__ recv, const int32_t* __restrict__ unique,
                                  const int32_t* __restrict__ off, const int32_t* __restrict__ pos, int64_t nunique,
                                  T* __restrict__ r) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * nunique; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t u = i / 3;
        const int c = (int)(i % 3);
        T sum = 0;
        for (int32_t j = off[u]; j < off[u + 1]; ++j) sum += recv[3 * (int64_t)pos[j] + c];
        r[3 * (int64_t)unique[u] + c] += sum;
    }
}

static int halo_grid(int64_t items) { return (int)std::max<int64_t>(1, std::min<int64_t>((items + 255) / 256, 148 * 8)); }

}  // namespace plb

using namespace plb;

extern "C" {

int pl_halo_create(pl_context ctx, int npeers, const int64_t* counts, const int32_t* nodes_host, pl_halo* out) {
    if (!ctx || !out || npeers < 0 || (npeers > 0 && !counts)) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    *out = nullptr;
    int64_t total = 0;
    for (int p = 0; p < npeers; ++p) {
        if (counts[p] < 0) return fail(PL_ERR_INVALID_ARG, "negative count");
        total += counts[p];
    }
    if (total > 0 && !nodes_host) return fail(PL_ERR_INVALID_ARG, "null node list");
    if (total >= (int64_t(1) << 31)) return fail(PL_ERR_UNSUPPORTED, "more than 2^31 shared entries");
    for (int64_t i = 0; i < total; ++i)
        if (nodes_host[i] < 0) return fail(PL_ERR_INVALID_ARG, "negative node index");
    // distinct nodes and, per node, its entries in neighbour order (entries are numbered
    // neighbour after neighbour, so sorting (node, entry) keeps that order)
    std::vector<std::pair<int32_t, int32_t>> ne((size_t)total);
    for (int64_t i = 0; i < total; ++i) ne[i] = {nodes_host[i], (int32_t)i};
    std::sort(ne.begin(), ne.end());
    std::vector<int32_t> unique, off(1, 0), pos;
    pos.reserve((size_t)total);
    for (size_t i = 0; i < ne.size(); ++i) {
        if (i == 0 || ne[i].first != ne[i - 1].first) {
            if (i) off.push_back((int32_t)pos.size());
            unique.push_back(ne[i].first);
        }
        pos.push_back(ne[i].second);
    }
    if (!ne.empty()) off.push_back((int32_t)pos.size());
    pl_halo h = new pl_halo_s();
    h->ctx = ctx;
    h->npeers = npeers;
    h->total = total;
    h->nunique = (int64_t)unique.size();
    h->counts.assign(counts, counts + npeers);
    cudaError_t e = cudaSetDevice(ctx->device);
    auto up = [&](int32_t** dst, const int32_t* src, size_t n) {
        if (e != cudaSuccess || n == 0) return;
        e = dev_alloc(dst, n);
        if (e == cudaSuccess) e = cudaMemcpy(*dst, src, n * sizeof(int32_t), cudaMemcpyHostToDevice);
    };
    up(&h->d_nodes, nodes_host, (size_t)total);
    up(&h->d_unique, unique.data(), unique.size());
    up(&h->d_off, off.data(), off.size());
    up(&h->d_pos, pos.data(), pos.size());
    if (e != cudaSuccess) {
        for (void* p : {(void*)h->d_nodes, (void*)h->d_unique, (void*)h->d_off, (void*)h->d_pos}) dev_free(p, nullptr);
        delete h;
        return cuda_fail(e, "pl_halo_create");
    }
    context_retain(ctx);
    *out = h;
    return PL_OK;
}

int64_t pl_halo_num_entries(pl_halo h) { return h ? h->total : 0; }

int pl_halo_pack(pl_halo h, const double* r_dev, double* send_dev) {
    if (!h || (h->total > 0 && (!r_dev || !send_dev))) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    if (h->total == 0) return PL_OK;
    PLB_CUDA(cudaSetDevice(h->ctx->device));
    k_halo_pack<double><<<halo_grid(3 * h->total), 256, 0, h->ctx->stream>>>(r_dev, h->d_nodes, h->total, send_dev);
    count_launch();
    PLB_CUDA(cudaGetLastError());
    return PL_OK;
}

int pl_halo_unpack_add(pl_halo h, const double* recv_dev, double* r_dev) {
    if (!h || (h->total > 0 && (!r_dev || !recv_dev))) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    if (h->total == 0) return PL_OK;
    PLB_CUDA(cudaSetDevice(h->ctx->device));
    k_halo_unpack_add<double><<<halo_grid(3 * h->nunique), 256, 0, h->ctx->stream>>>(
        recv_dev, h->d_unique, h->d_off, h->d_pos, h->nunique, r_dev);
    count_launch();
    PLB_CUDA(cudaGetLastError());
    return PL_OK;
}

int pl_halo_pack_f32(pl_halo h, const float* r_dev, float* send_dev) {
    if (!h || (h->total > 0 && (!r_dev || !send_dev))) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    if (h->total == 0) return PL_OK;
    PLB_CUDA(cudaSetDevice(h->ctx->device));
    k_halo_pack<float><<<halo_grid(3 * h->total), 256, 0, h->ctx->stream>>>(r_dev, h->d_nodes, h->total, send_dev);
    count_launch();
    PLB_CUDA(cudaGetLastError());
    return PL_OK;
}

int pl_halo_unpack_add_f32(pl_halo h, const float* recv_dev, float* r_dev) {
    if (!h || (h->total > 0 && (!r_dev || !recv_dev))) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    if (h->total == 0) return PL_OK;
    PLB_CUDA(cudaSetDevice(h->ctx->device));
    k_halo_unpack_add<float><<<halo_grid(3 * h->nunique), 256, 0, h->ctx->stream>>>(
        recv_dev, h->d_unique, h->d_off, h->d_pos, h->nunique, r_dev);
    count_launch();
    PLB_CUDA(cudaGetLastError());
    return PL_OK;
}

int pl_halo_destroy(pl_halo h) {
    if (!h) return PL_OK;
    cudaSetDevice(h->ctx->device);
    cudaStreamSynchronize(h->ctx->stream);
    for (void* p : {(void*)h->d_nodes, (void*)h->d_unique, (void*)h->d_off, (void*)h->d_pos}) dev_free(p, h->ctx->stream);
    pl_context c = h->ctx;
    delete h;
    context_release(c);
    return PL_OK;
}

}  // extern "C"
