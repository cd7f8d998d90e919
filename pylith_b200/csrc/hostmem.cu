// Page-locked host memory for the host side of host <-> device copies (pl_host_alloc).
//
// The buffers come from the CUDA driver (cudaHostAlloc), whose page-locked allocations the copy
// engines read at the link's rate; page-locked ranges made of scattered small pages (as some
// general-purpose pinned-memory caches hand out) can cap host-to-device DMA at a fraction of it.
// A host-to-device copy also reads host memory across the PCIe link with non-posted reads, so on
// a two-socket host pages on the far socket add the inter-socket link to every read: for the
// duration of the allocation the calling thread prefers the GPU's NUMA node (its previous policy
// is restored afterwards).
#include <cuda_runtime.h>
#include <sys/syscall.h>
#include <unistd.h>

#include <cctype>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>

#include "internal.hpp"

namespace {

constexpr int kMpolPreferred = 1;  // linux/mempolicy.h MPOL_PREFERRED

std::mutex g_host_mu;
std::map<void*, size_t> g_host_maps;  // registered mapping -> length

int gpu_numa_node(int device) {
    char bus[32] = {0};
    if (cudaDeviceGetPCIBusId(bus, sizeof(bus), device) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    for (char* p = bus; *p; ++p) *p = (char)std::tolower((unsigned char)*p);
    char path[96];
    std::snprintf(path, sizeof(path), "/sys/bus/pci/devices/%s/numa_node", bus);
    FILE* f = std::fopen(path, "r");
    if (!f) return -1;
    int node = -1;
    if (std::fscanf(f, "%d", &node) != 1) node = -1;
    std::fclose(f);
    return node;
}

}  // namespace

using namespace plb;

extern "C" {

int pl_context_numa_node(pl_context c, int* node) {
    if (!c || !node) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    *node = gpu_numa_node(c->device);
    return PL_OK;
}

int pl_host_alloc(pl_context c, size_t bytes, void** out) {
    if (!c || !out || bytes == 0) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    *out = nullptr;
    PLB_CUDA(cudaSetDevice(c->device));
    const int node = gpu_numa_node(c->device);
    // the calling thread's memory policy, restored after the allocation
    int old_mode = 0;
    unsigned long old_mask[16] = {0};
    bool policy = false;
    if (node >= 0 && node < 64 &&
        syscall(SYS_get_mempolicy, &old_mode, old_mask, 16ul * 64ul, nullptr, 0ul) == 0) {
        unsigned long mask = 1ul << node;
        // a refused policy (no NUMA support, the node outside the process's cpuset) leaves the
        // default placement, which still works
        policy = syscall(SYS_set_mempolicy, kMpolPreferred, &mask, 64ul) == 0;
    }
    void* p = nullptr;
    const cudaError_t e = cudaHostAlloc(&p, bytes, cudaHostAllocPortable);
    if (policy) syscall(SYS_set_mempolicy, old_mode, old_mask, 16ul * 64ul);
    if (e != cudaSuccess) return cuda_fail(e, "cudaHostAlloc");
    std::memset(p, 0, bytes);
    {
        std::lock_guard<std::mutex> lk(g_host_mu);
        g_host_maps[p] = bytes;
    }
    *out = p;
    return PL_OK;
}

int pl_host_free(void* ptr) {
    if (!ptr) return PL_OK;
    {
        std::lock_guard<std::mutex> lk(g_host_mu);
        auto it = g_host_maps.find(ptr);
        if (it == g_host_maps.end()) return fail(PL_ERR_INVALID_ARG, "pointer not from pl_host_alloc");
        g_host_maps.erase(it);
    }
    PLB_CUDA(cudaFreeHost(ptr));
    return PL_OK;
}

}  // extern "C"
