// Page-locked host memory for the host side of host <-> device copies (pl_host_alloc).
//
// A host-to-device DMA copy reads host memory with non-posted PCIe reads, so its rate depends
// on where the pages are: on a two-socket host, pages on the other socket make every read cross
// the inter-socket link, and page-locked buffers from cudaHostAlloc land wherever the
// allocating thread happens to run. pl_host_alloc maps anonymous memory, prefers the GPU's
// node (a node without free memory still yields a buffer), advises transparent huge pages for
// buffers of 2 MiB and more, faults every page in under that policy and registers the range
// with CUDA.
#include <cuda_runtime.h>
#include <sys/mman.h>
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
    const size_t page = (size_t)sysconf(_SC_PAGESIZE);
    const size_t len = (bytes + page - 1) / page * page;
    void* p = mmap(nullptr, len, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
    if (p == MAP_FAILED) return fail(PL_ERR_OUT_OF_MEMORY, "mmap of host buffer failed");
    const int node = gpu_numa_node(c->device);
    if (node >= 0 && node < 64) {
        unsigned long mask = 1ul << node;
        // a refused policy (no NUMA support in the kernel, the node outside the process's
        // cpuset) leaves the default placement, which still works
        syscall(SYS_mbind, p, len, kMpolPreferred, &mask, 64ul, 0u);
    }
    if (len >= (2u << 20)) madvise(p, len, MADV_HUGEPAGE);
    std::memset(p, 0, len);  // fault the pages in under the node policy
    cudaError_t e = cudaSetDevice(c->device);
    if (e == cudaSuccess) e = cudaHostRegister(p, len, cudaHostRegisterPortable);
    if (e != cudaSuccess) {
        munmap(p, len);
        return cuda_fail(e, "cudaHostRegister");
    }
    {
        std::lock_guard<std::mutex> lk(g_host_mu);
        g_host_maps[p] = len;
    }
    *out = p;
    return PL_OK;
}

int pl_host_free(void* ptr) {
    if (!ptr) return PL_OK;
    size_t len = 0;
    {
        std::lock_guard<std::mutex> lk(g_host_mu);
        auto it = g_host_maps.find(ptr);
        if (it == g_host_maps.end()) return fail(PL_ERR_INVALID_ARG, "pointer not from pl_host_alloc");
        len = it->second;
        g_host_maps.erase(it);
    }
    cudaError_t e = cudaHostUnregister(ptr);
    munmap(ptr, len);
    if (e != cudaSuccess) return cuda_fail(e, "cudaHostUnregister");
    return PL_OK;
}

}  // extern "C"
