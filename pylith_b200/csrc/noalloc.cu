// Host-buffer residual that allocates no device memory.
//
// pl_compute_lhs_residual_host copies the host solution to the device, computes the residual
// there and copies it back, through staging buffers that the context allocates (cudaMalloc) on
// first use and regrows when a larger mesh comes along; for P1 tetrahedra it also builds the
// cell-block layout on first use. Some callers cannot let a call allocate:
//  * a process whose device memory is all handed out up front by a pool it does not own
//    (a solver service that reserves nearly all of HBM for resident meshes), where a cudaMalloc
//    inside a call fails or evicts someone else's data;
//  * a time-step loop with a latency bound, where cudaMalloc/cudaFree can synchronise the whole
//    device and stall every stream for an unbounded time;
//  * code that reports its device memory to a budget at start-up (the serving admission in
//    pylith_b200/serving.py) and must not grow behind that budget's back.
// pl_compute_lhs_residual_host_noalloc stages through one fixed file-scope device array
// instead and computes the residual with the thread-per-cell kernels, which need no layout.
//
// Limits and rules:
//  * The array holds kNoAllocMaxDof solution values and kNoAllocMaxDof residual values
//    (2 x 2^20 doubles = 16 MiB). Every GPU on which the library's module is loaded holds it
//    until the process exits. Meshes with more DOFs are rejected with PL_ERR_INVALID_ARG.
//  * Its device address is looked up on the first call made on each device (with that device
//    current); make that first call before any stream capture begins. The address is kept for the
//    life of the process: after cudaDeviceReset (or any teardown of the device's primary context)
//    the module may be loaded at another address, so the entry point must not be used on that
//    device again.
//  * All calls share the array, and it keeps the last call's contents; the residual half is
//    cleared at the start of every call. Calls whose GPU work overlaps (from two host threads,
//    or on two contexts with different streams) race on the array. Each call ends by waiting
//    for its own stream, so calls made one after another from one thread do not overlap.
#include <mutex>

#include "domain_kernels.cuh"
#include "internal.hpp"
#include "launch.hpp"

namespace plb {

constexpr int64_t kNoAllocMaxDof = int64_t(1) << 20;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[2 * kNoAllocMaxDof];

static std::mutex g_noalloc_mutex;
static double* g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};

// Device address of the scratch array on `device` (the current device); looked up once.
static int noalloc_scratch(int device, double** out) {
    if (device < 0 || device >= kNoAllocMaxDevices) return fail(PL_ERR_INVALID_ARG, "device index out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[device]) {
        void* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(staging array)");
        g_noalloc_ptr[device] = static_cast<double*>(ptr);
    }
    *out = g_noalloc_ptr[device];
    return PL_OK;
}

}  // namespace plb

using namespace plb;

extern "C" int pl_compute_lhs_residual_host_noalloc(pl_integrator ig, double t, double dt, const double* u_host,
                                                    double* r_host) {
    if (!ig || !u_host || !r_host) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    pl_mesh m = ig->mesh;
    pl_context c = m->ctx;
    const int64_t n = pl_mesh_num_dof(m);
    if (n > kNoAllocMaxDof)
        return fail(PL_ERR_INVALID_ARG,
                    "pl_compute_lhs_residual_host_noalloc: " + std::to_string(n) +
                        " DOFs exceed the fixed staging array of 1048576 DOFs");
    PLB_CUDA(cudaSetDevice(c->device));
    double* scratch = nullptr;
    int rc = noalloc_scratch(c->device, &scratch);
    if (rc) return rc;
    double* du = scratch;
    double* dr = scratch + kNoAllocMaxDof;
    const cudaStream_t s = c->stream;
    if (ig->is_interface) {
        CohesiveParams p;
        if ((rc = bind_cohesive_residual(ig, &p))) return rc;
        p.u = du;
        p.out = dr;
        p.t = t;
        PLB_CUDA(cudaMemcpyAsync(du, u_host, n * sizeof(double), cudaMemcpyHostToDevice, s));
        PLB_CUDA(cudaMemsetAsync(dr, 0, n * sizeof(double), s));
        launch_cohesive_residual(p, s);
    } else {
        if (ig->r1 == K_NONE) return fail(PL_ERR_NOT_READY, "no residual kernels registered");
        DomainParams p;
        int rheo = 0;
        bool bf = false;
        if ((rc = bind_domain_residual(ig, &p, &rheo, &bf))) return rc;
        p.u = du;
        p.out = dr;
        p.t = t;
        p.dt = dt;
        PLB_CUDA(cudaMemcpyAsync(du, u_host, n * sizeof(double), cudaMemcpyHostToDevice, s));
        PLB_CUDA(cudaMemsetAsync(dr, 0, n * sizeof(double), s));
        launch_domain_apply_atomic(p, m->cell_type, rheo, bf, OP_RESIDUAL, s);
    }
    PLB_CUDA(cudaGetLastError());
    PLB_CUDA(cudaMemcpyAsync(r_host, dr, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    return pl_context_synchronize(c);
}
