// C ABI of the pylith_b200 engine (include/pylith_b200.h): contexts, meshes, integrators with
// PyLith's kernel registration, the compute entry points and the assembled Jacobian.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "domain_kernels.cuh"
#include "internal.hpp"
#include "launch.hpp"

namespace plb {

static thread_local std::string g_last_error;
static std::atomic<long long> g_launches{0};
static std::atomic<unsigned long long> g_epoch{1};

void bump_state_epoch() { ++g_epoch; }
unsigned long long state_epoch() { return g_epoch.load(); }

void count_launch(int n) { g_launches += n; }

void ensure_kernel_smem(const void* kernel, size_t bytes) {
    if (bytes <= 48 * 1024) return;
    static std::mutex mu;
    static std::vector<std::pair<std::pair<const void*, int>, size_t>> set;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    for (auto& e : set)
        if (e.first.first == kernel && e.first.second == dev) {
            if (e.second >= bytes) return;
            cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
            e.second = bytes;
            return;
        }
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    set.push_back({{kernel, dev}, bytes});
}

int sm_count() {
    static int counts[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return 148;
    if (!counts[dev]) {
        int n = 148;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        counts[dev] = n;
    }
    return counts[dev];
}

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_pool_mutex;
cudaMemPool_t g_pools[kMaxDevices] = {};

cudaMemPool_t device_pool(int dev) {
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (!g_pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
        // keep up to 4 GiB of freed memory for reuse; never make an allocation wait on another
        // stream's frees (reuse only what is already free)
        uint64_t keep = 4ull << 30;
        int no = 0;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no);
        g_pools[dev] = pool;
    }
    return g_pools[dev];
}

// The calling thread's allocation stream on `dev` (one per thread, so that one thread's pending
// frees never hold up another thread's allocations).
cudaStream_t thread_alloc_stream(int dev) {
    thread_local cudaStream_t streams[kMaxDevices] = {};
    if (!streams[dev]) cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking);
    return streams[dev];
}

}  // namespace

cudaError_t dev_alloc(void** p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    cudaMemPool_t pool = device_pool(dev);
    cudaStream_t s = thread_alloc_stream(dev);
    if (!pool || !s) return cudaErrorNotSupported;
    e = cudaMallocFromPoolAsync(p, bytes, pool, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e;
}

void dev_free(void* p, cudaStream_t after) {
    if (!p) return;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return;
    cudaStream_t s = thread_alloc_stream(dev);
    if (after) {
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing(after, &cap);
        if (cap != cudaStreamCaptureStatusNone) return;  // no ordering is possible during a capture: keep it
        cudaEvent_t ev = nullptr;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess) {
            cudaEventRecord(ev, after);
            cudaStreamWaitEvent(s, ev, 0);
            cudaEventDestroy(ev);
        } else {
            cudaStreamSynchronize(after);
        }
    }
    cudaFreeAsync(p, s);
}

void dev_pool_trim(int device) {
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (device >= 0 && device < kMaxDevices && g_pools[device]) cudaMemPoolTrimTo(g_pools[device], 0);
}

int cuda_fail(cudaError_t e, const char* what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? PL_ERR_OUT_OF_MEMORY : PL_ERR_CUDA;
}

template <typename T>
static int alloc_n(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) return PL_OK;
    PLB_CUDA(dev_alloc(p, count));
    return PL_OK;
}

template <typename T>
static int upload(T** p, const T* host, size_t count, cudaStream_t s) {
    int rc = alloc_n(p, count);
    if (rc) return rc;
    if (count) PLB_CUDA(cudaMemcpyAsync(*p, host, count * sizeof(T), cudaMemcpyHostToDevice, s));
    return PL_OK;
}

static int nodes_per_cell(int type) { return type == PL_CELL_TET4 ? 4 : (type == PL_CELL_HEX8 ? 8 : 27); }
static int quad_points(int type) { return type == PL_CELL_TET4 ? 1 : (type == PL_CELL_HEX8 ? 8 : 27); }

static const AuxField* find_aux(const pl_integrator_s* ig, const char* name) {
    for (const AuxField& f : ig->aux)
        if (f.name == name) return &f;
    return nullptr;
}

static Rheology rheology_of(const pl_integrator_s* ig, bool jacobian) {
    const KernelId k = jacobian ? ig->j3 : ig->r1;
    if (k == K_ILE_F1V || k == K_ILE_JF3VU) return RHEO_ILE;
    if (k == K_GM_F1V || k == K_GM_JF3VU) return RHEO_GENMAXWELL;
    return RHEO_NONE;
}

// Fill the aux pointers of DomainParams; checks that every subfield the rheology reads exists.
static int bind_domain(pl_integrator_s* ig, Rheology rheo, bool bf, DomainParams* p) {
    std::memset(p, 0, sizeof(*p));
    pl_mesh m = ig->mesh;
    p->cells = m->d_cells;
    p->coords = m->d_coords;
    p->cell_ids = ig->d_cell_ids;
    p->ncells = ig->ncells;
    p->err = m->ctx->d_err;
    const AuxField* mu = find_aux(ig, "shear_modulus");
    const AuxField* K = find_aux(ig, "bulk_modulus");
    if (!mu || !K) return fail(PL_ERR_INVALID_ARG, "aux subfields shear_modulus and bulk_modulus are required");
    p->mu = mu->d;
    p->K = K->d;
    if (bf) {
        const AuxField* b = find_aux(ig, "body_force");
        if (!b || b->ncomp != 3) return fail(PL_ERR_INVALID_ARG, "aux subfield body_force(3) is required");
        p->body_force = b->d;
    }
    if (rheo == RHEO_GENMAXWELL) {
        const AuxField* tau = find_aux(ig, "maxwell_time");
        const AuxField* ratio = find_aux(ig, "shear_modulus_ratio");
        const AuxField* visc = find_aux(ig, "viscous_strain");
        const AuxField* tot = find_aux(ig, "total_strain");
        if (!tau || !ratio || !visc || !tot || tau->ncomp != 3 || ratio->ncomp != 3 ||
            visc->ncomp != 18 || tot->ncomp != 6 || visc->storage != PL_AUX_PER_QUADPT ||
            tot->storage != PL_AUX_PER_QUADPT)
            return fail(PL_ERR_INVALID_ARG,
                        "generalized Maxwell needs maxwell_time(3), shear_modulus_ratio(3) per cell "
                        "and viscous_strain(18), total_strain(6) per quadrature point");
        p->tau = tau->d;
        p->ratio = ratio->d;
        p->visc = visc->d;
        p->total = tot->d;
        if (ig->constants.empty()) return fail(PL_ERR_INVALID_ARG, "generalized Maxwell needs constants[0] = dt");
    }
    if (ig->constants.size() > 8) return fail(PL_ERR_UNSUPPORTED, "at most 8 kernel constants are supported");
    p->num_constants = (int)ig->constants.size();
    for (int i = 0; i < p->num_constants; ++i) p->constants[i] = ig->constants[i];
    return PL_OK;
}

static int bind_cohesive(pl_integrator_s* ig, CohesiveParams* p) {
    std::memset(p, 0, sizeof(*p));
    pl_mesh m = ig->mesh;
    if (!m->d_coh || m->ncoh == 0) return fail(PL_ERR_INVALID_ARG, "mesh has no cohesive cells");
    p->coh = m->d_coh;
    p->ncoh = m->ncoh;
    p->coords = m->d_coords;
    p->lag_offset = 3 * m->nnodes;
    const AuxField* slip = find_aux(ig, "slip");
    p->slip = slip ? slip->d : nullptr;
    if (ig->constants.size() > 8) return fail(PL_ERR_UNSUPPORTED, "at most 8 kernel constants are supported");
    p->num_constants = (int)ig->constants.size();
    for (int i = 0; i < p->num_constants; ++i) p->constants[i] = ig->constants[i];
    for (int f = 0; f < 3; ++f) {
        p->kr[f] = ig->if_r[f];
        p->kj[f] = ig->if_j[f];
    }
    return PL_OK;
}

int bind_domain_jacobian(pl_integrator_s* ig, DomainParams* p) {
    return bind_domain(ig, rheology_of(ig, true), false, p);
}

int bind_domain_residual(pl_integrator_s* ig, DomainParams* p, int* rheo, bool* bf) {
    *rheo = rheology_of(ig, false);
    *bf = ig->r0 == K_G0V_BODYFORCE;
    return bind_domain(ig, (Rheology)*rheo, *bf, p);
}

int bind_cohesive_residual(pl_integrator_s* ig, CohesiveParams* p) {
    int rc = bind_cohesive(ig, p);
    if (rc) return rc;
    if (ig->if_r[2] != K_NONE && !p->slip) return fail(PL_ERR_INVALID_ARG, "aux subfield slip is required");
    return PL_OK;
}

}  // namespace plb

using namespace plb;

// ---------------------------------------------------------------------------------------
extern "C" {

const char* pl_error_string(int code) {
    switch (code) {
        case PL_OK: return "ok";
        case PL_ERR_INVALID_ARG: return "invalid argument";
        case PL_ERR_UNKNOWN_KERNEL: return "unknown pointwise kernel";
        case PL_ERR_CUDA: return "CUDA error";
        case PL_ERR_OUT_OF_MEMORY: return "out of device memory";
        case PL_ERR_NOT_CONVERGED: return "solver did not converge";
        case PL_ERR_DEVICE_CHECK: return "device-side check failed";
        case PL_ERR_UNSUPPORTED: return "unsupported configuration";
        case PL_ERR_NOT_READY: return "not ready";
        default: return "unknown error";
    }
}

const char* pl_last_error(void) { return g_last_error.c_str(); }

int64_t pl_kernel_launches(void) { return (int64_t)g_launches.load(); }

int pl_context_create(int device, pl_context* out) {
    if (!out) return fail(PL_ERR_INVALID_ARG, "null output");
    *out = nullptr;
    int n = 0;
    PLB_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) return fail(PL_ERR_INVALID_ARG, "no such CUDA device");
    PLB_CUDA(cudaSetDevice(device));
    pl_context c = new pl_context_s();
    c->device = device;
    cudaError_t e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return cuda_fail(e, "cudaStreamCreate");
    }
    c->stream = c->own_stream;
    e = dev_alloc(&c->d_err, 1);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->d_err, 0, sizeof(unsigned int), c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        cudaStreamDestroy(c->own_stream);
        delete c;
        return cuda_fail(e, "device memory for the error word");
    }
    *out = c;
    return PL_OK;
}

static void context_free(pl_context c) {
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    dev_free(c->d_err, c->stream);
    dev_free(c->d_stage, c->stream);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    dev_pool_trim(c->device);
    delete c;
}

int pl_context_destroy(pl_context c) {
    if (!c) return PL_OK;
    if (c->refs > 0) {
        c->destroy_requested = true;
        return PL_OK;
    }
    context_free(c);
    return PL_OK;
}

int pl_context_set_stream(pl_context c, void* stream) {
    if (!c) return fail(PL_ERR_INVALID_ARG, "null context");
    c->stream = (cudaStream_t)stream;
    return PL_OK;
}

int pl_context_use_own_stream(pl_context c) {
    if (!c) return fail(PL_ERR_INVALID_ARG, "null context");
    c->stream = c->own_stream;
    return PL_OK;
}

void* pl_context_get_stream(pl_context c) { return c ? (void*)c->stream : nullptr; }

int pl_context_synchronize(pl_context c) {
    if (!c) return fail(PL_ERR_INVALID_ARG, "null context");
    PLB_CUDA(cudaSetDevice(c->device));
    PLB_CUDA(cudaStreamSynchronize(c->stream));
    PLB_CUDA(cudaGetLastError());
    unsigned int err = 0;
    PLB_CUDA(cudaMemcpy(&err, c->d_err, sizeof(err), cudaMemcpyDeviceToHost));
    if (err) {
        PLB_CUDA(cudaMemset(c->d_err, 0, sizeof(err)));
        char msg[128];
        std::snprintf(msg, sizeof(msg), "device check failed (flags 0x%x: %s)", err,
                      (err & CHECK_NONPOSITIVE_DETJ) ? "non-positive Jacobian determinant" : "index/value check");
        return fail(PL_ERR_DEVICE_CHECK, msg);
    }
    return PL_OK;
}

// ---- mesh -------------------------------------------------------------------------------
int pl_mesh_create(pl_context c, int cell_type, int64_t num_cells, const int32_t* cells,
                   int64_t num_nodes, const double* coords, pl_mesh* out) {
    if (!c || !out || !cells || !coords) return fail(PL_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    if (cell_type < PL_CELL_TET4 || cell_type > PL_CELL_HEX27)
        return fail(PL_ERR_INVALID_ARG, "unknown cell type");
    if (num_cells <= 0 || num_nodes <= 0 || num_nodes > INT32_MAX)
        return fail(PL_ERR_INVALID_ARG, "bad mesh sizes");
    const int nen = nodes_per_cell(cell_type);
    for (int64_t i = 0; i < num_cells * nen; ++i)
        if (cells[i] < 0 || cells[i] >= num_nodes)
            return fail(PL_ERR_INVALID_ARG, "cell node index out of range");
    PLB_CUDA(cudaSetDevice(c->device));
    pl_mesh m = new pl_mesh_s();
    m->ctx = c;
    c->refs++;
    m->cell_type = cell_type;
    m->nen = nen;
    m->nq = quad_points(cell_type);
    m->ncells = num_cells;
    m->nnodes = num_nodes;
    m->h_cells.assign(cells, cells + num_cells * nen);
    m->h_coords.assign(coords, coords + num_nodes * 3);
    int rc = upload(&m->d_cells, cells, num_cells * nen, c->stream);
    if (!rc) rc = upload(&m->d_coords, coords, num_nodes * 3, c->stream);
    if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = fail(PL_ERR_CUDA, "mesh upload");
    if (rc) {
        pl_mesh_destroy(m);
        return rc;
    }
    *out = m;
    return PL_OK;
}

int pl_mesh_set_cohesive(pl_mesh m, int64_t ncoh, const int32_t* coh, int64_t nlag) {
    if (!m || (ncoh > 0 && !coh) || ncoh < 0 || nlag < 0) return fail(PL_ERR_INVALID_ARG, "bad cohesive arguments");
    for (int64_t c = 0; c < ncoh; ++c)
        for (int k = 0; k < 12; ++k) {
            const int32_t v = coh[12 * c + k];
            const int64_t lim = k < 8 ? m->nnodes : nlag;
            if (v < 0 || v >= lim) return fail(PL_ERR_INVALID_ARG, "cohesive cell index out of range");
        }
    PLB_CUDA(cudaSetDevice(m->ctx->device));
    dev_free(m->d_coh, m->ctx->stream);
    m->d_coh = nullptr;
    dev_free(m->d_cells_red, m->ctx->stream);
    m->d_cells_red = nullptr;
    m->h_node_red.clear();
    if (m->blocked) {
        dev_free(m->blocked->d_pipe_ids_red, m->ctx->stream);
        m->blocked->d_pipe_ids_red = nullptr;
        dev_free(m->blocked->d_slot_node_red, m->ctx->stream);
        m->blocked->d_slot_node_red = nullptr;
    }
    bump_state_epoch();  // captured solver graphs hold the reduced connectivity
    m->ncoh = ncoh;
    m->nlag = nlag;
    m->h_coh.assign(coh, coh + 12 * ncoh);
    int rc = upload(&m->d_coh, coh, 12 * ncoh, m->ctx->stream);
    if (rc) return rc;
    PLB_CUDA(cudaStreamSynchronize(m->ctx->stream));
    return PL_OK;
}


static void mesh_free(pl_mesh m) {
    pl_context c = m->ctx;
    cudaSetDevice(m->ctx->device);
    cudaStreamSynchronize(m->ctx->stream);
    dev_free(m->d_cells, m->ctx->stream);
    dev_free(m->d_coords, m->ctx->stream);
    dev_free(m->d_coh, m->ctx->stream);
    dev_free(m->d_cells_red, m->ctx->stream);
    if (m->blocked) free_blocked_layout(m->blocked, m->ctx->stream);
    delete m;
    if (--c->refs == 0 && c->destroy_requested) context_free(c);
}

int pl_mesh_destroy(pl_mesh m) {
    if (!m) return PL_OK;
    if (m->refs > 0) {
        m->destroy_requested = true;
        return PL_OK;
    }
    mesh_free(m);
    return PL_OK;
}

extern "C++" {
namespace plb {
void context_retain(pl_context_s* c) { c->refs++; }
void context_release(pl_context_s* c) {
    if (--c->refs == 0 && c->destroy_requested) context_free(c);
}
void mesh_retain(pl_mesh_s* m) { m->refs++; }
void mesh_release(pl_mesh_s* m) {
    if (--m->refs == 0 && m->destroy_requested) mesh_free(m);
}
}  // namespace plb
}

int64_t pl_mesh_num_dof(pl_mesh m) { return m ? 3 * (m->nnodes + m->nlag) : 0; }

// ---- integrators --------------------------------------------------------------------------
int pl_integrator_domain_create(pl_mesh m, int64_t num_ids, const int32_t* ids, pl_integrator* out) {
    if (!m || !out || num_ids < 0) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    *out = nullptr;
    pl_integrator ig = new pl_integrator_s();
    ig->mesh = m;
    mesh_retain(m);
    ig->subset = ids != nullptr;  // a label that matches no cells gives an empty integrator
    if (ids && num_ids > 0) {
        for (int64_t i = 0; i < num_ids; ++i)
            if (ids[i] < 0 || ids[i] >= m->ncells) {
                delete ig;
                mesh_release(m);
                return fail(PL_ERR_INVALID_ARG, "cell id out of range");
            }
        ig->ncells = num_ids;
        ig->h_cell_ids.assign(ids, ids + num_ids);
        cudaSetDevice(m->ctx->device);
        int rc = upload(&ig->d_cell_ids, ids, num_ids, m->ctx->stream);
        if (rc) {
            delete ig;
            mesh_release(m);
            return rc;
        }
    } else {
        ig->ncells = ids ? 0 : m->ncells;
    }
    *out = ig;
    return PL_OK;
}

int pl_integrator_interface_create(pl_mesh m, pl_integrator* out) {
    if (!m || !out) return fail(PL_ERR_INVALID_ARG, "null argument");
    if (m->ncoh == 0) return fail(PL_ERR_INVALID_ARG, "mesh has no cohesive cells");
    pl_integrator ig = new pl_integrator_s();
    ig->mesh = m;
    mesh_retain(m);
    ig->is_interface = true;
    ig->ncells = m->ncoh;
    *out = ig;
    return PL_OK;
}

int pl_integrator_set_kernels_residual(pl_integrator ig, const pl_residual_kernels* k, int num) {
    bump_state_epoch();  // captured solver graphs hold kernel arguments
    if (!ig || ig->is_interface || (num > 0 && !k)) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    KernelId r0 = K_NONE, r1 = K_NONE;
    for (int i = 0; i < num; ++i) {
        if (!k[i].subfield || std::strcmp(k[i].subfield, "displacement") != 0)
            return fail(PL_ERR_UNSUPPORTED, "only the displacement subfield is supported");
        if (k[i].part != PL_LHS) return fail(PL_ERR_UNSUPPORTED, "only LHS (quasi-static) residual kernels are supported");
        const KernelId a = lookup_kernel((const void*)k[i].r0);
        const KernelId b = lookup_kernel((const void*)k[i].r1);
        if (a == (KernelId)-1 || b == (KernelId)-1)
            return fail(PL_ERR_UNKNOWN_KERNEL, "residual kernel address is not a registered pointwise kernel");
        if (a != K_NONE && a != K_G0V_BODYFORCE) return fail(PL_ERR_UNKNOWN_KERNEL, "unsupported f0 kernel");
        if (b != K_NONE && b != K_ILE_F1V && b != K_GM_F1V) return fail(PL_ERR_UNKNOWN_KERNEL, "unsupported f1 kernel");
        if (a != K_NONE) r0 = a;
        if (b != K_NONE) r1 = b;
    }
    if (r1 == K_NONE) return fail(PL_ERR_UNSUPPORTED, "an f1 (stress) kernel is required");
    ig->r0 = r0;
    ig->r1 = r1;
    return PL_OK;
}

int pl_integrator_set_kernels_jacobian(pl_integrator ig, const pl_jacobian_kernels* k, int num) {
    bump_state_epoch();  // captured solver graphs hold kernel arguments
    if (!ig || ig->is_interface || (num > 0 && !k)) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    KernelId j3 = K_NONE;
    for (int i = 0; i < num; ++i) {
        if (k[i].part != PL_LHS) return fail(PL_ERR_UNSUPPORTED, "only LHS Jacobian kernels are supported");
        if (k[i].j0 || k[i].j1 || k[i].j2) return fail(PL_ERR_UNKNOWN_KERNEL, "unsupported Jf0/Jf1/Jf2 kernel");
        const KernelId c = lookup_kernel((const void*)k[i].j3);
        if (c == (KernelId)-1) return fail(PL_ERR_UNKNOWN_KERNEL, "Jf3 address is not a registered pointwise kernel");
        if (c != K_NONE && c != K_ILE_JF3VU && c != K_GM_JF3VU) return fail(PL_ERR_UNKNOWN_KERNEL, "unsupported Jf3 kernel");
        if (c != K_NONE) j3 = c;
    }
    ig->j3 = j3;
    ig->lm32_valid = false;  // the cached FP32 tangent was evaluated with the previous Jf3
    return PL_OK;
}

int pl_integrator_set_kernels_update_state_vars(pl_integrator ig, const pl_project_kernels* k, int num) {
    bump_state_epoch();  // captured solver graphs hold kernel arguments
    if (!ig || ig->is_interface || (num > 0 && !k)) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    std::vector<KernelId> ids;
    std::vector<std::string> names;
    for (int i = 0; i < num; ++i) {
        const KernelId c = lookup_kernel((const void*)k[i].f);
        if (c != K_GM_VISCOUS_STRAIN && c != K_EL_STRAIN_VECTOR)
            return fail(PL_ERR_UNKNOWN_KERNEL, "unsupported state-update kernel");
        ids.push_back(c);
        names.push_back(k[i].subfield ? k[i].subfield : "");
    }
    ig->project = ids;
    ig->project_subfields = names;
    return PL_OK;
}

int pl_integrator_set_kernels_derived_field(pl_integrator ig, const pl_project_kernels* k, int num) {
    bump_state_epoch();  // captured solver graphs hold kernel arguments
    if (!ig || ig->is_interface || num < 0 || num > 4 || (num > 0 && !k))
        return fail(PL_ERR_INVALID_ARG, "bad arguments (at most 4 derived-field kernels)");
    std::vector<KernelId> ids;
    std::vector<std::string> names;
    for (int i = 0; i < num; ++i) {
        const KernelId c = lookup_kernel((const void*)k[i].f);
        if (c != K_EL_STRAIN_VECTOR && c != K_ILE_STRESS_VECTOR && c != K_GM_STRESS_VECTOR)
            return fail(PL_ERR_UNKNOWN_KERNEL, "unsupported derived-field kernel");
        ids.push_back(c);
        names.push_back(k[i].subfield ? k[i].subfield : "");
    }
    ig->derived = ids;
    ig->derived_subfields = names;
    return PL_OK;
}

int pl_integrator_interface_set_kernels_residual(pl_integrator ig, const pl_interface_residual_kernels* k, int num) {
    bump_state_epoch();  // captured solver graphs hold kernel arguments
    if (!ig || !ig->is_interface || (num > 0 && !k)) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    KernelId r[3] = {K_NONE, K_NONE, K_NONE};
    for (int i = 0; i < num; ++i) {
        if (k[i].face < 0 || k[i].face > 2) return fail(PL_ERR_INVALID_ARG, "bad face");
        if (k[i].r1) return fail(PL_ERR_UNKNOWN_KERNEL, "unsupported f1 interface kernel");
        const KernelId c = lookup_kernel((const void*)k[i].r0);
        const KernelId want = k[i].face == PL_FACE_NEGATIVE ? K_FCK_F0U_NEG
                              : (k[i].face == PL_FACE_POSITIVE ? K_FCK_F0U_POS : K_FCK_F0L_SLIP);
        if (c == (KernelId)-1) return fail(PL_ERR_UNKNOWN_KERNEL, "interface kernel address is not registered");
        if (c != K_NONE && c != want) return fail(PL_ERR_UNKNOWN_KERNEL, "kernel does not match its face");
        r[k[i].face] = c;
    }
    for (int f = 0; f < 3; ++f) ig->if_r[f] = r[f];
    return PL_OK;
}

int pl_integrator_interface_set_kernels_jacobian(pl_integrator ig, const pl_interface_jacobian_kernels* k, int num) {
    bump_state_epoch();  // captured solver graphs hold kernel arguments
    if (!ig || !ig->is_interface || (num > 0 && !k)) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    KernelId r[3] = {K_NONE, K_NONE, K_NONE};
    for (int i = 0; i < num; ++i) {
        if (k[i].face < 0 || k[i].face > 2) return fail(PL_ERR_INVALID_ARG, "bad face");
        if (k[i].j1 || k[i].j2 || k[i].j3) return fail(PL_ERR_UNKNOWN_KERNEL, "unsupported interface Jacobian kernel");
        const KernelId c = lookup_kernel((const void*)k[i].j0);
        const KernelId want = k[i].face == PL_FACE_NEGATIVE ? K_FCK_JF0UL_NEG
                              : (k[i].face == PL_FACE_POSITIVE ? K_FCK_JF0UL_POS : K_FCK_JF0LU);
        if (c == (KernelId)-1) return fail(PL_ERR_UNKNOWN_KERNEL, "interface kernel address is not registered");
        if (c != K_NONE && c != want) return fail(PL_ERR_UNKNOWN_KERNEL, "kernel does not match its face");
        r[k[i].face] = c;
    }
    for (int f = 0; f < 3; ++f) ig->if_j[f] = r[f];
    return PL_OK;
}

int pl_integrator_set_aux(pl_integrator ig, const char* name, int storage, int ncomp, const double* values) {
    bump_state_epoch();  // captured solver graphs hold kernel arguments
    if (!ig || !name || !values || ncomp <= 0 || ncomp > 64) return fail(PL_ERR_INVALID_ARG, "bad aux arguments");
    ig->lm32_valid = false;
    pl_mesh m = ig->mesh;
    int64_t nc = ig->ncells;
    int nq = 1;
    if (storage == PL_AUX_PER_QUADPT) {
        if (ig->is_interface) return fail(PL_ERR_UNSUPPORTED, "per-point aux on interfaces");
        nq = m->nq;
    } else if (storage == PL_AUX_PER_FAULT_NODE) {
        if (!ig->is_interface) return fail(PL_ERR_INVALID_ARG, "fault-node aux on a domain integrator");
        nc = m->nlag;
    } else if (storage != PL_AUX_PER_CELL) {
        return fail(PL_ERR_INVALID_ARG, "bad aux storage");
    }
    const size_t count = (size_t)nc * nq * ncomp;
    std::vector<double> dev(count);
    if (storage == PL_AUX_PER_FAULT_NODE) {
        std::memcpy(dev.data(), values, count * sizeof(double));  // [nlag][ncomp]
    } else {
        for (int64_t c = 0; c < nc; ++c)
            for (int q = 0; q < nq; ++q)
                for (int k = 0; k < ncomp; ++k)
                    dev[((size_t)k * nq + q) * nc + c] = values[((size_t)c * nq + q) * ncomp + k];
    }
    PLB_CUDA(cudaSetDevice(m->ctx->device));
    AuxField* f = nullptr;
    for (AuxField& a : ig->aux)
        if (a.name == name) f = &a;
    if (f && (f->ncomp != ncomp || f->storage != storage)) {
        dev_free(f->d, m->ctx->stream);
        f->d = nullptr;
    }
    if (!f) {
        ig->aux.push_back(AuxField());
        f = &ig->aux.back();
        f->name = name;
    }
    f->storage = storage;
    f->ncomp = ncomp;
    if (!f->d) {
        int rc = alloc_n(&f->d, count);
        if (rc) return rc;
    }
    PLB_CUDA(cudaMemcpyAsync(f->d, dev.data(), count * sizeof(double), cudaMemcpyHostToDevice, m->ctx->stream));
    PLB_CUDA(cudaStreamSynchronize(m->ctx->stream));
    return PL_OK;
}

int pl_integrator_get_aux(pl_integrator ig, const char* name, double* values) {
    if (!ig || !name || !values) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    const AuxField* f = find_aux(ig, name);
    if (!f) return fail(PL_ERR_INVALID_ARG, std::string("no aux subfield ") + name);
    pl_mesh m = ig->mesh;
    const int64_t nc = f->storage == PL_AUX_PER_FAULT_NODE ? m->nlag : ig->ncells;
    const int nq = f->storage == PL_AUX_PER_QUADPT ? m->nq : 1;
    const size_t count = (size_t)nc * nq * f->ncomp;
    std::vector<double> dev(count);
    PLB_CUDA(cudaSetDevice(m->ctx->device));
    PLB_CUDA(cudaMemcpyAsync(dev.data(), f->d, count * sizeof(double), cudaMemcpyDeviceToHost, m->ctx->stream));
    PLB_CUDA(cudaStreamSynchronize(m->ctx->stream));
    if (f->storage == PL_AUX_PER_FAULT_NODE) {
        std::memcpy(values, dev.data(), count * sizeof(double));
    } else {
        for (int64_t c = 0; c < nc; ++c)
            for (int q = 0; q < nq; ++q)
                for (int k = 0; k < f->ncomp; ++k)
                    values[((size_t)c * nq + q) * f->ncomp + k] = dev[((size_t)k * nq + q) * nc + c];
    }
    return PL_OK;
}

int pl_integrator_set_constants(pl_integrator ig, int num, const double* constants) {
    bump_state_epoch();  // captured solver graphs hold kernel arguments
    if (!ig || num < 0 || (num > 0 && !constants)) return fail(PL_ERR_INVALID_ARG, "bad constants");
    if (num > 8) return fail(PL_ERR_UNSUPPORTED, "at most 8 kernel constants are supported");
    ig->lm32_valid = false;
    ig->constants.assign(constants, constants + num);
    return PL_OK;
}

int pl_integrator_set_scatter(pl_integrator ig, int scatter) {
    bump_state_epoch();  // captured solver graphs hold kernel arguments
    if (!ig || scatter < PL_SCATTER_AUTO || scatter > PL_SCATTER_DETERMINISTIC) return fail(PL_ERR_INVALID_ARG, "bad scatter");
    ig->scatter = scatter;
    return PL_OK;
}

static void integrator_free(pl_integrator ig) {
    cudaSetDevice(ig->mesh->ctx->device);
    cudaStreamSynchronize(ig->mesh->ctx->stream);
    cudaStream_t s = ig->mesh->ctx->stream;
    for (AuxField& f : ig->aux) dev_free(f.d, s);
    dev_free(ig->d_cell_ids, s);
    dev_free(ig->d_block_partial, s);
    dev_free(ig->d_lm32, s);
    pl_mesh m = ig->mesh;
    delete ig;
    mesh_release(m);
}

int pl_integrator_destroy(pl_integrator ig) {
    bump_state_epoch();  // captured solver graphs hold kernel arguments
    if (!ig) return PL_OK;
    if (ig->refs > 0) {  // still used by a solver: freed when the last one releases it
        ig->destroy_requested = true;
        return PL_OK;
    }
    integrator_free(ig);
    return PL_OK;
}

// ---- compute ----------------------------------------------------------------------------


extern "C++" {
namespace plb {
void integrator_retain(pl_integrator_s* ig) { ig->refs++; }
void integrator_release(pl_integrator_s* ig) {
    if (--ig->refs == 0 && ig->destroy_requested) integrator_free(ig);
}

int prepare_jv32_tangent(pl_integrator_s* ig, double t, double dt) {
    pl_mesh m = ig->mesh;
    if (ig->is_interface || (m->cell_type != PL_CELL_HEX8 && m->cell_type != PL_CELL_TET4) || ig->j3 == K_NONE)
        return PL_OK;
    const Rheology rheo = rheology_of(ig, true);
    if (rheo != RHEO_ILE && rheo != RHEO_GENMAXWELL) return PL_OK;
    if (ig->lm32_valid && ig->lm32_t == t && ig->lm32_dt == dt) return PL_OK;
    DomainParams p;
    int rc = bind_domain(ig, rheo, false, &p);
    if (rc) return rc;
    p.t = t;
    p.dt = dt;
    if (!ig->d_lm32 && ig->ncells > 0) PLB_CUDA(dev_alloc(&ig->d_lm32, 2 * ig->ncells));
    launch_tangent_lm32(p, rheo, ig->d_lm32, m->ctx->stream);
    PLB_CUDA(cudaGetLastError());
    ig->lm32_valid = true;
    ig->lm32_t = t;
    ig->lm32_dt = dt;
    return PL_OK;
}

static bool use_blocked(pl_integrator ig) {
    pl_mesh m = ig->mesh;
    if (ig->scatter == PL_SCATTER_ATOMIC) return false;
    if (ig->subset) return false;  // the blocked layout covers whole meshes
    return m->cell_type == PL_CELL_TET4 || ig->scatter == PL_SCATTER_BLOCKED || ig->scatter == PL_SCATTER_DETERMINISTIC;
}

// The reduced fault space's connectivity (each positive-side node replaced by its negative-side
// partner) and node map. Refused (PL_ERR_UNSUPPORTED) when a pair's two nodes do not coincide:
// the kernels then read the partner's coordinates in place of the node's own.
int ensure_reduced_cells(pl_mesh_s* m) {
    if (m->d_cells_red) return PL_OK;
    if (m->ncoh == 0) return PL_ERR_UNSUPPORTED;
    std::vector<int32_t> red(m->nnodes);
    for (int64_t v = 0; v < m->nnodes; ++v) red[v] = (int32_t)v;
    double scale = 0.0;
    for (double x : m->h_coords) scale = std::max(scale, std::fabs(x));
    for (int64_t c = 0; c < m->ncoh; ++c)
        for (int a = 0; a < 4; ++a) {
            const int32_t neg = m->h_coh[12 * c + a], pos = m->h_coh[12 * c + 4 + a];
            for (int d = 0; d < 3; ++d)
                if (std::fabs(m->h_coords[3 * (size_t)neg + d] - m->h_coords[3 * (size_t)pos + d]) > 1e-12 * scale)
                    return PL_ERR_UNSUPPORTED;
            red[pos] = neg;
        }
    std::vector<int32_t> cells(m->h_cells.size());
    for (size_t i = 0; i < cells.size(); ++i) cells[i] = red[m->h_cells[i]];
    int32_t* d = nullptr;
    PLB_CUDA(dev_alloc(&d, cells.size()));
    PLB_CUDA(cudaMemcpyAsync(d, cells.data(), cells.size() * sizeof(int32_t), cudaMemcpyHostToDevice, m->ctx->stream));
    PLB_CUDA(cudaStreamSynchronize(m->ctx->stream));
    m->d_cells_red = d;
    m->h_node_red.swap(red);
    return PL_OK;
}

// Whether jacobian_action_reduced(_f32) serves this integrator (domain cells of a mesh with
// faults whose node pairs coincide, not the deterministic scatter, and for cell blocks a padded
// layout kernel).
bool jacobian_action_reduced_supported(pl_integrator_s* ig) {
    if (!ig || ig->is_interface || ig->j3 == K_NONE || ig->scatter == PL_SCATTER_DETERMINISTIC) return false;
    pl_mesh m = ig->mesh;
    if (ensure_reduced_cells(m) != PL_OK) return false;
    // the cell-block path of tetrahedra needs the reduced slot ids (built here, outside capture)
    if (use_blocked(ig) && m->cell_type == PL_CELL_TET4)
        return prepare_blocked(ig) == PL_OK && ensure_reduced_ids(m) == PL_OK;
    return true;
}

// J v of the solvers' reduced fault space without unfolding v or folding the result: every
// positive-side node is read as, and adds into, its negative-side partner (v's positive-side
// entries are not read; the result's are zero after INSERT).
int jacobian_action_reduced(pl_integrator_s* ig, double t, double dt, const double* v, double* jv, int mode) {
    pl_mesh m = ig->mesh;
    cudaStream_t s = m->ctx->stream;
    int rc = ensure_reduced_cells(m);
    if (rc) return rc;
    const Rheology rheo = rheology_of(ig, true);
    DomainParams p;
    if ((rc = bind_domain(ig, rheo, false, &p)) != PL_OK) return rc;
    p.cells = m->d_cells_red;
    p.v = v;
    p.out = jv;
    p.t = t;
    p.dt = dt;
    if (mode == PL_INSERT) PLB_CUDA(cudaMemsetAsync(jv, 0, pl_mesh_num_dof(m) * sizeof(double), s));
    if (use_blocked(ig) && m->cell_type == PL_CELL_TET4) {
        if ((rc = prepare_blocked(ig)) != PL_OK || (rc = ensure_reduced_ids(m)) != PL_OK) return rc;
        if (!launch_domain_apply_blocked(p, *m->blocked, m->cell_type, rheo, false, OP_JACOBIAN_ACTION, false, m->nnodes,
                                         nullptr, s, true))
            return PL_ERR_UNSUPPORTED;
    } else if (ig->scatter == PL_SCATTER_ATOMIC ||
               !launch_domain_apply_hexgroup(p, m->cell_type, rheo, false, OP_JACOBIAN_ACTION, s)) {
        launch_domain_apply_atomic(p, m->cell_type, rheo, false, OP_JACOBIAN_ACTION, s);
    }
    PLB_CUDA(cudaGetLastError());
    return PL_OK;
}

int jacobian_action_reduced_f32(pl_integrator_s* ig, double t, double dt, const float* v, float* jv, int mode) {
    pl_mesh m = ig->mesh;
    cudaStream_t s = m->ctx->stream;
    int rc = ensure_reduced_cells(m);
    if (rc) return rc;
    const Rheology rheo = rheology_of(ig, true);
    DomainParams p;
    if ((rc = bind_domain(ig, rheo, false, &p)) != PL_OK) return rc;
    p.cells = m->d_cells_red;
    p.v32 = v;
    p.out32 = jv;
    p.t = t;
    p.dt = dt;
    if ((m->cell_type == PL_CELL_HEX8 || m->cell_type == PL_CELL_TET4) && ig->lm32_valid && ig->lm32_t == t &&
        ig->lm32_dt == dt)
        p.lm32 = ig->d_lm32;
    if (mode == PL_INSERT) PLB_CUDA(cudaMemsetAsync(jv, 0, pl_mesh_num_dof(m) * sizeof(float), s));
    if (use_blocked(ig) && m->cell_type == PL_CELL_TET4) {
        if ((rc = ensure_blocked_layout(m)) != PL_OK || (rc = ensure_reduced_ids(m)) != PL_OK) return rc;
        if (!launch_domain_jv32_blocked(p, *m->blocked, m->cell_type, rheo, m->nnodes, s, true)) return PL_ERR_UNSUPPORTED;
    } else if (ig->scatter == PL_SCATTER_ATOMIC || !launch_domain_jv32_hexgroup(p, m->cell_type, rheo, s)) {
        launch_domain_jv_f32_atomic(p, m->cell_type, rheo, s);
    }
    PLB_CUDA(cudaGetLastError());
    return PL_OK;
}

int prepare_blocked(pl_integrator_s* ig) {
    pl_mesh m = ig->mesh;
    int rc = ensure_blocked_layout(m);
    if (rc) return rc;
    if (ig->scatter == PL_SCATTER_DETERMINISTIC && !ig->d_block_partial && m->blocked->num_slots > 0)
        PLB_CUDA(dev_alloc(&ig->d_block_partial, 3 * m->blocked->num_slots));
    return PL_OK;
}
}  // namespace plb
}


int pl_compute_lhs_residual(pl_integrator ig, double t, double dt, const double* u, const double* u_t,
                            double* r, int mode) {
    if (!ig || !u || !r || (mode != PL_INSERT && mode != PL_ADD)) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    pl_mesh m = ig->mesh;
    cudaStream_t s = m->ctx->stream;
    PLB_CUDA(cudaSetDevice(m->ctx->device));
    if (ig->is_interface) {
        CohesiveParams p;
        int rc = bind_cohesive(ig, &p);
        if (rc) return rc;
        if (ig->if_r[2] != K_NONE && !p.slip) return fail(PL_ERR_INVALID_ARG, "aux subfield slip is required");
        p.u = u;
        p.out = r;
        p.t = t;
        if (mode == PL_INSERT) PLB_CUDA(cudaMemsetAsync(r, 0, pl_mesh_num_dof(m) * sizeof(double), s));
        launch_cohesive_residual(p, s);
        PLB_CUDA(cudaGetLastError());
        return PL_OK;
    }
    if (ig->r1 == K_NONE) return fail(PL_ERR_NOT_READY, "no residual kernels registered");
    const Rheology rheo = rheology_of(ig, false);
    const bool bf = ig->r0 == K_G0V_BODYFORCE;
    DomainParams p;
    int rc = bind_domain(ig, rheo, bf, &p);
    if (rc) return rc;
    p.u = u;
    p.out = r;
    p.t = t;
    p.dt = dt;
    if (use_blocked(ig) && (rc = prepare_blocked(ig)) == PL_OK &&
        launch_domain_apply_blocked(p, *m->blocked, m->cell_type, rheo, bf, OP_RESIDUAL, mode == PL_INSERT,
                                    m->nnodes, ig->scatter == PL_SCATTER_DETERMINISTIC ? ig->d_block_partial : nullptr,
                                    s)) {
        if (mode == PL_INSERT && m->nlag > 0)
            PLB_CUDA(cudaMemsetAsync(r + 3 * m->nnodes, 0, 3 * m->nlag * sizeof(double), s));
        PLB_CUDA(cudaGetLastError());
        return PL_OK;
    }
    if (rc) return rc;
    if (mode == PL_INSERT) PLB_CUDA(cudaMemsetAsync(r, 0, pl_mesh_num_dof(m) * sizeof(double), s));
    if (ig->scatter == PL_SCATTER_ATOMIC ||
        !launch_domain_apply_hexgroup(p, m->cell_type, rheo, bf, OP_RESIDUAL, s))
        launch_domain_apply_atomic(p, m->cell_type, rheo, bf, OP_RESIDUAL, s);
    PLB_CUDA(cudaGetLastError());
    return PL_OK;
}

int pl_compute_lhs_jacobian_action(pl_integrator ig, double t, double dt, double s_tshift, const double* u,
                                   const double* v, double* jv, int mode) {
    if (!ig || !v || !jv || (mode != PL_INSERT && mode != PL_ADD)) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    pl_mesh m = ig->mesh;
    cudaStream_t s = m->ctx->stream;
    PLB_CUDA(cudaSetDevice(m->ctx->device));
    if (ig->is_interface) {
        CohesiveParams p;
        int rc = bind_cohesive(ig, &p);
        if (rc) return rc;
        p.u = u;
        p.v = v;
        p.out = jv;
        p.t = t;
        p.s_tshift = s_tshift;
        if (mode == PL_INSERT) PLB_CUDA(cudaMemsetAsync(jv, 0, pl_mesh_num_dof(m) * sizeof(double), s));
        launch_cohesive_jv(p, s);
        PLB_CUDA(cudaGetLastError());
        return PL_OK;
    }
    if (ig->j3 == K_NONE) return fail(PL_ERR_NOT_READY, "no Jacobian kernels registered");
    const Rheology rheo = rheology_of(ig, true);
    DomainParams p;
    int rc = bind_domain(ig, rheo, false, &p);
    if (rc) return rc;
    p.u = u;
    p.v = v;
    p.out = jv;
    p.t = t;
    p.dt = dt;
    p.s_tshift = s_tshift;
    if (use_blocked(ig) && (rc = prepare_blocked(ig)) == PL_OK &&
        launch_domain_apply_blocked(p, *m->blocked, m->cell_type, rheo, false, OP_JACOBIAN_ACTION, mode == PL_INSERT,
                                    m->nnodes, ig->scatter == PL_SCATTER_DETERMINISTIC ? ig->d_block_partial : nullptr,
                                    s)) {
        if (mode == PL_INSERT && m->nlag > 0)
            PLB_CUDA(cudaMemsetAsync(jv + 3 * m->nnodes, 0, 3 * m->nlag * sizeof(double), s));
        PLB_CUDA(cudaGetLastError());
        return PL_OK;
    }
    if (rc) return rc;
    if (mode == PL_INSERT) PLB_CUDA(cudaMemsetAsync(jv, 0, pl_mesh_num_dof(m) * sizeof(double), s));
    if (ig->scatter == PL_SCATTER_ATOMIC ||
        !launch_domain_apply_hexgroup(p, m->cell_type, rheo, false, OP_JACOBIAN_ACTION, s))
        launch_domain_apply_atomic(p, m->cell_type, rheo, false, OP_JACOBIAN_ACTION, s);
    PLB_CUDA(cudaGetLastError());
    return PL_OK;
}

int pl_compute_lhs_jacobian_action_f32(pl_integrator ig, double t, double dt, const float* v, float* jv, int mode) {
    if (!ig || !v || !jv || (mode != PL_INSERT && mode != PL_ADD)) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    pl_mesh m = ig->mesh;
    cudaStream_t s = m->ctx->stream;
    PLB_CUDA(cudaSetDevice(m->ctx->device));
    if (mode == PL_INSERT) PLB_CUDA(cudaMemsetAsync(jv, 0, pl_mesh_num_dof(m) * sizeof(float), s));
    if (ig->is_interface) {
        CohesiveParams p;
        int rc = bind_cohesive(ig, &p);
        if (rc) return rc;
        p.v32 = v;
        p.out32 = jv;
        p.t = t;
        launch_cohesive_jv_f32(p, s);
        PLB_CUDA(cudaGetLastError());
        return PL_OK;
    }
    if (ig->j3 == K_NONE) return fail(PL_ERR_NOT_READY, "no Jacobian kernels registered");
    const Rheology rheo = rheology_of(ig, true);
    DomainParams p;
    int rc = bind_domain(ig, rheo, false, &p);
    if (rc) return rc;
    p.v32 = v;
    p.out32 = jv;
    p.t = t;
    p.dt = dt;
    if ((m->cell_type == PL_CELL_HEX8 || m->cell_type == PL_CELL_TET4) && ig->lm32_valid && ig->lm32_t == t &&
        ig->lm32_dt == dt)
        p.lm32 = ig->d_lm32;
    if (use_blocked(ig) && (rc = ensure_blocked_layout(m)) == PL_OK &&
        launch_domain_jv32_blocked(p, *m->blocked, m->cell_type, rheo, m->nnodes, s)) {
        PLB_CUDA(cudaGetLastError());
        return PL_OK;
    }
    if (rc) return rc;
    if (ig->scatter == PL_SCATTER_ATOMIC || !launch_domain_jv32_hexgroup(p, m->cell_type, rheo, s))
        launch_domain_jv_f32_atomic(p, m->cell_type, rheo, s);
    PLB_CUDA(cudaGetLastError());
    return PL_OK;
}

int pl_compute_lhs_residual_host(pl_integrator ig, double t, double dt, const double* u_host, double* r_host) {
    if (!ig || !u_host || !r_host) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    pl_mesh m = ig->mesh;
    pl_context c = m->ctx;
    const size_t n = (size_t)pl_mesh_num_dof(m);
    const size_t bytes = 2 * n * sizeof(double);
    PLB_CUDA(cudaSetDevice(c->device));
    if (c->d_stage_bytes < bytes) {
        dev_free(c->d_stage, c->stream);
        c->d_stage = nullptr;
        c->d_stage_bytes = 0;
        PLB_CUDA(dev_alloc((void**)&c->d_stage, bytes));
        c->d_stage_bytes = bytes;
    }
    double* du = c->d_stage;
    double* dr = c->d_stage + n;
    PLB_CUDA(cudaMemcpyAsync(du, u_host, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    int rc = pl_compute_lhs_residual(ig, t, dt, du, nullptr, dr, PL_INSERT);
    if (rc) return rc;
    PLB_CUDA(cudaMemcpyAsync(r_host, dr, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    return pl_context_synchronize(c);
}

int pl_update_state_vars(pl_integrator ig, double t, double dt, const double* u) {
    if (!ig || !u || ig->is_interface) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    if (ig->project.empty()) return fail(PL_ERR_NOT_READY, "no state-update kernels registered");
    bool has_visc = false, has_total = false;
    for (KernelId k : ig->project) {
        has_visc |= k == K_GM_VISCOUS_STRAIN;
        has_total |= k == K_EL_STRAIN_VECTOR;
    }
    if (!has_visc || !has_total)
        return fail(PL_ERR_UNSUPPORTED, "state update needs the viscous-strain and total-strain kernels");
    pl_mesh m = ig->mesh;
    PLB_CUDA(cudaSetDevice(m->ctx->device));
    DomainParams p;
    int rc = bind_domain(ig, RHEO_GENMAXWELL, false, &p);
    if (rc) return rc;
    p.u = u;
    p.t = t;
    p.dt = dt;
    launch_domain_update_state(p, m->cell_type, m->ctx->stream);
    PLB_CUDA(cudaGetLastError());
    return PL_OK;
}

int pl_compute_derived_field(pl_integrator ig, double t, double dt, const double* u, double* out) {
    if (!ig || !u || !out || ig->is_interface) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    if (ig->derived.empty()) return fail(PL_ERR_NOT_READY, "no derived-field kernels registered");
    pl_mesh m = ig->mesh;
    const Rheology rheo = rheology_of(ig, false) != RHEO_NONE ? rheology_of(ig, false) : rheology_of(ig, true);
    DerivedSpec spec;
    spec.n = (int)ig->derived.size();
    for (int i = 0; i < spec.n; ++i) {
        const KernelId k = ig->derived[i];
        if (k == K_ILE_STRESS_VECTOR && rheo != RHEO_ILE)
            return fail(PL_ERR_INVALID_ARG, "the isotropic linear elastic stress needs an isotropic linear elastic material");
        if (k == K_GM_STRESS_VECTOR && rheo != RHEO_GENMAXWELL)
            return fail(PL_ERR_INVALID_ARG, "the generalized Maxwell stress needs a generalized Maxwell material");
        if (k == K_GM_STRESS_VECTOR && m->cell_type != PL_CELL_TET4)
            return fail(PL_ERR_UNSUPPORTED,
                        "the generalized Maxwell stress of basis order 0 needs the state at the centroid "
                        "(P1 tetrahedra, whose single quadrature point is the centroid)");
        spec.kind[i] = (int)k;
    }
    if (rheo == RHEO_NONE) return fail(PL_ERR_NOT_READY, "register the material's residual or Jacobian kernels first");
    PLB_CUDA(cudaSetDevice(m->ctx->device));
    DomainParams p;
    int rc = bind_domain(ig, rheo, false, &p);
    if (rc) return rc;
    p.u = u;
    p.out = out;
    p.t = t;
    p.dt = dt;
    launch_domain_derived(p, m->cell_type, rheo, spec, m->ctx->stream);
    PLB_CUDA(cudaGetLastError());
    return PL_OK;
}

}  // extern "C"
