// Internal host-side structures shared by the pylith_b200 translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/pylith_b200.h"

namespace plb {

// Device implementations of the pointwise kernels the registry knows about.
enum KernelId {
    K_NONE = 0,
    K_G0V_BODYFORCE,
    K_ILE_F1V,
    K_ILE_JF3VU,
    K_GM_F1V,
    K_GM_JF3VU,
    K_GM_VISCOUS_STRAIN,
    K_EL_STRAIN_VECTOR,
    K_ILE_STRESS_VECTOR,
    K_GM_STRESS_VECTOR,
    K_FCK_F0U_NEG,
    K_FCK_F0U_POS,
    K_FCK_F0L_SLIP,
    K_FCK_JF0UL_NEG,
    K_FCK_JF0UL_POS,
    K_FCK_JF0LU,
};

KernelId lookup_kernel(const void* fn);

// Incremented whenever an integrator's kernels, aux fields, constants or scatter change (or it is
// destroyed): solvers re-capture their CUDA graphs when the value differs from their capture's.
void bump_state_epoch();
unsigned long long state_epoch();

void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

// Device memory of the library's objects comes from a stream-ordered pool per device: creating
// and destroying meshes, integrators and solvers then neither maps memory nor synchronises the
// device (cudaMalloc and cudaFree do both), which matters when one process builds and drops
// problems on several streams at once. dev_alloc returns memory ready for use on any stream;
// dev_free returns p to the pool once the work enqueued on `after` so far has completed (pass the
// object's context stream: a call's work on private streams is joined into it before the call
// returns), without blocking the host.
cudaError_t dev_alloc(void** p, size_t bytes);
template <typename T>
inline cudaError_t dev_alloc(T** p, size_t count) {
    return dev_alloc(reinterpret_cast<void**>(p), count * sizeof(T));
}
void dev_free(void* p, cudaStream_t after);
// Releases the pool memory of `device` that no allocation holds.
void dev_pool_trim(int device);

#define PLB_CUDA(call)                                             \
    do {                                                           \
        cudaError_t _e = (call);                                   \
        if (_e != cudaSuccess) return ::plb::cuda_fail(_e, #call); \
    } while (0)

// Cell-block layout of a tetrahedral mesh for the shared-memory kernels (built once per mesh).
struct BlockedLayout {
    int cells_per_block = 0;
    int64_t num_blocks = 0;
    int max_local_nodes = 0;
    int32_t* d_cell_begin = nullptr;        // [num_blocks + 1] first cell of each block
    int32_t* d_block_node_begin = nullptr;  // [num_blocks + 1] into slot_node
    uint32_t* d_slot_node = nullptr;        // global node of each block-local slot (sorted per block),
                                            // high bit set if other blocks also touch the node
    uint16_t* d_local_cells = nullptr;      // [ncells][4] block-local slot of each cell corner
    uint32_t* d_inc_off = nullptr;          // per block: ns+1 offsets into the block's incidence list
    uint16_t* d_inc = nullptr;              // [num_blocks][4 * cells_per_block] (cell * 4 + corner)
    int64_t num_shared_nodes = 0;
    int64_t num_untouched = 0;
    int64_t num_slots = 0;                  // block-local node slots over all blocks
    // Nodes not owned by exactly one block (shared between blocks, or in no cell): the FP64
    // kernels leave them to a second pass that sums the blocks' partial sums in block order.
    int64_t num_fix = 0;
    int32_t* d_fix_node = nullptr;          // [num_fix] node ids
    int32_t* d_fix_off = nullptr;           // [num_fix + 1] offsets into d_fix_slot
    int32_t* d_fix_slot = nullptr;          // global slot ids of each node, in block order
    // Padded per-block regions of the pipelined kernel (k_tet_pipe): block b's slots start at
    // d_pipe_begin[b] (a multiple of 4) and span its slot count rounded up to 4.
    int32_t* d_pipe_begin = nullptr;        // [num_blocks + 1]
    uint32_t* d_pipe_ids = nullptr;         // node id | shared bit, per padded slot
    double* d_pipe_coords = nullptr;        // per block [3][padded slots] coordinates
    uint32_t* d_pipe_off = nullptr;         // per block, at d_pipe_begin[b] + 4 b: ns + 1 offsets
    uint32_t* d_pipe_ids_red = nullptr;     // as d_pipe_ids in the reduced fault space (node of the
                                            // reduced space | shared bit: the node has more than one
                                            // slot), built on first use
    uint32_t* d_slot_node_red = nullptr;    // as d_slot_node in the reduced fault space (same build)
    uint16_t* d_pipe_inc = nullptr;         // [num_blocks][4 * cells_per_block] staging offsets
                                            // corner * 3 * cells_per_block + cell, node groups of
                                            // the pipelined kernel
    size_t device_bytes = 0;
    // host copies for the reduced slot ids
    std::vector<uint32_t> h_pipe_ids;
    std::vector<int32_t> h_pipe_begin, h_block_node_begin;
};

void context_retain(pl_context_s* c);
void context_release(pl_context_s* c);
void mesh_retain(pl_mesh_s* m);
void mesh_release(pl_mesh_s* m);
void solver_retain(pl_solver_s* S);
void solver_release(pl_solver_s* S);
void integrator_retain(pl_integrator_s* ig);
void integrator_release(pl_integrator_s* ig);

}  // namespace plb

// Object lifetimes: meshes hold a reference on their context, integrators, matrices and solvers
// on their mesh, solvers on the integrators added to them, batched solvers on their solver; a
// destroy request on an object that is still referenced is deferred until the last dependent
// object is destroyed, so any destroy order is safe.
struct pl_context_s {
    int refs = 0;
    bool destroy_requested = false;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    unsigned int* d_err = nullptr;
    // staging buffer for the host-buffer entry points
    double* d_stage = nullptr;
    size_t d_stage_bytes = 0;
};

struct pl_mesh_s {
    int refs = 0;
    bool destroy_requested = false;
    pl_context ctx = nullptr;
    int cell_type = 0;
    int nen = 0;
    int nq = 0;
    int64_t ncells = 0;
    int64_t nnodes = 0;
    int32_t* d_cells = nullptr;
    double* d_coords = nullptr;
    std::vector<int32_t> h_cells;
    std::vector<double> h_coords;
    int64_t ncoh = 0;
    int64_t nlag = 0;
    int32_t* d_coh = nullptr;
    std::vector<int32_t> h_coh;
    plb::BlockedLayout* blocked = nullptr;
    // The solvers' reduced fault space (each fault node's positive side follows its negative
    // side): the connectivity with every positive-side node replaced by its negative-side
    // partner, built on first use, and dropped when the cohesive cells change.
    int32_t* d_cells_red = nullptr;
    std::vector<int32_t> h_node_red;  // node -> node of the reduced space
};

namespace plb {
struct AuxField {
    std::string name;
    int storage = PL_AUX_PER_CELL;
    int ncomp = 0;
    double* d = nullptr;  // device SoA: [ncomp][(nq)][ncells]
};
}  // namespace plb

struct pl_integrator_s {
    int refs = 0;
    bool destroy_requested = false;
    pl_mesh mesh = nullptr;
    bool is_interface = false;
    int64_t ncells = 0;                 // cells integrated over
    bool subset = false;                // created with a cell list (possibly empty)
    int32_t* d_cell_ids = nullptr;      // NULL: all cells of the mesh, in order (or none, for an empty subset)
    double* d_block_partial = nullptr;  // [num_slots][3] partial sums of shared nodes (cell-block kernels)
    std::vector<int32_t> h_cell_ids;
    // domain kernels
    plb::KernelId r0 = plb::K_NONE, r1 = plb::K_NONE;
    plb::KernelId j0 = plb::K_NONE, j3 = plb::K_NONE;
    std::vector<plb::KernelId> project;
    std::vector<std::string> project_subfields;
    std::vector<plb::KernelId> derived;  // derived-field (output) project kernels
    std::vector<std::string> derived_subfields;
    // interface kernels: residual per face and Jacobian per face
    plb::KernelId if_r[3] = {plb::K_NONE, plb::K_NONE, plb::K_NONE};
    plb::KernelId if_j[3] = {plb::K_NONE, plb::K_NONE, plb::K_NONE};
    std::vector<plb::AuxField> aux;
    std::vector<double> constants;
    int scatter = PL_SCATTER_AUTO;
    // per-cell (lambda, mu) for the FP32 Jacobian action (hexahedra, tetrahedra), valid for (lm32_t,
    // lm32_dt) until the aux fields or constants change
    float* d_lm32 = nullptr;
    bool lm32_valid = false;
    double lm32_t = 0.0, lm32_dt = 0.0;
};

struct pl_matrix_s {
    pl_mesh mesh = nullptr;
    int64_t nrows = 0;  // block rows: nodes + Lagrange nodes
    int64_t nnzb = 0;
    int32_t* d_row_ptr = nullptr;
    int32_t* d_col = nullptr;
    double* d_val = nullptr;
    int32_t* d_cell_pos = nullptr;  // [ncells][nen][nen] block index of each element block
    int32_t* d_coh_pos = nullptr;   // [ncoh][4 (blocks)][4][4]
};

// Device Krylov solver state (csrc/solver.cu); the batched solver (csrc/multirhs.cu) reuses its
// operator, mask, preconditioner and fault pairs.
struct pl_solver_s {
    int refs = 0;
    bool destroy_requested = false;
    pl_mesh mesh = nullptr;
    std::vector<pl_integrator> ops;
    bool reduced = false;  // the operator runs in the reduced fault space directly (set up by pl_solver_setup)
    int64_t n = 0;       // DOFs (3 per node)
    int64_t nnodes = 0;  // node rows
    uint8_t* d_mask = nullptr;
    uint8_t* d_dirichlet = nullptr;  // the caller's constrained DOFs alone (boundary-value insertion)
    double* d_diag = nullptr;
    double* d_pinv = nullptr;
    float* d_pinv32 = nullptr;
    double *d_r = nullptr, *d_p = nullptr, *d_q = nullptr, *d_z = nullptr, *d_x = nullptr;
    float *f_r = nullptr, *f_p = nullptr, *f_q = nullptr, *f_z = nullptr, *f_x = nullptr;
    double* d_scal = nullptr;
    double* d_partials = nullptr;
    int64_t npairs = 0;               // fault nodes (Lagrange nodes)
    int32_t* d_pair_neg = nullptr;    // negative-side node of each fault node
    int32_t* d_pair_pos = nullptr;    // positive-side node
    double* d_pair_normal = nullptr;  // fault normal at each fault node
    double rtol = 1e-12, atol = 0.0, inner_rtol = 1e-5;
    int max_iter = 10000, precision = 0, check_every = 10;
    // FP32_REFINED: reliable updates (residual replacement when the iterated residual has dropped
    // by reliable_delta) or, when off, restarted iterative refinement to inner_rtol per pass
    bool reliable = true;
    double reliable_delta = 0.1;
    double t = 0.0, dt = 0.0;
    int iterations = 0, inner_iterations = 0, outer_iterations = 0;
    double rel_residual = 0.0;
    bool ready = false;
    // PCG iterations run as a CUDA graph of check_every iterations (index 0: FP64, 1: FP32) on a
    // private stream fenced against the context's stream with events.
    double* d_xs = nullptr;  // FP64 PCG solution (the graph's fixed output buffer)
    cudaStream_t cstream = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int graph_iters[2] = {0, 0};
    unsigned long long graph_epoch[2] = {0, 0};
    // geometric multigrid preconditioner (pl_solver_set_multigrid): when set, pl_solver_solve runs
    // multigrid-preconditioned flexible CG instead of point-block-Jacobi PCG
    struct pl_multigrid_s* mg = nullptr;
};

namespace plb {
int multigrid_setup(pl_multigrid_s* mg, double t, double dt);
int multigrid_solve(pl_multigrid_s* mg, const double* b, double* x);
void multigrid_detach(pl_multigrid_s* mg);
// A hierarchy as the batched solver's V-cycles read it (csrc/multirhs.cu): per level its solver,
// sizes, transfer operators (prolongation columns and restriction rows in the coarse level's
// reduced fault space) and lambda_max(D^-1 A); the smoothing; the coarsest level's dense FP32
// inverse (dense_n 0: none). multigrid_prepare makes the eigenvalue estimates and the dense
// inverse current (outside stream capture).
struct MgLevelView {
    pl_solver_s* S;
    int64_t n, nn, nmesh;
    const int32_t *p_row, *p_col, *r_row, *r_col;
    const double *p_val, *r_val;
    double lmax;
};
struct MgView {
    std::vector<MgLevelView> levels;
    int degree;
    double lower;
    int coarse_degree;
    double coarse_lower;
    bool pre_smooth, post_smooth;
    const float* dense_inv32;
    const int32_t* dense_idx;
    int dense_n;
};
int multigrid_prepare(pl_multigrid_s* mg);
MgView multigrid_view(const pl_multigrid_s* mg);
void multigrid_batch_use(pl_multigrid_s* mg, int delta);
}  // namespace plb
