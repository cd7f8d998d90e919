// Kernel launchers shared between translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

struct pl_mesh_s;

struct pl_integrator_s;
struct pl_solver_s;

namespace plb {

struct DomainParams;
void launch_domain_diag_blocks(const DomainParams& p, int cell, int rheo, double* diag, cudaStream_t s);
struct BlockedLayout;

// Counts kernel launches made by this library (reported by pl_kernel_launches).
void count_launch(int n = 1);
// Raises a kernel's dynamic shared-memory limit to at least `bytes` on the current device; the
// attribute is set once per (kernel, device, size) instead of on every launch.
void ensure_kernel_smem(const void* kernel, size_t bytes);
// Multiprocessor count of the current device (queried once per device).
int sm_count();
bool launch_tangent_lm32(const DomainParams& p, int rheo, float* out, cudaStream_t s);

void launch_domain_apply_atomic(const DomainParams& p, int cell, int rheo, bool bf, int op,
                                cudaStream_t s);
void launch_domain_jv_f32_atomic(const DomainParams& p, int cell, int rheo, cudaStream_t s);
// Hexahedra (Q1, Q2) with a group of lanes per cell (FP64 residual / Jacobian action, FP64
// reductions into the output); returns false for other cell types.
bool launch_domain_apply_hexgroup(const DomainParams& p, int cell, int rheo, bool bf, int op, cudaStream_t s);
// FP32 Jacobian action of hexahedra with a group of lanes per cell (FP64 geometry and tangent).
bool launch_domain_jv32_hexgroup(const DomainParams& p, int cell, int rheo, cudaStream_t s);
void launch_domain_jacobian(const DomainParams& p, int cell, int rheo, const int32_t* pos,
                            double* vals, cudaStream_t s);
// Aux binding of a domain integrator for its registered Jacobian kernels.
int bind_domain_jacobian(pl_integrator_s* ig, DomainParams* p);
void launch_domain_update_state(const DomainParams& p, int cell, cudaStream_t s);
// Derived fields of basis order 0: up to 4 registered project kernels, 6 values each per cell.
struct DerivedSpec {
    int n;
    int kind[4];
};
void launch_domain_derived(const DomainParams& p, int cell, int rheo, const DerivedSpec& spec, cudaStream_t s);
// Builds (once per mesh) the cell-block layout used by the blocked scatter.
int ensure_blocked_layout(pl_mesh_s* m);
void free_blocked_layout(BlockedLayout* b, cudaStream_t after);
// Cell-block (shared-memory, deterministic) residual / Jacobian action; returns false when the
// layout does not support the configuration. reduced: the solvers' reduced fault space (slot ids
// of d_pipe_ids_red; padded-layout kernels only, no partial-sum buffer, output zeroed or holding
// the sum to add to).
bool launch_domain_apply_blocked(const DomainParams& p, const BlockedLayout& b, int cell,
                                 int rheo, bool bf, int op, bool insert, int64_t nnodes, double* partial,
                                 cudaStream_t s, bool reduced = false);
// The padded layout's slot ids in the reduced fault space (mesh with faults, after
// ensure_reduced_cells); call outside stream capture.
int ensure_reduced_ids(pl_mesh_s* m);
// The reduced fault space of a mesh with faults (csrc/capi.cu): connectivity and node map.
int ensure_reduced_cells(pl_mesh_s* m);
// J v in the solvers' reduced fault space without unfold and fold (csrc/capi.cu); supported: see
// jacobian_action_reduced_supported.
bool jacobian_action_reduced_supported(pl_integrator_s* ig);
int jacobian_action_reduced(pl_integrator_s* ig, double t, double dt, const double* v, double* jv, int mode);
int jacobian_action_reduced_f32(pl_integrator_s* ig, double t, double dt, const float* v, float* jv, int mode);
// The cell-block layout of the integrator's mesh and the integrator's partial-sum buffer
// (allocations: call outside stream capture).
int prepare_blocked(pl_integrator_s* ig);
// Fills the integrator's per-cell FP32 (lambda, mu) for the Jacobian action of hexahedra at
// (t, dt) when that path applies (no-op otherwise); call outside stream capture.
int prepare_jv32_tangent(pl_integrator_s* ig, double t, double dt);

// FP32 Q1 Jacobian action over many members' cells in one launch (the ragged batch; device
// tables: per-member operator arguments, warp-chunk prefix, active flags, member count).
void launch_hex8_jv32_ragged(const DomainParams* ops, const int64_t* chunk0, const int* active, const int* nmembers,
                             cudaStream_t s);
// Step-by-step FP32 reliable-update PCG of one solver for an outside iteration loop (solver.cu).
int solver32_begin(pl_solver_s* S, const double* b, double* x, double* b0);
int solver32_replace(pl_solver_s* S, const double* b, double* x, bool restart, bool keep_correction, double* rt);
// q = J v of a solver's integrators with its faults' unfold and fold; the unfold and fold alone.
int solver_apply_J(pl_solver_s* S, const double* v, double* out);
int solver_apply_J32(pl_solver_s* S, const float* v, float* out);
void solver_unfold(pl_solver_s* S, double* v);
void solver_unfold32(pl_solver_s* S, float* v);
void solver_fold(pl_solver_s* S, double* v);
void solver_fold32(pl_solver_s* S, float* v);
// P^T b for a solver with faults (in the solver's scratch vector), b otherwise.
const double* solver_reduced_rhs(pl_solver_s* S, const double* b);

// FP32 Jacobian action on the cell blocks (the output must be zeroed or hold the sum to add to).
bool launch_domain_jv32_blocked(const DomainParams& p, const BlockedLayout& b, int cell, int rheo, int64_t nnodes,
                                cudaStream_t s, bool reduced = false);

struct CohesiveParams {
    const int32_t* coh;      // [ncoh][12]
    int64_t ncoh;
    const double* coords;
    const double* u;         // full local vector
    const double* v;         // Jacobian-action direction
    double* out;
    const float* v32;
    float* out32;
    const double* slip;      // [nlag][3]
    int64_t lag_offset;      // 3 * nnodes
    double t, s_tshift;
    int num_constants;
    double constants[8];
    int kr[3];               // residual kernel per face (KernelId)
    int kj[3];               // Jacobian kernel per face
};

void launch_cohesive_residual(const CohesiveParams& p, cudaStream_t s);
void launch_cohesive_jv(const CohesiveParams& p, cudaStream_t s);
void launch_cohesive_jv_f32(const CohesiveParams& p, cudaStream_t s);
void launch_cohesive_jacobian(const CohesiveParams& p, const int32_t* pos, double* vals,
                              cudaStream_t s);

// Aux binding of an integrator for its registered residual kernels (rheology and body-force
// switch of a domain integrator are returned).
int bind_domain_residual(pl_integrator_s* ig, DomainParams* p, int* rheo, bool* bf);
int bind_cohesive_residual(pl_integrator_s* ig, CohesiveParams* p);

}  // namespace plb
