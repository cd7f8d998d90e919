/*
 * pylith_b200 — C ABI of the B200 (sm_100a) finite-element residual/Jacobian engine.
 *
 * This is the drop-in boundary for PyLith's per-cell residual and Jacobian loop. In the
 * reference that loop is PETSc's DMPlexComputeResidualByKey / DMPlexComputeJacobianByKey /
 * DMPlexCompute{Residual,Jacobian}HybridByKey / DMProjectFieldLocal, driven by
 * IntegratorDomain and IntegratorInterface. Each entry point below names the reference
 * interface it replaces (paths relative to the PyLith source tree).
 *
 * Conventions
 *   - Every function returns PL_OK (0) or a negative PL_ERR_* code; nothing throws across
 *     the ABI. pl_last_error() returns a message for the calling thread's last failure.
 *   - Pointers named *_dev are device pointers (cudaMalloc'd or torch-owned); *_host are
 *     host pointers. The library never frees caller memory.
 *   - Local vectors follow the reference's local-vector semantics
 *     (docs/developer/implementation/petsc-fem.md:60-75): 3 displacement DOFs per mesh node
 *     (constrained DOFs included, holding their boundary values), followed, for meshes with
 *     a fault, by 3 Lagrange-multiplier DOFs per fault node.
 *   - Work is enqueued on the context's stream; results are ready after that stream
 *     synchronises. A context is used by one host thread at a time.
 *   - Pointwise kernels are identified by the address of the host function with PETSc's
 *     pointwise signature (the same function pointers PyLith hands to PetscWeakForm). The
 *     library maps each known address to its device implementation; an unknown address is
 *     rejected with PL_ERR_UNKNOWN_KERNEL (there is no CPU fallback).
 */
#ifndef PYLITH_B200_H
#define PYLITH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PL_OK 0
#define PL_ERR_INVALID_ARG (-1)
#define PL_ERR_UNKNOWN_KERNEL (-2)
#define PL_ERR_CUDA (-3)
#define PL_ERR_OUT_OF_MEMORY (-4)
#define PL_ERR_NOT_CONVERGED (-5)
#define PL_ERR_DEVICE_CHECK (-6)
#define PL_ERR_UNSUPPORTED (-7)
#define PL_ERR_NOT_READY (-8)

/* Scalar types of the reference (libsrc/pylith/utils/types.hh:14-16 with PETSc real
 * double, 32-bit indices). */
typedef int PylithInt;
typedef double PylithReal;
typedef double PylithScalar;

/* PETSc pointwise-function signatures (docs/developer/implementation/petsc-fem.md:438-600;
 * libsrc/pylith/fekernels/Elasticity.hh:125-142, FaultCohesiveKin.hh:74-92,298-317). */
typedef void (*PetscPointFn)(PylithInt dim, PylithInt numS, PylithInt numA, const PylithInt sOff[],
                             const PylithInt sOff_x[], const PylithScalar s[],
                             const PylithScalar s_t[], const PylithScalar s_x[],
                             const PylithInt aOff[], const PylithInt aOff_x[],
                             const PylithScalar a[], const PylithScalar a_t[],
                             const PylithScalar a_x[], PylithReal t, const PylithScalar x[],
                             PylithInt numConstants, const PylithScalar constants[],
                             PylithScalar f[]);
typedef void (*PetscPointJacFn)(PylithInt dim, PylithInt numS, PylithInt numA,
                                const PylithInt sOff[], const PylithInt sOff_x[],
                                const PylithScalar s[], const PylithScalar s_t[],
                                const PylithScalar s_x[], const PylithInt aOff[],
                                const PylithInt aOff_x[], const PylithScalar a[],
                                const PylithScalar a_t[], const PylithScalar a_x[], PylithReal t,
                                PylithReal s_tshift, const PylithScalar x[],
                                PylithInt numConstants, const PylithScalar constants[],
                                PylithScalar g[]);
typedef void (*PetscBdPointFn)(PylithInt dim, PylithInt numS, PylithInt numA,
                               const PylithInt sOff[], const PylithInt sOff_x[],
                               const PylithScalar s[], const PylithScalar s_t[],
                               const PylithScalar s_x[], const PylithInt aOff[],
                               const PylithInt aOff_x[], const PylithScalar a[],
                               const PylithScalar a_t[], const PylithScalar a_x[], PylithReal t,
                               const PylithScalar x[], const PylithReal n[],
                               PylithInt numConstants, const PylithScalar constants[],
                               PylithScalar f[]);
typedef void (*PetscBdPointJacFn)(PylithInt dim, PylithInt numS, PylithInt numA,
                                  const PylithInt sOff[], const PylithInt sOff_x[],
                                  const PylithScalar s[], const PylithScalar s_t[],
                                  const PylithScalar s_x[], const PylithInt aOff[],
                                  const PylithInt aOff_x[], const PylithScalar a[],
                                  const PylithScalar a_t[], const PylithScalar a_x[],
                                  PylithReal t, PylithReal s_tshift, const PylithScalar x[],
                                  const PylithReal n[], PylithInt numConstants,
                                  const PylithScalar constants[], PylithScalar g[]);

/* Equation parts (libsrc/pylith/feassemble/Integrator.hh:26-31). */
enum { PL_LHS = 0, PL_RHS = 1, PL_LHS_LUMPED_INV = 2, PL_LHS_WEIGHTED = 3 };

/* Cell types. Node order: see pylith_b200/meshing.py. */
enum { PL_CELL_TET4 = 0, PL_CELL_HEX8 = 1, PL_CELL_HEX27 = 2 };

/* Aux subfield storage: one value set per cell (basis order 0) or per quadrature point
 * ("point" finite-element space, pylith/topology/Subfield.py:28-30). Host layouts are
 * [ncells][ncomp] and [ncells][nquad][ncomp]. */
enum { PL_AUX_PER_CELL = 0, PL_AUX_PER_QUADPT = 1, PL_AUX_PER_FAULT_NODE = 2 };

/* Output modes of the compute calls: overwrite the whole output vector with this
 * integrator's contribution, or add into it (ADD_VALUES). */
enum { PL_INSERT = 0, PL_ADD = 1 };

/* Scatter (assembly) strategies of the domain kernels. */
enum {
    PL_SCATTER_AUTO = 0,      /* library choice: cell-block gather for P1 tetrahedra, a group of
                                 lanes per cell with FP64 reductions for hexahedra */
    PL_SCATTER_ATOMIC = 1,    /* one thread per cell, FP64 atomics into the output */
    PL_SCATTER_BLOCKED = 2,   /* cell blocks staged in shared memory, per-node gather, one FP64
                                 reduction per node shared between blocks (P1 tetrahedra) */
    PL_SCATTER_DETERMINISTIC = 3 /* as BLOCKED, but a shared node's block sums are added by a second
                                    pass in block order: bit-identical results run to run, about
                                    7% slower (FP64 P1 residual and Jacobian action) */
};

typedef struct pl_context_s* pl_context;
typedef struct pl_mesh_s* pl_mesh;
typedef struct pl_integrator_s* pl_integrator;
typedef struct pl_matrix_s* pl_matrix;

/* Registration records (libsrc/pylith/feassemble/IntegratorDomain.hh:25-86,
 * IntegratorInterface.hh:31-120). Unused kernels are NULL. */
typedef struct {
    const char* subfield;
    int part;
    PetscPointFn r0;
    PetscPointFn r1;
} pl_residual_kernels;

typedef struct {
    const char* subfield_trial;
    const char* subfield_basis;
    int part;
    PetscPointJacFn j0, j1, j2, j3;
} pl_jacobian_kernels;

typedef struct {
    const char* subfield;
    PetscPointFn f;
} pl_project_kernels;

/* Interface faces (IntegratorInterface::FaceEnum): negative side, positive side, fault. */
enum { PL_FACE_NEGATIVE = 0, PL_FACE_POSITIVE = 1, PL_FACE_FAULT = 2 };

typedef struct {
    const char* subfield;
    int part;
    int face;
    PetscBdPointFn r0;
    PetscBdPointFn r1;
} pl_interface_residual_kernels;

typedef struct {
    const char* subfield_trial;
    const char* subfield_basis;
    int part;
    int face;
    PetscBdPointJacFn j0, j1, j2, j3;
} pl_interface_jacobian_kernels;

/* ---- errors, kernels ------------------------------------------------------------------ */
const char* pl_error_string(int code);
const char* pl_last_error(void);
/* Number of device kernels this library has launched in the process (all contexts). */
int64_t pl_kernel_launches(void);
/* Address of a pointwise kernel by its PyLith name, e.g.
 * "IsotropicLinearElasticity3D::f1v_infinitesimalStrain"; NULL if unknown. The addresses are
 * those of the pylith::fekernels declarations in include/pylith_b200/fekernels.hh. */
void* pl_fekernel_lookup(const char* name);
/* Registers the caller's own compiled copy of a pointwise kernel under its PyLith name, so that a
 * material or fault compiled against the reference's libsrc/pylith/fekernels/*.hh can pass the
 * same function pointers it hands to PetscWeakFormAddResidual / PetscWeakFormAddJacobian
 * (IntegratorDomain.cc:135-205, IntegratorInterface.cc:243-310) to the registration calls below.
 * The function is first run on the host on a fixed set of probe inputs and must compute what the
 * named kernel computes (relative 1e-12); the engine then runs its device implementation of that
 * name for the address. Returns PL_ERR_UNKNOWN_KERNEL for a name without a device implementation
 * or a function that computes something else, PL_ERR_INVALID_ARG for an address already
 * registered under another name. Registering the same pair again is a no-op. Thread-safe. */
int pl_fekernel_register(const char* name, const void* fn);
/* PyLith name of a known or registered kernel address; NULL if the address is unknown. */
const char* pl_fekernel_name(const void* fn);

/* ---- context -------------------------------------------------------------------------- */
int pl_context_create(int device, pl_context* out);
/* Destroy calls may come in any order: an object still referenced by a dependent one (a mesh by
 * an integrator, a context by a mesh, an integrator by a solver it was added to, a solver by a
 * batched solver) is released when its last dependent is destroyed. */
int pl_context_destroy(pl_context ctx);
/* Enqueue all work on a caller-owned cudaStream_t; NULL is CUDA's legacy default stream
 * (torch's default stream). A new context starts on its own non-blocking stream. */
int pl_context_set_stream(pl_context ctx, void* stream);
int pl_context_use_own_stream(pl_context ctx);
void* pl_context_get_stream(pl_context ctx);
int pl_context_synchronize(pl_context ctx);

/* ---- host memory ---------------------------------------------------------------------- */
/* No counterpart in the reference (PETSc keeps its Vecs in pageable host memory). Page-locked
 * host memory for the host buffers of calls that copy between host and device (the
 * pl_compute_*_host entry points, or a caller's own copies around the device entry points):
 * the CUDA driver's page-locked allocation (cudaHostAlloc, portable), made while the calling
 * thread prefers the NUMA node the host reports for the context's GPU, so that on a two-socket
 * host the device's reads do not cross the inter-socket link. Copy engines read such buffers at
 * the link's rate, where page-locked ranges of scattered small pages can cap host-to-device
 * copies far below it. The node is a preference: with no NUMA information (one-node hosts) or
 * no free memory on that node the pages land where the kernel puts them. *out is zero-filled
 * and at least 256-byte aligned; release it with pl_host_free (not cudaFreeHost). Thread-safe. */
int pl_host_alloc(pl_context ctx, size_t bytes, void** out);
int pl_host_free(void* ptr);
/* NUMA node the host reports for the context's GPU; -1 when it reports none. */
int pl_context_numa_node(pl_context ctx, int* node);

/* ---- mesh ----------------------------------------------------------------------------- */
/* Uploads cells [num_cells][nodes_per_cell] (int32) and coordinates [num_nodes][3] (FP64).
 * Replaces the mesh/closure data PETSc keeps in the DMPlex (topology/Field.cc:276-440,
 * CoordsVisitor.icc:145-157). */
int pl_mesh_create(pl_context ctx, int cell_type, int64_t num_cells, const int32_t* cells_host,
                   int64_t num_nodes, const double* coords_host, pl_mesh* out);
/* Adds cohesive cells [num_cohesive][12] (4 negative, 4 positive, 4 Lagrange nodes) and the
 * number of Lagrange nodes (fault vertices). */
int pl_mesh_set_cohesive(pl_mesh mesh, int64_t num_cohesive, const int32_t* cohesive_host,
                         int64_t num_lagrange);
int pl_mesh_destroy(pl_mesh mesh);
int64_t pl_mesh_num_dof(pl_mesh mesh);

/* ---- domain integrator (libsrc/pylith/feassemble/IntegratorDomain.cc) ------------------ */
/* Integrates over cells [cell_ids] of the mesh (NULL = all cells; a non-NULL list with
 * num_ids = 0 is an empty integrator, as for a material label that matches no cells). */
int pl_integrator_domain_create(pl_mesh mesh, int64_t num_ids, const int32_t* cell_ids_host,
                                pl_integrator* out);
/* IntegratorDomain::setKernelsResidual (IntegratorDomain.cc:135-167). */
int pl_integrator_set_kernels_residual(pl_integrator integ, const pl_residual_kernels* kernels,
                                       int num);
/* IntegratorDomain::setKernelsJacobian (IntegratorDomain.cc:172-205). */
int pl_integrator_set_kernels_jacobian(pl_integrator integ, const pl_jacobian_kernels* kernels,
                                       int num);
/* IntegratorDomain::setKernelsUpdateStateVars (IntegratorDomain.cc:221-228). */
int pl_integrator_set_kernels_update_state_vars(pl_integrator integ,
                                                const pl_project_kernels* kernels, int num);
/* Auxiliary subfields in the reference's order (the registered kernels index them from the
 * back, e.g. IsotropicLinearElasticity.hh:95-127). Names: density, body_force,
 * shear_modulus, bulk_modulus, maxwell_time, shear_modulus_ratio, viscous_strain,
 * total_strain (domain); slip (interface). Values are copied to the device. */
int pl_integrator_set_aux(pl_integrator integ, const char* name, int storage, int ncomp,
                          const double* values_host);
/* Copies an aux subfield back in the host layout of pl_integrator_set_aux. */
int pl_integrator_get_aux(pl_integrator integ, const char* name, double* values_host);
/* Integrator::_setKernelConstants (Integrator.cc:264-290). At most 8 constants (the kernels on
 * this path use 1 or 6); more return PL_ERR_UNSUPPORTED and leave the previous constants. */
int pl_integrator_set_constants(pl_integrator integ, int num, const double* constants);
int pl_integrator_set_scatter(pl_integrator integ, int scatter);
int pl_integrator_destroy(pl_integrator integ);

/* ---- interface integrator (libsrc/pylith/feassemble/IntegratorInterface.cc) ------------ */
int pl_integrator_interface_create(pl_mesh mesh, pl_integrator* out);
/* IntegratorInterface::setKernels (IntegratorInterface.cc:243-310). */
int pl_integrator_interface_set_kernels_residual(pl_integrator integ,
                                                 const pl_interface_residual_kernels* kernels,
                                                 int num);
int pl_integrator_interface_set_kernels_jacobian(pl_integrator integ,
                                                 const pl_interface_jacobian_kernels* kernels,
                                                 int num);

/* ---- compute (Integrator.hh:164-200) --------------------------------------------------- */
/* computeLHSResidual: DMPlexComputeResidualByKey (IntegratorDomain.cc:448) or
 * DMPlexComputeResidualHybridByKey (IntegratorInterface.cc:653). u_t may be NULL for
 * quasi-static problems. */
int pl_compute_lhs_residual(pl_integrator integ, double t, double dt, const double* u_dev,
                            const double* u_t_dev, double* r_dev, int mode);
/* Matrix-free Jacobian action Jv with the registered Jacobian kernels
 * (DMPlexComputeJacobianActionByKey, IntegratorDomain.cc:540). */
int pl_compute_lhs_jacobian_action(pl_integrator integ, double t, double dt, double s_tshift,
                                   const double* u_dev, const double* v_dev, double* jv_dev,
                                   int mode);
/* FP32 variant of the Jacobian action (FP32 operands, FP32 accumulation, FP64 geometry);
 * used inside the mixed-precision Krylov iterations. */
int pl_compute_lhs_jacobian_action_f32(pl_integrator integ, double t, double dt,
                                       const float* v_dev, float* jv_dev, int mode);
/* Host-buffer convenience: copies u to the device, computes the residual and copies it
 * back (the end-to-end path a CPU caller takes). */
int pl_compute_lhs_residual_host(pl_integrator integ, double t, double dt, const double* u_host,
                                 double* r_host);
/* No counterpart in the reference. The host-buffer residual above, for callers that must not
 * allocate device memory during a call (a process whose HBM is reserved up front by a pool it
 * does not own, or a latency-bound step loop where cudaMalloc would stall the device). It
 * stages u and r through one fixed 16 MiB device array built into the library (held on every
 * GPU that loads it until exit) and so accepts meshes of at most 1048576 DOFs, returning
 * PL_ERR_INVALID_ARG beyond that. Uses the thread-per-cell kernels. The first call on each
 * device looks up the array's address and should come before any stream capture; the address is
 * kept for the life of the process and not looked up again, so the entry point must not be used
 * on a device after cudaDeviceReset (or another teardown of its primary context). All calls
 * share the array: calls whose GPU work overlaps (two host threads, two streams) race on it;
 * each call waits for its stream before returning. */
int pl_compute_lhs_residual_host_noalloc(pl_integrator integ, double t, double dt,
                                         const double* u_host, double* r_host);
/* DMProjectFieldLocal with the registered update-state kernels (IntegratorDomain.cc:555-590):
 * replaces the per-quadrature-point state subfields in place. */
int pl_update_state_vars(pl_integrator integ, double t, double dt, const double* u_dev);

/* Derived (output) fields of basis order 0, the default for cauchy_stress and cauchy_strain
 * (IntegratorDomain::setKernelsDerivedField, IntegratorDomain.cc:233-240; Elasticity.cc:629-651
 * registers them). Supported project kernels: Elasticity3D::infinitesimalStrain_asVector and the
 * cauchyStress_infinitesimalStrain_asVector of the integrator's material; at most 4. */
int pl_integrator_set_kernels_derived_field(pl_integrator integ, const pl_project_kernels* kernels,
                                            int num_kernels);
/* IntegratorDomain::_computeDerivedField (IntegratorDomain.cc:596-630): every registered
 * kernel evaluated at each cell's centroid (PETSc's order-0 dual basis), written to
 * out_dev[cell][6 * k + i] (Voigt order xx, yy, zz, xy, yz, xz) for the integrator's cells in
 * order. The generalized Maxwell stress is available on P1 tetrahedra. */
int pl_compute_derived_field(pl_integrator integ, double t, double dt, const double* u_dev,
                             double* out_dev);

/* ---- assembled Jacobian (DMPlexComputeJacobianByKey, IntegratorDomain.cc:489) ---------- */
/* Block-CSR matrix with 3x3 blocks over the mesh's node graph (plus Lagrange nodes). */
int pl_matrix_create(pl_mesh mesh, pl_matrix* out);
int pl_matrix_zero(pl_matrix mat);
int pl_compute_lhs_jacobian(pl_integrator integ, double t, double dt, double s_tshift,
                            const double* u_dev, pl_matrix mat);
/* Sizes and device arrays: row_ptr [nrows+1] int32, col_idx [nnzb] int32, values
 * [nnzb][3][3] FP64 (row-major blocks). */
int pl_matrix_info(pl_matrix mat, int64_t* nrows_blocks, int64_t* nnz_blocks,
                   const int32_t** row_ptr_dev, const int32_t** col_idx_dev,
                   double** values_dev);
/* Copies the matrix to host arrays sized by pl_matrix_info (synchronises the stream). */
int pl_matrix_copy_to_host(pl_matrix mat, int32_t* row_ptr_host, int32_t* col_idx_host,
                           double* values_host);
int pl_matrix_spmv(pl_matrix mat, const double* x_dev, double* y_dev);
int pl_matrix_destroy(pl_matrix mat);

/* ---- device Krylov solver (replaces the PETSc KSP of the quasi-static step;
 *      libsrc/pylith/materials/Elasticity.cc:298-330, petsc/Options.cc:320-331) ------------ */
/* Solves A x = b with A = -(sum of the added domain integrators' Jacobians), on the DOFs whose
 * constrained flag is 0 (Dirichlet DOFs of x are returned as 0). Preconditioned conjugate
 * gradients with point-block Jacobi. PL_SOLVER_FP32_REFINED runs the iterations in FP32 (FP64
 * dot products) and reaches FP64 accuracy through FP64 residuals (pl_solver_set_reliable).
 * Meshes with cohesive cells are solved in the reduced space of the slip constraint
 * u+ = u- + d: the positive-side DOFs of fault nodes follow the negative side and the two sides'
 * equations are summed, where the Lagrange-multiplier terms of f0u_neg/f0u_pos cancel; this
 * reduced operator is SPD. Vectors span the whole local vector (nodes, then Lagrange nodes);
 * the Lagrange-multiplier entries of x are returned as 0. */
enum { PL_SOLVER_FP64 = 0, PL_SOLVER_FP32_REFINED = 1 };
typedef struct pl_solver_s* pl_solver;
int pl_solver_create(pl_mesh mesh, const uint8_t* constrained_host, pl_solver* out);
int pl_solver_add_integrator(pl_solver solver, pl_integrator integ);
int pl_solver_set_tolerances(pl_solver solver, double rtol, double atol, int max_iter);
int pl_solver_set_precision(pl_solver solver, int precision, double inner_rtol);
/* How PL_SOLVER_FP32_REFINED reaches FP64 accuracy. enable != 0 (the default, delta 0.1):
 * reliable updates, one FP32 PCG without restarts whose iterated residual is replaced by the FP64
 * true residual (the FP32 correction added to the FP64 solution) whenever it has dropped by
 * `delta`. enable == 0: iterative refinement that restarts the FP32 PCG from every new FP64
 * residual until it has dropped by inner_rtol. Either way the solve ends when the FP64 residual
 * meets the tolerances. pl_solver_get_stats reports the replacements (or refinement passes) as
 * outer iterations. */
int pl_solver_set_reliable(pl_solver solver, int enable, double delta);
/* Builds the preconditioner at (t, dt). For PL_SOLVER_FP32_REFINED on hexahedra it also evaluates
 * each integrator's isotropic tangent once per cell at (t, dt), which the FP32 Jacobian action
 * (pl_compute_lhs_jacobian_action_f32) then reads until the integrator's aux fields or constants
 * change; call it again after such a change or a new time step. */
int pl_solver_setup(pl_solver solver, double t, double dt);
int pl_solver_solve(pl_solver solver, const double* b_dev, double* x_dev);
/* The Dirichlet values into a solution vector: u[i] = values[i] at every DOF marked in the
 * constrained mask given to pl_solver_create, every other entry untouched (fault DOFs included); values is a full local vector whose
 * constrained entries hold the boundary values (ConstraintSpatialDB::setSolution,
 * feassemble/ConstraintSpatialDB.cc:116-159, DMPlexInsertBoundaryValuesEssentialBdField). */
int pl_solver_insert_constrained(pl_solver solver, const double* values_dev, double* u_dev);
/* Sets the positive side of every fault node to u+ = u- + d from the interface integrator's
 * slip and reference directions (planar faults: one normal per fault node). */
int pl_solver_apply_fault_slip(pl_solver solver, pl_integrator iface, double* u_dev);
int pl_solver_get_stats(pl_solver solver, int* iterations, int* inner_iterations,
                        int* outer_iterations, double* rel_residual);
int pl_solver_destroy(pl_solver solver);

/* ---- geometric multigrid preconditioner (the class of preconditioner the reference configures:
 *      PETSc GAMG, libsrc/pylith/materials/Elasticity.cc:298-330) ------------------------------ */
/* A hierarchy of solvers on successively coarser meshes of the same domain (each with its own
 * integrators, constraint mask and faults; all on one context), tied by prolongations from level
 * l + 1 to level l given as host CSR node matrices: prolong_row_ptr[l] has (mesh nodes of level l)
 * + 1 entries, prolong_col[l] holds level-(l+1) mesh-node indices and prolong_val[l] the weights
 * (Lagrange-multiplier nodes are eliminated by the solvers' reduced space; applied to
 * each of the 3 components; positive-side fault nodes interpolate from their own side).
 * pylith_b200/multigrid.py builds them for structured hexahedral boxes. */
typedef struct pl_multigrid_s* pl_multigrid;
int pl_multigrid_create(pl_solver fine, int num_coarse, const pl_solver* coarse,
                        const int32_t* const* prolong_row_ptr, const int32_t* const* prolong_col,
                        const double* const* prolong_val, pl_multigrid* out);
/* Smoother: Chebyshev polynomial of point-block Jacobi of `degree` on [lower_ratio b, b],
 * b = 1.1 lambda_max(D^-1 A) estimated by power iterations at the first solve after each setup.
 * A coarsest level with at most 1536 unknowns is solved exactly (the inverse of its reduced matrix,
 * assembled and inverted on the device at the first solve after each setup); a larger one takes
 * degree coarse_degree on [coarse_lower_ratio b, b]. precision
 * PL_SOLVER_FP32_REFINED runs the V-cycle in FP32 (the outer conjugate gradients stay FP64).
 * Defaults: 2, 0.1, 40, 0.01, PL_SOLVER_FP64. */
int pl_multigrid_set_smoother(pl_multigrid mg, int degree, double lower_ratio, int coarse_degree,
                              double coarse_lower_ratio, int precision);
/* Makes pl_solver_solve run flexible conjugate gradients in FP64 preconditioned by one V-cycle
 * of `mg` (NULL: back to point-block Jacobi); pl_solver_setup then sets up every level. */
int pl_solver_set_multigrid(pl_solver solver, pl_multigrid mg);
/* The cycle: pre- and post-smoothing on (1) or off (0) on every level but the coarsest (default
 * both). Without pre-smoothing the residual is restricted as it is and the V-cycle is no longer
 * symmetric, which the flexible conjugate gradients accept. */
int pl_multigrid_set_cycle(pl_multigrid mg, int pre_smooth, int post_smooth);
/* Levels and each level's lambda_max(D^-1 A) estimate (0 before the first solve, and for a
 * coarsest level solved with its dense inverse). */
int pl_multigrid_get_levels(pl_multigrid mg, int* num_levels, double* lambda_max);
/* Refused while the hierarchy is attached to its solver (pl_solver_set_multigrid(solver, NULL)
 * or pl_solver_destroy detaches it). */
int pl_multigrid_destroy(pl_multigrid mg);

/* ---- batched right-hand sides (Green's functions; replaces the one-impulse-at-a-time
 *      SNES loop of libsrc/pylith/problems/GreensFns.cc:291-337) ------------------------------ */
/* Solves A x_i = b_i for many right-hand sides with the operator, constraints, preconditioner and
 * tolerances of `base` (after pl_solver_setup). Tiles of `tile` (1, 2, 4, 8 or 16) right-hand sides
 * share every launch of an FP32 PCG (FP64 dot products, CUDA-graph replay between convergence
 * checks), brought to FP64 accuracy per right-hand side (pl_batch_solver_set_reliable). b_dev/x_dev are arrays of nrhs
 * device pointers to full local vectors. P1 tetrahedra with isotropic linear elasticity. */
typedef struct pl_batch_solver_s* pl_batch_solver;
int pl_batch_solver_create(pl_solver base, int tile, pl_batch_solver* out);
int pl_batch_solver_solve(pl_batch_solver solver, int nrhs, const double* const* b_dev,
                          double* const* x_dev);
/* Preconditioner of the FP32 tile PCG. degree 0 or 1: point-block Jacobi (the default). degree
 * 2-8: Chebyshev-Jacobi, the Chebyshev iteration of that degree for A z = r from z = 0 with the
 * point-block Jacobi inverse P (degree - 1 operator applications per PCG iteration), on the
 * interval [lower_ratio b, b] with b = 1.1 lambda_max(P A); lambda_max is estimated by eig_iters
 * power iterations at the next solve (and again after the integrators change). The reference
 * smooths the fine level of its algebraic multigrid with the same kind of iteration: PETSc GAMG
 * (-pc_type gamg, -mg_fine_ksp_max_it 5, -mg_fine_pc_type vpbjacobi with faults;
 * libsrc/pylith/materials/Elasticity.cc:310-317), whose level smoother is PETSc's Chebyshev
 * iteration with bounds 0.1 and 1.1 times an estimated largest eigenvalue. */
int pl_batch_solver_set_chebyshev(pl_batch_solver solver, int degree, double lower_ratio, int eig_iters);
/* FP64 accuracy of the FP32 tile PCG. enable != 0 (the default, delta 0.01): reliable updates, one
 * FP32 PCG per right-hand side without restarts, whose iterated residual is replaced by the FP64
 * true residual (the FP32 correction added to the FP64 solution) whenever it has dropped by
 * `delta`; the solve ends when the true residual meets the base solver's rtol. enable == 0: FP64
 * iterative refinement that restarts the FP32 PCG from every new FP64 residual until it has
 * dropped by the base solver's inner_rtol. pl_batch_solver_get_stats counts FP64 true residuals
 * after the first as outer iterations with reliable updates, refinement passes without. */
int pl_batch_solver_set_reliable(pl_batch_solver solver, int enable, double delta);
/* Preconditions the tile's FP32 PCG with one V-cycle of `mg` per iteration on all K vectors at
 * once (NULL: back to the Chebyshev or point-block Jacobi setting): the hierarchy's smoothing,
 * transfers and dense coarsest inverse, with the batched cell-block operator on every level (P1
 * tetrahedra, isotropic linear elasticity; tiles of at most 8). The hierarchy's fine level must be
 * the base solver's mesh, and its fine solver set up at the same (t, dt); the eigenvalue estimates
 * come from the hierarchy (made at the next solve if not yet). pl_multigrid_destroy is refused while
 * a batched solver uses the hierarchy. */
int pl_batch_solver_set_multigrid(pl_batch_solver solver, pl_multigrid mg);
int pl_batch_solver_get_chebyshev(pl_batch_solver solver, double* lambda_max);
int pl_batch_solver_get_stats(pl_batch_solver solver, int64_t* solves, int64_t* inner_iterations,
                              int64_t* outer_iterations, double* max_rel_residual);
int pl_batch_solver_destroy(pl_batch_solver solver);

/* ---- ragged batches: many meshes of uneven size solved together (replaces one problem per
 *      solve, libsrc/pylith/problems/GreensFns.cc:291-337 and one run per forward problem) ---- */
/* A ragged batch runs the FP32 PCG iterations (with reliable updates to FP64 accuracy) of many
 * solvers at once: per iteration one operator launch covers the cells of every active member and
 * seven vector/reduction launches cover all their vectors, with dot products, step lengths and
 * convergence kept per member, so each member follows exactly its own PCG. Members join
 * (pl_ragged_add) and leave (on convergence, or pl_ragged_remove) between iteration chunks.
 * Members: solvers of Q1 hexahedral meshes with one domain integrator (and any faults), set up
 * with PL_SOLVER_FP32_REFINED, all on the batch's context. */
typedef struct pl_ragged_s* pl_ragged;
int pl_ragged_create(pl_context ctx, int capacity, pl_ragged* out);
/* Adds a solve A x = b (b_dev, x_dev: the solver's full local vectors, device memory that must
 * stay valid while the member is in the batch). Computes the member's initial FP64 residual with
 * its own launches (synchronises the context's stream); *member is its slot. */
int pl_ragged_add(pl_ragged batch, pl_solver solver, const double* b_dev, double* x_dev, int* member);
/* Runs one chunk of PCG iterations (pl_ragged_set_chunk, default 10) on every active member as
 * one CUDA graph, then checks each member: residual replacement (FP64 true residual) when its
 * iterated residual has dropped by the solver's reliable delta, completion when the true residual
 * meets the solver's tolerances. *active_left: members still iterating. */
int pl_ragged_iterate(pl_ragged batch, int* active_left);
/* status: PL_ERR_NOT_READY while iterating, PL_OK when converged (x_dev holds the solution), an
 * error code otherwise; iterations and the final relative FP64 residual. */
int pl_ragged_member_status(pl_ragged batch, int member, int* status, int* iterations, double* rel_residual);
/* Frees a member's slot (for a later pl_ragged_add); the other members keep theirs. */
int pl_ragged_remove(pl_ragged batch, int member);
int pl_ragged_set_chunk(pl_ragged batch, int iterations);
int pl_ragged_destroy(pl_ragged batch);

/* ---- partitioned meshes: shared-node exchange (replaces DMLocalToGlobal with ADD_VALUES
 *      over the PetscSF, libsrc/pylith/topology/Field.cc:394-402, TimeDependent.cc:667) ------ */
/* Exchange plan of one partition: npeers neighbouring partitions, counts[p] nodes shared with
 * neighbour p, and nodes_host the local node indices of those lists concatenated neighbour after
 * neighbour, each list in an order both partitions agree on (e.g. by global node id). */
typedef struct pl_halo_s* pl_halo;
int pl_halo_create(pl_context ctx, int npeers, const int64_t* counts, const int32_t* nodes_host,
                   pl_halo* out);
/* Number of listed entries (the send and receive buffers hold 3 values per entry). */
int64_t pl_halo_num_entries(pl_halo halo);
/* Copies the 3 values of every listed node of r_dev, neighbour after neighbour, into send_dev
 * (one launch on the context's stream). */
int pl_halo_pack(pl_halo halo, const double* r_dev, double* send_dev);
/* Adds the neighbours' partial sums recv_dev (laid out as send_dev) into r_dev: each shared node
 * gets its neighbours' values summed in neighbour order and added once (no atomics: the same
 * result every run). After it every partition holds the global residual at all of its nodes. */
int pl_halo_unpack_add(pl_halo halo, const double* recv_dev, double* r_dev);
/* FP32 versions for the inner iterations of the mixed-precision solvers. */
int pl_halo_pack_f32(pl_halo halo, const float* r_dev, float* send_dev);
int pl_halo_unpack_add_f32(pl_halo halo, const float* recv_dev, float* r_dev);
int pl_halo_destroy(pl_halo halo);

#ifdef __cplusplus
}
#endif

#endif /* PYLITH_B200_H */
