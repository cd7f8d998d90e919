"""Python mirror of PyLith's integrator registration API over the C ABI.

Same names, argument meaning and error behaviour as
libsrc/pylith/feassemble/IntegratorDomain.hh:25-86 and IntegratorInterface.hh:31-120:
kernels are registered as (subfield, part, pointwise functions) records; an unknown
pointwise function raises (PL_ERR_UNKNOWN_KERNEL) instead of falling back to the CPU.
Device buffers are torch CUDA tensors (float64, or float32 for the mixed-precision action).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib as C
from ._lib import check

LHS, RHS, LHS_LUMPED_INV, LHS_WEIGHTED = C.PL_LHS, C.PL_RHS, C.PL_LHS_LUMPED_INV, C.PL_LHS_WEIGHTED
PER_CELL, PER_QUADPT, PER_FAULT_NODE = C.PL_AUX_PER_CELL, C.PL_AUX_PER_QUADPT, C.PL_AUX_PER_FAULT_NODE
INSERT, ADD = C.PL_INSERT, C.PL_ADD
SCATTER_AUTO, SCATTER_ATOMIC, SCATTER_BLOCKED, SCATTER_DETERMINISTIC = (
    C.PL_SCATTER_AUTO, C.PL_SCATTER_ATOMIC, C.PL_SCATTER_BLOCKED, C.PL_SCATTER_DETERMINISTIC)
FACE_NEGATIVE, FACE_POSITIVE, FACE_FAULT = C.PL_FACE_NEGATIVE, C.PL_FACE_POSITIVE, C.PL_FACE_FAULT


class _Kernels:
    """Addresses of the registered pointwise kernels, by PyLith class and function name."""

    def __getattr__(self, cls):
        return _KernelClass(cls)


class _KernelClass:
    def __init__(self, cls):
        self.cls = cls

    def __getattr__(self, fn):
        addr = C.lib().pl_fekernel_lookup(f"{self.cls}::{fn}".encode())
        if not addr:
            raise AttributeError(f"no pointwise kernel {self.cls}::{fn}")
        return addr


fekernels = _Kernels()


def register_fekernel(name: str, address: int) -> None:
    """Registers a caller-compiled copy of the pointwise kernel `name` (e.g.
    "IsotropicLinearElasticity3D::f1v_infinitesimalStrain") so that its address can be passed to
    the set_kernels_* calls (pl_fekernel_register)."""
    check(C.lib().pl_fekernel_register(name.encode(), address))


def fekernel_name(address: int):
    """PyLith name of a known or registered kernel address, or None."""
    n = C.lib().pl_fekernel_name(address)
    return n.decode() if n else None


def _ptr(t) -> int:
    if t is None:
        return 0
    return t.data_ptr()


@dataclass
class ResidualKernels:
    subfield: str
    part: int
    r0: Optional[int]
    r1: Optional[int]


@dataclass
class JacobianKernels:
    subfield_trial: str
    subfield_basis: str
    part: int
    j0: Optional[int]
    j1: Optional[int]
    j2: Optional[int]
    j3: Optional[int]


@dataclass
class ProjectKernels:
    subfield: str
    f: int


@dataclass
class InterfaceResidualKernels:
    subfield: str
    part: int
    face: int
    r0: Optional[int]
    r1: Optional[int] = None


@dataclass
class InterfaceJacobianKernels:
    subfield_trial: str
    subfield_basis: str
    part: int
    face: int
    j0: Optional[int]
    j1: Optional[int] = None
    j2: Optional[int] = None
    j3: Optional[int] = None


class _HostBuffer:
    """Owner of one pl_host_alloc allocation, exposed to numpy through the array interface (the
    array keeps this object alive as its base; the memory is freed with it)."""

    def __init__(self, ctx, nbytes: int, shape, dtype):
        self.ptr = ctypes.c_void_p()
        check(C.lib().pl_host_alloc(ctx.handle, nbytes, ctypes.byref(self.ptr)))
        self.__array_interface__ = {"shape": shape, "typestr": dtype.str, "data": (self.ptr.value, False),
                                    "version": 3}

    def __del__(self):
        ptr, self.ptr = getattr(self, "ptr", None), None
        if ptr:
            try:
                C.lib().pl_host_free(ptr)
            except Exception:
                pass


class Context:
    """One CUDA device and the stream all work is enqueued on (torch's current stream)."""

    def __init__(self, device: int = 0, use_torch_stream: bool = True):
        self.handle = ctypes.c_void_p()
        check(C.lib().pl_context_create(device, ctypes.byref(self.handle)))
        self.device = device
        if use_torch_stream:
            import torch

            self.set_stream(torch.cuda.current_stream(device).cuda_stream)

    def set_stream(self, stream_handle: int) -> None:
        check(C.lib().pl_context_set_stream(self.handle, stream_handle))

    def synchronize(self) -> None:
        check(C.lib().pl_context_synchronize(self.handle))

    @property
    def numa_node(self) -> int:
        """NUMA node the host reports for this context's GPU (-1: none reported)."""
        node = ctypes.c_int(-1)
        check(C.lib().pl_context_numa_node(self.handle, ctypes.byref(node)))
        return node.value

    def host_empty(self, shape, dtype=np.float64) -> np.ndarray:
        """A zero-filled numpy array in page-locked host memory on the NUMA node of this
        context's GPU (pl_host_alloc), for the host side of copies to and from the device; the
        memory is released with the last array that views it."""
        dtype = np.dtype(dtype)
        shape = (shape,) if np.isscalar(shape) else tuple(shape)
        nbytes = int(np.prod(shape, dtype=np.int64)) * dtype.itemsize
        return np.asarray(_HostBuffer(self, max(nbytes, 1), shape, dtype))

    def close(self):
        if self.handle:
            C.lib().pl_context_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceMesh:
    """A mesh resident on the device (pylith_b200.meshing.Mesh uploaded once)."""

    def __init__(self, ctx: Context, mesh):
        self.ctx = ctx
        self.mesh = mesh
        self.handle = ctypes.c_void_p()
        cells = np.ascontiguousarray(mesh.cells, dtype=np.int32)
        coords = np.ascontiguousarray(mesh.coords, dtype=np.float64)
        check(C.lib().pl_mesh_create(ctx.handle, mesh.cell_type, mesh.num_cells,
                                     cells.ctypes.data, mesh.num_nodes, coords.ctypes.data,
                                     ctypes.byref(self.handle)))
        if mesh.cohesive is not None and len(mesh.cohesive):
            coh = np.ascontiguousarray(mesh.cohesive, dtype=np.int32)
            check(C.lib().pl_mesh_set_cohesive(self.handle, len(coh), coh.ctypes.data,
                                               mesh.num_lagrange))

    @property
    def num_dof(self) -> int:
        return int(C.lib().pl_mesh_num_dof(self.handle))

    def close(self):
        if self.handle:
            C.lib().pl_mesh_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Integrator:
    def __init__(self, mesh: DeviceMesh):
        self.dmesh = mesh
        self.handle = ctypes.c_void_p()

    def set_aux(self, name: str, storage: int, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        ncomp = v.shape[-1]
        check(C.lib().pl_integrator_set_aux(self.handle, name.encode(), storage, ncomp, v.ctypes.data))

    def get_aux(self, name: str, shape) -> np.ndarray:
        out = np.zeros(shape, dtype=np.float64)
        check(C.lib().pl_integrator_get_aux(self.handle, name.encode(), out.ctypes.data))
        return out

    def set_constants(self, constants: Sequence[float]) -> None:
        c = np.ascontiguousarray(constants, dtype=np.float64)
        check(C.lib().pl_integrator_set_constants(self.handle, len(c), c.ctypes.data if len(c) else None))

    def set_scatter(self, scatter: int) -> None:
        check(C.lib().pl_integrator_set_scatter(self.handle, scatter))

    def compute_lhs_residual(self, t, dt, u, r, u_t=None, mode=INSERT) -> None:
        check(C.lib().pl_compute_lhs_residual(self.handle, t, dt, _ptr(u), _ptr(u_t), _ptr(r), mode))

    def compute_lhs_jacobian_action(self, t, dt, s_tshift, u, v, jv, mode=INSERT) -> None:
        check(C.lib().pl_compute_lhs_jacobian_action(self.handle, t, dt, s_tshift, _ptr(u), _ptr(v),
                                                     _ptr(jv), mode))

    def compute_lhs_jacobian_action_f32(self, t, dt, v, jv, mode=INSERT) -> None:
        check(C.lib().pl_compute_lhs_jacobian_action_f32(self.handle, t, dt, _ptr(v), _ptr(jv), mode))

    def compute_lhs_residual_host(self, t, dt, u: np.ndarray, r: np.ndarray) -> None:
        assert u.dtype == np.float64 and r.dtype == np.float64
        check(C.lib().pl_compute_lhs_residual_host(self.handle, t, dt, u.ctypes.data, r.ctypes.data))

    def compute_lhs_jacobian(self, t, dt, s_tshift, u, matrix: "Matrix") -> None:
        check(C.lib().pl_compute_lhs_jacobian(self.handle, t, dt, s_tshift, _ptr(u), matrix.handle))

    def close(self):
        if self.handle:
            C.lib().pl_integrator_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class IntegratorDomain(Integrator):
    """IntegratorDomain (libsrc/pylith/feassemble/IntegratorDomain.cc) over all or some cells."""

    def __init__(self, mesh: DeviceMesh, cell_ids: Optional[np.ndarray] = None):
        super().__init__(mesh)
        ids = None if cell_ids is None else np.ascontiguousarray(cell_ids, dtype=np.int32)
        check(C.lib().pl_integrator_domain_create(mesh.handle, 0 if ids is None else len(ids),
                                                  None if ids is None else ids.ctypes.data,
                                                  ctypes.byref(self.handle)))

    def set_kernels_residual(self, kernels: Sequence[ResidualKernels]) -> None:
        arr = (C.ResidualKernelsC * len(kernels))(
            *[C.ResidualKernelsC(k.subfield.encode(), k.part, k.r0, k.r1) for k in kernels])
        check(C.lib().pl_integrator_set_kernels_residual(self.handle, arr, len(kernels)))

    def set_kernels_jacobian(self, kernels: Sequence[JacobianKernels]) -> None:
        arr = (C.JacobianKernelsC * len(kernels))(
            *[C.JacobianKernelsC(k.subfield_trial.encode(), k.subfield_basis.encode(), k.part,
                                 k.j0, k.j1, k.j2, k.j3) for k in kernels])
        check(C.lib().pl_integrator_set_kernels_jacobian(self.handle, arr, len(kernels)))

    def set_kernels_update_state_vars(self, kernels: Sequence[ProjectKernels]) -> None:
        arr = (C.ProjectKernelsC * len(kernels))(
            *[C.ProjectKernelsC(k.subfield.encode(), k.f) for k in kernels])
        check(C.lib().pl_integrator_set_kernels_update_state_vars(self.handle, arr, len(kernels)))

    def update_state_vars(self, t, dt, u) -> None:
        check(C.lib().pl_update_state_vars(self.handle, t, dt, _ptr(u)))

    def set_kernels_derived_field(self, kernels: Sequence[ProjectKernels]) -> None:
        """IntegratorDomain::setKernelsDerivedField (IntegratorDomain.cc:233-240)."""
        arr = (C.ProjectKernelsC * len(kernels))(
            *[C.ProjectKernelsC(k.subfield.encode(), k.f) for k in kernels])
        check(C.lib().pl_integrator_set_kernels_derived_field(self.handle, arr, len(kernels)))
        self.derived_subfields = [k.subfield for k in kernels]

    def compute_derived_field(self, t, dt, u, out) -> None:
        """Basis-order-0 derived fields at the cell centroids into out [ncells, 6 * nkernels]
        (IntegratorDomain::_computeDerivedField, IntegratorDomain.cc:596-630)."""
        check(C.lib().pl_compute_derived_field(self.handle, t, dt, _ptr(u), _ptr(out)))


class IntegratorInterface(Integrator):
    """IntegratorInterface (libsrc/pylith/feassemble/IntegratorInterface.cc) over the mesh's
    cohesive cells."""

    def __init__(self, mesh: DeviceMesh):
        super().__init__(mesh)
        check(C.lib().pl_integrator_interface_create(mesh.handle, ctypes.byref(self.handle)))

    def set_kernels_residual(self, kernels: Sequence[InterfaceResidualKernels]) -> None:
        arr = (C.InterfaceResidualKernelsC * len(kernels))(
            *[C.InterfaceResidualKernelsC(k.subfield.encode(), k.part, k.face, k.r0, k.r1)
              for k in kernels])
        check(C.lib().pl_integrator_interface_set_kernels_residual(self.handle, arr, len(kernels)))

    def set_kernels_jacobian(self, kernels: Sequence[InterfaceJacobianKernels]) -> None:
        arr = (C.InterfaceJacobianKernelsC * len(kernels))(
            *[C.InterfaceJacobianKernelsC(k.subfield_trial.encode(), k.subfield_basis.encode(),
                                          k.part, k.face, k.j0, k.j1, k.j2, k.j3) for k in kernels])
        check(C.lib().pl_integrator_interface_set_kernels_jacobian(self.handle, arr, len(kernels)))


class Matrix:
    """Assembled Jacobian in 3x3-block CSR form on the device."""

    def __init__(self, mesh: DeviceMesh):
        self.dmesh = mesh
        self.handle = ctypes.c_void_p()
        check(C.lib().pl_matrix_create(mesh.handle, ctypes.byref(self.handle)))

    def zero(self):
        check(C.lib().pl_matrix_zero(self.handle))

    def spmv(self, x, y):
        check(C.lib().pl_matrix_spmv(self.handle, _ptr(x), _ptr(y)))

    def to_scipy(self):
        """Copy to a host scipy.sparse BSR matrix (synchronises)."""
        import scipy.sparse as sp

        nr, nb = ctypes.c_int64(), ctypes.c_int64()
        check(C.lib().pl_matrix_info(self.handle, ctypes.byref(nr), ctypes.byref(nb), None, None, None))
        nr, nb = nr.value, nb.value
        h_rp = np.zeros(nr + 1, dtype=np.int32)
        h_ci = np.zeros(nb, dtype=np.int32)
        h_val = np.zeros((nb, 3, 3), dtype=np.float64)
        check(C.lib().pl_matrix_copy_to_host(self.handle, h_rp.ctypes.data, h_ci.ctypes.data,
                                             h_val.ctypes.data))
        return sp.bsr_matrix((h_val, h_ci, h_rp), shape=(3 * nr, 3 * nr))

    def close(self):
        if self.handle:
            C.lib().pl_matrix_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Solver:
    """Device PCG for A x = b, A = -(sum of the integrators' Jacobians), on the unconstrained DOFs
    (include/pylith_b200.h, pl_solver_*)."""

    FP64 = C.PL_SOLVER_FP64
    FP32_REFINED = C.PL_SOLVER_FP32_REFINED

    def __init__(self, mesh: DeviceMesh, constrained: Optional[np.ndarray], integrators,
                 rtol=1e-12, atol=0.0, max_iter=20000, precision=C.PL_SOLVER_FP64, inner_rtol=1e-5,
                 reliable=True, reliable_delta=0.1):
        self.dmesh = mesh
        self.integrators = list(integrators)
        self.handle = ctypes.c_void_p()
        mask = None if constrained is None else np.ascontiguousarray(constrained, dtype=np.uint8)
        self._mask = mask
        check(C.lib().pl_solver_create(mesh.handle, None if mask is None else mask.ctypes.data,
                                       ctypes.byref(self.handle)))
        for ig in self.integrators:
            check(C.lib().pl_solver_add_integrator(self.handle, ig.handle))
        check(C.lib().pl_solver_set_tolerances(self.handle, rtol, atol, max_iter))
        check(C.lib().pl_solver_set_precision(self.handle, precision, inner_rtol))
        # FP32_REFINED: reliable updates (residual replacement) or restarted iterative refinement
        check(C.lib().pl_solver_set_reliable(self.handle, 1 if reliable else 0, reliable_delta))

    def setup(self, t=0.0, dt=0.0):
        check(C.lib().pl_solver_setup(self.handle, t, dt))

    def solve(self, b, x):
        check(C.lib().pl_solver_solve(self.handle, _ptr(b), _ptr(x)))

    def insert_constrained(self, values, u) -> None:
        """u[i] = values[i] at the constrained DOFs (pl_solver_insert_constrained)."""
        check(C.lib().pl_solver_insert_constrained(self.handle, _ptr(values), _ptr(u)))

    def apply_fault_slip(self, iface: "IntegratorInterface", u) -> None:
        check(C.lib().pl_solver_apply_fault_slip(self.handle, iface.handle, _ptr(u)))

    def stats(self):
        it, inner, outer, rel = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        check(C.lib().pl_solver_get_stats(self.handle, ctypes.byref(it), ctypes.byref(inner),
                                          ctypes.byref(outer), ctypes.byref(rel)))
        return {"iterations": it.value, "inner_iterations": inner.value,
                "outer_iterations": outer.value, "rel_residual": rel.value}

    def close(self):
        if self.handle:
            C.lib().pl_solver_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchSolver:
    """Many right-hand sides with the operator and preconditioner of a set-up `Solver`
    (pl_batch_solver_*): tiles of `tile` RHS share each FP32 PCG launch, FP64 residuals per RHS."""

    def __init__(self, solver: Solver, tile: int = 8):
        self.solver = solver
        self.tile = tile
        self.degree = 0
        self.reliable = True
        self.handle = ctypes.c_void_p()
        check(C.lib().pl_batch_solver_create(solver.handle, tile, ctypes.byref(self.handle)))

    def solve(self, bs, xs) -> None:
        n = len(bs)
        pb = (ctypes.c_void_p * max(n, 1))(*[_ptr(b) for b in bs])
        px = (ctypes.c_void_p * max(n, 1))(*[_ptr(x) for x in xs])
        check(C.lib().pl_batch_solver_solve(self.handle, n, pb, px))

    def set_chebyshev(self, degree: int, lower_ratio: float = 0.05, eig_iters: int = 20) -> None:
        """Preconditioner of the FP32 tile PCG: degree 0 or 1 point-block Jacobi, 2-8 Chebyshev-
        Jacobi on [lower_ratio b, b], b = 1.1 lambda_max(P A), estimated at the next solve."""
        check(C.lib().pl_batch_solver_set_chebyshev(self.handle, int(degree), float(lower_ratio), int(eig_iters)))
        self.degree = int(degree)

    def set_multigrid(self, mg: Optional["Multigrid"]) -> None:
        """One V-cycle of `mg` on all the tile's vectors per PCG iteration (None: back to
        Chebyshev or point-block Jacobi); keeps `mg` alive while set."""
        check(C.lib().pl_batch_solver_set_multigrid(self.handle, mg.handle if mg is not None else None))
        self._mg = mg

    def set_reliable(self, enable: bool = True, delta: float = 0.01) -> None:
        """FP64 accuracy of the FP32 tile PCG: reliable updates (residual replacement whenever the
        iterated residual has dropped by `delta`; the default, with delta 0.01) or restarted
        iterative refinement."""
        check(C.lib().pl_batch_solver_set_reliable(self.handle, 1 if enable else 0, float(delta)))
        self.reliable = bool(enable)

    @property
    def lambda_max(self) -> float:
        """The power-iteration estimate of lambda_max(P A) (0 before the first Chebyshev solve)."""
        v = ctypes.c_double()
        check(C.lib().pl_batch_solver_get_chebyshev(self.handle, ctypes.byref(v)))
        return v.value

    def stats(self):
        s, i, o, r = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_double()
        check(C.lib().pl_batch_solver_get_stats(self.handle, ctypes.byref(s), ctypes.byref(i), ctypes.byref(o),
                                                ctypes.byref(r)))
        return {"solves": s.value, "inner_iterations": i.value, "outer_iterations": o.value,
                "max_rel_residual": r.value}

    def close(self):
        if self.handle:
            C.lib().pl_batch_solver_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RaggedBatch:
    """Many solvers on meshes of uneven size iterated together (pl_ragged_*): every PCG iteration
    of every active member shares one operator launch and seven vector launches, with dot products
    and convergence kept per member. Members are FP32-refined Q1 hexahedral solvers."""

    def __init__(self, ctx: Context, capacity: int = 256, chunk: int = 10):
        self.ctx = ctx
        self.handle = ctypes.c_void_p()
        check(C.lib().pl_ragged_create(ctx.handle, capacity, ctypes.byref(self.handle)))
        check(C.lib().pl_ragged_set_chunk(self.handle, chunk))
        self._keep = {}

    def add(self, solver: Solver, b, x) -> int:
        """Adds the solve solver.A x = b (device vectors kept alive while the member is here)."""
        m = ctypes.c_int()
        check(C.lib().pl_ragged_add(self.handle, solver.handle, _ptr(b), _ptr(x), ctypes.byref(m)))
        self._keep[m.value] = (solver, b, x)
        return m.value

    def iterate(self) -> int:
        """One chunk of iterations for every active member; returns how many are still active."""
        left = ctypes.c_int()
        check(C.lib().pl_ragged_iterate(self.handle, ctypes.byref(left)))
        return left.value

    def status(self, member: int):
        st, it, rel = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        check(C.lib().pl_ragged_member_status(self.handle, member, ctypes.byref(st), ctypes.byref(it),
                                              ctypes.byref(rel)))
        return {"status": st.value, "done": st.value != C.ERRORS_NOT_READY, "iterations": it.value,
                "rel_residual": rel.value}

    def remove(self, member: int) -> None:
        check(C.lib().pl_ragged_remove(self.handle, member))
        self._keep.pop(member, None)

    def close(self):
        if self.handle:
            C.lib().pl_ragged_destroy(self.handle)
            self.handle = ctypes.c_void_p()
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Multigrid:
    """Geometric multigrid preconditioner of a `Solver` (pl_multigrid_*): coarse-level solvers (set
    up together with the fine one) and the prolongations between levels, as CSR node matrices
    (row_ptr, col, val) from level l + 1 to level l. Attaching it makes the fine solver run
    flexible CG preconditioned by V-cycles."""

    def __init__(self, fine: Solver, coarse, prolongations, degree=2, lower=0.1, coarse_degree=40,
                 coarse_lower=0.01, precision=C.PL_SOLVER_FP64):
        self.fine = fine
        self.coarse = list(coarse)
        self._P = [tuple(np.ascontiguousarray(a, dtype=t) for a, t in zip(P, (np.int32, np.int32, np.float64)))
                   for P in prolongations]
        n = len(self.coarse)
        solvers = (ctypes.c_void_p * n)(*[s.handle.value for s in self.coarse])
        rows = (ctypes.c_void_p * n)(*[P[0].ctypes.data for P in self._P])
        cols = (ctypes.c_void_p * n)(*[P[1].ctypes.data for P in self._P])
        vals = (ctypes.c_void_p * n)(*[P[2].ctypes.data for P in self._P])
        self.handle = ctypes.c_void_p()
        check(C.lib().pl_multigrid_create(fine.handle, n, solvers, rows, cols, vals, ctypes.byref(self.handle)))
        self.precision = precision
        self.set_smoother(degree, lower, coarse_degree, coarse_lower)
        check(C.lib().pl_solver_set_multigrid(fine.handle, self.handle))

    def set_cycle(self, pre_smooth: bool = True, post_smooth: bool = True):
        """Pre- and post-smoothing on or off (pl_multigrid_set_cycle)."""
        check(C.lib().pl_multigrid_set_cycle(self.handle, 1 if pre_smooth else 0, 1 if post_smooth else 0))
        self.pre_smooth, self.post_smooth = pre_smooth, post_smooth

    def set_smoother(self, degree, lower, coarse_degree=40, coarse_lower=0.01):
        """Chebyshev-Jacobi smoothing of `degree` on [lower b, b] (pl_multigrid_set_smoother)."""
        check(C.lib().pl_multigrid_set_smoother(self.handle, degree, lower, coarse_degree, coarse_lower, self.precision))
        self.degree, self.lower = degree, lower

    def lambda_max(self):
        n = ctypes.c_int()
        lam = (ctypes.c_double * (len(self.coarse) + 1))()
        check(C.lib().pl_multigrid_get_levels(self.handle, ctypes.byref(n), lam))
        return list(lam)[:n.value]

    def close(self):
        if self.handle:
            if self.fine.handle:
                C.lib().pl_solver_set_multigrid(self.fine.handle, None)
            C.lib().pl_multigrid_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
