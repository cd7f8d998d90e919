"""ctypes binding of the C ABI in include/pylith_b200.h (libpylith_b200.so).

The library is built in-tree (pylith_b200/libpylith_b200.so) for sm_100a. There is no
fallback: if the library is missing or cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# PYLITH_B200_LIB selects another build of the same library (e.g. a tuning variant).
LIB_PATH = os.environ.get("PYLITH_B200_LIB", os.path.join(HERE, "libpylith_b200.so"))

_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_D = ctypes.c_double

PL_OK = 0
ERRORS_NOT_READY = -8
ERRORS = {
    -1: "PL_ERR_INVALID_ARG", -2: "PL_ERR_UNKNOWN_KERNEL", -3: "PL_ERR_CUDA",
    -4: "PL_ERR_OUT_OF_MEMORY", -5: "PL_ERR_NOT_CONVERGED", -6: "PL_ERR_DEVICE_CHECK",
    -7: "PL_ERR_UNSUPPORTED", -8: "PL_ERR_NOT_READY",
}

PL_LHS, PL_RHS, PL_LHS_LUMPED_INV, PL_LHS_WEIGHTED = 0, 1, 2, 3
PL_AUX_PER_CELL, PL_AUX_PER_QUADPT, PL_AUX_PER_FAULT_NODE = 0, 1, 2
PL_INSERT, PL_ADD = 0, 1
PL_SCATTER_AUTO, PL_SCATTER_ATOMIC, PL_SCATTER_BLOCKED, PL_SCATTER_DETERMINISTIC = 0, 1, 2, 3
PL_FACE_NEGATIVE, PL_FACE_POSITIVE, PL_FACE_FAULT = 0, 1, 2


class PylithB200Error(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class ResidualKernelsC(ctypes.Structure):
    _fields_ = [("subfield", ctypes.c_char_p), ("part", _I), ("r0", _P), ("r1", _P)]


class JacobianKernelsC(ctypes.Structure):
    _fields_ = [("subfield_trial", ctypes.c_char_p), ("subfield_basis", ctypes.c_char_p),
                ("part", _I), ("j0", _P), ("j1", _P), ("j2", _P), ("j3", _P)]


class ProjectKernelsC(ctypes.Structure):
    _fields_ = [("subfield", ctypes.c_char_p), ("f", _P)]


class InterfaceResidualKernelsC(ctypes.Structure):
    _fields_ = [("subfield", ctypes.c_char_p), ("part", _I), ("face", _I), ("r0", _P), ("r1", _P)]


class InterfaceJacobianKernelsC(ctypes.Structure):
    _fields_ = [("subfield_trial", ctypes.c_char_p), ("subfield_basis", ctypes.c_char_p),
                ("part", _I), ("face", _I), ("j0", _P), ("j1", _P), ("j2", _P), ("j3", _P)]


# name -> (restype, argtypes)
SIGNATURES = {
    "pl_error_string": (ctypes.c_char_p, [_I]),
    "pl_last_error": (ctypes.c_char_p, []),
    "pl_kernel_launches": (_I64, []),
    "pl_fekernel_lookup": (_P, [ctypes.c_char_p]),
    "pl_fekernel_register": (_I, [ctypes.c_char_p, _P]),
    "pl_fekernel_name": (ctypes.c_char_p, [_P]),
    "pl_context_create": (_I, [_I, ctypes.POINTER(_P)]),
    "pl_context_destroy": (_I, [_P]),
    "pl_context_set_stream": (_I, [_P, _P]),
    "pl_context_use_own_stream": (_I, [_P]),
    "pl_context_get_stream": (_P, [_P]),
    "pl_context_synchronize": (_I, [_P]),
    "pl_host_alloc": (_I, [_P, ctypes.c_size_t, ctypes.POINTER(_P)]),
    "pl_host_free": (_I, [_P]),
    "pl_context_numa_node": (_I, [_P, ctypes.POINTER(_I)]),
    "pl_mesh_create": (_I, [_P, _I, _I64, _P, _I64, _P, ctypes.POINTER(_P)]),
    "pl_mesh_set_cohesive": (_I, [_P, _I64, _P, _I64]),
    "pl_mesh_destroy": (_I, [_P]),
    "pl_mesh_num_dof": (_I64, [_P]),
    "pl_integrator_domain_create": (_I, [_P, _I64, _P, ctypes.POINTER(_P)]),
    "pl_integrator_set_kernels_residual": (_I, [_P, ctypes.POINTER(ResidualKernelsC), _I]),
    "pl_integrator_set_kernels_jacobian": (_I, [_P, ctypes.POINTER(JacobianKernelsC), _I]),
    "pl_integrator_set_kernels_update_state_vars": (_I, [_P, ctypes.POINTER(ProjectKernelsC), _I]),
    "pl_integrator_set_aux": (_I, [_P, ctypes.c_char_p, _I, _I, _P]),
    "pl_integrator_get_aux": (_I, [_P, ctypes.c_char_p, _P]),
    "pl_integrator_set_constants": (_I, [_P, _I, _P]),
    "pl_integrator_set_scatter": (_I, [_P, _I]),
    "pl_integrator_destroy": (_I, [_P]),
    "pl_integrator_interface_create": (_I, [_P, ctypes.POINTER(_P)]),
    "pl_integrator_interface_set_kernels_residual": (
        _I, [_P, ctypes.POINTER(InterfaceResidualKernelsC), _I]),
    "pl_integrator_interface_set_kernels_jacobian": (
        _I, [_P, ctypes.POINTER(InterfaceJacobianKernelsC), _I]),
    "pl_compute_lhs_residual": (_I, [_P, _D, _D, _P, _P, _P, _I]),
    "pl_compute_lhs_jacobian_action": (_I, [_P, _D, _D, _D, _P, _P, _P, _I]),
    "pl_compute_lhs_jacobian_action_f32": (_I, [_P, _D, _D, _P, _P, _I]),
    "pl_compute_lhs_residual_host": (_I, [_P, _D, _D, _P, _P]),
    "pl_compute_lhs_residual_host_noalloc": (_I, [_P, _D, _D, _P, _P]),
    "pl_update_state_vars": (_I, [_P, _D, _D, _P]),
    "pl_integrator_set_kernels_derived_field": (_I, [_P, ctypes.POINTER(ProjectKernelsC), _I]),
    "pl_compute_derived_field": (_I, [_P, _D, _D, _P, _P]),
    "pl_matrix_create": (_I, [_P, ctypes.POINTER(_P)]),
    "pl_matrix_zero": (_I, [_P]),
    "pl_compute_lhs_jacobian": (_I, [_P, _D, _D, _D, _P, _P]),
    "pl_matrix_info": (_I, [_P, ctypes.POINTER(_I64), ctypes.POINTER(_I64), ctypes.POINTER(_P),
                            ctypes.POINTER(_P), ctypes.POINTER(_P)]),
    "pl_matrix_copy_to_host": (_I, [_P, _P, _P, _P]),
    "pl_matrix_spmv": (_I, [_P, _P, _P]),
    "pl_matrix_destroy": (_I, [_P]),
    "pl_solver_create": (_I, [_P, _P, ctypes.POINTER(_P)]),
    "pl_solver_add_integrator": (_I, [_P, _P]),
    "pl_solver_set_tolerances": (_I, [_P, _D, _D, _I]),
    "pl_solver_set_precision": (_I, [_P, _I, _D]),
    "pl_solver_set_reliable": (_I, [_P, _I, _D]),
    "pl_solver_setup": (_I, [_P, _D, _D]),
    "pl_solver_solve": (_I, [_P, _P, _P]),
    "pl_solver_get_stats": (_I, [_P, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I),
                                 ctypes.POINTER(_D)]),
    "pl_solver_insert_constrained": (_I, [_P, _P, _P]),
    "pl_solver_apply_fault_slip": (_I, [_P, _P, _P]),
    "pl_solver_destroy": (_I, [_P]),
    "pl_batch_solver_create": (_I, [_P, _I, ctypes.POINTER(_P)]),
    "pl_batch_solver_solve": (_I, [_P, _I, _P, _P]),
    "pl_batch_solver_get_stats": (_I, [_P, ctypes.POINTER(_I64), ctypes.POINTER(_I64), ctypes.POINTER(_I64),
                                       ctypes.POINTER(_D)]),
    "pl_batch_solver_destroy": (_I, [_P]),
    "pl_batch_solver_set_chebyshev": (_I, [_P, _I, _D, _I]),
    "pl_batch_solver_get_chebyshev": (_I, [_P, ctypes.POINTER(_D)]),
    "pl_batch_solver_set_reliable": (_I, [_P, _I, _D]),
    "pl_batch_solver_set_multigrid": (_I, [_P, _P]),
    "pl_multigrid_set_cycle": (_I, [_P, _I, _I]),
    "pl_multigrid_create": (_I, [_P, _I, _P, _P, _P, _P, ctypes.POINTER(_P)]),
    "pl_multigrid_set_smoother": (_I, [_P, _I, _D, _I, _D, _I]),
    "pl_solver_set_multigrid": (_I, [_P, _P]),
    "pl_multigrid_get_levels": (_I, [_P, ctypes.POINTER(_I), _P]),
    "pl_multigrid_destroy": (_I, [_P]),
    "pl_ragged_create": (_I, [_P, _I, ctypes.POINTER(_P)]),
    "pl_ragged_add": (_I, [_P, _P, _P, _P, ctypes.POINTER(_I)]),
    "pl_ragged_iterate": (_I, [_P, ctypes.POINTER(_I)]),
    "pl_ragged_member_status": (_I, [_P, _I, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_D)]),
    "pl_ragged_remove": (_I, [_P, _I]),
    "pl_ragged_set_chunk": (_I, [_P, _I]),
    "pl_ragged_destroy": (_I, [_P]),
    "pl_halo_create": (_I, [_P, _I, _P, _P, ctypes.POINTER(_P)]),
    "pl_halo_num_entries": (_I64, [_P]),
    "pl_halo_pack": (_I, [_P, _P, _P]),
    "pl_halo_unpack_add": (_I, [_P, _P, _P]),
    "pl_halo_pack_f32": (_I, [_P, _P, _P]),
    "pl_halo_unpack_add_f32": (_I, [_P, _P, _P]),
    "pl_halo_destroy": (_I, [_P]),
}
PL_SOLVER_FP64, PL_SOLVER_FP32_REFINED = 0, 1

_lib = None


def lib():
    """Load libpylith_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise PylithB200Error(-7, f"{LIB_PATH} is not built; run __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != PL_OK:
        msg = lib().pl_last_error()
        raise PylithB200Error(rc, msg.decode() if msg else "")


def exported_symbols():
    """Names of every entry point declared in include/pylith_b200.h that the library exports."""
    L = lib()
    return [n for n in SIGNATURES if getattr(L, n, None) is not None]
