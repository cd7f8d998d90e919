"""ORACLE — test infrastructure only.

Python bindings for the oracle (oracle/cellloop.cc: a CPU restatement of
PETSc's finite-element cell loop around PyLith's pointwise kernels) and for the
reference's own pointwise kernels built from the PyLith sources
(oracle/_ref/libref_fekernels.so, when present).

Only tests/, bench.py's CPU-baseline leg and __graft_entry__.smoke() import
this module; the product library (pylith_b200) never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libref_fekernels.so")

_I = ctypes.c_int
_I64 = ctypes.c_int64
_D = ctypes.c_double
_P = ctypes.c_void_p

POINT_FN = ctypes.CFUNCTYPE(None, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _D, _P, _I, _P, _P)
JAC_FN = ctypes.CFUNCTYPE(None, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _D, _D, _P, _I, _P, _P)
BD_FN = ctypes.CFUNCTYPE(None, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _D, _P, _P, _I, _P, _P)
BDJ_FN = ctypes.CFUNCTYPE(None, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _D, _D, _P, _P, _I, _P, _P)

_lib = None
_ref = None


def source_tree():
    """The PyLith source tree named by the PYLITH_SRC environment variable, or None when it is
    unset or holds no libsrc/ (tests that read the tree skip then)."""
    src = os.environ.get("PYLITH_SRC")
    return src if src and os.path.isdir(os.path.join(src, "libsrc")) else None


def build(ref: bool = True) -> None:
    """Compile the oracle, and the reference kernels when PYLITH_SRC names the PyLith sources
    (an existing oracle/_ref build is kept otherwise)."""
    subprocess.check_call(["make", "-s", "-C", HERE], stdout=subprocess.DEVNULL)
    src = source_tree()
    if ref and src:
        subprocess.check_call(["make", "-s", "-C", HERE, "ref", f"PYLITH_SRC={src}"], stdout=subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build(ref=False)
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.oracle_residual.restype = _I64
        _lib.oracle_jacobian_elements.restype = _I64
        _lib.oracle_jacobian_action.restype = _I64
        _lib.oracle_project_qp.restype = _I64
        _lib.oracle_project_centroid.restype = _I64
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def ref():
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(REF_PATH)
    return _ref


# Names of the pointwise kernels: restatement symbol in liboracle.so, reference symbol in
# libref_fekernels.so, and the kind of function pointer.
KERNELS = {
    "Elasticity::g0v_bodyforce": ("oracle_g0v_bodyforce", "ref_Elasticity_g0v_bodyforce", "point"),
    "IsotropicLinearElasticity3D::f1v_infinitesimalStrain": (
        "oracle_ile3d_f1v", "ref_IsotropicLinearElasticity3D_f1v_infinitesimalStrain", "point"),
    "IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain": (
        "oracle_ile3d_Jf3vu", "ref_IsotropicLinearElasticity3D_Jf3vu_infinitesimalStrain", "jac"),
    "IsotropicLinearGenMaxwell3D::f1v_infinitesimalStrain": (
        "oracle_gm3d_f1v", "ref_IsotropicLinearGenMaxwell3D_f1v_infinitesimalStrain", "point"),
    "IsotropicLinearGenMaxwell3D::Jf3vu_infinitesimalStrain": (
        "oracle_gm3d_Jf3vu", "ref_IsotropicLinearGenMaxwell3D_Jf3vu_infinitesimalStrain", "jac"),
    "IsotropicLinearGenMaxwell3D::viscousStrain_infinitesimalStrain_asVector": (
        "oracle_gm3d_viscous_strain",
        "ref_IsotropicLinearGenMaxwell3D_viscousStrain_infinitesimalStrain_asVector", "point"),
    "Elasticity3D::infinitesimalStrain_asVector": (
        "oracle_el3d_strain_vector", "ref_Elasticity3D_infinitesimalStrain_asVector", "point"),
    "IsotropicLinearElasticity3D::cauchyStress_infinitesimalStrain_asVector": (
        "oracle_ile3d_stress_vector", "ref_IsotropicLinearElasticity3D_cauchyStress_infinitesimalStrain_asVector",
        "point"),
    "IsotropicLinearGenMaxwell3D::cauchyStress_infinitesimalStrain_asVector": (
        "oracle_gm3d_stress_vector", "ref_IsotropicLinearGenMaxwell3D_cauchyStress_infinitesimalStrain_asVector",
        "point"),
    "FaultCohesiveKin::f0u_neg": ("oracle_fck_f0u_neg", "ref_FaultCohesiveKin_f0u_neg", "bd"),
    "FaultCohesiveKin::f0u_pos": ("oracle_fck_f0u_pos", "ref_FaultCohesiveKin_f0u_pos", "bd"),
    "FaultCohesiveKin::f0l_slip": ("oracle_fck_f0l_slip", "ref_FaultCohesiveKin_f0l_slip", "bd"),
    "FaultCohesiveKin::Jf0ul_neg": ("oracle_fck_Jf0ul_neg", "ref_FaultCohesiveKin_Jf0ul_neg", "bdj"),
    "FaultCohesiveKin::Jf0ul_pos": ("oracle_fck_Jf0ul_pos", "ref_FaultCohesiveKin_Jf0ul_pos", "bdj"),
    "FaultCohesiveKin::Jf0lu": ("oracle_fck_Jf0lu", "ref_FaultCohesiveKin_Jf0lu", "bdj"),
}


def kernel(name: str, source: str = "oracle"):
    """Address of a pointwise kernel: the restatement ('oracle') or the reference ('ref')."""
    sym_o, sym_r, _ = KERNELS[name]
    L = lib() if source == "oracle" else ref()
    return ctypes.cast(getattr(L, sym_o if source == "oracle" else sym_r), _P).value


def _p(a):
    return None if a is None else a.ctypes.data_as(_P)


class AuxFields:
    """Aux subfields in reference order: list of (values, kind) with kind 'cell', 'qp' or 'node'."""

    KIND = {"cell": 0, "qp": 1, "node": 2}

    def __init__(self, fields):
        self.arrays = [np.ascontiguousarray(v, dtype=np.float64) for v, _ in fields]
        self.kinds = np.array([self.KIND[k] for _, k in fields], dtype=np.int32)
        self.ncomp = np.array([a.shape[-1] for a in self.arrays], dtype=np.int32)
        self.ptrs = (_P * max(len(self.arrays), 1))(*[a.ctypes.data for a in self.arrays])

    @property
    def num(self):
        return len(self.arrays)


def residual(mesh, u, aux: AuxFields, f0=None, f1=None, t=0.0, constants=None, u_t=None,
             nthreads=0, source="oracle"):
    """Local residual (ADD into zeros) of a domain integrator over all cells of `mesh`."""
    L = lib()
    cells = np.ascontiguousarray(mesh.cells, dtype=np.int32)
    coords = np.ascontiguousarray(mesh.coords, dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.float64)
    r = np.zeros(mesh.num_nodes * 3)
    c = np.ascontiguousarray(constants if constants is not None else [0.0], dtype=np.float64)
    nc = 0 if constants is None else len(constants)
    fp0 = kernel(f0, source) if f0 else None
    fp1 = kernel(f1, source) if f1 else None
    ut = None if u_t is None else np.ascontiguousarray(u_t, dtype=np.float64)
    bad = L.oracle_residual(_I(mesh.cell_type), _I64(mesh.num_cells), _p(cells), _p(coords),
                            _I64(mesh.num_nodes), _p(u), _p(ut), _I(aux.num), _p(aux.kinds),
                            _p(aux.ncomp), aux.ptrs, _D(t), _I(nc), _p(c), _P(fp0), _P(fp1),
                            _p(r), _I(nthreads))
    if bad:
        raise ValueError(f"non-positive Jacobian determinant in cell {-bad - 1}")
    return r


def jacobian_action(mesh, v, aux: AuxFields, g3, g0=None, u=None, t=0.0, s_tshift=0.0,
                    constants=None, nthreads=0, source="oracle"):
    """Matrix-free Jacobian action J v (ADD into zeros) over all cells of `mesh`
    (DMPlexComputeJacobianActionByKey, IntegratorDomain.cc:540), the pointwise Jacobians
    evaluated at u (zero when None)."""
    L = lib()
    cells = np.ascontiguousarray(mesh.cells, dtype=np.int32)
    coords = np.ascontiguousarray(mesh.coords, dtype=np.float64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    uu = None if u is None else np.ascontiguousarray(u, dtype=np.float64)
    jv = np.zeros(mesh.num_nodes * 3)
    c = np.ascontiguousarray(constants if constants is not None else [0.0], dtype=np.float64)
    nc = 0 if constants is None else len(constants)
    ptr = lambda n: _P(kernel(n, source) if n else None)  # noqa: E731
    bad = L.oracle_jacobian_action(_I(mesh.cell_type), _I64(mesh.num_cells), _p(cells), _p(coords),
                                   _I64(mesh.num_nodes), _p(uu), _p(v), _I(aux.num), _p(aux.kinds),
                                   _p(aux.ncomp), aux.ptrs, _D(t), _D(s_tshift), _I(nc), _p(c),
                                   ptr(g0), _P(None), _P(None), ptr(g3), _p(jv), _I(nthreads))
    if bad:
        raise ValueError(f"non-positive Jacobian determinant in cell {-bad - 1}")
    return jv


def jacobian_elements(mesh, aux: AuxFields, g3, g0=None, u=None, t=0.0, s_tshift=0.0,
                      constants=None, nthreads=0, source="oracle"):
    L = lib()
    nen = mesh.cells.shape[1]
    Ke = np.zeros((mesh.num_cells, nen * 3, nen * 3))
    cells = np.ascontiguousarray(mesh.cells, dtype=np.int32)
    coords = np.ascontiguousarray(mesh.coords, dtype=np.float64)
    c = np.ascontiguousarray(constants if constants is not None else [0.0], dtype=np.float64)
    nc = 0 if constants is None else len(constants)
    uu = None if u is None else np.ascontiguousarray(u, dtype=np.float64)
    ptr = lambda n: _P(kernel(n, source) if n else None)  # noqa: E731
    bad = L.oracle_jacobian_elements(_I(mesh.cell_type), _I64(mesh.num_cells), _p(cells), _p(coords),
                                     _p(uu), _I(aux.num), _p(aux.kinds), _p(aux.ncomp), aux.ptrs,
                                     _D(t), _D(s_tshift), _I(nc), _p(c), ptr(g0), None, None,
                                     ptr(g3), _p(Ke), _I(nthreads))
    if bad:
        raise ValueError(f"non-positive Jacobian determinant in cell {-bad - 1}")
    return Ke


def assemble(mesh, Ke, ndof=None):
    """Assemble element matrices into a scipy CSR matrix over nodal DOFs (3 per node)."""
    import scipy.sparse as sp

    nen = mesh.cells.shape[1]
    dofs = (3 * mesh.cells[:, :, None].astype(np.int64) + np.arange(3)[None, None, :]).reshape(
        mesh.num_cells, nen * 3)
    rows = np.repeat(dofs[:, :, None], nen * 3, axis=2).ravel()
    cols = np.repeat(dofs[:, None, :], nen * 3, axis=1).ravel()
    n = ndof if ndof is not None else mesh.num_nodes * 3
    return sp.coo_matrix((Ke.ravel(), (rows, cols)), shape=(n, n)).tocsr()


def project_qp(mesh, u, aux: AuxFields, fns, out_ncomp, t=0.0, constants=None, nthreads=0,
               source="oracle"):
    L = lib()
    nq = L.oracle_num_quadrature_points(_I(mesh.cell_type))
    outs = [np.zeros((mesh.num_cells, nq, n)) for n in out_ncomp]
    cells = np.ascontiguousarray(mesh.cells, dtype=np.int32)
    coords = np.ascontiguousarray(mesh.coords, dtype=np.float64)
    c = np.ascontiguousarray(constants if constants is not None else [0.0], dtype=np.float64)
    nc = 0 if constants is None else len(constants)
    fptrs = (_P * len(fns))(*[kernel(f, source) for f in fns])
    optrs = (_P * len(outs))(*[o.ctypes.data for o in outs])
    oc = np.array(out_ncomp, dtype=np.int32)
    bad = L.oracle_project_qp(_I(mesh.cell_type), _I64(mesh.num_cells), _p(cells), _p(coords),
                              _p(np.ascontiguousarray(u, dtype=np.float64)), _I(aux.num),
                              _p(aux.kinds), _p(aux.ncomp), aux.ptrs, _D(t), _I(nc), _p(c),
                              _I(len(fns)), fptrs, _p(oc), optrs, _I(nthreads))
    if bad:
        raise ValueError(f"non-positive Jacobian determinant in cell {-bad - 1}")
    return outs


def project_centroid(mesh, u, aux: AuxFields, fns, out_ncomp, t=0.0, constants=None, nthreads=0,
                     source="oracle"):
    """Derived fields of basis order 0: each kernel at every cell centroid -> [ncells][ncomp]."""
    L = lib()
    outs = [np.zeros((mesh.num_cells, n)) for n in out_ncomp]
    cells = np.ascontiguousarray(mesh.cells, dtype=np.int32)
    coords = np.ascontiguousarray(mesh.coords, dtype=np.float64)
    c = np.ascontiguousarray(constants if constants is not None else [0.0], dtype=np.float64)
    nc = 0 if constants is None else len(constants)
    fptrs = (_P * len(fns))(*[kernel(f, source) for f in fns])
    optrs = (_P * len(outs))(*[o.ctypes.data for o in outs])
    oc = np.array(out_ncomp, dtype=np.int32)
    bad = L.oracle_project_centroid(_I(mesh.cell_type), _I64(mesh.num_cells), _p(cells), _p(coords),
                                    _p(np.ascontiguousarray(u, dtype=np.float64)), _I(aux.num),
                                    _p(aux.kinds), _p(aux.ncomp), aux.ptrs, _D(t), _I(nc), _p(c),
                                    _I(len(fns)), fptrs, _p(oc), optrs, _I(nthreads))
    if bad:
        raise ValueError(f"non-positive Jacobian determinant in cell {-bad - 1}")
    return outs


def cohesive_residual(mesh, u, slip, constants, t=0.0, source="oracle", r=None):
    """Add the cohesive-cell residual (f0u_neg, f0u_pos, f0l_slip) into r (full local vector)."""
    L = lib()
    lag_offset = 3 * mesh.num_nodes
    if r is None:
        r = np.zeros(mesh.num_dof)
    coh = np.ascontiguousarray(mesh.cohesive, dtype=np.int32)
    c = np.ascontiguousarray(constants, dtype=np.float64)
    L.oracle_cohesive_residual(
        _I64(len(coh)), _p(coh), _p(np.ascontiguousarray(mesh.coords)),
        _p(np.ascontiguousarray(u, dtype=np.float64)), _I64(lag_offset),
        _p(np.ascontiguousarray(slip, dtype=np.float64)), _D(t), _I(len(c)), _p(c),
        _P(kernel("FaultCohesiveKin::f0u_neg", source)), _P(kernel("FaultCohesiveKin::f0u_pos", source)),
        _P(kernel("FaultCohesiveKin::f0l_slip", source)), _p(r))
    return r


def cohesive_jacobian(mesh, constants, t=0.0, source="oracle"):
    """Assembled cohesive-cell Jacobian (scipy CSR over the full local vector)."""
    import scipy.sparse as sp

    L = lib()
    coh = np.ascontiguousarray(mesh.cohesive, dtype=np.int32)
    Ke = np.zeros((len(coh), 36, 36))
    c = np.ascontiguousarray(constants, dtype=np.float64)
    L.oracle_cohesive_jacobian_elements(
        _I64(len(coh)), _p(coh), _p(np.ascontiguousarray(mesh.coords)), _D(t), _D(0.0), _I(len(c)),
        _p(c), _P(kernel("FaultCohesiveKin::Jf0ul_neg", source)),
        _P(kernel("FaultCohesiveKin::Jf0ul_pos", source)), _P(kernel("FaultCohesiveKin::Jf0lu", source)),
        _p(Ke))
    lag_offset = 3 * mesh.num_nodes
    nodes = np.concatenate([3 * coh[:, :8].astype(np.int64),
                            lag_offset + 3 * coh[:, 8:].astype(np.int64)], axis=1)
    dofs = (nodes[:, :, None] + np.arange(3)[None, None, :]).reshape(len(coh), 36)
    rows = np.repeat(dofs[:, :, None], 36, axis=2).ravel()
    cols = np.repeat(dofs[:, None, :], 36, axis=1).ravel()
    n = mesh.num_dof
    return sp.coo_matrix((Ke.ravel(), (rows, cols)), shape=(n, n)).tocsr()


def csr_spmv(A, x, nthreads=0):
    L = lib()
    indptr = np.ascontiguousarray(A.indptr, dtype=np.int64)
    indices = np.ascontiguousarray(A.indices, dtype=np.int32)
    data = np.ascontiguousarray(A.data, dtype=np.float64)
    y = np.zeros(A.shape[0])
    L.oracle_csr_spmv(_I64(A.shape[0]), _p(indptr), _p(indices), _p(data),
                      _p(np.ascontiguousarray(x, dtype=np.float64)), _p(y), _I(nthreads))
    return y


def call_point(name, s, s_x, a, aOff, constants, source="oracle", t=0.0, x=None, n=None,
               s_tshift=0.0, numS=1, sOff=None, out_size=None):
    """Call one pointwise kernel directly (restatement or reference) and return its output."""
    _, _, kind = KERNELS[name]
    addr = kernel(name, source)
    s = np.ascontiguousarray(s, dtype=np.float64)
    s_x = np.ascontiguousarray(s_x, dtype=np.float64)
    a = np.ascontiguousarray(a, dtype=np.float64)
    aOff = np.ascontiguousarray(aOff, dtype=np.int32)
    sOff = np.ascontiguousarray(sOff if sOff is not None else [0, 6], dtype=np.int32)
    sOff_x = np.zeros(len(sOff), dtype=np.int32)
    c = np.ascontiguousarray(constants if constants is not None else [0.0], dtype=np.float64)
    nc = 0 if constants is None else len(constants)
    x = np.ascontiguousarray(x if x is not None else [0.0, 0.0, 0.0], dtype=np.float64)
    out = np.zeros(out_size or 81)
    st = np.zeros_like(s)
    args_common = (3, numS, len(aOff), _p(sOff), _p(sOff_x), _p(s), _p(st), _p(s_x), _p(aOff), None,
                   _p(a), None, None, t)
    if kind == "point":
        POINT_FN(addr)(*args_common, _p(x), nc, _p(c), _p(out))
    elif kind == "jac":
        JAC_FN(addr)(*args_common, s_tshift, _p(x), nc, _p(c), _p(out))
    elif kind == "bd":
        nn = np.ascontiguousarray(n, dtype=np.float64)
        BD_FN(addr)(*args_common, _p(x), _p(nn), nc, _p(c), _p(out))
    else:
        nn = np.ascontiguousarray(n, dtype=np.float64)
        BDJ_FN(addr)(*args_common, s_tshift, _p(x), _p(nn), nc, _p(c), _p(out))
    return out
