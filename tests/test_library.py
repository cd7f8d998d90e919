"""CPU checks of the product library: it loads, exports every entry point the C header
declares, resolves every registered pointwise kernel by name, and the host build of the
device pointwise code matches the reference's golden vectors bit for bit."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pylith_b200.h")
GOLDEN = os.path.join(ROOT, "tests", "golden", "pointwise_golden.npz")

KERNEL_NAMES = [
    "Elasticity::g0v_bodyforce",
    "IsotropicLinearElasticity3D::f1v_infinitesimalStrain",
    "IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain",
    "IsotropicLinearGenMaxwell3D::f1v_infinitesimalStrain",
    "IsotropicLinearGenMaxwell3D::Jf3vu_infinitesimalStrain",
    "IsotropicLinearGenMaxwell3D::viscousStrain_infinitesimalStrain_asVector",
    "Elasticity3D::infinitesimalStrain_asVector",
    "IsotropicLinearElasticity3D::cauchyStress_infinitesimalStrain_asVector",
    "IsotropicLinearGenMaxwell3D::cauchyStress_infinitesimalStrain_asVector",
    "FaultCohesiveKin::f0u_neg", "FaultCohesiveKin::f0u_pos", "FaultCohesiveKin::f0l_slip",
    "FaultCohesiveKin::Jf0ul_neg", "FaultCohesiveKin::Jf0ul_pos", "FaultCohesiveKin::Jf0lu",
]


@pytest.fixture(scope="module")
def L():
    from pylith_b200 import _lib

    return _lib.lib()


def header_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|void\*|const char\*)\s+(pl_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol(L):
    names = header_functions()
    assert len(names) >= 30
    missing = [n for n in names if getattr(L, n, None) is None]
    assert not missing, missing


def test_binding_covers_header():
    from pylith_b200 import _lib

    assert set(header_functions()) <= set(_lib.SIGNATURES)


def test_kernel_lookup_by_name(L):
    for n in KERNEL_NAMES:
        assert L.pl_fekernel_lookup(n.encode()), n
    assert not L.pl_fekernel_lookup(b"IsotropicPowerLaw3D::f1v_infinitesimalStrain")


def test_error_strings(L):
    assert L.pl_error_string(-2) == b"unknown pointwise kernel"
    assert L.pl_error_string(0) == b"ok"


def test_host_free_accepts_only_its_own_buffers(L):
    """pl_host_free: NULL is a no-op, a pointer pl_host_alloc did not return is refused (the
    check runs before any CUDA call)."""
    assert L.pl_host_free(None) == 0
    buf = ctypes.create_string_buffer(64)
    assert L.pl_host_free(ctypes.addressof(buf)) == -1
    assert L.pl_host_alloc(None, 64, ctypes.byref(ctypes.c_void_p())) == -1


@pytest.mark.parametrize("name", KERNEL_NAMES)
def test_host_pointwise_matches_reference_golden(L, name):
    """The exported pylith::fekernels::* host functions run the same pointwise code the device
    kernels inline; pin it against the reference's outputs."""
    import oracle as O

    g = np.load(GOLDEN)
    key = name.replace("::", "__")
    addr = L.pl_fekernel_lookup(name.encode())
    kind = O.KERNELS[name][2]
    ftype = {"point": O.POINT_FN, "jac": O.JAC_FN, "bd": O.BD_FN, "bdj": O.BDJ_FN}[kind]
    fn = ftype(addr)
    P = ctypes.c_void_p
    for i in range(len(g[f"{key}.out"])):
        nc = int(g[f"{key}.numConstants"][i])
        s = np.ascontiguousarray(g[f"{key}.s"][i])
        s_x = np.ascontiguousarray(g[f"{key}.s_x"][i])
        a = np.ascontiguousarray(g[f"{key}.a"][i])
        aoff = np.ascontiguousarray(g[f"{key}.aOff"][i], dtype=np.int32)
        c = np.ascontiguousarray(g[f"{key}.constants"][i])
        n = np.ascontiguousarray(g[f"{key}.n"][i])
        x = np.zeros(3)
        numS = 2 if "Fault" in name else 1
        sOff = np.array([0, 6], dtype=np.int32)
        sOff_x = np.zeros(2, dtype=np.int32)
        st = np.zeros_like(s)
        out = np.zeros(81)
        common = (3, numS, len(aoff), sOff.ctypes.data_as(P), sOff_x.ctypes.data_as(P), s.ctypes.data_as(P),
                  st.ctypes.data_as(P), s_x.ctypes.data_as(P), aoff.ctypes.data_as(P), None,
                  a.ctypes.data_as(P), None, None, 0.0)
        if kind == "point":
            fn(*common, x.ctypes.data_as(P), nc, c.ctypes.data_as(P), out.ctypes.data_as(P))
        elif kind == "jac":
            fn(*common, 0.0, x.ctypes.data_as(P), nc, c.ctypes.data_as(P), out.ctypes.data_as(P))
        elif kind == "bd":
            fn(*common, x.ctypes.data_as(P), n.ctypes.data_as(P), nc, c.ctypes.data_as(P), out.ctypes.data_as(P))
        else:
            fn(*common, 0.0, x.ctypes.data_as(P), n.ctypes.data_as(P), nc, c.ctypes.data_as(P),
               out.ctypes.data_as(P))
        np.testing.assert_array_equal(out, g[f"{key}.out"][i])


def test_argument_validation_without_a_device(L):
    """Host-side checks run before any CUDA call: null handles and bad arguments return
    PL_ERR_INVALID_ARG (-1) with a message, and every error code has a name."""
    from pylith_b200 import _lib

    P = ctypes.c_void_p
    null = P(0)
    out = P()
    assert L.pl_context_create(0, None) == -1
    assert L.pl_mesh_create(null, 0, 10, None, 5, None, ctypes.byref(out)) == -1
    assert L.pl_integrator_domain_create(null, 0, None, ctypes.byref(out)) == -1
    assert L.pl_integrator_set_scatter(null, 0) == -1
    assert L.pl_integrator_set_aux(null, b"shear_modulus", 0, 1, None) == -1
    assert L.pl_integrator_set_kernels_derived_field(null, None, 0) == -1
    assert L.pl_compute_lhs_residual(null, 0.0, 0.0, None, None, None, 0) == -1
    assert L.pl_compute_lhs_jacobian_action(null, 0.0, 0.0, 0.0, None, None, None, 0) == -1
    assert L.pl_compute_lhs_residual_host(null, 0.0, 0.0, None, None) == -1
    assert L.pl_compute_lhs_residual_host_noalloc(null, 0.0, 0.0, None, None) == -1
    assert L.pl_compute_derived_field(null, 0.0, 0.0, None, None) == -1
    assert L.pl_solver_solve(null, None, None) == -1
    assert L.pl_batch_solver_create(null, 3, ctypes.byref(out)) == -1
    assert L.pl_last_error()
    for code, name in _lib.ERRORS.items():
        assert L.pl_error_string(code) not in (None, b"unknown error"), name
    assert L.pl_error_string(0) == b"ok"
    # destroying nothing is a no-op
    assert L.pl_integrator_destroy(null) == 0
    assert L.pl_matrix_destroy(null) == 0


def test_registration_accepts_the_reference_build_and_refuses_other_functions():
    """pl_fekernel_register runs a candidate on host probe inputs: the reference's kernels built
    from its sources (oracle/_ref) are accepted under their names, and a function with the right
    signature that computes something else is refused (PL_ERR_UNKNOWN_KERNEL), as is a name the
    engine has no device implementation for."""
    from pylith_b200 import _lib
    from pylith_b200 import feassemble as FA

    import oracle as O  # tests/conftest.py puts oracle/ on the path

    if O.ref_available():
        for name in O.KERNELS:
            FA.register_fekernel(name, O.kernel(name, "ref"))
            assert FA.fekernel_name(O.kernel(name, "ref")) == name
    D = ctypes.c_double
    PI = ctypes.POINTER(ctypes.c_int)
    PD = ctypes.POINTER(D)
    POINT = ctypes.CFUNCTYPE(None, ctypes.c_int, ctypes.c_int, ctypes.c_int, PI, PI, PD, PD, PD, PI, PI, PD, PD, PD,
                             D, PD, ctypes.c_int, PD, PD)

    def half_stress(dim, numS, numA, sOff, sOff_x, s, s_t, s_x, aOff, aOff_x, a, a_t, a_x, t, x, nc, c, f):
        for i in range(9):
            f[i] -= 0.5 * a[aOff[numA - 2]] * (s_x[i] + s_x[3 * (i % 3) + i // 3])

    fn = POINT(half_stress)
    addr = ctypes.cast(fn, ctypes.c_void_p).value
    with pytest.raises(_lib.PylithB200Error) as e:
        FA.register_fekernel("IsotropicLinearElasticity3D::f1v_infinitesimalStrain", addr)
    assert e.value.code == -2
    assert FA.fekernel_name(addr) is None
    with pytest.raises(_lib.PylithB200Error) as e:
        FA.register_fekernel("IsotropicLinearElasticity3D::f1v_infinitesimalStrain_refState", addr)
    assert e.value.code == -2
