"""pl_compute_lhs_residual_host_noalloc (host-buffer residual staged through the library's
fixed device array) against pl_compute_lhs_residual_host and against the oracle on the same
inputs, two calls in a row per integrator, called through the C ABI; after a first call has
loaded the library's device code, a call leaves the device's free memory unchanged. FP64
tolerance: relative L2 <= 1e-12 (the entry points and the oracle may sum cell contributions in
different orders)."""
import ctypes

import numpy as np
import pytest

from pylith_b200 import materials as MAT
from pylith_b200 import meshing as M

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
MAX_DOF = 1 << 20


def rel_l2(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def ctx():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pylith_b200 import feassemble as FA

    return FA.Context(0)


def _call(fn, ig, t, dt, u):
    from pylith_b200 import _lib

    r = np.full(u.shape, np.nan)
    _lib.check(fn(ig.handle, ctypes.c_double(t), ctypes.c_double(dt), u.ctypes.data, r.ctypes.data))
    return r


def _elastic(mesh, seed, body_force):
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=seed)
    bf = np.random.default_rng(seed + 1).standard_normal((mesh.num_cells, 3)) * 1e3 if body_force else None
    return MAT.IsotropicLinearElasticity(rho, mu, K, bf)


def _genmaxwell(mesh, seed):
    rng = np.random.default_rng(seed)
    nc, nq = mesh.num_cells, M.QUAD_POINTS[mesh.cell_type]
    rho, mu, K = MAT.lognormal_elastic(nc, seed=seed)
    tau = MAT.genmaxwell_times(rho, np.sqrt(mu / rho), [1e18, 1e19, 1e20], [0.3, 0.3, 0.3])
    ratio = np.tile([0.3, 0.3, 0.3], (nc, 1))
    return MAT.IsotropicLinearGenMaxwell(rho, mu, K, tau, ratio, rng.standard_normal((nc, nq, 18)) * 1e-5,
                                         rng.standard_normal((nc, nq, 6)) * 1e-5)


F1_ILE = "IsotropicLinearElasticity3D::f1v_infinitesimalStrain"
F1_GM = "IsotropicLinearGenMaxwell3D::f1v_infinitesimalStrain"
GM_DT = 1e8 * 3.15e7


def _oracle_elastic(O, mat):
    fields = [(mat.density[:, None], "cell")]
    if mat.body_force is not None:
        fields.append((mat.body_force, "cell"))
    return O.AuxFields(fields + [(mat.shear_modulus[:, None], "cell"), (mat.bulk_modulus[:, None], "cell")])


def _integrators(ctx, O, case):
    """(mesh, device mesh, [(integrator, oracle residual of u)])."""
    from pylith_b200 import feassemble as FA

    if case == "tet4_bodyforce":
        mesh = M.box_tet_delaunay(6000, seed=5)
        dm = FA.DeviceMesh(ctx, mesh)
        mat = _elastic(mesh, 3, True)
        aux = _oracle_elastic(O, mat)
        return mesh, dm, [(mat.create_integrator(dm),
                           lambda u: O.residual(mesh, u, aux, f0="Elasticity::g0v_bodyforce", f1=F1_ILE))]
    if case == "hex27":
        mesh = M.box_hex27(3, 3, 2)
        dm = FA.DeviceMesh(ctx, mesh)
        mat = _elastic(mesh, 4, False)
        aux = _oracle_elastic(O, mat)
        return mesh, dm, [(mat.create_integrator(dm), lambda u: O.residual(mesh, u, aux, f1=F1_ILE))]
    if case == "hex8_genmaxwell":
        mesh = M.box_hex(6, 5, 4)
        dm = FA.DeviceMesh(ctx, mesh)
        g = _genmaxwell(mesh, 6)
        aux = O.AuxFields([(g.density[:, None], "cell"), (g.shear_modulus[:, None], "cell"),
                           (g.bulk_modulus[:, None], "cell"), (g.maxwell_time, "cell"),
                           (g.shear_modulus_ratio, "cell"), (g.viscous_strain, "qp"), (g.total_strain, "qp")])
        return mesh, dm, [(g.create_integrator(dm, GM_DT),
                           lambda u: O.residual(mesh, u, aux, f1=F1_GM, constants=[GM_DT]))]
    if case == "fault":
        mesh = M.insert_fault_x(M.box_hex(6, 4, 3))
        slip = np.random.default_rng(11).standard_normal((mesh.num_lagrange, 3))
        fault = MAT.FaultCohesiveKin(slip, ref_dir_1=(0, 0, 1), ref_dir_2=(0.5, 0, 0.5))
        dm = FA.DeviceMesh(ctx, mesh)
        mat = _elastic(mesh, 7, False)
        aux = _oracle_elastic(O, mat)
        nn = 3 * mesh.num_nodes

        def domain_ref(u):
            r = np.zeros(mesh.num_dof)
            r[:nn] = O.residual(mesh, u[:nn], aux, f1=F1_ILE)
            return r

        return mesh, dm, [(mat.create_integrator(dm), domain_ref),
                          (fault.create_integrator(dm), lambda u: O.cohesive_residual(mesh, u, fault.slip,
                                                                                      fault.constants))]
    raise ValueError(case)


@pytest.mark.parametrize("case", ["tet4_bodyforce", "hex27", "hex8_genmaxwell", "fault"])
def test_noalloc_matches_host_entry_point_on_two_calls(oracle_lib, ctx, case):
    import torch

    from pylith_b200 import _lib

    lib = _lib.lib()
    mesh, dm, igs = _integrators(ctx, oracle_lib, case)
    n = dm.num_dof
    rng = np.random.default_rng(["tet4_bodyforce", "hex27", "hex8_genmaxwell", "fault"].index(case))
    for call in range(2):
        for ig, oracle_residual in igs:
            u = rng.standard_normal(n) * (1.0 + 10.0 * call)
            free0 = torch.cuda.mem_get_info()[0]
            r_new = _call(lib.pl_compute_lhs_residual_host_noalloc, ig, 0.0, 0.0, u)
            free1 = torch.cuda.mem_get_info()[0]
            r_ref = _call(lib.pl_compute_lhs_residual_host, ig, 0.0, 0.0, u)
            r_orc = oracle_residual(u)
            assert np.isfinite(r_new).all()
            assert np.linalg.norm(r_ref) > 0
            assert rel_l2(r_new, r_ref) <= TOL64, (case, call)
            assert rel_l2(r_new, r_orc) <= TOL64, (case, call)
            if call == 1:  # the device code was loaded by the first call
                assert free1 == free0, (case, free0 - free1)


def test_noalloc_rejects_meshes_beyond_its_array(ctx):
    from pylith_b200 import _lib
    from pylith_b200 import feassemble as FA

    mesh = M.box_hex(70, 70, 70)  # 71^3 nodes = 1,073,733 DOFs > 2^20
    assert 3 * mesh.num_nodes > MAX_DOF
    ig = _elastic(mesh, 8, False).create_integrator(FA.DeviceMesh(ctx, mesh))
    u = np.zeros(3 * mesh.num_nodes)
    with pytest.raises(_lib.PylithB200Error) as e:
        _call(_lib.lib().pl_compute_lhs_residual_host_noalloc, ig, 0.0, 0.0, u)
    assert e.value.code == -1
    assert "1048576" in str(e.value)
    # a mesh that fits still works after the rejection
    small = M.box_hex(4, 4, 4)
    ig2 = _elastic(small, 9, False).create_integrator(FA.DeviceMesh(ctx, small))
    u2 = np.random.default_rng(10).standard_normal(3 * small.num_nodes)
    r_new = _call(_lib.lib().pl_compute_lhs_residual_host_noalloc, ig2, 0.0, 0.0, u2)
    r_ref = _call(_lib.lib().pl_compute_lhs_residual_host, ig2, 0.0, 0.0, u2)
    assert rel_l2(r_new, r_ref) <= TOL64
