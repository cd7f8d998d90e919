"""pl_compute_lhs_residual_host_noalloc (host-buffer residual staged through the library's
fixed device array) against pl_compute_lhs_residual_host on the same inputs, two calls in a
row per integrator, called through the C ABI. FP64 tolerance: relative L2 <= 1e-12 (the two
entry points may sum cell contributions in different orders)."""
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


def _integrators(ctx, case):
    from pylith_b200 import feassemble as FA

    if case == "tet4_bodyforce":
        mesh = M.box_tet_delaunay(6000, seed=5)
        dm = FA.DeviceMesh(ctx, mesh)
        return mesh, dm, [_elastic(mesh, 3, True).create_integrator(dm)]
    if case == "hex27":
        mesh = M.box_hex27(3, 3, 2)
        dm = FA.DeviceMesh(ctx, mesh)
        return mesh, dm, [_elastic(mesh, 4, False).create_integrator(dm)]
    if case == "hex8_genmaxwell":
        mesh = M.box_hex(6, 5, 4)
        dm = FA.DeviceMesh(ctx, mesh)
        return mesh, dm, [_genmaxwell(mesh, 6).create_integrator(dm, 1e8 * 3.15e7)]
    if case == "fault":
        mesh = M.insert_fault_x(M.box_hex(6, 4, 3))
        slip = np.random.default_rng(11).standard_normal((mesh.num_lagrange, 3))
        fault = MAT.FaultCohesiveKin(slip, ref_dir_1=(0, 0, 1), ref_dir_2=(0.5, 0, 0.5))
        dm = FA.DeviceMesh(ctx, mesh)
        return mesh, dm, [_elastic(mesh, 7, False).create_integrator(dm), fault.create_integrator(dm)]
    raise ValueError(case)


@pytest.mark.parametrize("case", ["tet4_bodyforce", "hex27", "hex8_genmaxwell", "fault"])
def test_noalloc_matches_host_entry_point_on_two_calls(ctx, case):
    from pylith_b200 import _lib

    lib = _lib.lib()
    mesh, dm, igs = _integrators(ctx, case)
    n = dm.num_dof
    rng = np.random.default_rng(["tet4_bodyforce", "hex27", "hex8_genmaxwell", "fault"].index(case))
    for call in range(2):
        for ig in igs:
            u = rng.standard_normal(n) * (1.0 + 10.0 * call)
            r_new = _call(lib.pl_compute_lhs_residual_host_noalloc, ig, 0.0, 0.0, u)
            r_ref = _call(lib.pl_compute_lhs_residual_host, ig, 0.0, 0.0, u)
            assert np.isfinite(r_new).all()
            assert np.linalg.norm(r_ref) > 0
            assert rel_l2(r_new, r_ref) <= TOL64, (case, call)


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
