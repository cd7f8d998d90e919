"""GPU parity at the benchmarked sizes and on the reference's own meshes, through the C ABI
against the oracle (relative L2 <= 1e-12 for FP64):
  * the benchmark's 1.2 M-cell Delaunay P1 mesh (seed 0, every cell block the planner makes):
    residual and Jacobian action, with the default and the deterministic cell-block scatter;
  * a 32^3 Q2 hexahedral box (the sum-factorised kernel): residual and Jacobian action;
  * one time step of the 96x96x72 generalized-Maxwell box with a fault at x = 0: domain residual,
    cohesive residual, Jacobian action and the quadrature-point state update;
  * the reference's test meshes (tests/golden/reference_meshes.npz): the UniformStrain3D MMS
    residual (zero off the `boundary` group) and the axialdisp.cfg solve (the analytic answer);
  * a fault whose normal is oblique (the mesh rotated), so that the device copy of
    BoundaryDirections::tangential_directions meets its refDir2[1] term (BoundaryDirections.hh:62).
"""
import os
import sys

import numpy as np
import pytest

import known_answers as KA
from golden import make_mesh_golden as MG
from pylith_b200 import materials as MAT
from pylith_b200 import meshing as M

pytestmark = pytest.mark.gpu

F1_ILE = "IsotropicLinearElasticity3D::f1v_infinitesimalStrain"
JF3_ILE = "IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain"
F1_GM = "IsotropicLinearGenMaxwell3D::f1v_infinitesimalStrain"
JF3_GM = "IsotropicLinearGenMaxwell3D::Jf3vu_infinitesimalStrain"
TOL64 = 1e-12


def rel_l2(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module")
def ctx(torch_cuda):
    from pylith_b200 import feassemble as FA

    return FA.Context(0)


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def elastic_aux(O, rho, mu, K):
    return O.AuxFields([(rho[:, None], "cell"), (mu[:, None], "cell"), (K[:, None], "cell")])


@pytest.fixture(scope="module")
def bench_problem(torch_cuda, ctx):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    mesh = bench.load_mesh(bench.TARGET_CELLS, 0)
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=0)
    return mesh, rho, mu, K


@pytest.mark.parametrize("scatter", [0, 3], ids=["default", "deterministic"])
def test_bench_mesh_residual_and_jacobian_action_match_oracle(oracle_lib, torch_cuda, ctx, bench_problem, scatter):
    from pylith_b200 import feassemble as FA

    O, torch = oracle_lib, torch_cuda
    mesh, rho, mu, K = bench_problem
    assert mesh.num_cells > 1_200_000 and (mesh.num_cells + 255) // 256 >= 4761
    rng = np.random.default_rng(101)
    u = rng.standard_normal(mesh.num_dof)
    v = rng.standard_normal(mesh.num_dof)
    aux = elastic_aux(O, rho, mu, K)
    r_ref = O.residual(mesh, u, aux, f1=F1_ILE)
    jv_ref = O.jacobian_action(mesh, v, aux, g3=JF3_ILE)
    ig = MAT.IsotropicLinearElasticity(rho, mu, K).create_integrator(FA.DeviceMesh(ctx, mesh))
    ig.set_scatter(scatter)
    du, dv = dev(torch, u), dev(torch, v)
    dr, djv = torch.full_like(du, np.nan), torch.full_like(du, np.nan)
    ig.compute_lhs_residual(0.0, 0.0, du, dr)
    ig.compute_lhs_jacobian_action(0.0, 0.0, 0.0, du, dv, djv)
    ctx.synchronize()
    assert rel_l2(dr.cpu().numpy(), r_ref) <= TOL64
    assert rel_l2(djv.cpu().numpy(), jv_ref) <= TOL64


def test_q2_box_32cubed_matches_oracle(oracle_lib, torch_cuda, ctx):
    from pylith_b200 import feassemble as FA

    O, torch = oracle_lib, torch_cuda
    mesh = M.box_hex27(32, 32, 32)
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=0)
    rng = np.random.default_rng(102)
    u = rng.standard_normal(mesh.num_dof)
    v = rng.standard_normal(mesh.num_dof)
    aux = elastic_aux(O, rho, mu, K)
    r_ref = O.residual(mesh, u, aux, f1=F1_ILE)
    jv_ref = O.jacobian_action(mesh, v, aux, g3=JF3_ILE)
    ig = MAT.IsotropicLinearElasticity(rho, mu, K).create_integrator(FA.DeviceMesh(ctx, mesh))
    du, dv = dev(torch, u), dev(torch, v)
    dr, djv = torch.full_like(du, np.nan), torch.full_like(du, np.nan)
    ig.compute_lhs_residual(0.0, 0.0, du, dr)
    ig.compute_lhs_jacobian_action(0.0, 0.0, 0.0, du, dv, djv)
    ctx.synchronize()
    assert rel_l2(dr.cpu().numpy(), r_ref) <= TOL64
    assert rel_l2(djv.cpu().numpy(), jv_ref) <= TOL64


def test_genmaxwell_fault_box_time_step_matches_oracle(oracle_lib, torch_cuda, ctx):
    """96x96x72 Q1 hexahedra, generalized Maxwell with non-zero state, fault at x = 0."""
    from pylith_b200 import feassemble as FA

    O, torch = oracle_lib, torch_cuda
    mesh = M.insert_fault_x(M.box_hex(96, 96, 72))
    nc, nq = mesh.num_cells, 8
    rng = np.random.default_rng(103)
    rho, mu, K = MAT.lognormal_elastic(nc, seed=0)
    tau = MAT.genmaxwell_times(rho, np.sqrt(mu / rho), [1e18, 1e19, 1e20], [0.3, 0.3, 0.3])
    ratio = np.tile([0.3, 0.3, 0.3], (nc, 1))
    visc = rng.standard_normal((nc, nq, 18)) * 1e-5
    total = rng.standard_normal((nc, nq, 6)) * 1e-5
    g = MAT.IsotropicLinearGenMaxwell(rho, mu, K, tau, ratio, visc, total)
    fault = MAT.FaultCohesiveKin(rng.standard_normal((mesh.num_lagrange, 3)), ref_dir_1=(0, 0, 1),
                                 ref_dir_2=(0.5, 0, 0.5))
    dt = MAT.YEAR
    aux = O.AuxFields([(rho[:, None], "cell"), (mu[:, None], "cell"), (K[:, None], "cell"), (tau, "cell"),
                       (ratio, "cell"), (visc, "qp"), (total, "qp")])
    nn = 3 * mesh.num_nodes
    u = rng.standard_normal(mesh.num_dof) * 1e-2
    v = rng.standard_normal(mesh.num_dof)
    r_ref = np.zeros(mesh.num_dof)
    r_ref[:nn] = O.residual(mesh, u[:nn], aux, f1=F1_GM, constants=[dt])
    O.cohesive_residual(mesh, u, fault.slip, fault.constants, r=r_ref)
    jv_ref = O.jacobian_action(mesh, v[:nn], aux, g3=JF3_GM, constants=[dt])
    visc_ref, total_ref = O.project_qp(
        mesh, u[:nn], aux, ["IsotropicLinearGenMaxwell3D::viscousStrain_infinitesimalStrain_asVector",
                            "Elasticity3D::infinitesimalStrain_asVector"], [18, 6], constants=[dt])
    dm = FA.DeviceMesh(ctx, mesh)
    ig = g.create_integrator(dm, dt)
    ifc = fault.create_integrator(dm)
    du, dv = dev(torch, u), dev(torch, v)
    dr, djv = torch.full_like(du, np.nan), torch.full_like(du, np.nan)
    ig.compute_lhs_residual(0.0, dt, du, dr)
    ifc.compute_lhs_residual(0.0, dt, du, dr, mode=FA.ADD)
    ig.compute_lhs_jacobian_action(0.0, dt, 0.0, du, dv, djv)
    ctx.synchronize()
    assert rel_l2(dr.cpu().numpy(), r_ref) <= TOL64
    assert rel_l2(djv.cpu().numpy()[:nn], jv_ref) <= TOL64
    ig.update_state_vars(0.0, dt, du)
    ctx.synchronize()
    assert rel_l2(ig.get_aux("viscous_strain", (nc, nq, 18)), visc_ref) <= TOL64
    assert rel_l2(ig.get_aux("total_strain", (nc, nq, 6)), total_ref) <= TOL64


@pytest.fixture(scope="module")
def ref_meshes():
    return MG.load()


@pytest.mark.parametrize("key", ["mms_tet", "mms_hex"])
def test_reference_mms_meshes_on_gpu(oracle_lib, torch_cuda, ctx, ref_meshes, key):
    """UniformStrain3D (tests/mmstests/linearelasticity/nofaults-3d): the GPU residual of a linear
    displacement field vanishes off the `boundary` group and equals the oracle's."""
    from pylith_b200 import feassemble as FA

    O, torch = oracle_lib, torch_cuda
    d = ref_meshes[key]
    m = d.mesh
    rho, mu, K = MAT.uniform_elastic(m.num_cells)
    X = m.coords
    u = np.stack([1e-4 * X[:, 0] + 2e-5 * X[:, 1] - 3e-5 * X[:, 2], 3e-5 * X[:, 0] - 1e-4 * X[:, 1] + 4e-5 * X[:, 2],
                  -2e-5 * X[:, 0] + 1e-5 * X[:, 1] + 5e-5 * X[:, 2]], axis=1).ravel()
    r_ref = O.residual(m, u, elastic_aux(O, rho, mu, K), f1=F1_ILE)
    ig = MAT.IsotropicLinearElasticity(rho, mu, K).create_integrator(FA.DeviceMesh(ctx, m))
    du = dev(torch, u)
    dr = torch.full_like(du, np.nan)
    ig.compute_lhs_residual(0.0, 0.0, du, dr)
    ctx.synchronize()
    r = dr.cpu().numpy()
    assert rel_l2(r, r_ref) <= TOL64
    interior = np.ones(m.num_nodes, dtype=bool)
    interior[d.vertex_groups["boundary"]] = False
    assert interior.sum() > 0
    assert np.abs(r.reshape(-1, 3)[interior]).max() <= 1e-12 * np.abs(r).max()


@pytest.mark.parametrize("key", ["axial_tet", "axial_hex"])
@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32_refined"])
def test_reference_exodus_meshes_axial_solve_on_gpu(oracle_lib, torch_cuda, ctx, ref_meshes, key, precision):
    """axialdisp.cfg on the reference's ExodusII meshes, one integrator per material block
    (ids 1 and 2): the GPU residual matches the oracle and the GPU solve reproduces the analytic
    displacement (axialdisp_soln.py)."""
    from pylith_b200 import feassemble as FA
    from pylith_b200 import meshio as MIO

    O, torch = oracle_lib, torch_cuda
    d = ref_meshes[key]
    m = d.mesh
    cons = MIO.constrained_mask(d, [("boundary_xneg", [0]), ("boundary_xpos", [0]), ("boundary_yneg", [1]),
                                    ("boundary_ypos", [1]), ("boundary_zneg", [2])])
    uex = KA.axial_displacement(m.coords).ravel()
    dm = FA.DeviceMesh(ctx, m)
    igs, r_ref = [], np.zeros(m.num_dof)
    u0 = np.where(cons, uex, 0.0)
    for mid in (1, 2):
        ids = np.flatnonzero(d.material_ids == mid).astype(np.int32)
        rho, mu, K = MAT.uniform_elastic(len(ids), KA.AXIAL_DENSITY, KA.AXIAL_VS, KA.AXIAL_VP)
        sub = M.Mesh(m.cell_type, m.coords, m.cells[ids])
        r_ref += O.residual(sub, u0, elastic_aux(O, rho, mu, K), f1=F1_ILE)
        igs.append(MAT.IsotropicLinearElasticity(rho, mu, K).create_integrator(dm, ids))
    u = dev(torch, u0)
    F = torch.full_like(u, np.nan)
    for k, ig in enumerate(igs):
        ig.compute_lhs_residual(0.0, 0.0, u, F, mode=FA.INSERT if k == 0 else FA.ADD)
    ctx.synchronize()
    assert rel_l2(F.cpu().numpy(), r_ref) <= TOL64
    S = FA.Solver(dm, cons, igs, rtol=1e-12, precision=precision)
    S.setup()
    du = torch.zeros_like(u)
    S.solve(F, du)
    ctx.synchronize()
    sol = (u + du).cpu().numpy()
    assert np.abs(sol - uex).max() <= 1e-9 * np.abs(uex).max(), S.stats()


def _rotation(axis, angle):
    axis = np.asarray(axis, dtype=float) / np.linalg.norm(axis)
    Kx = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    return np.eye(3) + np.sin(angle) * Kx + (1 - np.cos(angle)) * Kx @ Kx


@pytest.mark.parametrize("angle,ref_dir_2", [(0.7, (0.0, 0.3, 1.0)), (2.4, (0.6, 0.3, 0.0))],
                         ids=["normal_pos_x", "normal_neg_x"])
def test_oblique_fault_matches_oracle(oracle_lib, torch_cuda, ctx, angle, ref_dir_2):
    """The cohesive residual, Jacobian action and assembly with the fault x = 0 turned about an
    oblique axis, so the fault normal has non-zero y and z components; refDir2 is chosen so that
    the sign test of tangential_directions as the reference writes it (refDir2[0] n[0] +
    refDir2[1] n[1] + refDir2[1] n[1]) and the plain dot product refDir2 . n disagree, i.e. the
    repeated term decides whether tanDir2 flips. Plus the domain + interface residual of the
    whole rotated problem."""
    from pylith_b200 import feassemble as FA

    O, torch = oracle_lib, torch_cuda
    base = M.insert_fault_x(M.box_hex(6, 4, 3))
    R = _rotation((0.3, 0.5, 0.8), angle)
    mesh = M.Mesh(base.cell_type, np.ascontiguousarray(base.coords @ R.T), base.cells, base.cohesive,
                  base.num_lagrange)
    Xc = mesh.coords[mesh.cohesive[:, :3]]
    n = np.cross(Xc[:, 1] - Xc[:, 0], Xc[:, 2] - Xc[:, 0])
    assert np.abs(n[:, 1]).min() > 0.05 * np.abs(n).max() and np.abs(n[:, 2]).min() > 0.05 * np.abs(n).max()
    r2 = np.asarray(ref_dir_2)
    quirk = r2[0] * n[:, 0] + r2[1] * n[:, 1] + r2[1] * n[:, 1]
    assert (np.sign(quirk) != np.sign(n @ r2)).all()
    rng = np.random.default_rng(104)
    fault = MAT.FaultCohesiveKin(rng.standard_normal((mesh.num_lagrange, 3)), ref_dir_1=(0, 0, 1),
                                 ref_dir_2=ref_dir_2)
    u = rng.standard_normal(mesh.num_dof)
    v = rng.standard_normal(mesh.num_dof)
    r_ref = O.cohesive_residual(mesh, u, fault.slip, fault.constants)
    Jc = O.cohesive_jacobian(mesh, fault.constants)
    dm = FA.DeviceMesh(ctx, mesh)
    ifc = fault.create_integrator(dm)
    du, dv = dev(torch, u), dev(torch, v)
    dr, djv = torch.zeros_like(du), torch.zeros_like(du)
    ifc.compute_lhs_residual(0.0, 0.0, du, dr)
    ifc.compute_lhs_jacobian_action(0.0, 0.0, 0.0, du, dv, djv)
    ctx.synchronize()
    assert rel_l2(dr.cpu().numpy(), r_ref) <= TOL64
    assert rel_l2(djv.cpu().numpy(), Jc @ v) <= TOL64
    A = FA.Matrix(dm)
    ifc.compute_lhs_jacobian(0.0, 0.0, 0.0, None, A)
    assert abs(A.to_scipy().tocsr() - Jc).max() <= 1e-12 * abs(Jc).max()
    # domain + interface, as TimeDependent sums its integrators
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=105)
    nn = 3 * mesh.num_nodes
    full = np.zeros(mesh.num_dof)
    full[:nn] = O.residual(mesh, u[:nn], elastic_aux(O, rho, mu, K), f1=F1_ILE)
    O.cohesive_residual(mesh, u, fault.slip, fault.constants, r=full)
    ig = MAT.IsotropicLinearElasticity(rho, mu, K).create_integrator(dm)
    dr2 = torch.full_like(du, np.nan)
    ig.compute_lhs_residual(0.0, 0.0, du, dr2)
    ifc.compute_lhs_residual(0.0, 0.0, du, dr2, mode=FA.ADD)
    ctx.synchronize()
    assert rel_l2(dr2.cpu().numpy(), full) <= TOL64
