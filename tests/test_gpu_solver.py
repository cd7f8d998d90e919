"""GPU linear solves of the quasi-static step against the reference's analytic known answers
and the oracle's direct solve."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

import known_answers as KA
from pylith_b200 import materials as MAT
from pylith_b200 import meshing as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pylith_b200 import feassemble as FA

    return FA.Context(0)


def solve_quasistatic(ctx, mesh, mat, uex, cons, precision, rtol=1e-12):
    """u = Dirichlet values, F = residual(u), solve (-J) du = F on free DOFs, u += du."""
    import torch
    from pylith_b200 import feassemble as FA

    dm = FA.DeviceMesh(ctx, mesh)
    ig = mat.create_integrator(dm)
    u = torch.from_numpy(np.where(cons, uex, 0.0)).cuda()
    F = torch.zeros_like(u)
    ig.compute_lhs_residual(0.0, 0.0, u, F)
    S = FA.Solver(dm, cons, [ig], rtol=rtol, precision=precision)
    S.setup()
    du = torch.zeros_like(u)
    S.solve(F, du)
    ctx.synchronize()
    return (u + du).cpu().numpy(), S.stats()


@pytest.mark.parametrize("make", [lambda: M.box_hex(8, 8, 6), lambda: M.box_tet_delaunay(20000, seed=1),
                                  lambda: M.box_hex27(4, 4, 3)], ids=["hex8", "tet4", "hex27"])
@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32_refined"])
def test_axial_displacement_solve(ctx, make, precision):
    mesh = make()
    rho, mu, K = MAT.uniform_elastic(mesh.num_cells, KA.AXIAL_DENSITY, KA.AXIAL_VS, KA.AXIAL_VP)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    uex = KA.axial_displacement(mesh.coords).ravel()
    cons = KA.axial_constrained(mesh)
    u, stats = solve_quasistatic(ctx, mesh, mat, uex, cons, precision)
    assert stats["rel_residual"] <= 1e-12
    assert np.abs(u - uex).max() <= 1e-9 * np.abs(uex).max(), stats


def test_heterogeneous_solve_matches_oracle_direct_solve(ctx, oracle_lib):
    """Log-normal material on tets: FP64 PCG and FP32-refined PCG against scipy's direct solve
    of the oracle-assembled system (relative displacement error <= 1e-8 for FP32 refined)."""
    O = oracle_lib
    mesh = M.box_tet_delaunay(8000, seed=4)
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=3)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    cons[M.boundary_mask(mesh, 0, "neg"), 0] = True
    cons[M.boundary_mask(mesh, 0, "pos"), 0] = True
    cons[M.boundary_mask(mesh, 1, "neg"), 1] = True
    cons[M.boundary_mask(mesh, 2, "neg"), 2] = True
    cons = cons.ravel()
    ubc = np.zeros((mesh.num_nodes, 3))
    ubc[M.boundary_mask(mesh, 0, "neg"), 0] = -1.0
    ubc[M.boundary_mask(mesh, 0, "pos"), 0] = 1.0
    ubc = ubc.ravel()
    aux = O.AuxFields([(rho[:, None], "cell"), (mu[:, None], "cell"), (K[:, None], "cell")])
    J = O.assemble(mesh, O.jacobian_elements(mesh, aux, g3="IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain"))
    u_ref = np.where(cons, ubc, 0.0)
    r = O.residual(mesh, u_ref, aux, f1="IsotropicLinearElasticity3D::f1v_infinitesimalStrain")
    free = ~cons
    u_ref[free] += spla.spsolve(J[free][:, free].tocsc(), -r[free])
    u64, s64 = solve_quasistatic(ctx, mesh, mat, ubc, cons, 0)
    u32, s32 = solve_quasistatic(ctx, mesh, mat, ubc, cons, 1)
    err64 = np.linalg.norm(u64 - u_ref) / np.linalg.norm(u_ref)
    err32 = np.linalg.norm(u32 - u_ref) / np.linalg.norm(u_ref)
    assert err64 <= 1e-10, (err64, s64)
    assert err32 <= 1e-8, (err32, s32)
    assert s32["inner_iterations"] > 0


def test_fault_rigid_blocks_solve(ctx):
    """Prescribed slip between two blocks with Dirichlet x faces (twoblocks.cfg): the reduced
    (slip-constrained) PCG reproduces the rigid-block answer -/+ d/2."""
    import torch
    from pylith_b200 import feassemble as FA

    mesh = M.insert_fault_x(M.box_hex(6, 4, 4))
    rho, mu, K = MAT.uniform_elastic(mesh.num_cells)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    fault = MAT.FaultCohesiveKin(np.tile([0.0, -2.0, 1.0], (mesh.num_lagrange, 1)),
                                 ref_dir_1=(0, 0, 1), ref_dir_2=(0.5, 0, 0.5))
    d = np.array([0.0, -2.0, 1.0])  # n = +x, t1 = +y, t2 = +z
    plus = np.zeros(mesh.num_nodes, dtype=bool)
    plus[np.unique(mesh.cells[mesh.coords[mesh.cells].mean(axis=1)[:, 0] > 0])] = True
    uex = np.where(plus[:, None], 0.5 * d, -0.5 * d).ravel()
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    cons[M.boundary_mask(mesh, 0, "neg")] = True
    cons[M.boundary_mask(mesh, 0, "pos")] = True
    cons = np.concatenate([cons.ravel(), np.zeros(3 * mesh.num_lagrange, dtype=bool)])
    dm = FA.DeviceMesh(ctx, mesh)
    ig = mat.create_integrator(dm)
    iface = fault.create_integrator(dm)
    S = FA.Solver(dm, cons, [ig], rtol=1e-12)
    u0 = np.zeros(mesh.num_dof)
    u0[:3 * mesh.num_nodes] = np.where(cons[:3 * mesh.num_nodes], uex, 0.0)
    u = torch.from_numpy(u0).cuda()
    S.apply_fault_slip(iface, u)
    F = torch.zeros_like(u)
    ig.compute_lhs_residual(0.0, 0.0, u, F)
    S.setup()
    du = torch.zeros_like(u)
    S.solve(F, du)
    ctx.synchronize()
    got = (u + du).cpu().numpy()[:3 * mesh.num_nodes]
    np.testing.assert_allclose(got, uex, atol=1e-9)


def test_fault_random_slip_solve_matches_oracle_saddle_point(ctx, oracle_lib):
    """Non-uniform slip and log-normal material: the reduced PCG solution equals the oracle's
    direct solve of the full saddle-point system (u and lambda), and the full residual of the
    GPU solution (domain + cohesive integrators, lambda from the oracle's solve) vanishes."""
    import scipy.sparse as sp
    import torch
    from pylith_b200 import feassemble as FA

    O = oracle_lib
    mesh = M.insert_fault_x(M.box_hex(6, 5, 4))
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=7)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    rng = np.random.default_rng(3)
    slip = rng.uniform(-1, 1, (mesh.num_lagrange, 3))
    fault = MAT.FaultCohesiveKin(slip, ref_dir_1=(0, 0, 1), ref_dir_2=(0, 1, 0))
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    cons[M.boundary_mask(mesh, 0, "neg")] = True
    cons[M.boundary_mask(mesh, 0, "pos")] = True
    cons[M.boundary_mask(mesh, 2, "neg"), 2] = True
    cons = np.concatenate([cons.ravel(), np.zeros(3 * mesh.num_lagrange, dtype=bool)])
    ubc = np.zeros(mesh.num_dof)
    ubc[:3 * mesh.num_nodes] = rng.uniform(-0.5, 0.5, 3 * mesh.num_nodes)
    # oracle saddle point
    aux = O.AuxFields([(rho[:, None], "cell"), (mu[:, None], "cell"), (K[:, None], "cell")])
    Kd = O.assemble(mesh, O.jacobian_elements(mesh, aux, g3="IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain"),
                    ndof=mesh.num_dof)
    J = (Kd + O.cohesive_jacobian(mesh, fault.constants)).tocsr()
    u_ref = np.where(cons, ubc, 0.0)
    r = np.zeros(mesh.num_dof)
    r[:3 * mesh.num_nodes] = O.residual(mesh, u_ref[:3 * mesh.num_nodes], aux,
                                        f1="IsotropicLinearElasticity3D::f1v_infinitesimalStrain")
    O.cohesive_residual(mesh, u_ref, slip, fault.constants, r=r)
    free = ~cons
    u_ref[free] += spla.spsolve(sp.csc_matrix(J[free][:, free]), -r[free])
    # GPU reduced solve
    dm = FA.DeviceMesh(ctx, mesh)
    ig = mat.create_integrator(dm)
    iface = fault.create_integrator(dm)
    for precision, tol in ((0, 1e-10), (1, 1e-8)):
        S = FA.Solver(dm, cons, [ig], rtol=1e-13, precision=precision)
        u = torch.from_numpy(np.where(cons, ubc, 0.0)).cuda()
        S.apply_fault_slip(iface, u)
        F = torch.zeros_like(u)
        ig.compute_lhs_residual(0.0, 0.0, u, F)
        S.setup()
        du = torch.zeros_like(u)
        S.solve(F, du)
        ctx.synchronize()
        got = (u + du).cpu().numpy()
        nd = 3 * mesh.num_nodes
        err = np.linalg.norm(got[:nd] - u_ref[:nd]) / np.linalg.norm(u_ref[:nd])
        assert err <= tol, (precision, err, S.stats())
    # full residual with lambda from the reference solve vanishes at the GPU solution
    full = got.copy()
    full[nd:] = u_ref[nd:]
    dfull = torch.from_numpy(full).cuda()
    R = torch.zeros_like(dfull)
    ig.compute_lhs_residual(0.0, 0.0, dfull, R)
    iface.compute_lhs_residual(0.0, 0.0, dfull, R, mode=FA.ADD)
    ctx.synchronize()
    Rn = R.cpu().numpy()
    scale = np.abs(r).max()
    assert np.abs(Rn[free]).max() <= 1e-6 * scale
