"""Geometric multigrid preconditioning of the device solver (pl_multigrid_*): on a Q1 box with a
fault at x = 0, flexible CG with V-cycles (FP64, or FP32 V-cycles under FP64 CG) reaches the
point-block-Jacobi PCG solution (relative displacement difference <= 1e-8 at rtol 1e-12) in at
least five times fewer iterations, for isotropic elasticity and generalized Maxwell, with nested
levels and with levels whose grids are not nested."""
import numpy as np
import pytest

from pylith_b200 import materials as MAT
from pylith_b200 import meshing as M
from pylith_b200 import multigrid as MG

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pylith_b200 import feassemble as FA

    return FA.Context(0)


@pytest.mark.parametrize("rheology,dims", [("elastic", (16, 16, 12)), ("genmaxwell", (16, 16, 12)),
                                           ("elastic", (18, 14, 11))])  # the last: non-nested levels
def test_multigrid_matches_point_jacobi_in_fewer_iterations(ctx, rheology, dims):
    from pylith_b200 import feassemble as FA
    from pylith_b200 import problems as P

    levels = MG.build_hierarchy(*dims, fault_x=0.0, constrained_faces=[(0, "neg", (0, 1, 2)), (0, "pos", (0, 1, 2))])
    assert len(levels) >= 3
    mesh, cons = levels[0].mesh, levels[0].constrained
    nc = mesh.num_cells
    rho, mu, K = MAT.lognormal_elastic(nc, seed=3)
    dt = MAT.YEAR if rheology == "genmaxwell" else 0.0
    if rheology == "genmaxwell":
        tau = MAT.genmaxwell_times(rho, np.sqrt(mu / rho), [1e18, 1e19, 1e20], [0.3, 0.3, 0.3])
        mat = MAT.IsotropicLinearGenMaxwell(rho, mu, K, tau, np.tile([0.3, 0.3, 0.3], (nc, 1)),
                                            np.zeros((nc, 8, 18)), np.zeros((nc, 8, 6)))
    else:
        mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    slip = np.zeros((mesh.num_lagrange, 3))
    slip[: mesh.num_lagrange // 2, 1] = 2.0
    bc = np.zeros(mesh.num_dof)

    def run(precision=None):
        prob = P.QuasistaticProblem(ctx, mesh, [(mat, None)], cons, bc, faults=[MAT.FaultCohesiveKin(slip)], dt=dt,
                                    precision=FA.Solver.FP64, rtol=1e-12)
        mg = None
        if precision is not None:
            mg = MG.attach(ctx, prob.solver, levels, mat, fault_x=0.0, dt=dt, precision=precision)
        st = prob.step(dt)
        u = prob.u.cpu().numpy()
        lam = mg.lambda_max() if mg else None
        if mg:
            mg.close()
        return u, st, lam

    u_ref, st_ref, _ = run()
    for precision in (FA.Solver.FP64, FA.Solver.FP32_REFINED):
        u, st, lam = run(precision)
        assert st.rel_residual <= 1e-12
        assert np.linalg.norm(u - u_ref) <= 1e-8 * np.linalg.norm(u_ref), (precision, st)
        assert 5 * st.iterations <= st_ref.iterations, (st.iterations, st_ref.iterations)
        assert all(v > 0 for v in lam[:-1])  # the coarsest level is solved with its dense inverse


def test_multigrid_on_unstructured_tetrahedra_with_a_fault(ctx):
    """Multigrid over independent Delaunay meshes of the same box and fault plane (P1 tetrahedra,
    barycentric interpolation per fault side): FP64 and FP32 V-cycles under FP64 CG reach the
    point-block-Jacobi solution (<= 1e-8) in at least five times fewer iterations."""
    from pylith_b200 import feassemble as FA
    from pylith_b200 import problems as P

    lo, hi = (-6000.0, -6000.0, -9000.0), (6000.0, 6000.0, 0.0)
    mesh = M.box_tet_delaunay_fault_x(120000, seed=1, lo=lo, hi=hi)
    levels = MG.build_tet_hierarchy(mesh, lambda n, l: M.box_tet_delaunay_fault_x(n, seed=10 + l, lo=lo, hi=hi),
                                    fault_x=0.0, lo=lo, hi=hi,
                                    constrained_faces=[(0, "neg", (0, 1, 2)), (0, "pos", (0, 1, 2))], min_cells=500)
    assert len(levels) >= 3
    cons = levels[0].constrained
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=4)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    slip = np.zeros((mesh.num_lagrange, 3))
    slip[: mesh.num_lagrange // 3, 1] = 1.5
    bc = np.zeros(mesh.num_dof)

    def run(precision=None):
        prob = P.QuasistaticProblem(ctx, mesh, [(mat, None)], cons, bc, faults=[MAT.FaultCohesiveKin(slip)],
                                    precision=FA.Solver.FP64, rtol=1e-12)
        mg = None
        if precision is not None:
            mg = MG.attach(ctx, prob.solver, levels, mat, fault_x=0.0, precision=precision)
        st = prob.step(0.0)
        u = prob.u.cpu().numpy()
        if mg:
            mg.close()
        prob.close()
        return u, st

    u_ref, st_ref = run()
    for precision in (FA.Solver.FP64, FA.Solver.FP32_REFINED):
        u, st = run(precision)
        assert st.rel_residual <= 1e-12
        assert np.linalg.norm(u - u_ref) <= 1e-8 * np.linalg.norm(u_ref), (precision, st)
        assert 5 * st.iterations <= st_ref.iterations, (st.iterations, st_ref.iterations)


def test_batched_multigrid_green_functions(ctx):
    """Green's functions on a Delaunay fault mesh, batched: tiles of 8 impulses whose FP32 PCG is
    preconditioned by one V-cycle of the tet hierarchy on all 8 vectors at once. The solutions match
    one-at-a-time FP64 solves to <= 1e-8 with far fewer iterations than the point-Jacobi tiles."""
    from pylith_b200 import feassemble as FA
    from pylith_b200 import greensfns as GF

    lo, hi = (-6000.0, -6000.0, -9000.0), (6000.0, 6000.0, 0.0)
    mesh = M.box_tet_delaunay_fault_x(120000, seed=3, lo=lo, hi=hi)
    levels = MG.build_tet_hierarchy(mesh, lambda n, l: M.box_tet_delaunay_fault_x(n, seed=20 + l, lo=lo, hi=hi),
                                    fault_x=0.0, lo=lo, hi=hi,
                                    constrained_faces=[(0, "neg", (0, 1, 2)), (0, "pos", (0, 1, 2))], min_cells=500)
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=6)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    patches = GF.fault_patches(mesh, (-6000.0, 6000.0), (-9000.0, 0.0), 4, 3)
    g = GF.GreensFunctions(ctx, mesh, mat, levels[0].constrained, patches, rtol=1e-11, inner_rtol=1e-4, tile=8)
    g.attach_multigrid(levels, mat, FA.Solver.FP32_REFINED)
    bmg = g.batched_multigrid(8)
    imps = g.impulses[:8]
    ref, _ = g.solve(imps, batched=False)
    got, _ = g.solve(imps, batched=True, batch=bmg)
    st_mg = bmg.stats()
    _, _ = g.solve(imps, batched=True)
    st_j = g.batch.stats()
    for a, b in zip(got, ref):
        a, b = a.cpu().numpy(), b.cpu().numpy()
        assert np.linalg.norm(a - b) <= 1e-8 * np.linalg.norm(b)
    assert st_mg["max_rel_residual"] <= 1e-11
    assert 5 * st_mg["inner_iterations"] <= st_j["inner_iterations"], (st_mg, st_j)
