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
    # Dirichlet DOFs only away from the fault: a boundary value on a fault node that disagrees
    # with the prescribed slip would make the saddle-point system inconsistent.
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    cons[M.boundary_mask(mesh, 0, "neg")] = True
    cons[M.boundary_mask(mesh, 0, "pos")] = True
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
    # the oracle's direct saddle-point solve itself carries ~1e-10 relative error here
    for precision, tol in ((0, 1e-9), (1, 1e-8)):
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


def test_quasistatic_genmaxwell_relaxation_driver(ctx):
    """axialstrain_genmaxwell (tests/fullscale/viscoelasticity/nofaults-3d): Dirichlet normal
    displacements on all faces hold the axial strain e0; 20 steps of dt = 0.025 yr through the
    device driver reproduce the analytic stress relaxation."""
    import torch
    from pylith_b200 import problems as P

    mesh = M.box_hex(4, 4, 4, lo=(-4000.0, -4000.0, -8000.0), hi=(4000.0, 4000.0, 0.0))
    mu, K, lam, tau = KA.genmaxwell_params()
    nc, nq, e0 = mesh.num_cells, 8, KA.GM_E0
    g = MAT.IsotropicLinearGenMaxwell(
        np.full(nc, KA.GM_DENSITY), np.full(nc, mu), np.full(nc, K), np.tile(tau, (nc, 1)),
        np.tile(KA.GM_RATIO, (nc, 1)), np.tile([-e0 / 3, -e0 / 3, 2 * e0 / 3, 0, 0, 0] * 3, (nc, nq, 1)),
        np.tile([0, 0, e0, 0, 0, 0.0], (nc, nq, 1)))
    lo, hi = (-4000.0, -4000.0, -8000.0), (4000.0, 4000.0, 0.0)
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    for ax in range(3):
        for sd in ("neg", "pos"):
            cons[M.boundary_mask(mesh, ax, sd, lo, hi), ax] = True
    X = mesh.coords
    bc = np.stack([0 * X[:, 0], 0 * X[:, 1], e0 * (X[:, 2] + 8000.0)], axis=1).ravel()
    prob = P.QuasistaticProblem(ctx, mesh, [(g, None)], cons.ravel(), bc, dt=KA.GM_DT, rtol=1e-13)
    for step in range(1, KA.GM_STEPS + 1):
        t = step * KA.GM_DT
        # stress of this step is evaluated from the previous state before the update
        prob.u = torch.from_numpy(bc).cuda()
        R = prob.residual(t).cpu().numpy()
        sigma = KA.stress_from_residual(X, R, 8000.0**3)
        np.testing.assert_allclose(np.diag(sigma), KA.genmaxwell_stress(t), rtol=1e-10)
        st = prob.step(t)
        ctx.synchronize()
        np.testing.assert_allclose(prob.u.cpu().numpy(), bc, atol=1e-12)


def test_genmaxwell_fault_time_steps_match_oracle(ctx, oracle_lib):
    """Generalized Maxwell material with a prescribed-slip fault, three time steps on the device
    driver (reduced fault PCG) against the same steps on the oracle (assembled saddle point,
    direct solve, quadrature-point state projection)."""
    import scipy.sparse as sp
    import torch
    from pylith_b200 import problems as P

    O = oracle_lib
    mesh = M.insert_fault_x(M.box_hex(6, 4, 4))
    nc, nq = mesh.num_cells, 8
    rho, mu, K = MAT.lognormal_elastic(nc, seed=2)
    tau = MAT.genmaxwell_times(rho, np.sqrt(mu / rho), [1e18, 1e19, 1e20], [0.3, 0.3, 0.3])
    ratio = np.tile([0.3, 0.3, 0.3], (nc, 1))
    visc = np.zeros((nc, nq, 18))
    total = np.zeros((nc, nq, 6))
    g = MAT.IsotropicLinearGenMaxwell(rho, mu, K, tau, ratio, visc, total)
    slip = np.tile([0.0, 2.0, 0.0], (mesh.num_lagrange, 1))  # left-lateral 2 m
    fault = MAT.FaultCohesiveKin(slip)
    # Dirichlet DOFs away from the fault (a constrained DOF on both sides of a fault node leaves
    # that node's Lagrange multiplier without an equation)
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    cons[M.boundary_mask(mesh, 0, "neg")] = True
    cons[M.boundary_mask(mesh, 0, "pos")] = True
    cons = np.concatenate([cons.ravel(), np.zeros(3 * mesh.num_lagrange, dtype=bool)])
    bc = np.zeros(mesh.num_dof)
    dt = 1.0 * MAT.YEAR
    prob = P.QuasistaticProblem(ctx, mesh, [(g, None)], cons, bc, faults=[fault], dt=dt, rtol=1e-13)
    # oracle state
    o_visc, o_total = visc.copy(), total.copy()
    u_o = np.zeros(mesh.num_dof)
    nd = 3 * mesh.num_nodes
    free = ~cons
    F1 = "IsotropicLinearGenMaxwell3D::f1v_infinitesimalStrain"
    for step in range(1, 4):
        t = step * dt
        prob.step(t)
        ctx.synchronize()
        aux = O.AuxFields([(rho[:, None], "cell"), (mu[:, None], "cell"), (K[:, None], "cell"), (tau, "cell"),
                           (ratio, "cell"), (o_visc, "qp"), (o_total, "qp")])
        Kd = O.assemble(mesh, O.jacobian_elements(mesh, aux, g3="IsotropicLinearGenMaxwell3D::Jf3vu_infinitesimalStrain",
                                                  constants=[dt]), ndof=mesh.num_dof)
        J = (Kd + O.cohesive_jacobian(mesh, fault.constants)).tocsr()
        u_o = np.where(cons, bc, u_o)
        r = np.zeros(mesh.num_dof)
        r[:nd] = O.residual(mesh, u_o[:nd], aux, f1=F1, constants=[dt])
        O.cohesive_residual(mesh, u_o, slip, fault.constants, r=r)
        u_o[free] += spla.spsolve(sp.csc_matrix(J[free][:, free]), -r[free])
        o_visc, o_total = O.project_qp(
            mesh, u_o[:nd], aux, ["IsotropicLinearGenMaxwell3D::viscousStrain_infinitesimalStrain_asVector",
                                  "Elasticity3D::infinitesimalStrain_asVector"], [18, 6], constants=[dt])
        got = prob.u.cpu().numpy()
        err = np.linalg.norm(got[:nd] - u_o[:nd]) / np.linalg.norm(u_o[:nd])
        assert err <= 1e-9, (step, err)
        gv = prob.domain[0].get_aux("viscous_strain", (nc, nq, 18))
        assert np.linalg.norm(gv - o_visc) <= 1e-8 * np.linalg.norm(o_visc), step


def test_batched_green_functions_match_single_fp64_solves(ctx):
    """Unit-slip patch impulses (left-lateral and reverse) on a tetrahedral mesh with a planar
    fault: the batched FP32-refined solver (tiles of 1, 2, 4, 8 and 16 right-hand sides, CUDA-graph
    replay) matches one-at-a-time FP64 solves to <= 1e-8 relative displacement error."""
    from pylith_b200 import greensfns as GF

    mesh = M.box_tet_kuhn(8, 6, 5, fault_x=0.0, seed=3)
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=5)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    cons[M.boundary_mask(mesh, 0, "neg")] = True
    cons[M.boundary_mask(mesh, 0, "pos")] = True
    cons = np.concatenate([cons.ravel(), np.zeros(3 * mesh.num_lagrange, dtype=bool)])
    patches = GF.fault_patches(mesh, (-6000.0, 6000.0), (-9000.0, 0.0), 3, 2)
    for tile in (1, 2, 4, 8, 16):
        g = GF.GreensFunctions(ctx, mesh, mat, cons, patches, rtol=1e-11, tile=tile)
        imps = g.impulses[:10] if tile < 16 else g.impulses[:12]
        ref, _ = g.solve(imps, batched=False)
        got, _ = g.solve(imps, batched=True)
        for a, b in zip(got, ref):
            a, b = a.cpu().numpy(), b.cpu().numpy()
            assert np.linalg.norm(a - b) <= 1e-8 * np.linalg.norm(b)
        st = g.batch.stats()
        assert st["solves"] == len(imps) and st["inner_iterations"] > 0


def test_batched_chebyshev_jacobi_eigen_estimate_and_solutions(ctx, oracle_lib):
    """Chebyshev-Jacobi preconditioning of the batched FP32 PCG on a Kuhn tetrahedral mesh: the
    power-iteration estimate of lambda_max(P A) lies within [0.85, 1.0001] of the largest
    generalized eigenvalue of the oracle-assembled stiffness against its 3x3 node blocks
    (scipy), the solutions match one-at-a-time FP64 solves to <= 1e-8, and degree 3 needs fewer
    inner iterations than point-block Jacobi."""
    import scipy.linalg as sla
    import torch
    from pylith_b200 import feassemble as FA

    O = oracle_lib
    mesh = M.box_tet_kuhn(8, 6, 5, seed=3)
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=5)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    cons[M.boundary_mask(mesh, 0, "neg")] = True
    cons[M.boundary_mask(mesh, 0, "pos")] = True
    cons[M.boundary_mask(mesh, 2, "neg"), 2] = True
    cons = cons.ravel()
    aux = O.AuxFields([(rho[:, None], "cell"), (mu[:, None], "cell"), (K[:, None], "cell")])
    J = O.assemble(mesh, O.jacobian_elements(mesh, aux, g3="IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain"))
    A = -J.toarray()
    free = ~cons
    D = np.zeros_like(A)
    for nd in range(mesh.num_nodes):
        s = slice(3 * nd, 3 * nd + 3)
        D[s, s] = A[s, s]
    lam_true = sla.eigh(A[free][:, free], D[free][:, free], eigvals_only=True)[-1]

    dm = FA.DeviceMesh(ctx, mesh)
    ig = mat.create_integrator(dm)
    S64 = FA.Solver(dm, cons, [ig], rtol=1e-11)
    S64.setup()
    S32 = FA.Solver(dm, cons, [ig], rtol=1e-11, precision=FA.Solver.FP32_REFINED, inner_rtol=1e-4)
    S32.setup()
    g = torch.Generator(device="cuda").manual_seed(11)
    bs = [torch.randn(dm.num_dof, dtype=torch.float64, device="cuda", generator=g) * torch.from_numpy(free).cuda()
          for _ in range(8)]
    ref = []
    for b in bs:
        x = torch.zeros_like(b)
        S64.solve(b, x)
        ref.append(x.cpu().numpy())
    iters = {}
    for degree in (0, 3):
        B = FA.BatchSolver(S32, 8)
        B.set_chebyshev(degree, lower_ratio=0.05)
        xs = [torch.zeros_like(b) for b in bs]
        B.solve(bs, xs)
        ctx.synchronize()
        for a, r in zip(xs, ref):
            assert np.linalg.norm(a.cpu().numpy() - r) <= 1e-8 * np.linalg.norm(r), degree
        iters[degree] = B.stats()["inner_iterations"]
        if degree == 3:
            assert 0.85 * lam_true <= B.lambda_max <= 1.0001 * lam_true, (B.lambda_max, lam_true)
        B.close()
    assert iters[3] < iters[0], iters


def test_green_functions_autotune_keeps_the_fastest_configuration(ctx):
    """The tile/preconditioner autotuner times every (tile, degree) pair on a sample of impulses
    and keeps the fastest batched solver, whose solutions still match FP64 solves to <= 1e-8."""
    from pylith_b200 import greensfns as GF

    mesh = M.box_tet_kuhn(8, 6, 5, fault_x=0.0, seed=3)
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=5)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    cons[M.boundary_mask(mesh, 0, "neg")] = True
    cons[M.boundary_mask(mesh, 0, "pos")] = True
    cons = np.concatenate([cons.ravel(), np.zeros(3 * mesh.num_lagrange, dtype=bool)])
    patches = GF.fault_patches(mesh, (-6000.0, 6000.0), (-9000.0, 0.0), 3, 2)
    g = GF.GreensFunctions(ctx, mesh, mat, cons, patches, rtol=1e-11)
    res = g.autotune(g.impulses[:8], tiles=(2, 4), degrees=(0, 3))
    assert len(res) == 4 and res[0][2] >= res[-1][2]
    assert (g.batch.tile, g.batch.degree) == res[0][:2]
    imps = g.impulses[:6]
    ref, _ = g.solve(imps, batched=False)
    got, _ = g.solve(imps, batched=True)
    for a, b in zip(got, ref):
        a, b = a.cpu().numpy(), b.cpu().numpy()
        assert np.linalg.norm(a - b) <= 1e-8 * np.linalg.norm(b)


def test_batched_reliable_updates_match_fp64_with_fewer_iterations(ctx):
    """Reliable updates (one FP32 PCG per right-hand side, residual replacement by the FP64 true
    residual) and restarted FP64 refinement both match one-at-a-time FP64 solves to <= 1e-8; the
    reliable updates need no more tile iterations than the restarts."""
    import torch
    from pylith_b200 import greensfns as GF

    mesh = M.box_tet_kuhn(12, 10, 8, fault_x=0.0, seed=4)
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=6)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    cons[M.boundary_mask(mesh, 0, "neg")] = True
    cons[M.boundary_mask(mesh, 0, "pos")] = True
    cons = np.concatenate([cons.ravel(), np.zeros(3 * mesh.num_lagrange, dtype=bool)])
    patches = GF.fault_patches(mesh, (-6000.0, 6000.0), (-9000.0, 0.0), 4, 3)
    g = GF.GreensFunctions(ctx, mesh, mat, cons, patches, rtol=1e-11, inner_rtol=1e-4, tile=8)
    imps = g.impulses[:8]
    ref, _ = g.solve(imps, batched=False)
    iters = {}
    for reliable in (True, False):
        g.batch.set_reliable(reliable, 0.1)
        got, _ = g.solve(imps, batched=True)
        for a, b in zip(got, ref):
            a, b = a.cpu().numpy(), b.cpu().numpy()
            assert np.linalg.norm(a - b) <= 1e-8 * np.linalg.norm(b), reliable
        st = g.batch.stats()
        assert st["max_rel_residual"] <= 1e-11
        iters[reliable] = st["inner_iterations"]
    assert iters[True] <= iters[False], iters


def test_batched_energy_sums_in_the_operator_launch_match_the_reduction_kernel(ctx, monkeypatch):
    """The batched PCG sums p.(A p) inside the operator launch, from the cells' energies (on a
    fault mesh: the reduced space's fold must not change the sum); the solutions and iteration
    counts match those of the separate DOF-wise reduction kernel, and both match FP64 solves."""
    from pylith_b200 import greensfns as GF

    lo, hi = (-6000.0, -6000.0, -9000.0), (6000.0, 6000.0, 0.0)
    mesh = M.box_tet_delaunay_fault_x(20000, seed=2, lo=lo, hi=hi)
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=7)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    cons[M.boundary_mask(mesh, 0, "neg", lo, hi)] = True
    cons[M.boundary_mask(mesh, 0, "pos", lo, hi)] = True
    cons = np.concatenate([cons.ravel(), np.zeros(3 * mesh.num_lagrange, dtype=bool)])
    patches = GF.fault_patches(mesh, (-6000.0, 6000.0), (-9000.0, 0.0), 4, 2)
    out = {}
    for fused in ("1", "0"):
        monkeypatch.setenv("PYLITH_B200_BATCH_FUSED_PQ", fused)
        g = GF.GreensFunctions(ctx, mesh, mat, cons, patches, rtol=1e-11, inner_rtol=1e-4, tile=8)
        got, _ = g.solve(g.impulses[:8], batched=True)
        out[fused] = ([x.cpu().numpy() for x in got], g.batch.stats())
        if fused == "0":
            ref, _ = g.solve(g.impulses[:8], batched=False)
    for fused, (xs, st) in out.items():
        assert st["max_rel_residual"] <= 1e-11
        for a, b in zip(xs, ref):
            b = b.cpu().numpy()
            assert np.linalg.norm(a - b) <= 1e-8 * np.linalg.norm(b), fused
    i1, i0 = out["1"][1]["inner_iterations"], out["0"][1]["inner_iterations"]
    assert abs(i1 - i0) <= 0.05 * i0 + 20, (i1, i0)


def test_fp32_reliable_updates_and_restarted_refinement_match_the_oracle(ctx, oracle_lib):
    """The single-right-hand-side FP32 solver with reliable updates and with restarted iterative
    refinement both reach the FP64 tolerance on a heterogeneous tetrahedral problem and match
    scipy's direct solve of the oracle-assembled system to <= 1e-8; the reliable updates need no
    more FP32 iterations."""
    import torch
    from pylith_b200 import feassemble as FA

    O = oracle_lib
    mesh = M.box_tet_delaunay(8000, seed=4)
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=3)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    cons[M.boundary_mask(mesh, 0, "neg")] = True
    cons[M.boundary_mask(mesh, 0, "pos")] = True
    cons = cons.ravel()
    aux = O.AuxFields([(rho[:, None], "cell"), (mu[:, None], "cell"), (K[:, None], "cell")])
    J = O.assemble(mesh, O.jacobian_elements(mesh, aux, g3="IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain"))
    b = np.random.default_rng(9).standard_normal(3 * mesh.num_nodes) * (~cons)
    free = ~cons
    x_ref = np.zeros_like(b)
    x_ref[free] = spla.spsolve((-J)[free][:, free].tocsc(), b[free])
    dm = FA.DeviceMesh(ctx, mesh)
    ig = mat.create_integrator(dm)
    inner = {}
    for reliable in (True, False):
        S = FA.Solver(dm, cons, [ig], rtol=1e-11, precision=FA.Solver.FP32_REFINED, inner_rtol=1e-4,
                      reliable=reliable)
        S.setup()
        x = torch.zeros(dm.num_dof, dtype=torch.float64, device="cuda")
        S.solve(torch.from_numpy(b).cuda(), x)
        ctx.synchronize()
        st = S.stats()
        assert st["rel_residual"] <= 1e-11, (reliable, st)
        err = np.linalg.norm(x.cpu().numpy() - x_ref) / np.linalg.norm(x_ref)
        assert err <= 1e-8, (reliable, err, st)
        inner[reliable] = st["inner_iterations"]
        S.close()
    assert inner[True] <= inner[False], inner


def test_handles_can_be_destroyed_in_any_order():
    """Handles are reference-counted: closing the context, mesh and solver before the batched
    solver that uses them defers their release to the batched solver's destroy, which still solves
    and then frees everything (the order in which a garbage collector may run finalizers)."""
    import torch
    from pylith_b200 import feassemble as FA

    mesh = M.box_tet_kuhn(4, 4, 3, seed=2)
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=2)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    cons[M.boundary_mask(mesh, 0, "neg")] = True
    cons = cons.ravel()
    c = FA.Context(0)
    dm = FA.DeviceMesh(c, mesh)
    ig = mat.create_integrator(dm)
    S = FA.Solver(dm, cons, [ig], rtol=1e-10, precision=FA.Solver.FP32_REFINED, inner_rtol=1e-4)
    S.setup()
    B = FA.BatchSolver(S, 4)
    b = torch.from_numpy(np.random.default_rng(1).standard_normal(dm.num_dof) * ~cons).cuda()
    x0 = torch.zeros_like(b)
    B.solve([b], [x0])
    S.close()
    dm.close()
    c.close()
    x1 = torch.zeros_like(b)
    B.solve([b], [x1])
    torch.cuda.synchronize()
    assert float(torch.linalg.norm(x1 - x0)) <= 1e-8 * float(torch.linalg.norm(x0)) and float(torch.linalg.norm(x0)) > 0.0
    B.close()
    ig.close()


def test_fp32_hex_jacobian_action_uses_the_tangent_cached_by_solver_setup(ctx):
    """A FP32 solver's setup caches, per Q1 cell, the (lambda, mu) of the registered isotropic
    tangent; the FP32 Jacobian action then reads them instead of evaluating the generalized-
    Maxwell tangent (three exponentials of dt / tau) at every quadrature point. The cached action
    matches the per-point one, and new constants (the time step) or new aux values make the cache
    stale until the next setup."""
    import torch
    from pylith_b200 import feassemble as FA

    mesh = M.box_hex(6, 5, 4, lo=(-4000.0, -4000.0, -8000.0), hi=(4000.0, 4000.0, 0.0))
    mu, K, lam, tau = KA.genmaxwell_params()
    nc, nq = mesh.num_cells, 8
    rng = np.random.default_rng(5)
    g = MAT.IsotropicLinearGenMaxwell(
        np.full(nc, KA.GM_DENSITY), mu * rng.uniform(0.5, 1.5, nc), np.full(nc, K), np.tile(tau, (nc, 1)),
        np.tile(KA.GM_RATIO, (nc, 1)), np.zeros((nc, nq, 18)), np.zeros((nc, nq, 6)))
    dt = KA.GM_DT
    dm = FA.DeviceMesh(ctx, mesh)
    ig = g.create_integrator(dm, dt)
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    cons[M.boundary_mask(mesh, 2, "neg")] = True
    v = torch.from_numpy(rng.standard_normal(dm.num_dof).astype(np.float32)).cuda()

    def jv():
        out = torch.zeros_like(v)
        ig.compute_lhs_jacobian_action_f32(0.0, dt, v, out)
        torch.cuda.synchronize()
        return out.double()

    def close(a, b):
        return float(torch.linalg.norm(a - b)) <= 1e-6 * float(torch.linalg.norm(b))

    def setup():
        S = FA.Solver(dm, cons.ravel(), [ig], precision=FA.Solver.FP32_REFINED)
        S.setup(0.0, dt)
        return S

    ref = jv()  # no cache yet: the tangent at every point
    S1 = setup()
    assert close(jv(), ref)
    ig.set_constants([4.0 * dt])  # another time step: the cache is stale
    fresh = jv()
    assert not close(fresh, ref)
    S2 = setup()
    assert close(jv(), fresh)
    ig.set_aux("shear_modulus", FA.PER_CELL, np.full((nc, 1), 2.0 * mu))
    fresh2 = jv()
    assert not close(fresh2, fresh)
    S3 = setup()
    assert close(jv(), fresh2)
    # a new Jf3 kernel (here the elastic one, reading the same shear and bulk moduli) also makes
    # the cache stale: the action follows the new kernel at once, and again after the next setup
    ig.set_kernels_jacobian([FA.JacobianKernels(
        "displacement", "displacement", FA.LHS, None, None, None,
        FA.fekernels.IsotropicLinearElasticity3D.Jf3vu_infinitesimalStrain)])
    elastic = jv()
    assert not close(elastic, fresh2)
    S4 = setup()
    assert close(jv(), elastic)
    for S in (S1, S2, S3, S4):
        S.close()


@pytest.mark.parametrize("rheology", ["elastic", "genmaxwell"])
def test_fp32_tet_jacobian_action_with_the_cached_tangent(ctx, rheology):
    """P1 tetrahedra: after a FP32 solver's setup has cached each cell's (lambda, mu), the FP32
    Jacobian action (the padded cell-block kernel) reads them; it matches the action that
    evaluates the registered tangent per cell (<= 1e-6) and the FP64 action (<= 1e-5), for
    isotropic elasticity and for generalized Maxwell (whose per-cell tangent the cache makes
    available to the cell-block kernel)."""
    import torch
    from pylith_b200 import feassemble as FA

    mesh = M.box_tet_delaunay(60000, seed=6)
    nc = mesh.num_cells
    rng = np.random.default_rng(8)
    rho, mu, K = MAT.lognormal_elastic(nc, seed=9)
    dt = 0.0
    if rheology == "genmaxwell":
        mu_g, K_g, lam_g, tau = KA.genmaxwell_params()
        mat = MAT.IsotropicLinearGenMaxwell(
            np.full(nc, KA.GM_DENSITY), mu_g * rng.uniform(0.5, 1.5, nc), np.full(nc, K_g), np.tile(tau, (nc, 1)),
            np.tile(KA.GM_RATIO, (nc, 1)), np.zeros((nc, 1, 18)), np.zeros((nc, 1, 6)))
        dt = KA.GM_DT
    else:
        mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    dm = FA.DeviceMesh(ctx, mesh)
    ig = mat.create_integrator(dm, dt) if rheology == "genmaxwell" else mat.create_integrator(dm)
    v64 = torch.from_numpy(rng.standard_normal(dm.num_dof)).cuda()
    v = v64.float()

    def jv32():
        out = torch.zeros_like(v)
        ig.compute_lhs_jacobian_action_f32(0.0, dt, v, out)
        torch.cuda.synchronize()
        return out.double()

    per_cell = jv32()
    ref = torch.zeros_like(v64)
    ig.compute_lhs_jacobian_action(0.0, dt, 0.0, None, v.double(), ref)
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    cons[M.boundary_mask(mesh, 2, "neg")] = True
    S = FA.Solver(dm, cons.ravel(), [ig], precision=FA.Solver.FP32_REFINED)
    S.setup(0.0, dt)
    cached = jv32()
    rel = lambda a, b: float(torch.linalg.norm(a - b) / torch.linalg.norm(b))  # noqa: E731
    assert rel(cached, per_cell) <= 1e-6
    assert rel(cached, ref) <= 1e-5
    S.close()


@pytest.mark.parametrize("kind", ["tet", "hex"])
def test_reduced_fault_space_operator_matches_unfold_and_fold(ctx, monkeypatch, kind):
    """With faults, the solvers apply their operator in the reduced fault space directly (every
    positive-side node read as, and added into, its negative-side partner: no unfold and fold
    launches). FP64 and FP32-refined solves match the unfold-and-fold operator's to <= 1e-10 in
    about the same number of iterations."""
    from pylith_b200 import problems as P
    from pylith_b200 import feassemble as FA

    if kind == "tet":
        lo, hi = (-6000.0, -6000.0, -9000.0), (6000.0, 6000.0, 0.0)
        mesh = M.box_tet_delaunay_fault_x(40000, seed=5, lo=lo, hi=hi)
    else:
        lo, hi = M.BOX_LO, M.BOX_HI
        mesh = M.insert_fault_x(M.box_hex(12, 10, 8))
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=11)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    cons[M.boundary_mask(mesh, 0, "neg", lo, hi)] = True
    cons[M.boundary_mask(mesh, 0, "pos", lo, hi)] = True
    cons = np.concatenate([cons.ravel(), np.zeros(3 * mesh.num_lagrange, dtype=bool)])
    slip = np.zeros((mesh.num_lagrange, 3))
    slip[: mesh.num_lagrange // 2, 1] = 1.0
    out = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("PYLITH_B200_REDUCED_KERNELS", flag)
        for prec in (FA.Solver.FP64, FA.Solver.FP32_REFINED):
            prob = P.QuasistaticProblem(ctx, mesh, [(mat, None)], cons, np.zeros(mesh.num_dof),
                                        faults=[MAT.FaultCohesiveKin(slip)], precision=prec, rtol=1e-12)
            st = prob.step(0.0)
            out[(flag, prec)] = (prob.u.cpu().numpy(), st.iterations + st.inner_iterations)
            prob.close()
    for prec in (FA.Solver.FP64, FA.Solver.FP32_REFINED):
        (u1, i1), (u0, i0) = out[("1", prec)], out[("0", prec)]
        assert np.linalg.norm(u1 - u0) <= 1e-10 * np.linalg.norm(u0), prec
        assert abs(i1 - i0) <= 0.05 * i0 + 10, (prec, i1, i0)


def test_insert_constrained_sets_only_the_constrained_dofs(ctx):
    """pl_solver_insert_constrained: u takes the boundary values where the solver's mask is set
    and keeps every other entry (Lagrange-multiplier DOFs of a fault mesh included)."""
    import torch
    from pylith_b200 import feassemble as FA

    mesh = M.insert_fault_x(M.box_hex(4, 3, 3))
    dm = FA.DeviceMesh(ctx, mesh)
    mat = MAT.IsotropicLinearElasticity(*MAT.lognormal_elastic(mesh.num_cells, seed=1))
    ig = mat.create_integrator(dm)
    rng = np.random.default_rng(4)
    cons = rng.random(3 * mesh.num_nodes) < 0.3
    S = FA.Solver(dm, np.concatenate([cons, np.zeros(3 * mesh.num_lagrange, dtype=bool)]), [ig])
    u0 = rng.standard_normal(dm.num_dof)
    vals = rng.standard_normal(dm.num_dof)
    u = torch.from_numpy(u0.copy()).cuda()
    S.insert_constrained(torch.from_numpy(vals).cuda(), u)
    ctx.synchronize()
    got = u.cpu().numpy()
    want = u0.copy()
    want[:3 * mesh.num_nodes][cons] = vals[:3 * mesh.num_nodes][cons]
    assert np.array_equal(got, want)
    S.close()
