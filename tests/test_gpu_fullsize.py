"""Full-size checks (the headline's ~1.2 M-cell P1 size) through size-independent properties of
linear elasticity, where the oracle would take too long:
  * rigid-body motions (translation, infinitesimal rotation) give a zero residual;
  * F(u) = J u (the residual of isotropic linear elasticity is linear in u, F(u) = -K u);
  * linearity: F(a u + b w) = a F(u) + b F(w);
  * the deterministic cell-block scatter gives bit-identical reruns (shared nodes are summed
    over their blocks in block order by a second pass); the default scatter (FP64 reductions for
    shared nodes) reproduces itself to rounding; both agree with the thread-per-cell atomic
    kernel.
Relative tolerances are FP64 rounding levels (1e-12 of the residual scale)."""
import numpy as np
import pytest

from pylith_b200 import materials as MAT
from pylith_b200 import meshing as M

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


@pytest.fixture(scope="module")
def setup():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pylith_b200 import feassemble as FA

    mesh = M.box_tet_kuhn(56, 56, 64, seed=3)  # 1,204,224 tets, 211,185 nodes
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=4)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    ctx = FA.Context(0)
    dm = FA.DeviceMesh(ctx, mesh)
    ig = mat.create_integrator(dm)
    return torch, FA, ctx, dm, mesh, mat, ig


def _res(torch, ctx, ig, u):
    r = torch.empty_like(u)
    ig.compute_lhs_residual(0.0, 0.0, u, r)
    ctx.synchronize()
    return r


def test_rigid_motions_have_zero_residual(setup):
    torch, FA, ctx, dm, mesh, mat, ig = setup
    X = torch.from_numpy(mesh.coords).cuda()
    g = torch.Generator(device="cuda").manual_seed(5)
    scale = _res(torch, ctx, ig, torch.randn(mesh.num_dof, dtype=torch.float64, device="cuda", generator=g)).norm()
    t = torch.tensor([0.3, -1.1, 0.7], dtype=torch.float64, device="cuda")
    u_t = t.expand(mesh.num_nodes, 3).reshape(-1).contiguous()
    w = torch.tensor([2e-4, -1e-4, 3e-4], dtype=torch.float64, device="cuda")
    u_r = torch.linalg.cross(w.expand(mesh.num_nodes, 3), X).reshape(-1).contiguous()
    # scale of a residual of the same displacement size
    for u in (u_t, u_r):
        r = _res(torch, ctx, ig, u)
        ref = scale * u.norm() / np.sqrt(mesh.num_dof)
        assert float(r.norm()) <= 1e-10 * float(ref)


def test_residual_equals_jacobian_action_and_is_linear(setup):
    torch, FA, ctx, dm, mesh, mat, ig = setup
    g = torch.Generator(device="cuda").manual_seed(6)
    u = torch.randn(mesh.num_dof, dtype=torch.float64, device="cuda", generator=g)
    w = torch.randn(mesh.num_dof, dtype=torch.float64, device="cuda", generator=g)
    ru, rw = _res(torch, ctx, ig, u), _res(torch, ctx, ig, w)
    jv = torch.empty_like(u)
    ig.compute_lhs_jacobian_action(0.0, 0.0, 0.0, u, u, jv)
    ctx.synchronize()
    assert float((ru - jv).norm() / ru.norm()) <= TOL64
    a, b = 0.7, -2.3
    rab = _res(torch, ctx, ig, a * u + b * w)
    assert float((rab - (a * ru + b * rw)).norm() / rab.norm()) <= TOL64


def test_blocked_kernel_is_deterministic_and_matches_atomic(setup):
    torch, FA, ctx, dm, mesh, mat, ig = setup
    g = torch.Generator(device="cuda").manual_seed(7)
    u = torch.randn(mesh.num_dof, dtype=torch.float64, device="cuda", generator=g)
    idet = mat.create_integrator(dm)
    idet.set_scatter(FA.SCATTER_DETERMINISTIC)
    r1, r2 = _res(torch, ctx, idet, u), _res(torch, ctx, idet, u)
    assert torch.equal(r1, r2)
    jv1, jv2 = torch.empty_like(u), torch.empty_like(u)
    idet.compute_lhs_jacobian_action(0.0, 0.0, 0.0, u, u, jv1)
    idet.compute_lhs_jacobian_action(0.0, 0.0, 0.0, u, u, jv2)
    ctx.synchronize()
    assert torch.equal(jv1, jv2)
    # the default cell-block scatter reproduces itself to rounding
    rb1, rb2 = _res(torch, ctx, ig, u), _res(torch, ctx, ig, u)
    assert float((rb1 - r1).norm() / r1.norm()) <= TOL64
    assert float((rb1 - rb2).norm() / rb1.norm()) <= 1e-14
    ia = mat.create_integrator(dm)
    ia.set_scatter(FA.SCATTER_ATOMIC)
    ra = _res(torch, ctx, ia, u)
    assert float((ra - r1).norm() / r1.norm()) <= TOL64
