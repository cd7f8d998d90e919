"""Ragged batches and serving: many meshes of uneven size solved together (pl_ragged_*), every
PCG iteration of every member in the same launches with per-member dot products. Each result is
the same alone and in the mix and matches the FP64 one-at-a-time path (relative displacement
difference <= 1e-8, with solves converged to a relative residual of 1e-12); the launches of an
iteration do not grow with the number of members; admission respects the HBM budget."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_ragged_batch_matches_single_solves(cuda):
    """Three fault problems of 4^3, 6^3 and 10^3 cells in one ragged batch against each solved
    alone by pl_solver_solve (FP32 refined) and by the FP64 solver."""
    torch = cuda
    from pylith_b200 import _lib
    from pylith_b200 import feassemble as FA
    from pylith_b200 import serving as SV

    reqs = [SV.Request(i, n, 100 + i, 0.0, 1.0 + i, (0.1, 0.8, 0.2, 0.9)) for i, n in enumerate((4, 6, 10))]
    hps = [SV.prepare(r) for r in reqs]
    ctx = FA.Context(0)
    solo = {}
    for prec in (FA.Solver.FP64, FA.Solver.FP32_REFINED):
        for hp in hps:
            prob = SV.build_problem(ctx, hp, prec, 1e-12)
            prob.step(0.0)
            solo[(prec, hp.req.rid)] = prob.u.cpu().numpy()
            prob.close()
    batch = FA.RaggedBatch(ctx, capacity=8, chunk=5)
    probs, members = [], []
    for hp in hps:
        prob = SV.build_problem(ctx, hp, FA.Solver.FP32_REFINED, 1e-12)
        F, du = prob.begin_step(0.0)
        members.append(batch.add(prob.solver, F, du))
        probs.append(prob)
    # one chunk of 5 iterations for three members is one graph of 8 launches per iteration (plus a
    # few launches per member for any residual replacement), not 8 per member per iteration
    l0 = _lib.lib().pl_kernel_launches()
    left = batch.iterate()
    assert 8 * 5 <= _lib.lib().pl_kernel_launches() - l0 < 3 * 8 * 5 and left == 3
    while left:
        left = batch.iterate()
    for hp, prob, m in zip(hps, probs, members):
        st = batch.status(m)
        assert st["done"] and st["status"] == 0 and st["rel_residual"] <= 1e-12
        prob.end_step(0.0)
        u = prob.u.cpu().numpy()
        assert _rel(u, solo[(FA.Solver.FP32_REFINED, hp.req.rid)]) <= 1e-8
        assert _rel(u, solo[(FA.Solver.FP64, hp.req.rid)]) <= 1e-8
        batch.remove(m)
        prob.close()
    batch.close()


def test_results_same_alone_and_in_the_mix(cuda):
    from pylith_b200 import serving as SV

    reqs = SV.poisson_requests(10, rate=200.0, seed=4, n_min=4, n_max=12)
    hps = [SV.prepare(r) for r in reqs]
    server = SV.Server(slots=4, keep_solutions=True, rtol=1e-12)
    mixed = server.run(hps)
    alone = [SV.Server(slots=1, keep_solutions=True, rtol=1e-12).run([hp])[0] for hp in hps[:4]]
    seq = SV.serve_sequential(hps, keep_solutions=True, rtol=1e-12)
    by_id = {r.rid: r for r in mixed}
    for a in alone:
        m = by_id[a.rid]
        assert np.linalg.norm(m.u - a.u) <= 1e-8 * np.linalg.norm(a.u)
    for s in seq:
        m = by_id[s.rid]
        assert np.linalg.norm(m.u - s.u) <= 1e-8 * np.linalg.norm(s.u)
    summ = SV.summarize(mixed)
    assert summ["requests"] == 10 and summ["p99_latency_s"] >= summ["p50_latency_s"]
    # requests overlapped in the batch: some started before an earlier one had finished
    spans = sorted((r.start, r.end) for r in mixed)
    assert any(s1 < e0 for (s0, e0), (s1, e1) in zip(spans, spans[1:]))


def test_admission_respects_the_hbm_budget(cuda):
    from pylith_b200 import serving as SV

    reqs = SV.poisson_requests(3, rate=1000.0, seed=1, n_min=4, n_max=6)
    hps = [SV.prepare(r) for r in reqs]
    budget = max(SV.estimate_bytes(r.n) for r in reqs)
    # a budget that fits one request at a time serialises them, and still completes them all
    res = SV.Server(slots=3, hbm_budget=budget).run(hps)
    starts = sorted((r.start, r.end) for r in res)
    for (s0, e0), (s1, e1) in zip(starts, starts[1:]):
        assert s1 >= e0 - 1e-3
    with pytest.raises(ValueError):
        SV.Server(slots=1, hbm_budget=budget // 4).run(hps)


def test_large_boxes_take_the_multigrid_route(cuda):
    """Boxes of 32^3 cells and more (with a multigrid hierarchy, nested or not: 34 coarsens to 16) are solved beside the ragged batch
    with FP32 V-cycles under FP64 CG; their results, and the batched small ones', match the plain
    FP64 one-at-a-time path."""
    from pylith_b200 import serving as SV

    reqs = [SV.Request(0, 32, 11, 0.0, 1.5, (0.1, 0.9, 0.2, 0.7)), SV.Request(1, 8, 12, 0.001, 0.7, (0.3, 0.6, 0.1, 0.9)),
            SV.Request(2, 34, 13, 0.002, 2.0, (0.0, 0.5, 0.5, 1.0)), SV.Request(3, 10, 14, 0.003, 1.0, (0.2, 0.8, 0.2, 0.8))]
    hps = [SV.prepare(r) for r in reqs]
    assert [hp.levels is not None for hp in hps] == [True, False, True, False]
    server = SV.Server(slots=4, keep_solutions=True, rtol=1e-12)
    served = {r.rid: r for r in server.run(hps)}
    assert server.routes == {0: "multigrid", 1: "batch", 2: "multigrid", 3: "batch"}
    for s in SV.serve_sequential(hps, keep_solutions=True, rtol=1e-12):
        m = served[s.rid]
        assert np.linalg.norm(m.u - s.u) <= 1e-8 * np.linalg.norm(s.u), s.rid
