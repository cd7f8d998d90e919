"""Serving: requests of mixed sizes admitted by HBM budget into concurrent device slots; each
result is the same alone and in the mix and matches the FP64 one-at-a-time path (relative
displacement difference <= 1e-8, with solves converged to a relative residual of 1e-12)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_results_same_alone_and_in_the_mix(cuda):
    from pylith_b200 import serving as SV

    reqs = SV.poisson_requests(10, rate=200.0, seed=4, n_min=4, n_max=12)
    server = SV.Server(slots=4, keep_solutions=True, rtol=1e-12)
    mixed = server.run(reqs)
    alone = [SV.Server(slots=1, keep_solutions=True, rtol=1e-12).run([r])[0] for r in reqs[:4]]
    seq = SV.serve_sequential(reqs, keep_solutions=True, rtol=1e-12)
    by_id = {r.rid: r for r in mixed}
    for a in alone:
        m = by_id[a.rid]
        assert np.linalg.norm(m.u - a.u) <= 1e-8 * np.linalg.norm(a.u)
    for s in seq:
        m = by_id[s.rid]
        assert np.linalg.norm(m.u - s.u) <= 1e-8 * np.linalg.norm(s.u)
    summ = SV.summarize(mixed)
    assert summ["requests"] == 10 and summ["p99_latency_s"] >= summ["p50_latency_s"]


def test_admission_respects_the_hbm_budget(cuda):
    from pylith_b200 import serving as SV

    reqs = SV.poisson_requests(3, rate=1000.0, seed=1, n_min=4, n_max=6)
    budget = max(SV.estimate_bytes(r.n) for r in reqs)
    # a budget that fits one request at a time serialises them, and still completes them all
    res = SV.Server(slots=3, hbm_budget=budget).run(reqs)
    starts = sorted((r.start, r.end) for r in res)
    for (s0, e0), (s1, e1) in zip(starts, starts[1:]):
        assert s1 >= e0 - 1e-3
    with pytest.raises(ValueError):
        SV.Server(slots=1, hbm_budget=budget // 4).run(reqs)
