"""Serving forward solves: a request loop with HBM-budget admission and concurrent device slots.

Each request is a quasi-static forward solve (the same path as problems.QuasistaticProblem) on
its own box mesh with a prescribed-slip fault. The server admits a request when it has arrived,
a slot is free and the request's estimated device memory fits the remaining HBM budget; every
slot has its own CUDA stream and host thread, so requests that arrive while others run are
started at once and their kernels overlap on the GPU. Meshes, aux fields and solver state live on
the device for the life of the request. Latency is measured from arrival to completion.

The baseline is the same stream of requests served one at a time with the FP64 solver.
"""
from __future__ import annotations

import heapq
import queue
import threading
import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import feassemble as FA
from . import materials as MAT
from . import meshing as M


@dataclass
class Request:
    rid: int
    n: int                  # n^3 Q1 hexahedra
    seed: int
    arrival: float          # seconds after the stream starts
    slip: float             # m, left-lateral
    patch: tuple            # (y0, y1, z0, z1) fraction of the fault plane


@dataclass
class Result:
    rid: int
    n: int
    dof: int
    arrival: float
    start: float
    end: float
    iterations: int
    u: Optional[np.ndarray] = None

    @property
    def latency(self) -> float:
        return self.end - self.arrival


def poisson_requests(count: int, rate: float, seed: int = 0, n_min: int = 8, n_max: int = 96):
    """Poisson arrivals (mean `rate` per second); mesh size log-uniform in [n_min, n_max];
    slip 0.1-3 m on a random rectangle of the fault plane."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        n = int(round(np.exp(rng.uniform(np.log(n_min), np.log(n_max)))))
        n = max(2, n + (n % 2))  # even, so the fault plane x = 0 is a grid plane
        y0, y1 = np.sort(rng.uniform(0.0, 1.0, 2))
        z0, z1 = np.sort(rng.uniform(0.0, 1.0, 2))
        out.append(Request(i, n, int(rng.integers(1 << 30)), t, float(rng.uniform(0.1, 3.0)),
                           (y0, max(y1, y0 + 0.1), z0, max(z1, z0 + 0.1))))
    return out


def estimate_bytes(n: int) -> int:
    """Device memory of one request: mesh, aux, integrators and solver vectors."""
    cells = n ** 3
    nodes = (n + 1) ** 3 + (n + 1) ** 2
    return cells * (32 + 40) + nodes * 3 * 8 * 24 + (64 << 20)


def build_problem(ctx, req: Request, precision: int, rtol: float):
    from . import problems as P

    lo, hi = M.BOX_LO, M.BOX_HI
    mesh = M.insert_fault_x(M.box_hex(req.n, req.n, req.n))
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=req.seed)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    lag_nodes = np.zeros(mesh.num_lagrange, dtype=np.int64)
    lag_nodes[mesh.cohesive[:, 8:].ravel()] = mesh.cohesive[:, :4].ravel()
    yz = mesh.coords[lag_nodes][:, 1:]
    fy = (yz[:, 0] - lo[1]) / (hi[1] - lo[1])
    fz = (yz[:, 1] - lo[2]) / (hi[2] - lo[2])
    y0, y1, z0, z1 = req.patch
    on = (fy >= y0) & (fy <= y1) & (fz >= z0) & (fz <= z1)
    slip = np.zeros((mesh.num_lagrange, 3))
    slip[on, 1] = req.slip
    fault = MAT.FaultCohesiveKin(slip)
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    cons[M.boundary_mask(mesh, 0, "neg")] = True
    cons[M.boundary_mask(mesh, 0, "pos")] = True
    cons = np.concatenate([cons.ravel(), np.zeros(3 * mesh.num_lagrange, dtype=bool)])
    bc = np.zeros(mesh.num_dof)
    return P.QuasistaticProblem(ctx, mesh, [(mat, None)], cons, bc, faults=[fault], precision=precision,
                                rtol=rtol)


def solve_one(ctx, req: Request, precision: int, rtol: float, keep_solution: bool):
    prob = build_problem(ctx, req, precision, rtol)
    st = prob.step(0.0)
    ctx.synchronize()
    u = prob.u.cpu().numpy() if keep_solution else None
    return prob.dmesh.num_dof, st.iterations + st.inner_iterations, u


class Server:
    def __init__(self, device: int = 0, slots: int = 8, hbm_budget: Optional[int] = None,
                 precision: int = FA.Solver.FP32_REFINED, rtol: float = 1e-10, keep_solutions=False):
        import torch

        self.device = device
        self.slots = slots
        free, total = torch.cuda.mem_get_info(device)
        self.budget = hbm_budget if hbm_budget is not None else int(0.8 * free)
        self.precision = precision
        self.rtol = rtol
        self.keep = keep_solutions

    def run(self, requests: List[Request]) -> List[Result]:
        import torch

        pending = sorted(requests, key=lambda r: r.arrival)
        work = queue.Queue()
        results: List[Result] = []
        lock = threading.Lock()
        freed = threading.Condition(lock)
        state = {"used": 0, "busy": 0}
        t0 = time.perf_counter()
        errors = []

        def worker():
            torch.cuda.set_device(self.device)
            stream = torch.cuda.Stream(device=self.device)
            ctx = FA.Context(self.device, use_torch_stream=False)
            ctx.set_stream(stream.cuda_stream)
            with torch.cuda.stream(stream):
                while True:
                    item = work.get()
                    if item is None:
                        break
                    req, nbytes = item
                    start = time.perf_counter() - t0
                    try:
                        dof, iters, u = solve_one(ctx, req, self.precision, self.rtol, self.keep)
                    except Exception as e:  # surfaced after the run
                        errors.append((req.rid, repr(e)))
                        dof, iters, u = 0, 0, None
                    end = time.perf_counter() - t0
                    with lock:
                        results.append(Result(req.rid, req.n, dof, req.arrival, start, end, iters, u))
                        state["used"] -= nbytes
                        state["busy"] -= 1
                        freed.notify_all()
            ctx.close()

        threads = [threading.Thread(target=worker, daemon=True) for _ in range(self.slots)]
        for th in threads:
            th.start()
        for req in pending:
            nbytes = estimate_bytes(req.n)
            if nbytes > self.budget:
                raise ValueError(f"request {req.rid} ({req.n}^3) exceeds the HBM budget")
            wait = req.arrival - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
            with lock:
                while state["busy"] >= self.slots or state["used"] + nbytes > self.budget:
                    freed.wait()
                state["used"] += nbytes
                state["busy"] += 1
            work.put((req, nbytes))
        for _ in threads:
            work.put(None)
        for th in threads:
            th.join()
        if errors:
            raise RuntimeError(f"requests failed: {errors[:3]}")
        return sorted(results, key=lambda r: r.rid)


def serve_sequential(requests: List[Request], device: int = 0, precision: int = FA.Solver.FP64,
                     rtol: float = 1e-10, keep_solutions=False) -> List[Result]:
    """The baseline: requests in arrival order, one at a time, on one stream."""
    import torch

    torch.cuda.set_device(device)
    ctx = FA.Context(device)
    t0 = time.perf_counter()
    out = []
    for req in sorted(requests, key=lambda r: r.arrival):
        wait = req.arrival - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        start = time.perf_counter() - t0
        dof, iters, u = solve_one(ctx, req, precision, rtol, keep_solutions)
        out.append(Result(req.rid, req.n, dof, req.arrival, start, time.perf_counter() - t0, iters, u))
    return out


def summarize(results: List[Result]):
    lat = np.array([r.latency for r in results])
    span = max(r.end for r in results) - min(r.arrival for r in results)
    return {"requests": len(results), "solves_per_s": len(results) / span,
            "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
            "dof_total": int(sum(r.dof for r in results))}
