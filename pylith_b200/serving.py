"""Serving forward solves: a request loop with HBM-budget admission and continuous batching.

Each request is a quasi-static forward solve (the same path as problems.QuasistaticProblem) on its
own box mesh with a prescribed-slip fault. A request is admitted when it has arrived, a slot is free
and its estimated device memory fits the remaining HBM budget; its mesh, aux fields and solver are
then built on the device. Small boxes join one ragged batch (pl_ragged_*) at the next iteration
boundary: every PCG iteration of every request in it shares the same launches (one operator launch
over all their cells), each request converging on its own dot products, and a request leaves the
batch when its FP64 residual meets the tolerance. Large boxes (with a multigrid hierarchy) are solved
beside the batch, on a second stream, with FP32 V-cycles under FP64 conjugate gradients. A finished
request's slot and memory go to the next arrival. Latency is measured from arrival to completion.

Host mesh generation is not part of serving: the requests' host-side problem data (mesh, material
fields, slip, constraints) is prepared before the request stream starts, for the server and the
baseline alike. The baseline is the same stream served one at a time with the FP64 solver.
"""
from __future__ import annotations

import time
from dataclasses import dataclass
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


@dataclass
class HostProblem:
    """A request's host-side data, prepared before the request stream starts."""
    req: Request
    mesh: object
    rho: np.ndarray
    mu: np.ndarray
    K: np.ndarray
    slip: np.ndarray
    constrained: np.ndarray
    bc: np.ndarray
    levels: Optional[list] = None  # multigrid hierarchy (pylith_b200.multigrid) for large boxes


MULTIGRID_MIN_N = 32


def prepare(req: Request, multigrid_min_n: int = MULTIGRID_MIN_N) -> HostProblem:
    """Host-side problem data; boxes of at least multigrid_min_n cells per side also get their
    multigrid hierarchy (meshes, constraint masks and prolongations of every level)."""
    from . import multigrid as MGH

    lo, hi = M.BOX_LO, M.BOX_HI
    levels = None
    if req.n >= multigrid_min_n:
        levels = MGH.build_hierarchy(req.n, req.n, req.n, fault_x=0.0,
                                     constrained_faces=[(0, "neg", (0, 1, 2)), (0, "pos", (0, 1, 2))])
        if len(levels) < 3:
            levels = None
    mesh = levels[0].mesh if levels else M.insert_fault_x(M.box_hex(req.n, req.n, req.n))
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=req.seed)
    lag_nodes = np.zeros(mesh.num_lagrange, dtype=np.int64)
    lag_nodes[mesh.cohesive[:, 8:].ravel()] = mesh.cohesive[:, :4].ravel()
    yz = mesh.coords[lag_nodes][:, 1:]
    fy = (yz[:, 0] - lo[1]) / (hi[1] - lo[1])
    fz = (yz[:, 1] - lo[2]) / (hi[2] - lo[2])
    y0, y1, z0, z1 = req.patch
    on = (fy >= y0) & (fy <= y1) & (fz >= z0) & (fz <= z1)
    slip = np.zeros((mesh.num_lagrange, 3))
    slip[on, 1] = req.slip
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    cons[M.boundary_mask(mesh, 0, "neg")] = True
    cons[M.boundary_mask(mesh, 0, "pos")] = True
    cons = np.concatenate([cons.ravel(), np.zeros(3 * mesh.num_lagrange, dtype=bool)])
    return HostProblem(req, mesh, rho, mu, K, slip, cons, np.zeros(mesh.num_dof), levels)


def build_problem(ctx, hp: HostProblem, precision: int, rtol: float, multigrid: Optional[int] = None):
    """The request's device problem; with `multigrid` (a precision) and a hierarchy, its solver is
    preconditioned by V-cycles of that precision (the problem keeps the hierarchy alive)."""
    from . import multigrid as MGH
    from . import problems as P

    mat = MAT.IsotropicLinearElasticity(hp.rho, hp.mu, hp.K)
    prob = P.QuasistaticProblem(ctx, hp.mesh, [(mat, None)], hp.constrained, hp.bc,
                                faults=[MAT.FaultCohesiveKin(hp.slip)], precision=precision, rtol=rtol)
    prob.multigrid = None
    if multigrid is not None and hp.levels is not None:
        prob.multigrid = MGH.attach(ctx, prob.solver, hp.levels, mat, fault_x=0.0, precision=multigrid)
    return prob


def close_problem(prob) -> None:
    if getattr(prob, "multigrid", None) is not None:
        prob.multigrid.close()
    prob.close()


class Server:
    """Serving loop: an admission thread (arrival times, slots, HBM budget) and device workers, each
    with its own stream: the batch worker keeps one ragged batch (pl_ragged_*) of FP32-refined
    solves that requests join and leave between iteration chunks; multigrid_workers workers take
    the large boxes that have a multigrid hierarchy from one queue and solve each with FP32
    V-cycles under FP64 conjugate gradients (their solves overlap on the device)."""

    def __init__(self, device: int = 0, slots: int = 64, hbm_budget: Optional[int] = None, rtol: float = 1e-10,
                 keep_solutions=False, chunk: int = 10, multigrid: bool = True, multigrid_workers: int = 3):
        import torch

        self.device = device
        self.slots = slots
        free, total = torch.cuda.mem_get_info(device)
        self.budget = hbm_budget if hbm_budget is not None else int(0.8 * free)
        self.rtol = rtol
        self.keep = keep_solutions
        self.chunk = chunk
        self.multigrid = multigrid
        self.multigrid_workers = max(1, multigrid_workers)
        self.memory = []  # (request, predicted bytes, measured bytes)
        self.routes = {}  # request -> "batch" or "multigrid"
        self.workers = {}  # worker -> {"requests", "busy_s", "last_end_s"}

    def run(self, problems: List[HostProblem]) -> List[Result]:
        import queue
        import threading

        import torch

        self.workers = {}
        pending = sorted(problems, key=lambda hp: hp.req.arrival)
        for hp in pending:
            if estimate_bytes(hp.req.n) > self.budget:
                raise ValueError(f"request {hp.req.rid} ({hp.req.n}^3) exceeds the HBM budget")
        lock = threading.Lock()
        freed = threading.Condition(lock)
        state = {"used": 0, "busy": 0}
        results: List[Result] = []
        errors = []
        self.memory = []
        q_batch, q_mg = queue.Queue(), queue.Queue()
        t0 = time.perf_counter()

        def account(worker, t_begin):
            now = time.perf_counter() - t0
            with lock:
                w = self.workers.setdefault(worker, {"requests": 0, "busy_s": 0.0, "last_end_s": 0.0})
                w["requests"] += 1
                w["busy_s"] += now - t_begin
                w["last_end_s"] = max(w["last_end_s"], now)

        def finish(hp, prob, start, its, nbytes):
            end = time.perf_counter() - t0
            u = prob.u.cpu().numpy() if self.keep and prob.u is not None else None
            with lock:
                results.append(Result(hp.req.rid, hp.req.n, prob.dmesh.num_dof, hp.req.arrival, start, end, its, u))
                state["used"] -= nbytes
                state["busy"] -= 1
                freed.notify_all()

        def batch_worker():
            torch.cuda.set_device(self.device)
            stream = torch.cuda.Stream(device=self.device)
            ctx = FA.Context(self.device, use_torch_stream=False)
            ctx.set_stream(stream.cuda_stream)
            batch = FA.RaggedBatch(ctx, capacity=self.slots, chunk=self.chunk)
            active = {}
            done = False
            with torch.cuda.stream(stream):
                while not done or active:
                    while True:  # join the batch at this iteration boundary
                        try:
                            item = q_batch.get(block=not active and not done, timeout=0.05)
                        except queue.Empty:
                            break
                        if item is None:
                            done = True
                            break
                        hp, nbytes, start = item
                        try:
                            free0 = torch.cuda.mem_get_info(self.device)[0]
                            prob = build_problem(ctx, hp, FA.Solver.FP32_REFINED, self.rtol)
                            F, du = prob.begin_step(0.0)
                            member = batch.add(prob.solver, F, du)
                            self.memory.append((hp.req.rid, nbytes, free0 - torch.cuda.mem_get_info(self.device)[0]))
                            active[member] = (hp, prob, start, nbytes)
                        except Exception as e:
                            errors.append((hp.req.rid, repr(e)))
                            finish(hp, _Null(), start, 0, nbytes)
                    if not active:
                        continue
                    batch.iterate()
                    for member in list(active):
                        st = batch.status(member)
                        if not st["done"]:
                            continue
                        hp, prob, start, nbytes = active.pop(member)
                        if st["status"] != 0:
                            errors.append((hp.req.rid, C_error(st["status"])))
                        prob.end_step(0.0)
                        stream.synchronize()
                        finish(hp, prob, start, st["iterations"], nbytes)
                        batch.remove(member)
                        close_problem(prob)
                        account("batch", start)
            batch.close()
            ctx.close()

        def multigrid_worker(name):
            torch.cuda.set_device(self.device)
            stream = torch.cuda.Stream(device=self.device)
            ctx = FA.Context(self.device, use_torch_stream=False)
            ctx.set_stream(stream.cuda_stream)
            with torch.cuda.stream(stream):
                while True:
                    item = q_mg.get()
                    if item is None:
                        break
                    hp, nbytes, start = item
                    t_begin = time.perf_counter() - t0
                    try:
                        prob = build_problem(ctx, hp, FA.Solver.FP64, self.rtol, multigrid=FA.Solver.FP32_REFINED)
                        st = prob.step(0.0)
                        stream.synchronize()
                        finish(hp, prob, start, st.iterations, nbytes)
                        close_problem(prob)
                    except Exception as e:
                        errors.append((hp.req.rid, repr(e)))
                        finish(hp, _Null(), start, 0, nbytes)
                    account(name, t_begin)
            ctx.close()

        mg_names = [f"multigrid{i}" for i in range(self.multigrid_workers)]
        workers = [threading.Thread(target=batch_worker, daemon=True)]
        workers += [threading.Thread(target=multigrid_worker, args=(nm,), daemon=True) for nm in mg_names]
        for w in workers:
            w.start()
        for hp in pending:
            nbytes = estimate_bytes(hp.req.n)
            wait = hp.req.arrival - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
            with lock:
                while state["busy"] >= self.slots or state["used"] + nbytes > self.budget:
                    freed.wait()
                state["used"] += nbytes
                state["busy"] += 1
            start = time.perf_counter() - t0
            route = "multigrid" if self.multigrid and hp.levels is not None else "batch"
            self.routes[hp.req.rid] = route
            (q_mg if route == "multigrid" else q_batch).put((hp, nbytes, start))
        q_batch.put(None)
        for _ in mg_names:
            q_mg.put(None)
        for w in workers:
            w.join()
        if errors:
            raise RuntimeError(f"requests failed: {errors[:3]}")
        return sorted(results, key=lambda r: r.rid)


class _Null:
    """Stand-in for a problem that failed to build (its request is reported as an error)."""
    u = None

    class dmesh:
        num_dof = 0


def C_error(code: int) -> str:
    from . import _lib as C

    return C.ERRORS.get(code, str(code))


def serve_sequential(problems: List[HostProblem], device: int = 0, precision: int = FA.Solver.FP64,
                     rtol: float = 1e-10, keep_solutions=False, multigrid: Optional[int] = None) -> List[Result]:
    """The baseline: requests in arrival order, one at a time, each with its own solver (point-block
    Jacobi PCG; with `multigrid`, V-cycles of that precision where a hierarchy exists)."""
    import torch

    torch.cuda.set_device(device)
    ctx = FA.Context(device)
    t0 = time.perf_counter()
    out = []
    for hp in sorted(problems, key=lambda hp: hp.req.arrival):
        wait = hp.req.arrival - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        start = time.perf_counter() - t0
        prob = build_problem(ctx, hp, precision, rtol, multigrid=multigrid)
        st = prob.step(0.0)
        ctx.synchronize()
        u = prob.u.cpu().numpy() if keep_solutions else None
        out.append(Result(hp.req.rid, hp.req.n, prob.dmesh.num_dof, hp.req.arrival, start,
                          time.perf_counter() - t0, st.iterations + st.inner_iterations, u))
        close_problem(prob)
    ctx.close()
    return out


def summarize(results: List[Result]):
    lat = np.array([r.latency for r in results])
    span = max(r.end for r in results) - min(r.arrival for r in results)
    return {"requests": len(results), "solves_per_s": len(results) / span,
            "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
            "dof_total": int(sum(r.dof for r in results))}
