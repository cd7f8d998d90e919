"""Benchmark: FP64 residual + matrix-free Jacobian action (GDOF/s) of 3-D quasi-static isotropic
linear elasticity on an unstructured P1 tetrahedral box mesh of ~1.2 M cells (Delaunay of seeded
uniform-random interior points plus a jittered regular boundary grid, box [-6,6]x[-6,6]x[-9,0] km,
per-cell log-normal Vs with median 3000 m/s and sigma_log 0.2, Vp = sqrt(3) Vs, density 2700
kg/m^3 +-5%).

One step = one residual F(u) and one Jacobian action J v, each over the whole mesh
(2 applications x N_dof). value = 2 * N_dof * steps / (device time of the applications).
The L2 cache (126 MB) is flushed before every application (a 256 MiB write, then a 256 MiB read
of a second buffer that writes the flush's dirty lines back), because the application's working
set (~53 MB) would otherwise stay cached between applications.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl pylith_b200|reference]
  python bench.py --config c0|c1link|c1q2|c2|c3|c3tile|c3mg|c3bmg|c4  (the other configurations, one JSON line each)

Under torchrun (N > 1) the ranks share one mesh of N x 1.2 M cells (the same Delaunay box
stretched N times along x, so every rank's part is the single-GPU workload: weak scaling), cut into
N contiguous ranges of its Morton order. Every application on every rank computes its part's
residual (or J v) and sums the shared nodes with its neighbours: one pack kernel, NCCL send/receive
per neighbour, one add kernel (the DMLocalToGlobal ADD_VALUES step of the reference). The slowest
rank's device time defines the step time; value counts the global mesh's DOFs.
"""
from __future__ import annotations

import argparse
import json
import os
import platform
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

TARGET_CELLS = 1_200_000
METRIC = "GDOF/s residual+Jv (FP64), % of HBM roofline"
UNIT = "GDOF/s"
L2_FLUSH_BYTES = 256 << 20


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def _mesh_path(cells: int, seed: int, stretch: int = 1):
    cache = os.path.join(tempfile.gettempdir(), "pylith_b200_mesh_cache")
    os.makedirs(cache, exist_ok=True)
    tag = f"tet_{cells}_{seed}_v1" if stretch == 1 else f"tet_{cells}_{seed}_x{stretch}_v1"
    return os.path.join(cache, tag + ".npz")


class L2Flush:
    """Leaves the L2 cache holding none of the next application's data and no dirty lines: a
    256 MiB write (larger than the 126 MB L2), then a 256 MiB read of a second buffer, which
    writes the first one's dirty lines back to HBM before the timed region starts (otherwise the
    timed application pays for writing back up to 126 MB of flush data it never touched)."""

    def __init__(self):
        import torch

        self.write = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
        self.read = torch.zeros(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def __call__(self):
        self.write.zero_()
        self.read.sum()


def load_mesh(cells: int, seed: int, stretch: int = 1, build: bool = True):
    """The seeded benchmark mesh, cached under the temp directory between processes. stretch > 1:
    the box [-6, -6 + 12 stretch] x [-6, 6] x [-9, 0] km with `cells` tetrahedra (the multi-GPU
    mesh). With build=False, waits for another process to write the cache."""
    from pylith_b200 import meshing as M

    path = _mesh_path(cells, seed, stretch)
    if not build:
        t0 = time.time()
        while not os.path.exists(path):
            if time.time() - t0 > 1800:
                raise TimeoutError(f"{path} was not written")
            time.sleep(1.0)
    if os.path.exists(path):
        d = np.load(path)
        return M.Mesh(M.CELL_TET4, d["coords"], d["cells"])
    t0 = time.time()
    if stretch == 1:
        mesh = M.box_tet_delaunay(cells, seed=seed)
    else:
        lo, hi = M.BOX_LO, M.BOX_HI
        mesh = M.box_tet_delaunay(cells, seed=seed, lo=lo, hi=(lo[0] + stretch * (hi[0] - lo[0]), hi[1], hi[2]))
    log(f"mesh: {mesh.num_cells} tets, {mesh.num_nodes} nodes in {time.time() - t0:.1f} s")
    tmp = path + f".{os.getpid()}.tmp.npz"
    np.savez(tmp, coords=mesh.coords, cells=mesh.cells)
    os.replace(tmp, path)
    return mesh


def algorithmic_bytes(mesh) -> int:
    """Unique HBM bytes of one application with perfect on-chip reuse: connectivity (4 int32)
    and material (mu, K as FP64) per cell; coordinates, input and output (3 FP64 each) per node."""
    return mesh.num_cells * (16 + 16) + mesh.num_nodes * (24 + 24 + 24)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.out, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.out.flush()
        rows = []
        with open(self.out.name) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _profile_summary():
    path = os.path.join(ROOT, "profiles", "tet4_residual_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f)


def profiled_traffic(mesh):
    """DRAM bytes per residual launch from the committed ncu summary, scaled to this mesh."""
    d = _profile_summary()
    return None if d is None else float(d["dram_bytes_per_cell"]) * mesh.num_cells


def issue_limiter(mesh, seconds_per_launch, sm_mhz):
    """What bounds the residual kernel below the HBM roofline: the instruction-issue and FP64
    floors from the committed ncu warp-instruction counts (per cell, scaled to this mesh), at the
    clock sampled during the timed region. One warp-instruction per scheduler per cycle (4 per
    SM); an FP64 warp-instruction holds a scheduler's FP64 pipe for 2 cycles (64 FP64 lanes per
    SM)."""
    d = _profile_summary()
    if d is None or "warp_instructions_per_cell" not in d:
        return None
    import torch

    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    slots = 4 * sms * (sm_mhz or 1965.0) * 1e6
    t_issue = float(d["warp_instructions_per_cell"]) * mesh.num_cells / slots
    t_fp64 = 2.0 * float(d["fp64_warp_instructions_per_cell"]) * mesh.num_cells / slots
    return {"kind": "instruction issue and latency (FP64 arithmetic, shared-memory gather), not HBM",
            "issue_floor_us": t_issue * 1e6, "issue_frac": t_issue / seconds_per_launch,
            "fp64_floor_us": t_fp64 * 1e6, "fp64_frac": t_fp64 / seconds_per_launch,
            "warp_instructions_per_cell": d["warp_instructions_per_cell"],
            "source": "ncu warp-instruction counts of the same kernel (profiles/tet4_residual_traffic.json)"}


def host_cpu():
    """The host processor's model name and its logical cores (from /proc/cpuinfo)."""
    model = platform.processor() or "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": model, "logical_cores": os.cpu_count() or 1,
            "affinity_cores": len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else None}


def cudart():
    """The CUDA runtime library this process already uses (torch's), through ctypes."""
    import ctypes

    path = None
    try:
        with open("/proc/self/maps") as f:
            for ln in f:
                if "libcudart.so" in ln:
                    path = ln.split()[-1]
                    break
    except OSError:
        pass
    lib = ctypes.CDLL(path or "libcudart.so.12")
    P, I, S = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t
    lib.cudaMemcpyAsync.argtypes = [P, P, S, I, P]
    lib.cudaEventRecord.argtypes = [P, P]
    lib.cudaStreamWaitEvent.argtypes = [P, P, ctypes.c_uint]
    lib.cudaEventCreateWithFlags.argtypes = [ctypes.POINTER(P), ctypes.c_uint]
    lib.cudaEventDestroy.argtypes = [P]
    return lib


def native_e2e_steps(ig, hin, din, dr, djv, hr, hjv, s_in, s_comp, s_out, n, s_main):
    """run(k): k end-to-end steps through the C ABI with host buffers, double-buffered like the
    torch version: per step one pinned H2D copy of u and v, the residual and J v calls on the
    library's stream, and D2H copies of r (after the residual) and J v; events order the three
    streams, which start after the work on s_main and which s_main waits for at the end. The
    context's stream must be s_comp."""
    import ctypes

    from pylith_b200 import _lib as C

    rt = cudart()
    lib = C.lib()
    res, jac = lib.pl_compute_lhs_residual, lib.pl_compute_lhs_jacobian_action
    h = ig.handle
    P = ctypes.c_void_p
    si, sc, so = P(s_in.cuda_stream), P(s_comp.cuda_stream), P(s_out.cuda_stream)
    sm = P(s_main.cuda_stream)

    def events():
        out = []
        for _ in range(2):
            e = P()
            if rt.cudaEventCreateWithFlags(ctypes.byref(e), 2) != 0:  # cudaEventDisableTiming
                raise RuntimeError("cudaEventCreateWithFlags failed")
            out.append(e)
        return out

    ev_in, ev_res, ev_done, ev_out = events(), events(), events(), events()
    ev_edge = events()
    hin_p = [P(x.data_ptr()) for x in hin]
    din_p = [P(x.data_ptr()) for x in din]
    du_p = [P(x.data_ptr()) for x in din]
    dv_p = [P(x.data_ptr() + 8 * n) for x in din]
    dr_p, djv_p = [P(x.data_ptr()) for x in dr], [P(x.data_ptr()) for x in djv]
    hr_p, hjv_p = [P(x.data_ptr()) for x in hr], [P(x.data_ptr()) for x in hjv]
    bin_, bout = ctypes.c_size_t(16 * n), ctypes.c_size_t(8 * n)
    H2D, D2H = 1, 2
    for i in range(2):  # every buffer starts free
        rt.cudaEventRecord(ev_done[i], sc)
        rt.cudaEventRecord(ev_out[i], sc)

    def run(steps):
        rt.cudaEventRecord(ev_edge[0], sm)
        for st in (si, sc, so):
            rt.cudaStreamWaitEvent(st, ev_edge[0], 0)
        for k in range(steps):
            i = k & 1
            rt.cudaStreamWaitEvent(si, ev_done[i], 0)
            rt.cudaMemcpyAsync(din_p[i], hin_p[i], bin_, H2D, si)
            rt.cudaEventRecord(ev_in[i], si)
            rt.cudaStreamWaitEvent(sc, ev_in[i], 0)
            rt.cudaStreamWaitEvent(sc, ev_out[i], 0)
            rc = res(h, 0.0, 0.0, du_p[i], None, dr_p[i], 0)
            rt.cudaEventRecord(ev_res[i], sc)
            rc |= jac(h, 0.0, 0.0, 0.0, du_p[i], dv_p[i], djv_p[i], 0)
            rt.cudaEventRecord(ev_done[i], sc)
            rt.cudaStreamWaitEvent(so, ev_res[i], 0)
            rt.cudaMemcpyAsync(hr_p[i], dr_p[i], bout, D2H, so)
            rt.cudaStreamWaitEvent(so, ev_done[i], 0)
            rt.cudaMemcpyAsync(hjv_p[i], djv_p[i], bout, D2H, so)
            rt.cudaEventRecord(ev_out[i], so)
            if rc:
                raise RuntimeError(f"library call failed ({rc})")
        for i in range(2):  # s_main waits for the last copies out
            rt.cudaStreamWaitEvent(sc, ev_out[i], 0)
        rt.cudaEventRecord(ev_edge[1], sc)
        rt.cudaStreamWaitEvent(sm, ev_edge[1], 0)

    return run


def cpu_baseline(mesh, mat, source: str, budget_s: float = 10.0):
    """Oracle cell loop on every host core: residual F(u) plus a second pass of the same loop
    standing in for J v (linear elasticity: F(u) = J u), repeated within a time budget."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # the oracle; timed here as the CPU baseline only

    if source == "ref" and not O.ref_available():
        source = "oracle"
    aux = O.AuxFields([(mat.density[:, None], "cell"), (mat.shear_modulus[:, None], "cell"),
                       (mat.bulk_modulus[:, None], "cell")])
    u = np.random.default_rng(0).standard_normal(mesh.num_nodes * 3)
    cores = host_cpu()["affinity_cores"] or os.cpu_count() or 1
    f1 = "IsotropicLinearElasticity3D::f1v_infinitesimalStrain"
    O.residual(mesh, u, aux, f1=f1, source=source, nthreads=cores)  # warm-up
    apps = 0
    t0 = time.perf_counter()
    while True:
        O.residual(mesh, u, aux, f1=f1, source=source, nthreads=cores)
        apps += 1
        if time.perf_counter() - t0 > budget_s or apps >= 5000:
            break
    dt = time.perf_counter() - t0
    apps1 = 0
    t1 = time.perf_counter()
    while apps1 < 3 and (apps1 == 0 or time.perf_counter() - t1 < 0.25 * budget_s):
        O.residual(mesh, u, aux, f1=f1, source=source, nthreads=1)
        apps1 += 1
    dt1 = time.perf_counter() - t1
    return {"value": mesh.num_dof * apps / dt / 1e9, "unit": UNIT, "cores": cores,
            "one_core_value": mesh.num_dof * apps1 / dt1 / 1e9, "cpu": host_cpu(),
            "kind": "reference" if source == "ref" else "port",
            "sample": (f"{apps} applications over the full {mesh.num_cells}-cell mesh in {dt:.1f} s; "
                       "oracle cell loop (restated PETSc DMPlexComputeResidual) calling "
                       + ("the reference's compiled pointwise kernels (oracle/_ref)" if source == "ref"
                          else "the restated pointwise kernels")
                       + "; J v counted as one more pass of the same loop")}


def run_reference(args, rank, world):
    if rank != 0:
        return
    from pylith_b200 import materials as MAT

    mesh = load_mesh(TARGET_CELLS, 0)
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=0)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    base = cpu_baseline(mesh, mat, "ref", budget_s=max(5.0, 0.6 * args.steps))
    line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 2 * mesh.num_dof / (base["value"] * 1e9) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": "elasticity P1 tet residual+Jv",
                                            "cells": mesh.num_cells, "nodes": mesh.num_nodes,
                                            "dof": mesh.num_dof},
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="pylith_b200")
    ap.add_argument("--cells", type=int, default=TARGET_CELLS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--config", default="c1", choices=["c1", "c0", "c1link", "c1q2", "c2", "c3", "c3tile", "c3mg", "c3bmg", "c4"])
    ap.add_argument("--scale", type=float, default=1.0, help="size factor for the --config runs")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.config != "c1":
        print(json.dumps(CONFIGS[args.config](args)), flush=True)
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        # rank 0 builds the shared mesh (minutes for 8 x 1.2 M cells) before the process group
        # starts its collective timeouts; the other ranks wait for its cache file
        load_mesh(args.cells * world, seed=0, stretch=world, build=rank == 0)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from pylith_b200 import _lib
    from pylith_b200 import feassemble as FA
    from pylith_b200 import materials as MAT

    halo = None
    if world == 1:
        mesh = load_mesh(args.cells, seed=0)
        rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=0)
        global_dof = mesh.num_dof
    else:
        from pylith_b200.parallel import HaloExchange, partition_mesh

        gmesh = load_mesh(args.cells * world, seed=0, stretch=world)
        grho, gmu, gK = MAT.lognormal_elastic(gmesh.num_cells, seed=0)
        global_dof = gmesh.num_dof
        part = partition_mesh(gmesh, world)[rank]
        mesh = part.mesh
        ids = part.cell_ids
        rho, mu, K = grho[ids], gmu[ids], gK[ids]
        del gmesh, grho, gmu, gK
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    ctx = FA.Context(local_rank)
    dmesh = FA.DeviceMesh(ctx, mesh)
    ig = mat.create_integrator(dmesh)
    n = dmesh.num_dof
    if world > 1:
        halo = HaloExchange(part, device="cuda", ctx=ctx)
        hsend = torch.empty(3 * halo.total, dtype=torch.float64, device="cuda")
        hrecv = torch.empty_like(hsend)
    gen = torch.Generator(device="cuda").manual_seed(1234 + rank)
    u = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen)
    v = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen)
    r = torch.empty_like(u)
    jv = torch.empty_like(u)
    flush = L2Flush()
    stream = torch.cuda.current_stream()

    def exchange(out):
        if halo is not None:
            halo.sum_shared(out, hsend, hrecv)

    def app_residual():
        ig.compute_lhs_residual(0.0, 0.0, u, r)
        exchange(r)

    def app_jv():
        ig.compute_lhs_jacobian_action(0.0, 0.0, 0.0, u, v, jv)
        exchange(jv)

    for _ in range(args.warmup):
        flush()
        app_residual()
        flush()
        app_jv()
    ctx.synchronize()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(2 * args.steps)]
    launches0 = _lib.lib().pl_kernel_launches()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clocks:
        for k in range(args.steps):
            flush()
            ev[2 * k][0].record(stream)
            app_residual()
            ev[2 * k][1].record(stream)
            flush()
            ev[2 * k + 1][0].record(stream)
            app_jv()
            ev[2 * k + 1][1].record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = _lib.lib().pl_kernel_launches() - launches0
    ctx.synchronize()
    t_res = sum(ev[2 * k][0].elapsed_time(ev[2 * k][1]) for k in range(args.steps)) / 1e3
    t_jv = sum(ev[2 * k + 1][0].elapsed_time(ev[2 * k + 1][1]) for k in range(args.steps)) / 1e3
    t_total = t_res + t_jv
    if dist:
        tt = torch.tensor([t_total, t_res, t_jv], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_total, t_res, t_jv = tt.tolist()
    value = 2 * global_dof * args.steps / t_total / 1e9

    # End to end through the public API with host buffers: every step copies its u and v from
    # pinned host memory, computes the residual and J v, and copies both results back. Copies in
    # and out run on their own streams and the device buffers alternate between steps, so one
    # step's transfers overlap the neighbouring steps' work (PCIe is full duplex).
    # a step's u and v sit side by side in one pinned buffer and one device buffer, so that they
    # cross the link as one copy (fewer, larger copies run closer to the link's rate)
    # host buffers: page-locked memory on the GPU's NUMA node (pl_host_alloc), so that the
    # host-to-device reads do not cross the inter-socket link of a two-socket host
    def host(*shape):
        return torch.from_numpy(ctx.host_empty(shape))

    hin = [host(2, n) for _ in range(2)]
    for h in hin:
        h[0].copy_(u.cpu())
        h[1].copy_(v.cpu())
    hu = [h[0] for h in hin]
    hv = [h[1] for h in hin]
    hr = [host(n) for _ in range(2)]
    hjv = [host(n) for _ in range(2)]
    din = [torch.empty(2, n, dtype=torch.float64, device=u.device) for _ in range(2)]
    du = [d[0] for d in din]
    dv = [d[1] for d in din]
    dr = [r, torch.empty_like(r)]
    djv = [jv, torch.empty_like(jv)]
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_res = [torch.cuda.Event() for _ in range(2)]
    ev_done = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]
    for i in range(2):  # every buffer starts free
        ev_done[i].record(stream)
        ev_out[i].record(stream)

    def e2e_step(k, comp):
        """Step k on buffer set k % 2."""
        i = k % 2
        s_in.wait_event(ev_done[i])  # inputs of step k - 2 consumed
        with torch.cuda.stream(s_in):
            din[i].copy_(hin[i], non_blocking=True)
            ev_in[i].record(s_in)
        comp.wait_event(ev_in[i])
        comp.wait_event(ev_out[i])  # results of step k - 2 copied out
        with torch.cuda.stream(comp):  # the exchange's NCCL calls follow the current stream
            ig.compute_lhs_residual(0.0, 0.0, du[i], dr[i])
            exchange(dr[i])
            ev_res[i].record(comp)
            ig.compute_lhs_jacobian_action(0.0, 0.0, 0.0, du[i], dv[i], djv[i])
            exchange(djv[i])
            ev_done[i].record(comp)
        s_out.wait_event(ev_res[i])
        with torch.cuda.stream(s_out):
            hr[i].copy_(dr[i], non_blocking=True)
            s_out.wait_event(ev_done[i])
            hjv[i].copy_(djv[i], non_blocking=True)
            ev_out[i].record(s_out)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        if dist:
            tt = torch.tensor([t], dtype=torch.float64, device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = tt.item()
        return t

    # the library's calls go to a stream of their own for the end-to-end steps (the legacy default
    # stream would order them against every other blocking stream)
    comp_stream = torch.cuda.Stream()

    def eager():
        comp_stream.wait_stream(stream)
        s_in.wait_stream(stream)
        s_out.wait_stream(stream)
        for i in range(2):
            ev_done[i].record(comp_stream)
            ev_out[i].record(comp_stream)
        for k in range(args.steps):
            e2e_step(k, comp_stream)
        stream.wait_stream(comp_stream)
        for i in range(2):
            stream.wait_event(ev_out[i])

    ctx.set_stream(comp_stream.cuda_stream)
    for k in range(args.warmup):
        e2e_step(k, comp_stream)
    torch.cuda.synchronize()
    if world == 1:
        # the same steps issued as a C caller would: the C ABI and the CUDA runtime through ctypes,
        # every pointer and handle bound once (the torch calls above cost tens of microseconds of
        # host time each, more than a step's device time)
        eager_native = native_e2e_steps(ig, hin, din, dr, djv, hr, hjv, s_in, comp_stream, s_out, n, stream)
        eager_native(args.warmup)
        torch.cuda.synchronize()
        t_e2e = timed(lambda: eager_native(args.steps))
    else:
        t_e2e = timed(eager)
    ctx.set_stream(stream.cuda_stream)
    e2e_value = 2 * global_dof * args.steps / t_e2e / 1e9

    # the host link on this box: pinned copies of one step's bytes as the steps make them (inputs
    # as one copy, the two results as two), each direction alone and both directions at once (the
    # bound of the overlapped end-to-end steps)
    def link():
        out = {}
        reps = 5
        copy_in = [(din[0], hin[0])]
        copy_out = [(hr[0], dr[0]), (hjv[0], djv[0])]
        for name, plan in (("h2d", [(s_in, copy_in)]), ("d2h", [(s_out, copy_out)]),
                           ("duplex", [(s_in, copy_in), (s_out, copy_out)])):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            s_in.wait_stream(stream)
            s_out.wait_stream(stream)
            for _ in range(reps):
                for st, copies in plan:
                    with torch.cuda.stream(st):
                        for dst, src in copies:
                            dst.copy_(src, non_blocking=True)
            stream.wait_stream(s_in)
            stream.wait_stream(s_out)
            e1.record(stream)
            torch.cuda.synchronize()
            out[name + "_gbs"] = reps * 2 * n * 8 / (e0.elapsed_time(e1) / 1e3) / 1e9
        return out

    # the same steps captured once in a CUDA graph (the library's calls are capturable) and
    # replayed: every step still copies its inputs in and its results out
    def graph_e2e():
        gr = torch.cuda.CUDAGraph()
        cs = torch.cuda.Stream()

        def all_steps(comp):
            for i in range(2):
                ev_done[i].record(comp)
                ev_out[i].record(comp)
            s_in.wait_stream(comp)
            s_out.wait_stream(comp)
            for k in range(args.steps):
                e2e_step(k, comp)
            comp.wait_stream(s_in)
            comp.wait_stream(s_out)

        cs.wait_stream(stream)
        torch.cuda.synchronize()
        ctx.set_stream(cs.cuda_stream)  # the library's launches join the capture
        try:
            with torch.cuda.graph(gr, stream=cs):
                all_steps(torch.cuda.current_stream())
        finally:
            ctx.set_stream(stream.cuda_stream)
        torch.cuda.synchronize()
        gr.replay()  # warm-up
        torch.cuda.synchronize()
        t = timed(gr.replay)
        del gr
        return 2 * global_dof * args.steps / t / 1e9

    try:
        # the exchange's NCCL calls stay out of graph capture
        e2e_graph = graph_e2e() if world == 1 else None
    except RuntimeError as exc:  # capture not possible here: report the per-call figure only
        log(f"graph e2e skipped: {exc}")
        e2e_graph = None
    torch.cuda.synchronize()
    link_gbs = link()
    # steps/s the duplex link allows: one step moves 2n doubles in and 2n out
    link_bound = link_gbs["duplex_gbs"] * 1e9 / (2 * n * 8) * 2 * n / 1e9

    if rank == 0:
        peak, peak_kind = measured_peak()
        alg = algorithmic_bytes(mesh)
        achieved = alg / (t_res / args.steps) / 1e9
        traffic = profiled_traffic(mesh)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_total / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "elasticity P1 tet residual+Jv", "cells": mesh.num_cells,
                       "nodes": mesh.num_nodes, "dof": n, "l2": "flushed before every application (256 MiB write, then a 256 MiB read that writes its dirty lines back)",
                       "ms_residual": t_res / args.steps * 1e3, "ms_jv": t_jv / args.steps * 1e3,
                       "parallelism": "single GPU" if world == 1 else
                       f"{world} cell partitions of one {global_dof // 3}-node mesh; shared-node sums "
                       "by pack kernel + NCCL send/recv + add kernel inside every application",
                       "global_dof": global_dof},
            "roofline": {"bound": "hbm", "kernel": "residual (P1 tet, FP64)", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_kind, "algorithmic_bytes": alg, "traffic": traffic},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * n * 8,
                    "d2h_bytes_per_step": 2 * n * 8,
                    "overlap": "copies in and out on their own streams, device buffers alternating between steps",
                    "graph_replay_value": e2e_graph,
                    "method": "per step: one pinned H2D copy of u and v, residual and J v through the C ABI "
                              "(pl_compute_lhs_residual, pl_compute_lhs_jacobian_action), D2H of r and J v; value: "
                              "eager per-call steps issued through ctypes as a C caller would (one GPU; torch calls "
                              "under torchrun); graph_replay_value: the same steps captured once in a CUDA graph",
                    "host_buffers": f"pl_host_alloc: page-locked, GPU NUMA node {ctx.numa_node}",
                    "host_link": {**link_gbs, "bound_gdof_s": link_bound,
                                  "note": "pinned copies of one step's inputs (h2d), outputs (d2h) and both at once"}},
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
        }
        lim = issue_limiter(mesh, t_res / args.steps, line["clocks"].get("sm_mhz"))
        if lim is not None:
            line["roofline"]["limiter"] = lim
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline(mesh, mat, "oracle")
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------------------------
# The other configurations (one JSON line each). They are measurements recorded beside the
# headline, not driver bench lines.


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # CPU baseline leg only

    return O


def _ev_time(fn, reps=1):
    import torch

    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    for _ in range(reps):
        fn()
    e1.record(s)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / reps


def config_c0(args):
    """16^3 Q1 hex, uniform material, ux = -/+1 on the x faces, uy = 0 on the y faces (the
    reference test's y-face constraint, without which uy is a nullspace), uz = 0 at the bottom:
    residual, assembled Jacobian and the linear solve against the closed-form uniaxial answer."""
    import scipy.sparse.linalg as spla
    import torch

    from pylith_b200 import feassemble as FA
    from pylith_b200 import materials as MAT
    from pylith_b200 import meshing as M

    O = _oracle()
    mesh = M.box_hex(16, 16, 16)
    rho, mu, K = MAT.uniform_elastic(mesh.num_cells, 2500.0, 3000.0, 5291.503)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    bc = np.zeros((mesh.num_nodes, 3))
    for sd, val in (("neg", -1.0), ("pos", 1.0)):
        m = M.boundary_mask(mesh, 0, sd)
        cons[m, 0] = True
        bc[m, 0] = val
        cons[M.boundary_mask(mesh, 1, sd), 1] = True
    cons[M.boundary_mask(mesh, 2, "neg"), 2] = True
    cons, bc = cons.ravel(), bc.ravel()
    ctx = FA.Context(0)
    dm = FA.DeviceMesh(ctx, mesh)
    ig = mat.create_integrator(dm)
    u = torch.from_numpy(np.where(cons, bc, 0.0)).cuda()
    F = torch.zeros_like(u)
    t_res = _ev_time(lambda: ig.compute_lhs_residual(0.0, 0.0, u, F), reps=20)
    A = FA.Matrix(dm)
    t_jac = _ev_time(lambda: (A.zero(), ig.compute_lhs_jacobian(0.0, 0.0, 0.0, u, A)), reps=5)
    S = FA.Solver(dm, cons, [ig], rtol=1e-12)
    S.setup()
    du = torch.zeros_like(u)
    ig.compute_lhs_residual(0.0, 0.0, u, F)
    t_solve = _ev_time(lambda: S.solve(F, du))
    sol = (u + du).cpu().numpy().reshape(-1, 3)
    # closed form: exx = 2/12000, eyy = 0, szz = 0 -> ezz = -lam exx / (lam + 2 mu)
    lam = K[0] - 2.0 / 3.0 * mu[0]
    exx = 2.0 / 12000.0
    ezz = -lam * exx / (lam + 2.0 * mu[0])
    X = mesh.coords
    exact = np.stack([exx * X[:, 0], 0 * X[:, 1], ezz * (X[:, 2] + 9000.0)], axis=1)
    err = np.abs(sol - exact).max() / np.abs(exact).max()
    # CPU: oracle residual, element Jacobians + assembly, scipy direct solve
    aux = O.AuxFields([(rho[:, None], "cell"), (mu[:, None], "cell"), (K[:, None], "cell")])
    un = np.where(cons, bc, 0.0)
    t0 = time.perf_counter()
    r = O.residual(mesh, un, aux, f1="IsotropicLinearElasticity3D::f1v_infinitesimalStrain")
    c_res = time.perf_counter() - t0
    t0 = time.perf_counter()
    J = O.assemble(mesh, O.jacobian_elements(mesh, aux, g3="IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain"))
    c_jac = time.perf_counter() - t0
    free = ~cons
    t0 = time.perf_counter()
    spla.spsolve(J[free][:, free].tocsc(), -r[free])
    c_solve = time.perf_counter() - t0
    return {"config": "c0", "cells": mesh.num_cells, "dof": mesh.num_dof,
            "gpu_ms": {"residual": t_res * 1e3, "jacobian_assembly": t_jac * 1e3, "solve": t_solve * 1e3},
            "solve": S.stats(), "max_rel_error_vs_closed_form": float(err),
            "cpu_ms": {"residual": c_res * 1e3, "jacobian_assembly": c_jac * 1e3, "direct_solve": c_solve * 1e3,
                       "cores": os.cpu_count(), "what": "oracle cell loop + scipy spsolve"}}


def config_c1q2(args):
    """64^3 Q2 hexahedra (27 nodes, 3x3x3 Gauss), log-normal material: FP64 residual and Jacobian
    action GDOF/s; bound: FP64 arithmetic (reported against the nominal FP64 rate, 148 SMs x 64
    FP64 lanes x 2 flops x 1.965 GHz)."""
    import torch

    from pylith_b200 import feassemble as FA
    from pylith_b200 import materials as MAT
    from pylith_b200 import meshing as M

    n = max(4, int(round(64 * args.scale)))
    mesh = M.box_hex27(n, n, n)
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=0)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    ctx = FA.Context(0)
    ig = mat.create_integrator(FA.DeviceMesh(ctx, mesh))
    ndof = mesh.num_dof
    u = torch.randn(ndof, dtype=torch.float64, device="cuda")
    r = torch.empty_like(u)
    flush = L2Flush()
    for _ in range(3):
        ig.compute_lhs_residual(0.0, 0.0, u, r)
        ig.compute_lhs_jacobian_action(0.0, 0.0, 0.0, u, u, r)
    times = {"residual": [], "jv": []}
    for _ in range(max(args.steps, 3)):
        flush()
        times["residual"].append(_ev_time(lambda: ig.compute_lhs_residual(0.0, 0.0, u, r)))
        flush()
        times["jv"].append(_ev_time(lambda: ig.compute_lhs_jacobian_action(0.0, 0.0, 0.0, u, u, r)))
    tr, tj = np.mean(times["residual"]), np.mean(times["jv"])
    # FP64 operations of the sum-factorised kernel per Gauss point (a multiply-add counts 2):
    # forward 1-D contractions 72 FMA, trilinear Jacobian 72 FMA, inverse ~33, gradient
    # transform 27 FMA, flux ~35, test weights 36, reverse contractions 72 FMA.
    flop_per_cell = 27 * (2 * (72 + 72 + 27 + 36 + 72) + 33 + 35)
    return {"config": "c1q2", "cells": mesh.num_cells, "dof": ndof,
            "gdof_s_residual_plus_jv": 2 * ndof / (tr + tj) / 1e9,
            "ms_residual": tr * 1e3, "ms_jv": tj * 1e3,
            "fp64_tflops_residual": mesh.num_cells * flop_per_cell / tr / 1e12,
            "flop_per_cell_counted": flop_per_cell,
            "fp64_peak_tflops_nominal": 148 * 64 * 2 * 1.965e9 / 1e12}


def config_c2(args):
    """96x96x72 Q1 hex, generalized Maxwell (3 elements, 1e18/1e19/1e20 Pa s, ratios 0.3), planar
    vertical fault at x = 0 with 2 m left-lateral slip (step at t = 0), state per quadrature point,
    steps of 1 yr: FP64 vs FP32-refined solver, time per step and displacement difference."""
    import torch

    from pylith_b200 import materials as MAT
    from pylith_b200 import meshing as M
    from pylith_b200 import problems as P

    nx, ny, nz = (max(4, int(round(v * args.scale))) for v in (96, 96, 72))
    nx += nx % 2
    steps = max(1, int(round(50 * min(1.0, args.scale))))
    mesh = M.insert_fault_x(M.box_hex(nx, ny, nz))
    nc, nq = mesh.num_cells, 8
    rho, mu, K = MAT.lognormal_elastic(nc, seed=0)
    tau = MAT.genmaxwell_times(rho, np.sqrt(mu / rho), [1e18, 1e19, 1e20], [0.3, 0.3, 0.3])
    ratio = np.tile([0.3, 0.3, 0.3], (nc, 1))
    z = np.zeros((nc, nq, 18)), np.zeros((nc, nq, 6))
    slip = np.tile([0.0, 2.0, 0.0], (mesh.num_lagrange, 1))
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    cons[M.boundary_mask(mesh, 0, "neg")] = True
    cons[M.boundary_mask(mesh, 0, "pos")] = True
    cons = np.concatenate([cons.ravel(), np.zeros(3 * mesh.num_lagrange, dtype=bool)])
    bc = np.zeros(mesh.num_dof)
    dt = MAT.YEAR
    out = {"config": "c2", "cells": nc, "dof": mesh.num_dof, "steps": steps}
    from pylith_b200 import feassemble as FA
    from pylith_b200 import multigrid as MG

    ctx = FA.Context(0)
    levels = None
    if nx % 4 == 0 and ny % 4 == 0 and nz % 4 == 0:
        levels = MG.build_hierarchy(nx, ny, nz, fault_x=0.0,
                                    constrained_faces=[(0, "neg", (0, 1, 2)), (0, "pos", (0, 1, 2))])
        assert np.array_equal(levels[0].constrained, cons)
        out["multigrid_levels"] = [list(lv.n) for lv in levels]
    sols = {}
    variants = [("fp64", FA.Solver.FP64, None), ("fp32_refined", FA.Solver.FP32_REFINED, None)]
    if levels is not None:
        variants += [("fp64_multigrid", FA.Solver.FP64, FA.Solver.FP64),
                     ("fp32_vcycle_multigrid", FA.Solver.FP64, FA.Solver.FP32_REFINED)]
    for name, prec, mg_prec in variants:
        g = MAT.IsotropicLinearGenMaxwell(rho, mu, K, tau, ratio, z[0], z[1])
        prob = P.QuasistaticProblem(ctx, mesh, [(g, None)], cons, bc, faults=[MAT.FaultCohesiveKin(slip)],
                                    dt=dt, precision=prec, rtol=1e-10, inner_rtol=1e-4)
        mg = None
        if mg_prec is not None:
            mg = MG.attach(ctx, prob.solver, levels, g, fault_x=0.0, dt=dt, precision=mg_prec)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        its = 0
        for k in range(1, steps + 1):
            st = prob.step(k * dt)
            its += st.iterations + st.inner_iterations
        ctx.synchronize()
        el = time.perf_counter() - t0
        sols[name] = prob.u.cpu().numpy()
        out[name] = {"s_per_step": el / steps, "iterations_per_step": its / steps}
        if mg is not None:
            out[name]["lambda_max_per_level"] = mg.lambda_max()
            mg.close()
    nd = 3 * mesh.num_nodes
    ref = sols["fp64"][:nd]
    for name in sols:
        if name != "fp64":
            out[f"rel_displacement_diff_{name}_vs_fp64"] = float(np.linalg.norm(sols[name][:nd] - ref) / np.linalg.norm(ref))
            out[f"speedup_{name}"] = out["fp64"]["s_per_step"] / out[name]["s_per_step"]
    return out


def config_c3(args):
    """Green's functions: 1.5 M-cell Delaunay P1 mesh of [-12,12]x[-15,15]x[-20,0] km (the config-1
    mesh construction, mirrored across x = 0 so that the plane carries a conforming fault of
    cohesive cells) with the config-1 material statistics; 40x25 unit-slip patches over y in
    [-12,12] km, z in [-15,0] km, left-lateral then reverse: 2,000 impulses. Every impulse solved
    (a) batched (FP32 PCG tiles with reliable updates, tile and preconditioner picked by the
    autotuner), (b) one at a time by FP64 CG with FP32 multigrid V-cycles over independent
    coarser Delaunay meshes of the box, and (c) batched with one FP32 V-cycle on all 8 vectors of a
    tile per iteration; against one-at-a-time FP64 solves of a sample of at least 20 impulses with
    point-block Jacobi and with FP64 multigrid."""
    import torch

    from pylith_b200 import feassemble as FA
    from pylith_b200 import greensfns as GF
    from pylith_b200 import materials as MAT
    from pylith_b200 import meshing as M
    from pylith_b200 import multigrid as MG

    lo, hi = (-12000.0, -15000.0, -20000.0), (12000.0, 15000.0, 0.0)
    t0 = time.perf_counter()
    mesh = M.box_tet_delaunay_fault_x(int(1_500_000 * args.scale), seed=0, lo=lo, hi=hi)
    t_mesh = time.perf_counter() - t0
    faces = [(0, "neg", (0, 1, 2)), (0, "pos", (0, 1, 2))]
    t0 = time.perf_counter()
    levels = MG.build_tet_hierarchy(mesh, lambda n, l: M.box_tet_delaunay_fault_x(n, seed=l, lo=lo, hi=hi),
                                    fault_x=0.0, lo=lo, hi=hi, constrained_faces=faces)
    t_hier = time.perf_counter() - t0
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=0)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    cons = levels[0].constrained
    patches = GF.fault_patches(mesh, (-12000.0, 12000.0), (-15000.0, 0.0), 40, 25)
    ctx = FA.Context(0)
    # rtol 1e-11 for every solve: the Delaunay mesh's conditioning turns a 1e-10 residual into
    # displacement differences just above 1e-8
    g = GF.GreensFunctions(ctx, mesh, mat, cons, patches, rtol=1e-11, inner_rtol=1e-4, tile=8)
    usable = [imp for imp in g.impulses if len(patches[imp.patch]) > 0]  # every patch holds a node: all of them
    # the autotuner picks the tile size and the preconditioner (point-block Jacobi or Chebyshev-
    # Jacobi of degree 2-3) on a sample of 32 impulses
    step = max(1, len(usable) // 32)
    table = g.autotune(usable[step // 2::step][:32], tiles=(8, 16), degrees=(0, 2, 3))
    mg64 = g.attach_multigrid(levels, mat, FA.Solver.FP64)
    mg64_h = g.mg
    mg32 = g.attach_multigrid(levels, mat, FA.Solver.FP32_REFINED)
    # the smoothing of the FP32 V-cycles, picked on a sample of 6 impulses (the FP64 multigrid
    # baseline takes the same)
    mg_table = g.tune_multigrid(usable[step // 2::step][:6])
    mg64_h.set_smoother(g.mg.degree, g.mg.lower)
    bmg = g.batched_multigrid(8)  # (c) tiles of 8 impulses, one V-cycle on all 8 per iteration
    g.solve(usable[:8], batched=True, batch=bmg)  # warm-up: graph capture
    g.solve(usable[:8], batched=True)  # warm-up
    g.solve(usable[:1], batched=False)
    g.solve(usable[:2], batched=False, solver=mg32)
    g.solve(usable[:2], batched=False, solver=mg64)
    ns = max(20, int(args.steps))
    sample_s = usable[::max(1, len(usable) // ns)][:ns]
    want = {id(imp) for imp in sample_s}
    keep_b, keep_m, keep_bm, t_b, t_m, t_bm, its_m = {}, {}, {}, 0.0, 0.0, 0.0, []
    for c0 in range(0, len(usable), 400):  # 400 impulses' vectors at a time on the device
        part = usable[c0:c0 + 400]
        sols, dt_part = g.solve(part, batched=True)
        t_b += dt_part
        keep_b.update({id(imp): x for imp, x in zip(part, sols) if id(imp) in want})
        del sols
        sols, dt_part = g.solve(part, batched=True, batch=bmg)
        t_bm += dt_part
        keep_bm.update({id(imp): x for imp, x in zip(part, sols) if id(imp) in want})
        del sols
        sols, dt_part = g.solve(part, batched=False, solver=mg32)
        t_m += dt_part
        its_m.append(mg32.stats()["iterations"])
        keep_m.update({id(imp): x for imp, x in zip(part, sols) if id(imp) in want})
        del sols
    st_b = g.batch.stats()
    sol_s, t_s = g.solve(sample_s, batched=False)
    its_s = g.solver64.stats()["iterations"]
    sol_g, t_g = g.solve(sample_s, batched=False, solver=mg64)
    its_g = mg64.stats()["iterations"]

    def err(keep, ref):
        return max(float(torch.linalg.norm(keep[id(imp)] - b) / torch.linalg.norm(b)) for imp, b in zip(sample_s, ref))

    rate_b, rate_m, rate_bm = len(usable) / t_b, len(usable) / t_m, len(usable) / t_bm
    st_bm = bmg.stats()
    rate_s, rate_g = len(sample_s) / t_s, len(sample_s) / t_g
    return {"config": "c3", "cells": mesh.num_cells, "dof": mesh.num_dof, "mesh": "Delaunay, mirrored across the fault",
            "mesh_build_s": t_mesh, "impulses_total": len(g.impulses), "impulses_solved": len(usable),
            "multigrid_levels": [lv.mesh.num_cells for lv in levels], "hierarchy_build_s": t_hier,
            "batched": {"solves_per_s": rate_b, "seconds": t_b, "tile": g.batch.tile,
                        "chebyshev_degree": g.batch.degree, "lambda_max_estimate": g.batch.lambda_max,
                        "fp64_accuracy": "reliable updates (residual replacement, delta 0.01)",
                        "last_call_stats": st_b},
            "autotune": [{"tile": t, "chebyshev_degree": d, "solves_per_s": r} for t, d, r in table],
            "multigrid_fp32_vcycles": {"solves_per_s": rate_m, "seconds": t_m, "iterations_last": its_m[-1],
                                       "smoother": {"degree": g.mg.degree, "lower_ratio": g.mg.lower},
                                       "smoother_tuning": [{"degree": d, "lower_ratio": lo, "solves_per_s": r,
                                                            "iterations": it} for d, lo, r, it in mg_table],
                                       "how": "one impulse at a time: FP64 flexible CG, one FP32 V-cycle "
                                              "(Chebyshev-Jacobi smoothing) per iteration"},
            "batched_multigrid": {"solves_per_s": rate_bm, "seconds": t_bm, "tile": 8, "last_call_stats": st_bm,
                                  "how": "tiles of 8 impulses: FP32 PCG with reliable updates, one FP32 V-cycle "
                                         "on all 8 vectors per iteration (batched cell-block operator on every level)"},
            "fp64_one_at_a_time": {"sample": len(sample_s), "solves_per_s": rate_s, "iterations_last": its_s,
                                   "preconditioner": "point-block Jacobi"},
            "fp64_multigrid_one_at_a_time": {"sample": len(sample_s), "solves_per_s": rate_g, "iterations_last": its_g},
            "speedup": rate_b / rate_s,
            "speedup_multigrid_vs_fp64": rate_m / rate_s,
            "speedup_multigrid_vs_fp64_multigrid": rate_m / rate_g,
            "speedup_batched_multigrid_vs_fp64": rate_bm / rate_s,
            "speedup_batched_multigrid_vs_fp64_multigrid": rate_bm / rate_g,
            "max_rel_displacement_error_batched_multigrid_vs_fp64": err(keep_bm, sol_s),
            "max_rel_displacement_error_vs_fp64": err(keep_b, sol_s),
            "max_rel_displacement_error_multigrid_vs_fp64": err(keep_m, sol_s)}


def config_c3tile(args):
    """One batched tile of the C3 Green's functions (8 impulses, FP32 PCG with reliable updates) on
    the 1.5 M-cell mirrored Delaunay mesh: the profiling case of the batched operator kernel."""
    from pylith_b200 import feassemble as FA
    from pylith_b200 import greensfns as GF
    from pylith_b200 import materials as MAT
    from pylith_b200 import meshing as M

    lo, hi = (-12000.0, -15000.0, -20000.0), (12000.0, 15000.0, 0.0)
    mesh = M.box_tet_delaunay_fault_x(int(1_500_000 * args.scale), seed=0, lo=lo, hi=hi)
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=0)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    for sd in ("neg", "pos"):
        cons[M.boundary_mask(mesh, 0, sd, lo, hi)] = True
    cons = np.concatenate([cons.ravel(), np.zeros(3 * mesh.num_lagrange, dtype=bool)])
    patches = GF.fault_patches(mesh, (-12000.0, 12000.0), (-15000.0, 0.0), 40, 25)
    ctx = FA.Context(0)
    g = GF.GreensFunctions(ctx, mesh, mat, cons, patches, rtol=1e-11, inner_rtol=1e-4, tile=8)
    _, dt = g.solve(g.impulses[:8], batched=True)
    return {"config": "c3tile", "cells": mesh.num_cells, "dof": mesh.num_dof, "seconds": dt, "stats": g.batch.stats()}


def config_c3mg(args):
    """Four Green's-function impulses on the C3 mesh solved one at a time by FP64 CG with FP32
    V-cycles over the coarser Delaunay levels (smoother degree 3): the profiling case of the
    multigrid path."""
    from pylith_b200 import feassemble as FA
    from pylith_b200 import greensfns as GF
    from pylith_b200 import materials as MAT
    from pylith_b200 import meshing as M
    from pylith_b200 import multigrid as MG

    lo, hi = (-12000.0, -15000.0, -20000.0), (12000.0, 15000.0, 0.0)
    mesh = M.box_tet_delaunay_fault_x(int(1_500_000 * args.scale), seed=0, lo=lo, hi=hi)
    levels = MG.build_tet_hierarchy(mesh, lambda n, l: M.box_tet_delaunay_fault_x(n, seed=l, lo=lo, hi=hi),
                                    fault_x=0.0, lo=lo, hi=hi, constrained_faces=[(0, "neg", (0, 1, 2)), (0, "pos", (0, 1, 2))])
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=0)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    patches = GF.fault_patches(mesh, (-12000.0, 12000.0), (-15000.0, 0.0), 40, 25)
    ctx = FA.Context(0)
    g = GF.GreensFunctions(ctx, mesh, mat, levels[0].constrained, patches, rtol=1e-11, inner_rtol=1e-4, tile=8)
    solver = g.attach_multigrid(levels, mat, FA.Solver.FP32_REFINED)
    g.mg.set_smoother(3, 0.1)
    g.solve(g.impulses[:1], batched=False, solver=solver)  # setup, eigenvalue estimates, graph capture
    _, dt = g.solve(g.impulses[1:5], batched=False, solver=solver)
    return {"config": "c3mg", "cells": mesh.num_cells, "levels": [lv.mesh.num_cells for lv in levels],
            "seconds_per_solve": dt / 4, "iterations": solver.stats()["iterations"]}


def config_c3bmg(args):
    """Sixteen Green's-function impulses on the C3 mesh in tiles of 8, the tile's FP32 PCG
    preconditioned by one V-cycle on all 8 vectors per iteration: the profiling case of the
    batched multigrid path."""
    from pylith_b200 import feassemble as FA
    from pylith_b200 import greensfns as GF
    from pylith_b200 import materials as MAT
    from pylith_b200 import meshing as M
    from pylith_b200 import multigrid as MG

    lo, hi = (-12000.0, -15000.0, -20000.0), (12000.0, 15000.0, 0.0)
    mesh = M.box_tet_delaunay_fault_x(int(1_500_000 * args.scale), seed=0, lo=lo, hi=hi)
    levels = MG.build_tet_hierarchy(mesh, lambda n, l: M.box_tet_delaunay_fault_x(n, seed=l, lo=lo, hi=hi),
                                    fault_x=0.0, lo=lo, hi=hi, constrained_faces=[(0, "neg", (0, 1, 2)), (0, "pos", (0, 1, 2))])
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=0)
    mat = MAT.IsotropicLinearElasticity(rho, mu, K)
    patches = GF.fault_patches(mesh, (-12000.0, 12000.0), (-15000.0, 0.0), 40, 25)
    ctx = FA.Context(0)
    g = GF.GreensFunctions(ctx, mesh, mat, levels[0].constrained, patches, rtol=1e-11, inner_rtol=1e-4, tile=8)
    g.attach_multigrid(levels, mat, FA.Solver.FP32_REFINED)
    g.mg.set_smoother(3, 0.1)
    bmg = g.batched_multigrid(8)
    g.solve(g.impulses[:8], batched=True, batch=bmg)  # eigenvalue estimates, graph capture
    _, dt = g.solve(g.impulses[8:24], batched=True, batch=bmg)
    return {"config": "c3bmg", "cells": mesh.num_cells, "seconds_per_solve": dt / 16, "stats": bmg.stats()}


def config_c4(args):
    """Serving: Poisson requests (200 req/s), box meshes n^3 with n log-uniform in [8, 96], log-normal
    material, random rectangular left-lateral slip patch of 0.1-3 m. Server (HBM-budget admission;
    small boxes in one ragged batch of FP32-refined solves, boxes of 32^3 and more with a multigrid
    hierarchy solved beside it by three workers with FP32 V-cycles) vs the plain FP64 one-at-a-time path (point-block
    Jacobi), and vs FP64 one at a time with FP64 multigrid. The requests' host-side meshes (and
    multigrid hierarchies) are built before the stream starts, for all."""
    from pylith_b200 import feassemble as FA
    from pylith_b200 import serving as SV

    count = max(8, int(40 * args.scale))
    reqs = SV.poisson_requests(count, rate=200.0, seed=0, n_min=8, n_max=max(8, int(96 * min(1.0, args.scale))))
    t0 = time.perf_counter()
    hps = [SV.prepare(r) for r in reqs]
    t_host = time.perf_counter() - t0
    warm = [SV.prepare(SV.Request(0, n, 1, 0.0, 1.0, (0.2, 0.8, 0.2, 0.8))) for n in (8, 32)]
    SV.Server(slots=64).run(warm)  # warm-up: device code loading and the first graph captures
    variants = {}
    for k in (1, 2, 4):
        sv = SV.Server(slots=64, multigrid_workers=k)
        variants[k] = SV.summarize(sv.run(hps))["solves_per_s"]
    server = SV.Server(slots=64, multigrid_workers=3)
    served = server.run(hps)
    seq = SV.serve_sequential(hps)
    seq_mg = SV.serve_sequential(hps, multigrid=FA.Solver.FP64)
    a, b, c = SV.summarize(served), SV.summarize(seq), SV.summarize(seq_mg)
    mem = np.array([(p, m) for _, p, m in server.memory], dtype=float) if server.memory else np.zeros((1, 2))
    routes = list(server.routes.values())
    return {"config": "c4", "requests": count, "server": a, "fp64_one_at_a_time": b,
            "solves_per_s_ratio": a["solves_per_s"] / b["solves_per_s"],
            "fp64_multigrid_one_at_a_time": c, "solves_per_s_ratio_vs_fp64_multigrid": a["solves_per_s"] / c["solves_per_s"],
            "routes": {"ragged_batch": routes.count("batch"), "multigrid": routes.count("multigrid")},
            "multigrid_workers": server.multigrid_workers, "workers": server.workers,
            "solves_per_s_with_multigrid_workers": {str(k): v for k, v in variants.items()},
            "host_mesh_build_s_excluded": t_host,
            "admission_bytes": {"predicted_total_batch": float(mem[:, 0].sum()), "measured_total_batch": float(mem[:, 1].sum()),
                                "how": "predicted: estimate_bytes(n) formula used for admission; measured: free device "
                                       "memory before and after each batched request's build (approximate: the "
                                       "multigrid workers allocate concurrently, and the library's memory pool keeps "
                                       "freed memory for reuse)"}}


def config_c1link(args):
    """Where the end-to-end steps of the headline workload (1.2 M P1 tets, one step = u and v in,
    residual and J v, r and J v out) spend their time on this box: each piece alone and the
    pipelines, in microseconds per step over 40 steps, with host buffers from pl_host_alloc
    and, for comparison, torch's pinned-memory cache."""
    import ctypes

    import torch

    from pylith_b200 import _lib
    from pylith_b200 import feassemble as FA
    from pylith_b200 import materials as MAT

    mesh = load_mesh(args.cells, seed=0)
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=0)
    ctx = FA.Context(0)
    ig = MAT.IsotropicLinearElasticity(rho, mu, K).create_integrator(FA.DeviceMesh(ctx, mesh))
    n = 3 * mesh.num_nodes

    def host(*shape):
        return torch.from_numpy(ctx.host_empty(shape))

    hin = [host(2, n) for _ in range(2)]
    hr, hjv = [host(n) for _ in range(2)], [host(n) for _ in range(2)]
    for h in hin:
        h.normal_()
    din = [torch.empty(2, n, dtype=torch.float64, device="cuda") for _ in range(2)]
    dr = [torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(2)]
    djv = [torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(2)]
    s_in, s_comp, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    main = torch.cuda.current_stream()
    ctx.set_stream(s_comp.cuda_stream)
    rt, lib = cudart(), _lib.lib()
    P, S = ctypes.c_void_p, ctypes.c_size_t
    steps = 40

    def per_step(fn):
        fn(4)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(main)
        fn(steps)
        e1.record(main)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) * 1e3 / steps

    def copies(do_in, do_out, src=None):
        def fn(k):
            for st in (s_in, s_out):
                st.wait_stream(main)
            for j in range(k):
                i = j & 1
                if do_in:
                    p = src[i] if src is not None else hin[i].data_ptr()
                    rt.cudaMemcpyAsync(P(din[i].data_ptr()), P(p), S(16 * n), 1, P(s_in.cuda_stream))
                if do_out:
                    rt.cudaMemcpyAsync(P(hr[i].data_ptr()), P(dr[i].data_ptr()), S(8 * n), 2, P(s_out.cuda_stream))
                    rt.cudaMemcpyAsync(P(hjv[i].data_ptr()), P(djv[i].data_ptr()), S(8 * n), 2, P(s_out.cuda_stream))
            for st in (s_in, s_out):
                main.wait_stream(st)
        return fn

    def compute(k):
        s_comp.wait_stream(main)
        for j in range(k):
            i = j & 1
            lib.pl_compute_lhs_residual(ig.handle, 0.0, 0.0, P(din[i].data_ptr()), None, P(dr[i].data_ptr()), 0)
            lib.pl_compute_lhs_jacobian_action(ig.handle, 0.0, 0.0, 0.0, P(din[i].data_ptr()),
                                               P(din[i].data_ptr() + 8 * n), P(djv[i].data_ptr()), 0)
        main.wait_stream(s_comp)

    pinned = [torch.empty(2, n, dtype=torch.float64, pin_memory=True) for _ in range(2)]
    for t in pinned:
        t.normal_()
    out = {"in": per_step(copies(True, False)), "out": per_step(copies(False, True)),
           "in_and_out": per_step(copies(True, True)), "kernels": per_step(compute)}
    run = native_e2e_steps(ig, hin, din, dr, djv, hr, hjv, s_in, s_comp, s_out, n, main)
    out["e2e_per_call"] = per_step(run)
    out["in_from_torch_pinned"] = per_step(copies(True, False, [t.data_ptr() for t in pinned]))
    ctx.set_stream(main.cuda_stream)
    gbs = {k: 16 * n / (v * 1e-6) / 1e9 for k, v in out.items() if k.startswith("in") and k != "in_and_out"}
    return {"config": "c1link", "dof": n, "bytes_in_per_step": 16 * n, "bytes_out_per_step": 16 * n,
            "us_per_step": out, "h2d_gbs": gbs, "e2e_gdof_s": 2 * n / (out["e2e_per_call"] * 1e-6) / 1e9,
            "host_buffers": f"pl_host_alloc (GPU NUMA node {ctx.numa_node})"}


CONFIGS = {"c0": config_c0, "c1link": config_c1link, "c1q2": config_c1q2, "c2": config_c2, "c3": config_c3, "c3tile": config_c3tile,
           "c3mg": config_c3mg, "c3bmg": config_c3bmg, "c4": config_c4}


if __name__ == "__main__":
    main()
