"""Static Green's functions: one linear solve per fault impulse, many impulses per launch.

The reference's GreensFns problem (libsrc/pylith/problems/GreensFns.cc:190-337) forms one
Jacobian (SNESSetLagJacobian(-2), :236-241) and then, for every impulse, sets unit slip on one
fault vertex and component (FaultCohesiveImpulses::updateAuxiliaryField,
libsrc/pylith/faults/FaultCohesiveImpulses.cc:264-290) and calls SNESSolve (:326), one impulse
at a time. Here an impulse is unit slip on a rectangular patch of fault nodes (a sum of the
reference's vertex impulses), the right-hand side of each impulse is the residual of the
displacement that carries the slip on the positive side of the fault, and tiles of impulses are
solved together by the batched solver (pl_batch_solver_*), with the one-at-a-time FP64 solve
kept as the reference-shaped baseline.
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np

from . import feassemble as FA

COMPONENTS = {"opening": 0, "left_lateral": 1, "reverse": 2}


def fault_patches(mesh, y_range, z_range, ny: int, nz: int):
    """Fault-node index lists of an ny x nz grid of rectangular patches on the fault plane. A patch
    that holds no fault node (an unstructured fault mesh coarser than the patch grid) takes the
    fault node nearest its centre, so every patch carries an impulse."""
    lag_nodes = np.zeros(mesh.num_lagrange, dtype=np.int64)
    coh = mesh.cohesive
    lag_nodes[coh[:, 8:].ravel()] = coh[:, :4].ravel()  # negative-side node of each fault node
    yz = mesh.coords[lag_nodes][:, 1:]
    iy = np.floor((yz[:, 0] - y_range[0]) / (y_range[1] - y_range[0]) * ny).astype(int)
    iz = np.floor((yz[:, 1] - z_range[0]) / (z_range[1] - z_range[0]) * nz).astype(int)
    inside = (iy >= 0) & (iy < ny) & (iz >= 0) & (iz < nz)
    patches = []
    for kz in range(nz):
        for ky in range(ny):
            nodes = np.nonzero(inside & (iy == ky) & (iz == kz))[0]
            if len(nodes) == 0 and len(yz):
                cy = y_range[0] + (ky + 0.5) * (y_range[1] - y_range[0]) / ny
                cz = z_range[0] + (kz + 0.5) * (z_range[1] - z_range[0]) / nz
                nodes = np.array([int(np.argmin((yz[:, 0] - cy) ** 2 + (yz[:, 1] - cz) ** 2))])
            patches.append(nodes)
    return patches


@dataclass
class Impulse:
    patch: int
    component: str


class GreensFunctions:
    def __init__(self, ctx, mesh, material, constrained, patches, components=("left_lateral", "reverse"),
                 rtol=1e-10, inner_rtol=1e-4, tile=8, ref_dir_1=(0.0, 0.0, 1.0), ref_dir_2=(0.0, 1.0, 0.0),
                 cheb_degree=0, cheb_lower_ratio=0.05):
        from . import materials as MAT

        self.ctx = ctx
        self.mesh = mesh
        self.dmesh = FA.DeviceMesh(ctx, mesh)
        self.domain = material.create_integrator(self.dmesh)
        self.fault = MAT.FaultCohesiveKin(np.zeros((mesh.num_lagrange, 3)), ref_dir_1, ref_dir_2)
        self.iface = self.fault.create_integrator(self.dmesh)
        self.patches = patches
        self.impulses = [Impulse(p, c) for c in components for p in range(len(patches))]
        self.constrained = constrained
        self.rtol = rtol
        self.solver64 = FA.Solver(self.dmesh, constrained, [self.domain], rtol=rtol)
        self.solver64.setup()
        self.solver32 = FA.Solver(self.dmesh, constrained, [self.domain], rtol=rtol,
                                  precision=FA.Solver.FP32_REFINED, inner_rtol=inner_rtol)
        self.solver32.setup()
        self.batch = FA.BatchSolver(self.solver32, tile)
        self.cheb_lower_ratio = cheb_lower_ratio
        if cheb_degree >= 2:
            self.batch.set_chebyshev(cheb_degree, cheb_lower_ratio)

    def attach_multigrid(self, levels, material, precision=FA.Solver.FP32_REFINED, fault_x=0.0, rtol=None):
        """A solver for one impulse at a time by FP64 flexible CG preconditioned with V-cycles (of
        `precision`) over `levels` (pylith_b200.multigrid.build_tet_hierarchy of this mesh); returns
        it (solve with method="multigrid" uses the last one attached)."""
        from . import multigrid as MG

        solver = FA.Solver(self.dmesh, self.constrained, [self.domain], rtol=rtol or self.rtol)
        mg = MG.attach(self.ctx, solver, levels, material, fault_x=fault_x, precision=precision)
        solver.setup()
        self._mg_keep = getattr(self, "_mg_keep", []) + [(solver, mg)]
        self.solver_mg = solver
        self.mg = mg
        return solver

    def batched_multigrid(self, tile=8):
        """A batched solver (tiles of `tile` impulses, FP32 PCG with reliable updates on the
        single-impulse solvers' FP32 operator) preconditioned by one V-cycle of the last attached
        hierarchy on all the tile's vectors per iteration; solve(..., batch=it) uses it."""
        bs = FA.BatchSolver(self.solver32, tile)
        bs.set_multigrid(self.mg)
        self._mg_keep = getattr(self, "_mg_keep", []) + [(bs, None)]
        return bs

    def tune_multigrid(self, impulses, degrees=(2, 3, 4), lowers=(0.1, 0.3)):
        """Picks the Chebyshev smoothing (degree, lower ratio) of the last attached multigrid with
        the highest solves/s on `impulses` (each setting solves them once to warm up and once timed)
        and keeps it. Returns [(degree, lower, solves_per_s, iterations)], best first."""
        rhs = [self.impulse_rhs(imp)[1] for imp in impulses]
        import torch

        out = []
        for d in degrees:
            for lo in lowers:
                self.mg.set_smoother(d, lo)
                xs = [torch.zeros_like(b) for b in rhs]
                self.solver_mg.solve(rhs[0], xs[0])  # graph capture
                self.ctx.synchronize()
                t0 = time.perf_counter()
                for b, x in zip(rhs, xs):
                    self.solver_mg.solve(b, x)
                self.ctx.synchronize()
                out.append((d, lo, len(rhs) / (time.perf_counter() - t0), self.solver_mg.stats()["iterations"]))
        best = max(out, key=lambda r: r[2])
        self.mg.set_smoother(best[0], best[1])
        return sorted(out, key=lambda r: -r[2])

    def impulse_rhs(self, imp: Impulse):
        """(u_slip, b): the displacement carrying unit slip on the patch, and b = F(u_slip)."""
        import torch

        slip = np.zeros((self.mesh.num_lagrange, 3))
        slip[self.patches[imp.patch], COMPONENTS[imp.component]] = 1.0
        self.iface.set_aux("slip", FA.PER_FAULT_NODE, slip)
        u = torch.zeros(self.dmesh.num_dof, dtype=torch.float64, device="cuda")
        self.solver64.apply_fault_slip(self.iface, u)
        b = torch.zeros_like(u)
        self.domain.compute_lhs_residual(0.0, 0.0, u, b)
        return u, b

    def autotune(self, impulses, tiles=(4, 8), degrees=(0, 2, 3, 4)):
        """Picks the tile size and the preconditioner degree (0: point-block Jacobi, >= 2:
        Chebyshev-Jacobi) with the highest batched solves/s on `impulses` (a sample of the
        impulses to be solved; each configuration solves them once to warm up and once timed)
        and keeps that batched solver. Returns [(tile, degree, solves_per_s)], best first."""
        rhs = [self.impulse_rhs(imp)[1] for imp in impulses]
        import torch

        results = []
        best = None
        for tile in tiles:
            for degree in degrees:
                bs = FA.BatchSolver(self.solver32, tile)
                if degree >= 2:
                    bs.set_chebyshev(degree, self.cheb_lower_ratio)
                xs = [torch.zeros_like(b) for b in rhs]
                bs.solve(rhs[:tile], xs[:tile])  # graph capture and eigenvalue estimate
                self.ctx.synchronize()
                t0 = time.perf_counter()
                bs.solve(rhs, xs)
                self.ctx.synchronize()
                rate = len(rhs) / (time.perf_counter() - t0)
                results.append((tile, degree, rate))
                if best is None or rate > best[2]:
                    if best is not None:
                        best[3].close()
                    best = (tile, degree, rate, bs)
                else:
                    bs.close()
        self.batch.close()
        self.batch = best[3]
        return sorted(results, key=lambda r: -r[2])

    def solve(self, impulses, batched=True, solver=None, batch=None):
        """Solutions u = u_slip + du of the given impulses; returns (solutions, seconds). batched:
        the tiles of `batch` (default: the autotuned batched FP32 solver); else one at a time with
        `solver` (default: the FP64 point-block Jacobi solver)."""
        import torch

        rhs = [self.impulse_rhs(imp) for imp in impulses]
        xs = [torch.zeros_like(b) for _, b in rhs]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if batched:
            (batch or self.batch).solve([b for _, b in rhs], xs)
        else:
            one = solver or self.solver64
            for (_, b), x in zip(rhs, xs):
                one.solve(b, x)
        self.ctx.synchronize()
        dt = time.perf_counter() - t0
        return [u + x for (u, _), x in zip(rhs, xs)], dt
