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
    """Fault-node index lists of an ny x nz grid of rectangular patches on the fault plane."""
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
            patches.append(np.nonzero(inside & (iy == ky) & (iz == kz))[0])
    return patches


@dataclass
class Impulse:
    patch: int
    component: str


class GreensFunctions:
    def __init__(self, ctx, mesh, material, constrained, patches, components=("left_lateral", "reverse"),
                 rtol=1e-10, inner_rtol=1e-4, tile=8, ref_dir_1=(0.0, 0.0, 1.0), ref_dir_2=(0.0, 1.0, 0.0)):
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
        self.solver64 = FA.Solver(self.dmesh, constrained, [self.domain], rtol=rtol)
        self.solver64.setup()
        self.solver32 = FA.Solver(self.dmesh, constrained, [self.domain], rtol=rtol,
                                  precision=FA.Solver.FP32_REFINED, inner_rtol=inner_rtol)
        self.solver32.setup()
        self.batch = FA.BatchSolver(self.solver32, tile)

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

    def solve(self, impulses, batched=True):
        """Solutions u = u_slip + du of the given impulses; returns (solutions, seconds)."""
        import torch

        rhs = [self.impulse_rhs(imp) for imp in impulses]
        xs = [torch.zeros_like(b) for _, b in rhs]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if batched:
            self.batch.solve([b for _, b in rhs], xs)
        else:
            for (_, b), x in zip(rhs, xs):
                self.solver64.solve(b, x)
        self.ctx.synchronize()
        dt = time.perf_counter() - t0
        return [u + x for (u, _), x in zip(rhs, xs)], dt
