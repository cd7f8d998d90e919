"""Quasi-static problem driver on the device: the loop PyLith's TimeDependent runs around the
residual/Jacobian path (libsrc/pylith/problems/TimeDependent.cc:490-747), restated for the
C ABI:

  per step   set the local solution's Dirichlet values (ConstraintSpatialDB::setSolution,
             feassemble/ConstraintSpatialDB.cc:147) and the prescribed fault slip
             (FaultCohesiveKin::updateAuxiliaryField, faults/FaultCohesiveKin.cc:232-258),
             compute the LHS residual of every integrator (TimeDependent.cc:659-662),
             solve J du = -F with the device PCG (the reference's KSP), u += du,
             then update the state variables (poststep, TimeDependent.cc:490-538).

The Jacobian (preconditioner) is rebuilt only when its trigger fires: never for linear
elasticity (RheologyElasticity.cc:27), on a time-step change for generalized Maxwell
(IsotropicLinearGenMaxwell.cc:33).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import feassemble as FA


@dataclass
class StepStats:
    t: float
    iterations: int
    inner_iterations: int
    outer_iterations: int
    rel_residual: float


@dataclass
class QuasistaticProblem:
    ctx: FA.Context
    mesh: object                       # pylith_b200.meshing.Mesh
    materials: list                    # (material, cell_ids or None)
    constrained: np.ndarray            # bool [num_dof]: Dirichlet DOFs
    bc_values: np.ndarray              # float64 [num_dof]: values at the constrained DOFs
    faults: list = field(default_factory=list)
    dt: float = 0.0
    precision: int = FA.Solver.FP64
    rtol: float = 1e-12
    inner_rtol: float = 1e-5

    def __post_init__(self):
        import torch

        self.dmesh = FA.DeviceMesh(self.ctx, self.mesh)
        self.domain: List[FA.IntegratorDomain] = []
        self.viscous: List[FA.IntegratorDomain] = []
        for mat, ids in self.materials:
            if hasattr(mat, "maxwell_time"):
                ig = mat.create_integrator(self.dmesh, self.dt, ids)
                self.viscous.append(ig)
            else:
                ig = mat.create_integrator(self.dmesh, ids)
            self.domain.append(ig)
        self.interfaces = [f.create_integrator(self.dmesh) for f in self.faults]
        self.solver = FA.Solver(self.dmesh, self.constrained, self.domain, rtol=self.rtol,
                                precision=self.precision, inner_rtol=self.inner_rtol)
        n = self.dmesh.num_dof
        self.u = torch.zeros(n, dtype=torch.float64, device="cuda")
        self.F = torch.zeros_like(self.u)
        self.du = torch.zeros_like(self.u)
        self._bc = torch.from_numpy(np.ascontiguousarray(self.bc_values, dtype=np.float64)).cuda()
        if self._bc.numel() < n:
            raise ValueError(f"bc_values has {self._bc.numel()} entries, the solution {n}")
        self._setup_dt: Optional[float] = None
        self.history: List[StepStats] = []

    def residual(self, t: float, u=None, out=None):
        """Sum of every integrator's LHS residual (the full local residual, fault rows included)."""
        u = self.u if u is None else u
        out = self.F if out is None else out
        for i, ig in enumerate(self.domain + self.interfaces):
            ig.compute_lhs_residual(t, self.dt, u, out, mode=FA.INSERT if i == 0 else FA.ADD)
        return out

    def begin_step(self, t: float):
        """Everything of a step before the linear solve: the solution takes its Dirichlet values
        and the prescribed slip, F is the domain residual (the fault's lambda terms cancel in the
        reduced, slip-constrained space) and the solver is set up when its trigger fires. Returns
        (F, du): the solve is A du = F."""
        self.solver.insert_constrained(self._bc, self.u)
        for iface in self.interfaces:
            self.solver.apply_fault_slip(iface, self.u)
        for i, ig in enumerate(self.domain):
            ig.compute_lhs_residual(t, self.dt, self.u, self.F, mode=FA.INSERT if i == 0 else FA.ADD)
        if self._setup_dt is None or (self.viscous and self._setup_dt != self.dt):
            self.solver.setup(t, self.dt)
            self._setup_dt = self.dt
        return self.F, self.du

    def end_step(self, t: float) -> None:
        """After the solve: u += du and the state variables' update (poststep)."""
        self.u += self.du
        for ig in self.viscous:
            ig.update_state_vars(t, self.dt, self.u)

    def step(self, t: float) -> StepStats:
        F, du = self.begin_step(t)
        self.solver.solve(F, du)
        self.end_step(t)
        s = self.solver.stats()
        st = StepStats(t, s["iterations"], s["inner_iterations"], s["outer_iterations"], s["rel_residual"])
        self.history.append(st)
        return st

    def close(self) -> None:
        """Releases the device objects (solver, integrators, mesh) now rather than at collection."""
        self.solver.close()
        for ig in self.domain + self.interfaces:
            ig.close()
        self.dmesh.close()
