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
from ._lib import PylithB200Error

PL_ERR_UNSUPPORTED = -7  # include/pylith_b200.h


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
    observers: list = field(default_factory=list)  # OutputObserver: written after every step

    def __post_init__(self):
        import torch

        self.dmesh = FA.DeviceMesh(self.ctx, self.mesh)
        self.domain: List[FA.IntegratorDomain] = []
        self.viscous: List[FA.IntegratorDomain] = []
        self.domain_cells: List[np.ndarray] = []  # mesh cell ids of each domain integrator
        for mat, ids in self.materials:
            self.domain_cells.append(np.arange(self.mesh.num_cells) if ids is None else np.asarray(ids))
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
        for obs in self.observers:  # poststep: notify the observers (TimeDependent.cc:490-538)
            obs.update(self, t, len(self.history) - 1)
        return st

    def close(self) -> None:
        """Releases the device objects (solver, integrators, mesh) now rather than at collection;
        closes the observers' writers."""
        for obs in self.observers:
            obs.close()
        self.solver.close()
        for ig in self.domain + self.interfaces:
            ig.close()
        self.dmesh.close()


@dataclass
class OutputObserver:
    """The reference's solution and material observers over one writer (OutputSolnDomain,
    meshio/OutputSolnDomain.cc, and OutputPhysics, meshio/OutputPhysics.cc), triggered every
    num_steps_skip + 1 steps (OutputTriggerStep::shouldWrite, meshio/OutputTriggerStep.cc:54-66:
    a step is written when its index exceeds the last written one by more than num_steps_skip).

    At a written step the solution's displacement goes out as a vertex field and, when
    `derived` is set, every domain integrator's registered derived fields (cauchy_stress,
    cauchy_strain: basis order 0, pl_compute_derived_field) as cell fields over the whole mesh,
    each integrator filling its own cells. The writer is an output.DataWriterHDF5,
    DataWriterHDF5Ext or DataWriterVTK (one file per step, into `directory`); it is opened on the
    problem's mesh at the first update and closed by close()."""

    writer: object
    num_steps_skip: int = 0
    derived: bool = True  # (integrators whose derived fields the device does not evaluate for
    directory: str = "."  # their cell type, PL_ERR_UNSUPPORTED, are left out)
    _step_wrote: int = -(1 << 30)
    _opened: bool = False

    def should_write(self, tindex: int) -> bool:
        if tindex - self._step_wrote > self.num_steps_skip:
            self._step_wrote = tindex
            return True
        return False

    def _fields(self, problem, t: float):
        import torch

        nn = problem.mesh.num_nodes
        vertex = [("displacement", problem.u[:3 * nn].reshape(nn, 3).cpu().numpy(), "vector")]
        cell = []
        if self.derived:
            out = {}
            for ig, ids in zip(problem.domain, problem.domain_cells):
                names = getattr(ig, "derived_subfields", [])
                if not names:
                    continue
                vals = torch.empty((len(ids), 6 * len(names)), dtype=torch.float64, device="cuda")
                try:
                    ig.compute_derived_field(t, problem.dt, problem.u, vals)
                except PylithB200Error as e:
                    if e.code != PL_ERR_UNSUPPORTED:
                        raise
                    continue  # no device evaluation of these fields for this cell type
                v = vals.cpu().numpy()
                for k, name in enumerate(names):
                    full = out.setdefault(name, np.zeros((problem.mesh.num_cells, 6)))
                    full[ids] = v[:, 6 * k:6 * k + 6]
            cell = [(name, v, "tensor") for name, v in out.items()]
        return vertex, cell

    def update(self, problem, t: float, tindex: int) -> None:
        if not self.should_write(tindex):
            return
        w = self.writer
        if not self._opened:
            w.open(problem.mesh)
            self._opened = True
        vertex, cell = self._fields(problem, t)
        if hasattr(w, "open_time_step"):  # VTK: one file per step
            w.open_time_step(t)
            for name, v, vtype in vertex:
                w.write_vertex_field(name, v, vector=vtype == "vector")
            for name, v, _ in cell:
                w.write_cell_field(name, v)
            w.close_time_step(self.directory)
        else:
            for name, v, vtype in vertex:
                w.write_vertex_field(t, name, v, vector_field_type=vtype)
            for name, v, vtype in cell:
                w.write_cell_field(t, name, v, vector_field_type=vtype)

    def close(self) -> None:
        if self._opened:
            self.writer.close()
            self._opened = False


@dataclass
class OutputPointsObserver:
    """The reference's station observer (OutputSolnPoints, meshio/OutputSolnPoints.cc:110-140)
    over one writer: every num_steps_skip + 1 steps (OutputTriggerStep) the displacement
    interpolated at named points (output.PointInterpolator, the counterpart of DMInterpolation)
    goes to a file of a point mesh, with the names in /stations written before the first step
    (output.read_points_list reads PyLith's points files)."""

    writer: object
    names: list
    points: np.ndarray
    num_steps_skip: int = 0
    _step_wrote: int = -(1 << 30)
    _interp: Optional[object] = None

    def update(self, problem, t: float, tindex: int) -> None:
        if tindex - self._step_wrote <= self.num_steps_skip:
            return
        self._step_wrote = tindex
        from . import output as OUT

        if self._interp is None:
            self._interp = OUT.PointInterpolator(problem.mesh, self.points)
            self.writer.open(OUT.PointMesh(np.asarray(self.points, dtype=np.float64).reshape(-1, 3)))
            self.writer.write_point_names(list(self.names))
        disp = self._interp(problem.u).cpu().numpy()
        self.writer.write_vertex_field(t, "displacement", disp, vector_field_type="vector")

    def close(self) -> None:
        if self._interp is not None:
            self.writer.close()
