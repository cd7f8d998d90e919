"""Geometric multigrid hierarchy of a structured Q1 hexahedral box (with an optional planar fault at
x = x0 of cohesive cells), for the multigrid-preconditioned conjugate gradients of the device solver
(pl_multigrid_*).

The reference preconditions its elasticity solves with algebraic multigrid (PETSc GAMG, fine-level
smoother point-block Jacobi with faults; libsrc/pylith/materials/Elasticity.cc:298-330). The boxes
of the configurations this build runs are structured, so the hierarchy here is geometric: every
level is the same box with half the cells per direction (while the counts stay even), re-discretised
with the registered pointwise kernels on cell-averaged aux fields; the levels are tied by trilinear
prolongation, each side of the fault interpolating from its own side, and restriction is its
transpose. In the solver's reduced space (positive-side fault DOFs follow the negative side), the
device code unfolds the coarse vector before prolongation and folds the restricted one, so the
reduced restriction is the transpose of the reduced prolongation and the V-cycle is symmetric.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import meshing as M


@dataclass
class Level:
    n: tuple                 # cells per direction
    mesh: M.Mesh
    cell_parent: Optional[np.ndarray]  # for coarse levels: [8, ncells] fine cells of each coarse cell
    constrained: np.ndarray  # bool [num_dof]


def _node_maps(nx, ny, nz, fault_i):
    """For a box_hex(nx, ny, nz) (+ insert_fault_x at lattice index fault_i): the node id of lattice
    point (i, j, k) on the negative side and on the positive side (equal off the plane)."""
    base = np.arange((nx + 1) * (ny + 1) * (nz + 1)).reshape((nz + 1, ny + 1, nx + 1)).transpose(2, 1, 0)
    neg = base.copy()
    pos = base.copy()
    if fault_i is not None:
        plane = base[fault_i].ravel(order="F")  # the plane's nodes in increasing id order
        order = np.argsort(plane)
        copy = np.empty_like(plane)
        nn = (nx + 1) * (ny + 1) * (nz + 1)
        copy[order] = nn + np.arange(len(plane))
        pos[fault_i] = copy.reshape(base[fault_i].shape, order="F")
    return neg, pos


def _weights_1d(nf):
    """Fine index i = 0 .. nf -> two (coarse index, weight) pairs of 1-D linear interpolation
    (nf even): (i/2, 1) and (i/2, 0) for even i, (i//2, 1/2) and (i//2 + 1, 1/2) for odd i."""
    i = np.arange(nf + 1)
    c0 = i // 2
    odd = (i % 2).astype(bool)
    return c0, np.where(odd, 0.5, 1.0), np.where(odd, c0 + 1, c0), np.where(odd, 0.5, 0.0)


def prolongation(nf, fault_i_f, nc, fault_i_c, num_nodes_f, num_nodes_c):
    """CSR (row_ptr, col, val) of the node prolongation from a coarse box (nc) to the fine box
    nf = 2 nc: trilinear weights, fine nodes of the +x side (x > x0, and the plane's positive
    copies) interpolating from the coarse +x side."""
    negf, posf = _node_maps(*nf, fault_i_f)
    negc, posc = _node_maps(*nc, fault_i_c)
    w = [_weights_1d(n) for n in nf]
    I, J, K = np.meshgrid(np.arange(nf[0] + 1), np.arange(nf[1] + 1), np.arange(nf[2] + 1), indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    rows, cols, vals = [], [], []
    sides = [("neg", negf, negc, I <= (fault_i_f if fault_i_f is not None else nf[0]))]
    if fault_i_f is not None:
        sides.append(("pos", posf, posc, I >= fault_i_f))
    for _, fmap, cmap, sel in sides:
        i, j, k = I[sel], J[sel], K[sel]
        f = fmap[i, j, k]
        for a in (0, 1):
            ci, wa = w[0][2 * a][i], w[0][2 * a + 1][i]
            for b in (0, 1):
                cj, wb = w[1][2 * b][j], w[1][2 * b + 1][j]
                for c in (0, 1):
                    ck, wc = w[2][2 * c][k], w[2][2 * c + 1][k]
                    wt = wa * wb * wc
                    keep = wt != 0.0
                    rows.append(f[keep])
                    cols.append(cmap[ci[keep], cj[keep], ck[keep]])
                    vals.append(wt[keep])
    rows, cols, vals = np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    row_ptr = np.zeros(num_nodes_f + 1, dtype=np.int32)
    np.add.at(row_ptr, rows + 1, 1)
    return np.cumsum(row_ptr).astype(np.int32), cols.astype(np.int32), vals.astype(np.float64)


def build_hierarchy(nx, ny, nz, lo=M.BOX_LO, hi=M.BOX_HI, fault_x: Optional[float] = None,
                    constrained_faces=(), min_cells: int = 2, max_levels: int = 8) -> List[Level]:
    """Levels 0 (the fine box) .. L of a box_hex(nx, ny, nz) [+ insert_fault_x(fault_x)] with
    Dirichlet constraints on whole faces: constrained_faces = [(axis, side, components)], e.g.
    (0, "neg", (0, 1, 2)). Coarsening stops when a count is odd or below 2 * min_cells."""
    levels = []
    n = (nx, ny, nz)
    parent = None
    while True:
        mesh = M.box_hex(*n, lo=lo, hi=hi)
        fault_i = None
        if fault_x is not None:
            h = (hi[0] - lo[0]) / n[0]
            fault_i = int(round((fault_x - lo[0]) / h))
            mesh = M.insert_fault_x(mesh, fault_x)
        cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
        for axis, side, comps in constrained_faces:
            cons[np.ix_(M.boundary_mask(mesh, axis, side, lo, hi), list(comps))] = True
        cons = np.concatenate([cons.ravel(), np.zeros(3 * mesh.num_lagrange, dtype=bool)])
        levels.append(Level(n, mesh, parent, cons))
        if len(levels) >= max_levels or any(v % 2 or v < 2 * min_cells for v in n):
            break
        if fault_x is not None and (fault_i % 2):
            break
        nc = tuple(v // 2 for v in n)
        # the 8 fine cells of each coarse cell (box_hex orders cells with i fastest)
        ci, cj, ck = np.meshgrid(np.arange(nc[0]), np.arange(nc[1]), np.arange(nc[2]), indexing="ij")
        ci, cj, ck = (a.ravel(order="F") for a in (ci, cj, ck))
        kids = []
        for di in (0, 1):
            for dj in (0, 1):
                for dk in (0, 1):
                    kids.append((2 * ci + di) + n[0] * ((2 * cj + dj) + n[1] * (2 * ck + dk)))
        parent = np.stack(kids)
        n = nc
    return levels


def coarsen_cells(values: np.ndarray, parent: np.ndarray) -> np.ndarray:
    """Per-cell values of a coarse level: the mean over each coarse cell's 8 fine cells."""
    return values[parent].mean(axis=0)


def prolongations(levels: List[Level], fault_x: Optional[float], lo=M.BOX_LO, hi=M.BOX_HI):
    """[(row_ptr, col, val)] of the prolongation from level l + 1 to level l, l = 0 .. L - 1."""
    out = []
    for lf, lc in zip(levels[:-1], levels[1:]):
        fi = fc = None
        if fault_x is not None:
            fi = int(round((fault_x - lo[0]) / ((hi[0] - lo[0]) / lf.n[0])))
            fc = fi // 2
        out.append(prolongation(lf.n, fi, lc.n, fc, lf.mesh.num_nodes, lc.mesh.num_nodes))
    return out


def coarsen_material(mat, parent):
    """The material of a coarse level: every per-cell field averaged over the 8 fine cells of each
    coarse cell; per-quadrature-point state starts at zero (the Jacobians read no state)."""
    from . import materials as MAT

    cc = lambda v: coarsen_cells(np.asarray(v), parent)  # noqa: E731
    if isinstance(mat, MAT.IsotropicLinearGenMaxwell):
        nc = parent.shape[1]
        return MAT.IsotropicLinearGenMaxwell(cc(mat.density), cc(mat.shear_modulus), cc(mat.bulk_modulus),
                                             cc(mat.maxwell_time), cc(mat.shear_modulus_ratio),
                                             np.zeros((nc, 8, 18)), np.zeros((nc, 8, 6)))
    bf = None if mat.body_force is None else cc(mat.body_force)
    return MAT.IsotropicLinearElasticity(cc(mat.density), cc(mat.shear_modulus), cc(mat.bulk_modulus), bf)


def attach(ctx, fine_solver, levels: List[Level], material, fault_x=None, dt=0.0, lo=M.BOX_LO, hi=M.BOX_HI,
           degree=2, lower=0.1, coarse_degree=40, coarse_lower=0.01, precision=None):
    """Builds the coarse levels' device meshes, integrators (the fine material coarsened level by
    level) and solvers, and attaches the multigrid preconditioner to `fine_solver`; returns the
    FA.Multigrid (keep it alive with the solver). Call fine_solver.setup afterwards."""
    from . import feassemble as FA
    from . import materials as MAT

    if precision is None:
        precision = FA.Solver.FP64
    keep = []
    coarse = []
    mat = material
    for lv in levels[1:]:
        mat = coarsen_material(mat, lv.cell_parent)
        dm = FA.DeviceMesh(ctx, lv.mesh)
        ig = mat.create_integrator(dm, dt) if isinstance(mat, MAT.IsotropicLinearGenMaxwell) else mat.create_integrator(dm)
        s = FA.Solver(dm, lv.constrained, [ig])
        keep += [dm, ig]
        coarse.append(s)
    mg = FA.Multigrid(fine_solver, coarse, prolongations(levels, fault_x, lo, hi), degree, lower, coarse_degree,
                      coarse_lower, precision)
    mg._keep = keep
    return mg
