"""Geometric multigrid hierarchy of a structured Q1 hexahedral box (with an optional planar fault at
x = x0 of cohesive cells), for the multigrid-preconditioned conjugate gradients of the device solver
(pl_multigrid_*).

The reference preconditions its elasticity solves with algebraic multigrid (PETSc GAMG, fine-level
smoother point-block Jacobi with faults; libsrc/pylith/materials/Elasticity.cc:298-330). The boxes
of the benchmarked configurations are structured, so the hierarchy here is geometric: every
level is the same box with about half the cells per direction (exactly half while that keeps the
fault plane a grid plane; otherwise the nearest count that does, so the grids need not be nested),
re-discretised with the registered pointwise kernels on cell-averaged aux fields; the levels are
tied by trilinear interpolation (the prolongation), each side of the fault interpolating from its
own side, and restriction is its transpose. In the solver's reduced space (positive-side fault DOFs follow the negative side), the
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
    cell_map: Optional[np.ndarray]  # for coarse levels: this level's cell holding each cell of the finer level
    constrained: np.ndarray  # bool [num_dof]
    prolong: Optional[tuple] = None  # CSR (row_ptr, col, val) from the next coarser level to this one


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


def _weights_1d(nf, nc):
    """Fine index i = 0 .. nf of a uniform grid of nf cells -> two (coarse index, weight) pairs of
    1-D linear interpolation from the grid of nc <= nf cells over the same interval: with
    s = i nc / nf (exact integer arithmetic), (floor s, 1 - frac s) and (floor s + 1, frac s),
    floor s capped at nc - 1."""
    i = np.arange(nf + 1, dtype=np.int64)
    c0 = np.minimum((i * nc) // nf, nc - 1)
    w1 = (i * nc - c0 * nf) / nf
    return c0, 1.0 - w1, c0 + 1, w1


def prolongation(nf, fault_i_f, nc, fault_i_c, num_nodes_f, num_nodes_c):
    """CSR (row_ptr, col, val) of the node prolongation from a coarse box (nc cells per direction)
    to a fine box of the same extent (nf >= nc; nested or not): trilinear interpolation weights, fine nodes of the +x side (x > x0, and the plane's positive
    copies) interpolating from the coarse +x side. Every fine node is one (side, lattice point)
    pair, so the rows are laid out by scattering those pairs to their node ids; within a row the
    entries are in increasing column order, zero weights left out."""
    negf, posf = _node_maps(*nf, fault_i_f)
    negc, posc = _node_maps(*nc, fault_i_c)
    w = [_weights_1d(a, b) for a, b in zip(nf, nc)]
    I, J, K = np.meshgrid(np.arange(nf[0] + 1), np.arange(nf[1] + 1), np.arange(nf[2] + 1), indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    sides = [(negf, negc, I <= (fault_i_f if fault_i_f is not None else nf[0]))]
    if fault_i_f is not None:
        sides.append((posf, posc, I >= fault_i_f))
    cols = np.empty((num_nodes_f, 8), dtype=np.int64)
    vals = np.empty((num_nodes_f, 8), dtype=np.float64)
    seen = np.zeros(num_nodes_f, dtype=np.int32)
    sc = (nc[1] + 1) * (nc[2] + 1), nc[2] + 1  # strides of a C-ordered (i, j, k) coarse lattice
    for fmap, cmap, sel in sides:
        i, j, k = I[sel], J[sel], K[sel]
        f = fmap.ravel()[(i * (nf[1] + 1) + j) * (nf[2] + 1) + k]
        cflat = cmap.ravel()
        seen[f] += 1
        C = np.empty((8, len(f)), dtype=np.int64)
        W = np.empty((8, len(f)), dtype=np.float64)
        e = 0
        for a in (0, 1):
            ci, wa = w[0][2 * a][i], w[0][2 * a + 1][i]
            for b in (0, 1):
                cj, wb = w[1][2 * b][j], w[1][2 * b + 1][j]
                for c in (0, 1):
                    ck, wc = w[2][2 * c][k], w[2][2 * c + 1][k]
                    C[e] = cflat[ci * sc[0] + cj * sc[1] + ck]
                    W[e] = wa * wb * wc
                    e += 1
        cols[f] = C.T
        vals[f] = W.T
    if not np.all(seen == 1):
        raise ValueError("prolongation: fine node ids do not match one (side, lattice point) each")
    keep = vals != 0.0
    order = np.argsort(np.where(keep, cols, np.iinfo(np.int64).max), axis=1, kind="stable")
    cols = np.take_along_axis(cols, order, axis=1)
    vals = np.take_along_axis(vals, order, axis=1)
    keep = np.take_along_axis(keep, order, axis=1)
    row_ptr = np.zeros(num_nodes_f + 1, dtype=np.int64)
    np.cumsum(keep.sum(axis=1), out=row_ptr[1:])
    return row_ptr.astype(np.int32), cols[keep].astype(np.int32), vals[keep]


def _coarse_count(v: int, fault_i: Optional[int]) -> Optional[int]:
    """Cells of the next coarser grid along an axis of v cells: v / 2 when v is even (and the fault
    plane, at lattice index fault_i, stays a grid plane), else the count nearest v / 2 that keeps it
    one; None when there is none."""
    if fault_i is None:
        return v // 2 if v % 2 == 0 else (v + 1) // 2
    for m in sorted(range(max(1, v // 2 - 2), v // 2 + 3), key=lambda m: (abs(2 * m - v), m)):
        if m < v and (fault_i * m) % v == 0:
            return m
    return None


def _cell_map(nf, nc):
    """The coarse cell (box_hex numbering, i fastest) holding each fine cell's centroid."""
    ax = [((2 * np.arange(a) + 1) * b) // (2 * a) for a, b in zip(nf, nc)]
    ci, cj, ck = np.meshgrid(ax[0], ax[1], ax[2], indexing="ij")
    ci, cj, ck = (x.ravel(order="F") for x in (ci, cj, ck))
    return (ci + nc[0] * (cj + nc[1] * ck)).astype(np.int64)


# A level with at most this many nodes is small enough to be the coarsest: the device solver
# inverts its reduced matrix (up to 1536 unknowns) instead of smoothing it.
MAX_COARSE_NODES = 512


def build_hierarchy(nx, ny, nz, lo=M.BOX_LO, hi=M.BOX_HI, fault_x: Optional[float] = None,
                    constrained_faces=(), min_cells: int = 2, max_levels: int = 8,
                    max_coarse_nodes: int = MAX_COARSE_NODES) -> List[Level]:
    """Levels 0 (the fine box) .. L of a box_hex(nx, ny, nz) [+ insert_fault_x(fault_x)] with
    Dirichlet constraints on whole faces: constrained_faces = [(axis, side, components)], e.g.
    (0, "neg", (0, 1, 2)). Each coarser level has about half the cells per direction
    (_coarse_count); coarsening stops at a level of at most max_coarse_nodes nodes, or when a count
    would drop below min_cells. Each level but the coarsest carries the prolongation from the next
    coarser one (Level.prolong)."""
    levels = []
    n = (nx, ny, nz)
    cmap = None
    fault_is = []
    while True:
        mesh = M.box_hex(*n, lo=lo, hi=hi)
        fault_i = None
        if fault_x is not None:
            t = (fault_x - lo[0]) / ((hi[0] - lo[0]) / n[0])
            fault_i = int(round(t))
            if abs(t - fault_i) > 1e-9 * max(1.0, abs(t)) or not 0 < fault_i < n[0]:
                raise ValueError(f"fault plane x = {fault_x} is not an interior grid plane of {n[0]} cells")
            mesh = M.insert_fault_x(mesh, fault_x)
        fault_is.append(fault_i)
        cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
        for axis, side, comps in constrained_faces:
            cons[np.ix_(M.boundary_mask(mesh, axis, side, lo, hi), list(comps))] = True
        cons = np.concatenate([cons.ravel(), np.zeros(3 * mesh.num_lagrange, dtype=bool)])
        levels.append(Level(n, mesh, cmap, cons))
        if len(levels) >= max_levels or (len(levels) > 1 and mesh.num_nodes <= max_coarse_nodes):
            break
        nc = (_coarse_count(n[0], fault_i), _coarse_count(n[1], None), _coarse_count(n[2], None))
        if any(m is None or m < min_cells for m in nc):
            break
        cmap = _cell_map(n, nc)
        n = nc
    for l, (lf, lc) in enumerate(zip(levels[:-1], levels[1:])):
        lf.prolong = prolongation(lf.n, fault_is[l], lc.n, fault_is[l + 1], lf.mesh.num_nodes, lc.mesh.num_nodes)
    return levels


def coarsen_cells(values: np.ndarray, cell_map) -> np.ndarray:
    """Per-cell values of a coarse level: the mean over the finer level's cells whose centroids lie
    in each coarse cell (cell_map: the coarse cell of each fine cell, or a sparse row-normalised
    [coarse cells x fine cells] averaging matrix)."""
    if not isinstance(cell_map, np.ndarray):
        v = np.asarray(values, dtype=np.float64)
        return np.asarray(cell_map @ v.reshape(v.shape[0], -1)).reshape((cell_map.shape[0],) + v.shape[1:])
    nc = int(cell_map.max()) + 1
    cnt = np.bincount(cell_map, minlength=nc).astype(np.float64)
    v = np.asarray(values, dtype=np.float64)
    flat = v.reshape(len(cell_map), -1)
    out = np.stack([np.bincount(cell_map, weights=flat[:, j], minlength=nc) / cnt for j in range(flat.shape[1])], axis=1)
    return out.reshape((nc,) + v.shape[1:])


def prolongations(levels: List[Level], fault_x: Optional[float], lo=M.BOX_LO, hi=M.BOX_HI):
    """[(row_ptr, col, val)] of the prolongation from level l + 1 to level l, l = 0 .. L - 1 (the
    ones build_hierarchy stored with the levels, else built here)."""
    out = []
    for lf, lc in zip(levels[:-1], levels[1:]):
        if lf.prolong is not None:
            out.append(lf.prolong)
            continue
        fi = fc = None
        if fault_x is not None:
            fi = int(round((fault_x - lo[0]) / ((hi[0] - lo[0]) / lf.n[0])))
            fc = int(round((fault_x - lo[0]) / ((hi[0] - lo[0]) / lc.n[0])))
        out.append(prolongation(lf.n, fi, lc.n, fc, lf.mesh.num_nodes, lc.mesh.num_nodes))
    return out


def coarsen_material(mat, cell_map):
    """The material of a coarse level: every per-cell field averaged over the finer level's cells
    of each coarse cell (coarsen_cells); per-quadrature-point state starts at zero (the Jacobians
    read no state)."""
    from . import materials as MAT

    cc = lambda v: coarsen_cells(np.asarray(v), cell_map)  # noqa: E731
    if isinstance(mat, MAT.IsotropicLinearGenMaxwell):
        nc = cell_map.shape[0] if not isinstance(cell_map, np.ndarray) else int(cell_map.max()) + 1
        return MAT.IsotropicLinearGenMaxwell(cc(mat.density), cc(mat.shear_modulus), cc(mat.bulk_modulus),
                                             cc(mat.maxwell_time), cc(mat.shear_modulus_ratio),
                                             np.zeros((nc, 8, 18)), np.zeros((nc, 8, 6)))
    bf = None if mat.body_force is None else cc(mat.body_force)
    return MAT.IsotropicLinearElasticity(cc(mat.density), cc(mat.shear_modulus), cc(mat.bulk_modulus), bf)


# ---- unstructured tetrahedral hierarchies ------------------------------------------------------
# A P1 tetrahedral mesh has no halving; its coarser levels are independent meshes of the same
# domain with about 1/8 of the cells (for the mirrored Delaunay meshes with a fault, the same
# construction with fewer points), tied by the interpolation of the coarse P1 space at the fine
# nodes: each fine node is located in a coarse cell of its own side of the fault and takes that
# cell's barycentric weights. The interpolation is exact for fields linear on each side, nodes on a
# box face or on the fault plane interpolate from that face's or plane's coarse nodes only, and the
# cell averages use the coarse cell that holds each fine cell's centroid.


def node_sides(mesh, fault_x: Optional[float]) -> np.ndarray:
    """+1 / -1 per node: the side of the fault plane x = fault_x (the plane's negative-side copies
    are -1, its positive-side copies +1); all +1 without a fault."""
    if fault_x is None:
        return np.ones(mesh.num_nodes, dtype=np.int8)
    side = np.where(mesh.coords[:, 0] < fault_x, -1, 1).astype(np.int8)
    if mesh.cohesive is not None and len(mesh.cohesive):
        side[mesh.cohesive[:, :4].ravel()] = -1
        side[mesh.cohesive[:, 4:8].ravel()] = 1
    return side


def _cell_sides(mesh, fault_x: Optional[float]) -> np.ndarray:
    if fault_x is None:
        return np.ones(mesh.num_cells, dtype=np.int8)
    return np.where(mesh.coords[mesh.cells].mean(axis=1)[:, 0] < fault_x, -1, 1).astype(np.int8)


def _node_cell_index(mesh, cside):
    """Per side: a KD-tree of the nodes of that side's cells, and for every node the side's cells
    around it."""
    from scipy.spatial import cKDTree

    trees, cells_of = {}, {}
    for sgn in (-1, 1):
        ids = np.flatnonzero(cside == sgn)
        if len(ids) == 0:
            continue
        flat = mesh.cells[ids].ravel()
        order = np.argsort(flat, kind="stable")
        nodes, starts = np.unique(flat[order], return_index=True)
        owners = np.repeat(ids, 4)[order]
        bounds = np.append(starts, len(order))
        cells_of[sgn] = {int(v): owners[bounds[i]:bounds[i + 1]] for i, v in enumerate(nodes)}
        trees[sgn] = (cKDTree(mesh.coords[nodes]), nodes)
    return trees, cells_of


def locate_in_tets(mesh, points: np.ndarray, point_sides: np.ndarray, fault_x: Optional[float],
                   k: int = 12, chunk: int = 100_000):
    """For each point, a cell of `mesh` (P1 tetrahedra) on the point's side that holds it, and the
    point's barycentric coordinates there ([m, 4], negatives of rounding clipped, rows summing to
    one). Candidates are the k cells with the nearest centroids (64 for points none of those hold);
    the cell whose smallest barycentric coordinate is largest wins."""
    from scipy.spatial import cKDTree

    X = mesh.coords[mesh.cells]  # [nc, 4, 3]
    X0 = X[:, 0]
    M = np.transpose(X[:, 1:] - X0[:, None, :], (0, 2, 1))  # columns = edge vectors
    Minv = np.linalg.inv(M)
    cside = _cell_sides(mesh, fault_x)
    cell = np.empty(len(points), dtype=np.int64)
    bary = np.empty((len(points), 4))
    node_tree = node_cells = None
    for sgn in (-1, 1):
        ids = np.flatnonzero(cside == sgn)
        sel = np.flatnonzero(point_sides == sgn)
        if len(sel) == 0:
            continue
        if len(ids) == 0:
            raise ValueError("no coarse cells on a side that holds fine points")
        tree = cKDTree(X[ids].mean(axis=1))
        for c0 in range(0, len(sel), chunk):
            part = sel[c0:c0 + chunk]
            P = points[part]
            best_c = np.zeros(len(part), dtype=np.int64)
            best_b = np.full((len(part), 4), -np.inf)
            todo = np.arange(len(part))
            for kk in (min(k, len(ids)), min(64, len(ids))):
                if len(todo) == 0:
                    break
                _, cand = tree.query(P[todo], k=kk)
                cand = ids[np.asarray(cand).reshape(len(todo), kk)]
                lam = np.einsum("mkij,mkj->mki", Minv[cand], P[todo][:, None, :] - X0[cand])
                b4 = np.concatenate([1.0 - lam.sum(axis=2, keepdims=True), lam], axis=2)
                score = b4.min(axis=2)
                j = score.argmax(axis=1)
                better = score[np.arange(len(todo)), j] > best_b[todo].min(axis=1)
                upd = todo[better]
                best_c[upd] = cand[better, j[better]]
                best_b[upd] = b4[better, j[better]]
                todo = todo[best_b[todo].min(axis=1) < -1e-9]
            if len(todo):
                # slivers: a cell can hold a point far from its centroid; try every cell around
                # the point's nearest coarse nodes (few points take this path)
                if node_tree is None:
                    node_tree, node_cells = _node_cell_index(mesh, cside)
                tree_s, nodes_s = node_tree[sgn]
                for t in todo:
                    _, nn = tree_s.query(P[t], k=min(16, tree_s.n))
                    cand = np.unique(np.concatenate([node_cells[sgn][int(v)] for v in nodes_s[np.atleast_1d(nn)]]))
                    lam = np.einsum("kij,kj->ki", Minv[cand], P[t][None, :] - X0[cand])
                    b4 = np.concatenate([1.0 - lam.sum(axis=1, keepdims=True), lam], axis=1)
                    j = b4.min(axis=1).argmax()
                    if b4[j].min() > best_b[t].min():
                        best_c[t], best_b[t] = cand[j], b4[j]
            cell[part] = best_c
            bary[part] = best_b
    bary = np.clip(bary, 0.0, None)
    bary /= bary.sum(axis=1, keepdims=True)
    return cell, bary


def tet_prolongation(fine, coarse, fault_x: Optional[float]):
    """CSR (row_ptr, col, val) of the interpolation of the coarse P1 space at the fine mesh's nodes
    (rows: fine nodes; columns: coarse nodes), each node from a coarse cell of its own side."""
    cell, bary = locate_in_tets(coarse, fine.coords, node_sides(fine, fault_x), fault_x)
    cols = coarse.cells[cell].astype(np.int64)
    keep = bary > 1e-12
    # rows are in node order already (one located cell per fine node)
    row_ptr = np.zeros(fine.num_nodes + 1, dtype=np.int64)
    np.cumsum(keep.sum(axis=1), out=row_ptr[1:])
    val = bary[keep]
    rs = np.add.reduceat(val, row_ptr[:-1]) if len(val) else val
    val = val / np.repeat(rs, np.diff(row_ptr))
    return row_ptr.astype(np.int32), cols[keep].astype(np.int32), val


def tet_cell_average(fine, coarse, fault_x: Optional[float]):
    """Sparse row-normalised [coarse cells x fine cells] averaging matrix: each coarse cell averages
    the fine cells whose centroids it holds (a coarse cell that holds none takes the fine cell
    nearest its own centroid on its side)."""
    import scipy.sparse as sp
    from scipy.spatial import cKDTree

    fc = fine.coords[fine.cells].mean(axis=1)
    fside = _cell_sides(fine, fault_x)
    cell, _ = locate_in_tets(coarse, fc, fside, fault_x)
    rows, cols = [cell], [np.arange(fine.num_cells)]
    empty = np.setdiff1d(np.arange(coarse.num_cells), cell)
    if len(empty):
        cc = coarse.coords[coarse.cells[empty]].mean(axis=1)
        cside = _cell_sides(coarse, fault_x)[empty]
        near = np.empty(len(empty), dtype=np.int64)
        for sgn in (-1, 1):
            e = np.flatnonzero(cside == sgn)
            f = np.flatnonzero(fside == sgn)
            if len(e):
                near[e] = f[cKDTree(fc[f]).query(cc[e])[1]]
        rows.append(empty)
        cols.append(near)
    r, c = np.concatenate(rows), np.concatenate(cols)
    W = sp.csr_matrix((np.ones(len(r)), (r, c)), shape=(coarse.num_cells, fine.num_cells))
    cnt = np.asarray(W.sum(axis=1)).ravel()
    return sp.diags(1.0 / cnt) @ W


def build_tet_hierarchy(fine, make_mesh, fault_x: Optional[float] = None, lo=M.BOX_LO, hi=M.BOX_HI,
                        constrained_faces=(), ratio: int = 8, min_cells: int = 2000,
                        max_levels: int = 6, max_coarse_nodes: int = MAX_COARSE_NODES) -> List[Level]:
    """Levels of a P1 tetrahedral mesh `fine`: level l + 1 is make_mesh(cells of level l / ratio,
    l + 1), a mesh of the same box (with the same fault plane), built while it keeps at least
    min_cells cells and the level above has more than max_coarse_nodes nodes. Each level but the
    coarsest carries its prolongation (tet_prolongation), each coarse level the cell averaging from
    the level above (Level.cell_map: a sparse matrix)."""

    def constraints(mesh):
        cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
        for axis, side, comps in constrained_faces:
            cons[np.ix_(M.boundary_mask(mesh, axis, side, lo, hi), list(comps))] = True
        return np.concatenate([cons.ravel(), np.zeros(3 * mesh.num_lagrange, dtype=bool)])

    levels = [Level(None, fine, None, constraints(fine))]
    while len(levels) < max_levels and levels[-1].mesh.num_nodes > max_coarse_nodes:
        target = levels[-1].mesh.num_cells // ratio
        if target < min_cells:
            break
        coarse = make_mesh(target, len(levels))
        lf = levels[-1]
        lf.prolong = tet_prolongation(lf.mesh, coarse, fault_x)
        levels.append(Level(None, coarse, tet_cell_average(lf.mesh, coarse, fault_x), constraints(coarse)))
    return levels


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
        mat = coarsen_material(mat, lv.cell_map)
        dm = FA.DeviceMesh(ctx, lv.mesh)
        ig = mat.create_integrator(dm, dt) if isinstance(mat, MAT.IsotropicLinearGenMaxwell) else mat.create_integrator(dm)
        s = FA.Solver(dm, lv.constrained, [ig])
        keep += [dm, ig]
        coarse.append(s)
    mg = FA.Multigrid(fine_solver, coarse, prolongations(levels, fault_x, lo, hi), degree, lower, coarse_degree,
                      coarse_lower, precision)
    mg._keep = keep
    return mg
