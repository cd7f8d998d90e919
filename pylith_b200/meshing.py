"""Seeded synthetic meshes for the residual/Jacobian path.

The reference reads meshes through PETSc/Gmsh/ExodusII readers
(libsrc/pylith/meshio/MeshIOPetsc.cc, MeshIOCubit.cc) and inserts cohesive
cells with DMPlexTransform (libsrc/pylith/faults/TopologyOps.cc:26-310). Those
readers and PETSc are not part of this path, so the benchmark meshes are built
here directly, with the same geometry as the reference's test boxes
(tests/fullscale/linearelasticity/nofaults-3d: [-6000,6000]^2 x [-9000,0] m).

Conventions (shared with the CUDA kernels and the oracle):
  * coordinates: float64 [nnodes, 3];
  * Q1 hexahedra: int32 [ncells, 8], corners (0,0,0),(1,0,0),(1,1,0),(0,1,0),
    (0,0,1),(1,0,1),(1,1,1),(0,1,1) in (x, y, z) lattice steps;
  * Q2 hexahedra: int32 [ncells, 27], node (a, b, c) in {0,1,2}^3 at local
    index a + 3 b + 9 c; nodes 0, 2, 8, 6, 18, 20, 26, 24 are the corners;
  * P1 tetrahedra: int32 [ncells, 4], positively oriented;
  * cohesive cells: int32 [ncoh, 12], negative-side face vertices (4),
    positive-side vertices (4), Lagrange-multiplier nodes (4); the face normal
    (dx/dxi x dx/deta) from the negative-side order points to the positive side.
"""
from __future__ import annotations

import dataclasses

import numpy as np

BOX_LO = (-6000.0, -6000.0, -9000.0)
BOX_HI = (6000.0, 6000.0, 0.0)

CELL_TET4 = 0
CELL_HEX8 = 1
CELL_HEX27 = 2

NODES_PER_CELL = {CELL_TET4: 4, CELL_HEX8: 8, CELL_HEX27: 27}
QUAD_POINTS = {CELL_TET4: 1, CELL_HEX8: 8, CELL_HEX27: 27}

_HEX_CORNERS = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                         [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=np.int64)


@dataclasses.dataclass
class Mesh:
    cell_type: int
    coords: np.ndarray          # float64 [nnodes, 3]
    cells: np.ndarray           # int32 [ncells, nodes_per_cell]
    cohesive: np.ndarray | None = None  # int32 [ncoh, 12]
    num_lagrange: int = 0       # Lagrange-multiplier nodes (fault vertices)

    @property
    def num_cells(self) -> int:
        return int(self.cells.shape[0])

    @property
    def num_nodes(self) -> int:
        return int(self.coords.shape[0])

    @property
    def num_dof(self) -> int:
        return 3 * (self.num_nodes + self.num_lagrange)

    def corner_nodes(self) -> np.ndarray:
        """Geometry (corner) node of every cell, in the Q1 corner order."""
        if self.cell_type == CELL_HEX27:
            idx = [a + 3 * b + 9 * c for (a, b, c) in (2 * _HEX_CORNERS)]
            return self.cells[:, idx]
        return self.cells


def box_hex(nx: int, ny: int, nz: int, lo=BOX_LO, hi=BOX_HI) -> Mesh:
    """Uniform Q1 hexahedral box with nx*ny*nz cells."""
    xs = [np.linspace(lo[d], hi[d], n + 1) for d, n in enumerate((nx, ny, nz))]
    X, Y, Z = np.meshgrid(*xs, indexing="ij")
    coords = np.stack([X.ravel(order="F"), Y.ravel(order="F"), Z.ravel(order="F")], axis=1)
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    i, j, k = (a.ravel(order="F") for a in (i, j, k))
    node = lambda a, b, c: a + (nx + 1) * (b + (ny + 1) * c)  # noqa: E731
    cells = np.stack([node(i + ci, j + cj, k + ck) for (ci, cj, ck) in _HEX_CORNERS], axis=1)
    return Mesh(CELL_HEX8, np.ascontiguousarray(coords), cells.astype(np.int32))


def box_hex27(nx: int, ny: int, nz: int, lo=BOX_LO, hi=BOX_HI) -> Mesh:
    """Uniform Q2 hexahedral box: a (2n+1)^3 node lattice, 27 nodes per cell."""
    mx, my, mz = 2 * nx + 1, 2 * ny + 1, 2 * nz + 1
    xs = [np.linspace(lo[d], hi[d], m) for d, m in enumerate((mx, my, mz))]
    X, Y, Z = np.meshgrid(*xs, indexing="ij")
    coords = np.stack([X.ravel(order="F"), Y.ravel(order="F"), Z.ravel(order="F")], axis=1)
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    i, j, k = (2 * a.ravel(order="F") for a in (i, j, k))
    node = lambda a, b, c: a + mx * (b + my * c)  # noqa: E731
    cols = []
    for c in range(3):
        for b in range(3):
            for a in range(3):
                cols.append(node(i + a, j + b, k + c))
    cells = np.stack(cols, axis=1)
    return Mesh(CELL_HEX27, np.ascontiguousarray(coords), cells.astype(np.int32))


def _morton_keys(points: np.ndarray, bits: int = 21) -> np.ndarray:
    lo = points.min(axis=0)
    span = np.maximum(points.max(axis=0) - lo, 1e-300)
    q = np.minimum(((points - lo) / span * (2**bits - 1)).astype(np.uint64), 2**bits - 1)

    def spread(v):
        v = v & np.uint64(0x1FFFFF)
        v = (v | (v << np.uint64(32))) & np.uint64(0x1F00000000FFFF)
        v = (v | (v << np.uint64(16))) & np.uint64(0x1F0000FF0000FF)
        v = (v | (v << np.uint64(8))) & np.uint64(0x100F00F00F00F00F)
        v = (v | (v << np.uint64(4))) & np.uint64(0x10C30C30C30C30C3)
        v = (v | (v << np.uint64(2))) & np.uint64(0x1249249249249249)
        return v

    return spread(q[:, 0]) | (spread(q[:, 1]) << np.uint64(1)) | (spread(q[:, 2]) << np.uint64(2))


def reorder_for_locality(mesh: Mesh) -> Mesh:
    """Sort cells along a Morton curve of their centroids and renumber nodes by first touch.

    Plays the role of the reference's optional reordering (RCM,
    libsrc/pylith/topology/ReverseCuthillMcKee.cc:23-72): neighbouring cells and
    their nodes end up close in memory, which is what the cell-block kernels and
    the L2 cache need.
    """
    corners = mesh.corner_nodes()
    centroids = mesh.coords[corners].mean(axis=1)
    order = np.argsort(_morton_keys(centroids), kind="stable")
    cells = mesh.cells[order]
    flat = cells.ravel()
    _, first = np.unique(flat, return_index=True)
    touched = flat[np.sort(first)]
    untouched = np.setdiff1d(np.arange(mesh.num_nodes), touched)
    new_order = np.concatenate([touched, untouched])
    perm = np.empty(mesh.num_nodes, dtype=np.int64)
    perm[new_order] = np.arange(mesh.num_nodes)
    out = Mesh(mesh.cell_type, np.ascontiguousarray(mesh.coords[new_order]),
               perm[cells].astype(np.int32))
    if mesh.cohesive is not None:
        coh = mesh.cohesive.copy()
        coh[:, :8] = perm[coh[:, :8]]
        out.cohesive = coh
        out.num_lagrange = mesh.num_lagrange
    return out


def _tet_volumes(coords: np.ndarray, cells: np.ndarray) -> np.ndarray:
    p = coords[cells]
    a = p[:, 1] - p[:, 0]
    b = p[:, 2] - p[:, 0]
    c = p[:, 3] - p[:, 0]
    return np.einsum("ij,ij->i", a, np.cross(b, c)) / 6.0


def box_tet_delaunay(target_cells: int, seed: int = 0, lo=BOX_LO, hi=BOX_HI,
                     reorder: bool = True) -> Mesh:
    """Delaunay tetrahedralisation of seeded uniform-random interior points plus a regular grid
    on the box faces (scipy/Qhull), sized to about `target_cells` tetrahedra.

    Zero-volume tetrahedra that Qhull forms among coplanar face-grid points are dropped, every
    cell is oriented positively, and (optionally) cells and nodes are reordered for locality.
    """
    from scipy.spatial import Delaunay

    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    ext = hi - lo
    npts = max(int(target_cells / 6.3), 64)
    h = (np.prod(ext) / npts) ** (1.0 / 3.0)
    nb = np.maximum(np.round(ext / h).astype(int), 2)
    axes = [np.linspace(lo[d], hi[d], nb[d] + 1) for d in range(3)]
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    grid = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    on_face = np.zeros(len(grid), dtype=bool)
    for d in range(3):
        on_face |= np.isclose(grid[:, d], lo[d]) | np.isclose(grid[:, d], hi[d])
    boundary = grid[on_face]
    rng = np.random.default_rng(seed)
    # Jitter the boundary grid inside its face (or along its edge) so that no four points of
    # two different faces are coplanar or cospherical: Qhull would otherwise emit flat
    # tetrahedra across the box edges whose removal leaves non-conforming cracks.
    pinned = np.zeros_like(boundary, dtype=bool)
    for d in range(3):
        pinned[:, d] = np.isclose(boundary[:, d], lo[d]) | np.isclose(boundary[:, d], hi[d])
    step = ext / nb
    jitter = rng.uniform(-0.3, 0.3, boundary.shape) * step
    boundary = np.where(pinned, boundary, boundary + jitter)
    nint = max(npts - len(boundary), 8)
    margin = 0.25 * h
    interior = lo + margin + rng.random((nint, 3)) * (ext - 2 * margin)
    pts = np.concatenate([boundary, interior], axis=0)
    tri = Delaunay(pts)
    cells = tri.simplices.astype(np.int64)
    vol = _tet_volumes(pts, cells)
    keep = np.abs(vol) > 1e-9 * np.abs(vol).mean()
    if not keep.all():
        # Only flat tetrahedra lying in one box face may be dropped (the boundary stays
        # conforming); any other degenerate cell means the triangulation is unusable.
        flat = pts[cells[~keep]]
        same_face = np.zeros(len(flat), dtype=bool)
        for d in range(3):
            for v in (lo[d], hi[d]):
                same_face |= np.isclose(flat[:, :, d], v).all(axis=1)
        if not same_face.all():
            raise RuntimeError("Delaunay produced degenerate tetrahedra off the box faces")
    cells = cells[keep]
    vol = vol[keep]
    neg = vol < 0
    cells[neg, 2], cells[neg, 3] = cells[neg, 3].copy(), cells[neg, 2].copy()
    used = np.unique(cells)
    remap = np.full(len(pts), -1, dtype=np.int64)
    remap[used] = np.arange(len(used))
    mesh = Mesh(CELL_TET4, np.ascontiguousarray(pts[used]), remap[cells].astype(np.int32))
    return reorder_for_locality(mesh) if reorder else mesh


def box_tet_delaunay_fault_x(target_cells: int, seed: int = 0, lo=BOX_LO, hi=BOX_HI, x0: float = 0.0,
                             reorder: bool = True) -> Mesh:
    """Delaunay P1 tetrahedra of a box symmetric about the plane x = x0, with a planar vertical
    fault of cohesive cells on that plane.

    The half box x >= x0 is triangulated as in `box_tet_delaunay` (seeded random interior points,
    a grid on its faces jittered inside each face), and mirrored across x = x0, so the two halves'
    triangulations of the plane are the same: the mesh is conforming across the fault. The plane's
    nodes are split (the +x cells take new positive-side copies) and every cell of the plane's
    face grid becomes a cohesive quadrilateral (negative side, positive side, Lagrange nodes; the
    normal points from - to +), whose corners are the plane grid's points: the solver uses the
    cohesive cells for their node pairs and the fault normal (libsrc/pylith/faults/TopologyOps.cc
    inserts cohesive cells on the mesh's own faces; here the faces of the two halves coincide).
    """
    from scipy.spatial import Delaunay

    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    if not np.isclose(x0 - lo[0], hi[0] - x0):
        raise ValueError("the box must be symmetric about x = x0")
    hlo = np.array([x0, lo[1], lo[2]])
    ext = hi - hlo
    npts = max(int(0.5 * target_cells / 6.3), 64)
    h = (np.prod(ext) / npts) ** (1.0 / 3.0)
    nb = np.maximum(np.round(ext / h).astype(int), 2)
    axes = [np.linspace(hlo[d], hi[d], nb[d] + 1) for d in range(3)]
    I, J, K = np.meshgrid(*[np.arange(n + 1) for n in nb], indexing="ij")
    ijk = np.stack([I.ravel(), J.ravel(), K.ravel()], axis=1)
    grid = np.stack([axes[d][ijk[:, d]] for d in range(3)], axis=1)
    on_face = np.zeros(len(grid), dtype=bool)
    for d in range(3):
        on_face |= (ijk[:, d] == 0) | (ijk[:, d] == nb[d])
    boundary, bijk = grid[on_face], ijk[on_face]
    rng = np.random.default_rng(seed)
    pinned = np.zeros_like(boundary, dtype=bool)
    for d in range(3):
        pinned[:, d] = (bijk[:, d] == 0) | (bijk[:, d] == nb[d])
    step = ext / nb
    boundary = np.where(pinned, boundary, boundary + rng.uniform(-0.3, 0.3, boundary.shape) * step)
    nint = max(npts - len(boundary), 8)
    margin = 0.25 * h
    interior = hlo + margin + rng.random((nint, 3)) * (ext - 2 * margin)
    pts = np.concatenate([boundary, interior], axis=0)
    cells = Delaunay(pts).simplices.astype(np.int64)
    vol = _tet_volumes(pts, cells)
    keep = np.abs(vol) > 1e-9 * np.abs(vol).mean()
    if not keep.all():
        flat = pts[cells[~keep]]
        same_face = np.zeros(len(flat), dtype=bool)
        for d in range(3):
            for v in (hlo[d], hi[d]):
                same_face |= np.isclose(flat[:, :, d], v).all(axis=1)
        if not same_face.all():
            raise RuntimeError("Delaunay produced degenerate tetrahedra off the box faces")
    cells, vol = cells[keep], vol[keep]
    neg = vol < 0
    cells[neg, 2], cells[neg, 3] = cells[neg, 3].copy(), cells[neg, 2].copy()
    npt = len(pts)
    # the fault plane's points (grid i == 0) and their (j, k) grid indices
    plane = np.zeros(npt, dtype=bool)
    plane[:len(boundary)] = bijk[:, 0] == 0
    jk_of = np.full((nb[1] + 1, nb[2] + 1), -1, dtype=np.int64)
    pidx = np.flatnonzero(plane)
    jk_of[bijk[pidx, 1], bijk[pidx, 2]] = pidx
    # nodes: the negative half (mirror; plane points shared), then the positive half's own points,
    # then the positive-side copies of the plane points
    off_pos = np.flatnonzero(~plane)
    neg_id = np.arange(npt)                      # mirror: plane points keep their ids
    mir = pts.copy()
    mir[:, 0] = 2 * x0 - mir[:, 0]
    pos_id = np.full(npt, -1, dtype=np.int64)
    pos_id[off_pos] = npt + np.arange(len(off_pos))
    pos_id[pidx] = npt + len(off_pos) + np.arange(len(pidx))
    coords = np.concatenate([mir, pts[off_pos], pts[pidx]], axis=0)
    neg_cells = neg_id[cells][:, [0, 1, 3, 2]]  # the mirror reverses orientation
    pos_cells = pos_id[cells]
    all_cells = np.concatenate([neg_cells, pos_cells], axis=0)
    # cohesive quads of the plane grid, corners (j,k), (j+1,k), (j+1,k+1), (j,k+1): +y then +z
    jj, kk = np.meshgrid(np.arange(nb[1]), np.arange(nb[2]), indexing="ij")
    jj, kk = jj.ravel(), kk.ravel()
    quad = np.stack([jk_of[jj, kk], jk_of[jj + 1, kk], jk_of[jj + 1, kk + 1], jk_of[jj, kk + 1]], axis=1)
    lag_of = np.full(npt, -1, dtype=np.int64)
    lag_of[pidx] = np.arange(len(pidx))
    coh = np.concatenate([neg_id[quad], pos_id[quad], lag_of[quad]], axis=1).astype(np.int32)
    used = np.unique(all_cells)
    if len(used) != len(coords):
        raise RuntimeError("unused nodes in the mirrored mesh")
    mesh = Mesh(CELL_TET4, np.ascontiguousarray(coords), all_cells.astype(np.int32), coh, len(pidx))
    return reorder_for_locality(mesh) if reorder else mesh


def boundary_mask(mesh: Mesh, axis: int, side: str, lo=BOX_LO, hi=BOX_HI, tol: float = 1e-6):
    """Boolean mask of nodes on the box face x_axis = lo (side 'neg') or hi ('pos')."""
    val = lo[axis] if side == "neg" else hi[axis]
    scale = max(abs(hi[axis] - lo[axis]), 1.0)
    return np.abs(mesh.coords[:, axis] - val) <= tol * scale


def insert_fault_x(mesh: Mesh, x0: float = 0.0, tol: float = 1e-6) -> Mesh:
    """Insert a planar vertical fault of cohesive cells at x = x0 into a Q1 hex mesh.

    Nodes on the plane are split: cells on the +x side are reconnected to new
    positive-side copies. Every quad face on the plane becomes a cohesive cell,
    and every split node carries one Lagrange-multiplier node (the reference's
    fault vertices, libsrc/pylith/faults/TopologyOps.cc:26-310).
    """
    if mesh.cell_type != CELL_HEX8:
        raise ValueError("insert_fault_x expects a Q1 hex mesh")
    coords = mesh.coords
    scale = np.abs(coords).max()
    on_plane = np.abs(coords[:, 0] - x0) <= tol * scale
    plane_nodes = np.nonzero(on_plane)[0]
    nn = mesh.num_nodes
    pos_of = np.full(nn, -1, dtype=np.int64)
    pos_of[plane_nodes] = nn + np.arange(len(plane_nodes))
    lag_of = np.full(nn, -1, dtype=np.int64)
    lag_of[plane_nodes] = np.arange(len(plane_nodes))
    cells = mesh.cells.astype(np.int64).copy()
    centroid_x = coords[mesh.cells].mean(axis=1)[:, 0]
    pos_cells = centroid_x > x0
    sub = cells[pos_cells]
    mask = on_plane[sub]
    sub[mask] = pos_of[sub[mask]]
    cells[pos_cells] = sub
    new_coords = np.concatenate([coords, coords[plane_nodes]], axis=0)
    # Faces on the plane: the x-min face (corners 0,3,7,4) of +x cells touching the plane.
    face_local = [0, 3, 7, 4]
    plus = np.nonzero(pos_cells)[0]
    orig = mesh.cells[plus][:, face_local]
    onf = on_plane[orig].all(axis=1)
    faces = orig[onf]
    # Orientation: corners 0,3,7,4 of a hex go (y, z) = (0,0),(1,0),(1,1),(0,1), so
    # dx/dxi = +y and dx/deta = +z and their cross product is +x: from the - side to the + side.
    neg = faces
    pos = pos_of[faces]
    lag = lag_of[faces]
    coh = np.concatenate([neg, pos, lag], axis=1).astype(np.int32)
    return Mesh(CELL_HEX8, np.ascontiguousarray(new_coords), cells.astype(np.int32), coh,
                len(plane_nodes))


# Kuhn split of a hexahedron (corner order above) into 6 tetrahedra around the 0-6 diagonal;
# every hexahedron uses the same diagonal direction, so the split is conforming across faces.
_KUHN = np.array([[0, 1, 2, 6], [0, 2, 3, 6], [0, 3, 7, 6], [0, 7, 4, 6], [0, 4, 5, 6], [0, 5, 1, 6]])


def box_tet_kuhn(nx: int, ny: int, nz: int, lo=BOX_LO, hi=BOX_HI, fault_x: float | None = None,
                 jitter: float = 0.1, seed: int = 0, reorder: bool = True) -> Mesh:
    """P1 tetrahedra from a Kuhn split of a hex grid, nodes jittered by up to `jitter` times the
    spacing (boundary nodes stay on their faces, fault nodes on the fault plane).

    With `fault_x`, a planar vertical fault of cohesive cells is inserted at x = fault_x first
    (`insert_fault_x`); the cohesive cells stay the quadrilateral hex faces on the plane, whose
    two triangles are faces of the adjacent tetrahedra. This is how the Green's-function mesh
    gets a fault that is a union of cell faces, which a Delaunay triangulation of random points
    does not provide.
    """
    hexes = box_hex(nx, ny, nz, lo, hi)
    if fault_x is not None:
        hexes = insert_fault_x(hexes, fault_x)
    coords = hexes.coords.copy()
    lo_a, hi_a = np.asarray(lo, float), np.asarray(hi, float)
    h = (hi_a - lo_a) / np.array([nx, ny, nz])
    rng = np.random.default_rng(seed)
    delta = rng.uniform(-jitter, jitter, coords.shape) * h
    for d in range(3):
        on = np.isclose(coords[:, d], lo_a[d]) | np.isclose(coords[:, d], hi_a[d])
        delta[on, d] = 0.0
    if fault_x is not None:
        delta[np.isclose(coords[:, 0], fault_x), 0] = 0.0
        # both sides of a split node move together
        nn0 = (nx + 1) * (ny + 1) * (nz + 1)
        plane = np.nonzero(np.isclose(hexes.coords[:nn0, 0], fault_x))[0]
        delta[nn0:nn0 + len(plane)] = delta[plane]
    coords = coords + delta
    tets = hexes.cells[:, _KUHN].reshape(-1, 4).astype(np.int64)
    vol = _tet_volumes(coords, tets)
    neg = vol < 0
    tets[neg, 2], tets[neg, 3] = tets[neg, 3].copy(), tets[neg, 2].copy()
    if np.any(np.abs(vol) < 1e-12 * np.abs(vol).mean()):
        raise RuntimeError("degenerate tetrahedron after jitter; lower the jitter")
    mesh = Mesh(CELL_TET4, np.ascontiguousarray(coords), tets.astype(np.int32), hexes.cohesive,
                hexes.num_lagrange)
    return reorder_for_locality(mesh) if reorder else mesh
