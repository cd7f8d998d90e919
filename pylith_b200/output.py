"""Output of solution and derived fields as VTK unstructured-grid files (.vtu).

The reference writes VTK output with its DataWriterVTK (libsrc/pylith/meshio/DataWriterVTK.cc),
which hands every field to PETSc's VTU viewer (PetscViewerVTKOpen/PetscViewerVTKAddField,
DataWriterVTK.cc:154-236). The file layout kept here is that viewer's, byte for byte (the
reference's golden files tests/libtests/meshio/data/*_t10.vtu pin it):

  * an XML `UnstructuredGrid` with one `Piece`, little-endian, UInt64 block headers;
  * every array in one raw `AppendedData` section, each block a UInt64 byte count followed by the
    values; `offset` attributes count bytes from the start of that section;
  * Float64 `Position`, Int32 `connectivity` and `offsets`, UInt8 `types`, and an Int32 `Rank`
    cell array (the MPI rank of every cell: 0 here) before the cell fields;
  * array names are the field name followed by the component name; a vector field is one
    3-component array, any other field one array per component with the suffix `.i` (a
    single-component cell field has no suffix).

File names follow DataWriterVTK::_vtkFilename (DataWriterVTK.cc:242-262): `<base>_t<stamp>.vtu`,
the stamp being the time format applied to t * time_scale / time_constant with its first
decimal point removed, or `<base>_info.vtu` for time-independent information.

Cells are written in this package's corner orders, which are VTK's for P1 tetrahedra (VTK_TETRA)
and Q1 hexahedra (VTK_HEXAHEDRON, corners (0,0,0),(1,0,0),(1,1,0),(0,1,0) then the top face).
Q2 hexahedra are written through their 8 corner nodes.
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import meshing as M

VTK_TETRA = 10
VTK_HEXAHEDRON = 12

_TYPE_NAMES = {np.dtype(np.float64): "Float64", np.dtype(np.int32): "Int32", np.dtype(np.uint8): "UInt8"}


@dataclass
class _Array:
    name: str
    data: np.ndarray  # C-contiguous, little-endian
    ncomp: int

    @property
    def type_name(self) -> str:
        return _TYPE_NAMES[self.data.dtype]


def _block(a: np.ndarray) -> bytes:
    raw = np.ascontiguousarray(a).astype(a.dtype.newbyteorder("<"), copy=False).tobytes()
    return struct.pack("<Q", len(raw)) + raw


def _array_line(a: _Array, offset: int, name_field: str) -> str:
    return (f'        <DataArray type="{a.type_name}" Name={name_field} NumberOfComponents="{a.ncomp}" '
            f'format="appended" offset="{offset}" />\n')


def write_vtu(path: str, points: np.ndarray, cells: np.ndarray, vtk_type: int,
              point_data: Sequence[Tuple[str, np.ndarray]] = (),
              cell_data: Sequence[Tuple[str, np.ndarray]] = (), rank: int = 0) -> None:
    """One .vtu file. points [npoints][3] (FP64), cells [ncells][nen] (corner indices in VTK order),
    point_data / cell_data: (array name, values [n] or [n][ncomp]) in file order."""
    points = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
    cells = np.ascontiguousarray(cells, dtype=np.int32)
    if cells.ndim != 2:
        raise ValueError("cells must be [ncells][corners]")
    npts, (ncells, nen) = points.shape[0], cells.shape
    if ncells and (cells.min() < 0 or cells.max() >= npts):
        raise ValueError("cell corner index out of range")

    def arrays(items, n, what):
        out = []
        for name, values in items:
            v = np.ascontiguousarray(values, dtype=np.float64)
            v = v.reshape(n, -1) if v.size else v.reshape(n, 0)
            if v.shape[0] != n:
                raise ValueError(f"{what} array {name!r} has {v.shape[0]} rows, expected {n}")
            out.append(_Array(name, v, v.shape[1]))
        return out

    pdata = arrays(point_data, npts, "point")
    cdata = arrays(cell_data, ncells, "cell")
    pos = _Array("Position", points, 3)
    conn = _Array("connectivity", cells.reshape(-1), 1)
    offs = _Array("offsets", (np.arange(1, ncells + 1, dtype=np.int32) * nen).astype(np.int32), 1)
    types = _Array("types", np.full(ncells, vtk_type, dtype=np.uint8), 1)
    rank_a = _Array("Rank", np.full(ncells, rank, dtype=np.int32), 1)

    blocks: List[bytes] = []
    offset = 0

    def place(a: _Array) -> int:
        nonlocal offset
        b = _block(a.data)
        here = offset
        blocks.append(b)
        offset += len(b)
        return here

    head = ['<?xml version="1.0"?>\n',
            '<VTKFile type="UnstructuredGrid" version="0.1" byte_order="LittleEndian" header_type="UInt64">\n',
            "  <UnstructuredGrid>\n",
            f'    <Piece NumberOfPoints="{npts}" NumberOfCells="{ncells}">\n',
            "      <Points>\n"]
    head.append(_array_line(pos, place(pos), '"Position"'))
    head.append("      </Points>\n      <Cells>\n")
    head.append(_array_line(conn, place(conn), '"connectivity"'))
    head.append(_array_line(offs, place(offs), '"offsets"     '))
    head.append(_array_line(types, place(types), '"types"       '))
    head.append("      </Cells>\n      <CellData>\n")
    head.append(_array_line(rank_a, place(rank_a), '"Rank"'))
    for a in cdata:
        head.append(_array_line(a, place(a), f'"{a.name}"'))
    head.append("      </CellData>\n      <PointData>\n")
    for a in pdata:
        head.append(_array_line(a, place(a), f'"{a.name}"'))
    head.append("      </PointData>\n    </Piece>\n  </UnstructuredGrid>\n")
    head.append('  <AppendedData encoding="raw">\n_')
    with open(path, "wb") as f:
        f.write("".join(head).encode("ascii"))
        for b in blocks:
            f.write(b)
        f.write(b"\n  </AppendedData>\n</VTKFile>\n")


def read_vtu(path: str):
    """Reads a file in the layout write_vtu produces: (points, connectivity, offsets, types,
    {cell array name: values}, {point array name: values}); values are [n][ncomp]."""
    import re

    data = open(path, "rb").read()
    start = data.index(b'<AppendedData encoding="raw">')
    base = data.index(b"_", start) + 1
    head = data[:start].decode("ascii")
    out = {}
    section = None
    npts = int(re.search(r'NumberOfPoints="(\d+)"', head).group(1))
    ncells = int(re.search(r'NumberOfCells="(\d+)"', head).group(1))
    dtypes = {"Float64": "<f8", "Int32": "<i4", "UInt8": "u1"}
    cell, point = {}, {}
    for line in head.splitlines():
        s = line.strip()
        if s in ("<Points>", "<Cells>", "<CellData>", "<PointData>"):
            section = s
            continue
        m = re.match(r'<DataArray type="(\w+)" Name="([^"]+)"\s+NumberOfComponents="(\d+)" format="appended" '
                     r'offset="(\d+)" />', s)
        if not m:
            continue
        t, name, nc, off = m.group(1), m.group(2), int(m.group(3)), int(m.group(4))
        (nbytes,) = struct.unpack_from("<Q", data, base + off)
        v = np.frombuffer(data, dtype=dtypes[t], count=nbytes // np.dtype(dtypes[t]).itemsize, offset=base + off + 8)
        if section == "<CellData>":
            cell[name] = v.reshape(ncells, nc)
        elif section == "<PointData>":
            point[name] = v.reshape(npts, nc)
        else:
            out[name] = v
    return (out["Position"].reshape(npts, 3), out["connectivity"], out["offsets"], out["types"], cell, point)


def vtk_cells(mesh: M.Mesh) -> Tuple[np.ndarray, int]:
    """Corner connectivity and VTK cell type of a mesh (Q2 hexahedra through their corners)."""
    if mesh.cell_type == M.CELL_TET4:
        return mesh.cells, VTK_TETRA
    if mesh.cell_type in (M.CELL_HEX8, M.CELL_HEX27):
        return mesh.corner_nodes(), VTK_HEXAHEDRON
    raise ValueError(f"cell type {mesh.cell_type} has no VTK output here")


@dataclass
class DataWriterVTK:
    """The reference's DataWriterVTK (libsrc/pylith/meshio/DataWriterVTK.hh) over write_vtu: one
    file per time step, fields added between openTimeStep and closeTimeStep."""

    filename: str = "output.vtu"
    time_format: str = "%f"
    time_constant: float = 1.0
    time_scale: float = 1.0
    is_info: bool = False
    _mesh: Optional[M.Mesh] = None
    _t: Optional[float] = None
    _point: List[Tuple[str, np.ndarray]] = field(default_factory=list)
    _cell: List[Tuple[str, np.ndarray]] = field(default_factory=list)

    def __post_init__(self):
        if not self.time_constant > 0.0:
            raise ValueError("Time used to normalize time stamp in VTK data files must be positive.")

    def vtk_filename(self, t: float) -> str:
        """DataWriterVTK::_vtkFilename (DataWriterVTK.cc:242-262)."""
        base = self.filename[:self.filename.find(".vtu")] if ".vtu" in self.filename else self.filename
        if self.is_info:
            return f"{base}_info.vtu"
        stamp = self.time_format % (t * self.time_scale / self.time_constant)
        stamp = stamp.replace(".", "", 1)
        return f"{base}_t{stamp}.vtu"

    def open(self, mesh: M.Mesh) -> None:
        self._mesh = mesh

    def open_time_step(self, t: float) -> None:
        if self._mesh is None:
            raise RuntimeError("open() the writer with a mesh first")
        self._t = t
        self._point, self._cell = [], []

    @staticmethod
    def _arrays(name: str, values: np.ndarray, vector: bool, cell: bool):
        v = np.asarray(values, dtype=np.float64)
        v = v.reshape(v.shape[0], -1)
        if vector:
            return [(name, v)]
        if v.shape[1] == 1 and cell:
            return [(name, v)]
        return [(f"{name}.{i}", v[:, i]) for i in range(v.shape[1])]

    def write_vertex_field(self, name: str, values: np.ndarray, vector: bool = False) -> None:
        """A field at the mesh nodes, [nnodes] or [nnodes][ncomp]; vector=True writes it as one
        3-component array."""
        self._point += self._arrays(name, values, vector, cell=False)

    def write_cell_field(self, name: str, values: np.ndarray, vector: bool = False) -> None:
        """A field per cell (basis order 0, e.g. the derived cauchy_stress), [ncells][ncomp]."""
        self._cell += self._arrays(name, values, vector, cell=True)

    def close_time_step(self, directory: str = ".") -> str:
        """Writes the step's file and returns its path."""
        if self._t is None:
            raise RuntimeError("no open time step")
        cells, vtk_type = vtk_cells(self._mesh)
        path = os.path.join(directory, self.vtk_filename(self._t))
        write_vtu(path, self._mesh.coords, cells, vtk_type, self._point, self._cell)
        self._t = None
        return path

    def close(self) -> None:
        self._mesh = None


# ---------------------------------------------------------------------------------------------
# HDF5 output
# ---------------------------------------------------------------------------------------------

@dataclass
class PointMesh:
    """A mesh of points alone, one vertex cell per point (the point mesh of station output,
    MeshOps::createFromPoints in topology/MeshOps.cc, used by OutputSolnPoints)."""

    coords: np.ndarray  # float64 [npoints, 3]

    @property
    def num_nodes(self) -> int:
        return int(len(self.coords))

    @property
    def num_cells(self) -> int:
        return int(len(self.coords))


def _q1_basis(xi: np.ndarray) -> np.ndarray:
    """Trilinear basis on [0, 1]^3 in this package's Q1 corner order, [n][8]."""
    x, y, z = xi[:, 0], xi[:, 1], xi[:, 2]
    cols = []
    for (a, b, c) in ((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)):
        cols.append((x if a else 1 - x) * (y if b else 1 - y) * (z if c else 1 - z))
    return np.stack(cols, axis=1)


def _q1_jacobian(X: np.ndarray, xi: np.ndarray) -> np.ndarray:
    """d x / d xi of the trilinear map of corners X [n][8][3] at xi [n][3], [n][3][3]."""
    x, y, z = xi[:, 0], xi[:, 1], xi[:, 2]
    J = np.zeros((len(xi), 3, 3))
    for k, (a, b, c) in enumerate(((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1),
                                   (0, 1, 1))):
        fx, fy, fz = (x if a else 1 - x), (y if b else 1 - y), (z if c else 1 - z)
        dx, dy, dz = (1.0 if a else -1.0), (1.0 if b else -1.0), (1.0 if c else -1.0)
        grad = np.stack([dx * fy * fz, fx * dy * fz, fx * fy * dz], axis=1)  # [n][3]
        J += X[:, k, :, None] * grad[:, None, :]
    return J


def _q2_basis(xi: np.ndarray) -> np.ndarray:
    """Triquadratic basis on [0, 1]^3, node (a, b, c) at index a + 3 b + 9 c, [n][27]."""
    def lag(t):
        return np.stack([2 * (t - 0.5) * (t - 1), -4 * t * (t - 1), 2 * t * (t - 0.5)], axis=1)

    lx, ly, lz = lag(xi[:, 0]), lag(xi[:, 1]), lag(xi[:, 2])
    return np.einsum("na,nb,nc->ncba", lx, ly, lz).reshape(len(xi), 27)


class PointInterpolator:
    """DMInterpolation for station output (OutputSolnPoints, meshio/OutputSolnPoints.cc:160-260):
    each point is located once in a cell of the mesh on the host (cells nearest by centroid,
    then the point's coordinates in the cell: barycentric for P1 tetrahedra, the inverse of the
    trilinear corner map by Newton iterations for Q1 and Q2 hexahedra), and the solution's nodal
    displacement is then interpolated with the cell's basis at the point on the device. A point
    outside the mesh is an error, as DMInterpolationSetUp reports without ignoreOutsideDomain."""

    def __init__(self, mesh, points, tol: float = 1e-9, device: str = "cuda"):
        from scipy.spatial import cKDTree

        pts = np.asarray(points, dtype=np.float64).reshape(-1, 3)
        corners = mesh.corner_nodes()
        cent = mesh.coords[corners].mean(axis=1)
        k = min(64, mesh.num_cells)
        _, cand = cKDTree(cent).query(pts, k=k)
        cand = np.asarray(cand).reshape(len(pts), k)
        cell = np.full(len(pts), -1)
        ref = np.zeros((len(pts), 3))
        for j in range(k):
            todo = np.flatnonzero(cell < 0)
            if len(todo) == 0:
                break
            c = cand[todo, j]
            xi = self._reference(mesh, corners[c], pts[todo])
            if mesh.cell_type == M.CELL_TET4:
                inside = (xi >= -tol).all(axis=1) & (xi.sum(axis=1) <= 1 + tol)
            else:
                inside = ((xi >= -tol) & (xi <= 1 + tol)).all(axis=1)
            cell[todo[inside]] = c[inside]
            ref[todo[inside]] = xi[inside]
        if (cell < 0).any():
            raise ValueError(f"{int((cell < 0).sum())} points are outside the mesh, e.g. {pts[cell < 0][0]}")
        if mesh.cell_type == M.CELL_TET4:
            w = np.concatenate([1 - ref.sum(axis=1, keepdims=True), ref], axis=1)
        elif mesh.cell_type == M.CELL_HEX8:
            w = _q1_basis(ref)
        else:
            w = _q2_basis(ref)
        import torch

        self.cells = cell
        self.nodes = torch.from_numpy(mesh.cells[cell].astype(np.int64)).to(device)
        self.weights = torch.from_numpy(w).to(device)

    @staticmethod
    def _reference(mesh, X_idx, pts):
        X = mesh.coords[X_idx]  # [n][corners][3]
        if mesh.cell_type == M.CELL_TET4:
            A = np.transpose(X[:, 1:, :] - X[:, :1, :], (0, 2, 1))  # columns x_k - x_0
            return np.linalg.solve(A, (pts - X[:, 0, :])[..., None])[..., 0]
        xi = np.full((len(pts), 3), 0.5)
        for _ in range(20):  # Newton on the trilinear map (exact in one step for affine cells)
            r = np.einsum("nk,nkd->nd", _q1_basis(xi), X) - pts
            xi = xi - np.linalg.solve(_q1_jacobian(X, xi), r[..., None])[..., 0]
        return xi

    def __call__(self, u):
        """Displacement at the points, [npoints][3], from a device solution vector (3 DOFs per
        mesh node first)."""
        disp = u.reshape(-1, 3)  # mesh nodes first, then the fault's Lagrange-multiplier nodes
        return (disp[self.nodes] * self.weights[..., None]).sum(dim=1)


def read_points_list(path: str, comment: str = "#", delimiter: Optional[str] = None):
    """Station names and coordinates from a points file as PyLith's PointsList reads it
    (pylith/meshio/PointsList.py): one point per line, `name x y z`, fields split on whitespace
    (or `delimiter`), lines starting with the comment delimiter skipped."""
    names, coords = [], []
    with open(path) as fh:
        for line in fh:
            line = line.strip()
            if not line or line.startswith(comment):
                continue
            fields = line.split(delimiter)
            names.append(fields[0].strip())
            coords.append([float(v) for v in fields[1:4]])
    return names, np.array(coords, dtype=np.float64).reshape(-1, 3)


VECTOR_FIELD_TYPES = ("scalar", "vector", "tensor", "other", "multi_scalar", "multi_vector", "multi_tensor",
                      "multi_other")  # FieldBase::vectorFieldString (topology/FieldBase.cc:34-56)


def _vector_field_type(ncomp: int) -> str:
    return {1: "scalar", 3: "vector", 6: "tensor"}.get(ncomp, "other")


@dataclass
class DataWriterHDF5:
    """The reference's DataWriterHDF5 (libsrc/pylith/meshio/DataWriterHDF5.hh) over
    pylith_b200.hdf5.H5Writer, with the layout PETSc's HDF5 viewer gives that writer's files
    (the reference's golden files tests/libtests/meshio/data/*.h5 pin it):

      * /geometry/vertices: float64 [nvertices][3], coordinates times the length scale
        (DataWriter.cc:235-237);
      * /viz/topology/cells: int32 [ncells][ncorners] with int32 attributes cell_corners and
        cell_dim; cohesive cells in /viz/topology_1/cells (negative-side then positive-side face
        vertices);
      * /cell_fields/partition_rank: float64 [ncells][1] (the MPI rank of every cell, 0 here),
        attributes vector_field_type "scalar" and componentName0 "0";
      * /time: float64 [nsteps][1][1], t times the time scale, one entry per output step
        (DataWriterHDF5.cc:441-463); attribute timestepping = 1 (uint8);
      * /vertex_fields/<name>, /cell_fields/<name>: float64 [nsteps][npoints][ncomp], attributes
        timestepping = 1 and vector_field_type (FieldBase::vectorFieldString);
      * /stations: fixed-length strings (longest name + 1 bytes) from write_point_names.

    The file is written as the calls come: after every call it is complete and readable
    (datasets grow one step at a time). Steps follow the reference's rule: the k-th write of a
    field is its step k, and the first field written at a new step adds that step's time."""

    filename: str = "output.h5"
    time_scale: float = 1.0
    length_scale: float = 1.0
    is_info: bool = False
    _h5: Optional[object] = None
    _mesh: Optional[M.Mesh] = None
    _steps: dict = field(default_factory=dict)
    _tstamp_index: int = 0

    def hdf5_filename(self) -> str:
        """DataWriterHDF5::hdf5Filename (DataWriterHDF5.cc:422-435)."""
        if self.is_info:
            i = self.filename.find(".h5")
            return (self.filename[:i] if i >= 0 else self.filename[:-1]) + "_info.h5"
        return self.filename

    def open(self, mesh: M.Mesh, is_info: Optional[bool] = None) -> None:
        """DataWriterHDF5::open (DataWriterHDF5.cc:82-117): a new file with the mesh."""
        from . import hdf5 as H5

        if is_info is not None:
            self.is_info = is_info
        self.close()
        self._mesh = mesh
        self._steps, self._tstamp_index = {}, 0
        w = H5.H5Writer(self.hdf5_filename())
        w.create_dataset("/geometry/vertices", np.asarray(mesh.coords, dtype=np.float64) * self.length_scale)
        if isinstance(mesh, PointMesh):  # stations: vertex cells, the rank as a vertex field
            n = mesh.num_nodes
            w.create_dataset("/viz/topology/cells", np.arange(n, dtype=np.int32).reshape(n, 1),
                             {"cell_corners": np.int32(1), "cell_dim": np.int32(0)})
            w.create_dataset("/vertex_fields/partition_rank", np.zeros((n, 1)),
                             {"vector_field_type": "scalar", "componentName0": "0"})
            self._h5 = w
            return
        corners = vtk_cells(mesh)[0].astype(np.int32)
        w.create_dataset("/viz/topology/cells", corners,
                         {"cell_corners": np.int32(corners.shape[1]), "cell_dim": np.int32(3)})
        if mesh.cohesive is not None and len(mesh.cohesive):
            coh = np.ascontiguousarray(mesh.cohesive[:, :8], dtype=np.int32)
            w.create_dataset("/viz/topology_1/cells", coh, {"cell_corners": np.int32(8), "cell_dim": np.int32(3)})
        w.create_dataset("/cell_fields/partition_rank", np.zeros((mesh.num_cells, 1)),
                         {"vector_field_type": "scalar", "componentName0": "0"})
        self._h5 = w

    def _write_time(self, t: float) -> None:
        w = self._h5
        if "/time" not in w.series:
            w.create_series("/time", (1, 1), attrs={"timestepping": np.uint8(1)})
        w.append("/time", [[t * self.time_scale]])
        self._tstamp_index += 1

    def _write_field(self, group: str, t: float, name: str, values, npoints: int, vector_field_type) -> None:
        v = np.asarray(values, dtype=np.float64)
        if v.shape[0] != npoints:
            raise ValueError(f"field '{name}' has {v.shape[0]} points, the mesh {npoints}")
        v = v.reshape(npoints, -1)
        vtype = vector_field_type or _vector_field_type(v.shape[1])
        if vtype not in VECTOR_FIELD_TYPES:
            raise ValueError(f"unknown vector field type '{vtype}'")
        key = f"{group}/{name}"
        istep = self._steps[key] = self._steps.get(key, -1) + 1
        if self._tstamp_index == istep:
            self._write_time(t)
        self._store(key, name, v, vtype, istep)

    def _store(self, key: str, name: str, v: np.ndarray, vtype: str, istep: int) -> None:
        """One step of a field: a chunk of the dataset (created at the field's first step)."""
        if istep == 0:
            self._h5.create_series(key, v.shape, attrs={"timestepping": np.uint8(1), "vector_field_type": vtype})
        self._h5.append(key, v)

    def write_vertex_field(self, t: float, name: str, values, vector_field_type: Optional[str] = None) -> None:
        """DataWriterHDF5::writeVertexField (DataWriterHDF5.cc:162-216): values [nvertices] or
        [nvertices][ncomp]; the vector field type defaults from the component count (1 scalar,
        3 vector, 6 tensor, else other)."""
        if self._h5 is None:
            raise RuntimeError("open() the writer with a mesh first")
        self._write_field("/vertex_fields", t, name, values, self._mesh.num_nodes, vector_field_type)

    def write_cell_field(self, t: float, name: str, values, vector_field_type: Optional[str] = None) -> None:
        """DataWriterHDF5::writeCellField (DataWriterHDF5.cc:222-276): values [ncells] or
        [ncells][ncomp] over the domain cells (e.g. the derived cauchy_stress)."""
        if self._h5 is None:
            raise RuntimeError("open() the writer with a mesh first")
        self._write_field("/cell_fields", t, name, values, self._mesh.num_cells, vector_field_type)

    def write_point_names(self, names: Sequence[str]) -> None:
        """DataWriterHDF5::writePointNames (DataWriterHDF5.cc:282-416): /stations as
        null-padded fixed-length strings of the longest name plus one byte."""
        if self._h5 is None:
            raise RuntimeError("open() the writer with a mesh first")
        width = max([len(n) for n in names] + [0]) + 1
        self._h5.create_dataset("/stations", np.array([n.encode() for n in names], dtype=f"S{width}"))

    def close(self) -> None:
        """DataWriterHDF5::close (DataWriterHDF5.cc:137-160): closes the file and writes its Xdmf
        description next to it (write_xdmf)."""
        if self._h5 is not None:
            self._h5.close()
            self._h5 = None
            write_xdmf(self.hdf5_filename())


# ---------------------------------------------------------------------------------------------
# Xdmf metadata for HDF5 output
# ---------------------------------------------------------------------------------------------

_XDMF_CELL_TYPES = {(0, 1): "Polyvertex", (1, 2): "Polyline", (2, 3): "Triangle", (2, 4): "Quadrilateral",
                    (3, 4): "Tetrahedron", (3, 8): "Hexahedron"}
_XDMF_VECTOR_TYPES = {"scalar": "Scalar", "vector": "Vector", "tensor": "Tensor6"}
_XDMF_TENSOR_SUFFIXES = {2: ("_xx", "_yy", "_xy"), 3: ("_xx", "_yy", "_zz", "_xy", "_yz", "_xz")}
_HEAVY = "&HeavyData;:"


class _XdmfLines:
    """Lines of an Xdmf document, each indented by two spaces per depth."""

    def __init__(self):
        self.lines: List[str] = []

    def __call__(self, depth: int, text: str) -> None:
        self.lines.append("  " * depth + text)

    def item(self, depth: int, attrs: str, body: str) -> None:
        """<DataItem attrs> body </DataItem>, the body one level deeper."""
        self(depth, f"<DataItem {attrs}>")
        self(depth + 1, body)
        self(depth, "</DataItem>")

    def text(self) -> str:
        return "\n".join(self.lines) + "\n"


def _xdmf_field(f, group: str, name: str):
    """(name, Xdmf type, center, HDF5 path, steps, points, components) of one field dataset."""
    path = f"/{group}/{name}"
    shape = f.dataset(path).shape
    vtype = f.attrs(path).get("vector_field_type")
    if vtype is not None:
        xtype = _XDMF_VECTOR_TYPES.get(str(vtype).lower(), "Matrix")
    else:  # no attribute: guess from the component count
        xtype = {1: "Scalar", 3: "Vector"}.get(shape[-1], "Matrix") if len(shape) in (2, 3) else "Matrix"
    if len(shape) == 2:
        steps, points, comps = 1, shape[0], shape[1]
    elif len(shape) == 3:
        steps, points, comps = shape
    else:
        raise ValueError(f"unexpected shape {shape} of dataset '{path}'")
    center = "Node" if group == "vertex_fields" else "Cell"
    return name, xtype, center, path, steps, points, comps


def write_xdmf(filename_h5: str, filename_xdmf: Optional[str] = None) -> Optional[str]:
    """Writes the Xdmf file describing an HDF5 output file for visualization tools, as the
    reference's Xdmf writer does (pylith/meshio/Xdmf.py, called from DataWriterHDF5::close,
    meshio/DataWriterHDF5.cc:146-157); its golden files tests/pytests/meshio/data/*.xmf pin the
    text line for line. Returns the path written, or None for a 1-D mesh (Xdmf has no 1-D grids).

    The document references the HDF5 datasets by path: the cells and vertices once in the domain
    (a 2-D mesh gets a zero z coordinate through a JOIN function), then one uniform grid per time
    stamp of /time (in a temporal collection) or one grid without time, each with the fields of
    /vertex_fields and /cell_fields in name order. Scalars and vectors are one attribute per
    field (2-D vectors joined with a zero z); tensors become one scalar attribute per component
    (_xx, _yy, _zz, _xy, _yz, _xz; _xx, _yy, _xy in 2-D) and other fields one per component
    (_0, _1, ...)."""
    from . import hdf5 as H5

    f = H5.H5File(filename_h5)
    out_path = filename_xdmf or filename_h5.replace(".h5", ".xmf")
    verts = f.dataset("/geometry/vertices")
    cells = f.dataset("/viz/topology/cells")
    nv, dim = verts.shape
    if dim == 1:
        return None
    nc, ncorners = cells.shape
    cell_dim = int(f.attrs("/viz/topology/cells").get("cell_dim", dim))
    cell_type = _XDMF_CELL_TYPES.get((cell_dim, ncorners), "Unknown")
    times = f.dataset("/time").ravel() if f.has("/time") else None
    fields = [_xdmf_field(f, g, k) for g in ("vertex_fields", "cell_fields") if f.has("/" + g) for k in f.keys("/" + g)]

    x = _XdmfLines()
    x(0, '<?xml version="1.0" ?>')
    x(0, '<!DOCTYPE Xdmf SYSTEM "Xdmf.dtd" [')
    x(0, f'<!ENTITY HeavyData "{os.path.basename(filename_h5)}">')
    x(0, "]>")
    x(0, "")
    x(0, "<Xdmf>")
    x(1, '<Domain Name="domain">')
    x.item(2, f'Name="cells" ItemType="Uniform" Format="HDF" NumberType="Float" Precision="8" '
              f'Dimensions="{nc} {ncorners}"', _HEAVY + "/viz/topology/cells")
    if dim == 3:
        x.item(2, f'Name="vertices" ItemType="Uniform" Format="HDF" Dimensions="{nv} {dim}"',
               _HEAVY + "/geometry/vertices")
    elif dim == 2:
        x(2, f'<DataItem Name="vertices" ItemType="Function" Dimensions="{nv} 3" Function="JOIN($0, $1, $2)">')
        for axis, comp in (("X", 0), ("Y", 1)):
            x(3, f'<DataItem Name="vertices{axis}" ItemType="Hyperslab" Type="HyperSlab" Dimensions="{nv} 1">')
            x.item(4, 'Dimensions="3 2" Format="XML"', f"0 {comp}   1 1   {nv} 1")
            x.item(4, f'Dimensions="{nv} 1" Format="HDF"', _HEAVY + "/geometry/vertices")
            x(3, "</DataItem>")
        x(3, f'<DataItem Name="verticesZ" ItemType="Function" Dimensions="{nv} 1" Function="0*$0">')
        x.item(4, 'Reference="XML"', '/Xdmf/Domain/DataItem[@Name="vertices"]/DataItem[@Name="verticesX"]')
        x(3, "</DataItem>")
        x(2, "</DataItem>")
    else:
        raise ValueError(f"unexpected spatial dimension {dim} of the domain vertices")

    def grid(step: Optional[int]) -> None:
        x(3, '<Grid Name="domain" GridType="Uniform">')
        x(4, f'<Topology TopologyType="{cell_type}" NumberOfElements="{nc}">')
        x.item(5, 'Reference="XML"', '/Xdmf/Domain/DataItem[@Name="cells"]')
        x(4, "</Topology>")
        x(4, '<Geometry GeometryType="XYZ">')
        x.item(5, 'Reference="XML"', '/Xdmf/Domain/DataItem[@Name="vertices"]')
        x(4, "</Geometry>")
        at = 0 if step is None else step
        for name, xtype, center, path, steps, points, comps in fields:
            hdf = f'DataType="Float" Precision="8" Dimensions="{steps} {points} {comps}" Format="HDF"'
            if xtype in ("Tensor6", "Matrix"):
                suffixes = (_XDMF_TENSOR_SUFFIXES[dim] if xtype == "Tensor6" else
                            tuple(f"_{i}" for i in range(comps)))
                for i in range(comps):
                    x(4, f'<Attribute Name="{name}{suffixes[i]}" Type="Scalar" Center="{center}">')
                    x(5, f'<DataItem ItemType="HyperSlab" Dimensions="1 {points} 1" Type="HyperSlab">')
                    x.item(6, 'Dimensions="3 3" Format="XML"', f"{at} 0 {i}    1 1 1    1 {points} 1")
                    x.item(6, hdf, _HEAVY + path)
                    x(5, "</DataItem>")
                    x(4, "</Attribute>")
                continue
            x(4, f'<Attribute Name="{name}" Type="{xtype}" Center="{center}">')
            if dim == 2 and xtype == "Vector":
                x(5, f'<DataItem ItemType="Function" Dimensions="{points} 3" Function="JOIN($0, $1, $2)">')
                for comp in (0, 1):
                    x(6, f'<DataItem ItemType="HyperSlab" Dimensions="{points} 1" Type="HyperSlab">')
                    x.item(7, 'Dimensions="3 3" Format="XML"', f"{at} 0 {comp}    1 1 1    1 {points} 1")
                    x.item(7, hdf, _HEAVY + path)
                    x(6, "</DataItem>")
                grid_ref = "/Xdmf/Domain/Grid" if step is None else "/Xdmf/Domain/Grid/Grid[1]"
                x(6, f'<DataItem ItemType="Function" Dimensions="{points} 1" Function="0*$0">')
                x.item(7, 'Reference="XML"', f'{grid_ref}/Attribute[@Name="{name}"]/DataItem[1]/DataItem[1]')
                x(6, "</DataItem>")
                x(5, "</DataItem>")
            else:
                x(5, f'<DataItem ItemType="HyperSlab" Dimensions="1 {points} {comps}" Type="HyperSlab">')
                x.item(6, 'Dimensions="3 3" Format="XML"', f"{at} 0 0    1 1 1    1 {points} {comps}")
                x.item(6, hdf, _HEAVY + path)
                x(5, "</DataItem>")
            x(4, "</Attribute>")
        x(3, "</Grid>")

    if times is not None:
        x(2, '<Grid Name="TimeSeries" GridType="Collection" CollectionType="Temporal">')
        x(3, '<Time TimeType="List">')
        x(4, f'<DataItem Format="XML" NumberType="Float" Dimensions="{len(times)}">')
        x(4, "".join("  %16.8e" % t for t in times))
        x(4, "</DataItem>")
        x(3, "</Time>")
        for step in range(len(times)):
            grid(step)
        x(2, "</Grid>")
    else:
        grid(None)
    x(1, "</Domain>")
    x(0, "</Xdmf>")
    with open(out_path, "w") as fh:
        fh.write(x.text())
    return out_path


@dataclass
class DataWriterHDF5Ext(DataWriterHDF5):
    """The reference's DataWriterHDF5Ext (libsrc/pylith/meshio/DataWriterHDF5Ext.hh): the HDF5
    file holds the mesh and /time as DataWriterHDF5 writes them, while every field's values go
    to a raw file of big-endian FP64 values, <file base>_<field>.dat (_datasetFilename,
    DataWriterHDF5Ext.cc:518-529), one step after another; the field's dataset in the HDF5 file
    refers to that file (an external dataset, HDF5::createDatasetRawExternal) with dimensions
    steps x points x components (at most one step for an info file) and carries the attribute
    vector_field_type. No Xdmf file is written (DataWriterHDF5Ext::close)."""

    _raw: dict = field(default_factory=dict)

    def dataset_filename(self, name: str) -> str:
        base = self.hdf5_filename()
        i = base.find(".h5")
        return (base[:i] if i >= 0 else base) + f"_{name}.dat"

    def _store(self, key: str, name: str, v: np.ndarray, vtype: str, istep: int) -> None:
        if istep == 0:
            fn = self.dataset_filename(name)
            self._raw[key] = open(fn, "wb")
            self._h5.create_external(key, fn, v.shape, ">f8", 1 if self.is_info else None,
                                     attrs={"vector_field_type": vtype})
        fh = self._raw[key]
        fh.write(v.astype(">f8").tobytes())
        fh.flush()
        self._h5.extend(key, istep + 1)

    def close(self) -> None:
        for fh in self._raw.values():
            fh.close()
        self._raw = {}
        if self._h5 is not None:
            self._h5.close()
            self._h5 = None
