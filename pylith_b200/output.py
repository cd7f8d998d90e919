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
        w = self._h5
        if istep == 0:
            w.create_series(key, v.shape, attrs={"timestepping": np.uint8(1), "vector_field_type": vtype})
        w.append(key, v)

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
        if self._h5 is not None:
            self._h5.close()
            self._h5 = None
