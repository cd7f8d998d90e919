"""Mesh ingest: Gmsh 4.1 (ASCII and binary) and ExodusII (NetCDF classic / 64-bit offset) readers.

The reference reads Gmsh files through PETSc's DMPlex Gmsh reader
(libsrc/pylith/meshio/MeshIOPetsc.cc:126-240, with `dm_plex_gmsh_use_regions` and vertex marking)
and ExodusII files with its own NetCDF reader (libsrc/pylith/meshio/MeshIOCubit.cc:241-400). The
conventions kept here are the reference's:

  * cells carry a material id: the physical tag of their Gmsh volume entity, or the ExodusII
    element-block id (`eb_prop1`, MeshIOCubit.cc:291-336);
  * boundary conditions refer to vertex groups: the vertices of every lower-dimensional Gmsh
    physical group, named by `$PhysicalNames` (MeshIOPetsc.cc:329-380 keeps only the vertices of
    such labels), or ExodusII node sets named by `ns_names` (MeshIOCubit.cc:346-393);
  * ExodusII connectivity and node sets are 1-based (MeshIOCubit.cc:333,385).

Cells come back in the engine's conventions (see pylith_b200.meshing): positively oriented P1
tetrahedra and Q1 hexahedra with corners (0,0,0),(1,0,0),(1,1,0),(0,1,0),(0,0,1),... (the Gmsh and
ExodusII HEX8 order); tetrahedra and hexahedra with a negative Jacobian determinant are
reflected. Only the nodes that cells use are kept.
"""
from __future__ import annotations

import dataclasses
import struct
from typing import Dict

import numpy as np

from . import meshing as M

# Gmsh element types and their node counts (Gmsh reference manual, "MSH file format")
_GMSH_NODES = {1: 2, 2: 3, 3: 4, 4: 4, 5: 8, 6: 6, 7: 5, 8: 3, 9: 6, 10: 9, 11: 10, 12: 27, 15: 1}
_GMSH_CELLS = {4: M.CELL_TET4, 5: M.CELL_HEX8}


@dataclasses.dataclass
class MeshData:
    mesh: M.Mesh
    material_ids: np.ndarray                 # int32 [ncells]
    vertex_groups: Dict[str, np.ndarray]     # name -> sorted node indices (int64)


class MeshIOError(ValueError):
    pass


def _orient(cell_type: int, coords: np.ndarray, cells: np.ndarray) -> np.ndarray:
    cells = cells.copy()
    if cell_type == M.CELL_TET4:
        X = coords[cells]
        det = np.einsum("ij,ij->i", np.cross(X[:, 1] - X[:, 0], X[:, 2] - X[:, 0]), X[:, 3] - X[:, 0])
        if np.any(det == 0.0):
            raise MeshIOError("degenerate tetrahedron in mesh")
        neg = det < 0
        cells[neg] = cells[neg][:, [0, 2, 1, 3]]
    else:
        X = coords[cells]
        # Jacobian at the cell centre from the trilinear map
        dx = (X[:, 1] + X[:, 2] + X[:, 5] + X[:, 6] - X[:, 0] - X[:, 3] - X[:, 4] - X[:, 7]) / 4
        dy = (X[:, 2] + X[:, 3] + X[:, 6] + X[:, 7] - X[:, 0] - X[:, 1] - X[:, 4] - X[:, 5]) / 4
        dz = (X[:, 4] + X[:, 5] + X[:, 6] + X[:, 7] - X[:, 0] - X[:, 1] - X[:, 2] - X[:, 3]) / 4
        det = np.einsum("ij,ij->i", np.cross(dx, dy), dz)
        if np.any(det == 0.0):
            raise MeshIOError("degenerate hexahedron in mesh")
        neg = det < 0
        cells[neg] = cells[neg][:, [4, 5, 6, 7, 0, 1, 2, 3]]
    return cells


def _compact(cell_type, coords, cells, material_ids, groups) -> MeshData:
    used = np.unique(cells)
    remap = -np.ones(coords.shape[0], dtype=np.int64)
    remap[used] = np.arange(used.size)
    coords = np.ascontiguousarray(coords[used], dtype=np.float64)
    cells = remap[cells].astype(np.int32)
    cells = _orient(cell_type, coords, cells)
    out = {}
    for name, nodes in groups.items():
        r = remap[np.asarray(nodes, dtype=np.int64)]
        out[name] = np.unique(r[r >= 0])
    return MeshData(M.Mesh(cell_type, coords, np.ascontiguousarray(cells)),
                    np.asarray(material_ids, dtype=np.int32), out)


# ---------------------------------------------------------------------------------------------
# Gmsh 4.1


class _Tokens:
    """Reads the values of one Gmsh section: whitespace-separated text, or packed binary
    (int = int32, size_t = uint64, double = float64, native little-endian)."""

    def __init__(self, data: bytes, pos: int, binary: bool):
        self.data = data
        self.pos = pos
        self.binary = binary

    def _word(self) -> bytes:
        d, n = self.data, len(self.data)
        i = self.pos
        while i < n and d[i] in b" \t\r\n":
            i += 1
        j = i
        while j < n and d[j] not in b" \t\r\n":
            j += 1
        if i == j:
            raise MeshIOError("unexpected end of Gmsh file")
        self.pos = j
        return d[i:j]

    def ints(self, count: int, size_t: bool = False) -> np.ndarray:
        if not self.binary:
            return np.array([int(self._word()) for _ in range(count)], dtype=np.int64)
        dt = np.uint64 if size_t else np.int32
        nbytes = count * np.dtype(dt).itemsize
        a = np.frombuffer(self.data, dtype=dt, count=count, offset=self.pos).astype(np.int64)
        self.pos += nbytes
        return a

    def int(self) -> int:
        return int(self.ints(1)[0])

    def size(self) -> int:
        return int(self.ints(1, size_t=True)[0])

    def doubles(self, count: int) -> np.ndarray:
        if not self.binary:
            return np.array([float(self._word()) for _ in range(count)], dtype=np.float64)
        a = np.frombuffer(self.data, dtype=np.float64, count=count, offset=self.pos).copy()
        self.pos += 8 * count
        return a


def _line(data: bytes, pos: int):
    j = data.find(b"\n", pos)
    if j < 0:
        j = len(data)
    return data[pos:j].strip(), j + 1


def _expect_end(data: bytes, pos: int, name: str) -> int:
    tag = b"$End" + name.encode()
    j = data.find(tag, pos)
    if j < 0:
        raise MeshIOError(f"missing {tag.decode()}")
    return data.find(b"\n", j) + 1 if data.find(b"\n", j) >= 0 else len(data)


def read_gmsh(path: str) -> MeshData:
    """Gmsh MSH 4.1 file (ASCII or binary) with P1 tetrahedra or Q1 hexahedra."""
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    binary = False
    names: Dict[tuple, str] = {}
    entity_phys: Dict[tuple, list] = {}
    node_tags, node_xyz = [], []
    blocks = []  # (dim, entity tag, element type, connectivity tags [n, k])
    while pos < len(data):
        line, pos = _line(data, pos)
        if not line:
            continue
        if not line.startswith(b"$"):
            raise MeshIOError(f"unexpected line in Gmsh file: {line[:40]!r}")
        section = line[1:].decode()
        if section == "MeshFormat":
            fmt, pos = _line(data, pos)
            version, ftype, dsize = fmt.split()
            if not version.startswith(b"4"):
                raise MeshIOError(f"Gmsh format {version.decode()} is not supported (4.1 is)")
            binary = int(ftype) == 1
            if binary:
                if int(dsize) != 8:
                    raise MeshIOError("binary Gmsh files need 8-byte size_t")
                (one,) = struct.unpack_from("<i", data, pos)
                if one != 1:
                    raise MeshIOError("big-endian binary Gmsh files are not supported")
                pos += 4
            pos = _expect_end(data, pos, section)
        elif section == "PhysicalNames":
            count, pos = _line(data, pos)
            for _ in range(int(count)):
                ln, pos = _line(data, pos)
                dim, tag, name = ln.split(maxsplit=2)
                names[(int(dim), int(tag))] = name.decode().strip('"')
            pos = _expect_end(data, pos, section)
        elif section == "Entities":
            t = _Tokens(data, pos, binary)
            counts = [t.size() for _ in range(4)]
            for dim in range(4):
                for _ in range(counts[dim]):
                    tag = t.int()
                    t.doubles(3 if dim == 0 else 6)
                    phys = [int(v) for v in t.ints(t.size())]
                    if dim > 0:
                        t.ints(t.size())  # bounding entities
                    entity_phys[(dim, tag)] = phys
            pos = _expect_end(data, t.pos, section)
        elif section == "PartitionedEntities":
            raise MeshIOError("partitioned Gmsh files are not supported")
        elif section == "Nodes":
            t = _Tokens(data, pos, binary)
            nblocks = t.size()
            t.size(), t.size(), t.size()
            for _ in range(nblocks):
                t.int()
                t.int()
                parametric = t.int()
                n = t.size()
                if parametric:
                    raise MeshIOError("parametric Gmsh nodes are not supported")
                node_tags.append(t.ints(n, size_t=True))
                node_xyz.append(t.doubles(3 * n).reshape(n, 3))
            pos = _expect_end(data, t.pos, section)
        elif section == "Elements":
            t = _Tokens(data, pos, binary)
            nblocks = t.size()
            t.size(), t.size(), t.size()
            for _ in range(nblocks):
                dim = t.int()
                etag = t.int()
                etype = t.int()
                n = t.size()
                if etype not in _GMSH_NODES:
                    raise MeshIOError(f"Gmsh element type {etype} is not supported")
                k = _GMSH_NODES[etype]
                conn = t.ints(n * (k + 1), size_t=True).reshape(n, k + 1)[:, 1:]
                blocks.append((dim, etag, etype, conn))
            pos = _expect_end(data, t.pos, section)
        else:
            pos = _expect_end(data, pos, section)
    if not node_tags or not blocks:
        raise MeshIOError("Gmsh file has no nodes or no elements")
    tags = np.concatenate(node_tags)
    xyz = np.concatenate(node_xyz)
    lookup = -np.ones(int(tags.max()) + 1, dtype=np.int64)
    lookup[tags] = np.arange(tags.size)
    cell_blocks = [b for b in blocks if b[0] == 3]
    if not cell_blocks:
        raise MeshIOError("Gmsh file has no 3-D elements")
    types = {b[2] for b in cell_blocks}
    if len(types) != 1 or next(iter(types)) not in _GMSH_CELLS:
        raise MeshIOError(f"3-D Gmsh elements must all be tetrahedra or all hexahedra (found types {sorted(types)})")
    cell_type = _GMSH_CELLS[next(iter(types))]
    cells = np.concatenate([lookup[b[3]] for b in cell_blocks])
    mats = np.concatenate([np.full(len(b[3]), (entity_phys.get((3, b[1])) or [0])[0]) for b in cell_blocks])
    groups: Dict[str, list] = {}
    for dim, etag, _, conn in blocks:
        if dim == 3:
            continue
        for ptag in entity_phys.get((dim, etag), []):
            name = names.get((dim, ptag), str(ptag))
            groups.setdefault(name, []).append(lookup[conn].ravel())
    groups = {k: np.concatenate(v) for k, v in groups.items()}
    if np.any(cells < 0):
        raise MeshIOError("element refers to an undefined node")
    return _compact(cell_type, xyz, cells, mats, groups)


def write_gmsh(path: str, data: MeshData, binary: bool = False) -> None:
    """MSH 4.1 writer (one volume entity per material id, one point entity per vertex group,
    written as point elements): enough for round trips through read_gmsh."""
    mesh = data.mesh
    etype = {M.CELL_TET4: 4, M.CELL_HEX8: 5}[mesh.cell_type]
    mats = sorted(set(int(m) for m in data.material_ids))
    gnames = list(data.vertex_groups)
    out = bytearray()

    def text(s: str):
        out.extend(s.encode())

    def put(fmt: str, *vals):
        if binary:
            out.extend(struct.pack("<" + fmt, *vals))
        else:
            text(" ".join(repr(float(v)) if c == "d" else str(int(v)) for c, v in zip(fmt, vals)) + "\n")

    def put_array(a: np.ndarray, dt):
        if binary:
            out.extend(np.ascontiguousarray(a, dtype=dt).tobytes())
        else:
            for row in np.atleast_2d(a):
                text(" ".join(repr(float(v)) if dt == np.float64 else str(int(v)) for v in row) + "\n")

    text("$MeshFormat\n4.1 %d 8\n" % (1 if binary else 0))
    if binary:
        out.extend(struct.pack("<i", 1))
        text("\n")
    text("$EndMeshFormat\n$PhysicalNames\n%d\n" % (len(mats) + len(gnames)))
    for m in mats:
        text('3 %d "material-id:%d"\n' % (m, m))
    for i, g in enumerate(gnames):
        text('0 %d "%s"\n' % (i + 1, g))
    text("$EndPhysicalNames\n$Entities\n")
    put("QQQQ", len(gnames), 0, 0, len(mats))
    for i in range(len(gnames)):
        put("idddQi", i + 1, 0.0, 0.0, 0.0, 1, i + 1)
    for m in mats:
        put("iddddddQiQ", m, 0, 0, 0, 0, 0, 0, 1, m, 0)
    text("$EndEntities\n$Nodes\n")
    n = mesh.num_nodes
    put("QQQQ", 1, n, 1, n)
    put("iiiQ", 3, mats[0], 0, n)
    put_array(np.arange(1, n + 1)[:, None], np.uint64)
    put_array(mesh.coords, np.float64)
    text("$EndNodes\n$Elements\n")
    npoint = sum(len(v) for v in data.vertex_groups.values())
    put("QQQQ", len(mats) + len(gnames), mesh.num_cells + npoint, 1, mesh.num_cells + npoint)
    tag = 1
    for m in mats:
        sel = np.flatnonzero(np.asarray(data.material_ids) == m)
        put("iiiQ", 3, m, etype, sel.size)
        rows = np.concatenate([np.arange(tag, tag + sel.size)[:, None], mesh.cells[sel] + 1], axis=1)
        put_array(rows, np.uint64)
        tag += sel.size
    for i, g in enumerate(gnames):
        v = np.asarray(data.vertex_groups[g])
        put("iiiQ", 0, i + 1, 15, v.size)
        put_array(np.stack([np.arange(tag, tag + v.size), v + 1], axis=1), np.uint64)
        tag += v.size
    text("$EndElements\n")
    with open(path, "wb") as f:
        f.write(bytes(out))


# ---------------------------------------------------------------------------------------------
# ExodusII


def _names(var) -> list:
    raw = np.asarray(var[:])
    return [b"".join(r).split(b"\0")[0].decode().strip() for r in raw]


def read_exodus(path: str) -> MeshData:
    """ExodusII file (NetCDF classic or 64-bit offset) with TETRA or HEX8 element blocks."""
    from scipy.io import netcdf_file

    with netcdf_file(path, "r", mmap=False) as nc:
        v = nc.variables
        if "coord" in v:
            coords = np.asarray(v["coord"][:], dtype=np.float64).T.copy()
        else:
            coords = np.stack([np.asarray(v[f"coord{c}"][:], dtype=np.float64) for c in "xyz"], axis=1)
        nblk = int(nc.dimensions["num_el_blk"])
        ids = np.asarray(v["eb_prop1"][:], dtype=np.int64)
        cells, mats, ctype = [], [], None
        for b in range(1, nblk + 1):
            conn = v[f"connect{b}"]
            et = conn._attributes.get("elem_type", b"").decode().upper()
            t = M.CELL_TET4 if et.startswith("TET") else M.CELL_HEX8 if et.startswith("HEX") else None
            if t is None or (t == M.CELL_HEX8 and conn.shape[1] != 8) or (t == M.CELL_TET4 and conn.shape[1] != 4):
                raise MeshIOError(f"element block {b}: type {et} with {conn.shape[1]} nodes is not supported")
            if ctype is not None and t != ctype:
                raise MeshIOError("all element blocks must have the same cell type")
            ctype = t
            cells.append(np.asarray(conn[:], dtype=np.int64) - 1)
            mats.append(np.full(conn.shape[0], ids[b - 1]))
        groups = {}
        if "num_node_sets" in nc.dimensions and int(nc.dimensions["num_node_sets"]) > 0:
            nns = int(nc.dimensions["num_node_sets"])
            gnames = _names(v["ns_names"]) if "ns_names" in v else [str(i) for i in v["ns_prop1"][:]]
            for i in range(nns):
                groups[gnames[i]] = np.asarray(v[f"node_ns{i + 1}"][:], dtype=np.int64) - 1
    return _compact(ctype, coords, np.concatenate(cells), np.concatenate(mats), groups)


def read(path: str) -> MeshData:
    """Dispatch on the file suffix (.msh: Gmsh; .exo/.e/.gen: ExodusII), as
    MeshIOPetsc.cc:126-130 dispatches on `.msh`."""
    low = path.lower()
    if low.endswith(".msh"):
        return read_gmsh(path)
    if low.endswith((".exo", ".e", ".gen", ".g")):
        return read_exodus(path)
    raise MeshIOError(f"unknown mesh file type: {path}")


def constrained_mask(data: MeshData, bcs) -> np.ndarray:
    """Boolean mask over the displacement DOFs (3 per node) of Dirichlet conditions given as
    (vertex-group name, constrained components), the `label` and `constrained_dof` of the
    reference's DirichletTimeDependent (libsrc/pylith/bc/DirichletTimeDependent.cc,
    ConstraintSpatialDB.cc:85)."""
    mask = np.zeros((data.mesh.num_nodes, 3), dtype=bool)
    for name, comps in bcs:
        if name not in data.vertex_groups:
            raise MeshIOError(f"no vertex group named {name!r}")
        for c in comps:
            mask[data.vertex_groups[name], int(c)] = True
    return mask.ravel()
