"""Generate tests/golden/h5_golden.npz from the reference's golden HDF5 files.

The reference's HDF5 writer tests (tests/libtests/meshio/TestDataWriterHDF5*.cc) compare their
output with tests/libtests/meshio/data/*.h5, files written through PETSc's HDF5 viewer by the
HDF5 library. No HDF5 library is available here, so this script reads them with
pylith_b200.hdf5 (written from the file-format specification) and first pins that reader with
facts that do not come from the files' encoding:

  * every file of the reference tree parses, every dataset and attribute decodes;
  * /geometry/vertices of the mesh cases are the vertices of the ASCII meshes the tests read
    (tests/libtests/meshio/data/{tri3,quad4,tet4,hex8}.mesh), fault vertices repeated;
  * the vertex and cell fields equal the tests' analytic field (TestDataWriterMesh.cc:235-270):
    value[i] = +-1.1 + 2 ncomp / 7 + i + sum_d x_d / (0.1 c_d), c = (11, 13, 17), x the vertex or
    the cell centroid in coordinates scaled by the tests' length scale 0.1, the sign that of the
    cell centroid's x (so that of x for vertices off the fault);
  * /time holds the tests' one time, 1.0, and each field's vector_field_type is its name.

It then keeps, for the tet4 and hex8 vertex, cell and station (points) files, every dataset (values, shapes) and
attribute, and the SHA-256 of each file, so that tests/test_hdf5.py can check the writer in
pylith_b200/output.py against them without the PyLith sources.

    PYLITH_SRC=path/to/pylith python tests/golden/make_h5_golden.py
"""
import glob
import hashlib
import json
import os
import re
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from pylith_b200 import hdf5 as H5  # noqa: E402

KEEP = ["tet4_vertex.h5", "tet4_cell.h5", "hex8_vertex.h5", "hex8_cell.h5", "tet4_points_vertex.h5",
        "hex8_points_vertex.h5"]
MESH_CASES = {"tri3": 2, "quad4": 2, "tet4": 3, "hex8": 3}
LENGTH_SCALE = 0.1
CONSTANTS = (11.0, 13.0, 17.0)


def ascii_mesh_vertices(path: str) -> np.ndarray:
    """Vertex coordinates of a PyLith ASCII mesh (MeshIOAscii): the `coordinates` block."""
    text = open(path).read()
    m = re.search(r"vertices\s*=\s*\{(.*?)coordinates\s*=\s*\{(.*?)\}", text, re.S)
    dim = int(re.search(r"dimension\s*=\s*(\d+)", m.group(1)).group(1))
    rows = [ln.split() for ln in m.group(2).strip().splitlines() if ln.strip()]
    return np.array([[float(v) for v in r[1:1 + dim]] for r in rows])


def analytic(x: np.ndarray, ncomp: int) -> np.ndarray:
    """The tests' field without its fault-side offset: 2 ncomp / 7 + i + sum_d x_d / c_d."""
    xs = x / LENGTH_SCALE
    base = sum(xs[:, d] / CONSTANTS[d] for d in range(x.shape[1]))
    return 2.0 * ncomp / 7.0 + np.arange(ncomp)[None, :] + base[:, None]


def check_offsets(res: np.ndarray, side_x: np.ndarray, what: str) -> None:
    """res = value - analytic must be -1.1 where side_x < 0 and +1.1 where side_x > 0 (either
    sign where side_x = 0, the same for all components of a point)."""
    assert np.allclose(np.abs(res), 1.1, rtol=0, atol=1e-12), what
    assert np.allclose(res, res[:, :1], rtol=0, atol=1e-12), what
    neg, pos = side_x < -1e-12, side_x > 1e-12
    assert np.all(res[neg] < 0) and np.all(res[pos] > 0), what


def pin(data_dir: str, f: H5.H5File, case: str, where: str) -> None:
    dim = MESH_CASES[case]
    verts = f.dataset("/geometry/vertices")
    mesh = ascii_mesh_vertices(os.path.join(data_dir, f"{case}.mesh"))
    assert verts.shape[1] == dim == mesh.shape[1]
    on_mesh = [np.min(np.abs(mesh - v).max(axis=1)) == 0.0 for v in verts]
    assert all(on_mesh) and len({tuple(v) for v in verts}) == len(mesh), case
    cells = f.dataset("/viz/topology/cells")
    a = f.attrs("/viz/topology/cells")
    assert int(a["cell_corners"]) == cells.shape[1] and int(a["cell_dim"]) == dim
    centroids = verts[cells].mean(axis=1)
    assert np.array_equal(f.dataset("/time"), np.ones((1, 1, 1)))
    group, points, side = (("/vertex_fields", verts, None) if where == "vertex" else
                           ("/cell_fields", centroids, centroids[:, 0]))
    names = [k for k in f.keys(group) if k != "partition_rank"]
    assert names == ["other", "scalar", "tensor", "vector"], names
    for k in names:
        v = f.dataset(f"{group}/{k}")
        assert v.shape[:2] == (1, len(points)), (case, k, v.shape)
        assert f.attrs(f"{group}/{k}")["vector_field_type"] == k
        res = v[0] - analytic(points, v.shape[2])
        if side is None:  # a vertex takes the side of the cell it was evaluated in
            side_v = np.where(np.abs(points[:, 0]) > 1e-12, points[:, 0], 0.0)
            check_offsets(res, side_v, f"{case} {k}")
        else:
            check_offsets(res, side, f"{case} {k}")


def main(pylith=None):
    pylith = pylith or os.environ.get("PYLITH_SRC")
    if not pylith:
        sys.exit("set PYLITH_SRC to the PyLith source tree")
    data_dir = os.path.join(pylith, "tests", "libtests", "meshio", "data")
    every = sorted(glob.glob(os.path.join(pylith, "tests", "**", "*.h5"), recursive=True))
    for path in every:  # every file parses and decodes
        f = H5.H5File(path)
        for p in f.walk():
            f.attrs(p)
            if not f.is_group(p):
                f.dataset(p)
    for case in MESH_CASES:
        for where in ("vertex", "cell"):
            pin(data_dir, H5.H5File(os.path.join(data_dir, f"{case}_{where}.h5")), case, where)
    arrays, meta = {}, {"files_read": len(every)}
    for i, name in enumerate(KEEP):
        path = os.path.join(data_dir, name)
        f = H5.H5File(path)
        entry = {"sha256": hashlib.sha256(open(path, "rb").read()).hexdigest(), "datasets": {}, "groups": []}
        for j, p in enumerate(f.walk()):
            attrs = {k: (v if isinstance(v, str) else np.asarray(v).tolist()) for k, v in f.attrs(p).items()}
            if f.is_group(p):
                entry["groups"].append(p)
                continue
            arrays[f"f{i}_d{j}"] = f.dataset(p)
            entry["datasets"][p] = {"key": f"f{i}_d{j}", "attrs": attrs}
        meta[name] = entry
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "h5_golden.npz")
    np.savez_compressed(out, meta=json.dumps(meta), **arrays)
    print(f"pinned the reader on {len(every)} files; wrote {out}")


if __name__ == "__main__":
    main()
