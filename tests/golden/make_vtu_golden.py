"""Generate tests/golden/vtu_golden.npz from the reference's golden VTK files.

The reference's writer tests (tests/libtests/meshio/TestDataWriterVTK*.cc) compare their output
with the files tests/libtests/meshio/data/{tet4,hex8}_{vertex,cell}_t10.vtu. This script reads
those files (the PyLith source tree must be present), keeps their mesh, cell types and field
arrays (names and values, in file order) and the SHA-256 of every file, so that the writer in
pylith_b200/output.py can be checked byte for byte against them without the PyLith sources.

    PYLITH_SRC=path/to/pylith python tests/golden/make_vtu_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from pylith_b200 import output as OUT  # noqa: E402

FILES = ["tet4_vertex_t10.vtu", "tet4_cell_t10.vtu", "hex8_vertex_t10.vtu", "hex8_cell_t10.vtu"]


def main(pylith=None):
    pylith = pylith or os.environ.get("PYLITH_SRC")
    if not pylith:
        sys.exit("set PYLITH_SRC to the PyLith source tree")
    data_dir = os.path.join(pylith, "tests", "libtests", "meshio", "data")
    arrays, meta = {}, {}
    for i, name in enumerate(FILES):
        path = os.path.join(data_dir, name)
        raw = open(path, "rb").read()
        pts, conn, offs, types, cell, point = OUT.read_vtu(path)
        nen = int(offs[0]) if len(offs) else 0
        arrays[f"f{i}_points"] = pts
        arrays[f"f{i}_cells"] = conn.reshape(-1, nen)
        for j, (k, v) in enumerate(cell.items()):
            arrays[f"f{i}_cell{j}"] = v
        for j, (k, v) in enumerate(point.items()):
            arrays[f"f{i}_point{j}"] = v
        meta[name] = {"index": i, "vtk_type": int(types[0]), "cell_names": list(cell.keys()),
                      "point_names": list(point.keys()), "sha256": hashlib.sha256(raw).hexdigest(),
                      "size": len(raw)}
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "vtu_golden.npz")
    np.savez(out, meta=np.array(json.dumps(meta)), **arrays)
    print(f"wrote {out}")


if __name__ == "__main__":
    main(*sys.argv[1:])
