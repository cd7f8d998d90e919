"""Generate tests/golden/xdmf_golden.json from the reference's golden Xdmf files.

The reference's Xdmf test (tests/pytests/meshio/TestXdmf.py) writes the Xdmf description of each
HDF5 file in tests/pytests/meshio/data and compares it line for line with the .xmf beside it.
An Xdmf file depends only on the HDF5 file's name, dataset shapes, a few attributes
(cell_dim, vector_field_type) and the time stamps. This script reads each pair (the PyLith source
tree must be present), checks that pylith_b200.output.write_xdmf reproduces the .xmf byte for
byte from the .h5, and keeps that metadata with the SHA-256 of each .xmf, so that
tests/test_hdf5.py can rebuild stand-in HDF5 files and check the Xdmf writer without the PyLith
sources.

    PYLITH_SRC=path/to/pylith python tests/golden/make_xdmf_golden.py
"""
import glob
import hashlib
import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from pylith_b200 import hdf5 as H5  # noqa: E402
from pylith_b200 import output as OUT  # noqa: E402

KEPT_ATTRS = ("cell_dim", "vector_field_type")


def describe(path: str) -> dict:
    f = H5.H5File(path)
    out = {"datasets": {}}
    for p in f.walk():
        if f.is_group(p):
            continue
        d = f.dataset(p)
        attrs = {k: (v if isinstance(v, str) else np.asarray(v).tolist()) for k, v in f.attrs(p).items()
                 if k in KEPT_ATTRS}
        entry = {"shape": list(d.shape), "dtype": d.dtype.str, "attrs": attrs}
        if p == "/time":
            entry["values"] = d.ravel().tolist()
        out["datasets"][p] = entry
    return out


def main(pylith=None):
    pylith = pylith or os.environ.get("PYLITH_SRC")
    if not pylith:
        sys.exit("set PYLITH_SRC to the PyLith source tree")
    data_dir = os.path.join(pylith, "tests", "pytests", "meshio", "data")
    meta = {}
    tmp = tempfile.mkdtemp()
    for xmf in sorted(glob.glob(os.path.join(data_dir, "*.xmf"))):
        h5 = xmf[:-4] + ".h5"
        name = os.path.basename(h5)
        golden = open(xmf, "rb").read()
        out = OUT.write_xdmf(h5, os.path.join(tmp, os.path.basename(xmf)))
        assert open(out, "rb").read() == golden, name
        meta[name] = {"xmf_sha256": hashlib.sha256(golden).hexdigest(), **describe(h5)}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "xdmf_golden.json")
    with open(path, "w") as fh:
        json.dump(meta, fh, indent=1, sort_keys=True)
    print(f"{len(meta)} Xdmf files reproduced; wrote {path}")


if __name__ == "__main__":
    main()
