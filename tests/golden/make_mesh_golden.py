"""Generate tests/golden/reference_meshes.npz from the reference's own test meshes.

The reference's 3-D elasticity tests run on four small meshes of an 8 km box:
  * tests/mmstests/linearelasticity/nofaults-3d/data/{tet,hex}.msh (Gmsh 4.1 ASCII; the
    UniformStrain3D MMS, material 24, vertex group `boundary`);
  * tests/fullscale/linearelasticity/nofaults-3d/mesh_{tet,hex}.exo (ExodusII; the axial
    displacement test axialdisp.cfg, materials 1 and 2, groups boundary_{x,y,z}{neg,pos}).
This script reads them with pylith_b200.meshio (the PyLith source tree must be present) and keeps
what the tests use -- cell type, coordinates, cells (as the reader numbers and orients them),
material ids and vertex groups -- so that GPU tests, which run where the PyLith sources are not,
can put the reference's meshes through the CUDA path. The CPU tests in tests/test_meshio.py check
that reading the files again reproduces this fixture.

    PYLITH_SRC=path/to/pylith python tests/golden/make_mesh_golden.py
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from pylith_b200 import meshio as MIO  # noqa: E402

MESHES = {
    "mms_tet": "tests/mmstests/linearelasticity/nofaults-3d/data/tet.msh",
    "mms_hex": "tests/mmstests/linearelasticity/nofaults-3d/data/hex.msh",
    "axial_tet": "tests/fullscale/linearelasticity/nofaults-3d/mesh_tet.exo",
    "axial_hex": "tests/fullscale/linearelasticity/nofaults-3d/mesh_hex.exo",
}
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_meshes.npz")


def read_all(pylith):
    return {key: MIO.read(os.path.join(pylith, rel)) for key, rel in MESHES.items()}


def pack(datas):
    arrays, meta = {}, {}
    for key, d in datas.items():
        arrays[f"{key}_coords"] = d.mesh.coords
        arrays[f"{key}_cells"] = d.mesh.cells.astype(np.int32)
        arrays[f"{key}_material_ids"] = d.material_ids.astype(np.int32)
        groups = sorted(d.vertex_groups)
        for j, g in enumerate(groups):
            arrays[f"{key}_group{j}"] = np.asarray(d.vertex_groups[g], dtype=np.int64)
        meta[key] = {"source": MESHES[key], "cell_type": int(d.mesh.cell_type), "groups": groups}
    return arrays, meta


def load(path=OUT):
    """{key: MeshData} from the fixture."""
    from pylith_b200 import meshing as M

    z = np.load(path)
    meta = json.loads(str(z["meta"]))
    out = {}
    for key, m in meta.items():
        mesh = M.Mesh(m["cell_type"], z[f"{key}_coords"], z[f"{key}_cells"])
        groups = {g: z[f"{key}_group{j}"] for j, g in enumerate(m["groups"])}
        out[key] = MIO.MeshData(mesh, z[f"{key}_material_ids"], groups)
    return out


def main(pylith=None):
    pylith = pylith or os.environ.get("PYLITH_SRC")
    if not pylith:
        sys.exit("set PYLITH_SRC to the PyLith source tree")
    arrays, meta = pack(read_all(pylith))
    np.savez_compressed(OUT, meta=np.array(json.dumps(meta)), **arrays)
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main(*sys.argv[1:])
