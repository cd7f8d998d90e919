"""VTK output (pylith_b200/output.py) against the reference's golden files.

tests/golden/vtu_golden.npz holds the meshes, field arrays and SHA-256 hashes of the reference's
tests/libtests/meshio/data/{tet4,hex8}_{vertex,cell}_t10.vtu (tests/golden/make_vtu_golden.py).
Writing the same mesh and fields must give the same bytes, both through write_vtu and through
the DataWriterVTK mirror with the reference's field names."""
import hashlib
import json
import os

import numpy as np
import pytest

from pylith_b200 import meshing as M
from pylith_b200 import output as OUT

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "vtu_golden.npz")


def _golden():
    d = np.load(GOLDEN)
    return d, json.loads(str(d["meta"]))


def _sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


@pytest.mark.parametrize("name", ["tet4_vertex_t10.vtu", "tet4_cell_t10.vtu", "hex8_vertex_t10.vtu",
                                  "hex8_cell_t10.vtu"])
def test_write_vtu_is_byte_identical_to_the_reference(tmp_path, name):
    d, meta = _golden()
    m = meta[name]
    i = m["index"]
    cell = [(k, d[f"f{i}_cell{j}"]) for j, k in enumerate(m["cell_names"]) if k != "Rank"]
    assert np.all(d[f"f{i}_cell{m['cell_names'].index('Rank')}"] == 0)
    point = [(k, d[f"f{i}_point{j}"]) for j, k in enumerate(m["point_names"])]
    path = str(tmp_path / name)
    OUT.write_vtu(path, d[f"f{i}_points"], d[f"f{i}_cells"], m["vtk_type"], point, cell)
    assert os.path.getsize(path) == m["size"]
    assert _sha(path) == m["sha256"]


@pytest.mark.parametrize("kind", ["tet4", "hex8"])
def test_data_writer_vtk_names_files_and_fields_as_the_reference(tmp_path, kind):
    d, meta = _golden()
    for where in ("vertex", "cell"):
        name = f"{kind}_{where}_t10.vtu"
        m = meta[name]
        i = m["index"]
        mesh = M.Mesh(M.CELL_TET4 if kind == "tet4" else M.CELL_HEX8, d[f"f{i}_points"],
                      d[f"f{i}_cells"].astype(np.int32))
        w = OUT.DataWriterVTK(filename=str(tmp_path / f"{kind}_{where}.vtu"), time_format="%3.1f")
        w.open(mesh)
        w.open_time_step(1.0)
        names = m["point_names"] if where == "vertex" else [k for k in m["cell_names"] if k != "Rank"]
        src = "point" if where == "vertex" else "cell"
        vals = {k: d[f"f{i}_{src}{(m['point_names'] if where == 'vertex' else m['cell_names']).index(k)}"]
                for k in names}
        add = w.write_vertex_field if where == "vertex" else w.write_cell_field
        add("scalarscalar", vals["scalarscalar.0" if where == "vertex" else "scalarscalar"])
        add("vectorvector", vals["vectorvector"], vector=True)
        add("tensortensor", np.concatenate([vals[f"tensortensor.{c}"] for c in range(6)], axis=1))
        add("otherother", np.concatenate([vals[f"otherother.{c}"] for c in range(2)], axis=1))
        path = w.close_time_step()
        assert os.path.basename(path) == name
        assert _sha(path) == m["sha256"], name
        w.close()


def test_vtk_filename_stamps():
    w = OUT.DataWriterVTK(filename="out/step.vtu", time_format="%05.2f", time_constant=2.0, time_scale=10.0)
    assert w.vtk_filename(0.5) == "out/step_t0250.vtu"
    assert OUT.DataWriterVTK(filename="a.vtu", is_info=True).vtk_filename(3.0) == "a_info.vtu"
    with pytest.raises(ValueError):
        OUT.DataWriterVTK(time_constant=0.0)


def test_q2_mesh_with_a_derived_cell_field_round_trips(tmp_path):
    mesh = M.box_hex27(3, 2, 2)
    rng = np.random.default_rng(3)
    u = rng.standard_normal((mesh.num_nodes, 3))
    stress = rng.standard_normal((mesh.num_cells, 6))
    w = OUT.DataWriterVTK(filename=str(tmp_path / "q2.vtu"), time_format="%4.2f")
    w.open(mesh)
    w.open_time_step(0.25)
    w.write_vertex_field("displacement", u, vector=True)
    w.write_cell_field("cauchy_stress", stress)
    path = w.close_time_step()
    assert path.endswith("q2_t025.vtu")
    pts, conn, offs, types, cell, point = OUT.read_vtu(path)
    assert np.array_equal(pts, mesh.coords)
    assert np.array_equal(conn.reshape(-1, 8), mesh.corner_nodes())
    assert np.all(types == OUT.VTK_HEXAHEDRON) and offs[-1] == 8 * mesh.num_cells
    assert np.array_equal(point["displacement"], u)
    assert np.array_equal(np.concatenate([cell[f"cauchy_stress.{c}"] for c in range(6)], axis=1), stress)
    assert np.all(cell["Rank"] == 0)


def test_write_vtu_rejects_bad_input(tmp_path):
    pts = np.zeros((4, 3))
    with pytest.raises(ValueError):
        OUT.write_vtu(str(tmp_path / "x.vtu"), pts, np.array([[0, 1, 2, 4]]), OUT.VTK_TETRA)
    with pytest.raises(ValueError):
        OUT.write_vtu(str(tmp_path / "x.vtu"), pts, np.array([[0, 1, 2, 3]]), OUT.VTK_TETRA,
                      point_data=[("f", np.zeros(3))])
