"""HDF5 output (pylith_b200/output.py DataWriterHDF5 over pylith_b200/hdf5.py) against the
reference's golden files, dataset by dataset, as the reference's own writer tests compare them
(tests/libtests/meshio/TestDataWriterHDF5.cc: geometry, viz topology and cell_dim, time, every
vertex and cell field with its vector_field_type).

tests/golden/h5_golden.npz holds the datasets and attributes of the reference's
tests/libtests/meshio/data/{tet4,hex8}_{vertex,cell}.h5, read with pylith_b200.hdf5 after that
reader was pinned on the reference's files (tests/golden/make_h5_golden.py). Where PYLITH_SRC
names the PyLith source tree, the pins run again on the files themselves."""
import json
import os

import numpy as np
import pytest

from pylith_b200 import hdf5 as H5
from pylith_b200 import meshing as M
from pylith_b200 import output as OUT

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "h5_golden.npz")


def _golden(name):
    d = np.load(GOLDEN)
    meta = json.loads(str(d["meta"]))[name]
    return {p: (d[v["key"]], v["attrs"]) for p, v in meta["datasets"].items()}, meta["groups"]


def _attrs(f, p):
    return {k: (v if isinstance(v, str) else np.asarray(v).tolist()) for k, v in f.attrs(p).items()}


@pytest.mark.parametrize("name", ["tet4_vertex.h5", "tet4_cell.h5", "hex8_vertex.h5", "hex8_cell.h5"])
def test_writer_reproduces_the_reference_datasets(tmp_path, name):
    ds, groups = _golden(name)
    kind, where = name[:-3].split("_")
    verts, cells = ds["/geometry/vertices"][0], ds["/viz/topology/cells"][0]
    cohesive = None
    if kind == "hex8":  # cohesive hexahedral prisms: negative then positive face (4 + 4)
        prisms = ds["/viz/topology_1/cells"][0]
        cohesive = np.concatenate([prisms, np.zeros((len(prisms), 4), dtype=np.int32)], axis=1)
    else:  # triangular cohesive prisms are not a cell of this package's meshes
        ds.pop("/viz/topology_1/cells")
        groups.remove("/viz/topology_1")
    mesh = M.Mesh(M.CELL_TET4 if kind == "tet4" else M.CELL_HEX8, verts, cells.astype(np.int32), cohesive)
    w = OUT.DataWriterHDF5(filename=str(tmp_path / name))
    w.open(mesh)
    group = f"/{where}_fields"
    for p, (v, a) in ds.items():
        if p.startswith(group + "/") and "timestepping" in a:
            add = w.write_vertex_field if where == "vertex" else w.write_cell_field
            add(1.0, p.rsplit("/", 1)[1], v[0], vector_field_type=a["vector_field_type"])
    w.close()
    f = H5.H5File(str(tmp_path / name))
    paths = f.walk()
    assert sorted(p for p in paths if f.is_group(p)) == sorted(groups)
    assert sorted(p for p in paths if not f.is_group(p)) == sorted(ds)
    for p, (v, a) in ds.items():
        got = f.dataset(p)
        assert got.dtype == v.dtype and got.shape == v.shape, p
        assert np.array_equal(got, v), p
        assert _attrs(f, p) == a, p


@pytest.mark.parametrize("name", ["tet4_points_vertex.h5", "hex8_points_vertex.h5"])
def test_station_output_reproduces_the_reference_datasets(tmp_path, name):
    """Station output (TestDataWriterHDF5Points): a point mesh, its names in /stations, fields per
    point; the layout and values must be the golden file's."""
    ds, groups = _golden(name)
    pts = ds["/geometry/vertices"][0]
    names = [n.decode() for n in ds["/stations"][0]]
    w = OUT.DataWriterHDF5(filename=str(tmp_path / name))
    w.open(OUT.PointMesh(pts))
    w.write_point_names(names)
    for p, (v, a) in ds.items():
        if p.startswith("/vertex_fields/") and "timestepping" in a:
            w.write_vertex_field(1.0, p.rsplit("/", 1)[1], v[0], vector_field_type=a["vector_field_type"])
    w.close()
    f = H5.H5File(str(tmp_path / name))
    paths = f.walk()
    assert sorted(p for p in paths if f.is_group(p)) == sorted(groups)
    assert sorted(p for p in paths if not f.is_group(p)) == sorted(ds)
    for p, (v, a) in ds.items():
        got = f.dataset(p)
        assert got.dtype == v.dtype and got.shape == v.shape, p
        assert np.array_equal(got, v), p
        assert _attrs(f, p) == a, p
    assert '<Topology TopologyType="Polyvertex" NumberOfElements="4">' in open(tmp_path / name.replace(".h5", ".xmf")).read()


def test_points_list_reader(tmp_path):
    p = tmp_path / "points.txt"
    p.write_text("# Points for solution output\nZZ.1 -2200.0 +2100.0  -1000.0\n\nZZ.2  +100.0   +50.0  -1020.0\n")
    names, xyz = OUT.read_points_list(str(p))
    assert names == ["ZZ.1", "ZZ.2"]
    assert np.array_equal(xyz, [[-2200.0, 2100.0, -1000.0], [100.0, 50.0, -1020.0]])


def test_steps_times_and_growth(tmp_path):
    """The reference's step rule (DataWriterHDF5.cc:168-178): the k-th write of a field is its step
    k and the first field written at a new step adds that step's time (times the time scale). The
    file is complete after every call, including past 64 steps (a deeper chunk index)."""
    mesh = M.box_hex(2, 2, 1)
    path = str(tmp_path / "out.h5")
    w = OUT.DataWriterHDF5(filename=path, time_scale=2.0)
    w.open(mesh)
    rng = np.random.default_rng(3)
    disp, vel, stress = [], [], []
    for k in range(150):
        t = 0.5 * k
        disp.append(rng.standard_normal((mesh.num_nodes, 3)))
        w.write_vertex_field(t, "displacement", disp[-1])
        if k % 2 == 0:
            vel.append(rng.standard_normal(mesh.num_nodes))
            w.write_vertex_field(t, "velocity", vel[-1])
        stress.append(rng.standard_normal((mesh.num_cells, 6)))
        w.write_cell_field(t, "cauchy_stress", stress[-1])
        if k in (0, 1, 63, 64, 65, 149):
            f = H5.H5File(path)
            assert f.dataset("/time").shape == (k + 1, 1, 1)
            assert np.array_equal(f.dataset("/time")[:, 0, 0], 2.0 * 0.5 * np.arange(k + 1))
            assert np.array_equal(f.dataset("/vertex_fields/displacement"), np.array(disp))
            assert np.array_equal(f.dataset("/vertex_fields/velocity")[:, :, 0], np.array(vel))
            assert np.array_equal(f.dataset("/cell_fields/cauchy_stress"), np.array(stress))
    w.close()
    f = H5.H5File(path)
    assert f.attrs("/vertex_fields/displacement") == {"timestepping": 1, "vector_field_type": "vector"}
    assert f.attrs("/vertex_fields/velocity")["vector_field_type"] == "scalar"
    assert f.attrs("/cell_fields/cauchy_stress")["vector_field_type"] == "tensor"
    assert np.array_equal(f.dataset("/geometry/vertices"), mesh.coords)
    assert np.array_equal(f.dataset("/viz/topology/cells"), mesh.cells)


def test_info_file_names_and_stations(tmp_path):
    w = OUT.DataWriterHDF5(filename=str(tmp_path / "mat.h5"), is_info=True, length_scale=1e3)
    assert w.hdf5_filename() == str(tmp_path / "mat_info.h5")
    mesh = M.insert_fault_x(M.box_hex(2, 1, 1))
    w.open(mesh)
    w.write_point_names(["ZZ.A", "ZZ.B", "ZZ.C", "ZZ.DD"])  # as in tet4_points_vertex.h5
    w.write_cell_field(0.0, "density", np.full(mesh.num_cells, 2500.0))
    w.close()
    f = H5.H5File(w.hdf5_filename())
    st = f.dataset("/stations")
    assert st.dtype == np.dtype("S6") and list(st) == [b"ZZ.A", b"ZZ.B", b"ZZ.C", b"ZZ.DD"]
    assert np.array_equal(f.dataset("/geometry/vertices"), mesh.coords * 1e3)
    assert np.array_equal(f.dataset("/viz/topology_1/cells"), mesh.cohesive[:, :8])
    assert f.attrs("/viz/topology_1/cells") == {"cell_corners": 8, "cell_dim": 3}
    w2 = OUT.DataWriterHDF5(filename=str(tmp_path / "y.h5"))
    with pytest.raises(RuntimeError):
        w2.write_vertex_field(0.0, "u", np.zeros((mesh.num_nodes, 3)))  # not open
    w2.open(mesh)
    with pytest.raises(ValueError):
        w2.write_vertex_field(0.0, "u", np.zeros((mesh.num_nodes, 3)), vector_field_type="vectors")
    with pytest.raises(ValueError):
        w2.write_vertex_field(0.0, "u", np.zeros((mesh.num_nodes + 1, 3)))
    w2.close()


def test_reader_rejects_other_files(tmp_path):
    p = tmp_path / "not.h5"
    p.write_bytes(b"not an hdf5 file" * 10)
    with pytest.raises(H5.H5FormatError):
        H5.H5File(str(p))


def test_reader_pins_on_the_reference_files():
    src = os.environ.get("PYLITH_SRC")
    if not src or not os.path.isdir(os.path.join(src, "tests", "libtests", "meshio", "data")):
        pytest.skip("PYLITH_SRC (the PyLith source tree) is not set")
    import importlib.util

    spec = importlib.util.spec_from_file_location(
        "make_h5_golden", os.path.join(os.path.dirname(__file__), "golden", "make_h5_golden.py"))
    G = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(G)
    data_dir = os.path.join(src, "tests", "libtests", "meshio", "data")
    for case in G.MESH_CASES:
        for where in ("vertex", "cell"):
            G.pin(data_dir, H5.H5File(os.path.join(data_dir, f"{case}_{where}.h5")), case, where)
    d = np.load(GOLDEN)
    meta = json.loads(str(d["meta"]))
    import hashlib

    for name in G.KEEP:
        raw = open(os.path.join(data_dir, name), "rb").read()
        assert hashlib.sha256(raw).hexdigest() == meta[name]["sha256"]
        f = H5.H5File(raw)
        for p, v in meta[name]["datasets"].items():
            assert np.array_equal(f.dataset(p), d[v["key"]])


XDMF_GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "xdmf_golden.json")


def _xdmf_cases():
    with open(XDMF_GOLDEN) as fh:
        return json.load(fh)


@pytest.mark.parametrize("name", sorted(_xdmf_cases()))
def test_xdmf_is_byte_identical_to_the_reference(tmp_path, name):
    """write_xdmf against the reference's golden .xmf files (tests/pytests/meshio/data, compared
    line for line by its TestXdmf.py). The HDF5 file is rebuilt from the golden metadata (dataset
    shapes and types, cell_dim, vector_field_type, time stamps; values are irrelevant to Xdmf)."""
    import hashlib

    case = _xdmf_cases()[name]
    path = str(tmp_path / name)
    with H5.H5Writer(path) as w:
        for p, d in case["datasets"].items():
            data = np.asarray(d["values"]).reshape(d["shape"]) if "values" in d else np.zeros(d["shape"], d["dtype"])
            w.create_dataset(p, data.astype(d["dtype"]), attrs={k: (np.int32(v) if k == "cell_dim" else v)
                                                                for k, v in d["attrs"].items()})
    out = OUT.write_xdmf(path)
    assert out == path.replace(".h5", ".xmf")
    assert hashlib.sha256(open(out, "rb").read()).hexdigest() == case["xmf_sha256"]


def test_data_writer_hdf5_writes_its_xdmf(tmp_path):
    mesh = M.box_hex(2, 1, 1)
    w = OUT.DataWriterHDF5(filename=str(tmp_path / "soln.h5"))
    w.open(mesh)
    for t in (0.0, 1.0):
        w.write_vertex_field(t, "displacement", np.zeros((mesh.num_nodes, 3)))
        w.write_cell_field(t, "cauchy_stress", np.zeros((mesh.num_cells, 6)))
    w.close()
    text = open(tmp_path / "soln.xmf").read()
    assert '<!ENTITY HeavyData "soln.h5">' in text
    assert text.count('<Grid Name="domain" GridType="Uniform">') == 2
    assert '<Attribute Name="cauchy_stress_xz" Type="Scalar" Center="Cell">' in text
    assert '<Topology TopologyType="Hexahedron" NumberOfElements="2">' in text


@pytest.mark.parametrize("name", ["tet4_vertex.h5", "hex8_cell.h5"])
def test_external_writer_reproduces_the_reference_datasets(tmp_path, name):
    """DataWriterHDF5Ext: the reference's HDF5Ext tests compare against the same golden files as
    the HDF5 ones (TestDataWriterHDF5ExtMesh_Cases.cc), reading fields through the external raw
    files; values, shapes and vector_field_type must match."""
    ds, _ = _golden(name)
    kind, where = name[:-3].split("_")
    cohesive = None
    if kind == "hex8":
        prisms = ds["/viz/topology_1/cells"][0]
        cohesive = np.concatenate([prisms, np.zeros((len(prisms), 4), dtype=np.int32)], axis=1)
    mesh = M.Mesh(M.CELL_TET4 if kind == "tet4" else M.CELL_HEX8, ds["/geometry/vertices"][0],
                  ds["/viz/topology/cells"][0].astype(np.int32), cohesive)
    w = OUT.DataWriterHDF5Ext(filename=str(tmp_path / name))
    w.open(mesh)
    group = f"/{where}_fields"
    fields = {p: (v, a) for p, (v, a) in ds.items() if p.startswith(group + "/") and "timestepping" in a}
    for p, (v, a) in fields.items():
        add = w.write_vertex_field if where == "vertex" else w.write_cell_field
        add(1.0, p.rsplit("/", 1)[1], v[0], vector_field_type=a["vector_field_type"])
    w.close()
    f = H5.H5File(str(tmp_path / name))
    assert np.array_equal(f.dataset("/time"), ds["/time"][0])
    assert np.array_equal(f.dataset("/geometry/vertices"), ds["/geometry/vertices"][0])
    for p, (v, a) in fields.items():
        assert np.array_equal(f.dataset(p), v), p
        assert f.attrs(p) == {"vector_field_type": a["vector_field_type"]}
        raw = np.fromfile(w.dataset_filename(p.rsplit("/", 1)[1]), dtype=">f8")
        assert np.array_equal(raw, v.ravel())


def test_external_writer_steps(tmp_path):
    mesh = M.box_hex(2, 1, 1)
    w = OUT.DataWriterHDF5Ext(filename=str(tmp_path / "soln.h5"), time_scale=10.0)
    w.open(mesh)
    disp = [np.random.default_rng(k).standard_normal((mesh.num_nodes, 3)) for k in range(5)]
    for k, d in enumerate(disp):
        w.write_vertex_field(float(k), "displacement", d)
        f = H5.H5File(str(tmp_path / "soln.h5"))
        assert np.array_equal(f.dataset("/vertex_fields/displacement"), np.array(disp[:k + 1]))
        assert np.array_equal(f.dataset("/time")[:, 0, 0], 10.0 * np.arange(k + 1))
    w.close()
    assert not (tmp_path / "soln.xmf").exists()
    assert (tmp_path / "soln_displacement.dat").stat().st_size == 5 * mesh.num_nodes * 3 * 8
