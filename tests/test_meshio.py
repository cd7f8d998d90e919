"""Mesh ingest (pylith_b200.meshio): Gmsh 4.1 ASCII/binary round trips, and the reference's own
test meshes solved with the oracle against the reference tests' known answers:
  * UniformStrain3D MMS on tests/mmstests/linearelasticity/nofaults-3d/data/{tet,hex}.msh;
  * axial displacement on tests/fullscale/linearelasticity/nofaults-3d/mesh_{tet,hex}.exo with the
    Dirichlet groups and components of axialdisp.cfg.
The meshes come from tests/golden/reference_meshes.npz (written by make_mesh_golden.py with this
reader); where PYLITH_SRC names the PyLith source tree, reading the files again must reproduce
the fixture."""
import os

import numpy as np
import pytest
import scipy.sparse.linalg as spla

import known_answers as KA
from golden import make_mesh_golden as MG
from pylith_b200 import materials as MAT
from pylith_b200 import meshing as M
from pylith_b200 import meshio as MIO

F1_ILE = "IsotropicLinearElasticity3D::f1v_infinitesimalStrain"
JF3_ILE = "IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain"


@pytest.fixture(scope="module")
def ref_meshes():
    return MG.load()


@pytest.mark.parametrize("binary", [False, True], ids=["ascii", "binary"])
@pytest.mark.parametrize("make", [lambda: M.box_tet_kuhn(3, 4, 2), lambda: M.box_hex(3, 2, 2)], ids=["tet", "hex"])
def test_gmsh_round_trip(tmp_path, make, binary):
    mesh = make()
    rng = np.random.default_rng(0)
    data = MIO.MeshData(mesh, rng.integers(1, 4, mesh.num_cells).astype(np.int32),
                        {"boundary_xneg": np.flatnonzero(M.boundary_mask(mesh, 0, "neg")),
                         "points": np.array([0, 3, 7])})
    path = str(tmp_path / "m.msh")
    MIO.write_gmsh(path, data, binary=binary)
    back = MIO.read(path)
    # nodes and cells come back grouped by material
    assert back.mesh.cell_type == mesh.cell_type
    assert back.mesh.num_cells == mesh.num_cells and back.mesh.num_nodes == mesh.num_nodes
    key = lambda X: np.lexsort(X.T)  # noqa: E731
    np.testing.assert_array_equal(back.mesh.coords[key(back.mesh.coords)], mesh.coords[key(mesh.coords)])
    assert sorted(back.material_ids.tolist()) == sorted(data.material_ids.tolist())
    cent = lambda m: np.sort(m.coords[m.cells].mean(axis=1).round(6), axis=0)  # noqa: E731
    np.testing.assert_array_equal(cent(back.mesh), cent(mesh))
    for name, nodes in data.vertex_groups.items():
        got = back.mesh.coords[back.vertex_groups[name]]
        np.testing.assert_array_equal(got[key(got)], mesh.coords[nodes][key(mesh.coords[nodes])])


def test_orientation_is_fixed(tmp_path):
    mesh = M.box_tet_kuhn(2, 2, 2)
    flipped = M.Mesh(mesh.cell_type, mesh.coords, mesh.cells[:, [0, 2, 1, 3]].copy())
    path = str(tmp_path / "f.msh")
    MIO.write_gmsh(path, MIO.MeshData(flipped, np.ones(mesh.num_cells, np.int32), {}))
    back = MIO.read(path).mesh
    X = back.coords[back.cells]
    det = np.einsum("ij,ij->i", np.cross(X[:, 1] - X[:, 0], X[:, 2] - X[:, 0]), X[:, 3] - X[:, 0])
    assert (det > 0).all()


def test_rejects_unknown_format(tmp_path):
    p = tmp_path / "m.vtk"
    p.write_text("x")
    with pytest.raises(MIO.MeshIOError):
        MIO.read(str(p))


def test_reading_the_reference_files_reproduces_the_fixture():
    src = os.environ.get("PYLITH_SRC")
    if not src or not os.path.isdir(src):
        pytest.skip("PYLITH_SRC (the PyLith source tree) is not set")
    fresh = MG.read_all(src)
    fixture = MG.load()
    assert sorted(fresh) == sorted(fixture)
    for key, d in fresh.items():
        f = fixture[key]
        assert d.mesh.cell_type == f.mesh.cell_type
        np.testing.assert_array_equal(d.mesh.coords, f.mesh.coords)
        np.testing.assert_array_equal(d.mesh.cells, f.mesh.cells)
        np.testing.assert_array_equal(d.material_ids, f.material_ids)
        assert sorted(d.vertex_groups) == sorted(f.vertex_groups)
        for g in d.vertex_groups:
            np.testing.assert_array_equal(d.vertex_groups[g], f.vertex_groups[g])


@pytest.mark.parametrize("key,ctype,ncells", [("mms_tet", M.CELL_TET4, 307), ("mms_hex", M.CELL_HEX8, 125)])
def test_reference_gmsh_meshes_mms_uniform_strain(oracle_lib, ref_meshes, key, ctype, ncells):
    """The reference's MMS meshes: 8 km box, material 24, vertex group `boundary`; a linear
    displacement field gives zero residual at every vertex outside `boundary`
    (UniformStrain3D.cc)."""
    O = oracle_lib
    d = ref_meshes[key]
    m = d.mesh
    assert m.cell_type == ctype and m.num_cells == ncells
    np.testing.assert_allclose(m.coords.min(0), [-4000, -4000, -8000])
    np.testing.assert_allclose(m.coords.max(0), [4000, 4000, 0])
    assert set(d.material_ids.tolist()) == {24}
    rho, mu, K = MAT.uniform_elastic(m.num_cells)
    aux = O.AuxFields([(rho[:, None], "cell"), (mu[:, None], "cell"), (K[:, None], "cell")])
    X = m.coords
    u = np.stack([1e-4 * X[:, 0] + 2e-5 * X[:, 1] - 3e-5 * X[:, 2], 3e-5 * X[:, 0] - 1e-4 * X[:, 1] + 4e-5 * X[:, 2],
                  -2e-5 * X[:, 0] + 1e-5 * X[:, 1] + 5e-5 * X[:, 2]], axis=1).ravel()
    r = O.residual(m, u, aux, f1=F1_ILE, source="ref" if O.ref_available() else "oracle").reshape(-1, 3)
    interior = np.ones(m.num_nodes, dtype=bool)
    interior[d.vertex_groups["boundary"]] = False
    assert interior.sum() > 0
    assert np.abs(r[interior]).max() <= 1e-12 * np.abs(r).max()


@pytest.mark.parametrize("key", ["axial_tet", "axial_hex"])
def test_reference_exodus_meshes_axial_displacement(oracle_lib, ref_meshes, key):
    """axialdisp.cfg on the reference's ExodusII meshes: ux on boundary_x*, uy on boundary_y*,
    uz on boundary_zneg from the analytic solution; the oracle's solve reproduces it."""
    O = oracle_lib
    d = ref_meshes[key]
    m = d.mesh
    assert set(d.material_ids.tolist()) == {1, 2}
    cons = MIO.constrained_mask(d, [("boundary_xneg", [0]), ("boundary_xpos", [0]), ("boundary_yneg", [1]),
                                    ("boundary_ypos", [1]), ("boundary_zneg", [2])])
    rho, mu, K = MAT.uniform_elastic(m.num_cells, KA.AXIAL_DENSITY, KA.AXIAL_VS, KA.AXIAL_VP)
    aux = O.AuxFields([(rho[:, None], "cell"), (mu[:, None], "cell"), (K[:, None], "cell")])
    uex = KA.axial_displacement(m.coords).ravel()
    J = O.assemble(m, O.jacobian_elements(m, aux, g3=JF3_ILE))
    u = np.where(cons, uex, 0.0)
    r = O.residual(m, u, aux, f1=F1_ILE)
    free = ~cons
    u[free] += spla.spsolve(J[free][:, free].tocsc(), -r[free])
    assert np.abs(u - uex).max() <= 1e-10 * np.abs(uex).max()
