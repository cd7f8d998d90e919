"""The host side of the geometric multigrid (pylith_b200/multigrid.py): level sizes, and the
prolongation between levels -- trilinear, exact for fields that are linear on each side of the
fault (with any jump across it), rows summing to one -- and the cell averaging of materials."""
import numpy as np
import scipy.sparse as sp

from pylith_b200 import materials as MAT
from pylith_b200 import multigrid as MG


def _side_linear(mesh):
    X = mesh.coords
    f = 2.0 * X[:, 0] - 3.0 * X[:, 1] + 0.5 * X[:, 2]
    plus = np.zeros(mesh.num_nodes, dtype=bool)
    plus[np.unique(mesh.cells[mesh.coords[mesh.cells].mean(axis=1)[:, 0] > 0])] = True
    return f + np.where(plus, 1000.0, 0.0)


def test_levels_and_prolongation_with_a_fault():
    levels = MG.build_hierarchy(16, 8, 12, fault_x=0.0, constrained_faces=[(0, "neg", (0,)), (2, "neg", (2,))],
                                max_coarse_nodes=0)
    assert [lv.n for lv in levels] == [(16, 8, 12), (8, 4, 6), (4, 2, 3)]
    for (row, col, val), lf, lc in zip(MG.prolongations(levels, 0.0), levels[:-1], levels[1:]):
        P = sp.csr_matrix((val, col, row), shape=(lf.mesh.num_nodes, lc.mesh.num_nodes))
        np.testing.assert_allclose(np.asarray(P.sum(axis=1)).ravel(), 1.0)
        np.testing.assert_allclose(P @ _side_linear(lc.mesh), _side_linear(lf.mesh), rtol=0, atol=1e-9)
        # constrained faces line up: a coarse constrained DOF's node coincides with a constrained fine one
        cf = lf.constrained[: 3 * lf.mesh.num_nodes].reshape(-1, 3)
        cc = lc.constrained[: 3 * lc.mesh.num_nodes].reshape(-1, 3)
        assert cc.sum() > 0 and cf.sum() > cc.sum()


def test_prolongation_without_a_fault_reproduces_linear_fields():
    levels = MG.build_hierarchy(8, 8, 8)
    for (row, col, val), lf, lc in zip(MG.prolongations(levels, None), levels[:-1], levels[1:]):
        P = sp.csr_matrix((val, col, row), shape=(lf.mesh.num_nodes, lc.mesh.num_nodes))
        lin = lambda m: m.coords @ np.array([1.0, -2.0, 0.25])  # noqa: E731
        np.testing.assert_allclose(P @ lin(lc.mesh), lin(lf.mesh), rtol=1e-12, atol=1e-9)


def test_materials_are_averaged_over_child_cells():
    levels = MG.build_hierarchy(4, 4, 4)
    nc0 = levels[0].mesh.num_cells
    rho, mu, K = MAT.lognormal_elastic(nc0, seed=1)
    coarse = MG.coarsen_material(MAT.IsotropicLinearElasticity(rho, mu, K), levels[1].cell_map)
    assert coarse.shear_modulus.shape == (levels[1].mesh.num_cells,)
    np.testing.assert_allclose(coarse.shear_modulus.sum() * 8, mu.sum())
    # nested levels: every coarse cell holds exactly 8 fine cells
    assert levels[1].cell_map.shape == (nc0,)
    assert np.array_equal(np.bincount(levels[1].cell_map), np.full(levels[1].mesh.num_cells, 8))


def test_non_nested_levels_keep_the_fault_plane():
    """Counts that are not powers of two (and halves that would move the fault plane off the grid)
    coarsen to the nearest count that keeps the plane a grid plane; the interpolation between such
    non-nested grids is still exact for fields linear on each side of the fault."""
    levels = MG.build_hierarchy(30, 14, 9, fault_x=0.0, constrained_faces=[(0, "neg", (0, 1, 2))])
    ns = [lv.n for lv in levels]
    assert ns[0] == (30, 14, 9) and len(ns) >= 3
    for (nx, ny, nz), (mx, my, mz) in zip(ns[:-1], ns[1:]):
        assert mx % 2 == 0 and abs(2 * mx - nx) <= 4 and my == (ny + 1) // 2 and mz == (nz + 1) // 2
    for (row, col, val), lf, lc in zip(MG.prolongations(levels, 0.0), levels[:-1], levels[1:]):
        P = sp.csr_matrix((val, col, row), shape=(lf.mesh.num_nodes, lc.mesh.num_nodes))
        np.testing.assert_allclose(np.asarray(P.sum(axis=1)).ravel(), 1.0)
        assert val.min() > 0.0
        np.testing.assert_allclose(P @ _side_linear(lc.mesh), _side_linear(lf.mesh), rtol=0, atol=1e-8)
    # every coarse cell holds at least one finer cell, and a cell-wise constant averages to itself
    for lf, lc in zip(levels[:-1], levels[1:]):
        cnt = np.bincount(lc.cell_map, minlength=lc.mesh.num_cells)
        assert cnt.min() >= 1
        np.testing.assert_allclose(MG.coarsen_cells(np.full(lf.mesh.num_cells, 3.5), lc.cell_map), 3.5)
        # cells stay on their side of the fault
        xf = lf.mesh.coords[lf.mesh.cells].mean(axis=1)[:, 0]
        xc = lc.mesh.coords[lc.mesh.cells].mean(axis=1)[:, 0]
        assert np.all(np.sign(xf) == np.sign(xc[lc.cell_map]))


def test_tetrahedral_levels_interpolate_fields_linear_on_each_side():
    """Unstructured P1 levels (independent Delaunay meshes of the same box and fault plane): the
    interpolation at the fine nodes reproduces fields linear on each side of the fault with any
    jump across it, uses non-negative weights summing to one, keeps box-face and fault-plane nodes
    on their face's coarse nodes, and the cell averaging preserves constants."""
    from pylith_b200 import meshing as M

    lo, hi = (-6000.0, -6000.0, -9000.0), (6000.0, 6000.0, 0.0)
    fine = M.box_tet_delaunay_fault_x(40000, seed=0, lo=lo, hi=hi)
    levels = MG.build_tet_hierarchy(fine, lambda n, l: M.box_tet_delaunay_fault_x(n, seed=l, lo=lo, hi=hi),
                                    fault_x=0.0, lo=lo, hi=hi, constrained_faces=[(0, "neg", (0, 1, 2))],
                                    min_cells=100)
    assert len(levels) >= 3
    for (row, col, val), lf, lc in zip(MG.prolongations(levels, 0.0), levels[:-1], levels[1:]):
        P = sp.csr_matrix((val, col, row), shape=(lf.mesh.num_nodes, lc.mesh.num_nodes))
        np.testing.assert_allclose(np.asarray(P.sum(axis=1)).ravel(), 1.0, rtol=1e-12)
        assert val.min() > 0.0
        X = lf.mesh.coords
        f = lambda m: (m.coords @ np.array([2.0, -3.0, 0.5])  # noqa: E731
                       + np.where(MG.node_sides(m, 0.0) > 0, 1000.0, 0.0))
        np.testing.assert_allclose(P @ f(lc.mesh), f(lf.mesh), rtol=0, atol=1e-7)
        # nodes on the face x = lo take weights from coarse nodes on that face only
        face_f = np.isclose(X[:, 0], lo[0])
        face_c = np.isclose(lc.mesh.coords[:, 0], lo[0])
        rows = np.repeat(np.arange(lf.mesh.num_nodes), np.diff(row))
        assert face_c[col[face_f[rows]]].all()
        # fault-plane copies interpolate from coarse copies of their own side
        sf, sc = MG.node_sides(lf.mesh, 0.0), MG.node_sides(lc.mesh, 0.0)
        assert np.array_equal(sf[rows], sc[col])
        W = lc.cell_map
        assert W.shape == (lc.mesh.num_cells, lf.mesh.num_cells)
        np.testing.assert_allclose(MG.coarsen_cells(np.full(lf.mesh.num_cells, 2.5), W), 2.5)
