"""Output of a device time-stepping run: problems.OutputObserver (the reference's OutputSolnDomain
and OutputPhysics with OutputTriggerStep) writing the solution and the derived fields of two
materials on cell subsets through DataWriterHDF5 and DataWriterVTK; every written value must equal
the device state of its step."""
import numpy as np
import pytest

from pylith_b200 import materials as MAT
from pylith_b200 import meshing as M

pytestmark = pytest.mark.gpu

LO, HI = (-4000.0, -4000.0, -8000.0), (4000.0, 4000.0, 0.0)
E0 = 1e-4
DT = 1e8 * 3.15e7  # the Maxwell times below are 1e18-1e20 s: visible relaxation per step


@pytest.fixture(scope="module")
def ctx():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pylith_b200 import feassemble as FA

    return FA.Context(0)


def _problem(ctx, observers):
    from pylith_b200 import problems as P

    mesh = M.box_tet_delaunay(4000, seed=3, lo=LO, hi=HI)
    cx = mesh.coords[mesh.cells].mean(axis=1)[:, 0]
    left, right = np.flatnonzero(cx < 0), np.flatnonzero(cx >= 0)
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=5)
    elastic = MAT.IsotropicLinearElasticity(rho[left], mu[left], K[left])
    nr, nq = len(right), M.QUAD_POINTS[mesh.cell_type]
    tau = MAT.genmaxwell_times(rho[right], np.sqrt(mu[right] / rho[right]), [1e18, 1e19, 1e20], [0.3, 0.3, 0.3])
    maxwell = MAT.IsotropicLinearGenMaxwell(rho[right], mu[right], K[right], tau, np.tile([0.3, 0.3, 0.3], (nr, 1)),
                                            np.zeros((nr, nq, 18)), np.zeros((nr, nq, 6)))
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    for ax in range(3):
        for sd in ("neg", "pos"):
            cons[M.boundary_mask(mesh, ax, sd, LO, HI)] = True
    X = mesh.coords
    bc = np.stack([0 * X[:, 0], 0 * X[:, 1], E0 * (X[:, 2] - LO[2])], axis=1).ravel()
    prob = P.QuasistaticProblem(ctx, mesh, [(elastic, left), (maxwell, right)], cons.ravel(), bc, dt=DT,
                                rtol=1e-12, observers=observers)
    return prob


def _expected(prob, t):
    """Displacement and the full-mesh cauchy_stress / cauchy_strain of the problem's state."""
    import torch

    nn = prob.mesh.num_nodes
    disp = prob.u[:3 * nn].reshape(nn, 3).cpu().numpy()
    out = {"cauchy_stress": np.zeros((prob.mesh.num_cells, 6)), "cauchy_strain": np.zeros((prob.mesh.num_cells, 6))}
    for ig, ids in zip(prob.domain, prob.domain_cells):
        vals = torch.empty((len(ids), 12), dtype=torch.float64, device="cuda")
        ig.compute_derived_field(t, prob.dt, prob.u, vals)
        v = vals.cpu().numpy()
        out["cauchy_stress"][ids] = v[:, :6]
        out["cauchy_strain"][ids] = v[:, 6:]
    return disp, out


def test_observer_writes_every_other_step_to_hdf5(ctx, tmp_path):
    from pylith_b200 import hdf5 as H5
    from pylith_b200 import output as OUT
    from pylith_b200 import problems as P

    w = OUT.DataWriterHDF5(filename=str(tmp_path / "domain.h5"))
    prob = _problem(ctx, [P.OutputObserver(w, num_steps_skip=1)])
    written = []
    for k in range(5):
        t = (k + 1) * DT
        prob.step(t)
        if k % 2 == 0:  # OutputTriggerStep with numStepsSkip = 1: steps 0, 2, 4
            written.append((t,) + _expected(prob, t))
    prob.close()
    f = H5.H5File(str(tmp_path / "domain.h5"))
    assert np.array_equal(f.dataset("/time")[:, 0, 0], [entry[0] for entry in written])
    disp = f.dataset("/vertex_fields/displacement")
    assert disp.shape == (3, prob.mesh.num_nodes, 3)
    for s, (t, d, cell) in enumerate(written):
        assert np.array_equal(disp[s], d)
        for name, v in cell.items():
            assert np.array_equal(f.dataset(f"/cell_fields/{name}")[s], v), (s, name)
    assert f.attrs("/cell_fields/cauchy_stress")["vector_field_type"] == "tensor"
    # the stress relaxes on the Maxwell side between written steps
    stress = f.dataset("/cell_fields/cauchy_stress")
    right = prob.domain_cells[1]
    assert not np.allclose(stress[0][right], stress[2][right])
    assert (tmp_path / "domain.xmf").exists()


def test_observer_writes_vtk_files_per_step(ctx, tmp_path):
    from pylith_b200 import output as OUT
    from pylith_b200 import problems as P

    w = OUT.DataWriterVTK(filename="domain.vtu", time_format="%03.0f", time_constant=DT)
    prob = _problem(ctx, [P.OutputObserver(w, directory=str(tmp_path))])
    prob.step(DT)
    d, cell = _expected(prob, DT)
    prob.close()
    pts, conn, offs, types, cfields, pfields = OUT.read_vtu(str(tmp_path / "domain_t001.vtu"))
    assert np.array_equal(pfields["displacement"], d)
    assert np.array_equal(cfields["cauchy_stress.0"].ravel(), cell["cauchy_stress"][:, 0])


def test_station_observer_interpolates_the_device_solution(ctx, tmp_path):
    """OutputPointsObserver: the displacement at stations read from a points file, interpolated
    on the device (exact for the uniform strain the boundaries impose on a homogeneous box),
    written with the station names to a point-mesh HDF5 file."""
    from pylith_b200 import hdf5 as H5
    from pylith_b200 import output as OUT
    from pylith_b200 import problems as P

    pts_file = tmp_path / "points.txt"
    pts_file.write_text("# stations\nZZ.1 -2200.0 +2100.0 -1000.0\nZZ.2 +100.0 +50.0 -1020.0\n"
                        "ZZ.3 +1100.0 +3400.0 -3230.0\nZZ.44 0.0 0.0 -7999.0\n")
    names, pts = OUT.read_points_list(str(pts_file))
    mesh = M.box_tet_delaunay(3000, seed=4, lo=LO, hi=HI)
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=2, sigma_log=0.0, density_spread=0.0)
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    for ax in range(3):
        for sd in ("neg", "pos"):
            cons[M.boundary_mask(mesh, ax, sd, LO, HI)] = True
    X = mesh.coords
    bc = np.stack([0 * X[:, 0], 0 * X[:, 1], E0 * (X[:, 2] - LO[2])], axis=1).ravel()
    w = OUT.DataWriterHDF5(filename=str(tmp_path / "stations.h5"))
    obs = P.OutputPointsObserver(w, names, pts)
    prob = P.QuasistaticProblem(ctx, mesh, [(MAT.IsotropicLinearElasticity(rho, mu, K), None)], cons.ravel(), bc,
                                rtol=1e-13, observers=[obs])
    prob.step(1.0)
    prob.step(2.0)
    prob.close()
    f = H5.H5File(str(tmp_path / "stations.h5"))
    assert [s.decode() for s in f.dataset("/stations")] == names
    assert f.dataset("/stations").dtype == np.dtype("S6")
    d = f.dataset("/vertex_fields/displacement")
    assert d.shape == (2, 4, 3)
    want = np.stack([0 * pts[:, 0], 0 * pts[:, 1], E0 * (pts[:, 2] - LO[2])], axis=1)
    np.testing.assert_allclose(d[1], want, rtol=0, atol=1e-9 * E0 * (HI[2] - LO[2]))
    assert np.array_equal(f.dataset("/viz/topology/cells").ravel(), np.arange(4))
    assert f.attrs("/viz/topology/cells") == {"cell_corners": 1, "cell_dim": 0}
