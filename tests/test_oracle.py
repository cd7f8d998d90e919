"""Pins the oracle (CPU restatement) before the GPU tests compare against it.

1. Pointwise kernels: the restatement against golden vectors produced by the
   reference's own kernels (tests/golden/pointwise_golden.npz), and against
   the reference kernels themselves when oracle/_ref is built.
2. Cell loop: the reference's known answers (MMS uniform strain, axial
   displacement, generalized-Maxwell relaxation, rigid two-block slip).
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

import known_answers as KA
from pylith_b200 import materials as MAT
from pylith_b200 import meshing as M

F1_ILE = "IsotropicLinearElasticity3D::f1v_infinitesimalStrain"
JF3_ILE = "IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain"
GOLDEN = __import__("os").path.join(__import__("os").path.dirname(__file__), "golden",
                                    "pointwise_golden.npz")


def elastic_aux(O, rho, mu, K):
    return O.AuxFields([(rho[:, None], "cell"), (mu[:, None], "cell"), (K[:, None], "cell")])


@pytest.mark.parametrize("name", [
    "Elasticity::g0v_bodyforce",
    "IsotropicLinearElasticity3D::f1v_infinitesimalStrain",
    "IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain",
    "IsotropicLinearGenMaxwell3D::f1v_infinitesimalStrain",
    "IsotropicLinearGenMaxwell3D::Jf3vu_infinitesimalStrain",
    "IsotropicLinearGenMaxwell3D::viscousStrain_infinitesimalStrain_asVector",
    "Elasticity3D::infinitesimalStrain_asVector",
    "IsotropicLinearElasticity3D::cauchyStress_infinitesimalStrain_asVector",
    "IsotropicLinearGenMaxwell3D::cauchyStress_infinitesimalStrain_asVector",
    "FaultCohesiveKin::f0u_neg", "FaultCohesiveKin::f0u_pos", "FaultCohesiveKin::f0l_slip",
    "FaultCohesiveKin::Jf0ul_neg", "FaultCohesiveKin::Jf0ul_pos", "FaultCohesiveKin::Jf0lu",
])
def test_pointwise_restatement_matches_reference_golden(oracle_lib, name):
    O = oracle_lib
    g = np.load(GOLDEN)
    key = name.replace("::", "__")
    n = len(g[f"{key}.out"])
    for i in range(n):
        nc = int(g[f"{key}.numConstants"][i])
        out = O.call_point(name, g[f"{key}.s"][i], g[f"{key}.s_x"][i], g[f"{key}.a"][i],
                           g[f"{key}.aOff"][i], g[f"{key}.constants"][i][:nc] if nc else None,
                           "oracle", n=g[f"{key}.n"][i], numS=2 if "Fault" in name else 1)
        # bit-exact: same operations in the same order as the reference kernel
        np.testing.assert_array_equal(out, g[f"{key}.out"][i])
    if O.ref_available():
        for i in range(n):
            nc = int(g[f"{key}.numConstants"][i])
            out = O.call_point(name, g[f"{key}.s"][i], g[f"{key}.s_x"][i], g[f"{key}.a"][i],
                               g[f"{key}.aOff"][i], g[f"{key}.constants"][i][:nc] if nc else None,
                               "ref", n=g[f"{key}.n"][i], numS=2 if "Fault" in name else 1)
            np.testing.assert_array_equal(out, g[f"{key}.out"][i])


def test_tangential_directions_golden(oracle_lib):
    import ctypes

    O = oracle_lib
    g = np.load(GOLDEN)["tangential_directions"]
    P = ctypes.c_void_p
    for row in g:
        n, r1, r2, t1, t2 = row[0:3], row[3:6], row[6:9], row[9:12], row[12:15]
        o1 = np.zeros(3)
        o2 = np.zeros(3)
        O.lib().oracle_tangential_directions(o1.ctypes.data_as(P), o2.ctypes.data_as(P),
                                             np.ascontiguousarray(r1).ctypes.data_as(P),
                                             np.ascontiguousarray(r2).ctypes.data_as(P),
                                             np.ascontiguousarray(n).ctypes.data_as(P))
        np.testing.assert_array_equal(o1, t1)
        np.testing.assert_array_equal(o2, t2)


def _linear_field(X):
    return np.stack([1e-4 * X[:, 0] + 2e-5 * X[:, 1] - 3e-5 * X[:, 2],
                     3e-5 * X[:, 0] - 1e-4 * X[:, 1] + 4e-5 * X[:, 2],
                     -2e-5 * X[:, 0] + 1e-5 * X[:, 1] + 5e-5 * X[:, 2]], axis=1).ravel()


@pytest.mark.parametrize("make", [lambda: M.box_hex(4, 4, 3), lambda: M.box_tet_delaunay(3000, seed=3),
                                  lambda: M.box_hex27(3, 3, 2)], ids=["hex8", "tet4", "hex27"])
@pytest.mark.parametrize("source", ["oracle", "ref"])
def test_mms_uniform_strain_residual_vanishes(oracle_lib, make, source):
    """UniformStrain3D MMS (tests/mmstests/linearelasticity/nofaults-3d/UniformStrain3D.cc):
    a linear displacement field gives a zero residual at every interior node (tol 1e-8 in the
    reference's MMSTest.cc:40; here relative to the boundary residual scale)."""
    O = oracle_lib
    if source == "ref" and not O.ref_available():
        pytest.skip("reference kernels not built")
    mesh = make()
    rho, mu, K = MAT.uniform_elastic(mesh.num_cells)
    aux = elastic_aux(O, rho, mu, K)
    u = _linear_field(mesh.coords)
    r = O.residual(mesh, u, aux, f1=F1_ILE, source=source).reshape(-1, 3)
    bnd = np.zeros(mesh.num_nodes, dtype=bool)
    for ax in range(3):
        for sd in ("neg", "pos"):
            bnd |= M.boundary_mask(mesh, ax, sd)
    scale = np.abs(r).max()
    assert np.abs(r[~bnd]).max() <= 1e-13 * scale
    # The Jacobian is exactly linear: J u reproduces the residual (isJacobianLinear).
    J = O.assemble(mesh, O.jacobian_elements(mesh, aux, g3=JF3_ILE, source=source))
    np.testing.assert_allclose(J @ u, r.ravel(), rtol=0, atol=1e-12 * scale)


@pytest.mark.parametrize("make", [lambda: M.box_hex(6, 6, 4), lambda: M.box_tet_delaunay(4000, seed=1),
                                  lambda: M.box_hex27(3, 3, 2)], ids=["hex8", "tet4", "hex27"])
def test_axial_displacement_known_answer(oracle_lib, make):
    """Axial extension (tests/fullscale/linearelasticity/nofaults-3d/axialdisp_soln.py): the
    uniform-strain solution is reproduced exactly by the discretisation."""
    O = oracle_lib
    mesh = make()
    rho, mu, K = MAT.uniform_elastic(mesh.num_cells, KA.AXIAL_DENSITY, KA.AXIAL_VS, KA.AXIAL_VP)
    aux = elastic_aux(O, rho, mu, K)
    uex = KA.axial_displacement(mesh.coords).ravel()
    cons = KA.axial_constrained(mesh)
    J = O.assemble(mesh, O.jacobian_elements(mesh, aux, g3=JF3_ILE))
    u = np.where(cons, uex, 0.0)
    r = O.residual(mesh, u, aux, f1=F1_ILE)
    free = ~cons
    u[free] += spla.spsolve(J[free][:, free].tocsc(), -r[free])
    assert np.abs(u - uex).max() <= 1e-10 * np.abs(uex).max()


def test_genmaxwell_relaxation_known_answer(oracle_lib):
    """Generalized-Maxwell axial strain relaxation
    (tests/fullscale/viscoelasticity/nofaults-3d/axialstrain_genmaxwell_soln.py): with the
    initial viscous strain dev(e0) and constant strain e0 in z, the discrete update reproduces
    sigma(t_n) = K tr(e) + 2 mu dev(e) (r0 + sum r_i exp(-t_n/tau_i)) at every step."""
    O = oracle_lib
    mesh = M.box_hex(2, 2, 2, lo=(-4000.0, -4000.0, -8000.0), hi=(4000.0, 4000.0, 0.0))
    mu, K, lam, tau = KA.genmaxwell_params()
    nc = mesh.num_cells
    nq = 8
    e0 = KA.GM_E0
    visc = np.tile(np.array([-e0 / 3, -e0 / 3, 2 * e0 / 3, 0, 0, 0] * 3), (nc, nq, 1))
    total = np.tile(np.array([0, 0, e0, 0, 0, 0.0]), (nc, nq, 1))
    X = mesh.coords
    u = np.stack([0 * X[:, 0], 0 * X[:, 1], e0 * (X[:, 2] + 8000.0)], axis=1).ravel()
    vol = 8000.0 * 8000.0 * 8000.0
    for step in range(1, KA.GM_STEPS + 1):
        aux = O.AuxFields([(np.full((nc, 1), KA.GM_DENSITY), "cell"), (np.full((nc, 1), mu), "cell"),
                           (np.full((nc, 1), K), "cell"), (np.tile(tau, (nc, 1)), "cell"),
                           (np.tile(np.array(KA.GM_RATIO), (nc, 1)), "cell"), (visc, "qp"),
                           (total, "qp")])
        r = O.residual(mesh, u, aux, f1="IsotropicLinearGenMaxwell3D::f1v_infinitesimalStrain",
                       constants=[KA.GM_DT])
        sigma = KA.stress_from_residual(X, r, vol)
        expect = KA.genmaxwell_stress(step * KA.GM_DT)
        np.testing.assert_allclose(np.diag(sigma), expect, rtol=1e-10)
        visc, total = O.project_qp(
            mesh, u, aux, ["IsotropicLinearGenMaxwell3D::viscousStrain_infinitesimalStrain_asVector",
                           "Elasticity3D::infinitesimalStrain_asVector"], [18, 6], constants=[KA.GM_DT])


def test_rigid_two_block_slip_known_answer(oracle_lib):
    """Prescribed slip between two rigid blocks (tests/fullscale/linearelasticity/faults-3d/
    twoblocks.cfg: ll = -2 m, reverse = 1 m, ref_dir_1 = [0,0,1], ref_dir_2 = [0.5,0,0.5]) on a
    vertical fault at x = 0: each block translates by -/+ slip/2, lambda = 0, and the full
    saddle-point system solved with Dirichlet x faces reproduces that state."""
    import scipy.sparse as sp

    O = oracle_lib
    mesh = M.insert_fault_x(M.box_hex(4, 3, 3))
    rho, mu, K = MAT.uniform_elastic(mesh.num_cells)
    aux = elastic_aux(O, rho, mu, K)
    consts = [0.0, 0.0, 1.0, 0.5, 0.0, 0.5]
    slip = np.tile([0.0, -2.0, 1.0], (mesh.num_lagrange, 1))
    # n = +x, t1 = ref_dir_1 x n = +y, t2 = n x t1 = +z (no flip: 0.5*1 + 0*0 + 0*0 >= 0)
    d = np.array([0.0, -2.0, 1.0])
    plus = np.zeros(mesh.num_nodes, dtype=bool)
    plus[np.unique(mesh.cells[mesh.coords[mesh.cells].mean(axis=1)[:, 0] > 0])] = True
    uex = np.where(plus[:, None], 0.5 * d, -0.5 * d)
    uex_full = np.concatenate([uex.ravel(), np.zeros(3 * mesh.num_lagrange)])
    r = np.zeros(mesh.num_dof)
    r[:3 * mesh.num_nodes] = O.residual(mesh, uex_full[:3 * mesh.num_nodes], aux, f1=F1_ILE)
    O.cohesive_residual(mesh, uex_full, slip, consts, r=r)
    # A unit strain error would give residuals of order mu * |d| * h.
    h = 3000.0
    assert np.abs(r).max() <= 1e-12 * mu.max() * np.linalg.norm(d) * h
    # Solve the saddle point from zero with Dirichlet values on the x faces.
    Kd = O.assemble(mesh, O.jacobian_elements(mesh, aux, g3=JF3_ILE), ndof=mesh.num_dof)
    J = (Kd + O.cohesive_jacobian(mesh, consts)).tocsr()
    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    cons[M.boundary_mask(mesh, 0, "neg")] = True
    cons[M.boundary_mask(mesh, 0, "pos")] = True
    cons = np.concatenate([cons.ravel(), np.zeros(3 * mesh.num_lagrange, dtype=bool)])
    u = np.where(cons, uex_full, 0.0)
    r = np.zeros(mesh.num_dof)
    r[:3 * mesh.num_nodes] = O.residual(mesh, u[:3 * mesh.num_nodes], aux, f1=F1_ILE)
    O.cohesive_residual(mesh, u, slip, consts, r=r)
    free = ~cons
    u[free] += spla.spsolve(sp.csc_matrix(J[free][:, free]), -r[free])
    nd = 3 * mesh.num_nodes
    np.testing.assert_allclose(u[:nd], uex_full[:nd], atol=1e-9)
    # lambda is a traction (Pa); zero to rounding relative to mu
    np.testing.assert_allclose(u[nd:], 0.0, atol=1e-12 * mu.max())


@pytest.mark.parametrize("make", [lambda: M.box_hex(3, 3, 2), lambda: M.box_tet_delaunay(1500, seed=4),
                                  lambda: M.box_hex27(2, 2, 2)], ids=["hex8", "tet4", "hex27"])
def test_derived_fields_known_answer(oracle_lib, make):
    """Basis-order-0 derived fields (Elasticity::_setKernelsDerivedField, Elasticity.cc:629-651):
    for a linear displacement the centroid strain is the imposed strain and the stress is
    K tr(e) I + 2 mu dev(e) in every cell; the restatement and the reference kernels agree bit for
    bit through the same projection."""
    O = oracle_lib
    mesh = make()
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=2)
    aux = elastic_aux(O, rho, mu, K)
    G = np.array([[1e-4, 2e-5, -3e-5], [3e-5, -1e-4, 4e-5], [-2e-5, 1e-5, 5e-5]])
    u = (mesh.coords @ G.T).ravel()
    fns = ["IsotropicLinearElasticity3D::cauchyStress_infinitesimalStrain_asVector",
           "Elasticity3D::infinitesimalStrain_asVector"]
    stress, strain = O.project_centroid(mesh, u, aux, fns, [6, 6])
    e = 0.5 * (G + G.T)
    ev = np.array([e[0, 0], e[1, 1], e[2, 2], e[0, 1], e[1, 2], e[0, 2]])
    np.testing.assert_allclose(strain, np.tile(ev, (mesh.num_cells, 1)), rtol=0, atol=1e-13 * np.abs(ev).max())
    tr = np.trace(e)
    dev = ev - np.array([tr / 3, tr / 3, tr / 3, 0, 0, 0])
    sig = K[:, None] * np.array([tr, tr, tr, 0, 0, 0]) + 2 * mu[:, None] * dev
    np.testing.assert_allclose(stress, sig, rtol=1e-12, atol=1e-12 * np.abs(sig).max())
    if O.ref_available():
        s_ref, e_ref = O.project_centroid(mesh, u, aux, fns, [6, 6], source="ref")
        np.testing.assert_array_equal(stress, s_ref)
        np.testing.assert_array_equal(strain, e_ref)


@pytest.mark.parametrize("make", [lambda: M.box_tet_delaunay(2000, seed=3), lambda: M.box_hex(4, 3, 3),
                                  lambda: M.box_hex27(2, 2, 2)], ids=["tet4", "hex8", "hex27"])
def test_jacobian_action_equals_assembled_elements(oracle_lib, make):
    """The matrix-free action (DMPlexComputeJacobianActionByKey) is the assembled element Jacobians
    applied to v, for the elastic and the generalized-Maxwell tangents."""
    O = oracle_lib
    mesh = make()
    rng = np.random.default_rng(7)
    nc, nq = mesh.num_cells, M.QUAD_POINTS[mesh.cell_type]
    rho, mu, K = MAT.lognormal_elastic(nc, seed=2)
    tau = MAT.genmaxwell_times(rho, np.sqrt(mu / rho), [1e18, 1e19, 1e20], [0.3, 0.3, 0.3])
    gm = O.AuxFields([(rho[:, None], "cell"), (mu[:, None], "cell"), (K[:, None], "cell"), (tau, "cell"),
                      (np.tile([0.3, 0.3, 0.3], (nc, 1)), "cell"), (np.zeros((nc, nq, 18)), "qp"),
                      (np.zeros((nc, nq, 6)), "qp")])
    el = O.AuxFields([(rho[:, None], "cell"), (mu[:, None], "cell"), (K[:, None], "cell")])
    v = rng.standard_normal(mesh.num_dof)
    for aux, g3, consts in ((el, "IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain", None),
                            (gm, "IsotropicLinearGenMaxwell3D::Jf3vu_infinitesimalStrain", [MAT.YEAR])):
        J = O.assemble(mesh, O.jacobian_elements(mesh, aux, g3=g3, constants=consts))
        jv = O.jacobian_action(mesh, v, aux, g3=g3, constants=consts)
        assert np.linalg.norm(jv - J @ v) <= 1e-13 * np.linalg.norm(J @ v)
