"""Analytic known answers from the reference's own tests, restated as functions.

  * axial displacement: tests/fullscale/linearelasticity/nofaults-3d/axialdisp_soln.py
  * generalized Maxwell axial strain relaxation:
    tests/fullscale/viscoelasticity/nofaults-3d/axialstrain_genmaxwell_soln.py
  * uniform-strain MMS: tests/mmstests/linearelasticity/nofaults-3d/UniformStrain3D.cc
    (a linear displacement field makes the interior residual vanish)
"""
import numpy as np

from pylith_b200 import materials as MAT

# axialdisp_soln.py:27-47
AXIAL_DENSITY = 2500.0
AXIAL_VS = 3000.0
AXIAL_VP = 5291.502622129181


def axial_strain():
    mu = AXIAL_DENSITY * AXIAL_VS**2
    lam = AXIAL_DENSITY * AXIAL_VP**2 - 2 * mu
    sxx, syy, szz = 1.0e7, -0.8e7, 0.0
    tr = sxx + syy + szz
    exx = 1.0 / (2 * mu) * (sxx - lam / (3 * lam + 2 * mu) * tr)
    eyy = 1.0 / (2 * mu) * (syy - lam / (3 * lam + 2 * mu) * tr)
    ezz = 1.0 / (2 * mu) * (szz - lam / (3 * lam + 2 * mu) * tr)
    return exx, eyy, ezz


def axial_displacement(coords):
    exx, eyy, ezz = axial_strain()
    return np.stack([exx * coords[:, 0], eyy * coords[:, 1], ezz * coords[:, 2]], axis=1)


def axial_constrained(mesh):
    """bc_xneg/xpos constrain ux, bc_yneg/ypos uy, bc_zneg uz (axialdisp.cfg)."""
    from pylith_b200 import meshing as M

    cons = np.zeros((mesh.num_nodes, 3), dtype=bool)
    for side in ("neg", "pos"):
        cons[M.boundary_mask(mesh, 0, side), 0] = True
        cons[M.boundary_mask(mesh, 1, side), 1] = True
    cons[M.boundary_mask(mesh, 2, "neg"), 2] = True
    return cons.ravel()


# axialstrain_genmaxwell_soln.py:22-47
GM_DENSITY = 2500.0
GM_VS = 3464.1016
GM_VP = 6000.0
GM_VISCOSITY = (9.46728e17, 4.73364e17, 1.893456e18)
GM_RATIO = (0.25, 0.25, 0.25)
GM_E0 = 1.0 / 8000.0
GM_DT = 0.025 * MAT.YEAR
GM_STEPS = 20


def genmaxwell_params():
    mu = GM_DENSITY * GM_VS**2
    lam = GM_DENSITY * GM_VP**2 - 2.0 * mu
    K = lam + 2.0 * mu / 3.0
    tau = np.array([GM_VISCOSITY[i] / (mu * GM_RATIO[i]) for i in range(3)])
    return mu, K, lam, tau


def genmaxwell_stress(t):
    """Analytic Cauchy stress (xx, yy, zz) at time t for the constant axial strain e0 in z."""
    mu, K, lam, tau = genmaxwell_params()
    ezz = GM_E0
    emean = ezz / 3.0
    edev = np.array([-emean, -emean, ezz - emean])
    r0 = 1.0 - sum(GM_RATIO)
    fac = r0 + sum(GM_RATIO[i] * np.exp(-t / tau[i]) for i in range(3))
    smean = GM_E0 * (3.0 * lam + 2.0 * mu) / 3.0
    return 2.0 * mu * edev * fac + smean


def stress_from_residual(coords, r, volume):
    """Uniform Cauchy stress recovered from a residual with f1 = -sigma:
    sum_a r_a (x) X_a = -sigma V for any basis that reproduces linear fields."""
    R = r.reshape(-1, 3)
    return -(R.T @ coords) / volume
