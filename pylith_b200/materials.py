"""Material parameters and seeded synthetic material fields.

Conversions follow the reference's spatial-database queries
(libsrc/pylith/materials/Query.cc):
  shear modulus   mu = rho vs^2                       (_Query::vmToShearModulus)
  bulk modulus    K  = rho (vp^2 - 4/3 vs^2)          (_Query::vmToBulkModulus)
  Maxwell times   tau_i = eta_i / (r_i mu)            (_Query::vmToGeneralizedMaxwellTimes)
"""
from __future__ import annotations

import numpy as np

YEAR = 60.0 * 60.0 * 24.0 * 365.25


def shear_modulus(density, vs):
    return np.asarray(density) * np.asarray(vs) ** 2


def bulk_modulus(density, vs, vp):
    vs = np.asarray(vs)
    vp = np.asarray(vp)
    return np.asarray(density) * (vp * vp - 4.0 / 3.0 * vs * vs)


def genmaxwell_times(density, vs, viscosities, ratios):
    mu = shear_modulus(density, vs)
    eta = np.asarray(viscosities, dtype=np.float64)
    r = np.asarray(ratios, dtype=np.float64)
    mu_i = np.multiply.outer(np.atleast_1d(mu), r)
    with np.errstate(divide="ignore"):
        tau = np.where(mu_i > 0.0, eta / mu_i, np.finfo(np.float64).max)
    return tau if np.ndim(mu) else tau[0]


def uniform_elastic(ncells, density=2500.0, vs=3000.0, vp=5291.503):
    """Per-cell (density, mu, K) for a uniform material (the small hex box)."""
    rho = np.full(ncells, density)
    return rho, shear_modulus(rho, vs), bulk_modulus(rho, vs, vp)


def lognormal_elastic(ncells, seed=0, vs_median=3000.0, sigma_log=0.2, density=2700.0,
                      density_spread=0.05):
    """Per-cell log-normal material: Vs = median * exp(sigma N(0,1)), Vp = sqrt(3) Vs,
    density = 2700 * U(1 - 5%, 1 + 5%)."""
    rng = np.random.default_rng(seed)
    vs = vs_median * np.exp(sigma_log * rng.standard_normal(ncells))
    vp = np.sqrt(3.0) * vs
    rho = density * rng.uniform(1.0 - density_spread, 1.0 + density_spread, ncells)
    return rho, shear_modulus(rho, vs), bulk_modulus(rho, vs, vp)


# ---- kernel registration (what PyLith's material and fault objects do) --------------------
class IsotropicLinearElasticity:
    """Quasi-static isotropic linear elasticity; registers the kernels PyLith's Elasticity
    chooses for this rheology (libsrc/pylith/materials/Elasticity.cc:448-563):
    f0u = g0v_bodyforce (when a body force is given), f1u = f1v_infinitesimalStrain,
    Jf3uu = Jf3vu_infinitesimalStrain."""

    def __init__(self, density, shear_modulus, bulk_modulus, body_force=None):
        self.density = np.asarray(density, dtype=np.float64)
        self.shear_modulus = np.asarray(shear_modulus, dtype=np.float64)
        self.bulk_modulus = np.asarray(bulk_modulus, dtype=np.float64)
        self.body_force = None if body_force is None else np.asarray(body_force, dtype=np.float64)

    def create_integrator(self, dmesh, cell_ids=None):
        from . import feassemble as FA

        k = FA.fekernels
        ig = FA.IntegratorDomain(dmesh, cell_ids)
        ig.set_aux("density", FA.PER_CELL, self.density[:, None])
        if self.body_force is not None:
            ig.set_aux("body_force", FA.PER_CELL, self.body_force)
        ig.set_aux("shear_modulus", FA.PER_CELL, self.shear_modulus[:, None])
        ig.set_aux("bulk_modulus", FA.PER_CELL, self.bulk_modulus[:, None])
        r0 = k.Elasticity.g0v_bodyforce if self.body_force is not None else None
        ig.set_kernels_residual([FA.ResidualKernels(
            "displacement", FA.LHS, r0, k.IsotropicLinearElasticity3D.f1v_infinitesimalStrain)])
        ig.set_kernels_jacobian([FA.JacobianKernels(
            "displacement", "displacement", FA.LHS, None, None, None,
            k.IsotropicLinearElasticity3D.Jf3vu_infinitesimalStrain)])
        # Elasticity::_setKernelsDerivedField (Elasticity.cc:629-651)
        ig.set_kernels_derived_field([
            FA.ProjectKernels("cauchy_stress", k.IsotropicLinearElasticity3D.cauchyStress_infinitesimalStrain_asVector),
            FA.ProjectKernels("cauchy_strain", k.Elasticity3D.infinitesimalStrain_asVector)])
        return ig


class IsotropicLinearGenMaxwell:
    """Generalized Maxwell viscoelasticity with 3 Maxwell elements and state kept per
    quadrature point (libsrc/pylith/materials/IsotropicLinearGenMaxwell.cc:33,94-102,200-243).
    constants = [dt]."""

    def __init__(self, density, shear_modulus, bulk_modulus, maxwell_time, shear_modulus_ratio,
                 viscous_strain, total_strain):
        self.density = np.asarray(density, dtype=np.float64)
        self.shear_modulus = np.asarray(shear_modulus, dtype=np.float64)
        self.bulk_modulus = np.asarray(bulk_modulus, dtype=np.float64)
        self.maxwell_time = np.asarray(maxwell_time, dtype=np.float64)
        self.shear_modulus_ratio = np.asarray(shear_modulus_ratio, dtype=np.float64)
        self.viscous_strain = np.asarray(viscous_strain, dtype=np.float64)
        self.total_strain = np.asarray(total_strain, dtype=np.float64)

    def create_integrator(self, dmesh, dt, cell_ids=None):
        from . import feassemble as FA

        k = FA.fekernels
        ig = FA.IntegratorDomain(dmesh, cell_ids)
        ig.set_aux("density", FA.PER_CELL, self.density[:, None])
        ig.set_aux("shear_modulus", FA.PER_CELL, self.shear_modulus[:, None])
        ig.set_aux("bulk_modulus", FA.PER_CELL, self.bulk_modulus[:, None])
        ig.set_aux("maxwell_time", FA.PER_CELL, self.maxwell_time)
        ig.set_aux("shear_modulus_ratio", FA.PER_CELL, self.shear_modulus_ratio)
        ig.set_aux("viscous_strain", FA.PER_QUADPT, self.viscous_strain)
        ig.set_aux("total_strain", FA.PER_QUADPT, self.total_strain)
        ig.set_constants([dt])
        ig.set_kernels_residual([FA.ResidualKernels(
            "displacement", FA.LHS, None, k.IsotropicLinearGenMaxwell3D.f1v_infinitesimalStrain)])
        ig.set_kernels_jacobian([FA.JacobianKernels(
            "displacement", "displacement", FA.LHS, None, None, None,
            k.IsotropicLinearGenMaxwell3D.Jf3vu_infinitesimalStrain)])
        ig.set_kernels_update_state_vars([
            FA.ProjectKernels("viscous_strain",
                              k.IsotropicLinearGenMaxwell3D.viscousStrain_infinitesimalStrain_asVector),
            FA.ProjectKernels("total_strain", k.Elasticity3D.infinitesimalStrain_asVector)])
        # Elasticity::_setKernelsDerivedField (Elasticity.cc:629-651)
        ig.set_kernels_derived_field([
            FA.ProjectKernels("cauchy_stress", k.IsotropicLinearGenMaxwell3D.cauchyStress_infinitesimalStrain_asVector),
            FA.ProjectKernels("cauchy_strain", k.Elasticity3D.infinitesimalStrain_asVector)])
        return ig


class FaultCohesiveKin:
    """Prescribed-slip fault on cohesive cells (libsrc/pylith/faults/FaultCohesiveKin.cc:330-461;
    constants refDir1, refDir2 from FaultCohesive.cc:526-539). slip: [nlag][3] as (opening,
    left-lateral, reverse)."""

    def __init__(self, slip, ref_dir_1=(0.0, 0.0, 1.0), ref_dir_2=(0.0, 1.0, 0.0)):
        self.slip = np.asarray(slip, dtype=np.float64)
        self.constants = list(ref_dir_1) + list(ref_dir_2)

    def create_integrator(self, dmesh):
        from . import feassemble as FA

        k = FA.fekernels
        ig = FA.IntegratorInterface(dmesh)
        ig.set_aux("slip", FA.PER_FAULT_NODE, self.slip)
        ig.set_constants(self.constants)
        ig.set_kernels_residual([
            FA.InterfaceResidualKernels("displacement", FA.LHS, FA.FACE_NEGATIVE, k.FaultCohesiveKin.f0u_neg),
            FA.InterfaceResidualKernels("displacement", FA.LHS, FA.FACE_POSITIVE, k.FaultCohesiveKin.f0u_pos),
            FA.InterfaceResidualKernels("lagrange_multiplier_fault", FA.LHS, FA.FACE_FAULT,
                                        k.FaultCohesiveKin.f0l_slip)])
        ig.set_kernels_jacobian([
            FA.InterfaceJacobianKernels("displacement", "lagrange_multiplier_fault", FA.LHS,
                                        FA.FACE_NEGATIVE, k.FaultCohesiveKin.Jf0ul_neg),
            FA.InterfaceJacobianKernels("displacement", "lagrange_multiplier_fault", FA.LHS,
                                        FA.FACE_POSITIVE, k.FaultCohesiveKin.Jf0ul_pos),
            FA.InterfaceJacobianKernels("lagrange_multiplier_fault", "displacement", FA.LHS,
                                        FA.FACE_FAULT, k.FaultCohesiveKin.Jf0lu)])
        return ig
