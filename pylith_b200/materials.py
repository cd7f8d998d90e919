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
