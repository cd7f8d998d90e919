// ORACLE — test infrastructure only. Nothing in the product library includes,
// links or calls this file; tests/, bench.py's CPU-baseline leg and smoke()
// use it as the oracle.
//
// CPU restatement of the PyLith pointwise kernels on the residual/Jacobian hot
// path, written against PETSc's pointwise-function signature
// (docs/developer/implementation/petsc-fem.md:438-600). Each function cites
// the reference kernel it restates. The arithmetic follows the reference's
// order of operations so that results agree to rounding; the tests check this
// against the reference kernels compiled from the PyLith sources (oracle/_ref).
#pragma once

#include <cmath>

namespace oracle {
namespace pw {

typedef int Int;
typedef double Real;

#define ORACLE_POINT_ARGS                                                                    \
    Int dim, Int numS, Int numA, const Int sOff[], const Int sOff_x[], const Real s[],       \
    const Real s_t[], const Real s_x[], const Int aOff[], const Int aOff_x[], const Real a[], \
    const Real a_t[], const Real a_x[], Real t

typedef void (*PointFn)(ORACLE_POINT_ARGS, const Real x[], Int numConstants, const Real constants[],
                        Real f[]);
typedef void (*PointJacFn)(ORACLE_POINT_ARGS, Real s_tshift, const Real x[], Int numConstants,
                           const Real constants[], Real g[]);
typedef void (*BdPointFn)(ORACLE_POINT_ARGS, const Real x[], const Real n[], Int numConstants,
                          const Real constants[], Real f[]);
typedef void (*BdPointJacFn)(ORACLE_POINT_ARGS, Real s_tshift, const Real x[], const Real n[],
                             Int numConstants, const Real constants[], Real g[]);

// Symmetric 3x3 tensor, component order xx, yy, zz, xy, yz, xz
// (libsrc/pylith/fekernels/Tensor.hh:21-24).
struct Sym {
    Real xx = 0, yy = 0, zz = 0, xy = 0, yz = 0, xz = 0;
};

static inline Sym sym_from_vector(const Real* v) {
    Sym t;
    t.xx = v[0]; t.yy = v[1]; t.zz = v[2]; t.xy = v[3]; t.yz = v[4]; t.xz = v[5];
    return t;
}

// Elasticity3D::infinitesimalStrain (Elasticity.hh:560-575).
static inline Sym strain_from_grad(const Real* u_x) {
    Sym e;
    e.xx = u_x[0];
    e.yy = u_x[4];
    e.zz = u_x[8];
    e.xy = 0.5 * (u_x[1] + u_x[3]);
    e.yz = 0.5 * (u_x[5] + u_x[7]);
    e.xz = 0.5 * (u_x[2] + u_x[6]);
    return e;
}

// Elasticity::deviatoric (Elasticity.hh:392-407).
static inline Sym deviatoric(const Sym& t) {
    const Real mean = (t.xx + t.yy + t.zz) / 3.0;
    Sym d;
    d.xx = t.xx - mean; d.yy = t.yy - mean; d.zz = t.zz - mean;
    d.xy = t.xy; d.yz = t.yz; d.xz = t.xz;
    return d;
}

// IsotropicLinearElasticity::meanStress (IsotropicLinearElasticity.hh:222-234).
static inline void add_mean_stress(Real K, const Sym& e, Sym* s) {
    const Real m = K * (e.xx + e.yy + e.zz);
    s->xx += m; s->yy += m; s->zz += m;
}

// IsotropicLinearElasticity::deviatoricStress (IsotropicLinearElasticity.hh:240-255).
static inline void add_dev_stress(Real mu, const Sym& e, Sym* s) {
    const Real tr = e.xx + e.yy + e.zz;
    const Real trace_term = -2.0 / 3.0 * mu * tr;
    s->xx += 2.0 * mu * e.xx + trace_term;
    s->yy += 2.0 * mu * e.yy + trace_term;
    s->zz += 2.0 * mu * e.zz + trace_term;
    s->xy += 2.0 * mu * e.xy;
    s->yz += 2.0 * mu * e.yz;
    s->xz += 2.0 * mu * e.xz;
}

// Elasticity::f1v accumulation into the 3x3 row-major f1 (Elasticity.hh:172-191,
// TensorOps::_toTensor3D at Tensor.hh:235-247).
static inline void f1_minus_stress(const Sym& s, Real f1[]) {
    f1[0] -= s.xx; f1[1] -= s.xy; f1[2] -= s.xz;
    f1[3] -= s.xy; f1[4] -= s.yy; f1[5] -= s.yz;
    f1[6] -= s.xz; f1[7] -= s.yz; f1[8] -= s.zz;
}

// Elasticity::g0v_bodyforce (Elasticity.hh:300-334): g0 += body_force, aux index 1.
static inline void g0v_bodyforce(ORACLE_POINT_ARGS, const Real x[], Int numConstants,
                                 const Real constants[], Real g0[]) {
    const Real* bf = &a[aOff[1]];
    for (Int i = 0; i < dim; ++i) g0[i] += bf[i];
}

// IsotropicLinearElasticity3D::f1v_infinitesimalStrain (IsotropicLinearElasticity.hh:804-838):
// mu = a[aOff[numA-2]], K = a[aOff[numA-1]]; f1 -= K tr(e) I + 2 mu dev(e).
static inline void ile3d_f1v(ORACLE_POINT_ARGS, const Real x[], Int numConstants,
                             const Real constants[], Real f1[]) {
    const Real mu = a[aOff[numA - 2]];
    const Real K = a[aOff[numA - 1]];
    const Sym e = strain_from_grad(&s_x[sOff_x[0]]);
    Sym sig;
    add_mean_stress(K, e, &sig);
    add_dev_stress(mu, e, &sig);
    f1_minus_stress(sig, f1);
}

// Nonzero pattern of the isotropic elastic tangent, j(f,g,df,dg) = C(f,df,g,dg), index
// ((f*3+g)*3+df)*3+dg (IsotropicLinearElasticity.hh:928-1034).
static inline void jf3_isotropic(Real C1111, Real C1122, Real C1212, Real Jf3[]) {
    Jf3[0] -= C1111;  Jf3[4] -= C1212;  Jf3[8] -= C1212;  Jf3[10] -= C1122;
    Jf3[12] -= C1212; Jf3[20] -= C1122; Jf3[24] -= C1212; Jf3[28] -= C1212;
    Jf3[30] -= C1122; Jf3[36] -= C1212; Jf3[40] -= C1111; Jf3[44] -= C1212;
    Jf3[50] -= C1122; Jf3[52] -= C1212; Jf3[56] -= C1212; Jf3[60] -= C1122;
    Jf3[68] -= C1212; Jf3[70] -= C1122; Jf3[72] -= C1212; Jf3[76] -= C1212;
    Jf3[80] -= C1111;
}

// IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain (IsotropicLinearElasticity.hh:891-1035).
static inline void ile3d_Jf3vu(ORACLE_POINT_ARGS, Real s_tshift, const Real x[], Int numConstants,
                               const Real constants[], Real Jf3[]) {
    const Real mu = a[aOff[numA - 2]];
    const Real K = a[aOff[numA - 1]];
    const Real lambda = K - 2.0 / 3.0 * mu;
    const Real lambda2mu = lambda + 2.0 * mu;
    jf3_isotropic(lambda2mu, lambda, mu, Jf3);
}

// IsotropicLinearMaxwell::viscousStrainCoeff (IsotropicLinearMaxwell.hh:220-223).
static inline Real maxwell_dq(Real dt, Real tau) { return tau * (1.0 - std::exp(-dt / tau)) / dt; }

// IsotropicLinearMaxwell::viscousStrain (IsotropicLinearMaxwell.hh:256-278).
static inline Sym maxwell_viscous_strain(Real tau, const Sym& prev, const Sym& total_prev,
                                         const Sym& e, Real dt) {
    const Sym de = deviatoric(e);
    const Sym dt_prev = deviatoric(total_prev);
    const Real dq = maxwell_dq(dt, tau);
    const Real ef = std::exp(-dt / tau);
    Sym v;
    v.xx = ef * prev.xx + dq * (de.xx - dt_prev.xx);
    v.yy = ef * prev.yy + dq * (de.yy - dt_prev.yy);
    v.zz = ef * prev.zz + dq * (de.zz - dt_prev.zz);
    v.xy = ef * prev.xy + dq * (de.xy - dt_prev.xy);
    v.yz = ef * prev.yz + dq * (de.yz - dt_prev.yz);
    v.xz = ef * prev.xz + dq * (de.xz - dt_prev.xz);
    return v;
}

// Generalized Maxwell aux layout, indexed from the back of the aux list
// (IsotropicLinearGenMaxwell.hh:136-141): mu, K, maxwell_time(3), shear_modulus_ratio(3),
// viscous_strain(18), total_strain(6); constants[0] = dt (IsotropicLinearGenMaxwell.cc:200-214).
struct GenMaxwellCtx {
    Real mu, K, dt;
    const Real* tau;
    const Real* ratio;
    Sym visc[3];
    Sym total;
};

static inline GenMaxwellCtx genmaxwell_ctx(Int numA, const Int aOff[], const Real a[],
                                           const Real constants[]) {
    GenMaxwellCtx c;
    c.mu = a[aOff[numA - 6]];
    c.K = a[aOff[numA - 5]];
    c.tau = &a[aOff[numA - 4]];
    c.ratio = &a[aOff[numA - 3]];
    c.dt = constants[0];
    for (int i = 0; i < 3; ++i) c.visc[i] = sym_from_vector(&a[aOff[numA - 2] + 6 * i]);
    c.total = sym_from_vector(&a[aOff[numA - 1]]);
    return c;
}

// IsotropicLinearGenMaxwell::cauchyStress + _deviatoricStress
// (IsotropicLinearGenMaxwell.hh:267-292, 404-447).
static inline Sym genmaxwell_stress(const GenMaxwellCtx& c, const Sym& e) {
    Sym s;
    add_mean_stress(c.K, e, &s);
    Sym v[3];
    for (int i = 0; i < 3; ++i) v[i] = maxwell_viscous_strain(c.tau[i], c.visc[i], c.total, e, c.dt);
    const Sym de = deviatoric(e);
    Real ratio = 1.0;
    for (int i = 0; i < 3; ++i) ratio -= c.ratio[i];
    const Real mu_el = c.mu * ratio;  // shearModulusElastic (:389-396)
    s.xx += 2.0 * mu_el * de.xx;
    for (int i = 0; i < 3; ++i) s.xx += 2.0 * c.mu * c.ratio[i] * v[i].xx;
    s.yy += 2.0 * mu_el * de.yy;
    for (int i = 0; i < 3; ++i) s.yy += 2.0 * c.mu * c.ratio[i] * v[i].yy;
    s.zz += 2.0 * mu_el * de.zz;
    for (int i = 0; i < 3; ++i) s.zz += 2.0 * c.mu * c.ratio[i] * v[i].zz;
    s.xy += 2.0 * mu_el * de.xy;
    for (int i = 0; i < 3; ++i) s.xy += 2.0 * c.mu * c.ratio[i] * v[i].xy;
    s.yz += 2.0 * mu_el * de.yz;
    for (int i = 0; i < 3; ++i) s.yz += 2.0 * c.mu * c.ratio[i] * v[i].yz;
    s.xz += 2.0 * mu_el * de.xz;
    for (int i = 0; i < 3; ++i) s.xz += 2.0 * c.mu * c.ratio[i] * v[i].xz;
    return s;
}

// IsotropicLinearGenMaxwell3D::f1v_infinitesimalStrain (IsotropicLinearGenMaxwell.hh:1054-1087).
static inline void gm3d_f1v(ORACLE_POINT_ARGS, const Real x[], Int numConstants,
                            const Real constants[], Real f1[]) {
    const GenMaxwellCtx c = genmaxwell_ctx(numA, aOff, a, constants);
    const Sym e = strain_from_grad(&s_x[sOff_x[0]]);
    f1_minus_stress(genmaxwell_stress(c, e), f1);
}

// IsotropicLinearGenMaxwell3D::Jf3vu_infinitesimalStrain (IsotropicLinearGenMaxwell.hh:1143-1300).
static inline void gm3d_Jf3vu(ORACLE_POINT_ARGS, Real s_tshift, const Real x[], Int numConstants,
                              const Real constants[], Real Jf3[]) {
    const GenMaxwellCtx c = genmaxwell_ctx(numA, aOff, a, constants);
    const Real r0 = 1.0 - c.ratio[0] - c.ratio[1] - c.ratio[2];
    Real shear = c.mu * r0;
    for (int i = 0; i < 3; ++i) shear += c.mu * maxwell_dq(c.dt, c.tau[i]) * c.ratio[i];
    const Real C1111 = c.K + 4.0 * shear / 3.0;
    const Real C1122 = c.K - 2.0 * shear / 3.0;
    jf3_isotropic(C1111, C1122, shear, Jf3);
}

// IsotropicLinearGenMaxwell3D::viscousStrain_infinitesimalStrain_asVector
// (IsotropicLinearGenMaxwell.hh:1507-1549): 18 values, element i at offset 6*i.
static inline void gm3d_viscous_strain(ORACLE_POINT_ARGS, const Real x[], Int numConstants,
                                       const Real constants[], Real out[]) {
    const GenMaxwellCtx c = genmaxwell_ctx(numA, aOff, a, constants);
    const Sym e = strain_from_grad(&s_x[sOff_x[0]]);
    for (int i = 0; i < 3; ++i) {
        const Sym v = maxwell_viscous_strain(c.tau[i], c.visc[i], c.total, e, c.dt);
        Real* o = out + 6 * i;
        o[0] = v.xx; o[1] = v.yy; o[2] = v.zz; o[3] = v.xy; o[4] = v.yz; o[5] = v.xz;
    }
}

// Elasticity3D::infinitesimalStrain_asVector (Elasticity.hh:587-612).
static inline void el3d_strain_vector(ORACLE_POINT_ARGS, const Real x[], Int numConstants,
                                      const Real constants[], Real out[]) {
    const Sym e = strain_from_grad(&s_x[sOff_x[0]]);
    out[0] = e.xx; out[1] = e.yy; out[2] = e.zz; out[3] = e.xy; out[4] = e.yz; out[5] = e.xz;
}

// Stress tensor as a vector, xx, yy, zz, xy, yz, xz (Elasticity::stress_asVector,
// Elasticity.hh:441-456).
static inline void stress_to_vector(const Sym& s, Real out[]) {
    out[0] = s.xx; out[1] = s.yy; out[2] = s.zz; out[3] = s.xy; out[4] = s.yz; out[5] = s.xz;
}

// IsotropicLinearElasticity3D::cauchyStress_infinitesimalStrain_asVector
// (IsotropicLinearElasticity.hh:1243-1273): IsotropicLinearElasticity::cauchyStress
// (:183-193) = meanStress then deviatoricStress.
static inline void ile3d_stress_vector(ORACLE_POINT_ARGS, const Real x[], Int numConstants,
                                       const Real constants[], Real out[]) {
    const Real mu = a[aOff[numA - 2]];
    const Real K = a[aOff[numA - 1]];
    const Sym e = strain_from_grad(&s_x[sOff_x[0]]);
    Sym sig;
    add_mean_stress(K, e, &sig);
    add_dev_stress(mu, e, &sig);
    stress_to_vector(sig, out);
}

// IsotropicLinearGenMaxwell3D::cauchyStress_infinitesimalStrain_asVector
// (IsotropicLinearGenMaxwell.hh:1556-1589) with cauchyStress_stateVars (:340-357): the stored
// viscous strains, not updated.
static inline void gm3d_stress_vector(ORACLE_POINT_ARGS, const Real x[], Int numConstants,
                                      const Real constants[], Real out[]) {
    const GenMaxwellCtx c = genmaxwell_ctx(numA, aOff, a, constants);
    const Sym e = strain_from_grad(&s_x[sOff_x[0]]);
    Sym sig;
    add_mean_stress(c.K, e, &sig);
    const Sym de = deviatoric(e);
    Real ratio = 1.0;
    for (int i = 0; i < 3; ++i) ratio -= c.ratio[i];
    const Real mu_el = c.mu * ratio;
    sig.xx += 2.0 * mu_el * de.xx;
    for (int i = 0; i < 3; ++i) sig.xx += 2.0 * c.mu * c.ratio[i] * c.visc[i].xx;
    sig.yy += 2.0 * mu_el * de.yy;
    for (int i = 0; i < 3; ++i) sig.yy += 2.0 * c.mu * c.ratio[i] * c.visc[i].yy;
    sig.zz += 2.0 * mu_el * de.zz;
    for (int i = 0; i < 3; ++i) sig.zz += 2.0 * c.mu * c.ratio[i] * c.visc[i].zz;
    sig.xy += 2.0 * mu_el * de.xy;
    for (int i = 0; i < 3; ++i) sig.xy += 2.0 * c.mu * c.ratio[i] * c.visc[i].xy;
    sig.yz += 2.0 * mu_el * de.yz;
    for (int i = 0; i < 3; ++i) sig.yz += 2.0 * c.mu * c.ratio[i] * c.visc[i].yz;
    sig.xz += 2.0 * mu_el * de.xz;
    for (int i = 0; i < 3; ++i) sig.xz += 2.0 * c.mu * c.ratio[i] * c.visc[i].xz;
    stress_to_vector(sig, out);
}

// BoundaryDirections::_unitCrossProduct (BoundaryDirections.hh:248-270).
static inline void unit_cross(Real r[3], const Real a[3], const Real b[3]) {
    r[0] = +a[1] * b[2] - a[2] * b[1];
    r[1] = +a[2] * b[0] - a[0] * b[2];
    r[2] = +a[0] * b[1] - a[1] * b[0];
    Real mag = 0.0;
    for (int i = 0; i < 3; ++i) mag += r[i] * r[i];
    mag = std::sqrt(mag);
    for (int i = 0; i < 3; ++i) r[i] /= mag;
}

// BoundaryDirections::tangential_directions (BoundaryDirections.hh:35-67). The sign test on
// the second tangent uses refDir2[1]*n[1] twice, exactly as the reference does (:62).
static inline void tangential_directions(Real t1[3], Real t2[3], const Real ref1[3],
                                         const Real ref2[3], const Real n[3]) {
    Real ref[3] = {ref1[0], ref1[1], ref1[2]};
    if (std::fabs(ref[0] * n[0] + ref[1] * n[1] + ref[2] * n[2]) > 0.999) {
        for (int i = 0; i < 3; ++i) ref[i] = ref2[i];
    }
    unit_cross(t1, ref, n);
    unit_cross(t2, n, t1);
    if (ref2[0] * n[0] + ref2[1] * n[1] + ref2[1] * n[1] < 0.0) {
        for (int i = 0; i < 3; ++i) t2[i] *= -1.0;
    }
}

// FaultCohesiveKin::f0u_neg / f0u_pos (FaultCohesiveKin.hh:74-150): f0 -/+= lambda,
// lambda = s[sOff[numS-1]].
static inline void fck_f0u_neg(ORACLE_POINT_ARGS, const Real x[], const Real n[], Int numConstants,
                               const Real constants[], Real f0[]) {
    const Real* lam = &s[sOff[numS - 1]];
    for (Int i = 0; i < dim; ++i) f0[i] += -lam[i];
}
static inline void fck_f0u_pos(ORACLE_POINT_ARGS, const Real x[], const Real n[], Int numConstants,
                               const Real constants[], Real f0[]) {
    const Real* lam = &s[sOff[numS - 1]];
    for (Int i = 0; i < dim; ++i) f0[i] += +lam[i];
}

// FaultCohesiveKin::f0l_slip, 3D branch (FaultCohesiveKin.hh:158-225): slip = a[aOff[0]]
// (opening, left-lateral, reverse); u- at sOff[0], u+ at sOff[0]+3; constants = refDir1, refDir2.
static inline void fck_f0l_slip(ORACLE_POINT_ARGS, const Real x[], const Real n[],
                                Int numConstants, const Real constants[], Real f0[]) {
    const Real* slip = &a[aOff[0]];
    const Real* uN = &s[sOff[0]];
    const Real* uP = &s[sOff[0] + 3];
    Real t1[3], t2[3];
    tangential_directions(t1, t2, &constants[0], &constants[3], n);
    for (int i = 0; i < 3; ++i) {
        const Real slip_xyz = n[i] * slip[0] + t1[i] * slip[1] + t2[i] * slip[2];
        f0[i] += uP[i] - uN[i] - slip_xyz;
    }
}

// FaultCohesiveKin::Jf0ul_neg / Jf0ul_pos / Jf0lu (FaultCohesiveKin.hh:298-412).
static inline void fck_Jf0ul_neg(ORACLE_POINT_ARGS, Real s_tshift, const Real x[], const Real n[],
                                 Int numConstants, const Real constants[], Real Jf0[]) {
    for (Int i = 0; i < dim; ++i) Jf0[i * dim + i] += -1.0;
}
static inline void fck_Jf0ul_pos(ORACLE_POINT_ARGS, Real s_tshift, const Real x[], const Real n[],
                                 Int numConstants, const Real constants[], Real Jf0[]) {
    for (Int i = 0; i < dim; ++i) Jf0[i * dim + i] += +1.0;
}
static inline void fck_Jf0lu(ORACLE_POINT_ARGS, Real s_tshift, const Real x[], const Real n[],
                             Int numConstants, const Real constants[], Real Jf0[]) {
    for (Int i = 0; i < dim; ++i) {
        Jf0[i * dim + i] += -1.0;
        Jf0[dim * dim + i * dim + i] += +1.0;
    }
}

}  // namespace pw
}  // namespace oracle
