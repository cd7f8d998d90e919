// Pointwise physics kernels of the residual/Jacobian path, as host+device code.
//
// Each function keeps the argument list of PETSc's pointwise functions
// (docs/developer/implementation/petsc-fem.md:438-600) so that the cell-loop kernels call
// them exactly the way PETSc's DMPlexComputeResidual calls PyLith's fekernels. They are
// __forceinline__ templates on the scalar type: inside a kernel the offset arrays are
// compile-time constants, so the indirection folds away and the arithmetic stays in
// registers. The same code, instantiated for double, is what the exported
// pylith::fekernels::* host symbols run (include/pylith_b200/fekernels.hh).
#pragma once

#include "common.cuh"

namespace plb {
namespace pw {

#define PLB_POINT_ARGS(R)                                                                  \
    int dim, int numS, int numA, const int* sOff, const int* sOff_x, const R* s,           \
        const R* s_t, const R* s_x, const int* aOff, const int* aOff_x, const R* a,        \
        const R* a_t, const R* a_x, R t

template <typename R>
struct Sym {
    R xx, yy, zz, xy, yz, xz;
};

template <typename R>
PL_HD Sym<R> sym_zero() {
    return Sym<R>{R(0), R(0), R(0), R(0), R(0), R(0)};
}

template <typename R>
PL_HD Sym<R> sym_from_vector(const R* v) {
    return Sym<R>{v[0], v[1], v[2], v[3], v[4], v[5]};
}

// Infinitesimal strain from the row-major displacement gradient (Elasticity.hh:560-575).
template <typename R>
PL_HD Sym<R> strain(const R* u_x) {
    Sym<R> e;
    e.xx = u_x[0];
    e.yy = u_x[4];
    e.zz = u_x[8];
    e.xy = R(0.5) * (u_x[1] + u_x[3]);
    e.yz = R(0.5) * (u_x[5] + u_x[7]);
    e.xz = R(0.5) * (u_x[2] + u_x[6]);
    return e;
}

// Deviatoric part (Elasticity.hh, Elasticity::deviatoric).
template <typename R>
PL_HD Sym<R> deviatoric(const Sym<R>& t) {
    const R mean = (t.xx + t.yy + t.zz) / R(3.0);
    return Sym<R>{t.xx - mean, t.yy - mean, t.zz - mean, t.xy, t.yz, t.xz};
}

// Mean and deviatoric stress of isotropic linear elasticity
// (IsotropicLinearElasticity.hh:222-255).
template <typename R>
PL_HD void add_mean_stress(R K, const Sym<R>& e, Sym<R>* s) {
    const R m = K * (e.xx + e.yy + e.zz);
    s->xx += m;
    s->yy += m;
    s->zz += m;
}

template <typename R>
PL_HD void add_dev_stress(R mu, const Sym<R>& e, Sym<R>* s) {
    const R tr = e.xx + e.yy + e.zz;
    const R trace_term = R(-2.0) / R(3.0) * mu * tr;
    s->xx += R(2.0) * mu * e.xx + trace_term;
    s->yy += R(2.0) * mu * e.yy + trace_term;
    s->zz += R(2.0) * mu * e.zz + trace_term;
    s->xy += R(2.0) * mu * e.xy;
    s->yz += R(2.0) * mu * e.yz;
    s->xz += R(2.0) * mu * e.xz;
}

// f1 -= sigma as a full row-major 3x3 tensor (Elasticity::f1v, Elasticity.hh:172-191).
template <typename R>
PL_HD void f1_minus_stress(const Sym<R>& s, R* f1) {
    f1[0] -= s.xx; f1[1] -= s.xy; f1[2] -= s.xz;
    f1[3] -= s.xy; f1[4] -= s.yy; f1[5] -= s.yz;
    f1[6] -= s.xz; f1[7] -= s.yz; f1[8] -= s.zz;
}

// Elasticity::g0v_bodyforce (Elasticity.hh:300-334): g0 += body_force (aux subfield 1).
template <typename R>
PL_HD void g0v_bodyforce(PLB_POINT_ARGS(R), const R* x, int numConstants, const R* constants,
                         R* g0) {
    const R* bf = &a[aOff[1]];
    for (int i = 0; i < 3; ++i) g0[i] += bf[i];
}

// IsotropicLinearElasticity3D::f1v_infinitesimalStrain (IsotropicLinearElasticity.hh:804-838).
template <typename R>
PL_HD void ile3d_f1v(PLB_POINT_ARGS(R), const R* x, int numConstants, const R* constants,
                     R* f1) {
    const R mu = a[aOff[numA - 2]];
    const R K = a[aOff[numA - 1]];
    const Sym<R> e = strain(&s_x[sOff_x[0]]);
    Sym<R> sig = sym_zero<R>();
    add_mean_stress(K, e, &sig);
    add_dev_stress(mu, e, &sig);
    f1_minus_stress(sig, f1);
}

// Isotropic tangent pattern j(f,g,df,dg) = C(f,df,g,dg) at ((f*3+g)*3+df)*3+dg
// (IsotropicLinearElasticity.hh:928-1034).
template <typename R>
PL_HD void jf3_isotropic(R C1111, R C1122, R C1212, R* Jf3) {
    Jf3[0] -= C1111;  Jf3[4] -= C1212;  Jf3[8] -= C1212;  Jf3[10] -= C1122;
    Jf3[12] -= C1212; Jf3[20] -= C1122; Jf3[24] -= C1212; Jf3[28] -= C1212;
    Jf3[30] -= C1122; Jf3[36] -= C1212; Jf3[40] -= C1111; Jf3[44] -= C1212;
    Jf3[50] -= C1122; Jf3[52] -= C1212; Jf3[56] -= C1212; Jf3[60] -= C1122;
    Jf3[68] -= C1212; Jf3[70] -= C1122; Jf3[72] -= C1212; Jf3[76] -= C1212;
    Jf3[80] -= C1111;
}

// IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain (IsotropicLinearElasticity.hh:891-1035).
template <typename R>
PL_HD void ile3d_Jf3vu(PLB_POINT_ARGS(R), R s_tshift, const R* x, int numConstants,
                       const R* constants, R* Jf3) {
    const R mu = a[aOff[numA - 2]];
    const R K = a[aOff[numA - 1]];
    const R lambda = K - R(2.0) / R(3.0) * mu;
    const R lambda2mu = lambda + R(2.0) * mu;
    jf3_isotropic(lambda2mu, lambda, mu, Jf3);
}

// IsotropicLinearMaxwell::viscousStrainCoeff and the per-element exponential factor
// (IsotropicLinearMaxwell.hh:220-223, 256-278).
template <typename R>
PL_HD R maxwell_dq(R dt, R tau) {
    return tau * (R(1.0) - exp(-dt / tau)) / dt;
}

template <typename R>
PL_HD Sym<R> maxwell_viscous_strain(R tau, const Sym<R>& prev, const Sym<R>& total_prev,
                                    const Sym<R>& e, R dt) {
    const Sym<R> de = deviatoric(e);
    const Sym<R> dp = deviatoric(total_prev);
    const R dq = maxwell_dq(dt, tau);
    const R ef = exp(-dt / tau);
    Sym<R> v;
    v.xx = ef * prev.xx + dq * (de.xx - dp.xx);
    v.yy = ef * prev.yy + dq * (de.yy - dp.yy);
    v.zz = ef * prev.zz + dq * (de.zz - dp.zz);
    v.xy = ef * prev.xy + dq * (de.xy - dp.xy);
    v.yz = ef * prev.yz + dq * (de.yz - dp.yz);
    v.xz = ef * prev.xz + dq * (de.xz - dp.xz);
    return v;
}

// Generalized Maxwell: aux indexed from the back (IsotropicLinearGenMaxwell.hh:136-141):
// mu, K, maxwell_time(3), shear_modulus_ratio(3), viscous_strain(18), total_strain(6);
// constants[0] = dt.
template <typename R>
PL_HD Sym<R> genmaxwell_stress(int numA, const int* aOff, const R* a, const R* constants,
                               const Sym<R>& e) {
    const R mu = a[aOff[numA - 6]];
    const R K = a[aOff[numA - 5]];
    const R* tau = &a[aOff[numA - 4]];
    const R* ratio = &a[aOff[numA - 3]];
    const R* visc = &a[aOff[numA - 2]];
    const Sym<R> total = sym_from_vector(&a[aOff[numA - 1]]);
    const R dt = constants[0];
    Sym<R> s = sym_zero<R>();
    add_mean_stress(K, e, &s);
    Sym<R> v[3];
    for (int i = 0; i < 3; ++i)
        v[i] = maxwell_viscous_strain(tau[i], sym_from_vector(&visc[6 * i]), total, e, dt);
    const Sym<R> de = deviatoric(e);
    R r = R(1.0);
    for (int i = 0; i < 3; ++i) r -= ratio[i];
    const R mu_el = mu * r;  // IsotropicLinearGenMaxwell::shearModulusElastic
    // _deviatoricStress (IsotropicLinearGenMaxwell.hh:404-447), same summation order
    s.xx += R(2.0) * mu_el * de.xx;
    for (int i = 0; i < 3; ++i) s.xx += R(2.0) * mu * ratio[i] * v[i].xx;
    s.yy += R(2.0) * mu_el * de.yy;
    for (int i = 0; i < 3; ++i) s.yy += R(2.0) * mu * ratio[i] * v[i].yy;
    s.zz += R(2.0) * mu_el * de.zz;
    for (int i = 0; i < 3; ++i) s.zz += R(2.0) * mu * ratio[i] * v[i].zz;
    s.xy += R(2.0) * mu_el * de.xy;
    for (int i = 0; i < 3; ++i) s.xy += R(2.0) * mu * ratio[i] * v[i].xy;
    s.yz += R(2.0) * mu_el * de.yz;
    for (int i = 0; i < 3; ++i) s.yz += R(2.0) * mu * ratio[i] * v[i].yz;
    s.xz += R(2.0) * mu_el * de.xz;
    for (int i = 0; i < 3; ++i) s.xz += R(2.0) * mu * ratio[i] * v[i].xz;
    return s;
}

// IsotropicLinearGenMaxwell3D::f1v_infinitesimalStrain (IsotropicLinearGenMaxwell.hh:1054-1087).
template <typename R>
PL_HD void gm3d_f1v(PLB_POINT_ARGS(R), const R* x, int numConstants, const R* constants, R* f1) {
    const Sym<R> e = strain(&s_x[sOff_x[0]]);
    f1_minus_stress(genmaxwell_stress(numA, aOff, a, constants, e), f1);
}

// IsotropicLinearGenMaxwell3D::Jf3vu_infinitesimalStrain (IsotropicLinearGenMaxwell.hh:1143-1300).
template <typename R>
PL_HD void gm3d_Jf3vu(PLB_POINT_ARGS(R), R s_tshift, const R* x, int numConstants,
                      const R* constants, R* Jf3) {
    const R mu = a[aOff[numA - 6]];
    const R K = a[aOff[numA - 5]];
    const R* tau = &a[aOff[numA - 4]];
    const R* ratio = &a[aOff[numA - 3]];
    const R dt = constants[0];
    const R r0 = R(1.0) - ratio[0] - ratio[1] - ratio[2];
    R shear = mu * r0;
    for (int i = 0; i < 3; ++i) shear += mu * maxwell_dq(dt, tau[i]) * ratio[i];
    jf3_isotropic(K + R(4.0) * shear / R(3.0), K - R(2.0) * shear / R(3.0), shear, Jf3);
}

// IsotropicLinearGenMaxwell3D::viscousStrain_infinitesimalStrain_asVector
// (IsotropicLinearGenMaxwell.hh:1507-1549).
template <typename R>
PL_HD void gm3d_viscous_strain(PLB_POINT_ARGS(R), const R* x, int numConstants,
                               const R* constants, R* out) {
    const R* tau = &a[aOff[numA - 4]];
    const R* visc = &a[aOff[numA - 2]];
    const Sym<R> total = sym_from_vector(&a[aOff[numA - 1]]);
    const Sym<R> e = strain(&s_x[sOff_x[0]]);
    for (int i = 0; i < 3; ++i) {
        const Sym<R> v =
            maxwell_viscous_strain(tau[i], sym_from_vector(&visc[6 * i]), total, e, constants[0]);
        R* o = out + 6 * i;
        o[0] = v.xx; o[1] = v.yy; o[2] = v.zz; o[3] = v.xy; o[4] = v.yz; o[5] = v.xz;
    }
}

// Elasticity3D::infinitesimalStrain_asVector (Elasticity.hh:587-612).
template <typename R>
PL_HD void el3d_strain_vector(PLB_POINT_ARGS(R), const R* x, int numConstants,
                              const R* constants, R* out) {
    const Sym<R> e = strain(&s_x[sOff_x[0]]);
    out[0] = e.xx; out[1] = e.yy; out[2] = e.zz; out[3] = e.xy; out[4] = e.yz; out[5] = e.xz;
}

// Cauchy stress as a vector (xx, yy, zz, xy, yz, xz) for output, basis order 0 derived field
// (Elasticity::stress_asVector, Elasticity.hh:441-456).
template <typename R>
PL_HD void sym_to_vector(const Sym<R>& t, R* out) {
    out[0] = t.xx; out[1] = t.yy; out[2] = t.zz; out[3] = t.xy; out[4] = t.yz; out[5] = t.xz;
}

// IsotropicLinearElasticity3D::cauchyStress_infinitesimalStrain_asVector
// (IsotropicLinearElasticity.hh:1243-1273): mean stress, then deviatoric stress.
template <typename R>
PL_HD void ile3d_stress_vector(PLB_POINT_ARGS(R), const R* x, int numConstants, const R* constants,
                               R* out) {
    const R mu = a[aOff[numA - 2]];
    const R K = a[aOff[numA - 1]];
    const Sym<R> e = strain(&s_x[sOff_x[0]]);
    Sym<R> sig = sym_zero<R>();
    add_mean_stress(K, e, &sig);
    add_dev_stress(mu, e, &sig);
    sym_to_vector(sig, out);
}

// IsotropicLinearGenMaxwell3D::cauchyStress_infinitesimalStrain_asVector
// (IsotropicLinearGenMaxwell.hh:1556-1589) through cauchyStress_stateVars (:340-357): the
// stored viscous strains enter as they are (no update with dt).
template <typename R>
PL_HD void gm3d_stress_vector(PLB_POINT_ARGS(R), const R* x, int numConstants, const R* constants,
                              R* out) {
    const R mu = a[aOff[numA - 6]];
    const R K = a[aOff[numA - 5]];
    const R* ratio = &a[aOff[numA - 3]];
    const R* visc = &a[aOff[numA - 2]];
    const Sym<R> e = strain(&s_x[sOff_x[0]]);
    Sym<R> sig = sym_zero<R>();
    add_mean_stress(K, e, &sig);
    Sym<R> v[3];
    for (int i = 0; i < 3; ++i) v[i] = sym_from_vector(&visc[6 * i]);
    const Sym<R> de = deviatoric(e);
    R r = R(1.0);
    for (int i = 0; i < 3; ++i) r -= ratio[i];
    const R mu_el = mu * r;
    sig.xx += R(2.0) * mu_el * de.xx;
    for (int i = 0; i < 3; ++i) sig.xx += R(2.0) * mu * ratio[i] * v[i].xx;
    sig.yy += R(2.0) * mu_el * de.yy;
    for (int i = 0; i < 3; ++i) sig.yy += R(2.0) * mu * ratio[i] * v[i].yy;
    sig.zz += R(2.0) * mu_el * de.zz;
    for (int i = 0; i < 3; ++i) sig.zz += R(2.0) * mu * ratio[i] * v[i].zz;
    sig.xy += R(2.0) * mu_el * de.xy;
    for (int i = 0; i < 3; ++i) sig.xy += R(2.0) * mu * ratio[i] * v[i].xy;
    sig.yz += R(2.0) * mu_el * de.yz;
    for (int i = 0; i < 3; ++i) sig.yz += R(2.0) * mu * ratio[i] * v[i].yz;
    sig.xz += R(2.0) * mu_el * de.xz;
    for (int i = 0; i < 3; ++i) sig.xz += R(2.0) * mu * ratio[i] * v[i].xz;
    sym_to_vector(sig, out);
}

// BoundaryDirections::tangential_directions and _unitCrossProduct
// (BoundaryDirections.hh:35-67, 248-270). The sign test on the second tangent repeats
// refDir2[1]*n[1], as the reference does.
template <typename R>
PL_HD void unit_cross(R* r, const R* a, const R* b) {
    r[0] = +a[1] * b[2] - a[2] * b[1];
    r[1] = +a[2] * b[0] - a[0] * b[2];
    r[2] = +a[0] * b[1] - a[1] * b[0];
    R mag = R(0.0);
    for (int i = 0; i < 3; ++i) mag += r[i] * r[i];
    mag = sqrt(mag);
    for (int i = 0; i < 3; ++i) r[i] /= mag;
}

template <typename R>
PL_HD void tangential_directions(R* t1, R* t2, const R* ref1, const R* ref2, const R* n) {
    R ref[3] = {ref1[0], ref1[1], ref1[2]};
    if (fabs(ref[0] * n[0] + ref[1] * n[1] + ref[2] * n[2]) > R(0.999)) {
        for (int i = 0; i < 3; ++i) ref[i] = ref2[i];
    }
    unit_cross(t1, ref, n);
    unit_cross(t2, n, t1);
    if (ref2[0] * n[0] + ref2[1] * n[1] + ref2[1] * n[1] < R(0.0)) {
        for (int i = 0; i < 3; ++i) t2[i] *= R(-1.0);
    }
}

// FaultCohesiveKin::f0u_neg / f0u_pos (FaultCohesiveKin.hh:74-150).
template <typename R>
PL_HD void fck_f0u_neg(PLB_POINT_ARGS(R), const R* x, const R* n, int numConstants,
                       const R* constants, R* f0) {
    const R* lam = &s[sOff[numS - 1]];
    for (int i = 0; i < 3; ++i) f0[i] += -lam[i];
}
template <typename R>
PL_HD void fck_f0u_pos(PLB_POINT_ARGS(R), const R* x, const R* n, int numConstants,
                       const R* constants, R* f0) {
    const R* lam = &s[sOff[numS - 1]];
    for (int i = 0; i < 3; ++i) f0[i] += +lam[i];
}

// FaultCohesiveKin::f0l_slip, 3D (FaultCohesiveKin.hh:158-225).
template <typename R>
PL_HD void fck_f0l_slip(PLB_POINT_ARGS(R), const R* x, const R* n, int numConstants,
                        const R* constants, R* f0) {
    const R* slip = &a[aOff[0]];
    const R* uN = &s[sOff[0]];
    const R* uP = &s[sOff[0] + 3];
    R t1[3], t2[3];
    tangential_directions(t1, t2, &constants[0], &constants[3], n);
    for (int i = 0; i < 3; ++i) {
        const R slip_xyz = n[i] * slip[0] + t1[i] * slip[1] + t2[i] * slip[2];
        f0[i] += uP[i] - uN[i] - slip_xyz;
    }
}

// FaultCohesiveKin::Jf0ul_neg / Jf0ul_pos / Jf0lu (FaultCohesiveKin.hh:298-412).
template <typename R>
PL_HD void fck_Jf0ul_neg(PLB_POINT_ARGS(R), R s_tshift, const R* x, const R* n,
                         int numConstants, const R* constants, R* Jf0) {
    for (int i = 0; i < 3; ++i) Jf0[i * 3 + i] += R(-1.0);
}
template <typename R>
PL_HD void fck_Jf0ul_pos(PLB_POINT_ARGS(R), R s_tshift, const R* x, const R* n,
                         int numConstants, const R* constants, R* Jf0) {
    for (int i = 0; i < 3; ++i) Jf0[i * 3 + i] += R(+1.0);
}
template <typename R>
PL_HD void fck_Jf0lu(PLB_POINT_ARGS(R), R s_tshift, const R* x, const R* n, int numConstants,
                     const R* constants, R* Jf0) {
    for (int i = 0; i < 3; ++i) {
        Jf0[i * 3 + i] += R(-1.0);
        Jf0[9 + i * 3 + i] += R(+1.0);
    }
}

}  // namespace pw
}  // namespace plb
