// Host definitions of the registered pointwise kernels and the address -> device-kernel
// registry. The bodies run the same pointwise code the device kernels inline
// (pointwise.cuh); the registry compares addresses. A caller's own compiled copy of a kernel (the
// address PyLith itself hands to PetscWeakFormAddResidual, IntegratorDomain.cc:145,183) joins the
// registry through pl_fekernel_register, after it has computed what the named kernel computes on
// a set of probe inputs; the engine then runs its device implementation of that name.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/pylith_b200/fekernels.hh"
#include "internal.hpp"
#include "pointwise.cuh"

#define ARGS dim, numS, numA, sOff, sOff_x, s, s_t, s_x, aOff, aOff_x, a, a_t, a_x, t

namespace fk = pylith::fekernels;

void fk::Elasticity::g0v_bodyforce(PYLITH_B200_POINT_ARGS, const PylithScalar x[],
                                   const PylithInt numConstants, const PylithScalar constants[],
                                   PylithScalar f[]) {
    plb::pw::g0v_bodyforce<double>(ARGS, x, numConstants, constants, f);
}
void fk::Elasticity3D::infinitesimalStrain_asVector(PYLITH_B200_POINT_ARGS, const PylithScalar x[],
                                                    const PylithInt numConstants,
                                                    const PylithScalar constants[], PylithScalar f[]) {
    plb::pw::el3d_strain_vector<double>(ARGS, x, numConstants, constants, f);
}
void fk::IsotropicLinearElasticity3D::f1v_infinitesimalStrain(PYLITH_B200_POINT_ARGS,
                                                              const PylithScalar x[],
                                                              const PylithInt numConstants,
                                                              const PylithScalar constants[],
                                                              PylithScalar f[]) {
    plb::pw::ile3d_f1v<double>(ARGS, x, numConstants, constants, f);
}
void fk::IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain(
    PYLITH_B200_POINT_ARGS, const PylithReal s_tshift, const PylithScalar x[],
    const PylithInt numConstants, const PylithScalar constants[], PylithScalar g[]) {
    plb::pw::ile3d_Jf3vu<double>(ARGS, s_tshift, x, numConstants, constants, g);
}
void fk::IsotropicLinearGenMaxwell3D::f1v_infinitesimalStrain(PYLITH_B200_POINT_ARGS,
                                                              const PylithScalar x[],
                                                              const PylithInt numConstants,
                                                              const PylithScalar constants[],
                                                              PylithScalar f[]) {
    plb::pw::gm3d_f1v<double>(ARGS, x, numConstants, constants, f);
}
void fk::IsotropicLinearGenMaxwell3D::Jf3vu_infinitesimalStrain(
    PYLITH_B200_POINT_ARGS, const PylithReal s_tshift, const PylithScalar x[],
    const PylithInt numConstants, const PylithScalar constants[], PylithScalar g[]) {
    plb::pw::gm3d_Jf3vu<double>(ARGS, s_tshift, x, numConstants, constants, g);
}
void fk::IsotropicLinearGenMaxwell3D::viscousStrain_infinitesimalStrain_asVector(
    PYLITH_B200_POINT_ARGS, const PylithScalar x[], const PylithInt numConstants,
    const PylithScalar constants[], PylithScalar f[]) {
    plb::pw::gm3d_viscous_strain<double>(ARGS, x, numConstants, constants, f);
}
void fk::IsotropicLinearElasticity3D::cauchyStress_infinitesimalStrain_asVector(
    PYLITH_B200_POINT_ARGS, const PylithScalar x[], const PylithInt numConstants,
    const PylithScalar constants[], PylithScalar f[]) {
    plb::pw::ile3d_stress_vector<double>(ARGS, x, numConstants, constants, f);
}
void fk::IsotropicLinearGenMaxwell3D::cauchyStress_infinitesimalStrain_asVector(
    PYLITH_B200_POINT_ARGS, const PylithScalar x[], const PylithInt numConstants,
    const PylithScalar constants[], PylithScalar f[]) {
    plb::pw::gm3d_stress_vector<double>(ARGS, x, numConstants, constants, f);
}
void fk::FaultCohesiveKin::f0u_neg(PYLITH_B200_POINT_ARGS, const PylithScalar x[],
                                   const PylithReal n[], const PylithInt numConstants,
                                   const PylithScalar constants[], PylithScalar f[]) {
    plb::pw::fck_f0u_neg<double>(ARGS, x, n, numConstants, constants, f);
}
void fk::FaultCohesiveKin::f0u_pos(PYLITH_B200_POINT_ARGS, const PylithScalar x[],
                                   const PylithReal n[], const PylithInt numConstants,
                                   const PylithScalar constants[], PylithScalar f[]) {
    plb::pw::fck_f0u_pos<double>(ARGS, x, n, numConstants, constants, f);
}
void fk::FaultCohesiveKin::f0l_slip(PYLITH_B200_POINT_ARGS, const PylithScalar x[],
                                    const PylithReal n[], const PylithInt numConstants,
                                    const PylithScalar constants[], PylithScalar f[]) {
    plb::pw::fck_f0l_slip<double>(ARGS, x, n, numConstants, constants, f);
}
void fk::FaultCohesiveKin::Jf0ul_neg(PYLITH_B200_POINT_ARGS, const PylithReal s_tshift,
                                     const PylithScalar x[], const PylithReal n[],
                                     const PylithInt numConstants, const PylithScalar constants[],
                                     PylithScalar g[]) {
    plb::pw::fck_Jf0ul_neg<double>(ARGS, s_tshift, x, n, numConstants, constants, g);
}
void fk::FaultCohesiveKin::Jf0ul_pos(PYLITH_B200_POINT_ARGS, const PylithReal s_tshift,
                                     const PylithScalar x[], const PylithReal n[],
                                     const PylithInt numConstants, const PylithScalar constants[],
                                     PylithScalar g[]) {
    plb::pw::fck_Jf0ul_pos<double>(ARGS, s_tshift, x, n, numConstants, constants, g);
}
void fk::FaultCohesiveKin::Jf0lu(PYLITH_B200_POINT_ARGS, const PylithReal s_tshift,
                                 const PylithScalar x[], const PylithReal n[],
                                 const PylithInt numConstants, const PylithScalar constants[],
                                 PylithScalar g[]) {
    plb::pw::fck_Jf0lu<double>(ARGS, s_tshift, x, n, numConstants, constants, g);
}

namespace {
// Argument layout a registered kernel is probed with: the aux subfields, solution fields and
// constants its family reads (indexed as the reference kernels index them).
enum Family { F_ELASTIC, F_BODYFORCE, F_GENMAXWELL, F_FAULT };
enum Kind { POINT, JAC, BDPOINT, BDJAC };

struct Entry {
    const char* name;
    const void* fn;
    plb::KernelId id;
    Kind kind;
    Family family;
};

const Entry kRegistry[] = {
    {"Elasticity::g0v_bodyforce", (const void*)&fk::Elasticity::g0v_bodyforce, plb::K_G0V_BODYFORCE, POINT,
     F_BODYFORCE},
    {"IsotropicLinearElasticity3D::f1v_infinitesimalStrain",
     (const void*)&fk::IsotropicLinearElasticity3D::f1v_infinitesimalStrain, plb::K_ILE_F1V, POINT, F_ELASTIC},
    {"IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain",
     (const void*)&fk::IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain, plb::K_ILE_JF3VU, JAC, F_ELASTIC},
    {"IsotropicLinearGenMaxwell3D::f1v_infinitesimalStrain",
     (const void*)&fk::IsotropicLinearGenMaxwell3D::f1v_infinitesimalStrain, plb::K_GM_F1V, POINT, F_GENMAXWELL},
    {"IsotropicLinearGenMaxwell3D::Jf3vu_infinitesimalStrain",
     (const void*)&fk::IsotropicLinearGenMaxwell3D::Jf3vu_infinitesimalStrain, plb::K_GM_JF3VU, JAC, F_GENMAXWELL},
    {"IsotropicLinearGenMaxwell3D::viscousStrain_infinitesimalStrain_asVector",
     (const void*)&fk::IsotropicLinearGenMaxwell3D::viscousStrain_infinitesimalStrain_asVector,
     plb::K_GM_VISCOUS_STRAIN, POINT, F_GENMAXWELL},
    {"Elasticity3D::infinitesimalStrain_asVector",
     (const void*)&fk::Elasticity3D::infinitesimalStrain_asVector, plb::K_EL_STRAIN_VECTOR, POINT, F_ELASTIC},
    {"IsotropicLinearElasticity3D::cauchyStress_infinitesimalStrain_asVector",
     (const void*)&fk::IsotropicLinearElasticity3D::cauchyStress_infinitesimalStrain_asVector, plb::K_ILE_STRESS_VECTOR,
     POINT, F_ELASTIC},
    {"IsotropicLinearGenMaxwell3D::cauchyStress_infinitesimalStrain_asVector",
     (const void*)&fk::IsotropicLinearGenMaxwell3D::cauchyStress_infinitesimalStrain_asVector, plb::K_GM_STRESS_VECTOR,
     POINT, F_GENMAXWELL},
    {"FaultCohesiveKin::f0u_neg", (const void*)&fk::FaultCohesiveKin::f0u_neg, plb::K_FCK_F0U_NEG, BDPOINT, F_FAULT},
    {"FaultCohesiveKin::f0u_pos", (const void*)&fk::FaultCohesiveKin::f0u_pos, plb::K_FCK_F0U_POS, BDPOINT, F_FAULT},
    {"FaultCohesiveKin::f0l_slip", (const void*)&fk::FaultCohesiveKin::f0l_slip, plb::K_FCK_F0L_SLIP, BDPOINT, F_FAULT},
    {"FaultCohesiveKin::Jf0ul_neg", (const void*)&fk::FaultCohesiveKin::Jf0ul_neg, plb::K_FCK_JF0UL_NEG, BDJAC, F_FAULT},
    {"FaultCohesiveKin::Jf0ul_pos", (const void*)&fk::FaultCohesiveKin::Jf0ul_pos, plb::K_FCK_JF0UL_POS, BDJAC, F_FAULT},
    {"FaultCohesiveKin::Jf0lu", (const void*)&fk::FaultCohesiveKin::Jf0lu, plb::K_FCK_JF0LU, BDJAC, F_FAULT},
};

// Addresses registered by callers (pl_fekernel_register), each with the entry it stands for.
std::mutex g_reg_mutex;
std::vector<std::pair<const void*, const Entry*>> g_registered;

const Entry* entry_by_name(const char* name) {
    for (const Entry& e : kRegistry)
        if (std::strcmp(e.name, name) == 0) return &e;
    return nullptr;
}

uint64_t mix(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double uniform(uint64_t& x) { return (double)(mix(x) >> 11) * (1.0 / 9007199254740992.0); }  // [0, 1)

// Calls kernel `fn` of `kind` on probe case `k` of family `fam`; out has 128 zeroed entries.
void probe_call(const void* fn, Kind kind, Family fam, int k, double* out) {
    uint64_t seed = 0x5EEDull + 977ull * (uint64_t)k;
    double s[12], s_t[12] = {0}, s_x[36], a[40], a_t[40] = {0}, a_x[120] = {0}, x[3], n[3], c[6];
    for (double& v : s) v = 2.0 * uniform(seed) - 1.0;
    for (double& v : s_x) v = (2.0 * uniform(seed) - 1.0) * 1e-3;
    for (double& v : x) v = (2.0 * uniform(seed) - 1.0) * 4000.0;
    double nn = 0.0;
    for (double& v : n) nn += (v = 2.0 * uniform(seed) - 1.0) * v;
    for (double& v : n) v /= std::sqrt(nn);
    PylithInt numS = 1, numA = 3, nc = 0;
    PylithInt sOff[2] = {0, 6}, sOff_x[2] = {0, 18}, aOff[7] = {0, 1, 2, 3, 6, 9, 27}, aOff_x[7] = {0};
    a[0] = 2500.0;
    a[1] = 3e10 * (0.5 + uniform(seed));
    a[2] = 5e10 * (0.5 + uniform(seed));
    switch (fam) {
        case F_ELASTIC: break;
        case F_BODYFORCE:
            numA = 2;
            for (int i = 1; i < 4; ++i) a[i] = 2.0 * uniform(seed) - 1.0;
            break;
        case F_GENMAXWELL:
            numA = 7;
            for (int i = 3; i < 6; ++i) a[i] = 1.0 + 9.0 * uniform(seed);
            for (int i = 6; i < 9; ++i) a[i] = 0.1 + 0.2 * uniform(seed);
            for (int i = 9; i < 33; ++i) a[i] = (2.0 * uniform(seed) - 1.0) * 1e-4;
            c[0] = 0.1 + 1.9 * uniform(seed);
            nc = 1;
            break;
        case F_FAULT:
            numS = 2;
            numA = 1;
            for (int i = 0; i < 3; ++i) a[i] = 2.0 * uniform(seed) - 1.0;
            c[0] = 0.0, c[1] = 0.0, c[2] = 1.0;
            c[3] = 2.0 * uniform(seed) - 1.0, c[4] = 2.0 * uniform(seed) - 1.0, c[5] = 2.0 * uniform(seed) - 1.0;
            nc = 6;
            break;
    }
    const double t = 0.25, shift = 0.0;
    switch (kind) {
        case POINT:
            ((PetscPointFn)fn)(3, numS, numA, sOff, sOff_x, s, s_t, s_x, aOff, aOff_x, a, a_t, a_x, t, x, nc, c, out);
            break;
        case JAC:
            ((PetscPointJacFn)fn)(3, numS, numA, sOff, sOff_x, s, s_t, s_x, aOff, aOff_x, a, a_t, a_x, t, shift, x, nc,
                                  c, out);
            break;
        case BDPOINT:
            ((PetscBdPointFn)fn)(3, numS, numA, sOff, sOff_x, s, s_t, s_x, aOff, aOff_x, a, a_t, a_x, t, x, n, nc, c,
                                 out);
            break;
        case BDJAC:
            ((PetscBdPointJacFn)fn)(3, numS, numA, sOff, sOff_x, s, s_t, s_x, aOff, aOff_x, a, a_t, a_x, t, shift, x,
                                    n, nc, c, out);
            break;
    }
}

// True when `fn` computes what `e` computes on 8 probe cases (relative 1e-12: the caller's
// compiler may contract multiply-adds differently).
bool computes_the_same(const Entry& e, const void* fn) {
    for (int k = 0; k < 8; ++k) {
        double want[128] = {0}, got[128] = {0};
        probe_call(e.fn, e.kind, e.family, k, want);
        probe_call(fn, e.kind, e.family, k, got);
        double scale = 0.0;
        for (double v : want) scale = std::max(scale, std::fabs(v));
        for (int i = 0; i < 128; ++i)
            if (!(std::fabs(got[i] - want[i]) <= 1e-12 * scale)) return false;
    }
    return true;
}
}  // namespace

plb::KernelId plb::lookup_kernel(const void* fn) {
    if (!fn) return K_NONE;
    for (const Entry& e : kRegistry)
        if (e.fn == fn) return e.id;
    std::lock_guard<std::mutex> lock(g_reg_mutex);
    for (const auto& r : g_registered)
        if (r.first == fn) return r.second->id;
    return (KernelId)-1;
}

extern "C" void* pl_fekernel_lookup(const char* name) {
    if (!name) return nullptr;
    const Entry* e = entry_by_name(name);
    return e ? const_cast<void*>(e->fn) : nullptr;
}

extern "C" int pl_fekernel_register(const char* name, const void* fn) {
    if (!name || !fn) return plb::fail(PL_ERR_INVALID_ARG, "pl_fekernel_register: null name or function");
    const Entry* e = entry_by_name(name);
    if (!e) return plb::fail(PL_ERR_UNKNOWN_KERNEL, std::string("no device implementation of ") + name);
    if (fn == e->fn) return PL_OK;
    {
        std::lock_guard<std::mutex> lock(g_reg_mutex);
        for (const auto& r : g_registered)
            if (r.first == fn) {
                if (r.second == e) return PL_OK;
                return plb::fail(PL_ERR_INVALID_ARG, std::string("address already registered as ") + r.second->name);
            }
    }
    for (const Entry& o : kRegistry)
        if (o.fn == fn) return plb::fail(PL_ERR_INVALID_ARG, std::string("address is the library's ") + o.name);
    if (!computes_the_same(*e, fn))
        return plb::fail(PL_ERR_UNKNOWN_KERNEL,
                         std::string("the function does not compute ") + name + " on the registration probes");
    std::lock_guard<std::mutex> lock(g_reg_mutex);
    g_registered.emplace_back(fn, e);
    return PL_OK;
}

extern "C" const char* pl_fekernel_name(const void* fn) {
    if (!fn) return nullptr;
    for (const Entry& e : kRegistry)
        if (e.fn == fn) return e.name;
    std::lock_guard<std::mutex> lock(g_reg_mutex);
    for (const auto& r : g_registered)
        if (r.first == fn) return r.second->name;
    return nullptr;
}
