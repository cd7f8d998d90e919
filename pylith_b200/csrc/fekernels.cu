// Host definitions of the registered pointwise kernels and the address -> device-kernel
// registry. The bodies run the same pointwise code the device kernels inline
// (pointwise.cuh); the registry only compares addresses.
#include <cstring>

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
struct Entry {
    const char* name;
    const void* fn;
    plb::KernelId id;
};

const Entry kRegistry[] = {
    {"Elasticity::g0v_bodyforce", (const void*)&fk::Elasticity::g0v_bodyforce, plb::K_G0V_BODYFORCE},
    {"IsotropicLinearElasticity3D::f1v_infinitesimalStrain",
     (const void*)&fk::IsotropicLinearElasticity3D::f1v_infinitesimalStrain, plb::K_ILE_F1V},
    {"IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain",
     (const void*)&fk::IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain, plb::K_ILE_JF3VU},
    {"IsotropicLinearGenMaxwell3D::f1v_infinitesimalStrain",
     (const void*)&fk::IsotropicLinearGenMaxwell3D::f1v_infinitesimalStrain, plb::K_GM_F1V},
    {"IsotropicLinearGenMaxwell3D::Jf3vu_infinitesimalStrain",
     (const void*)&fk::IsotropicLinearGenMaxwell3D::Jf3vu_infinitesimalStrain, plb::K_GM_JF3VU},
    {"IsotropicLinearGenMaxwell3D::viscousStrain_infinitesimalStrain_asVector",
     (const void*)&fk::IsotropicLinearGenMaxwell3D::viscousStrain_infinitesimalStrain_asVector,
     plb::K_GM_VISCOUS_STRAIN},
    {"Elasticity3D::infinitesimalStrain_asVector",
     (const void*)&fk::Elasticity3D::infinitesimalStrain_asVector, plb::K_EL_STRAIN_VECTOR},
    {"IsotropicLinearElasticity3D::cauchyStress_infinitesimalStrain_asVector",
     (const void*)&fk::IsotropicLinearElasticity3D::cauchyStress_infinitesimalStrain_asVector, plb::K_ILE_STRESS_VECTOR},
    {"IsotropicLinearGenMaxwell3D::cauchyStress_infinitesimalStrain_asVector",
     (const void*)&fk::IsotropicLinearGenMaxwell3D::cauchyStress_infinitesimalStrain_asVector, plb::K_GM_STRESS_VECTOR},
    {"FaultCohesiveKin::f0u_neg", (const void*)&fk::FaultCohesiveKin::f0u_neg, plb::K_FCK_F0U_NEG},
    {"FaultCohesiveKin::f0u_pos", (const void*)&fk::FaultCohesiveKin::f0u_pos, plb::K_FCK_F0U_POS},
    {"FaultCohesiveKin::f0l_slip", (const void*)&fk::FaultCohesiveKin::f0l_slip, plb::K_FCK_F0L_SLIP},
    {"FaultCohesiveKin::Jf0ul_neg", (const void*)&fk::FaultCohesiveKin::Jf0ul_neg, plb::K_FCK_JF0UL_NEG},
    {"FaultCohesiveKin::Jf0ul_pos", (const void*)&fk::FaultCohesiveKin::Jf0ul_pos, plb::K_FCK_JF0UL_POS},
    {"FaultCohesiveKin::Jf0lu", (const void*)&fk::FaultCohesiveKin::Jf0lu, plb::K_FCK_JF0LU},
};
}  // namespace

plb::KernelId plb::lookup_kernel(const void* fn) {
    if (!fn) return K_NONE;
    for (const Entry& e : kRegistry)
        if (e.fn == fn) return e.id;
    return (KernelId)-1;
}

extern "C" void* pl_fekernel_lookup(const char* name) {
    if (!name) return nullptr;
    for (const Entry& e : kRegistry)
        if (std::strcmp(e.name, name) == 0) return const_cast<void*>(e.fn);
    return nullptr;
}
