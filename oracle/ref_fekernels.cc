// Test infrastructure only (never linked into the product library).
//
// Exposes the reference's own pointwise kernels, compiled unchanged from the
// PyLith sources (libsrc/pylith/fekernels/*.hh), under plain C symbol names so
// that the oracle's cell loop and the tests can call them through PETSc-style
// function pointers, exactly as PETSc's DMPlexComputeResidual calls them.
//
// Built by oracle/Makefile into oracle/_ref/libref_fekernels.so from the
// reference tree; nothing of the reference is copied into this repository.
#include "pylith/fekernels/IsotropicLinearElasticity.hh"
#include "pylith/fekernels/IsotropicLinearGenMaxwell.hh"
#include "pylith/fekernels/FaultCohesiveKin.hh"
#include "pylith/fekernels/BoundaryDirections.hh"
#include "pylith/fekernels/Elasticity.hh"

namespace fk = pylith::fekernels;

#define PL_POINT_ARGS                                                                    \
    const PylithInt dim, const PylithInt numS, const PylithInt numA, const PylithInt sOff[], \
    const PylithInt sOff_x[], const PylithScalar s[], const PylithScalar s_t[],            \
    const PylithScalar s_x[], const PylithInt aOff[], const PylithInt aOff_x[],            \
    const PylithScalar a[], const PylithScalar a_t[], const PylithScalar a_x[],            \
    const PylithReal t
#define PL_POINT_PASS dim, numS, numA, sOff, sOff_x, s, s_t, s_x, aOff, aOff_x, a, a_t, a_x, t

#define REF_POINT(cname, qualified)                                                         \
    extern "C" void cname(PL_POINT_ARGS, const PylithScalar x[], const PylithInt numConstants, \
                          const PylithScalar constants[], PylithScalar f[]) {               \
        qualified(PL_POINT_PASS, x, numConstants, constants, f);                            \
    }
#define REF_JAC(cname, qualified)                                                           \
    extern "C" void cname(PL_POINT_ARGS, const PylithReal s_tshift, const PylithScalar x[],  \
                          const PylithInt numConstants, const PylithScalar constants[],     \
                          PylithScalar g[]) {                                               \
        qualified(PL_POINT_PASS, s_tshift, x, numConstants, constants, g);                  \
    }
#define REF_BD_POINT(cname, qualified)                                                      \
    extern "C" void cname(PL_POINT_ARGS, const PylithScalar x[], const PylithReal n[],       \
                          const PylithInt numConstants, const PylithScalar constants[],     \
                          PylithScalar f[]) {                                               \
        qualified(PL_POINT_PASS, x, n, numConstants, constants, f);                         \
    }
#define REF_BD_JAC(cname, qualified)                                                        \
    extern "C" void cname(PL_POINT_ARGS, const PylithReal s_tshift, const PylithScalar x[],  \
                          const PylithReal n[], const PylithInt numConstants,               \
                          const PylithScalar constants[], PylithScalar g[]) {               \
        qualified(PL_POINT_PASS, s_tshift, x, n, numConstants, constants, g);               \
    }

REF_POINT(ref_Elasticity_g0v_bodyforce, fk::Elasticity::g0v_bodyforce)
REF_POINT(ref_IsotropicLinearElasticity3D_f1v_infinitesimalStrain,
          fk::IsotropicLinearElasticity3D::f1v_infinitesimalStrain)
REF_JAC(ref_IsotropicLinearElasticity3D_Jf3vu_infinitesimalStrain,
        fk::IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain)
REF_POINT(ref_IsotropicLinearGenMaxwell3D_f1v_infinitesimalStrain,
          fk::IsotropicLinearGenMaxwell3D::f1v_infinitesimalStrain)
REF_JAC(ref_IsotropicLinearGenMaxwell3D_Jf3vu_infinitesimalStrain,
        fk::IsotropicLinearGenMaxwell3D::Jf3vu_infinitesimalStrain)
REF_POINT(ref_IsotropicLinearGenMaxwell3D_viscousStrain_infinitesimalStrain_asVector,
          fk::IsotropicLinearGenMaxwell3D::viscousStrain_infinitesimalStrain_asVector)
REF_POINT(ref_Elasticity3D_infinitesimalStrain_asVector,
          fk::Elasticity3D::infinitesimalStrain_asVector)
REF_POINT(ref_IsotropicLinearElasticity3D_cauchyStress_infinitesimalStrain_asVector,
          fk::IsotropicLinearElasticity3D::cauchyStress_infinitesimalStrain_asVector)
REF_POINT(ref_IsotropicLinearGenMaxwell3D_cauchyStress_infinitesimalStrain_asVector,
          fk::IsotropicLinearGenMaxwell3D::cauchyStress_infinitesimalStrain_asVector)
REF_BD_POINT(ref_FaultCohesiveKin_f0u_neg, fk::FaultCohesiveKin::f0u_neg)
REF_BD_POINT(ref_FaultCohesiveKin_f0u_pos, fk::FaultCohesiveKin::f0u_pos)
REF_BD_POINT(ref_FaultCohesiveKin_f0l_slip, fk::FaultCohesiveKin::f0l_slip)
REF_BD_JAC(ref_FaultCohesiveKin_Jf0ul_neg, fk::FaultCohesiveKin::Jf0ul_neg)
REF_BD_JAC(ref_FaultCohesiveKin_Jf0ul_pos, fk::FaultCohesiveKin::Jf0ul_pos)
REF_BD_JAC(ref_FaultCohesiveKin_Jf0lu, fk::FaultCohesiveKin::Jf0lu)

extern "C" void ref_BoundaryDirections_tangential_directions(double tanDir1[], double tanDir2[],
                                                             const double refDir1[],
                                                             const double refDir2[],
                                                             const double normalDir[]) {
    fk::BoundaryDirections::tangential_directions(tanDir1, tanDir2, refDir1, refDir2, normalDir);
}
