// Pointwise kernels known to the pylith_b200 device engine, declared with PyLith's names and
// PETSc's pointwise signatures (libsrc/pylith/fekernels/*.hh). Pass their addresses to the
// integrator registration calls exactly as PyLith passes them to PetscWeakForm; the engine
// maps each address to its device implementation. The host definitions compute the same
// pointwise values on the CPU (for callers that use them directly); the engine itself never
// runs them.
#pragma once

#include "../pylith_b200.h"

#define PYLITH_B200_POINT_ARGS                                                                 \
    const PylithInt dim, const PylithInt numS, const PylithInt numA, const PylithInt sOff[],  \
        const PylithInt sOff_x[], const PylithScalar s[], const PylithScalar s_t[],           \
        const PylithScalar s_x[], const PylithInt aOff[], const PylithInt aOff_x[],           \
        const PylithScalar a[], const PylithScalar a_t[], const PylithScalar a_x[],           \
        const PylithReal t
#define PYLITH_B200_POINTFN(name)                                                              \
    static void name(PYLITH_B200_POINT_ARGS, const PylithScalar x[], const PylithInt numConstants, \
                     const PylithScalar constants[], PylithScalar f[])
#define PYLITH_B200_JACFN(name)                                                                \
    static void name(PYLITH_B200_POINT_ARGS, const PylithReal s_tshift, const PylithScalar x[], \
                     const PylithInt numConstants, const PylithScalar constants[],            \
                     PylithScalar g[])
#define PYLITH_B200_BDPOINTFN(name)                                                            \
    static void name(PYLITH_B200_POINT_ARGS, const PylithScalar x[], const PylithReal n[],     \
                     const PylithInt numConstants, const PylithScalar constants[],            \
                     PylithScalar f[])
#define PYLITH_B200_BDJACFN(name)                                                              \
    static void name(PYLITH_B200_POINT_ARGS, const PylithReal s_tshift, const PylithScalar x[], \
                     const PylithReal n[], const PylithInt numConstants,                      \
                     const PylithScalar constants[], PylithScalar g[])

namespace pylith {
namespace fekernels {

// Elasticity.hh:300-334
struct Elasticity {
    PYLITH_B200_POINTFN(g0v_bodyforce);
};

// Elasticity.hh:587-612
struct Elasticity3D {
    PYLITH_B200_POINTFN(infinitesimalStrain_asVector);
};

// IsotropicLinearElasticity.hh:804-838, 891-1035, 1243-1273
struct IsotropicLinearElasticity3D {
    PYLITH_B200_POINTFN(f1v_infinitesimalStrain);
    PYLITH_B200_JACFN(Jf3vu_infinitesimalStrain);
    PYLITH_B200_POINTFN(cauchyStress_infinitesimalStrain_asVector);
};

// IsotropicLinearGenMaxwell.hh:1054-1087, 1143-1300, 1507-1549, 1556-1589
struct IsotropicLinearGenMaxwell3D {
    PYLITH_B200_POINTFN(f1v_infinitesimalStrain);
    PYLITH_B200_JACFN(Jf3vu_infinitesimalStrain);
    PYLITH_B200_POINTFN(viscousStrain_infinitesimalStrain_asVector);
    PYLITH_B200_POINTFN(cauchyStress_infinitesimalStrain_asVector);
};

// FaultCohesiveKin.hh:74-225, 298-412
struct FaultCohesiveKin {
    PYLITH_B200_BDPOINTFN(f0u_neg);
    PYLITH_B200_BDPOINTFN(f0u_pos);
    PYLITH_B200_BDPOINTFN(f0l_slip);
    PYLITH_B200_BDJACFN(Jf0ul_neg);
    PYLITH_B200_BDJACFN(Jf0ul_pos);
    PYLITH_B200_BDJACFN(Jf0lu);
};

}  // namespace fekernels
}  // namespace pylith
