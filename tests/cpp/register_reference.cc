// Registers the reference's own pointwise kernels -- compiled here from PyLith's
// libsrc/pylith/fekernels/*.hh, as a PyLith material or fault compiles them -- with the engine
// through the C ABI (pl_fekernel_register), and checks that a function computing something else
// is refused. Registration runs on the host only, so this program needs no GPU.
#include <cstdio>
#include <cstring>

#include "pylith/fekernels/Elasticity.hh"
#include "pylith/fekernels/FaultCohesiveKin.hh"
#include "pylith/fekernels/IsotropicLinearElasticity.hh"
#include "pylith/fekernels/IsotropicLinearGenMaxwell.hh"
#include "pylith_b200.h"

namespace fk = pylith::fekernels;

struct Kernel {
    const char* name;
    const void* fn;
};

int main() {
    const Kernel kernels[] = {
        {"Elasticity::g0v_bodyforce", (const void*)&fk::Elasticity::g0v_bodyforce},
        {"Elasticity3D::infinitesimalStrain_asVector", (const void*)&fk::Elasticity3D::infinitesimalStrain_asVector},
        {"IsotropicLinearElasticity3D::f1v_infinitesimalStrain",
         (const void*)&fk::IsotropicLinearElasticity3D::f1v_infinitesimalStrain},
        {"IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain",
         (const void*)&fk::IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain},
        {"IsotropicLinearElasticity3D::cauchyStress_infinitesimalStrain_asVector",
         (const void*)&fk::IsotropicLinearElasticity3D::cauchyStress_infinitesimalStrain_asVector},
        {"IsotropicLinearGenMaxwell3D::f1v_infinitesimalStrain",
         (const void*)&fk::IsotropicLinearGenMaxwell3D::f1v_infinitesimalStrain},
        {"IsotropicLinearGenMaxwell3D::Jf3vu_infinitesimalStrain",
         (const void*)&fk::IsotropicLinearGenMaxwell3D::Jf3vu_infinitesimalStrain},
        {"IsotropicLinearGenMaxwell3D::viscousStrain_infinitesimalStrain_asVector",
         (const void*)&fk::IsotropicLinearGenMaxwell3D::viscousStrain_infinitesimalStrain_asVector},
        {"IsotropicLinearGenMaxwell3D::cauchyStress_infinitesimalStrain_asVector",
         (const void*)&fk::IsotropicLinearGenMaxwell3D::cauchyStress_infinitesimalStrain_asVector},
        {"FaultCohesiveKin::f0u_neg", (const void*)&fk::FaultCohesiveKin::f0u_neg},
        {"FaultCohesiveKin::f0u_pos", (const void*)&fk::FaultCohesiveKin::f0u_pos},
        {"FaultCohesiveKin::f0l_slip", (const void*)&fk::FaultCohesiveKin::f0l_slip},
        {"FaultCohesiveKin::Jf0ul_neg", (const void*)&fk::FaultCohesiveKin::Jf0ul_neg},
        {"FaultCohesiveKin::Jf0ul_pos", (const void*)&fk::FaultCohesiveKin::Jf0ul_pos},
        {"FaultCohesiveKin::Jf0lu", (const void*)&fk::FaultCohesiveKin::Jf0lu},
    };
    int failures = 0;
    for (const Kernel& k : kernels) {
        const int rc = pl_fekernel_register(k.name, k.fn);
        const char* back = pl_fekernel_name(k.fn);
        if (rc != PL_OK || !back || std::strcmp(back, k.name) != 0) {
            std::printf("FAIL %s: rc %d (%s)\n", k.name, rc, pl_last_error());
            ++failures;
        }
    }
    // a kernel registered under a name whose computation it does not perform is refused
    // (gravity's g0 = density * gravity registered as the body-force g0 = body force)
    const int wrong = pl_fekernel_register("Elasticity::g0v_bodyforce", (const void*)&fk::Elasticity::g0v_grav);
    if (wrong != PL_ERR_UNKNOWN_KERNEL) {
        std::printf("FAIL: a mismatched kernel was accepted (rc %d)\n", wrong);
        ++failures;
    }
    // a name without a device implementation is refused
    if (pl_fekernel_register("IsotropicLinearElasticity3D::f1v_infinitesimalStrain_refState",
                             (const void*)&fk::IsotropicLinearElasticity3D::f1v_infinitesimalStrain_refState) !=
        PL_ERR_UNKNOWN_KERNEL) {
        std::printf("FAIL: a kernel without a device implementation was accepted\n");
        ++failures;
    }
    if (failures == 0) std::printf("ok: %d reference kernels registered\n", (int)(sizeof(kernels) / sizeof(kernels[0])));
    return failures == 0 ? 0 : 1;
}
