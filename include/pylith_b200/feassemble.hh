// C++ integrator API over the pylith_b200 C ABI, with PyLith's class and method names
// (libsrc/pylith/feassemble/IntegratorDomain.hh:25-86, IntegratorInterface.hh:31-120,
// Integrator.hh:26-59,164-200). Header-only: a PyLith build that links libpylith_b200.so can
// keep its material and fault code (which builds ResidualKernels/JacobianKernels/ProjectKernels
// records from pylith::fekernels function pointers) and route the compute calls here.
// Errors from the C ABI are thrown as pylith_b200::Error (PyLith reports PETSc errors as C++
// exceptions the same way, libsrc/pylith/exceptions/error.hh:33-44).
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "../pylith_b200.h"
#include "fekernels.hh"

namespace pylith_b200 {

class Error : public std::runtime_error {
public:
    Error(int code, const std::string& msg) : std::runtime_error(msg), code(code) {}
    int code;
};

inline void check(int rc) {
    if (rc != PL_OK) throw Error(rc, std::string(pl_error_string(rc)) + ": " + pl_last_error());
}

}  // namespace pylith_b200

namespace pylith {
namespace feassemble {

class Integrator {
public:
    enum EquationPart { LHS = PL_LHS, RHS = PL_RHS, LHS_LUMPED_INV = PL_LHS_LUMPED_INV, LHS_WEIGHTED = PL_LHS_WEIGHTED };

    // Data of one compute call (IntegrationData.hh:26-38 keys used on this path).
    struct IntegrationData {
        double time = 0.0;
        double time_step = 0.0;
        double s_tshift = 0.0;
        const double* solution = nullptr;      // device local vector
        const double* solution_dot = nullptr;  // device local vector or nullptr
    };

    explicit Integrator(pl_integrator h) : _h(h) {}
    virtual ~Integrator() { pl_integrator_destroy(_h); }
    Integrator(const Integrator&) = delete;
    Integrator& operator=(const Integrator&) = delete;

    pl_integrator handle() const { return _h; }

    void setAuxiliarySubfield(const char* name, int storage, int ncomp, const double* hostValues) {
        pylith_b200::check(pl_integrator_set_aux(_h, name, storage, ncomp, hostValues));
    }

    // Integrator::_setKernelConstants (Integrator.cc:264-290)
    void setKernelConstants(const std::vector<double>& constants) {
        pylith_b200::check(pl_integrator_set_constants(_h, (int)constants.size(), constants.data()));
    }

    // computeLHSResidual: ADD into `residual` (a device local vector the caller zeroed), as the
    // reference's integrators add into TimeDependent's zeroed local residual.
    void computeLHSResidual(double* residual, const IntegrationData& d) {
        pylith_b200::check(pl_compute_lhs_residual(_h, d.time, d.time_step, d.solution, d.solution_dot, residual, PL_ADD));
    }

    void computeLHSJacobian(pl_matrix jacobian, const IntegrationData& d) {
        pylith_b200::check(pl_compute_lhs_jacobian(_h, d.time, d.time_step, d.s_tshift, d.solution, jacobian));
    }

    void computeLHSJacobianAction(const double* v, double* jv, const IntegrationData& d) {
        pylith_b200::check(pl_compute_lhs_jacobian_action(_h, d.time, d.time_step, d.s_tshift, d.solution, v, jv, PL_ADD));
    }

protected:
    pl_integrator _h;
};

class IntegratorDomain : public Integrator {
public:
    struct ResidualKernels {
        std::string subfield;
        EquationPart part;
        PetscPointFn r0;
        PetscPointFn r1;
        ResidualKernels(const char* s = "", EquationPart p = LHS, PetscPointFn a = nullptr, PetscPointFn b = nullptr)
            : subfield(s), part(p), r0(a), r1(b) {}
    };
    struct JacobianKernels {
        std::string subfieldTrial, subfieldBasis;
        EquationPart part;
        PetscPointJacFn j0, j1, j2, j3;
        JacobianKernels(const char* t = "", const char* b = "", EquationPart p = LHS, PetscPointJacFn a = nullptr,
                        PetscPointJacFn c = nullptr, PetscPointJacFn d = nullptr, PetscPointJacFn e = nullptr)
            : subfieldTrial(t), subfieldBasis(b), part(p), j0(a), j1(c), j2(d), j3(e) {}
    };
    struct ProjectKernels {
        std::string subfield;
        PetscPointFn f;
        ProjectKernels(const char* s = "", PetscPointFn fn = nullptr) : subfield(s), f(fn) {}
    };

    static pl_integrator create(pl_mesh mesh, const std::vector<int32_t>& cells) {
        pl_integrator h = nullptr;
        pylith_b200::check(pl_integrator_domain_create(mesh, (int64_t)cells.size(), cells.empty() ? nullptr : cells.data(), &h));
        return h;
    }
    explicit IntegratorDomain(pl_mesh mesh, const std::vector<int32_t>& cells = {}) : Integrator(create(mesh, cells)) {}

    // IntegratorDomain::setKernelsResidual (IntegratorDomain.cc:135-167)
    void setKernelsResidual(const std::vector<ResidualKernels>& kernels) {
        std::vector<pl_residual_kernels> k;
        for (const auto& r : kernels) k.push_back({r.subfield.c_str(), (int)r.part, r.r0, r.r1});
        pylith_b200::check(pl_integrator_set_kernels_residual(_h, k.data(), (int)k.size()));
    }

    // IntegratorDomain::setKernelsJacobian (IntegratorDomain.cc:172-205)
    void setKernelsJacobian(const std::vector<JacobianKernels>& kernels) {
        std::vector<pl_jacobian_kernels> k;
        for (const auto& j : kernels)
            k.push_back({j.subfieldTrial.c_str(), j.subfieldBasis.c_str(), (int)j.part, j.j0, j.j1, j.j2, j.j3});
        pylith_b200::check(pl_integrator_set_kernels_jacobian(_h, k.data(), (int)k.size()));
    }

    // IntegratorDomain::setKernelsUpdateStateVars (IntegratorDomain.cc:221-228)
    void setKernelsUpdateStateVars(const std::vector<ProjectKernels>& kernels) {
        std::vector<pl_project_kernels> k;
        for (const auto& p : kernels) k.push_back({p.subfield.c_str(), p.f});
        pylith_b200::check(pl_integrator_set_kernels_update_state_vars(_h, k.data(), (int)k.size()));
    }

    // IntegratorDomain::_updateStateVars (IntegratorDomain.cc:555-590)
    void updateStateVars(const IntegrationData& d) {
        pylith_b200::check(pl_update_state_vars(_h, d.time, d.time_step, d.solution));
    }
};

class IntegratorInterface : public Integrator {
public:
    enum FaceEnum { NEGATIVE_FACE = PL_FACE_NEGATIVE, POSITIVE_FACE = PL_FACE_POSITIVE, FAULT_FACE = PL_FACE_FAULT };

    struct ResidualKernels {
        std::string subfield;
        EquationPart part;
        FaceEnum face;
        PetscBdPointFn r0;
        PetscBdPointFn r1;
        ResidualKernels(const char* s = "", EquationPart p = LHS, FaceEnum f = FAULT_FACE, PetscBdPointFn a = nullptr,
                        PetscBdPointFn b = nullptr)
            : subfield(s), part(p), face(f), r0(a), r1(b) {}
    };
    struct JacobianKernels {
        std::string subfieldTrial, subfieldBasis;
        EquationPart part;
        FaceEnum face;
        PetscBdPointJacFn j0, j1, j2, j3;
        JacobianKernels(const char* t = "", const char* b = "", EquationPart p = LHS, FaceEnum f = FAULT_FACE,
                        PetscBdPointJacFn a = nullptr, PetscBdPointJacFn c = nullptr, PetscBdPointJacFn d = nullptr,
                        PetscBdPointJacFn e = nullptr)
            : subfieldTrial(t), subfieldBasis(b), part(p), face(f), j0(a), j1(c), j2(d), j3(e) {}
    };

    static pl_integrator create(pl_mesh mesh) {
        pl_integrator h = nullptr;
        pylith_b200::check(pl_integrator_interface_create(mesh, &h));
        return h;
    }
    explicit IntegratorInterface(pl_mesh mesh) : Integrator(create(mesh)) {}

    // IntegratorInterface::setKernels (IntegratorInterface.cc:243-310)
    void setKernels(const std::vector<ResidualKernels>& residual, const std::vector<JacobianKernels>& jacobian) {
        std::vector<pl_interface_residual_kernels> r;
        for (const auto& k : residual) r.push_back({k.subfield.c_str(), (int)k.part, (int)k.face, k.r0, k.r1});
        pylith_b200::check(pl_integrator_interface_set_kernels_residual(_h, r.data(), (int)r.size()));
        std::vector<pl_interface_jacobian_kernels> j;
        for (const auto& k : jacobian)
            j.push_back({k.subfieldTrial.c_str(), k.subfieldBasis.c_str(), (int)k.part, (int)k.face, k.j0, k.j1, k.j2, k.j3});
        pylith_b200::check(pl_integrator_interface_set_kernels_jacobian(_h, j.data(), (int)j.size()));
    }
};

}  // namespace feassemble
}  // namespace pylith
