// C++ use of the integrator API (include/pylith_b200/feassemble.hh) the way PyLith's material
// code registers kernels: by the addresses of the pylith::fekernels functions. Builds a small
// hex box, registers isotropic linear elasticity, and checks on the GPU that
//   * the residual of a linear displacement field vanishes at interior nodes (MMS uniform
//     strain, tests/mmstests/linearelasticity/nofaults-3d/UniformStrain3D.cc), and
//   * the Jacobian action reproduces the residual (the residual is linear: F(u) = J u).
// Exit status 0 on success.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <vector>

#include "pylith_b200/feassemble.hh"

namespace fk = pylith::fekernels;
using pylith::feassemble::Integrator;
using pylith::feassemble::IntegratorDomain;

int main() {
    const int n = 4;
    const int nn = (n + 1) * (n + 1) * (n + 1);
    std::vector<double> X(3 * nn);
    for (int k = 0; k <= n; ++k)
        for (int j = 0; j <= n; ++j)
            for (int i = 0; i <= n; ++i) {
                const int id = i + (n + 1) * (j + (n + 1) * k);
                X[3 * id] = -6000.0 + 12000.0 * i / n;
                X[3 * id + 1] = -6000.0 + 12000.0 * j / n;
                X[3 * id + 2] = -9000.0 + 9000.0 * k / n;
            }
    const int corner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    std::vector<int32_t> cells;
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i)
                for (auto& c : corner) cells.push_back((i + c[0]) + (n + 1) * ((j + c[1]) + (n + 1) * (k + c[2])));
    const int nc = n * n * n;
    pl_context ctx = nullptr;
    pylith_b200::check(pl_context_create(0, &ctx));
    pl_mesh mesh = nullptr;
    pylith_b200::check(pl_mesh_create(ctx, PL_CELL_HEX8, nc, cells.data(), nn, X.data(), &mesh));
    int status = 0;
    {
        IntegratorDomain ig(mesh);
        std::vector<double> rho(nc, 2500.0), mu(nc, 2.25e10), K(nc, 4.0e10);
        ig.setAuxiliarySubfield("density", PL_AUX_PER_CELL, 1, rho.data());
        ig.setAuxiliarySubfield("shear_modulus", PL_AUX_PER_CELL, 1, mu.data());
        ig.setAuxiliarySubfield("bulk_modulus", PL_AUX_PER_CELL, 1, K.data());
        ig.setKernelsResidual({IntegratorDomain::ResidualKernels(
            "displacement", Integrator::LHS, nullptr, fk::IsotropicLinearElasticity3D::f1v_infinitesimalStrain)});
        ig.setKernelsJacobian({IntegratorDomain::JacobianKernels(
            "displacement", "displacement", Integrator::LHS, nullptr, nullptr, nullptr,
            fk::IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain)});
        std::vector<double> u(3 * nn);
        for (int i = 0; i < nn; ++i) {
            u[3 * i] = 1e-4 * X[3 * i] + 2e-5 * X[3 * i + 1];
            u[3 * i + 1] = -1e-4 * X[3 * i + 1] + 3e-5 * X[3 * i + 2];
            u[3 * i + 2] = 5e-5 * X[3 * i + 2] - 2e-5 * X[3 * i];
        }
        double *du, *dr, *djv;
        cudaMalloc(&du, 8 * u.size());
        cudaMalloc(&dr, 8 * u.size());
        cudaMalloc(&djv, 8 * u.size());
        cudaMemcpy(du, u.data(), 8 * u.size(), cudaMemcpyHostToDevice);
        cudaMemset(dr, 0, 8 * u.size());
        cudaMemset(djv, 0, 8 * u.size());
        cudaDeviceSynchronize();
        Integrator::IntegrationData d;
        d.solution = du;
        ig.computeLHSResidual(dr, d);
        ig.computeLHSJacobianAction(du, djv, d);
        pylith_b200::check(pl_context_synchronize(ctx));
        std::vector<double> r(u.size()), jv(u.size());
        cudaMemcpy(r.data(), dr, 8 * r.size(), cudaMemcpyDeviceToHost);
        cudaMemcpy(jv.data(), djv, 8 * jv.size(), cudaMemcpyDeviceToHost);
        double scale = 0.0, interior = 0.0, diff = 0.0;
        for (size_t i = 0; i < r.size(); ++i) {
            scale = std::fmax(scale, std::fabs(r[i]));
            diff = std::fmax(diff, std::fabs(r[i] - jv[i]));
        }
        for (int k = 1; k < n; ++k)
            for (int j = 1; j < n; ++j)
                for (int i = 1; i < n; ++i) {
                    const int id = i + (n + 1) * (j + (n + 1) * k);
                    for (int c = 0; c < 3; ++c) interior = std::fmax(interior, std::fabs(r[3 * id + c]));
                }
        std::printf("residual scale %.3e interior %.3e |F(u) - J u| %.3e\n", scale, interior, diff);
        if (!(interior <= 1e-12 * scale) || !(diff <= 1e-12 * scale)) status = 1;
        // an unknown pointwise function is rejected, not run on the CPU
        try {
            ig.setKernelsResidual({IntegratorDomain::ResidualKernels(
                "displacement", Integrator::LHS, nullptr, (PetscPointFn)&std::printf)});
            status = 1;
        } catch (const pylith_b200::Error& e) {
            if (e.code != PL_ERR_UNKNOWN_KERNEL) status = 1;
        }
        cudaFree(du);
        cudaFree(dr);
        cudaFree(djv);
    }
    pl_mesh_destroy(mesh);
    pl_context_destroy(ctx);
    std::printf(status == 0 ? "ok\n" : "FAILED\n");
    return status;
}
