// Cohesive-cell kernels: the device form of DMPlexCompute{Residual,Jacobian}HybridByKey for
// PyLith's FaultCohesiveKin (libsrc/pylith/feassemble/IntegratorInterface.cc:603-720,
// libsrc/pylith/fekernels/FaultCohesiveKin.hh).
//
// One thread per cohesive cell (a quadrilateral fault face with negative-side, positive-side
// and Lagrange-multiplier nodes). Face geometry and the normal come from the negative-side
// vertices at 2x2 Gauss points; the normal points from the negative to the positive side.
// At each point the solution is packed as PETSc packs a hybrid closure,
// s = [u-(3), u+(3), lambda(3)] with sOff = {0, 6}, and aux = slip(3).
#include "elements.cuh"
#include "internal.hpp"
#include "launch.hpp"
#include "pointwise.cuh"

namespace plb {

struct FacePt {
    double phi[4];
    double x[3];
    double n[3];
    double w;
};

PL_D void face_point(const double X[4][3], int q, FacePt* fp) {
    const int qi = q & 1, qj = q >> 1;
    const double xi = gauss2_x(qi), eta = gauss2_x(qj);
    const int ci[4] = {0, 1, 1, 0}, cj[4] = {0, 0, 1, 1};
    double dxi[3] = {0, 0, 0}, deta[3] = {0, 0, 0};
    fp->x[0] = fp->x[1] = fp->x[2] = 0.0;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        fp->phi[a] = lin_v(ci[a], xi) * lin_v(cj[a], eta);
        const double dx = lin_d(ci[a]) * lin_v(cj[a], eta);
        const double dy = lin_v(ci[a], xi) * lin_d(cj[a]);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            fp->x[d] += fp->phi[a] * X[a][d];
            dxi[d] += dx * X[a][d];
            deta[d] += dy * X[a][d];
        }
    }
    const double nn[3] = {dxi[1] * deta[2] - dxi[2] * deta[1], dxi[2] * deta[0] - dxi[0] * deta[2],
                          dxi[0] * deta[1] - dxi[1] * deta[0]};
    const double area = sqrt(nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2]);
#pragma unroll
    for (int d = 0; d < 3; ++d) fp->n[d] = nn[d] / area;
    fp->w = area;  // 2-point Gauss weights are 1
}

PL_D void call_face_residual(int k, const double* s, const double* a, const FacePt& fp,
                             const CohesiveParams& p, double* f0) {
    const int sOff[2] = {0, 6}, sOff_x[2] = {0, 0}, aOff[1] = {0};
    switch (k) {
        case K_FCK_F0U_NEG:
            pw::fck_f0u_neg<double>(3, 2, 1, sOff, sOff_x, s, nullptr, nullptr, aOff, nullptr, a,
                                    nullptr, nullptr, p.t, fp.x, fp.n, p.num_constants,
                                    p.constants, f0);
            break;
        case K_FCK_F0U_POS:
            pw::fck_f0u_pos<double>(3, 2, 1, sOff, sOff_x, s, nullptr, nullptr, aOff, nullptr, a,
                                    nullptr, nullptr, p.t, fp.x, fp.n, p.num_constants,
                                    p.constants, f0);
            break;
        case K_FCK_F0L_SLIP:
            pw::fck_f0l_slip<double>(3, 2, 1, sOff, sOff_x, s, nullptr, nullptr, aOff, nullptr, a,
                                     nullptr, nullptr, p.t, fp.x, fp.n, p.num_constants,
                                     p.constants, f0);
            break;
        default:
            break;
    }
}

// Pointwise Jacobian blocks for face k: g0 = 3x3 (Jf0ul_*) or two 3x3 blocks (Jf0lu).
PL_D void call_face_jacobian(int k, const FacePt& fp, const CohesiveParams& p, double* g0) {
    const int sOff[2] = {0, 6}, sOff_x[2] = {0, 0}, aOff[1] = {0};
    switch (k) {
        case K_FCK_JF0UL_NEG:
            pw::fck_Jf0ul_neg<double>(3, 2, 1, sOff, sOff_x, nullptr, nullptr, nullptr, aOff,
                                      nullptr, nullptr, nullptr, nullptr, p.t, p.s_tshift, fp.x,
                                      fp.n, p.num_constants, p.constants, g0);
            break;
        case K_FCK_JF0UL_POS:
            pw::fck_Jf0ul_pos<double>(3, 2, 1, sOff, sOff_x, nullptr, nullptr, nullptr, aOff,
                                      nullptr, nullptr, nullptr, nullptr, p.t, p.s_tshift, fp.x,
                                      fp.n, p.num_constants, p.constants, g0);
            break;
        case K_FCK_JF0LU:
            pw::fck_Jf0lu<double>(3, 2, 1, sOff, sOff_x, nullptr, nullptr, nullptr, aOff, nullptr,
                                  nullptr, nullptr, nullptr, p.t, p.s_tshift, fp.x, fp.n,
                                  p.num_constants, p.constants, g0);
            break;
        default:
            break;
    }
}

PL_D void load_face(const CohesiveParams& p, const int32_t* cc, double X[4][3]) {
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int d = 0; d < 3; ++d) X[a][d] = p.coords[3 * (int64_t)cc[a] + d];
}

__global__ void __launch_bounds__(128) k_cohesive_residual(CohesiveParams p) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < p.ncoh;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int32_t* cc = p.coh + 12 * c;
        double X[4][3];
        load_face(p, cc, X);
        double U[12][3];  // u- (4), u+ (4), lambda (4)
        double S[4][3];
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                U[k][d] = p.u[3 * (int64_t)cc[k] + d];
                U[4 + k][d] = p.u[3 * (int64_t)cc[4 + k] + d];
                U[8 + k][d] = p.u[p.lag_offset + 3 * (int64_t)cc[8 + k] + d];
                S[k][d] = p.slip[3 * (int64_t)cc[8 + k] + d];
            }
        double acc[3][12];
#pragma unroll
        for (int f = 0; f < 3; ++f)
#pragma unroll
            for (int i = 0; i < 12; ++i) acc[f][i] = 0.0;
#pragma unroll 1
        for (int q = 0; q < 4; ++q) {
            FacePt fp;
            face_point(X, q, &fp);
            double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, a[3] = {0, 0, 0};
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    s[d] += fp.phi[k] * U[k][d];
                    s[3 + d] += fp.phi[k] * U[4 + k][d];
                    s[6 + d] += fp.phi[k] * U[8 + k][d];
                    a[d] += fp.phi[k] * S[k][d];
                }
#pragma unroll
            for (int f = 0; f < 3; ++f) {
                if (p.kr[f] == K_NONE) continue;
                double f0[3] = {0, 0, 0};
                call_face_residual(p.kr[f], s, a, fp, p, f0);
#pragma unroll
                for (int k = 0; k < 4; ++k)
#pragma unroll
                    for (int d = 0; d < 3; ++d) acc[f][k * 3 + d] += fp.w * fp.phi[k] * f0[d];
            }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                if (p.kr[0] != K_NONE) red_add(&p.out[3 * (int64_t)cc[k] + d], acc[0][k * 3 + d]);
                if (p.kr[1] != K_NONE) red_add(&p.out[3 * (int64_t)cc[4 + k] + d], acc[1][k * 3 + d]);
                if (p.kr[2] != K_NONE)
                    red_add(&p.out[p.lag_offset + 3 * (int64_t)cc[8 + k] + d], acc[2][k * 3 + d]);
            }
    }
}

// Jacobian action of the cohesive blocks: u- rows take Jf0ul_neg * v_lambda, u+ rows
// Jf0ul_pos * v_lambda, lambda rows Jf0lu * [v-, v+].
template <typename T>
__global__ void __launch_bounds__(128) k_cohesive_jv(CohesiveParams p, const T* v, T* out) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < p.ncoh;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int32_t* cc = p.coh + 12 * c;
        double X[4][3];
        load_face(p, cc, X);
        T V[12][3];
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                V[k][d] = v[3 * (int64_t)cc[k] + d];
                V[4 + k][d] = v[3 * (int64_t)cc[4 + k] + d];
                V[8 + k][d] = v[p.lag_offset + 3 * (int64_t)cc[8 + k] + d];
            }
        T acc[3][12];
#pragma unroll
        for (int f = 0; f < 3; ++f)
#pragma unroll
            for (int i = 0; i < 12; ++i) acc[f][i] = T(0);
#pragma unroll 1
        for (int q = 0; q < 4; ++q) {
            FacePt fp;
            face_point(X, q, &fp);
            T vl[3] = {0, 0, 0}, vn[3] = {0, 0, 0}, vp[3] = {0, 0, 0};
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    vn[d] += T(fp.phi[k]) * V[k][d];
                    vp[d] += T(fp.phi[k]) * V[4 + k][d];
                    vl[d] += T(fp.phi[k]) * V[8 + k][d];
                }
#pragma unroll
            for (int f = 0; f < 3; ++f) {
                if (p.kj[f] == K_NONE) continue;
                double g0[18];
#pragma unroll
                for (int i = 0; i < 18; ++i) g0[i] = 0.0;
                call_face_jacobian(p.kj[f], fp, p, g0);
                T r[3];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    if (f < 2) {
                        r[i] = T(g0[i * 3 + 0]) * vl[0] + T(g0[i * 3 + 1]) * vl[1] + T(g0[i * 3 + 2]) * vl[2];
                    } else {
                        r[i] = T(g0[i * 3 + 0]) * vn[0] + T(g0[i * 3 + 1]) * vn[1] + T(g0[i * 3 + 2]) * vn[2] +
                               T(g0[9 + i * 3 + 0]) * vp[0] + T(g0[9 + i * 3 + 1]) * vp[1] +
                               T(g0[9 + i * 3 + 2]) * vp[2];
                    }
                }
#pragma unroll
                for (int k = 0; k < 4; ++k)
#pragma unroll
                    for (int d = 0; d < 3; ++d) acc[f][k * 3 + d] += T(fp.w * fp.phi[k]) * r[d];
            }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                if (p.kj[0] != K_NONE) red_add(&out[3 * (int64_t)cc[k] + d], acc[0][k * 3 + d]);
                if (p.kj[1] != K_NONE) red_add(&out[3 * (int64_t)cc[4 + k] + d], acc[1][k * 3 + d]);
                if (p.kj[2] != K_NONE)
                    red_add(&out[p.lag_offset + 3 * (int64_t)cc[8 + k] + d], acc[2][k * 3 + d]);
            }
    }
}

// Cohesive element blocks into the 3x3-block CSR matrix. pos[c][blk][a][b] holds the block
// index for blk = 0 (u-_a, lambda_b), 1 (u+_a, lambda_b), 2 (lambda_a, u-_b),
// 3 (lambda_a, u+_b).
__global__ void __launch_bounds__(128) k_cohesive_jacobian(CohesiveParams p, const int32_t* pos,
                                                           double* vals) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < p.ncoh;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int32_t* cc = p.coh + 12 * c;
        double X[4][3];
        load_face(p, cc, X);
        const int32_t* cpos = pos + 64 * c;
#pragma unroll 1
        for (int q = 0; q < 4; ++q) {
            FacePt fp;
            face_point(X, q, &fp);
#pragma unroll 1
            for (int f = 0; f < 3; ++f) {
                if (p.kj[f] == K_NONE) continue;
                double g0[18];
#pragma unroll
                for (int i = 0; i < 18; ++i) g0[i] = 0.0;
                call_face_jacobian(p.kj[f], fp, p, g0);
#pragma unroll 1
                for (int a = 0; a < 4; ++a)
#pragma unroll 1
                    for (int b = 0; b < 4; ++b) {
                        const double w = fp.w * fp.phi[a] * fp.phi[b];
                        if (f < 2) {
                            double* blk = vals + 9 * (int64_t)cpos[(f * 4 + a) * 4 + b];
                            for (int i = 0; i < 9; ++i) red_add(&blk[i], w * g0[i]);
                        } else {
                            double* bn = vals + 9 * (int64_t)cpos[(2 * 4 + a) * 4 + b];
                            double* bp = vals + 9 * (int64_t)cpos[(3 * 4 + a) * 4 + b];
                            for (int i = 0; i < 9; ++i) {
                                red_add(&bn[i], w * g0[i]);
                                red_add(&bp[i], w * g0[9 + i]);
                            }
                        }
                    }
            }
        }
    }
}

static int grid_coh(int64_t n) {
    const int64_t b = (n + 127) / 128;
    return (int)(b < 148 * 32 ? (b > 0 ? b : 1) : 148 * 32);
}

void launch_cohesive_residual(const CohesiveParams& p, cudaStream_t s) {
    if (p.ncoh == 0) return;
    k_cohesive_residual<<<grid_coh(p.ncoh), 128, 0, s>>>(p);
    count_launch();
}

void launch_cohesive_jv(const CohesiveParams& p, cudaStream_t s) {
    if (p.ncoh == 0) return;
    k_cohesive_jv<double><<<grid_coh(p.ncoh), 128, 0, s>>>(p, p.v, p.out);
    count_launch();
}

void launch_cohesive_jv_f32(const CohesiveParams& p, cudaStream_t s) {
    if (p.ncoh == 0) return;
    k_cohesive_jv<float><<<grid_coh(p.ncoh), 128, 0, s>>>(p, p.v32, p.out32);
    count_launch();
}

void launch_cohesive_jacobian(const CohesiveParams& p, const int32_t* pos, double* vals,
                              cudaStream_t s) {
    if (p.ncoh == 0) return;
    k_cohesive_jacobian<<<grid_coh(p.ncoh), 128, 0, s>>>(p, pos, vals);
    count_launch();
}

}  // namespace plb
