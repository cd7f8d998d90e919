// Shared device helpers for the pylith_b200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define PL_HD __host__ __device__ __forceinline__
#define PL_D __device__ __forceinline__

namespace plb {

// Material model (rheology) selected by the registered f1/Jf3 kernels.
enum Rheology { RHEO_NONE = 0, RHEO_ILE = 1, RHEO_GENMAXWELL = 2 };

// Device-side check codes, OR-ed into the context's error word and returned to the host
// as PL_ERR_DEVICE_CHECK after the next synchronisation.
enum DeviceCheck : unsigned int {
    CHECK_NONPOSITIVE_DETJ = 1u << 0,
    CHECK_INDEX_RANGE = 1u << 1,
    CHECK_NONFINITE = 1u << 2,
};

PL_D void flag_error(unsigned int* err, unsigned int code) {
    if (err) atomicOr(err, code);
}

// Reduction into global memory without a return value (red.global.add).
// CG step length rz / pq for the SPD operator: 0 when pq <= 0 or the step is not a finite float
// (a search direction that collapsed to rounding noise in FP32 iterations past convergence).
PL_D float safe_step_f32(double rz, double pq) {
    const float a = pq > 0.0 ? (float)(rz / pq) : 0.0f;
    return isfinite(a) ? a : 0.0f;
}

PL_D void red_add(double* p, double v) { atomicAdd(p, v); }
PL_D void red_add(float* p, float v) { atomicAdd(p, v); }

}  // namespace plb
