// collide_math.cuh -- the pair test and impulse of the two-pass collision
// step (BHTree.cu:642-660), shared by the stand-alone neighbour search and
// the force walk with fused collisions, so both find the same pairs and
// round each impulse the same way.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace nb {

// Squared distance of a pair, one fixed rounding.
__device__ __forceinline__ float coll_dist2(float dx, float dy, float dz) {
  return fmaf(dz, dz, fmaf(dy, dy, __fmul_rn(dx, dx)));
}

// Adds to dv_i the impulse of source j at d = x_j - x_i (dist2 = coll_dist2(d),
// already known to be < r_coll^2), relative velocity v_j - v_i: with
// n = d / (|d| + 1e-10), dvn = (v_j - v_i) . n; when approaching (dvn < 0),
// dv_i -= (1 + e) dvn / 2 n.
__device__ __forceinline__ void coll_impulse(float dx, float dy, float dz, float dist2,
                                             float rvx, float rvy, float rvz, float e,
                                             float& dvx, float& dvy, float& dvz) {
  const float dist = sqrtf(dist2) + 1e-10f;
  const float nx = dx / dist, ny = dy / dist, nz = dz / dist;
  const float dvn = rvx * nx + rvy * ny + rvz * nz;
  if (dvn < 0.f) {
    const float J = -(1.f + e) * dvn * 0.5f;
    dvx += -J * nx;
    dvy += -J * ny;
    dvz += -J * nz;
  }
}

// A velocity component as the FP32 impulse uses it: the float value, the
// double rounded to float, or the hi word of a hi/lo pair (the conversions
// of the state's float read-out).
__device__ __forceinline__ float coll_vel(const void* p, int vtype, uint32_t i) {
  if (vtype == 1) return (float)__ldg((const double*)p + i);
  if (vtype == 2) return __ldg((const float2*)p + i).x;
  return __ldg((const float*)p + i);
}

}  // namespace nb
