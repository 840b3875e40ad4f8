// walk_math.cuh -- the per-interaction arithmetic of the force walk, shared
// by the tree walk and the tape replays so that a replayed interaction
// rounds exactly as the recorded one did.
#pragma once
#include <cuda_runtime.h>

namespace nb {

// 1/sqrt(x) by the hardware approximation (rsqrt.approx, ~2^-22 relative),
// with subnormal inputs and results flushed to zero: r^2 >= eps^2 or a
// squared distance between distinct bodies is never subnormal here, and the
// flush spares the range fix-up the non-flushing form needs.
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// acc += m_s (s - p) / (|s - p|^2 + eps^2)^{3/2}  (s.w = m_s; FP32, FMA form)
template <bool kSoft>
__device__ __forceinline__ void interact(const float4 s, const float4 p, float eps2,
                                         float3& acc) {
  float dx = s.x - p.x, dy = s.y - p.y, dz = s.z - p.z;
  float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
  float inv = rsqrt_ftz(r2);
  if (!kSoft) inv = (r2 > 0.f) ? inv : 0.f;
  float f = s.w * (inv * inv * inv);
  acc.x = fmaf(f, dx, acc.x);
  acc.y = fmaf(f, dy, acc.y);
  acc.z = fmaf(f, dz, acc.z);
}

// Vector-Jacobian product of one interaction: with d = s - p and
// K(d) = d / (|d|^2 + eps^2)^{3/2}, returns g = m_s (dK/dd) lam
//   = m_s (lam r^-3 - 3 d (d . lam) r^-5),   r^2 = |d|^2 + eps^2.
// The target's position adjoint receives -g, the source's +g.
template <bool kSoft>
__device__ __forceinline__ float3 interact_vjp(const float4 s, const float4 p, float eps2,
                                               const float3 lam) {
  float dx = s.x - p.x, dy = s.y - p.y, dz = s.z - p.z;
  float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
  float inv = rsqrt_ftz(r2);
  if (!kSoft) inv = (r2 > 0.f) ? inv : 0.f;
  const float inv2 = inv * inv;
  const float f = s.w * (inv2 * inv);
  const float dl = fmaf(dx, lam.x, fmaf(dy, lam.y, dz * lam.z));
  const float t = 3.f * dl * inv2;
  return make_float3(f * fmaf(-t, dx, lam.x), f * fmaf(-t, dy, lam.y), f * fmaf(-t, dz, lam.z));
}

}  // namespace nb
