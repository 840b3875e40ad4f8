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

// A target's accelerations as pairs: .x sums the even-indexed sources of a
// list, .y the odd-indexed ones, added together once the walk is done.
struct PairAcc {
  float2 x, y, z;
};

// A target's negated coordinates, each in both halves of a pair.
struct PairTgt {
  float2 x, y, z;
};

// interact() on two sources at once in packed FP32 (f32x2, sm_100): the same
// operations in the same order on each half, so each interaction rounds as
// interact() rounds it (s + (-p) is s - p exactly).  sx .. sm hold the two
// sources' coordinates and masses.  Returns the two softened r^2.
template <bool kSoft>
__device__ __forceinline__ float2 interact2(const float2 sx, const float2 sy, const float2 sz,
                                            const float2 sm, const PairTgt& p, const float2 e2,
                                            PairAcc& acc) {
  const float2 dx = __fadd2_rn(sx, p.x), dy = __fadd2_rn(sy, p.y), dz = __fadd2_rn(sz, p.z);
  const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, e2)));
  float2 inv = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
  if (!kSoft) {
    inv.x = (r2.x > 0.f) ? inv.x : 0.f;
    inv.y = (r2.y > 0.f) ? inv.y : 0.f;
  }
  const float2 f = __fmul2_rn(sm, __fmul2_rn(__fmul2_rn(inv, inv), inv));
  acc.x = __ffma2_rn(f, dx, acc.x);
  acc.y = __ffma2_rn(f, dy, acc.y);
  acc.z = __ffma2_rn(f, dz, acc.z);
  return r2;
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

// interact_vjp() on two sources (or two targets) at once in packed FP32,
// added into acc: acc += m_s (lam r^-3 - 3 d (d . lam) r^-5), pair half by
// pair half.  p holds the negated target coordinates, sx .. sm the sources'
// coordinates and masses (a mass of 0 drops its half), lx .. lz the
// adjoints.
template <bool kSoft>
__device__ __forceinline__ void interact_vjp2(const float2 sx, const float2 sy, const float2 sz,
                                              const float2 sm, const PairTgt& p, const float2 e2,
                                              const float2 lx, const float2 ly, const float2 lz,
                                              PairAcc& acc) {
  const float2 dx = __fadd2_rn(sx, p.x), dy = __fadd2_rn(sy, p.y), dz = __fadd2_rn(sz, p.z);
  const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, e2)));
  float2 inv = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
  if (!kSoft) {
    inv.x = (r2.x > 0.f) ? inv.x : 0.f;
    inv.y = (r2.y > 0.f) ? inv.y : 0.f;
  }
  const float2 inv2 = __fmul2_rn(inv, inv);
  const float2 f = __fmul2_rn(sm, __fmul2_rn(inv2, inv));
  const float2 dl = __ffma2_rn(dx, lx, __ffma2_rn(dy, ly, __fmul2_rn(dz, lz)));
  const float2 nt = __fmul2_rn(__fmul2_rn(make_float2(-3.f, -3.f), dl), inv2);
  acc.x = __ffma2_rn(f, __ffma2_rn(nt, dx, lx), acc.x);
  acc.y = __ffma2_rn(f, __ffma2_rn(nt, dy, ly), acc.y);
  acc.z = __ffma2_rn(f, __ffma2_rn(nt, dz, lz), acc.z);
}

}  // namespace nb
