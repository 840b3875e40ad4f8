// moments.cuh -- FP64 moment prefix sums shared by the octree emit and the
// tape replay: a node's (m, m x, m y, m z) over its sorted body range
// [lo, end) is two differences of tile-local prefix sums, and its centre of
// mass is rounded to float the same way wherever it is needed, so a replayed
// interaction sees the very float4 the recorded walk saw.
#pragma once
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace nb {

__device__ __forceinline__ double4 d4add(double4 a, double4 b) {
  return make_double4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}
__device__ __forceinline__ double4 d4sub(double4 a, double4 b) {
  return make_double4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
}

// Moments of sorted bodies [lo, end): ploc holds tile-local exclusive prefix
// sums (index i: sum over [tile start, i)), tpre the exclusive prefix of the
// tile sums.
__device__ __forceinline__ double4 range_moments(const double4* __restrict__ ploc,
                                                 const double4* __restrict__ tpre, int lo,
                                                 int end) {
  double4 r = d4sub(ploc[end], ploc[lo]);
  const int t0 = lo / kMomentTile, t1 = end / kMomentTile;
  if (t0 != t1) r = d4add(r, d4sub(tpre[t1], tpre[t0]));
  return r;
}

// Float centre of mass and mass of a moment sum (fallback: the given point).
__device__ __forceinline__ float4 com_of(double4 s, float cx, float cy, float cz) {
  if (s.x > 0.0) {
    const double inv = 1.0 / s.x;
    return make_float4((float)(s.y * inv), (float)(s.z * inv), (float)(s.w * inv), (float)s.x);
  }
  return make_float4(cx, cy, cz, 0.f);
}

}  // namespace nb
