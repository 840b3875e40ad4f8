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

// One moment tile is kMomentTile bodies, scanned by kMomentThreads threads
// holding two consecutive bodies each.
constexpr int kMomentThreads = 1024;
static_assert(kMomentTile == 2 * kMomentThreads, "two bodies per thread");
static_assert(kMomentThreads % 32 == 0 && kMomentThreads <= 1024, "one warp scans the warp sums");

__device__ __forceinline__ double4 d4shfl_up(double4 v, int o) {
  return make_double4(__shfl_up_sync(0xffffffffu, v.x, o), __shfl_up_sync(0xffffffffu, v.y, o),
                      __shfl_up_sync(0xffffffffu, v.z, o), __shfl_up_sync(0xffffffffu, v.w, o));
}

__device__ __forceinline__ double4 d4warp_incl_scan(double4 v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double4 t = d4shfl_up(v, o);
    if (lane >= o) v = d4add(v, t);
  }
  return v;
}

// Moment value (m, m x, m y, m z) of one body.
__device__ __forceinline__ double4 body_moment(double m, double x, double y, double z) {
  return make_double4(m, m * x, m * y, m * z);
}

// The tile-local exclusive prefix of tile blockIdx.x: thread t of the block
// (kMomentThreads threads) passes the moments v0, v1 of bodies base, base + 1
// (base = tile start + 2 t; zero past n).  Writes ploc[i] for i <= n of the
// tile (index n gets the tile's local prefix at n) and the tile's sum.
__device__ __forceinline__ void moment_tile_scan(double4 v0, double4 v1, long long base, int n,
                                                 double4* __restrict__ ploc,
                                                 double4* __restrict__ tile_sum) {
  __shared__ double4 s_w[kMomentThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double4 sum = d4add(v0, v1);
  const double4 inc = d4warp_incl_scan(sum, lane);
  if (lane == 31) s_w[warp] = inc;
  __syncthreads();
  if (warp == 0) {  // exclusive prefix of the warp sums (kMomentThreads / 32 <= 32 of them)
    constexpr int kWarps = kMomentThreads / 32;
    const double4 x = (lane < kWarps) ? s_w[lane] : make_double4(0, 0, 0, 0);
    const double4 y = d4warp_incl_scan(x, lane);
    __syncwarp();
    if (lane < kWarps) s_w[lane] = d4sub(y, x);
  }
  __syncthreads();
  double4 run = d4add(s_w[warp], d4sub(inc, sum));
  if (base <= n) ploc[base] = run;
  run = d4add(run, v0);
  if (base + 1 <= n) ploc[base + 1] = run;
  run = d4add(run, v1);
  if (tid == kMomentThreads - 1) tile_sum[blockIdx.x] = run;
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
