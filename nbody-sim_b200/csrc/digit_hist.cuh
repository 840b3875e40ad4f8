// digit_hist.cuh -- per-block digit histograms of radix-sort keys, shared by
// the sort's own histogram kernel and the key kernel that counts the digits
// of the keys it writes (one pass over the keys instead of two).
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace nb {

constexpr int kHistBins = 256;       // 8-bit digits
constexpr int kHistMaxPasses = 8;    // up to 64-bit keys

// Adds the digits of one key per lane to the block's histograms s_h[pass][d].
// Every lane of the warp calls it (valid = false for lanes without a key):
// lanes with equal digits are merged by __match_any_sync into one atomic,
// which matters for nearly sorted keys, whose high digits mostly agree.
template <typename K>
__device__ __forceinline__ void hist_add(uint32_t (*s_h)[kHistBins], K key, bool valid,
                                         int passes) {
  const int lane = threadIdx.x & 31;
  for (int p = 0; p < passes; ++p) {
    const uint32_t d = valid ? (uint32_t)(key >> (8 * p)) & 0xffu : (uint32_t)kHistBins;
    const unsigned peers = __match_any_sync(kFull, d);
    if (valid && lane == __ffs(peers) - 1) atomicAdd(&s_h[p][d], (uint32_t)__popc(peers));
  }
}

// Adds the block's histograms into the global ones (after a __syncthreads).
__device__ __forceinline__ void hist_flush(uint32_t (*s_h)[kHistBins], int passes,
                                           uint32_t* __restrict__ hist) {
  for (int i = threadIdx.x; i < passes * kHistBins; i += blockDim.x) {
    const uint32_t c = (&s_h[0][0])[i];
    if (c) atomicAdd(hist + i, c);
  }
}

}  // namespace nb
