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
// Every lane of the warp calls it (valid = false for lanes without a key).
// Lanes whose digit equals the previous lane's join that lane's run, and the
// first lane of each run adds the run's length in one atomic: the keys come
// nearly sorted, so their high digits form a few long runs.  Equal digits in
// separate runs each add their own run (one count per key either way).
template <typename K>
__device__ __forceinline__ void hist_add(uint32_t (*s_h)[kHistBins], K key, bool valid,
                                         int passes) {
  const int lane = threadIdx.x & 31;
  const unsigned above = ~((2u << lane) - 1u);  // lanes after this one (none for lane 31)
  for (int p = 0; p < passes; ++p) {
    const uint32_t d = valid ? (uint32_t)(key >> (8 * p)) & 0xffu : (uint32_t)kHistBins;
    const uint32_t prev = __shfl_up_sync(kFull, d, 1);
    const unsigned heads = __ballot_sync(kFull, lane == 0 || d != prev);
    if (valid && ((heads >> lane) & 1u)) {
      const unsigned later = heads & above;
      const int next = later ? __ffs(later) - 1 : 32;
      atomicAdd(&s_h[p][d], (uint32_t)(next - lane));
    }
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
