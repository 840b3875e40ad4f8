// direct.cu -- FP64 direct-sum self-gravity: the accuracy yardstick of the
// tree walk and the pair potential of the softened energy.
//
// For each target i (a list, or every body):
//   a_i   =  sum_{j != i} m_j (x_j - x_i) / (|x_j - x_i|^2 + eps^2)^{3/2}
//   phi_i = -sum_{j != i} m_j / (|x_j - x_i|^2 + eps^2)^{1/2}
// in FP64 with a fixed source order (j ascending), so results are
// deterministic.  One thread per target; sources stream through shared
// memory in tiles of kTile bodies.  The softened star term of
// src/physics/BHTree.cu:547-553 is not included: callers add it in FP64.
#include <algorithm>

#include "capi_util.h"
#include "common.cuh"
#include "kernels.cuh"

namespace nb {
namespace {

constexpr int kThreadsD = 256;
constexpr int kTile = 256;

__global__ void __launch_bounds__(kThreadsD)
k_direct(const double* __restrict__ x, const double* __restrict__ y,
         const double* __restrict__ z, const float* __restrict__ m, int n,
         const int* __restrict__ targets, int nt, double eps2, double* __restrict__ ax,
         double* __restrict__ ay, double* __restrict__ az, double* __restrict__ phi) {
  __shared__ double4 src[kTile];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = t < nt;
  const int i = live ? (targets ? targets[t] : t) : -1;
  const double xi = live ? x[i] : 0.0, yi = live ? y[i] : 0.0, zi = live ? z[i] : 0.0;
  double sx = 0.0, sy = 0.0, sz = 0.0, sp = 0.0;
  for (int base = 0; base < n; base += kTile) {
    const int j = base + threadIdx.x;
    __syncthreads();
    src[threadIdx.x] = (j < n) ? make_double4(x[j], y[j], z[j], (double)m[j])
                               : make_double4(0.0, 0.0, 0.0, 0.0);
    __syncthreads();
    const int cnt = min(kTile, n - base);
    if (!live) continue;
#pragma unroll 4
    for (int k = 0; k < cnt; ++k) {
      const double4 s = src[k];
      const double dx = s.x - xi, dy = s.y - yi, dz = s.z - zi;
      const double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
      const double inv = (base + k == i) ? 0.0 : rsqrt(r2);
      const double minv = s.w * inv;
      const double f = minv * inv * inv;
      sx = fma(f, dx, sx);
      sy = fma(f, dy, sy);
      sz = fma(f, dz, sz);
      sp -= minv;
    }
  }
  if (live) {
    if (ax) ax[t] = sx;
    if (ay) ay[t] = sy;
    if (az) az[t] = sz;
    if (phi) phi[t] = sp;
  }
}

}  // namespace
}  // namespace nb

extern "C" int nbody_direct_f64(const double* x, const double* y, const double* z,
                                const float* mass, int n, const int* targets, int n_targets,
                                double eps, double* ax, double* ay, double* az, double* phi) {
  NBODY_API_BODY({
    NBODY_REQUIRE(x && y && z && mass, "nbody_direct_f64: null array");
    NBODY_REQUIRE(n >= 0, "nbody_direct_f64: negative n");
    const int nt = targets ? n_targets : n;
    NBODY_REQUIRE(nt >= 0, "nbody_direct_f64: negative target count");
    if (nt == 0 || n == 0) return NBODY_OK;
    nb::k_direct<<<nb::div_up(nt, nb::kThreadsD), nb::kThreadsD>>>(
        x, y, z, mass, n, targets, nt, eps * eps, ax, ay, az, phi);
    nb::check(cudaGetLastError(), "k_direct launch");
    nb::check(cudaDeviceSynchronize(), "k_direct");
  })
}

namespace {
template <typename K>
int radix_sort_api(K* keys, uint32_t* values, int n, int bits, const char* what) {
  NBODY_API_BODY({
    NBODY_REQUIRE(n >= 0, std::string(what) + ": negative n");
    NBODY_REQUIRE(bits >= 1 && bits <= 8 * (int)sizeof(K), std::string(what) + ": bad bit count");
    if (n <= 1) return NBODY_OK;
    NBODY_REQUIRE(keys && values, std::string(what) + ": null array");
    K* ka = nullptr;
    uint32_t *va = nullptr, *counts = nullptr;
    int* status = nullptr;
    auto release = [&]() {
      cudaFree(ka);
      cudaFree(va);
      cudaFree(counts);
      cudaFree(status);
    };
    try {
      nb::check(cudaMalloc(&ka, sizeof(K) * (size_t)n), "sort scratch");
      nb::check(cudaMalloc(&va, sizeof(uint32_t) * (size_t)n), "sort scratch");
      nb::check(cudaMalloc(&counts, sizeof(uint32_t) * nb::radix_sort_count_words(n)),
                "sort scratch");
      nb::check(cudaMalloc(&status, sizeof(int)), "sort status");
      nb::check(cudaMemset(status, 0, sizeof(int)), "sort status");
      nb::radix_sort_pairs<K>(keys, values, ka, va, counts, n, bits, 0, status);
      int st = 0;
      nb::check(cudaMemcpy(&st, status, sizeof(int), cudaMemcpyDeviceToHost), "sort status");
      if (st) throw nb::CudaError(std::string(what) + ": a look-back wait gave up");
    } catch (...) {
      release();
      throw;
    }
    release();
  })
}
}  // namespace

extern "C" int nbody_radix_sort_u32(uint32_t* keys, uint32_t* values, int n, int bits) {
  return radix_sort_api<uint32_t>(keys, values, n, bits, "nbody_radix_sort_u32");
}

extern "C" int nbody_radix_sort_u64(uint64_t* keys, uint32_t* values, int n, int bits) {
  return radix_sort_api<uint64_t>(keys, values, n, bits, "nbody_radix_sort_u64");
}

extern "C" int nbody_radix_tree_u32(const uint32_t* keys, int n, int key_bits, int* left,
                                    int* right, int* lo, int* hi, uint8_t* prefix) {
  NBODY_API_BODY({
    NBODY_REQUIRE(n >= 0, "nbody_radix_tree_u32: negative n");
    NBODY_REQUIRE(key_bits >= 1 && key_bits <= 32, "nbody_radix_tree_u32: bad bit count");
    if (n < 2) return NBODY_OK;
    NBODY_REQUIRE(keys && left && right && lo && hi && prefix,
                  "nbody_radix_tree_u32: null array");
    nb::radix_tree_u32(keys, n, key_bits, left, right, lo, hi, prefix);
  })
}

extern "C" int nbody_selftest_sort_wait(int* status_bits) {
  NBODY_API_BODY({
    NBODY_REQUIRE(status_bits, "nbody_selftest_sort_wait: null argument");
    *status_bits = nb::sort_wait_selftest();
  })
}
