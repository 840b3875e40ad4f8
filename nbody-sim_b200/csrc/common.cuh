// common.cuh -- device helpers shared by the nbody-b200 kernels (sm_100a).
#pragma once
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>
#include <stdexcept>
#include <string>

namespace nb {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

// Status bits raised by kernels into a device word; the host reads it once per
// call (no per-kernel sync).  Every bounded loop that gives up sets one.
enum StatusBits : int {
  kStatusStackOverflow = 1,   // walk stack spill area exhausted
  kStatusUnionFindLimit = 2,  // FoF union loop hit its iteration cap
  kStatusTreeLimit = 4,       // tree bottom-up climb exceeded its bound
  kStatusNonFinite = 8,       // a non-finite position reached key generation
  kStatusTapeFull = 16,       // a recording walk ran out of tape chunks
  kStatusSortWait = 32,       // a radix-sort look-back wait gave up
};

// Hi/lo float pair state (NBODY_STATE_F32X2): value = hi + lo with
// |lo| <= ulp(hi)/2, about 48 significant bits in 8 bytes.  Kernels convert
// to double, compute in FP64 and split back; the tree reads hi.
struct __align__(8) HiLo {
  float hi, lo;
  HiLo() = default;
  __host__ __device__ explicit HiLo(double v) {
    hi = (float)v;
    lo = (float)(v - (double)hi);
  }
  __host__ __device__ explicit HiLo(float v) : hi(v), lo(0.f) {}
  __host__ __device__ explicit operator double() const { return (double)hi + (double)lo; }
  __host__ __device__ explicit operator float() const { return hi; }
};

// Arithmetic type of a state storage type.
template <typename R>
struct ComputeOf {
  using type = R;
};
template <>
struct ComputeOf<HiLo> {
  using type = double;
};

struct CudaError : std::runtime_error {
  explicit CudaError(const std::string& s) : std::runtime_error(s) {}
};

// Throws on a failed runtime call.  The runtime also keeps that error as its
// "last error" until read; it is read here, so that a later
// cudaGetLastError() after a kernel launch reports that launch, not this call.
inline void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    throw CudaError(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
  }
}

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

// Order-preserving map of a double onto uint64 (for atomicMin/Max bboxes).
__device__ __forceinline__ unsigned long long ordered_bits(double v) {
  unsigned long long u = (unsigned long long)__double_as_longlong(v);
  return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__host__ __device__ inline double from_ordered_bits(unsigned long long u) {
  u = (u & 0x8000000000000000ull) ? (u & 0x7fffffffffffffffull) : ~u;
  double d;
  memcpy(&d, &u, sizeof(d));
  return d;
}

__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ __forceinline__ int warp_incl_scan(int v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(kFull, v, o);
    if (lane >= o) v += t;
  }
  return v;
}
__device__ __forceinline__ unsigned warp_incl_scan(unsigned v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned t = __shfl_up_sync(kFull, v, o);
    if (lane >= o) v += t;
  }
  return v;
}
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Programmatic dependent launch (sm_90+).  A kernel launched with the
// programmatic-serialization attribute may start before the kernel ahead of
// it in the stream has finished: grid_dependency_wait() returns once that
// kernel has completed and its writes are visible (at once for a kernel
// launched without the attribute), and grid_dependents_launch() lets the
// next such kernel start early.
__device__ __forceinline__ void grid_dependency_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}
__device__ __forceinline__ void grid_dependents_launch() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Spreads the low 10 bits of v so that bit k lands on bit 3k.
__device__ __forceinline__ uint32_t spread3(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

// 30-bit Morton key with z as the most significant bit of each triple, so the
// key order inside a cell is the reference octant order k = x | y<<1 | z<<2
// (BHTree.cu:164-170).
__device__ __forceinline__ uint32_t morton30(uint32_t cx, uint32_t cy, uint32_t cz) {
  return spread3(cx) | (spread3(cy) << 1) | (spread3(cz) << 2);
}

}  // namespace nb
