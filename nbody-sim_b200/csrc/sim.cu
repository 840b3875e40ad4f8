// sim.cu -- the step engine: src/main.cu:85-139 with the state resident on
// the GPU, kept in the Morton order of the last tree build.
//
// One step (reference launch order K1, D, tree, force, perturber, collision,
// K2, drag) becomes:
//   k_stream  : [dv + K2 + drag of the previous step] + K1 + drift + bbox
//   k_keys    : 30-bit Morton keys of the new positions (bbox from k_stream)
//   sort      : 4-pass radix sort -> permutation
//   k_permute : state gathered into the new key order (+ float4 bodies)
//   Karras tree, bottom-up FP64 moments, octree layout
//   k_walk    : star + Barnes-Hut + perturber accelerations
//   k_neighbors (collisions only): dv
// and the trailing dv + K2 + drag is fused into the next step's k_stream.
// Both kicks of a step boundary use the same acceleration, so fusing K2(n)
// with K1(n+1) changes no arithmetic.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "capi_util.h"
#include "common.cuh"
#include "kernels.cuh"
#include "moments.cuh"
#include "output.h"
#include "physics.cuh"

namespace nb {
namespace {

constexpr int kThreads = 256;

// State storage: float (the reference's), double, or hi/lo float pairs.
template <typename R>
constexpr bool kIsF32 = std::is_same<R, float>::value;
template <typename R>
constexpr bool kIsF64 = std::is_same<R, double>::value;

int stream_grid(int n) { return std::max(1, std::min(div_up(n, kThreads), 148 * 8)); }

template <typename R>
struct StateArrays {
  R* v[6];  // x y z vx vy vz
  float* m;
  int* id;
  int* disk;  // ensembles: the body's disk (nullptr for one disk)
};

template <typename Tin, typename Tout>
__global__ void k_convert(const Tin* __restrict__ in, Tout* __restrict__ out, int n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = (Tout)in[i];
}

__global__ void k_iota(int* __restrict__ id, int n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    id[i] = (int)i;
}

// What the permute kernel also zeroes, in its first block: the encoded
// bounding boxes (6 words per disk, after the key kernel has read them) that
// the next stream kernel accumulates, and the walk's group counter and
// statistics (the walk is then launched with counters_zeroed).
struct StepReset {
  unsigned long long* enc = nullptr;
  int enc_words = 0;
  int* work = nullptr;
  unsigned long long* inter = nullptr;
  unsigned long long* counters = nullptr;
};

// State gathered into the new key order, plus the float4 bodies, in the
// moment tiles' layout (kMomentThreads threads with two consecutive bodies
// each, one block per tile of kMomentTile bodies): the gathered bodies' FP64
// moments (m, m x, m y, m z) -- from the FP64 positions for a double state,
// else from the float4 bodies, as k_moment_tiles takes them -- are scanned
// into the tile-local prefix and the tile sums on the way, so the octree
// build needs no pass of its own over the bodies.
template <typename R>
__global__ void __launch_bounds__(kMomentThreads)
k_permute(const uint32_t* __restrict__ perm, StateArrays<R> in, StateArrays<R> out, int n,
          float4* __restrict__ body4, const StepReset r, double4* __restrict__ ploc,
          double4* __restrict__ tile_sum) {
  if (blockIdx.x == 0) {  // counters the step uses next (each has a sole writer)
    for (int i = threadIdx.x; i < r.enc_words; i += blockDim.x)
      r.enc[i] = ((i % 6) < 3) ? ~0ull : 0ull;
    if (threadIdx.x == 0 && r.work) *r.work = 0;
    if (threadIdx.x == 1 && r.inter) *r.inter = 0ull;
    if (threadIdx.x >= 2 && threadIdx.x < 5 && r.counters) r.counters[threadIdx.x - 2] = 0ull;
  }
  const long long base = (long long)blockIdx.x * kMomentTile + 2ll * threadIdx.x;
  double4 v[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const long long s = base + k;
    v[k] = make_double4(0, 0, 0, 0);
    if (s >= n) continue;
    // every gather first, then every store: the arrays carry no restrict, so
    // interleaving them would make each load wait for the store before it
    const uint32_t o = perm[s];
    R q[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) q[c] = in.v[c][o];
    const float m = in.m[o];
    const int id = in.id[o];
    const int dk = in.disk ? in.disk[o] : 0;
#pragma unroll
    for (int c = 0; c < 6; ++c) out.v[c][s] = q[c];
    out.m[s] = m;
    out.id[s] = id;
    if (in.disk) out.disk[s] = dk;
    const float4 b = make_float4((float)q[0], (float)q[1], (float)q[2], m);
    body4[s] = b;
    if constexpr (kIsF64<R>)
      v[k] = body_moment((double)m, (double)q[0], (double)q[1], (double)q[2]);
    else
      v[k] = body_moment((double)m, (double)b.x, (double)b.y, (double)b.z);
  }
  moment_tile_scan(v[0], v[1], base, n, ploc, tile_sum);
}

struct StreamArgs {
  const float* ax;
  const float* ay;
  const float* az;
  const float* dvx;  // nullptr: no collision pass
  const float* dvy;
  const float* dvz;
  double dt;
  double dth;
  double decay;      // drag retention factor; <= 0 disables drag
  float decay_f;     // expf(-rate dt), the reference's float factor
  float dt_f;
  float dth_f;
  double eps;
  double star_mass;
  unsigned long long* bbox;
};

// Fused step boundary.  kEnd: dv + K2 + drag (main.cu:131-139);
// kBegin: K1 + drift (main.cu:104-107) + bbox of the new positions.
template <typename R, bool kEnd, bool kBegin, bool kMulti>
__device__ __forceinline__ void stream_body(StateArrays<R> st, int n, const StreamArgs& a) {
  using C = typename ComputeOf<R>::type;
  // FP32 state: the bbox in FP32 (a min or max of floats is one of them, so
  // it equals the FP64 one it is widened to at the end)
  using B = typename std::conditional<std::is_same<C, float>::value, float, double>::type;
  B lo[3] = {(B)INFINITY, (B)INFINITY, (B)INFINITY};
  B hi[3] = {-(B)INFINITY, -(B)INFINITY, -(B)INFINITY};
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
       s += (long long)gridDim.x * blockDim.x) {
    C x = (C)st.v[0][s], y = (C)st.v[1][s], z = (C)st.v[2][s];
    C vx = (C)st.v[3][s], vy = (C)st.v[4][s], vz = (C)st.v[5][s];
    C ax = (C)a.ax[s], ay = (C)a.ay[s], az = (C)a.az[s];
    if (sizeof(C) == 8) {  // FP64 arithmetic: the stiff star term in FP64
      double sx, sy, sz;
      star_accel<double>((double)x, (double)y, (double)z, a.eps, a.star_mass, sx, sy, sz);
      ax += (C)sx; ay += (C)sy; az += (C)sz;
    }
    if (kEnd) {
      if (a.dvx) {  // bhtree_applyCollisionDeltaKernel (BHTree.cu:683-685)
        vx += (C)a.dvx[s]; vy += (C)a.dvy[s]; vz += (C)a.dvz[s];
      }
      if (sizeof(C) == 4) {  // integrator_halfKickKernel: v += a dt/2 (one FMA)
        vx = fmaf((float)ax, a.dth_f, (float)vx);
        vy = fmaf((float)ay, a.dth_f, (float)vy);
        vz = fmaf((float)az, a.dth_f, (float)vz);
        if (a.decay > 0.0) {
          float fvx = (float)vx, fvy = (float)vy, fvz = (float)vz;
          gas_drag<float>((float)x, (float)z, fvx, fvy, fvz, a.decay_f, (float)a.star_mass);
          vx = fvx; vy = fvy; vz = fvz;
        }
      } else {
        vx = fma(ax, (C)a.dth, vx); vy = fma(ay, (C)a.dth, vy); vz = fma(az, (C)a.dth, vz);
        if (a.decay > 0.0) gas_drag<C>(x, z, vx, vy, vz, (C)a.decay, (C)a.star_mass);
      }
    }
    if (kBegin) {
      if (sizeof(C) == 4) {
        vx = fmaf((float)ax, a.dth_f, (float)vx);
        vy = fmaf((float)ay, a.dth_f, (float)vy);
        vz = fmaf((float)az, a.dth_f, (float)vz);
        x = fmaf((float)vx, a.dt_f, (float)x);
        y = fmaf((float)vy, a.dt_f, (float)y);
        z = fmaf((float)vz, a.dt_f, (float)z);
      } else {
        vx = fma(ax, (C)a.dth, vx); vy = fma(ay, (C)a.dth, vy); vz = fma(az, (C)a.dth, vz);
        x = fma(vx, (C)a.dt, x); y = fma(vy, (C)a.dt, y); z = fma(vz, (C)a.dt, z);
      }
      if (kMulti) {
        // per-disk bbox: one warp-wide reduction when the warp's bodies share
        // a disk (the common case), per-lane atomics at a disk boundary
        const int d = st.disk[s];
        const unsigned act = __activemask();
        const int d0 = __shfl_sync(act, d, __ffs(act) - 1);
        const bool same = __all_sync(act, d == d0) && act == kFull;
        unsigned long long* bb = a.bbox + 6 * d;
        if (same) {
          double v6[6] = {(double)x, (double)y, (double)z, (double)x, (double)y, (double)z};
#pragma unroll
          for (int k = 0; k < 3; ++k) { v6[k] = warp_min(v6[k]); v6[3 + k] = warp_max(v6[3 + k]); }
          if ((threadIdx.x & 31) == 0) {
            for (int k = 0; k < 3; ++k) {
              atomicMin(bb + k, ordered_bits(v6[k]));
              atomicMax(bb + 3 + k, ordered_bits(v6[3 + k]));
            }
          }
        } else {
          atomicMin(bb + 0, ordered_bits((double)x)); atomicMax(bb + 3, ordered_bits((double)x));
          atomicMin(bb + 1, ordered_bits((double)y)); atomicMax(bb + 4, ordered_bits((double)y));
          atomicMin(bb + 2, ordered_bits((double)z)); atomicMax(bb + 5, ordered_bits((double)z));
        }
      } else {
        lo[0] = fmin(lo[0], (B)x); hi[0] = fmax(hi[0], (B)x);
        lo[1] = fmin(lo[1], (B)y); hi[1] = fmax(hi[1], (B)y);
        lo[2] = fmin(lo[2], (B)z); hi[2] = fmax(hi[2], (B)z);
      }
      st.v[0][s] = (R)x; st.v[1][s] = (R)y; st.v[2][s] = (R)z;
    }
    st.v[3][s] = (R)vx; st.v[4][s] = (R)vy; st.v[5][s] = (R)vz;
  }
  if (kBegin && !kMulti) {
    __shared__ double sb[6][kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double p = (double)warp_min(lo[k]), q = (double)warp_max(hi[k]);
      if (lane == 0) { sb[k][warp] = p; sb[3 + k][warp] = q; }
    }
    __syncthreads();
    if (threadIdx.x < 6) {
      const int k = threadIdx.x;
      double v = sb[k][0];
      for (int w = 1; w < kThreads / 32; ++w) v = (k < 3) ? fmin(v, sb[k][w]) : fmax(v, sb[k][w]);
      if (v == v && fabs(v) != INFINITY) {
        if (k < 3) atomicMin(a.bbox + k, ordered_bits(v));
        else atomicMax(a.bbox + k, ordered_bits(v));
      }
    }
  }
}

template <typename R, bool kEnd, bool kBegin, bool kMulti = false>
__global__ void __launch_bounds__(kThreads) k_stream(StateArrays<R> st, int n, StreamArgs a) {
  stream_body<R, kEnd, kBegin, kMulti>(st, n, a);
}

// The fused boundary of FP32 steps (second kick, drag, first kick, drift) at
// four blocks per SM (64 registers), so that more of its loads are in
// flight; the other forms keep the compiler's choice (bounded like this the
// FP64 ones would spill).
template <bool kMulti>
__global__ void __launch_bounds__(kThreads, 4)
    k_stream_f32(StateArrays<float> st, int n, StreamArgs a) {
  stream_body<float, true, true, kMulti>(st, n, a);
}

template <typename R, bool kEnd, bool kBegin, bool kMulti = false>
void launch_stream(const StateArrays<R>& st, int n, const StreamArgs& a, int g, cudaStream_t s) {
  if constexpr (std::is_same<R, float>::value && kEnd && kBegin)
    k_stream_f32<kMulti><<<g, kThreads, 0, s>>>(st, n, a);
  else
    k_stream<R, kEnd, kBegin, kMulti><<<g, kThreads, 0, s>>>(st, n, a);
}

// Writes the state back in caller order (out[id[s]] = state[s]); with
// accelerations, adds the FP64 star term in FP64 mode.
template <typename R, typename T>
__global__ void __launch_bounds__(kThreads)
k_unsort(StateArrays<R> st, int n, T* __restrict__ o0, T* __restrict__ o1, T* __restrict__ o2,
         T* __restrict__ o3, T* __restrict__ o4, T* __restrict__ o5, const float* __restrict__ ax,
         const float* __restrict__ ay, const float* __restrict__ az, float* __restrict__ oax,
         float* __restrict__ oay, float* __restrict__ oaz, double eps, double star_mass) {
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
       s += (long long)gridDim.x * blockDim.x) {
    const int o = st.id[s];
    const T q0 = (T)st.v[0][s], q1 = (T)st.v[1][s], q2 = (T)st.v[2][s];
    const T q3 = (T)st.v[3][s], q4 = (T)st.v[4][s], q5 = (T)st.v[5][s];
    o0[o] = q0; o1[o] = q1; o2[o] = q2;
    o3[o] = q3; o4[o] = q4; o5[o] = q5;
    if (oax) {
      double gx = ax[s], gy = ay[s], gz = az[s];
      if (sizeof(typename ComputeOf<R>::type) == 8) {  // the walk left the star out
        double sx, sy, sz;
        star_accel<double>((double)st.v[0][s], (double)st.v[1][s], (double)st.v[2][s], eps,
                           star_mass, sx, sy, sz);
        gx += sx; gy += sy; gz += sz;
      }
      oax[o] = (float)gx; oay[o] = (float)gy; oaz[o] = (float)gz;
    }
  }
}

// The caller-order read-back of nbody_sim_step_host in two halves: the
// positions (final once the last step's permute has run) and the velocities
// and accelerations (final at the end of the call).
template <typename R, typename T>
__global__ void __launch_bounds__(kThreads)
k_unsort_pos(StateArrays<R> st, int n, T* __restrict__ ox, T* __restrict__ oy,
             T* __restrict__ oz) {
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
       s += (long long)gridDim.x * blockDim.x) {
    const int o = st.id[s];
    const T px = (T)st.v[0][s], py = (T)st.v[1][s], pz = (T)st.v[2][s];
    ox[o] = px; oy[o] = py; oz[o] = pz;
  }
}

// Velocities and accelerations, as k_unsort writes them (with the star term
// an FP64 walk leaves out).
template <typename R, typename T>
__global__ void __launch_bounds__(kThreads)
k_unsort_vel_acc(StateArrays<R> st, int n, T* __restrict__ ovx, T* __restrict__ ovy,
                 T* __restrict__ ovz, const float* __restrict__ ax,
                 const float* __restrict__ ay, const float* __restrict__ az,
                 float* __restrict__ oax, float* __restrict__ oay, float* __restrict__ oaz,
                 double eps, double star_mass) {
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
       s += (long long)gridDim.x * blockDim.x) {
    const int o = st.id[s];
    const T vx = (T)st.v[3][s], vy = (T)st.v[4][s], vz = (T)st.v[5][s];
    double gx = ax[s], gy = ay[s], gz = az[s];
    if (sizeof(typename ComputeOf<R>::type) == 8) {  // the walk left the star out
      double sx, sy, sz;
      star_accel<double>((double)st.v[0][s], (double)st.v[1][s], (double)st.v[2][s], eps,
                         star_mass, sx, sy, sz);
      gx += sx; gy += sy; gz += sz;
    }
    ovx[o] = vx; ovy[o] = vy; ovz[o] = vz;
    oax[o] = (float)gx; oay[o] = (float)gy; oaz[o] = (float)gz;
  }
}

// The positions-first read-back of a host round trip: positions on rb (once
// ev_pos, recorded after the last permute, has fired), then velocities and
// accelerations on st; T is the caller's type.  stage holds 6 T + 3 floats
// per body.
template <typename R, typename T>
void read_back_split(const StateArrays<R>& a, int n, const float* ax, const float* ay,
                     const float* az, double eps, double star_mass, T* const* v,
                     float* const* acc, void* stage, cudaEvent_t ev_pos, cudaStream_t rb,
                     cudaStream_t st) {
  T* stg = (T*)stage;
  const size_t nn = (size_t)n, bytes = sizeof(T) * nn, fb = sizeof(float) * nn;
  check(cudaStreamWaitEvent(rb, ev_pos, 0), "read-back wait");
  k_unsort_pos<R, T><<<stream_grid(n), kThreads, 0, rb>>>(a, n, stg, stg + nn, stg + 2 * nn);
  check(cudaGetLastError(), "k_unsort_pos launch");
  for (int k = 0; k < 3; ++k)
    check(cudaMemcpyAsync(v[k], stg + k * nn, bytes, cudaMemcpyDeviceToHost, rb),
          "position D2H");
  T* sv = stg + 3 * nn;
  float* sa = (float*)(stg + 6 * nn);
  k_unsort_vel_acc<R, T><<<stream_grid(n), kThreads, 0, st>>>(
      a, n, sv, sv + nn, sv + 2 * nn, ax, ay, az, sa, sa + nn, sa + 2 * nn, eps, star_mass);
  check(cudaGetLastError(), "k_unsort_vel_acc launch");
  for (int k = 0; k < 3; ++k)
    check(cudaMemcpyAsync(v[3 + k], sv + k * nn, bytes, cudaMemcpyDeviceToHost, st),
          "velocity D2H");
  for (int k = 0; k < 3; ++k)
    check(cudaMemcpyAsync(acc[k], sa + k * nn, fb, cudaMemcpyDeviceToHost, st), "accel D2H");
  check(cudaStreamSynchronize(rb), "read-back sync");
  check(cudaStreamSynchronize(st), "step_host sync");
}

__global__ void k_scatter_labels(const int* __restrict__ in_l, const uint16_t* __restrict__ in_s,
                                 int n, int* __restrict__ out_l, uint16_t* __restrict__ out_s) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    out_l[i] = in_l[i];
    out_s[i] = in_s[i];
  }
}

// Ensemble: each body's disk from the per-disk offsets (binary search).
__global__ void k_disk_of(const int* __restrict__ offsets, int n_disks, int n,
                          int* __restrict__ disk) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = n_disks - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (offsets[mid] <= i) lo = mid;
      else hi = mid - 1;
    }
    disk[i] = lo;
  }
}

// Per-disk bbox of the current positions (warp-aggregated atomics).
template <typename R>
__global__ void __launch_bounds__(kThreads)
k_bbox_multi(StateArrays<R> st, int n, unsigned long long* __restrict__ bbox) {
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
       s += (long long)gridDim.x * blockDim.x) {
    const double p3[3] = {(double)st.v[0][s], (double)st.v[1][s], (double)st.v[2][s]};
    unsigned long long* bb = bbox + 6 * st.disk[s];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      atomicMin(bb + k, ordered_bits(p3[k]));
      atomicMax(bb + 3 + k, ordered_bits(p3[k]));
    }
  }
}

__global__ void k_increment(int* c) { *c += 1; }

template <typename T>
T* dalloc(size_t count, const char* what) {
  T* p = nullptr;
  check(cudaMalloc(&p, sizeof(T) * (count ? count : 1)), what);
  return p;
}

}  // namespace

// Writes the state back in the caller's order (by id) as float or double,
// with the accelerations (plus the star term the FP64 walk leaves out), into
// device buffers or, through the persistent device scratch `stage` (6 doubles
// + 3 floats per body), host buffers.
template <typename R>
void state_out(const StateArrays<R>& a, int n, const float* ax, const float* ay,
               const float* az, float eps, float star_mass, void* const* v, bool as_double,
               float* const* acc, bool on_device, void* stage, cudaStream_t st) {
  const size_t esz = as_double ? sizeof(double) : sizeof(float);
  char* scratch = (char*)stage;
  std::vector<void*> dst(6);
  for (int k = 0; k < 6; ++k) dst[k] = on_device ? v[k] : (void*)(scratch + k * esz * n);
  float* da[3] = {nullptr, nullptr, nullptr};
  if (acc && acc[0])
    for (int k = 0; k < 3; ++k)
      da[k] = on_device ? acc[k] : (float*)(scratch + 6 * sizeof(double) * n) + (size_t)k * n;
  if (as_double)
    k_unsort<R, double><<<stream_grid(n), kThreads, 0, st>>>(
        a, n, (double*)dst[0], (double*)dst[1], (double*)dst[2], (double*)dst[3],
        (double*)dst[4], (double*)dst[5], ax, ay, az, da[0], da[1], da[2], eps, star_mass);
  else
    k_unsort<R, float><<<stream_grid(n), kThreads, 0, st>>>(
        a, n, (float*)dst[0], (float*)dst[1], (float*)dst[2], (float*)dst[3], (float*)dst[4],
        (float*)dst[5], ax, ay, az, da[0], da[1], da[2], eps, star_mass);
  check(cudaGetLastError(), "k_unsort launch");
  if (!on_device) {
    for (int k = 0; k < 6; ++k)
      check(cudaMemcpyAsync(v[k], dst[k], esz * n, cudaMemcpyDeviceToHost, st), "state D2H");
    if (da[0])
      for (int k = 0; k < 3; ++k)
        check(cudaMemcpyAsync(acc[k], da[k], sizeof(float) * n, cudaMemcpyDeviceToHost, st),
              "accel D2H");
  }
  check(cudaStreamSynchronize(st), "get_state sync");
}

// The collision pass runs beside the force walk on the tree's second stream
// (it needs the tree and the half-step velocities, not the accelerations):
// its own group counter and stack-spill area, and the fork / join events.
struct CollSide {
  int* work = nullptr;
  int* spill = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  void alloc(size_t spill_words) {
    check(cudaMalloc(&work, sizeof(int)), "collision work");
    check(cudaMalloc(&spill, sizeof(int) * spill_words), "collision spill");
    check(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "collision fork");
    check(cudaEventCreateWithFlags(&join, cudaEventDisableTiming), "collision join");
  }
  void release() {
    if (work) cudaFree(work);
    if (spill) cudaFree(spill);
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
    *this = CollSide();
  }
};

// Bytes of the state_out scratch for n bodies.
inline size_t out_stage_bytes(int n) { return (size_t)n * (6 * sizeof(double) + 3 * sizeof(float)); }

struct SimBase {
  virtual ~SimBase() {}
  nbody_sim_params p{};
  int n = 0;
  cudaStream_t st = 0;
  int steps_done = 0;
  bool has_state = false;
  TreeWork tw;
  float *ax = nullptr, *ay = nullptr, *az = nullptr;
  float *dvx = nullptr, *dvy = nullptr, *dvz = nullptr;
  float4* pert_tab = nullptr;
  int pert_cap = 0;
  int* pert_step = nullptr;  // row of pert_tab the next walk reads (device)
  int* spill = nullptr;
  int spill_cap = 0;
  int* work = nullptr;
  unsigned long long* inter = nullptr;
  unsigned long long* counters = nullptr;  // walk: nodes visited, spills, groups
  // shared walk: per group its span, per span its lists, the lists' chunk pool
  int2* group_spans = nullptr;
  int4* span_lists = nullptr;
  int* span_pool = nullptr;
  int* span_next = nullptr;
  int* span_used = nullptr;
  int* span_work = nullptr;
  int span_cap = 0;  // chunks of 32 entries
  unsigned long long* span_counters = nullptr;  // shared entries, frontier entries, spans
  bool span_on() const {
    return p.span_walk == 1 && p.group_span > 1 && p.targets_per_lane == 1 &&
           !(p.r_coll > 0.f && p.fuse_collisions);
  }
  void span_alloc() {
    if (group_spans) return;
    group_spans = dalloc<int2>(n, "group spans");
    span_lists = dalloc<int4>(n, "span lists");
    span_cap = std::max(1024, n / 8);
    span_pool = dalloc<int>((size_t)span_cap * 32, "span pool");
    span_next = dalloc<int>(span_cap, "span chunk links");
    span_used = dalloc<int>(1, "span chunks used");
    span_work = dalloc<int>(1, "span counter");
    span_counters = dalloc<unsigned long long>(3, "span counters");
    check(cudaMemset(span_counters, 0, 3 * sizeof(unsigned long long)), "span counters");
  }
  int* parent = nullptr;
  int* labels = nullptr;
  int* sizes = nullptr;
  uint16_t* agg = nullptr;
  int* ngroups = nullptr;
  void* staging = nullptr;  // n doubles
  void* out_stage = nullptr;  // get_state to host: out_stage_bytes(n), on first use
  nbody_perturber pert{};
  // profiling: events at phase boundaries of every step, read lazily
  bool profiling = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::vector<cudaEvent_t>> ev_pending;  // per record: NBODY_PHASES + 1 events
  std::vector<bool> ev_is_step;
  std::vector<cudaEvent_t>* ev_cur = nullptr;
  double phase_ms[NBODY_PHASES] = {0};
  int profiled_steps = 0;
  unsigned long long launches = 0;

  cudaEvent_t take_event() {
    if (ev_pool.empty()) {
      cudaEvent_t e;
      check(cudaEventCreate(&e), "cudaEventCreate");
      return e;
    }
    cudaEvent_t e = ev_pool.back();
    ev_pool.pop_back();
    return e;
  }
  void mark(int phase) {  // boundary before `phase` (NBODY_PHASES = end)
    if (!ev_cur) return;
    // inside a capture: an event-record node of the step's graph
    check(cudaEventRecordWithFlags((*ev_cur)[phase], st,
                                   capturing ? cudaEventRecordExternal : cudaEventRecordDefault),
          "cudaEventRecord");
  }
  void begin_step_profile(bool is_step = true) {
    if (!profiling) { ev_cur = nullptr; return; }
    ev_is_step.push_back(is_step);
    ev_pending.emplace_back();
    ev_cur = &ev_pending.back();
    for (int k = 0; k <= NBODY_PHASES; ++k) ev_cur->push_back(take_event());
    for (int k = 0; k <= NBODY_PHASES; ++k) mark(k);  // phases skipped this step read 0
  }
  void collect_profile() {
    if (ev_pending.empty()) return;
    check(cudaStreamSynchronize(st), "profile sync");
    for (size_t r = 0; r < ev_pending.size(); ++r) {
      auto& evs = ev_pending[r];
      for (int k = 0; k < NBODY_PHASES; ++k) {
        float ms = 0.f;
        check(cudaEventElapsedTime(&ms, evs[k], evs[k + 1]), "cudaEventElapsedTime");
        phase_ms[k] += ms;
      }
      if (ev_is_step[r]) ++profiled_steps;
      for (cudaEvent_t e : evs) ev_pool.push_back(e);
    }
    ev_pending.clear();
    ev_is_step.clear();
    ev_cur = nullptr;
  }

  virtual void set_state(const void* const* v, bool is_double, const float* mass,
                         bool on_device, bool forces = true) = 0;
  virtual void get_state(void* const* v, bool as_double, float* const* a, bool on_device) = 0;
  // nsteps steps; close: end with the last step's second kick and drag.
  // Left open, the velocities stay at the last step's half step and the next
  // advance starts with its fused (second kick + drag, first kick) form.
  virtual void advance(int nsteps, bool close) = 0;
  void step(int nsteps) { advance(nsteps, true); }
  bool open = false;  // the last step's second kick and drag are pending
  virtual const uint32_t* ids() = 0;
  // Positions and velocities in caller order as float, on the engine stream.
  virtual void snapshot(float* const* dst) = 0;
  OutputPipe* pipe = nullptr;
  virtual void load_accel(const float* ax, const float* ay, const float* az) = 0;
  virtual void autotune(const int* cand, int nc, float* ms_out) = 0;
  // Host round trip of nbody_sim_step_host (float state and float arrays).
  virtual void step_host(float* const* v, float* const* a, const float* mass, int nsteps) = 0;
  // Recorded after every permute (an external event node inside the step
  // graphs): from there on the step leaves the positions alone.
  cudaEvent_t ev_pos = nullptr;
  cudaStream_t rb_st = nullptr;  // read-back stream of step_host
  CollSide cs;                   // collisions beside the walk (r_coll > 0)
  bool capturing = false;

  void common_alloc() {
    tree_alloc(tw, n);
    ax = dalloc<float>(n, "ax"); ay = dalloc<float>(n, "ay"); az = dalloc<float>(n, "az");
    dvx = dalloc<float>(n, "dvx"); dvy = dalloc<float>(n, "dvy"); dvz = dalloc<float>(n, "dvz");
    spill_cap = p.spill_cap > 0 ? p.spill_cap : 4096;
    spill = dalloc<int>((size_t)walk_spill_slots(0) * spill_cap, "walk spill");
    work = dalloc<int>(1, "work");
    inter = dalloc<unsigned long long>(1, "inter");
    counters = dalloc<unsigned long long>(3, "walk counters");
    parent = dalloc<int>(n, "fof parent");
    labels = dalloc<int>(n, "fof labels");
    sizes = dalloc<int>(n, "fof sizes");
    agg = dalloc<uint16_t>(n, "fof agg");
    ngroups = dalloc<int>(1, "fof ngroups");
    staging = dalloc<double>(n, "staging");
    pert_step = dalloc<int>(1, "perturber row");
    check(cudaMemset(pert_step, 0, sizeof(int)), "perturber row init");
  }

  // CUDA graphs of one step: [first step of a call?][state buffer at step
  // start]; captured on a private stream, replayed on the engine's.
  bool use_graphs = true;
  cudaStream_t cap_st = nullptr;
  cudaGraphExec_t gx[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  unsigned long long g_kernels[2][2] = {{0, 0}, {0, 0}};
  unsigned long long graph_launches = 0;
  // Profiled steps with graphs on: the same step graphs, captured with an
  // event-record node at each phase boundary (pev: their events).
  cudaGraphExec_t pgx[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  std::vector<cudaEvent_t> pev[2][2];
  void drop_graphs() {
    for (auto* set : {&gx, &pgx})
      for (auto& row : *set)
        for (auto& g : row)
          if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  }

  void common_free() {
    drop_graphs();
    for (void* q : {(void*)group_spans, (void*)span_lists, (void*)span_pool, (void*)span_next,
                    (void*)span_used, (void*)span_work, (void*)span_counters})
      if (q) cudaFree(q);
    if (cap_st) cudaStreamDestroy(cap_st);
    if (rb_st) cudaStreamDestroy(rb_st);
    if (ev_pos) cudaEventDestroy(ev_pos);
    cs.release();
    if (pipe) {
      delete pipe;
      pipe = nullptr;
    }
    for (auto& evs : ev_pending)
      for (cudaEvent_t e : evs) ev_pool.push_back(e);
    for (auto& row : pev)
      for (auto& evs : row)
        for (cudaEvent_t e : evs) ev_pool.push_back(e);
    for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
    tree_free(tw);
    void* ptrs[] = {ax, ay, az, dvx, dvy, dvz, pert_tab, pert_step, spill, work, inter,
                    counters, parent, labels, sizes, agg, ngroups, staging, out_stage};
    for (void* q : ptrs)
      if (q) cudaFree(q);
  }

  // Perturber positions for force times (k+1) dt, k in [k0, k0+count), by the
  // host arithmetic of updatePerturber (Perturber.h:60-66); the walk reads row
  // *pert_step, which every step advances (so a captured step needs no host
  // update).
  void upload_perturber(int k0, int count) {
    if (!p.perturber_enabled || count <= 0) return;
    if (count > pert_cap) {
      check(cudaStreamSynchronize(st), "perturber table sync");
      if (pert_tab) cudaFree(pert_tab);
      pert_cap = std::max(count, std::max(64, 2 * pert_cap));
      pert_tab = dalloc<float4>(pert_cap, "perturber table");
      drop_graphs();  // the captured walks hold the old table
    }
    std::vector<float4> h(count);
    for (int k = 0; k < count; ++k) {
      nbody_perturber q = pert;
      nbody_perturber_update(&q, (float)(k0 + k + 1) * p.dt);
      h[k] = make_float4(q.x, q.y, q.z, q.mass_msun);
    }
    check(cudaMemcpyAsync(pert_tab, h.data(), sizeof(float4) * count, cudaMemcpyHostToDevice, st),
          "perturber upload");
    check(cudaMemsetAsync(pert_step, 0, sizeof(int), st), "perturber row reset");
  }

  int check_status() {
    int s = 0;
    check(cudaStreamSynchronize(st), "engine sync");
    check(cudaMemcpy(&s, tw.status, sizeof(int), cudaMemcpyDeviceToHost), "status read");
    return s;
  }

  void fof(float ll, int* out_labels, uint16_t* out_agg, int* n_groups, bool on_device) {
    NeighborArgs na{tw.oct.info, tw.oct.box_lo, tw.oct.box_hi, tw.body4, n,
                    tw.groups, tw.n_groups, p.leaf_max, spill, spill_cap, work, tw.status};
    launch_fof_link(na, ids(), ll, parent, st);
    launch_fof_finish(parent, n, labels, sizes, agg, ngroups, tw.status, st);
    if (on_device) {
      k_scatter_labels<<<stream_grid(n), kThreads, 0, st>>>(labels, agg, n, out_labels, out_agg);
      check(cudaGetLastError(), "fof copy");
    } else {
      check(cudaMemcpyAsync(out_labels, labels, sizeof(int) * n, cudaMemcpyDeviceToHost, st),
            "fof labels D2H");
      check(cudaMemcpyAsync(out_agg, agg, sizeof(uint16_t) * n, cudaMemcpyDeviceToHost, st),
            "fof sizes D2H");
    }
    check(cudaMemcpyAsync(n_groups, ngroups, sizeof(int), cudaMemcpyDeviceToHost, st),
          "fof groups D2H");
    check(cudaStreamSynchronize(st), "fof sync");
  }
};

template <typename R>
struct SimImpl : SimBase {
  StateArrays<R> s[2]{};
  int cur = 0;

  SimImpl(const nbody_sim_params& prm, int nn) {
    p = prm;
    n = nn;
    if (p.leaf_max <= 0) p.leaf_max = default_leaf_max(n);
    if (p.targets_per_lane != 2) p.targets_per_lane = 1;
    if (p.walk_mode < 0 || p.walk_mode > 2) p.walk_mode = kDefaultWalkMode;
    if (p.group_span <= 0) p.group_span = (n >= kGroupSpanMinBodies) ? kDefaultGroupSpan : 1;
    if (p.group_span > 64) p.group_span = 64;
    nbody_config c;
    nbody_config_defaults(&c);
    c.perturber_enabled = p.perturber_enabled;
    c.perturber_mass_mjup = p.perturber_mass_mjup;
    c.perturber_radius_AU = p.perturber_radius_au;
    c.perturber_phase0 = p.perturber_phase0;
    c.star_mass_msun = p.star_mass;
    nbody_perturber_make(&c, &pert);
    common_alloc();
    tree_enable_overlap(tw);
    check(cudaEventCreateWithFlags(&ev_pos, cudaEventDisableTiming), "position event");
    check(cudaStreamCreateWithFlags(&rb_st, cudaStreamNonBlocking), "read-back stream");
    if (p.r_coll > 0.f) cs.alloc((size_t)walk_spill_slots(0) * spill_cap);
    tw.group_max = 32 * p.targets_per_lane;
    tw.group_span = p.group_span;
    for (int b = 0; b < 2; ++b) {
      for (int k = 0; k < 6; ++k) s[b].v[k] = dalloc<R>(n, "state");
      s[b].m = dalloc<float>(n, "mass");
      s[b].id = dalloc<int>(n, "id");
    }
  }

  ~SimImpl() override {
    for (int b = 0; b < 2; ++b) {
      for (int k = 0; k < 6; ++k) cudaFree(s[b].v[k]);
      cudaFree(s[b].m);
      cudaFree(s[b].id);
    }
    common_free();
  }

  const uint32_t* ids() override { return (const uint32_t*)s[cur].id; }

  void snapshot(float* const* d) override {
    k_unsort<R, float><<<stream_grid(n), kThreads, 0, st>>>(
        s[cur], n, d[0], d[1], d[2], d[3], d[4], d[5], ax, ay, az, nullptr, nullptr, nullptr,
        p.softening, p.star_mass);
    check(cudaGetLastError(), "snapshot launch");
    launches += 1;
  }

  void set_state(const void* const* v, bool is_double, const float* mass, bool on_device,
                 bool forces) override {
    cur = 0;
    const size_t esz = is_double ? sizeof(double) : sizeof(float);
    const bool same = (is_double && kIsF64<R>) || (!is_double && kIsF32<R>);
    for (int k = 0; k < 6; ++k) {
      const void* src = v[k];
      if (same) {  // the caller's type is the state's: one copy, no conversion pass
        check(cudaMemcpyAsync(s[0].v[k], src, esz * n,
                              on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st),
              "state copy");
        continue;
      }
      if (!on_device) {
        check(cudaMemcpyAsync(staging, src, esz * n, cudaMemcpyHostToDevice, st), "state H2D");
        src = staging;
      }
      if (is_double)
        k_convert<double, R><<<stream_grid(n), kThreads, 0, st>>>((const double*)src, s[0].v[k], n);
      else
        k_convert<float, R><<<stream_grid(n), kThreads, 0, st>>>((const float*)src, s[0].v[k], n);
      check(cudaGetLastError(), "state convert");
    }
    check(cudaMemcpyAsync(s[0].m, mass, sizeof(float) * n,
                          on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st),
          "mass copy");
    k_iota<<<stream_grid(n), kThreads, 0, st>>>(s[0].id, n);
    check(cudaGetLastError(), "iota");
    steps_done = 0;
    has_state = true;
    open = false;
    if (forces) {
      upload_perturber(-1, 1);  // (float)(0) * dt = 0
      launch_bbox<R>(tw, s[0].v[0], s[0].v[1], s[0].v[2], n, st);
      compute_forces(true);
    } else {
      launch_bbox_reset(tw, st);  // the next k_stream accumulates the bbox
    }
  }

  void load_accel(const float* hax, const float* hay, const float* haz) override {
    // caller order == current order right after set_state (id = iota)
    check(cudaMemcpyAsync(ax, hax, sizeof(float) * n, cudaMemcpyHostToDevice, st), "ax H2D");
    check(cudaMemcpyAsync(ay, hay, sizeof(float) * n, cudaMemcpyHostToDevice, st), "ay H2D");
    check(cudaMemcpyAsync(az, haz, sizeof(float) * n, cudaMemcpyHostToDevice, st), "az H2D");
  }

  // Tree + walk for the current positions; initial: the forces of t = 0 (the
  // perturber where makePerturber puts it), else of the step's row.
  void compute_forces(bool initial) {
    StateArrays<R>& a = s[cur];
    StateArrays<R>& b = s[1 - cur];
    mark(NBODY_PHASE_SORT);
    // the key kernel also counts the digits of the sort's four passes
    uint32_t* hist = radix_sort_prepare(tw.counts, 30, st);
    launch_keys<R>(tw, a.v[0], a.v[1], a.v[2], n, st, hist);
    radix_sort_pairs(tw.keys, tw.perm, tw.keys_alt, tw.perm_alt, tw.counts, n, 30, st,
                     tw.status, true);
    mark(NBODY_PHASE_PERMUTE);
    StepReset rs;
    rs.enc = tw.bbox_enc; rs.enc_words = 6;
    rs.work = work; rs.inter = inter; rs.counters = counters;
    k_permute<R><<<moment_tiles(n), kMomentThreads, 0, st>>>(tw.perm, a, b, n, tw.body4, rs,
                                                             tw.mom_ploc, tw.mom_tiles);
    check(cudaGetLastError(), "k_permute launch");
    check(cudaEventRecordWithFlags(ev_pos, st, capturing ? cudaEventRecordExternal
                                                         : cudaEventRecordDefault),
          "position event");
    cur = 1 - cur;
    mark(NBODY_PHASE_TREE);
    tw.prune_max = p.leaf_max;
    tw.boxes = p.r_coll > 0.f;  // only the collision searches read the records' boxes
    const bool span = span_on();
    if (span) span_alloc();
    tw.group_spans = span ? group_spans : nullptr;
    if (kIsF64<R>)
      launch_tree<uint32_t>(tw, tw.keys, n, 30, 0, 1, tw.geom, nullptr,
                            (const double*)s[cur].v[0], (const double*)s[cur].v[1],
                            (const double*)s[cur].v[2], st, true);
    else
      launch_tree<uint32_t>(tw, tw.keys, n, 30, 0, 1, tw.geom, nullptr, nullptr, nullptr, nullptr,
                            st, true);
    WalkArgs w{};
    w.com = tw.oct.com; w.info = tw.oct.info; w.body = tw.body4; w.n = n;
    w.groups = tw.groups; w.n_groups = tw.n_groups;
    w.theta2 = p.theta * p.theta; w.eps = p.softening; w.star_mass = p.star_mass;
    w.star_in_walk = kIsF32<R> ? 1 : 0;
    w.leaf_max = p.leaf_max;
    w.pert = p.perturber_enabled ? pert_tab : nullptr;
    w.pert_step = p.perturber_enabled ? pert_step : nullptr;
    w.n_disks = 1;
    w.ax = ax; w.ay = ay; w.az = az; w.scatter = nullptr;
    w.spill = spill; w.spill_cap = spill_cap; w.inter = inter; w.counters = counters;
    w.work = work; w.status = tw.status; w.targets_per_lane = tw.group_max / 32;
    w.walk_mode = p.walk_mode;
    w.counters_zeroed = true;
    if (!initial && coll_fused()) set_coll_args(w);
    const bool side_coll = !initial && p.r_coll > 0.f && !coll_fused();
    if (side_coll) {  // the collision pass on the second stream, beside the walk
      check(cudaEventRecord(cs.fork, st), "collision fork");
      check(cudaStreamWaitEvent(tw.side, cs.fork, 0), "collision fork");
      collide(tw.side, cs.work, cs.spill);
      check(cudaEventRecord(cs.join, tw.side), "collision join");
      launches += 1;
    }
    mark(NBODY_PHASE_WALK);
    if (span) {  // the shared walk's first traversal (one warp per span node), then the walk
      SpanArgs sa{tw.oct.com, tw.oct.info, tw.body4, tw.groups, group_spans, tw.n_groups,
                  p.theta * p.theta, p.leaf_max, span_lists, span_pool, span_next, span_used,
                  span_cap, span_work, span_counters};
      launch_span_walk(sa, n, st);
      w.group_span = group_spans; w.span_lists = span_lists;
      w.span_pool = span_pool; w.span_next = span_next;
      launches += 2;
    }
    launch_walk(w, st);
    if (side_coll) check(cudaStreamWaitEvent(st, cs.join, 0), "collision join");
    mark(NBODY_PHASE_COLLIDE);
    // keys (+ digit histograms), 4 one-sweep passes, permute (+ bbox and
    // walk counter resets, + moment tiles), moment tile scan, karras, mark,
    // tile scan, apply, emit, walk
    launches += 13;
  }

  // Collisions inside the walk (one warp per group of <= 32 targets).
  bool coll_fused() const {
    return p.r_coll > 0.f && p.fuse_collisions && tw.group_max == 32;
  }
  void set_coll_args(WalkArgs& w) {
    for (int k = 0; k < 3; ++k) w.coll_v[k] = s[cur].v[3 + k];
    w.coll_vtype = kIsF32<R> ? 0 : (kIsF64<R> ? 1 : 2);
    w.coll_r = p.r_coll;
    w.coll_e = p.restitution;
    w.coll_dv[0] = dvx; w.coll_dv[1] = dvy; w.coll_dv[2] = dvz;
    w.box_lo = tw.oct.box_lo; w.box_hi = tw.oct.box_hi;
  }

  void collide(cudaStream_t on, int* wk, int* sp) {
    NeighborArgs na{tw.oct.info, tw.oct.box_lo, tw.oct.box_hi, tw.body4, n,
                    tw.groups, tw.n_groups, p.leaf_max, sp, spill_cap, wk, tw.status};
    // the half-step velocities read in their storage type, rounded to float
    launch_collide_v(na, s[cur].v[3], s[cur].v[4], s[cur].v[5],
                     kIsF32<R> ? 0 : (kIsF64<R> ? 1 : 2), nullptr, p.r_coll, p.restitution,
                     dvx, dvy, dvz, on);
  }

  void stream_kernel(bool end, bool begin) {
    StreamArgs a{};
    a.ax = ax; a.ay = ay; a.az = az;
    const bool coll = p.r_coll > 0.f;
    a.dvx = coll ? dvx : nullptr; a.dvy = coll ? dvy : nullptr; a.dvz = coll ? dvz : nullptr;
    a.dt_f = p.dt;
    a.dth_f = p.dt * 0.5f;
    a.dt = (double)p.dt;
    a.dth = (double)p.dt * 0.5;
    const bool drag = p.gas_drag_rate > 0.f;
    a.decay_f = drag ? expf(-p.gas_drag_rate * p.dt) : 0.f;
    a.decay = drag ? std::exp(-(double)p.gas_drag_rate * (double)p.dt) : 0.0;
    a.eps = p.softening;
    a.star_mass = p.star_mass;
    a.bbox = tw.bbox_enc;
    const int g = stream_grid(n);
    if (end && begin)
      launch_stream<R, true, true>(s[cur], n, a, g, st);
    else if (end)
      launch_stream<R, true, false>(s[cur], n, a, g, st);
    else
      launch_stream<R, false, true>(s[cur], n, a, g, st);
    check(cudaGetLastError(), "k_stream launch");
  }

  // One step (main.cu:101-139): [dv + K2 + drag of the previous step] + K1 +
  // drift, tree + walk (+ star, + perturber row), collisions; the perturber
  // row advances.
  void one_step(bool first) {
    mark(NBODY_PHASE_STREAM);
    stream_kernel(!first, true);
    compute_forces(false);  // with the collision pass when r_coll > 0
    if (p.perturber_enabled) {
      k_increment<<<1, 1, 0, st>>>(pert_step);
      check(cudaGetLastError(), "k_increment launch");
      launches += 1;
    }
    mark(NBODY_PHASES);
    launches += 1;
  }

  cudaGraphExec_t graph_for(bool first) {
    const int f = first ? 1 : 0, c = cur;
    if (gx[f][c]) return gx[f][c];
    if (!cap_st) check(cudaStreamCreateWithFlags(&cap_st, cudaStreamNonBlocking), "capture stream");
    cudaGraph_t graph = nullptr;
    const unsigned long long l0 = launches;
    cudaStream_t user = st;
    st = cap_st;
    check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
    capturing = true;
    one_step(first);
    capturing = false;
    const cudaError_t ce = cudaStreamEndCapture(st, &graph);
    st = user;
    check(ce, "end capture");
    cur = c;  // captured, not run
    g_kernels[f][c] = launches - l0;
    launches = l0;
    check(cudaGraphInstantiate(&gx[f][c], graph, 0), "graph instantiate");
    cudaGraphDestroy(graph);
    return gx[f][c];
  }

  // A profiled step as the graphs run it: the step graph captured with an
  // event-record node at each phase boundary (kept like the plain graphs),
  // replayed, and its events read once it has run, so the phase times hold
  // the graph's own launch gaps and overlap.
  void profiled_graph_step(bool first) {
    const int f = first ? 1 : 0, c = cur;
    std::vector<cudaEvent_t>& evs = pev[f][c];
    if (evs.empty())
      for (int k = 0; k <= NBODY_PHASES; ++k) evs.push_back(take_event());
    if (!pgx[f][c]) {
      if (!cap_st) check(cudaStreamCreateWithFlags(&cap_st, cudaStreamNonBlocking), "capture stream");
      const unsigned long long l0 = launches;
      cudaStream_t user = st;
      st = cap_st;
      cudaGraph_t graph = nullptr;
      check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
      capturing = true;
      ev_cur = &evs;
      one_step(first);
      ev_cur = nullptr;
      capturing = false;
      const cudaError_t ce = cudaStreamEndCapture(st, &graph);
      st = user;
      check(ce, "end capture");
      cur = c;  // captured, not run
      g_kernels[f][c] = launches - l0;
      launches = l0;
      const cudaError_t ie = cudaGraphInstantiate(&pgx[f][c], graph, 0);
      cudaGraphDestroy(graph);
      check(ie, "graph instantiate");
    }
    check(cudaGraphLaunch(pgx[f][c], st), "graph launch");
    check(cudaStreamSynchronize(st), "profiled graph step");
    for (int k = 0; k < NBODY_PHASES; ++k) {
      float ms = 0.f;
      check(cudaEventElapsedTime(&ms, evs[k], evs[k + 1]), "cudaEventElapsedTime");
      phase_ms[k] += ms;
    }
    ++profiled_steps;
    launches += g_kernels[f][c];
    graph_launches += 1;
    cur = 1 - cur;
  }

  void advance(int nsteps, bool close) override {
    if (nsteps > 0) {
      upload_perturber(steps_done, nsteps);
      for (int k = 0; k < nsteps; ++k) {
        const bool first = (k == 0) && !open;  // no pending second kick before it
        if (use_graphs && !profiling) {
          const int f = first ? 1 : 0, c = cur;
          check(cudaGraphLaunch(graph_for(first), st), "graph launch");
          launches += g_kernels[f][c];
          graph_launches += 1;
          cur = 1 - cur;
        } else if (use_graphs) {
          profiled_graph_step(first);
        } else {
          begin_step_profile();
          one_step(first);
        }
      }
      steps_done += nsteps;
      open = true;
    }
    if (close && open) {
      // the last step's dv + K2 + drag: a record that adds to the stream phase only
      begin_step_profile(false);
      stream_kernel(true, false);
      for (int k = NBODY_PHASE_STREAM + 1; k <= NBODY_PHASES; ++k) mark(k);
      launches += 1;
      ev_cur = nullptr;
      open = false;
    }
  }

  void get_state(void* const* v, bool as_double, float* const* acc, bool on_device) override {
    if (!on_device && !out_stage) out_stage = dalloc<char>(out_stage_bytes(n), "output staging");
    state_out<R>(s[cur], n, ax, ay, az, p.softening, p.star_mass, v, as_double, acc, on_device,
                 out_stage, st);
  }

  // copyToGPU, nsteps, copyToCPU.  The positions are final once the last
  // step's permute has run, so their caller-order gather and copy to the host
  // go out on the read-back stream while the tree, the walk and the closing
  // kick still run; the velocities and accelerations follow at the end.
  void step_host(float* const* v, float* const* acc, const float* mass, int nsteps) override {
    const int steps0 = steps_done;
    const void* vin[6] = {v[0], v[1], v[2], v[3], v[4], v[5]};
    set_state(vin, false, mass, false, false);
    load_accel(acc[0], acc[1], acc[2]);
    steps_done = steps0;  // the caller's clock continues
    void* vout[6] = {v[0], v[1], v[2], v[3], v[4], v[5]};
    if (nsteps <= 0 || !kIsF32<R>) {
      step(nsteps);
      get_state(vout, false, acc, false);
      return;
    }
    step(nsteps);
    if (!out_stage) out_stage = dalloc<char>(out_stage_bytes(n), "output staging");
    read_back_split<R, float>(s[cur], n, ax, ay, az, p.softening, p.star_mass, v, acc, out_stage,
                              ev_pos, rb_st, st);
  }

  // Times force evaluations of the current state for each candidate
  // (targets_per_lane, leaf_max, walk_mode, group_span) and keeps the
  // fastest; the forces are recomputed with it, the state is unchanged.
  void autotune(const int* cand, int nc, float* ms_out) override {
    static const int kDefault[] = {1, 8, 1, 0, 1, 8, 0, 0, 1, 8, 2, 0,
                                   1, 16, 1, 0, 1, 16, 2, 0, 1, 4, 2, 0};
    if (!cand) {
      cand = kDefault;
      nc = 6;
    }
    auto apply = [&](int k) {
      p.targets_per_lane = cand[4 * k] == 2 ? 2 : 1;
      p.leaf_max = std::max(1, cand[4 * k + 1]);
      p.walk_mode = (cand[4 * k + 2] >= 0 && cand[4 * k + 2] <= 2) ? cand[4 * k + 2]
                                                                : kDefaultWalkMode;
      const int span = cand[4 * k + 3];
      p.group_span = span > 0 ? std::min(span, 64) : (n >= kGroupSpanMinBodies ? kDefaultGroupSpan : 1);
      tw.group_max = 32 * p.targets_per_lane;
      tw.group_span = p.group_span;
    };
    auto forces = [&]() {  // the forces of the current time, no collisions
      upload_perturber(steps_done - 1, 1);
      launch_bbox_reset(tw, st);
      launch_bbox<R>(tw, s[cur].v[0], s[cur].v[1], s[cur].v[2], n, st);
      compute_forces(true);
    };
    cudaEvent_t e0, e1;
    check(cudaEventCreate(&e0), "event");
    check(cudaEventCreate(&e1), "event");
    float best = 0.f;
    int best_k = -1;
    for (int k = 0; k < nc; ++k) {
      apply(k);
      forces();  // warm-up with this setting
      float ms = 0.f;
      for (int rep = 0; rep < 2; ++rep) {  // best of two timed evaluations
        check(cudaEventRecord(e0, st), "event");
        forces();
        check(cudaEventRecord(e1, st), "event");
        check(cudaEventSynchronize(e1), "event sync");
        float t = 0.f;
        check(cudaEventElapsedTime(&t, e0, e1), "event time");
        ms = (rep == 0) ? t : std::min(ms, t);
      }
      if (ms_out) ms_out[k] = ms;
      if (best_k < 0 || ms < best) {
        best = ms;
        best_k = k;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    apply(best_k);
    drop_graphs();
    forces();
    check(cudaStreamSynchronize(st), "autotune sync");
  }
};

SimBase* make_sim(const nbody_sim_params& p, int n) {
  if (p.state_precision == NBODY_STATE_F64) return new SimImpl<double>(p, n);
  if (p.state_precision == NBODY_STATE_F32X2) return new SimImpl<HiLo>(p, n);
  return new SimImpl<float>(p, n);
}

}  // namespace nb

struct nbody_sim {
  nb::SimBase* impl;
};

extern "C" {

void nbody_sim_params_from_config(const nbody_config* cfg, nbody_sim_params* out) {
  std::memset(out, 0, sizeof(*out));
  out->dt = cfg->dt;
  out->theta = cfg->theta;
  out->softening = cfg->softening_AU;
  out->star_mass = cfg->star_mass_msun;
  // main.cu:58-59: r_coll = collision_radius_factor * particlePhysicalRadius
  out->r_coll = cfg->collision_radius_factor * nbody_particle_radius(cfg->particle_mass_msun);
  out->restitution = cfg->restitution;
  out->gas_drag_rate = cfg->gas_drag_rate;
  out->perturber_enabled = cfg->perturber_enabled;
  out->perturber_mass_mjup = cfg->perturber_mass_mjup;
  out->perturber_radius_au = cfg->perturber_radius_AU;
  out->perturber_phase0 = cfg->perturber_phase0;
  out->state_precision = NBODY_STATE_F32;
  out->leaf_max = 0;  // by the body count
  out->targets_per_lane = 1;
  out->walk_mode = nb::kDefaultWalkMode;
  out->group_span = 0;
}

int nbody_sim_create(const nbody_sim_params* p, int n, nbody_sim** out) {
  NBODY_API_BODY({
    NBODY_REQUIRE(p && out, "nbody_sim_create: null argument");
    NBODY_REQUIRE(n > 0 && n < (1 << 27), "nbody_sim_create: n must be in [1, 2^27)");
    NBODY_REQUIRE(p->dt > 0.f, "nbody_sim_create: dt must be positive");
    NBODY_REQUIRE(p->state_precision >= NBODY_STATE_F32 && p->state_precision <= NBODY_STATE_F32X2,
                  "nbody_sim_create: unknown state precision");
    *out = nullptr;
    nbody_sim* s = new nbody_sim{nb::make_sim(*p, n)};
    *out = s;
  })
}

void nbody_sim_destroy(nbody_sim* s) {
  if (!s) return;
  cudaStreamSynchronize(s->impl->st);
  delete s->impl;
  delete s;
}

int nbody_sim_set_stream(nbody_sim* s, void* stream) {
  NBODY_API_BODY({
    NBODY_REQUIRE(s, "nbody_sim_set_stream: null sim");
    s->impl->st = (cudaStream_t)stream;
  })
}

int nbody_sim_set_state(nbody_sim* s, const float* x, const float* y, const float* z,
                        const float* vx, const float* vy, const float* vz, const float* mass,
                        int on_device) {
  NBODY_API_BODY({
    NBODY_REQUIRE(s && x && y && z && vx && vy && vz && mass, "nbody_sim_set_state: null array");
    const void* v[6] = {x, y, z, vx, vy, vz};
    s->impl->set_state(v, false, mass, on_device != 0);
  })
}

int nbody_sim_set_state_f64(nbody_sim* s, const double* x, const double* y, const double* z,
                            const double* vx, const double* vy, const double* vz,
                            const float* mass, int on_device) {
  NBODY_API_BODY({
    NBODY_REQUIRE(s && x && y && z && vx && vy && vz && mass,
                  "nbody_sim_set_state_f64: null array");
    const void* v[6] = {x, y, z, vx, vy, vz};
    s->impl->set_state(v, true, mass, on_device != 0);
  })
}

int nbody_sim_step(nbody_sim* s, int nsteps) {
  NBODY_API_BODY({
    NBODY_REQUIRE(s, "nbody_sim_step: null sim");
    NBODY_REQUIRE(s->impl->has_state, "nbody_sim_step: state not set");
    NBODY_REQUIRE(nsteps >= 0, "nbody_sim_step: negative step count");
    s->impl->step(nsteps);
  })
}

int nbody_sim_step_open(nbody_sim* s, int nsteps) {
  NBODY_API_BODY({
    NBODY_REQUIRE(s, "nbody_sim_step_open: null sim");
    NBODY_REQUIRE(s->impl->has_state, "nbody_sim_step_open: state not set");
    NBODY_REQUIRE(nsteps >= 0, "nbody_sim_step_open: negative step count");
    s->impl->advance(nsteps, false);
  })
}

int nbody_sim_close(nbody_sim* s) {
  NBODY_API_BODY({
    NBODY_REQUIRE(s, "nbody_sim_close: null sim");
    s->impl->advance(0, true);
  })
}

int nbody_sim_sync(nbody_sim* s) {
  NBODY_API_BODY({
    NBODY_REQUIRE(s, "nbody_sim_sync: null sim");
    int st = s->impl->check_status();
    if (st) {
      nb::check(cudaMemsetAsync(s->impl->tw.status, 0, sizeof(int), s->impl->st), "status reset");
      throw nb::ArgError("device status " + std::to_string(st) +
                             " (1 walk stack, 2 union-find, 4 tree, 8 non-finite position, 16 tape, 32 sort wait)",
                         NBODY_ERR_OVERFLOW);
    }
  })
}

int nbody_sim_get_state(nbody_sim* s, float* x, float* y, float* z, float* vx, float* vy,
                        float* vz, float* ax, float* ay, float* az, int on_device) {
  NBODY_API_BODY({
    NBODY_REQUIRE(s && x && y && z && vx && vy && vz, "nbody_sim_get_state: null array");
    NBODY_REQUIRE(s->impl->has_state, "nbody_sim_get_state: state not set");
    s->impl->advance(0, true);  // a pending second kick first
    void* v[6] = {x, y, z, vx, vy, vz};
    float* a[3] = {ax, ay, az};
    s->impl->get_state(v, false, (ax && ay && az) ? a : nullptr, on_device != 0);
  })
}

int nbody_sim_get_state_f64(nbody_sim* s, double* x, double* y, double* z, double* vx,
                            double* vy, double* vz, int on_device) {
  NBODY_API_BODY({
    NBODY_REQUIRE(s && x && y && z && vx && vy && vz, "nbody_sim_get_state_f64: null array");
    NBODY_REQUIRE(s->impl->has_state, "nbody_sim_get_state_f64: state not set");
    s->impl->advance(0, true);  // a pending second kick first
    void* v[6] = {x, y, z, vx, vy, vz};
    s->impl->get_state(v, true, nullptr, on_device != 0);
  })
}

int nbody_sim_fof(nbody_sim* s, float link_length, int* labels, uint16_t* agg_size,
                  int* n_groups, int on_device) {
  NBODY_API_BODY({
    NBODY_REQUIRE(s && labels && agg_size && n_groups, "nbody_sim_fof: null argument");
    NBODY_REQUIRE(s->impl->has_state, "nbody_sim_fof: state not set");
    s->impl->advance(0, true);  // a pending second kick first
    s->impl->fof(link_length, labels, agg_size, n_groups, on_device != 0);
  })
}

int nbody_sim_set_profiling(nbody_sim* s, int on) {
  NBODY_API_BODY({
    NBODY_REQUIRE(s, "nbody_sim_set_profiling: null sim");
    s->impl->profiling = on != 0;
  })
}

int nbody_sim_profile_get(nbody_sim* s, nbody_sim_profile* out, int reset) {
  NBODY_API_BODY({
    NBODY_REQUIRE(s && out, "nbody_sim_profile_get: null argument");
    nb::SimBase* b = s->impl;
    b->collect_profile();
    std::memset(out, 0, sizeof(*out));
    for (int k = 0; k < NBODY_PHASES; ++k) out->ms[k] = b->phase_ms[k];
    out->steps = b->profiled_steps;
    out->launches = b->launches;
    if (reset) {
      for (int k = 0; k < NBODY_PHASES; ++k) b->phase_ms[k] = 0.0;
      b->profiled_steps = 0;
      b->launches = 0;
    }
  })
}

int nbody_sim_stats_get(nbody_sim* s, nbody_sim_stats* out) {
  NBODY_API_BODY({
    NBODY_REQUIRE(s && out, "nbody_sim_stats_get: null argument");
    nb::SimBase* b = s->impl;
    nb::check(cudaStreamSynchronize(b->st), "stats sync");
    std::memset(out, 0, sizeof(*out));
    out->n = b->n;
    out->steps_done = b->steps_done;
    nb::check(cudaMemcpy(&out->n_nodes, b->tw.n_nodes, sizeof(int), cudaMemcpyDeviceToHost),
              "n_nodes");
    nb::check(cudaMemcpy(&out->interactions, b->inter, sizeof(unsigned long long),
                         cudaMemcpyDeviceToHost), "interactions");
    nb::check(cudaMemcpy(&out->status, b->tw.status, sizeof(int), cudaMemcpyDeviceToHost),
              "status");
    unsigned long long c[3];
    nb::check(cudaMemcpy(c, b->counters, sizeof(c), cudaMemcpyDeviceToHost), "counters");
    out->walk_nodes_visited = c[0];
    out->walk_stack_spills = c[1];
    out->walk_groups = c[2];
    out->launches = b->launches;
    out->graph_launches = b->graph_launches;
    out->targets_per_lane = b->p.targets_per_lane;
    out->leaf_max = b->p.leaf_max;
    out->walk_mode = b->p.walk_mode;
    out->group_span = b->p.group_span;
    out->span_walk = b->span_on() ? 1 : 0;
    if (b->span_counters) {
      unsigned long long sc[3];
      nb::check(cudaMemcpy(sc, b->span_counters, sizeof(sc), cudaMemcpyDeviceToHost),
                "span counters");
      out->span_shared = sc[0];
      out->span_frontier = sc[1];
      out->spans = sc[2];
    }
  })
}

int nbody_sim_autotune(nbody_sim* s, const int* candidates, int n_candidates, float* ms_out) {
  NBODY_API_BODY({
    NBODY_REQUIRE(s, "nbody_sim_autotune: null simulation");
    NBODY_REQUIRE(s->impl->has_state, "nbody_sim_autotune: no state set");
    s->impl->advance(0, true);  // a pending second kick first
    NBODY_REQUIRE(!candidates || n_candidates >= 1, "nbody_sim_autotune: no candidates");
    s->impl->autotune(candidates, n_candidates, ms_out);
  })
}

int nbody_sim_set_graphs(nbody_sim* s, int on) {
  NBODY_API_BODY({
    NBODY_REQUIRE(s, "nbody_sim_set_graphs: null sim");
    if (!on) s->impl->drop_graphs();
    s->impl->use_graphs = on != 0;
  })
}

int nbody_sim_output_begin(nbody_sim* s, float link_length, float particle_mass,
                           float sim_time, int frame_index) {
  NBODY_API_BODY({
    NBODY_REQUIRE(s, "nbody_sim_output_begin: null sim");
    nb::SimBase* b = s->impl;
    NBODY_REQUIRE(b->has_state, "nbody_sim_output_begin: state not set");
    b->advance(0, true);  // a pending second kick first
    NBODY_REQUIRE(link_length >= 0.f, "nbody_sim_output_begin: negative link length");
    if (!b->pipe) b->pipe = new nb::OutputPipe(b->n, b->p.leaf_max);
    const int k = b->pipe->begin_slot();
    b->snapshot(b->pipe->slot[k].snap);
    b->pipe->launch(k, b->st, link_length, particle_mass, sim_time, frame_index);
  })
}

int nbody_sim_output_wait(nbody_sim* s, nbody_frame* out) {
  NBODY_API_BODY({
    NBODY_REQUIRE(s && out, "nbody_sim_output_wait: null argument");
    NBODY_REQUIRE(s->impl->pipe, "nbody_sim_output_wait: no frame in flight");
    s->impl->pipe->wait(out);
  })
}

int nbody_sim_step_host(nbody_sim* s, float* x, float* y, float* z, float* vx, float* vy,
                        float* vz, float* ax, float* ay, float* az, const float* mass,
                        int nsteps) {
  NBODY_API_BODY({
    NBODY_REQUIRE(s && x && y && z && vx && vy && vz && ax && ay && az && mass,
                  "nbody_sim_step_host: null array");
    nb::SimBase* b = s->impl;
    NBODY_REQUIRE(b->p.state_precision == NBODY_STATE_F32,
                  "nbody_sim_step_host: needs NBODY_STATE_F32");
    NBODY_REQUIRE(nsteps >= 0, "nbody_sim_step_host: negative step count");
    float* v[6] = {x, y, z, vx, vy, vz};
    float* a[3] = {ax, ay, az};
    b->step_host(v, a, mass, nsteps);  // copyToGPU, nsteps, copyToCPU
  })
}

}  // extern "C"


// ======================================================================
// Ensemble: independent disks of uneven size advanced together, every phase
// one launch over all disks.  Bodies carry their disk index; the Morton key
// gets the disk index above its 30 bits, so one radix sort orders all disks
// and the Karras tree splits by disk first.  Each disk is its own octree
// (root slot = disk index, own root cube), warp groups never span disks, and
// every group walks its own disk's tree with its own perturber.  A step is
// captured once per variant as a CUDA graph and replayed; the perturber
// table row it reads is a device counter that the step increments.
namespace nb {

template <typename R>
struct EnsembleImpl;

struct EnsembleBase {
  virtual ~EnsembleBase() {}
  nbody_sim_params p{};
  int D = 0, n = 0;
  cudaStream_t st = 0;
  bool has_state = false;
  int steps_done = 0;
  unsigned long long launches = 0, graph_launches = 0;
  virtual void set_stream(cudaStream_t s) = 0;
  virtual void set_state(const void* const* v, bool is_double, const float* mass,
                         bool on_device, bool forces = true) = 0;
  virtual void load_accel(const float* const* acc) = 0;
  // Host round trip of nbody_ensemble_step_host (double state arrays).
  virtual void step_host(double* const* v, float* const* a, const float* mass, int nsteps) = 0;
  virtual void step(int nsteps) = 0;
  virtual void get_state(void* const* v, bool as_double, float* const* a, bool on_device) = 0;
  virtual void autotune(const int* cand, int nc, float* ms) = 0;
  virtual void set_graphs(bool on) = 0;
  virtual void stats(nbody_ensemble_stats* out) = 0;
  virtual void sync() = 0;
};

template <typename R>
struct EnsembleImpl : EnsembleBase {
  int disk_bits = 0;
  std::vector<int> off;
  std::vector<nbody_perturber> pert;
  bool own_stream = false;
  TreeWork tw;
  uint64_t *keys64 = nullptr, *keys64_alt = nullptr;
  StateArrays<R> s[2]{};
  int cur = 0;
  float *ax = nullptr, *ay = nullptr, *az = nullptr, *dvx = nullptr, *dvy = nullptr,
        *dvz = nullptr;
  TreeGeom* geoms = nullptr;
  unsigned long long* bbox = nullptr;
  int* group_disk = nullptr;
  int* d_off = nullptr;
  float4* pert_tab = nullptr;
  int pert_rows = 0;
  int* pert_step = nullptr;
  int* spill = nullptr;
  int spill_cap = 4096;
  int* work = nullptr;
  unsigned long long* inter = nullptr;
  unsigned long long* counters = nullptr;
  void* staging = nullptr;
  void* out_stage = nullptr;
  bool use_graphs = true;
  cudaStream_t cap_st = nullptr;
  // [first step of a call?][state buffer at step start]
  cudaGraphExec_t gx[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  unsigned long long g_kernels[2][2] = {{0, 0}, {0, 0}};

  EnsembleImpl(const nbody_sim_params& prm, const nbody_disk_spec* disks, int nd) {
    p = prm;
    if (p.leaf_max <= 0) p.leaf_max = kLeafMaxSmall;
    if (p.targets_per_lane != 2) p.targets_per_lane = 1;
    if (p.walk_mode < 0 || p.walk_mode > 2) p.walk_mode = kDefaultWalkMode;
    if (p.group_span <= 0) p.group_span = 1;  // small compact disks: keep every group
    if (p.group_span > 64) p.group_span = 64;
    D = nd;
    while ((1 << disk_bits) < D) ++disk_bits;
    off.assign(D + 1, 0);
    pert.resize(D);
    for (int d = 0; d < D; ++d) {
      off[d + 1] = off[d] + disks[d].n;
      nbody_config c;
      nbody_config_defaults(&c);
      c.perturber_enabled = disks[d].perturber_enabled;
      c.perturber_mass_mjup = disks[d].perturber_mass_mjup;
      c.perturber_radius_AU = disks[d].perturber_radius_au;
      c.perturber_phase0 = disks[d].perturber_phase0;
      c.star_mass_msun = p.star_mass;
      nbody_perturber_make(&c, &pert[d]);
    }
    n = off[D];
    check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "ensemble stream");
    own_stream = true;
    tree_alloc(tw, n);
    tree_enable_overlap(tw);
    tw.group_max = 32 * p.targets_per_lane;
    tw.group_span = p.group_span;
    keys64 = dalloc<uint64_t>(n, "keys64");
    keys64_alt = dalloc<uint64_t>(n, "keys64_alt");
    for (int b = 0; b < 2; ++b) {
      for (int k = 0; k < 6; ++k) s[b].v[k] = dalloc<R>(n, "state");
      s[b].m = dalloc<float>(n, "mass");
      s[b].id = dalloc<int>(n, "id");
      s[b].disk = dalloc<int>(n, "disk");
    }
    ax = dalloc<float>(n, "ax"); ay = dalloc<float>(n, "ay"); az = dalloc<float>(n, "az");
    dvx = dalloc<float>(n, "dvx"); dvy = dalloc<float>(n, "dvy"); dvz = dalloc<float>(n, "dvz");
    geoms = dalloc<TreeGeom>(D, "geoms");
    bbox = dalloc<unsigned long long>(6 * (size_t)D, "bboxes");
    group_disk = dalloc<int>(n, "group disk");
    d_off = dalloc<int>(D + 1, "offsets");
    check(cudaMemcpy(d_off, off.data(), sizeof(int) * (D + 1), cudaMemcpyHostToDevice),
          "offsets");
    pert_step = dalloc<int>(1, "perturber row");
    spill_cap = p.spill_cap > 0 ? p.spill_cap : 4096;
    spill = dalloc<int>((size_t)walk_spill_slots(0) * spill_cap, "walk spill");
    work = dalloc<int>(1, "work");
    inter = dalloc<unsigned long long>(1, "inter");
    if (p.r_coll > 0.f) cs.alloc((size_t)walk_spill_slots(0) * spill_cap);
    check(cudaEventCreateWithFlags(&ev_pos, cudaEventDisableTiming), "position event");
    check(cudaStreamCreateWithFlags(&rb_st, cudaStreamNonBlocking), "read-back stream");
    counters = dalloc<unsigned long long>(3, "counters");
    staging = dalloc<double>(n, "staging");
    reserve_perturber_rows(64);
  }

  ~EnsembleImpl() override {
    if (st) cudaStreamSynchronize(st);
    drop_graphs();
    for (int b = 0; b < 2; ++b) {
      for (int k = 0; k < 6; ++k) cudaFree(s[b].v[k]);
      cudaFree(s[b].m); cudaFree(s[b].id); cudaFree(s[b].disk);
    }
    void* ptrs[] = {keys64, keys64_alt, ax,    ay,    az,         dvx,   dvy,
                    dvz,    geoms, bbox,  group_disk, d_off, pert_tab,
                    pert_step, spill,   work,  inter, counters,   staging, out_stage};
    for (void* q : ptrs)
      if (q) cudaFree(q);
    tree_free(tw);
    cs.release();
    if (rb_st) cudaStreamDestroy(rb_st);
    if (ev_pos) cudaEventDestroy(ev_pos);
    if (cap_st) cudaStreamDestroy(cap_st);
    if (own_stream && st) cudaStreamDestroy(st);
  }

  void drop_graphs() {
    for (auto& row : gx)
      for (auto& g : row)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  }

  void set_stream(cudaStream_t stream) override {
    check(cudaStreamSynchronize(st), "ensemble sync");
    drop_graphs();
    if (own_stream) cudaStreamDestroy(st);
    own_stream = false;
    st = stream;
  }

  void set_graphs(bool on) override {
    if (!on) drop_graphs();
    use_graphs = on;
  }

  void reserve_perturber_rows(int rows) {
    if (rows <= pert_rows) return;
    check(cudaStreamSynchronize(st), "perturber table sync");
    if (pert_tab) cudaFree(pert_tab);
    pert_rows = std::max(rows, 2 * pert_rows);
    pert_tab = dalloc<float4>((size_t)pert_rows * D, "perturber table");
    drop_graphs();  // the captured walks hold the old table
  }

  // Row k: every disk's perturber at t = (k0 + k) dt (updatePerturber,
  // Perturber.h:60-66, on the host as in the reference), mass 0 when off.
  void upload_perturbers(int k0, int count) {
    reserve_perturber_rows(count);
    std::vector<float4> h((size_t)count * D);
    for (int k = 0; k < count; ++k)
      for (int d = 0; d < D; ++d) {
        nbody_perturber q = pert[d];
        nbody_perturber_update(&q, (float)(k0 + k) * p.dt);
        h[(size_t)k * D + d] = make_float4(q.x, q.y, q.z, q.enabled ? q.mass_msun : 0.f);
      }
    check(cudaMemcpyAsync(pert_tab, h.data(), sizeof(float4) * h.size(), cudaMemcpyHostToDevice,
                          st),
          "perturber upload");
    check(cudaMemsetAsync(pert_step, 0, sizeof(int), st), "perturber row reset");
  }

  void set_state(const void* const* v, bool is_double, const float* mass, bool on_device,
                 bool forces) override {
    check(cudaStreamSynchronize(st), "ensemble sync");
    cur = 0;
    const size_t esz = is_double ? sizeof(double) : sizeof(float);
    for (int k = 0; k < 6; ++k) {
      const void* src = v[k];
      if (!on_device) {
        check(cudaMemcpyAsync(staging, src, esz * n, cudaMemcpyHostToDevice, st), "state H2D");
        src = staging;
      }
      if (is_double)
        k_convert<double, R><<<stream_grid(n), kThreads, 0, st>>>((const double*)src, s[0].v[k],
                                                                   n);
      else
        k_convert<float, R><<<stream_grid(n), kThreads, 0, st>>>((const float*)src, s[0].v[k], n);
    }
    check(cudaMemcpyAsync(s[0].m, mass, sizeof(float) * n,
                          on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st),
          "mass copy");
    k_iota<<<stream_grid(n), kThreads, 0, st>>>(s[0].id, n);
    k_disk_of<<<stream_grid(n), kThreads, 0, st>>>(d_off, D, n, s[0].disk);
    check(cudaGetLastError(), "ensemble state");
    launches += 8;
    steps_done = 0;
    has_state = true;
    if (forces) {
      upload_perturbers(0, 1);
      forces_from_scratch();
    } else {
      launch_bbox_reset_n(bbox, D, st);  // the next stream kernel accumulates them
      launches += 1;
    }
  }

  // Accelerations of the state just set (caller order is the current order).
  void load_accel(const float* const* acc) override {
    float* dst[3] = {ax, ay, az};
    for (int k = 0; k < 3; ++k)
      check(cudaMemcpyAsync(dst[k], acc[k], sizeof(float) * n, cudaMemcpyHostToDevice, st),
            "accel H2D");
  }

  // Bounding boxes of the current positions, then forces (no step).
  void forces_from_scratch() {
    launch_bbox_reset_n(bbox, D, st);
    k_bbox_multi<R><<<stream_grid(n), kThreads, 0, st>>>(s[cur], n, bbox);
    check(cudaGetLastError(), "k_bbox_multi launch");
    launches += 2;
    compute_forces();
  }

  // Keys, sort, permute into key order, tree, walk.  Leaves the bounding
  // boxes reset for the next stream kernel to accumulate.
  // with_coll: the step's forces, which may carry the fused collisions.
  void compute_forces(bool with_coll = false) {
    StateArrays<R>& a = s[cur];
    StateArrays<R>& b = s[1 - cur];
    const int key_bits = 30 + disk_bits;
    launch_geoms(bbox, geoms, D, st);
    uint32_t* hist = radix_sort_prepare(tw.counts, key_bits, st);  // counted by the key kernel
    launch_keys_multi<R>(a.v[0], a.v[1], a.v[2], a.disk, n, geoms, keys64, tw.perm, tw.status,
                         st, hist, key_bits);
    radix_sort_pairs<uint64_t>(keys64, tw.perm, keys64_alt, tw.perm_alt, tw.counts, n, key_bits,
                               st, tw.status, true);
    StepReset rs;
    rs.enc = bbox; rs.enc_words = 6 * D;
    rs.work = work; rs.inter = inter; rs.counters = counters;
    k_permute<R><<<moment_tiles(n), kMomentThreads, 0, st>>>(tw.perm, a, b, n, tw.body4, rs,
                                                             tw.mom_ploc, tw.mom_tiles);
    check(cudaGetLastError(), "k_permute launch");
    check(cudaEventRecordWithFlags(ev_pos, st, capturing ? cudaEventRecordExternal
                                                         : cudaEventRecordDefault),
          "position event");
    cur = 1 - cur;
    tw.prune_max = p.leaf_max;
    tw.boxes = p.r_coll > 0.f;  // only the collision searches read the records' boxes
    if (kIsF64<R>)
      launch_tree<uint64_t>(tw, keys64, n, key_bits, disk_bits, D, geoms, group_disk,
                            (const double*)s[cur].v[0], (const double*)s[cur].v[1],
                            (const double*)s[cur].v[2], st, true);
    else
      launch_tree<uint64_t>(tw, keys64, n, key_bits, disk_bits, D, geoms, group_disk, nullptr,
                            nullptr, nullptr, st, true);
    WalkArgs w{};
    w.com = tw.oct.com; w.info = tw.oct.info; w.body = tw.body4; w.n = n;
    w.groups = tw.groups; w.n_groups = tw.n_groups;
    w.theta2 = p.theta * p.theta; w.eps = p.softening; w.star_mass = p.star_mass;
    w.star_in_walk = kIsF32<R> ? 1 : 0;
    w.leaf_max = p.leaf_max;
    w.pert = pert_tab; w.pert_step = pert_step; w.n_disks = D; w.group_disk = group_disk;
    w.ax = ax; w.ay = ay; w.az = az; w.scatter = nullptr;
    w.spill = spill; w.spill_cap = spill_cap; w.inter = inter; w.counters = counters;
    w.work = work; w.status = tw.status; w.targets_per_lane = tw.group_max / 32;
    w.walk_mode = p.walk_mode;
    w.counters_zeroed = true;
    if (with_coll && coll_fused()) {
      for (int k = 0; k < 3; ++k) w.coll_v[k] = s[cur].v[3 + k];
      w.coll_vtype = kIsF32<R> ? 0 : (kIsF64<R> ? 1 : 2);
      w.coll_r = p.r_coll;
      w.coll_e = p.restitution;
      w.coll_dv[0] = dvx; w.coll_dv[1] = dvy; w.coll_dv[2] = dvz;
      w.box_lo = tw.oct.box_lo; w.box_hi = tw.oct.box_hi;
    }
    const bool side_coll = with_coll && p.r_coll > 0.f && !coll_fused();
    if (side_coll) {  // the collision pass on the second stream, beside the walk
      check(cudaEventRecord(cs.fork, st), "collision fork");
      check(cudaStreamWaitEvent(tw.side, cs.fork, 0), "collision fork");
      collide(tw.side, cs.work, cs.spill);
      check(cudaEventRecord(cs.join, tw.side), "collision join");
    }
    launch_walk(w, st);
    if (side_coll) check(cudaStreamWaitEvent(st, cs.join, 0), "collision join");
    // geoms, keys (+ digit histograms), one one-sweep kernel per pass,
    // permute (+ bbox and walk counter resets, + moment tiles), moment tile
    // scan, karras, mark, tile scan, apply, emit, walk
    launches += 2 + (key_bits + 7) / 8 + 8;
  }

  void collide(cudaStream_t on, int* wk, int* sp) {
    NeighborArgs na{tw.oct.info, tw.oct.box_lo, tw.oct.box_hi, tw.body4, n, tw.groups,
                    tw.n_groups, p.leaf_max, sp, spill_cap, wk, tw.status, group_disk};
    // the half-step velocities read in their storage type, rounded to float
    launch_collide_v(na, s[cur].v[3], s[cur].v[4], s[cur].v[5],
                     kIsF32<R> ? 0 : (kIsF64<R> ? 1 : 2), nullptr, p.r_coll, p.restitution,
                     dvx, dvy, dvz, on);
    launches += 1;
  }

  void stream_kernel(bool end, bool begin) {
    StreamArgs a{};
    a.ax = ax; a.ay = ay; a.az = az;
    const bool coll = p.r_coll > 0.f;
    a.dvx = coll ? dvx : nullptr; a.dvy = coll ? dvy : nullptr; a.dvz = coll ? dvz : nullptr;
    a.dt_f = p.dt; a.dth_f = p.dt * 0.5f;
    a.dt = (double)p.dt; a.dth = (double)p.dt * 0.5;
    const bool drag = p.gas_drag_rate > 0.f;
    a.decay_f = drag ? expf(-p.gas_drag_rate * p.dt) : 0.f;
    a.decay = drag ? std::exp(-(double)p.gas_drag_rate * (double)p.dt) : 0.0;
    a.eps = p.softening; a.star_mass = p.star_mass; a.bbox = bbox;
    const int g = stream_grid(n);
    if (end && begin) launch_stream<R, true, true, true>(s[cur], n, a, g, st);
    else if (end) launch_stream<R, true, false, true>(s[cur], n, a, g, st);
    else launch_stream<R, false, true, true>(s[cur], n, a, g, st);
    check(cudaGetLastError(), "k_stream launch");
    launches += 1;
  }

  // main.cu:101-139 for every disk: (dv + K2 + drag of the previous step),
  // K1 + drift + bbox, tree + walk (+ star, + perturber at t_{n+1}),
  // collisions on v_1/2; then the perturber row advances.
  CollSide cs;  // collisions beside the walk (r_coll > 0)
  // Recorded after every permute (an external event node in the step
  // graphs); the read-back stream of step_host waits on it.
  cudaEvent_t ev_pos = nullptr;
  cudaStream_t rb_st = nullptr;
  bool capturing = false;

  bool coll_fused() const {
    return p.r_coll > 0.f && p.fuse_collisions && tw.group_max == 32;
  }

  void one_step(bool first) {
    stream_kernel(!first, true);
    compute_forces(true);
    // (the collision pass, when r_coll > 0, runs inside compute_forces)
    k_increment<<<1, 1, 0, st>>>(pert_step);
    check(cudaGetLastError(), "k_increment launch");
    launches += 1;
  }

  // The step's launches have fixed pointers and sizes; only the state buffer
  // the step starts from (it flips at the permute) and whether the previous
  // step's closing kick is pending change, so four graphs cover every step.
  cudaGraphExec_t graph_for(bool first) {
    const int f = first ? 1 : 0, c = cur;
    if (gx[f][c]) return gx[f][c];
    cudaGraph_t graph = nullptr;
    const unsigned long long l0 = launches;
    // Captured on a private stream (the caller's may be the legacy default
    // stream, which cannot capture) and launched on the caller's.
    if (!cap_st) check(cudaStreamCreateWithFlags(&cap_st, cudaStreamNonBlocking), "capture stream");
    cudaStream_t user = st;
    st = cap_st;
    check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
    capturing = true;
    one_step(first);
    capturing = false;
    const cudaError_t ce = cudaStreamEndCapture(st, &graph);
    st = user;
    check(ce, "end capture");
    cur = c;  // captured, not run
    g_kernels[f][c] = launches - l0;
    launches = l0;
    check(cudaGraphInstantiate(&gx[f][c], graph, 0), "graph instantiate");
    cudaGraphDestroy(graph);
    return gx[f][c];
  }

  void step(int nsteps) override {
    if (nsteps <= 0) return;
    upload_perturbers(steps_done + 1, nsteps);
    for (int k = 0; k < nsteps; ++k) {
      const bool first = (k == 0);
      if (use_graphs) {
        const int f = first ? 1 : 0, c = cur;
        check(cudaGraphLaunch(graph_for(first), st), "graph launch");
        launches += g_kernels[f][c];
        graph_launches += 1;
        cur = 1 - cur;
      } else {
        one_step(first);
      }
    }
    stream_kernel(true, false);
    steps_done += nsteps;
  }

  void get_state(void* const* v, bool as_double, float* const* acc, bool on_device) override {
    if (!on_device && !out_stage) out_stage = dalloc<char>(out_stage_bytes(n), "output staging");
    state_out<R>(s[cur], n, ax, ay, az, p.softening, p.star_mass, v, as_double, acc, on_device,
                 out_stage, st);
    launches += 1;
  }

  // copyToGPU, nsteps, copyToCPU; the positions go back on the read-back
  // stream as soon as the last permute has run.
  void step_host(double* const* v, float* const* acc, const float* mass, int nsteps) override {
    const int steps0 = has_state ? steps_done : 0;
    const void* vin[6] = {v[0], v[1], v[2], v[3], v[4], v[5]};
    const float* ain[3] = {acc[0], acc[1], acc[2]};
    set_state(vin, true, mass, false, false);
    load_accel(ain);
    steps_done = steps0;  // the caller's clock continues
    if (nsteps <= 0) {
      void* vout[6] = {v[0], v[1], v[2], v[3], v[4], v[5]};
      get_state(vout, true, acc, false);
      return;
    }
    step(nsteps);
    if (!out_stage) out_stage = dalloc<char>(out_stage_bytes(n), "output staging");
    read_back_split<R, double>(s[cur], n, ax, ay, az, p.softening, p.star_mass, v, acc,
                               out_stage, ev_pos, rb_st, st);
    launches += 2;
  }

  // Candidates are (targets per lane, leaf size, walk mode) triples.
  void autotune(const int* cand, int nc, float* ms_out) override {
    static const int kDefault[] = {1, 8, 0, 1, 8, 1, 1, 8, 2, 1, 4, 2, 1, 16, 2, 2, 8, 0};
    if (!cand) {
      cand = kDefault;
      nc = 6;
    }
    auto apply = [&](int k) {
      p.targets_per_lane = cand[3 * k] == 2 ? 2 : 1;
      p.leaf_max = std::max(1, cand[3 * k + 1]);
      p.walk_mode = (cand[3 * k + 2] >= 0 && cand[3 * k + 2] <= 2) ? cand[3 * k + 2]
                                                                : kDefaultWalkMode;
      tw.group_max = 32 * p.targets_per_lane;
    };
    upload_perturbers(steps_done, 1);  // the forces of the current time
    cudaEvent_t e0, e1;
    check(cudaEventCreate(&e0), "event");
    check(cudaEventCreate(&e1), "event");
    float best = 0.f;
    int best_k = -1;
    for (int k = 0; k < nc; ++k) {
      apply(k);
      forces_from_scratch();  // warm-up with this setting
      float ms = 0.f;
      for (int rep = 0; rep < 2; ++rep) {  // best of two timed evaluations
        check(cudaEventRecord(e0, st), "event");
        forces_from_scratch();
        check(cudaEventRecord(e1, st), "event");
        check(cudaEventSynchronize(e1), "event sync");
        float t = 0.f;
        check(cudaEventElapsedTime(&t, e0, e1), "event time");
        ms = (rep == 0) ? t : std::min(ms, t);
      }
      if (ms_out) ms_out[k] = ms;
      if (best_k < 0 || ms < best) {
        best = ms;
        best_k = k;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    apply(best_k);
    drop_graphs();
    forces_from_scratch();
  }

  void stats(nbody_ensemble_stats* out) override {
    check(cudaStreamSynchronize(st), "ensemble sync");
    out->n_disks = D;
    out->n_total = n;
    out->steps_done = steps_done;
    out->targets_per_lane = p.targets_per_lane;
    out->leaf_max = p.leaf_max;
    out->walk_mode = p.walk_mode;
    check(cudaMemcpy(&out->status, tw.status, sizeof(int), cudaMemcpyDeviceToHost), "status");
    check(cudaMemcpy(&out->interactions, inter, sizeof(unsigned long long),
                     cudaMemcpyDeviceToHost),
          "interactions");
    out->launches = launches;
    out->graph_launches = graph_launches;
  }

  void sync() override {
    int s = 0;
    check(cudaStreamSynchronize(st), "ensemble sync");
    check(cudaMemcpy(&s, tw.status, sizeof(int), cudaMemcpyDeviceToHost), "status read");
    if (s) {
      check(cudaMemsetAsync(tw.status, 0, sizeof(int), st), "status reset");
      throw ArgError("device status " + std::to_string(s) +
                         " (1 walk stack, 2 union-find, 4 tree, 8 non-finite position, 16 tape, 32 sort wait)",
                     NBODY_ERR_OVERFLOW);
    }
  }
};

EnsembleBase* make_ensemble(const nbody_sim_params& p, const nbody_disk_spec* d, int nd) {
  if (p.state_precision == NBODY_STATE_F64) return new EnsembleImpl<double>(p, d, nd);
  if (p.state_precision == NBODY_STATE_F32X2) return new EnsembleImpl<HiLo>(p, d, nd);
  return new EnsembleImpl<float>(p, d, nd);
}

}  // namespace nb

struct nbody_ensemble {
  nb::EnsembleBase* impl;
};

extern "C" {

int nbody_ensemble_create(const nbody_sim_params* p, const nbody_disk_spec* disks, int n_disks,
                          nbody_ensemble** out) {
  NBODY_API_BODY({
    NBODY_REQUIRE(p && disks && out, "nbody_ensemble_create: null argument");
    *out = nullptr;
    NBODY_REQUIRE(n_disks >= 1 && n_disks <= (1 << 20),
                  "nbody_ensemble_create: n_disks must be in [1, 2^20]");
    long long total = 0;
    for (int d = 0; d < n_disks; ++d) {
      NBODY_REQUIRE(disks[d].n >= 2, "nbody_ensemble_create: every disk needs >= 2 bodies");
      total += disks[d].n;
    }
    NBODY_REQUIRE(total < (1 << 27), "nbody_ensemble_create: total bodies must be < 2^27");
    NBODY_REQUIRE(p->dt > 0.f, "nbody_ensemble_create: dt must be positive");
    NBODY_REQUIRE(p->state_precision >= NBODY_STATE_F32 && p->state_precision <= NBODY_STATE_F32X2,
                  "nbody_ensemble_create: unknown state precision");
    *out = new nbody_ensemble{nb::make_ensemble(*p, disks, n_disks)};
  })
}

int nbody_ensemble_destroy(nbody_ensemble* e) {
  NBODY_API_BODY({
    if (e) {
      delete e->impl;
      delete e;
    }
  })
}

int nbody_ensemble_set_stream(nbody_ensemble* e, void* stream) {
  NBODY_API_BODY({
    NBODY_REQUIRE(e, "nbody_ensemble_set_stream: null ensemble");
    e->impl->set_stream((cudaStream_t)stream);
  })
}

int nbody_ensemble_set_state(nbody_ensemble* e, const float* x, const float* y, const float* z,
                             const float* vx, const float* vy, const float* vz,
                             const float* mass, int on_device) {
  NBODY_API_BODY({
    NBODY_REQUIRE(e && x && y && z && vx && vy && vz && mass,
                  "nbody_ensemble_set_state: null array");
    const void* v[6] = {x, y, z, vx, vy, vz};
    e->impl->set_state(v, false, mass, on_device != 0, true);
  })
}

int nbody_ensemble_set_state_f64(nbody_ensemble* e, const double* x, const double* y,
                                 const double* z, const double* vx, const double* vy,
                                 const double* vz, const float* mass, int on_device) {
  NBODY_API_BODY({
    NBODY_REQUIRE(e && x && y && z && vx && vy && vz && mass,
                  "nbody_ensemble_set_state_f64: null array");
    const void* v[6] = {x, y, z, vx, vy, vz};
    e->impl->set_state(v, true, mass, on_device != 0, true);
  })
}

int nbody_ensemble_step(nbody_ensemble* e, int nsteps) {
  NBODY_API_BODY({
    NBODY_REQUIRE(e, "nbody_ensemble_step: null ensemble");
    NBODY_REQUIRE(e->impl->has_state, "nbody_ensemble_step: state not set");
    NBODY_REQUIRE(nsteps >= 0, "nbody_ensemble_step: negative step count");
    e->impl->step(nsteps);
  })
}

int nbody_ensemble_sync(nbody_ensemble* e) {
  NBODY_API_BODY({
    NBODY_REQUIRE(e, "nbody_ensemble_sync: null ensemble");
    e->impl->sync();
  })
}

int nbody_ensemble_get_state(nbody_ensemble* e, float* x, float* y, float* z, float* vx,
                             float* vy, float* vz, float* ax, float* ay, float* az,
                             int on_device) {
  NBODY_API_BODY({
    NBODY_REQUIRE(e && x && y && z && vx && vy && vz, "nbody_ensemble_get_state: null array");
    NBODY_REQUIRE(e->impl->has_state, "nbody_ensemble_get_state: state not set");
    void* v[6] = {x, y, z, vx, vy, vz};
    float* a[3] = {ax, ay, az};
    e->impl->get_state(v, false, (ax && ay && az) ? a : nullptr, on_device != 0);
  })
}

int nbody_ensemble_get_state_f64(nbody_ensemble* e, double* x, double* y, double* z,
                                 double* vx, double* vy, double* vz, float* ax, float* ay,
                                 float* az, int on_device) {
  NBODY_API_BODY({
    NBODY_REQUIRE(e && x && y && z && vx && vy && vz,
                  "nbody_ensemble_get_state_f64: null array");
    NBODY_REQUIRE(e->impl->has_state, "nbody_ensemble_get_state_f64: state not set");
    void* v[6] = {x, y, z, vx, vy, vz};
    float* a[3] = {ax, ay, az};
    e->impl->get_state(v, true, (ax && ay && az) ? a : nullptr, on_device != 0);
  })
}

int nbody_ensemble_step_host(nbody_ensemble* e, double* x, double* y, double* z, double* vx,
                             double* vy, double* vz, float* ax, float* ay, float* az,
                             const float* mass, int nsteps) {
  NBODY_API_BODY({
    NBODY_REQUIRE(e && x && y && z && vx && vy && vz && ax && ay && az && mass,
                  "nbody_ensemble_step_host: null array");
    NBODY_REQUIRE(nsteps >= 0, "nbody_ensemble_step_host: negative step count");
    double* v[6] = {x, y, z, vx, vy, vz};
    float* a[3] = {ax, ay, az};
    e->impl->step_host(v, a, mass, nsteps);  // copyToGPU, nsteps, copyToCPU
  })
}

int nbody_ensemble_autotune(nbody_ensemble* e, const int* candidates, int n_candidates,
                            float* ms_out) {
  NBODY_API_BODY({
    NBODY_REQUIRE(e, "nbody_ensemble_autotune: null ensemble");
    NBODY_REQUIRE(e->impl->has_state, "nbody_ensemble_autotune: state not set");
    NBODY_REQUIRE(!candidates || n_candidates >= 1,
                  "nbody_ensemble_autotune: empty candidate list");
    e->impl->autotune(candidates, n_candidates, ms_out);
  })
}

int nbody_ensemble_set_graphs(nbody_ensemble* e, int on) {
  NBODY_API_BODY({
    NBODY_REQUIRE(e, "nbody_ensemble_set_graphs: null ensemble");
    e->impl->set_graphs(on != 0);
  })
}

int nbody_ensemble_stats_get(nbody_ensemble* e, nbody_ensemble_stats* out) {
  NBODY_API_BODY({
    NBODY_REQUIRE(e && out, "nbody_ensemble_stats_get: null argument");
    e->impl->stats(out);
  })
}

}  // extern "C"
