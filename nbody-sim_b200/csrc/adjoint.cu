// adjoint.cu -- reverse-mode derivatives of a disk's trajectory through the
// frozen Barnes-Hut tree.
//
// The differentiable step is the reference's step order (src/main.cu:101-139:
// K1, drift, tree + force, perturber, K2, gas drag; no collisions) with FP64
// state.  Self-gravity comes from the FP32 tree walk; the star pull
// (BHTree.cu:547-553 form), the perturber pull (Perturber.cu:20-34 form,
// position as updatePerturber, Perturber.h:60-66) and the drag
// (Integrator.cu:47-75) are FP64.
//
// Forward: every step records its tape -- the sort permutation, the warp
// groups and each group's source list as sorted body ranges in evaluation
// order (a recording variant of the walk) -- and the states of every time
// level.  All of it stays in HBM.
//
// Backward: the exact adjoint of that computation with the tree frozen
// (same permutations, groups and source lists).  Per level, the tape is
// replayed with the interaction's vector-Jacobian product: the target side
// accumulates -g (FP32 within a 32-source chunk, FP64 across chunks), the source side adds +g to its centre of mass,
// whose adjoint reaches each member body j in proportion m_j / M_node (a
// range add over the sorted body range, resolved by one prefix sum).  The
// star, perturber and drag Jacobians are applied per body in FP64; the
// perturber's position and mass adjoints are reduced per level and chained
// to (mass in M_J, orbit radius) on the host.
//
// Replay: the same frozen-tree forward with other initial conditions or
// perturber parameters -- the function the backward differentiates, used
// for finite-difference checks.
#include <algorithm>
#include <cmath>
#include <vector>

#include "capi_util.h"
#include "common.cuh"
#include "kernels.cuh"
#include "moments.cuh"
#include "physics.cuh"
#include "walk_math.cuh"

namespace nb {
namespace {

constexpr int kThreads = 256;
constexpr int kRW = 4;  // warps per block of the replay kernels
constexpr int kTapeChunk = 32;

int grid1(long long n) { return std::max(1, std::min(div_up(n, kThreads), 148 * 8)); }

template <typename T>
T* dalloc(size_t count, const char* what) {
  T* p = nullptr;
  check(cudaMalloc(&p, sizeof(T) * (count ? count : 1)), what);
  return p;
}

// Sorted FP64 positions and float bodies of level positions (caller order).
__global__ void k_gather_sorted(const uint32_t* __restrict__ perm, const double* __restrict__ x,
                                const double* __restrict__ y, const double* __restrict__ z,
                                const float* __restrict__ m, int n, double* __restrict__ xs,
                                double* __restrict__ ys, double* __restrict__ zs,
                                float4* __restrict__ body4) {
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
       s += (long long)gridDim.x * blockDim.x) {
    const uint32_t o = perm[s];
    const double px = x[o], py = y[o], pz = z[o];
    xs[s] = px; ys[s] = py; zs[s] = pz;
    body4[s] = make_float4((float)px, (float)py, (float)pz, m[o]);
  }
}

__global__ void k_copy_groups(const int2* __restrict__ src, const int* __restrict__ n_groups,
                              int n, int2* __restrict__ dst, int* __restrict__ n_dst) {
  const int ng = *n_groups;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < n;
       g += (long long)gridDim.x * blockDim.x)
    if (g < ng) dst[g] = src[g];
  if (blockIdx.x == 0 && threadIdx.x == 0) *n_dst = ng;
}

// FP64 acceleration of body o at level positions: float self-gravity plus the
// softened star and perturber pulls.
template <typename TA>
__device__ __forceinline__ void total_accel(double x, double y, double z, TA sx, TA sy, TA sz,
                                            double eps, double star_mass, double4 p, double& ax,
                                            double& ay, double& az) {
  double tx, ty, tz;
  star_accel<double>(x, y, z, eps, star_mass, tx, ty, tz);
  ax = (double)sx + tx;
  ay = (double)sy + ty;
  az = (double)sz + tz;
  if (p.w != 0.0) {
    const double dx = p.x - x, dy = p.y - y, dz = p.z - z;
    const double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, __dmul_rn(eps, eps))));
    const double f = p.w / __dmul_rn(r2, sqrt(r2));
    ax = fma(f, dx, ax);
    ay = fma(f, dy, ay);
    az = fma(f, dz, az);
  }
}

template <typename TA>
struct StepArgsT {
  const double* x;   // level-L positions (caller order)
  const double* y;
  const double* z;
  double* vx;        // in: v' of step L-1 (kEnd) or v_L; out: v_h of step L
  double* vy;
  double* vz;
  const TA* ax;      // level-L self-gravity (float from the walk, double from
  const TA* ay;      // the FP64 replay)
  const TA* az;
  double* lvx;       // out (optional): v_L
  double* lvy;
  double* lvz;
  double* nx;        // out (kBegin): level L+1 positions
  double* ny;
  double* nz;
  const double4* pert_tab;  // perturber (x, y, z, mass in M_sun) per level
  int level;
  double eps, star_mass, dt, dth, decay;
  int drag;
  int n;
};
using StepArgs = StepArgsT<float>;

// Boundary of level L: [K2 + drag of step L-1] then [K1 + drift of step L].
template <bool kEnd, bool kBegin, typename TA>
__global__ void __launch_bounds__(kThreads) k_dstep(const StepArgsT<TA> a) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n;
       i += (long long)gridDim.x * blockDim.x) {
    const double x = a.x[i], y = a.y[i], z = a.z[i];
    double vx = a.vx[i], vy = a.vy[i], vz = a.vz[i];
    double ax, ay, az;
    total_accel(x, y, z, a.ax[i], a.ay[i], a.az[i], a.eps, a.star_mass, a.pert_tab[a.level], ax,
                ay, az);
    if (kEnd) {
      vx = fma(ax, a.dth, vx); vy = fma(ay, a.dth, vy); vz = fma(az, a.dth, vz);
      if (a.drag) gas_drag<double>(x, z, vx, vy, vz, a.decay, a.star_mass);
    }
    if (a.lvx) { a.lvx[i] = vx; a.lvy[i] = vy; a.lvz[i] = vz; }
    if (kBegin) {
      vx = fma(ax, a.dth, vx); vy = fma(ay, a.dth, vy); vz = fma(az, a.dth, vz);
      a.nx[i] = fma(vx, a.dt, x); a.ny[i] = fma(vy, a.dt, y); a.nz[i] = fma(vz, a.dt, z);
    }
    a.vx[i] = vx; a.vy[i] = vy; a.vz[i] = vz;
  }
}

// ------------------------------------------------------------ tape replay
struct ReplayArgs {
  const float4* body4;      // level bodies, sorted order
  const double4* ploc;      // moment prefix (range_moments)
  const double4* tpre;
  const uint32_t* perm;     // sorted -> caller
  const int2* groups;
  const int* n_groups;
  const int2* group_tape;
  const int2* tape;
  const int* tape_next;
  float eps2;
  int* work;
  int* status;
  // forward replay: self-gravity out (caller order), float or (FP64 replay)
  // double
  float* ax;
  float* ay;
  float* az;
  double* dax;
  double* day;
  double* daz;
  const double* xs;         // FP64 replay: sorted FP64 positions
  const double* ys;
  const double* zs;
  // adjoint replay: lam in (caller order), mu out (sorted), range adds
  const double* lx;
  const double* ly;
  const double* lz;
  double* mux;
  double* muy;
  double* muz;
  double4* radd;            // n + 1 entries
};

struct ReplaySmem {
  double4 dlst[32];  // FP64 replay sources
  // FP32 sources, one row per component (x, y, z, mass): two entries of a
  // row from an even index are one 8-byte load into a register pair
  float src[4][32];
  int2 ent[32];
  double mass[32];
  // the group's targets, one row per component: negated x, y, z, then the
  // adjoint's x, y, z
  float tgt[6][32];
  int tid[32];
};

__device__ __forceinline__ float2 row2(const float* r, int j) {
  return *reinterpret_cast<const float2*>(r + j);
}

__device__ __forceinline__ float4 src_at(const ReplaySmem& w, int j) {
  return make_float4(w.src[0][j], w.src[1][j], w.src[2][j], w.src[3][j]);
}

// Loads up to 32 entries of the tape chain into the warp's list: source
// float4 (centre of mass from the FP64 prefix sums, or the body itself).
__device__ __forceinline__ void load_chunk(const ReplayArgs& a, ReplaySmem& w, int chunk, int k,
                                           int lane) {
  if (lane < k) {
    const int2 e = a.tape[(size_t)chunk * kTapeChunk + lane];
    float4 src;
    double m;
    if (e.y == 1) {
      src = a.body4[e.x];
      m = (double)src.w;
    } else {
      const double4 s = range_moments(a.ploc, a.tpre, e.x, e.x + e.y);
      src = com_of(s, 0.f, 0.f, 0.f);
      m = s.x;
    }
    w.src[0][lane] = src.x;
    w.src[1][lane] = src.y;
    w.src[2][lane] = src.z;
    w.src[3][lane] = src.w;
    w.ent[lane] = e;
    w.mass[lane] = m;
  }
  __syncwarp();
}

// FP64 replay source: the body's FP64 position, or the node's FP64 centre
// of mass, with its mass.
__device__ __forceinline__ void load_chunk64(const ReplayArgs& a, ReplaySmem& w, int chunk,
                                             int k, int lane) {
  if (lane < k) {
    const int2 e = a.tape[(size_t)chunk * kTapeChunk + lane];
    if (e.y == 1) {
      w.dlst[lane] = make_double4(a.xs[e.x], a.ys[e.x], a.zs[e.x], (double)a.body4[e.x].w);
    } else {
      const double4 s = range_moments(a.ploc, a.tpre, e.x, e.x + e.y);
      const double inv = 1.0 / s.x;
      w.dlst[lane] = make_double4(s.y * inv, s.z * inv, s.w * inv, s.x);
    }
  }
  __syncwarp();
}

// The frozen-tree forward with FP64 interactions (the finite-difference
// reference: free of the FP32 rounding that the perturbed body's own terms
// would otherwise add to a difference quotient).
__global__ void __launch_bounds__(kRW * 32) k_replay64(const ReplayArgs a) {
  __shared__ ReplaySmem smem[kRW];
  const int lane = threadIdx.x & 31;
  ReplaySmem& w = smem[threadIdx.x >> 5];
  const int n_groups = *a.n_groups;
  const double eps2 = (double)a.eps2;
  while (true) {
    int g = 0;
    if (lane == 0) g = atomicAdd(a.work, 1);
    g = __shfl_sync(kFull, g, 0);
    if (g >= n_groups) break;
    const int2 gr = a.groups[g];
    const int2 gt = a.group_tape[g];
    const bool valid = lane < gr.y;
    const int s = gr.x + (valid ? lane : 0);
    const double px = a.xs[s], py = a.ys[s], pz = a.zs[s];
    double sx = 0.0, sy = 0.0, sz = 0.0;
    int chunk = gt.x, done = 0;
    while (done < gt.y) {
      const int k = min(kTapeChunk, gt.y - done);
      load_chunk64(a, w, chunk, k, lane);
      for (int j = 0; j < k; ++j) {
        const double4 q = w.dlst[j];
        const double dx = q.x - px, dy = q.y - py, dz = q.z - pz;
        const double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
        if (r2 <= 0.0) continue;
        const double inv = 1.0 / sqrt(r2);
        const double f = q.w * inv * inv * inv;
        sx = fma(f, dx, sx); sy = fma(f, dy, sy); sz = fma(f, dz, sz);
      }
      __syncwarp();
      done += k;
      if (done < gt.y) chunk = a.tape_next[chunk];
      if (chunk < 0 && done < gt.y) {
        if (lane == 0) atomicOr(a.status, kStatusTapeFull);
        break;
      }
    }
    if (valid) {
      const uint32_t o = a.perm[s];
      a.dax[o] = sx; a.day[o] = sy; a.daz[o] = sz;
    }
  }
}

template <bool kSoft, bool kAdj>
__global__ void __launch_bounds__(kRW * 32) k_replay(const ReplayArgs a) {
  __shared__ ReplaySmem smem[kRW];
  const int lane = threadIdx.x & 31;
  ReplaySmem& w = smem[threadIdx.x >> 5];
  const int n_groups = *a.n_groups;
  while (true) {
    int g = 0;
    if (lane == 0) g = atomicAdd(a.work, 1);
    g = __shfl_sync(kFull, g, 0);
    if (g >= n_groups) break;
    const int2 gr = a.groups[g];
    const int2 gt = a.group_tape[g];
    if (gt.x < 0 && gt.y > 0) {  // never recorded (tape ran out)
      if (lane == 0) atomicOr(a.status, kStatusTapeFull);
      continue;
    }
    const bool valid = lane < gr.y;
    const int s = gr.x + (valid ? lane : 0);
    const float4 me = a.body4[s];
    const uint32_t o = a.perm[s];
    float3 acc = make_float3(0.f, 0.f, 0.f);
    float3 lam = make_float3(0.f, 0.f, 0.f);
    double mx = 0.0, my = 0.0, mz = 0.0;
    if (kAdj) {
      if (valid) lam = make_float3((float)a.lx[o], (float)a.ly[o], (float)a.lz[o]);
      w.tgt[0][lane] = -me.x;
      w.tgt[1][lane] = -me.y;
      w.tgt[2][lane] = -me.z;
      w.tgt[3][lane] = lam.x;
      w.tgt[4][lane] = lam.y;
      w.tgt[5][lane] = lam.z;
      w.tid[lane] = valid ? s : -1;
      __syncwarp();
    }
    int chunk = gt.x, done = 0;
    while (done < gt.y) {
      const int k = min(kTapeChunk, gt.y - done);
      load_chunk(a, w, chunk, k, lane);
      if (!kAdj) {
        for (int j = 0; j < k; ++j) interact<kSoft>(src_at(w, j), me, a.eps2, acc);
      } else {
        const float2 e2 = make_float2(a.eps2, a.eps2);
        // target side: -g for every source except the body itself (a mass of
        // 0), sources in pairs through the packed product, summed over the
        // chunk (<= 32 terms) in FP32, the chunk sums in FP64
        PairTgt me2;
        me2.x = make_float2(-me.x, -me.x);
        me2.y = make_float2(-me.y, -me.y);
        me2.z = make_float2(-me.z, -me.z);
        const float2 l2x = make_float2(lam.x, lam.x), l2y = make_float2(lam.y, lam.y);
        const float2 l2z = make_float2(lam.z, lam.z);
        PairAcc p2;
        p2.x = p2.y = p2.z = make_float2(0.f, 0.f);
        int j = 0;
        for (; j + 2 <= k; j += 2) {
          const int4 ee = *reinterpret_cast<const int4*>(&w.ent[j]);
          float2 m2 = row2(w.src[3], j);
          if (ee.y == 1 && ee.x == s) m2.x = 0.f;
          if (ee.w == 1 && ee.z == s) m2.y = 0.f;
          interact_vjp2<kSoft>(row2(w.src[0], j), row2(w.src[1], j), row2(w.src[2], j), m2, me2,
                               e2, l2x, l2y, l2z, p2);
        }
        float3 part = make_float3(p2.x.x + p2.x.y, p2.y.x + p2.y.y, p2.z.x + p2.z.y);
        for (; j < k; ++j) {
          const int2 e = w.ent[j];
          if (e.y == 1 && e.x == s) continue;
          const float3 gv = interact_vjp<kSoft>(src_at(w, j), me, a.eps2, lam);
          part.x += gv.x; part.y += gv.y; part.z += gv.z;
        }
        mx -= (double)part.x; my -= (double)part.y; mz -= (double)part.z;
        // source side: lane j sums +g over the group's targets, in pairs of
        // targets, and spreads it over the source's bodies in proportion to
        // their mass
        if (lane < k) {
          const float4 src = src_at(w, lane);
          const int2 e = w.ent[lane];
          const float2 s2x = make_float2(src.x, src.x), s2y = make_float2(src.y, src.y);
          const float2 s2z = make_float2(src.z, src.z);
          const bool single = e.y == 1;
          PairAcc g2;
          g2.x = g2.y = g2.z = make_float2(0.f, 0.f);
          int t = 0;
          for (; t + 2 <= gr.y; t += 2) {
            const int2 ids = *reinterpret_cast<const int2*>(&w.tid[t]);
            float2 m2 = make_float2(src.w, src.w);
            if (single && e.x == ids.x) m2.x = 0.f;
            if (single && e.x == ids.y) m2.y = 0.f;
            PairTgt tp;
            tp.x = row2(w.tgt[0], t);
            tp.y = row2(w.tgt[1], t);
            tp.z = row2(w.tgt[2], t);
            interact_vjp2<kSoft>(s2x, s2y, s2z, m2, tp, e2, row2(w.tgt[3], t),
                                 row2(w.tgt[4], t), row2(w.tgt[5], t), g2);
          }
          float3 gs = make_float3(g2.x.x + g2.x.y, g2.y.x + g2.y.y, g2.z.x + g2.z.y);
          for (; t < gr.y; ++t) {
            if (single && e.x == w.tid[t]) continue;
            const float4 tp = make_float4(-w.tgt[0][t], -w.tgt[1][t], -w.tgt[2][t], 0.f);
            const float3 gv = interact_vjp<kSoft>(src, tp, a.eps2,
                                                  make_float3(w.tgt[3][t], w.tgt[4][t],
                                                              w.tgt[5][t]));
            gs.x += gv.x; gs.y += gv.y; gs.z += gv.z;
          }
          const double inv = 1.0 / w.mass[lane];
          const double wx = (double)gs.x * inv, wy = (double)gs.y * inv, wz = (double)gs.z * inv;
          double4* lo = a.radd + e.x;
          double4* hi = a.radd + e.x + e.y;
          atomicAdd(&lo->x, wx); atomicAdd(&lo->y, wy); atomicAdd(&lo->z, wz);
          atomicAdd(&hi->x, -wx); atomicAdd(&hi->y, -wy); atomicAdd(&hi->z, -wz);
        }
      }
      __syncwarp();
      done += k;
      if (done < gt.y) chunk = a.tape_next[chunk];
      if (chunk < 0 && done < gt.y) {  // broken chain: stop, report
        if (lane == 0) atomicOr(a.status, kStatusTapeFull);
        break;
      }
    }
    if (valid) {
      if (!kAdj) {
        a.ax[o] = acc.x; a.ay[o] = acc.y; a.az[o] = acc.z;
      } else {
        a.mux[s] = mx; a.muy[s] = my; a.muz[s] = mz;
      }
    }
  }
}

// Exclusive tile-local prefix sums of a double4 array in the layout of the
// moment prefix (index i: sum over [tile start, i)), and the tile totals.
__global__ void __launch_bounds__(kThreads)
k_prefix4_tiles(const double4* __restrict__ in, int n, double4* __restrict__ ploc,
                double4* __restrict__ tile_sum) {
  constexpr int kPer = kMomentTile / kThreads;
  __shared__ double4 s_w[kThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long base = (long long)blockIdx.x * kMomentTile + (long long)tid * kPer;
  double4 v[kPer];
  double4 sum = make_double4(0, 0, 0, 0);
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    const long long i = base + k;
    v[k] = (i < n) ? in[i] : make_double4(0, 0, 0, 0);
    sum = d4add(sum, v[k]);
  }
  double4 inc = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double4 t = make_double4(__shfl_up_sync(kFull, inc.x, o), __shfl_up_sync(kFull, inc.y, o),
                                   __shfl_up_sync(kFull, inc.z, o), __shfl_up_sync(kFull, inc.w, o));
    if (lane >= o) inc = d4add(inc, t);
  }
  if (lane == 31) s_w[warp] = inc;
  __syncthreads();
  double4 run = d4sub(inc, sum);
  for (int q = 0; q < warp; ++q) run = d4add(run, s_w[q]);
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    const long long i = base + k;
    if (i <= n) ploc[i] = run;
    run = d4add(run, v[k]);
  }
  if (tid == kThreads - 1) tile_sum[blockIdx.x] = run;
}

// Exclusive scan of the tile totals (one warp, fixed order).
__global__ void k_tiles_scan4(const double4* __restrict__ tile_sum, int ntiles,
                              double4* __restrict__ tpre) {
  if (threadIdx.x != 0) return;
  double4 run = make_double4(0, 0, 0, 0);
  for (int t = 0; t <= ntiles; ++t) {
    tpre[t] = run;
    if (t < ntiles) run = d4add(run, tile_sum[t]);
  }
}

struct ApplyArgs {
  const uint32_t* perm;
  const float4* body4;
  const double* mux;
  const double* muy;
  const double* muz;
  const double4* rploc;     // prefix of the range adds
  const double4* rtpre;
  const double* x;          // level positions (caller order)
  const double* y;
  const double* z;
  const double* lx;         // adjoint of the level's acceleration
  const double* ly;
  const double* lz;
  double* gx;               // position adjoint (in/out)
  double* gy;
  double* gz;
  double* gvx;              // velocity adjoint: v_h of the step that ends here
  double* gvy;
  double* gvz;
  double* plx;              // out: pending acceleration adjoint dt/2 V_h
  double* ply;
  double* plz;
  const double4* pert_tab;
  int level;
  double eps, star_mass, dt, dth;
  double* pgrad;            // 4 per level: adjoint of perturber x, y, z, mass
  int n;
};

// Per body (sorted index s, caller index o): the walk adjoint (target side
// plus the mass-weighted share of its ancestors' centre-of-mass adjoints),
// the FP64 star and perturber Jacobians, then -- unless this is level 0 --
// the drift and first-kick adjoints of the step that produced the level.
// kDirect: the force adjoint came from the FP64 direct sum, already whole and
// in caller order (mu), with no centre-of-mass range adds.
template <bool kStep, bool kDirect = false>
__global__ void __launch_bounds__(kThreads) k_adj_apply(const ApplyArgs a) {
  __shared__ double red[4][kThreads / 32];
  double pg[4] = {0.0, 0.0, 0.0, 0.0};
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < a.n;
       s += (long long)gridDim.x * blockDim.x) {
    const uint32_t o = kDirect ? (uint32_t)s : a.perm[s];
    double gx, gy, gz;
    if (kDirect) {
      gx = a.gx[o] + a.mux[s];
      gy = a.gy[o] + a.muy[s];
      gz = a.gz[o] + a.muz[s];
    } else {
      const double4 P = range_moments(a.rploc, a.rtpre, 0, (int)s + 1);
      const double m = (double)a.body4[s].w;
      gx = a.gx[o] + a.mux[s] + m * P.x;
      gy = a.gy[o] + a.muy[s] + m * P.y;
      gz = a.gz[o] + a.muz[s] + m * P.z;
    }
    const double x = a.x[o], y = a.y[o], z = a.z[o];
    const double lx = a.lx[o], ly = a.ly[o], lz = a.lz[o];
    {  // star: a = -M x / r^3, da/dx = -M (I/r^3 - 3 x x^T / r^5)
      const double r2 = fma(x, x, fma(y, y, fma(z, z, a.eps * a.eps)));
      const double inv = 1.0 / sqrt(r2);
      const double inv3 = inv * inv * inv, inv5 = inv3 * inv * inv;
      const double xl = x * lx + y * ly + z * lz;
      gx -= a.star_mass * (lx * inv3 - 3.0 * x * xl * inv5);
      gy -= a.star_mass * (ly * inv3 - 3.0 * y * xl * inv5);
      gz -= a.star_mass * (lz * inv3 - 3.0 * z * xl * inv5);
    }
    const double4 pt = a.pert_tab[a.level];
    if (pt.w != 0.0) {  // a = m_p d / r^3 with d = p - x
      const double dx = pt.x - x, dy = pt.y - y, dz = pt.z - z;
      const double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, a.eps * a.eps)));
      const double inv = 1.0 / sqrt(r2);
      const double inv3 = inv * inv * inv, inv5 = inv3 * inv * inv;
      const double dl = dx * lx + dy * ly + dz * lz;
      const double jx = pt.w * (lx * inv3 - 3.0 * dx * dl * inv5);
      const double jy = pt.w * (ly * inv3 - 3.0 * dy * dl * inv5);
      const double jz = pt.w * (lz * inv3 - 3.0 * dz * dl * inv5);
      gx -= jx; gy -= jy; gz -= jz;
      pg[0] += jx; pg[1] += jy; pg[2] += jz;
      pg[3] += dl * inv3;
    }
    a.gx[o] = gx; a.gy[o] = gy; a.gz[o] = gz;
    if (kStep) {
      const double vx = fma(a.dt, gx, a.gvx[o]);
      const double vy = fma(a.dt, gy, a.gvy[o]);
      const double vz = fma(a.dt, gz, a.gvz[o]);
      a.gvx[o] = vx; a.gvy[o] = vy; a.gvz[o] = vz;
      a.plx[o] = a.dth * vx; a.ply[o] = a.dth * vy; a.plz[o] = a.dth * vz;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    double v = pg[k];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(kFull, v, off);
    if (lane == 0) red[k][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0.0;
    for (int q = 0; q < kThreads / 32; ++q) v += red[threadIdx.x][q];
    if (v != 0.0) atomicAdd(a.pgrad + threadIdx.x, v);
  }
}

template <typename TA>
struct DragAdjArgsT {
  // level L (start of the step) and L+1 (end), caller order
  const double* x0;
  const double* y0;
  const double* z0;
  const double* v0x;
  const double* v0y;
  const double* v0z;
  const TA* a0x;
  const TA* a0y;
  const TA* a0z;
  const double* x1;
  const double* y1;
  const double* z1;
  const TA* a1x;
  const TA* a1y;
  const TA* a1z;
  const double4* pert_tab;  // levels L and L+1
  int level;
  double eps, star_mass, dth, decay;
  int drag;
  // adjoints
  double* gx;   // of x_{L+1} (in/out)
  double* gy;
  double* gz;
  double* gvx;  // in: of v_{L+1}; out: of v' (= of v_h)
  double* gvy;
  double* gvz;
  double* plx;  // in: pending (dt/2 V_h of step L+1, or 0); out: lam_{L+1}
  double* ply;
  double* plz;
  int n;
};

// Second kick + drag of step L in reverse: v' = v_h + dt/2 A_{L+1} is
// recomputed as the forward did (its v_phi sign selects the drag branch);
// drag(x, v') = decay v' + (1 - decay) s sqrt(M) (-z, 0, x) r_xz^{-3/2}.
template <typename TA>
__global__ void __launch_bounds__(kThreads) k_adj_drag(const DragAdjArgsT<TA> a) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n;
       i += (long long)gridDim.x * blockDim.x) {
    double gvx = a.gvx[i], gvy = a.gvy[i], gvz = a.gvz[i];
    if (a.drag) {
      const double x = a.x1[i], z = a.z1[i];
      const double rxz2 = fma(x, x, __dmul_rn(z, z));
      if (!(rxz2 < 1e-12)) {
        double ax0, ay0, az0, ax1, ay1, az1;
        total_accel(a.x0[i], a.y0[i], a.z0[i], a.a0x[i], a.a0y[i], a.a0z[i], a.eps, a.star_mass,
                    a.pert_tab[a.level], ax0, ay0, az0);
        total_accel(x, a.y1[i], z, a.a1x[i], a.a1y[i], a.a1z[i], a.eps, a.star_mass,
                    a.pert_tab[a.level + 1], ax1,
                    ay1, az1);
        double vx = fma(ax0, a.dth, a.v0x[i]), vz = fma(az0, a.dth, a.v0z[i]);
        vx = fma(ax1, a.dth, vx);
        vz = fma(az1, a.dth, vz);
        const double inv_r = 1.0 / sqrt(rxz2);
        const double v_phi = __dmul_rn(fma(vx, -z, __dmul_rn(vz, x)), inv_r);
        const double sgn = (v_phi >= 0.0) ? 1.0 : -1.0;
        // u = (-z, 0, x) r^-3/2, r = r_xz; c = (1 - decay) s sqrt(M)
        const double c = (1.0 - a.decay) * sgn * sqrt(a.star_mass);
        const double r = sqrt(rxz2);
        const double rm32 = 1.0 / (r * sqrt(r));          // r^-3/2
        const double rm72 = rm32 / (rxz2);                // r^-7/2
        const double dux_dx = 1.5 * x * z * rm72;
        const double dux_dz = -rm32 + 1.5 * z * z * rm72;
        const double duz_dx = rm32 - 1.5 * x * x * rm72;
        const double duz_dz = -1.5 * x * z * rm72;
        a.gx[i] += c * (dux_dx * gvx + duz_dx * gvz);
        a.gz[i] += c * (dux_dz * gvx + duz_dz * gvz);
        gvx *= a.decay; gvy *= a.decay; gvz *= a.decay;
      }
    }
    a.gvx[i] = gvx; a.gvy[i] = gvy; a.gvz[i] = gvz;
    a.plx[i] = fma(a.dth, gvx, a.plx[i]);
    a.ply[i] = fma(a.dth, gvy, a.ply[i]);
    a.plz[i] = fma(a.dth, gvz, a.plz[i]);
  }
}

// ------------------------------------------------- time-reversed leapfrog
struct RevArgs {
  const double* x;   // level L positions, velocities (caller order)
  const double* vx;
  const float* ax;   // level L self-gravity
  const double4* pert_tab;
  int level;
  double* px;        // out: level L-1 positions
  double* vh;        // out: v_h of step L-1
  double eps, star_mass, dt, dth, decay;
  int drag;
  int n;
};

// Step L-1 run backwards from level L: the drag is inverted in closed form
// (drag(x, v') = decay v' + (1 - decay) s sqrt(M) (-z, 0, x) r_xz^{-3/2},
// s the sign of v_phi, which the drag keeps), then the second kick
// (v_h = v' - dt/2 acc_L) and the drift (x_{L-1} = x_L - dt v_h).
__global__ void __launch_bounds__(kThreads) k_dstep_rev(const RevArgs a) {
  const size_t n1 = a.n, n2 = 2 * (size_t)a.n;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n;
       i += (long long)gridDim.x * blockDim.x) {
    const double x = a.x[i], y = a.x[n1 + i], z = a.x[n2 + i];
    double vx = a.vx[i], vy = a.vx[n1 + i], vz = a.vx[n2 + i];
    if (a.drag) {
      const double rxz2 = fma(x, x, __dmul_rn(z, z));
      if (!(rxz2 < 1e-12)) {
        const double inv_r = 1.0 / sqrt(rxz2);
        const double v_phi = __dmul_rn(fma(vx, -z, __dmul_rn(vz, x)), inv_r);
        const double sgn = (v_phi >= 0.0) ? 1.0 : -1.0;
        const double c = (1.0 - a.decay) * sgn * sqrt(a.star_mass) * inv_r * sqrt(inv_r);
        const double inv_d = 1.0 / a.decay;
        vx = (vx + c * z) * inv_d;
        vz = (vz - c * x) * inv_d;
        vy = vy * inv_d;
      }
    }
    double ax, ay, az;
    total_accel(x, y, z, a.ax[i], a.ax[n1 + i], a.ax[n2 + i], a.eps, a.star_mass,
                a.pert_tab[a.level], ax, ay, az);
    vx = fma(-a.dth, ax, vx); vy = fma(-a.dth, ay, vy); vz = fma(-a.dth, az, vz);
    a.vh[i] = vx; a.vh[n1 + i] = vy; a.vh[n2 + i] = vz;
    a.px[i] = fma(-a.dt, vx, x); a.px[n1 + i] = fma(-a.dt, vy, y);
    a.px[n2 + i] = fma(-a.dt, vz, z);
  }
}

// The first kick of step L-1 undone once level L-1's self-gravity is known:
// v_{L-1} = v_h - dt/2 acc_{L-1}.
__global__ void __launch_bounds__(kThreads) k_kick_rev(const double* __restrict__ x,
                                                       const double* __restrict__ vh,
                                                       const float* __restrict__ sg,
                                                       const double4* __restrict__ pert_tab,
                                                       int level, double eps, double star_mass,
                                                       double dth, double* __restrict__ v,
                                                       int n) {
  const size_t n1 = n, n2 = 2 * (size_t)n;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double ax, ay, az;
    total_accel(x[i], x[n1 + i], x[n2 + i], sg[i], sg[n1 + i], sg[n2 + i], eps, star_mass,
                pert_tab[level], ax, ay, az);
    v[i] = fma(-dth, ax, vh[i]);
    v[n1 + i] = fma(-dth, ay, vh[n1 + i]);
    v[n2 + i] = fma(-dth, az, vh[n2 + i]);
  }
}

// ------------------------------------------------ FP64 direct-sum dynamics
// The reference gradient's dynamics: self-gravity by FP64 direct summation
// over every pair (softened, no tree), a_i = sum_j m_j d_ij / r_ij^3 with
// d_ij = x_j - x_i and r^2 = |d|^2 + eps^2.  Caller order; the source tile
// is staged in shared memory.
constexpr int kDirTile = 256;

__global__ void __launch_bounds__(kDirTile) k_direct_acc(const double* __restrict__ x,
                                                          const float* __restrict__ m, int n,
                                                          double eps2, double* __restrict__ a) {
  __shared__ double4 src[kDirTile];
  const size_t n1 = n, n2 = 2 * (size_t)n;
  const int i = blockIdx.x * kDirTile + threadIdx.x;
  const bool valid = i < n;
  const double px = valid ? x[i] : 0.0, py = valid ? x[n1 + i] : 0.0,
               pz = valid ? x[n2 + i] : 0.0;
  double sx = 0.0, sy = 0.0, sz = 0.0;
  for (int t0 = 0; t0 < n; t0 += kDirTile) {
    const int j = t0 + threadIdx.x;
    src[threadIdx.x] = (j < n) ? make_double4(x[j], x[n1 + j], x[n2 + j], (double)m[j])
                               : make_double4(0.0, 0.0, 0.0, 0.0);
    __syncthreads();
    const int k = min(kDirTile, n - t0);
    for (int q = 0; q < k; ++q) {
      const double4 s = src[q];
      const double dx = s.x - px, dy = s.y - py, dz = s.z - pz;
      const double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
      if (t0 + q == i || r2 <= 0.0) continue;
      const double inv = 1.0 / sqrt(r2);
      const double f = s.w * inv * inv * inv;
      sx = fma(f, dx, sx); sy = fma(f, dy, sy); sz = fma(f, dz, sz);
    }
    __syncthreads();
  }
  if (valid) { a[i] = sx; a[n1 + i] = sy; a[n2 + i] = sz; }
}

// Vector-Jacobian product of the direct sum: with lam_i the adjoint of a_i
// and J(d) = (I r^2 - 3 d d^T) / r^5 (symmetric, even in d), the adjoint of
// x_k is sum_{j != k} J(d_kj) (m_k lam_j - m_j lam_k).  Written to mu
// (caller order), which the apply kernel adds to the position adjoint.
__global__ void __launch_bounds__(kDirTile) k_direct_vjp(const double* __restrict__ x,
                                                          const float* __restrict__ m,
                                                          const double* __restrict__ lam, int n,
                                                          double eps2, double* __restrict__ mu) {
  __shared__ double4 src[kDirTile];
  __shared__ double3 sl[kDirTile];
  const size_t n1 = n, n2 = 2 * (size_t)n;
  const int k = blockIdx.x * kDirTile + threadIdx.x;
  const bool valid = k < n;
  const double px = valid ? x[k] : 0.0, py = valid ? x[n1 + k] : 0.0,
               pz = valid ? x[n2 + k] : 0.0;
  const double mk = valid ? (double)m[k] : 0.0;
  const double lkx = valid ? lam[k] : 0.0, lky = valid ? lam[n1 + k] : 0.0,
               lkz = valid ? lam[n2 + k] : 0.0;
  double gx = 0.0, gy = 0.0, gz = 0.0;
  for (int t0 = 0; t0 < n; t0 += kDirTile) {
    const int j = t0 + threadIdx.x;
    src[threadIdx.x] = (j < n) ? make_double4(x[j], x[n1 + j], x[n2 + j], (double)m[j])
                               : make_double4(0.0, 0.0, 0.0, 0.0);
    sl[threadIdx.x] = (j < n) ? make_double3(lam[j], lam[n1 + j], lam[n2 + j])
                              : make_double3(0.0, 0.0, 0.0);
    __syncthreads();
    const int kk = min(kDirTile, n - t0);
    for (int q = 0; q < kk; ++q) {
      const double4 s = src[q];
      const double3 l = sl[q];
      const double dx = s.x - px, dy = s.y - py, dz = s.z - pz;
      const double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
      if (t0 + q == k || r2 <= 0.0) continue;
      const double inv = 1.0 / sqrt(r2);
      const double inv3 = inv * inv * inv, inv5 = inv3 * inv * inv;
      const double wx = mk * l.x - s.w * lkx, wy = mk * l.y - s.w * lky,
                   wz = mk * l.z - s.w * lkz;
      const double dw = dx * wx + dy * wy + dz * wz;
      gx += wx * inv3 - 3.0 * dx * dw * inv5;
      gy += wy * inv3 - 3.0 * dy * dw * inv5;
      gz += wz * inv3 - 3.0 * dz * dw * inv5;
    }
    __syncthreads();
  }
  if (valid) { mu[k] = gx; mu[n1 + k] = gy; mu[n2 + k] = gz; }
}

}  // namespace

// ================================================================== host
// How the backward gets the forward's levels (nbody_adjoint_create_mode):
//  kModeTape        every level's state and tape kept in HBM from the forward;
//  kModeCheckpoint  FP64 states every `every` levels only: the backward
//                   rebuilds each level by running the step backwards in time
//                   (time-reversed leapfrog) from the level after it, re-records
//                   its tree and tape, and restarts every segment from its
//                   exact checkpoint, so rounding drift never spans more than
//                   `every` steps; two levels of state and tape are held;
//  kModeDirect      FP64 direct-sum self-gravity instead of the tree walk (every
//                   level kept): the reference gradient of the same loss.
constexpr int kModeTape = NBODY_ADJOINT_TAPE, kModeCheckpoint = NBODY_ADJOINT_CHECKPOINT,
              kModeDirect = NBODY_ADJOINT_DIRECT;

struct AdjointImpl {
  nbody_sim_params p{};
  int n = 0, steps = 0;
  int mode = kModeTape;
  int every = 0;  // checkpoint spacing (kModeCheckpoint)
  cudaStream_t st = 0;
  bool own_stream = false;
  TreeWork tw;
  // level buffers (caller order): positions, velocities, self-gravity; one
  // per level, or two (slot L & 1) in checkpoint mode
  std::vector<double*> X, V;
  std::vector<float*> A;
  std::vector<double*> AD;  // direct mode: FP64 self-gravity per level
  std::vector<double*> CK;  // checkpoint mode: x, v (6n) at levels 0, every, 2 every, ...
  double* vh = nullptr;     // checkpoint mode: v_h of the step being reversed
  // per level tape: sort permutation, groups, group tape; tape chunks come
  // from pool 0 (tape mode, every level) or pool L & 1 (checkpoint mode)
  std::vector<uint32_t*> perm;
  std::vector<int2*> groups, gtape;
  int* ngroups = nullptr;  // per level slot, device
  // Checkpoint mode holds three levels at a time (and a tape pool each): the
  // backward re-records level L-1 while it differentiates level L, and
  // level L+1's slot may still be in use then.
  static constexpr int kCkSlots = 3;
  int2* pool[kCkSlots] = {nullptr, nullptr, nullptr};
  int* pool_next[kCkSlots] = {nullptr, nullptr, nullptr};
  int* pool_used = nullptr;  // device, one counter per pool
  int pool_cap = 0;          // chunks per pool
  // scratch
  double *xs = nullptr, *ys = nullptr, *zs = nullptr;  // sorted positions of the tree builds
  // A level's bodies for the replays and the force adjoints (level_bodies):
  // sorted FP64 positions (lev_x..z), float bodies and their moment prefix
  // (tv holds body4, mom_ploc and mom_tiles only), apart from the tree
  // builds' own so that a backward can rebuild one level while it
  // differentiates another.
  double *lev_x = nullptr, *lev_y = nullptr, *lev_z = nullptr;
  TreeWork tv;
  int* work_b = nullptr;  // the replays' group counter
  // checkpoint-mode backward: the rebuilds of earlier levels run on rev_st
  // beside the differentiation on the engine stream, ordered by these events
  cudaStream_t rev_st = nullptr;
  std::vector<cudaEvent_t> bwd_events;
  double *vw = nullptr, *xw = nullptr;      // work velocity (3n) and positions (2 x 3n)
  float* aw = nullptr;                       // work self-gravity (3n)
  double* aw64 = nullptr;                    // FP64 replay self-gravity (3n)
  double *gx = nullptr, *gv = nullptr, *lam = nullptr, *mu = nullptr;  // 3n each
  double4 *radd = nullptr, *rploc = nullptr, *rtiles = nullptr;
  double* pgrad = nullptr;                   // 4 per level
  float* mass = nullptr;
  int* spill = nullptr;
  int spill_cap = 4096;
  int* work = nullptr;
  unsigned long long* inter = nullptr;
  double mjup = 0.0;
  double pm = 0.0, pr = 1.0;  // perturber mass (M_J) and radius (AU) of the recorded forward
  bool recorded = false;
  float ms_forward = 0.f, ms_backward = 0.f, ms_replay = 0.f;
  unsigned long long launches = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  // perturber (x, y, z, mass in M_sun) per level: recorded run, replays
  double4* pert_fwd = nullptr;
  double4* pert_rep = nullptr;
  // The recording forward, the backward and the two replays are each captured
  // once as a CUDA graph (every buffer they touch is fixed for the engine's
  // life; inputs and outputs are copied in and out around the launch) and
  // replayed: at small n a level is a few tens of microseconds of GPU work,
  // less than launching its kernels one by one.
  struct Captured {
    cudaGraphExec_t g = nullptr;
    unsigned long long kernels = 0;
  };
  Captured g_fwd, g_bwd, g_rep[2];
  double* rep_final[2] = {nullptr, nullptr};  // buffer holding a replay's final positions
  cudaStream_t cap_st = nullptr;

  int slot(int L) const { return mode == kModeCheckpoint ? (L % kCkSlots) : L; }
  int pidx(int L) const { return mode == kModeCheckpoint ? (L % kCkSlots) : 0; }
  int n_pools() const { return mode == kModeCheckpoint ? kCkSlots : (mode == kModeTape ? 1 : 0); }

  AdjointImpl(const nbody_sim_params& prm, int nn, int nsteps, int md, int ck_every) {
    p = prm;
    n = nn;
    steps = nsteps;
    mode = md;
    every = ck_every;
    if (p.leaf_max <= 0) p.leaf_max = kLeafMaxSmall;
    check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "adjoint stream");
    own_stream = true;
    tree_alloc(tw, n);
    // no side stream for the moment prefix: beside the Karras pass it
    // slowed the build (N = 2^20: 115 us against 88 us in one stream)
    tw.group_max = 32;
    const size_t n3 = 3 * (size_t)n;
    const int nslot = (mode == kModeCheckpoint) ? kCkSlots : steps + 1;
    for (int L = 0; L < nslot; ++L) {
      X.push_back(dalloc<double>(n3, "level positions"));
      V.push_back(dalloc<double>(n3, "level velocities"));
      if (mode == kModeDirect) {
        AD.push_back(dalloc<double>(n3, "level self-gravity"));
        continue;
      }
      A.push_back(dalloc<float>(n3, "level self-gravity"));
      perm.push_back(dalloc<uint32_t>(n, "level permutation"));
      groups.push_back(dalloc<int2>(n, "level groups"));
      gtape.push_back(dalloc<int2>(n, "level group tape"));
    }
    if (mode == kModeCheckpoint) {
      for (int L = 0; L <= steps; L += every) CK.push_back(dalloc<double>(2 * n3, "checkpoint"));
      vh = dalloc<double>(n3, "reversed half-step velocity");
    }
    ngroups = dalloc<int>(nslot, "level group counts");
    xs = dalloc<double>(n, "sorted x"); ys = dalloc<double>(n, "sorted y");
    lev_x = dalloc<double>(n, "level sorted x"); lev_y = dalloc<double>(n, "level sorted y");
    lev_z = dalloc<double>(n, "level sorted z");
    tv.body4 = dalloc<float4>(n, "level bodies");
    tv.mom_ploc = dalloc<double4>(n + 1, "level moment prefix");
    tv.mom_tiles = dalloc<double4>(2 * (moment_tiles(n) + 1), "level moment tiles");
    work_b = dalloc<int>(1, "replay work");
    zs = dalloc<double>(n, "sorted z");
    vw = dalloc<double>(n3, "work velocity");
    xw = dalloc<double>(2 * n3, "work positions");
    aw = dalloc<float>(n3, "work self-gravity");
    gx = dalloc<double>(n3, "position adjoint");
    gv = dalloc<double>(n3, "velocity adjoint");
    lam = dalloc<double>(n3, "acceleration adjoint");
    mu = dalloc<double>(n3, "walk target adjoint");
    radd = dalloc<double4>(n + 1, "range adds");
    rploc = dalloc<double4>(n + 2, "range prefix");
    rtiles = dalloc<double4>(2 * ((n + 1) / kMomentTile + 3), "range tiles");
    pgrad = dalloc<double>(4 * (size_t)(steps + 1), "perturber adjoints");
    mass = dalloc<float>(n, "mass");
    spill = dalloc<int>((size_t)walk_spill_slots(0) * spill_cap, "walk spill");
    work = dalloc<int>(1, "work");
    inter = dalloc<unsigned long long>(1, "interactions");
    pool_used = dalloc<int>(kCkSlots, "tape chunks used");
    aw64 = dalloc<double>(n3, "FP64 replay self-gravity");
    pert_fwd = dalloc<double4>(steps + 1, "perturber per level");
    pert_rep = dalloc<double4>(steps + 1, "replay perturber per level");
    nbody_config c;
    nbody_config_defaults(&c);
    c.perturber_enabled = 1;
    c.perturber_mass_mjup = 1.f;
    c.perturber_radius_AU = 1.f;
    nbody_perturber q;
    nbody_perturber_make(&c, &q);
    mjup = (double)q.mass_msun;
    check(cudaEventCreate(&e0), "event");
    check(cudaEventCreate(&e1), "event");
  }

  ~AdjointImpl() {
    if (st) cudaStreamSynchronize(st);
    drop_graphs();
    if (cap_st) cudaStreamDestroy(cap_st);
    for (auto* q : X) cudaFree(q);
    for (auto* q : V) cudaFree(q);
    for (auto* q : A) cudaFree(q);
    for (auto* q : AD) cudaFree(q);
    for (auto* q : CK) cudaFree(q);
    for (auto* q : perm) cudaFree(q);
    for (auto* q : groups) cudaFree(q);
    for (auto* q : gtape) cudaFree(q);
    void* ptrs[] = {ngroups, pool[0], pool[1], pool[2], pool_next[0], pool_next[1], pool_next[2],
                    pool_used, xs, ys, zs, lev_x, lev_y, lev_z, work_b, vw, xw, aw, aw64, gx, gv, lam, mu,
                    radd, rploc, rtiles, pgrad, mass, spill, work, inter, pert_fwd, pert_rep, vh};
    for (void* q : ptrs)
      if (q) cudaFree(q);
    for (cudaEvent_t e : bwd_events)
      cudaEventDestroy(e);
    if (rev_st) cudaStreamDestroy(rev_st);
    tree_free(tw);
    tree_free(tv);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (own_stream && st) cudaStreamDestroy(st);
  }

  void set_stream(cudaStream_t s) {
    check(cudaStreamSynchronize(st), "adjoint sync");
    if (own_stream) cudaStreamDestroy(st);
    own_stream = false;
    st = s;
  }

  // Perturber (x, y, z, mass in M_sun) at t_L = L dt in FP64: the orbit of
  // makePerturber/updatePerturber (Perturber.h:39-66) evaluated in double.
  double4 pert_at(int L, double mass_mj, double radius) const {
    if (!p.perturber_enabled) return make_double4(0, 0, 0, 0);
    const double om = std::sqrt((double)p.star_mass / (radius * radius * radius));
    const double phi = (double)p.perturber_phase0 + om * ((double)L * (double)p.dt);
    return make_double4(radius * std::cos(phi), 0.0, radius * std::sin(phi), mass_mj * mjup);
  }

  template <typename TA = float>
  StepArgsT<TA> step_args(const double* x, double* v, const TA* a, double* lv, double* nx,
                          const double4* tab, int level) const {
    StepArgsT<TA> s{};
    s.x = x; s.y = x + n; s.z = x + 2 * (size_t)n;
    s.vx = v; s.vy = v + n; s.vz = v + 2 * (size_t)n;
    s.ax = a; s.ay = a + n; s.az = a + 2 * (size_t)n;
    s.lvx = lv; s.lvy = lv ? lv + n : nullptr; s.lvz = lv ? lv + 2 * (size_t)n : nullptr;
    s.nx = nx; s.ny = nx ? nx + n : nullptr; s.nz = nx ? nx + 2 * (size_t)n : nullptr;
    s.pert_tab = tab;
    s.level = level;
    s.eps = p.softening; s.star_mass = p.star_mass;
    s.dt = (double)p.dt; s.dth = (double)p.dt * 0.5;
    s.drag = p.gas_drag_rate > 0.f;
    s.decay = s.drag ? std::exp(-(double)p.gas_drag_rate * (double)p.dt) : 1.0;
    s.n = n;
    return s;
  }

  template <typename TA>
  void launch_step(bool end, bool begin, const StepArgsT<TA>& s) {
    if (end && begin) k_dstep<true, true, TA><<<grid1(n), kThreads, 0, st>>>(s);
    else if (end) k_dstep<true, false, TA><<<grid1(n), kThreads, 0, st>>>(s);
    else k_dstep<false, true, TA><<<grid1(n), kThreads, 0, st>>>(s);
    check(cudaGetLastError(), "k_dstep launch");
    launches += 1;
  }

  // Tree + recording walk at level L's positions -> its self-gravity and tape
  // (level slot L; checkpoint mode starts the slot's tape pool afresh).
  void record_level(int L) {
    const int sl = slot(L), pi = pidx(L);
    const double* x = X[sl];
    if (mode == kModeCheckpoint)
      check(cudaMemsetAsync(pool_used + pi, 0, sizeof(int), st), "tape reset");
    const size_t n1 = n, n2 = 2 * (size_t)n;
    launch_bbox<double>(tw, x, x + n1, x + n2, n, st);
    uint32_t* hist = radix_sort_prepare(tw.counts, 30, st);  // counted by the key kernel
    launch_keys<double>(tw, x, x + n1, x + n2, n, st, hist);
    radix_sort_pairs(tw.keys, tw.perm, tw.keys_alt, tw.perm_alt, tw.counts, n, 30, st,
                     tw.status, true);
    k_gather_sorted<<<grid1(n), kThreads, 0, st>>>(tw.perm, x, x + n1, x + n2, mass, n, xs, ys,
                                                   zs, tw.body4);
    tw.prune_max = p.leaf_max;
    launch_tree<uint32_t>(tw, tw.keys, n, 30, 0, 1, tw.geom, nullptr, xs, ys, zs, st);
    check(cudaMemcpyAsync(perm[sl], tw.perm, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice,
                          st), "tape permutation");
    k_copy_groups<<<grid1(n), kThreads, 0, st>>>(tw.groups, tw.n_groups, n, groups[sl],
                                                 ngroups + sl);
    WalkArgs w{};
    w.com = tw.oct.com; w.info = tw.oct.info; w.body = tw.body4; w.n = n;
    w.groups = tw.groups; w.n_groups = tw.n_groups;
    w.theta2 = p.theta * p.theta; w.eps = p.softening; w.star_mass = 0.f;
    w.star_in_walk = 0; w.leaf_max = p.leaf_max; w.pert = nullptr;
    float* a = A[sl];
    w.ax = a; w.ay = a + n1; w.az = a + n2; w.scatter = tw.perm;
    w.spill = spill; w.spill_cap = spill_cap; w.inter = inter; w.counters = nullptr;
    w.work = work; w.status = tw.status; w.targets_per_lane = 1;
    w.tape = pool[pi]; w.tape_next = pool_next[pi]; w.tape_used = pool_used + pi;
    w.tape_cap = pool_cap;
    w.group_tape = gtape[sl];
    launch_walk(w, st);
    // bbox, keys, 20 sort, gather, copy groups, karras, mark, 6 scans,
    // moment tiles, tile scan, emit, walk
    launches += 36;
  }

  void drop_graphs() {
    for (Captured* c : {&g_fwd, &g_bwd, &g_rep[0], &g_rep[1]})
      if (c->g) {
        cudaGraphExecDestroy(c->g);
        c->g = nullptr;
      }
  }

  // Runs body's launches as one graph (captured on first use, on a private
  // stream; the caller's stream may be the legacy one), on the engine stream.
  template <typename F>
  void run_graph(Captured& c, F&& body) {
    if (!c.g) {
      if (!cap_st)
        check(cudaStreamCreateWithFlags(&cap_st, cudaStreamNonBlocking), "capture stream");
      cudaStream_t user = st;
      const unsigned long long l0 = launches;
      cudaGraph_t graph = nullptr;
      st = cap_st;
      check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
      try {
        body();
      } catch (...) {
        cudaStreamEndCapture(st, &graph);
        if (graph) cudaGraphDestroy(graph);
        st = user;
        launches = l0;
        throw;
      }
      const cudaError_t ce = cudaStreamEndCapture(st, &graph);
      st = user;
      check(ce, "end capture");
      c.kernels = launches - l0;
      launches = l0;
      const cudaError_t ie = cudaGraphInstantiate(&c.g, graph, 0);
      cudaGraphDestroy(graph);
      check(ie, "graph instantiate");
    }
    check(cudaGraphLaunch(c.g, st), "graph launch");
    launches += c.kernels;
  }

  void upload_pert(double4* tab, double mass_mj, double radius) {
    std::vector<double4> h(steps + 1);
    for (int L = 0; L <= steps; ++L) h[L] = pert_at(L, mass_mj, radius);
    check(cudaMemcpyAsync(tab, h.data(), sizeof(double4) * h.size(), cudaMemcpyHostToDevice, st),
          "perturber table");
  }

  void ensure_pool(int chunks) {
    if (chunks <= pool_cap) return;
    check(cudaStreamSynchronize(st), "tape pool sync");
    drop_graphs();  // the captured runs hold the old pool
    const int npools = n_pools();
    pool_cap = chunks;
    for (int k = 0; k < npools; ++k) {
      if (pool[k]) cudaFree(pool[k]);
      if (pool_next[k]) cudaFree(pool_next[k]);
      pool[k] = dalloc<int2>((size_t)pool_cap * kTapeChunk, "tape pool");
      pool_next[k] = dalloc<int>(pool_cap, "tape links");
    }
  }

  int read_status() {
    int s = 0;
    check(cudaStreamSynchronize(st), "adjoint sync");
    check(cudaMemcpy(&s, tw.status, sizeof(int), cudaMemcpyDeviceToHost), "status");
    return s;
  }

  // Forward with recording: initial state (device, caller order SoA) and the
  // perturber's mass (M_J) and orbit radius (AU).
  void forward(const double* const* x0, const float* m, double mass_mj, double radius) {
    pm = mass_mj;
    pr = radius;
    check(cudaMemcpyAsync(mass, m, sizeof(float) * n, cudaMemcpyDeviceToDevice, st), "mass");
    for (int k = 0; k < 3; ++k)
      check(cudaMemcpyAsync(X[0] + (size_t)k * n, x0[k], sizeof(double) * n,
                            cudaMemcpyDeviceToDevice, st),
            "initial positions");
    // size the tape pool(s) from level 0, then record the whole run (again
    // if the estimate fell short)
    if (mode != kModeDirect) {
      if (pool_cap == 0) ensure_pool(std::max(1024, n / 32 * 24));
      for (int attempt = 0; attempt < 4; ++attempt) {
        check(cudaMemsetAsync(tw.status, 0, sizeof(int), st), "status reset");
        check(cudaMemsetAsync(pool_used, 0, kCkSlots * sizeof(int), st), "tape reset");
        record_level(0);
        int used = 0;
        check(cudaStreamSynchronize(st), "adjoint sync");
        check(cudaMemcpy(&used, pool_used, sizeof(int), cudaMemcpyDeviceToHost), "tape used");
        const long long need = (mode == kModeTape)
                                   ? (long long)used * (steps + 1) * 5 / 4 + 1024
                                   : (long long)used * 2 + 1024;
        if (need > pool_cap) {
          ensure_pool((int)std::min<long long>(need, 0x7fffffffLL / kTapeChunk));
          continue;
        }
        break;
      }
    }
    upload_pert(pert_fwd, pm, pr);
    for (int attempt = 0; attempt < 3; ++attempt) {
      for (int k = 0; k < 3; ++k)
        check(cudaMemcpyAsync(vw + (size_t)k * n, x0[3 + k], sizeof(double) * n,
                              cudaMemcpyDeviceToDevice, st),
              "initial velocities");
      check(cudaEventRecord(e0, st), "event");
      run_graph(g_fwd, [&] { forward_levels(); });
      check(cudaEventRecord(e1, st), "event");
      const int s = read_status();
      if (s & kStatusTapeFull) {
        int used[kCkSlots] = {0, 0, 0};
        check(cudaMemcpy(used, pool_used, kCkSlots * sizeof(int), cudaMemcpyDeviceToHost),
              "tape used");
        const int u = std::max(used[0], std::max(used[1], used[2]));
        ensure_pool((int)std::min<long long>((long long)u * 3 / 2 + 1024,
                                             0x7fffffffLL / kTapeChunk));
        continue;
      }
      if (s) throw ArgError("adjoint forward: device status " + std::to_string(s),
                            NBODY_ERR_OVERFLOW);
      check(cudaEventElapsedTime(&ms_forward, e0, e1), "event time");
      recorded = true;
      return;
    }
    throw ArgError("adjoint forward: tape pool could not be sized", NBODY_ERR_OVERFLOW);
  }

  // The forward's launches (captured as one graph): every level's forces and
  // the step to the next level.  Tape mode keeps every level; checkpoint mode
  // writes two level slots and copies (x, v) out every `every` levels; direct
  // mode sums the self-gravity pair by pair in FP64.
  void forward_levels() {
    check(cudaMemsetAsync(tw.status, 0, sizeof(int), st), "status reset");
    check(cudaMemsetAsync(pool_used, 0, kCkSlots * sizeof(int), st), "tape reset");
    const size_t n3 = 3 * (size_t)n;
    if (mode == kModeDirect) {
      const double eps2 = (double)p.softening * (double)p.softening;
      for (int L = 0; L <= steps; ++L) {
        k_direct_acc<<<div_up(n, kDirTile), kDirTile, 0, st>>>(X[L], mass, n, eps2, AD[L]);
        const bool end = L > 0, begin = L < steps;
        launch_step(end, begin, step_args<double>(X[L], vw, AD[L], V[L],
                                                  begin ? X[L + 1] : nullptr, pert_fwd, L));
        launches += 1;
      }
      return;
    }
    record_level(0);
    for (int L = 0; L <= steps; ++L) {
      const bool end = L > 0, begin = L < steps;
      const int sl = slot(L);
      launch_step(end, begin, step_args<float>(X[sl], vw, A[sl], V[sl],
                                               begin ? X[slot(L + 1)] : nullptr, pert_fwd, L));
      if (mode == kModeCheckpoint && L % every == 0) {
        double* c = CK[L / every];
        check(cudaMemcpyAsync(c, X[sl], sizeof(double) * n3, cudaMemcpyDeviceToDevice, st),
              "checkpoint x");
        check(cudaMemcpyAsync(c + n3, V[sl], sizeof(double) * n3, cudaMemcpyDeviceToDevice, st),
              "checkpoint v");
      }
      if (begin) record_level(L + 1);
    }
  }

  // Level L's bodies in its recorded order and their moment prefix.
  void level_bodies(int L, const double* x) {
    const size_t n1 = n, n2 = 2 * (size_t)n;
    k_gather_sorted<<<grid1(n), kThreads, 0, st>>>(perm[slot(L)], x, x + n1, x + n2, mass, n,
                                                   lev_x, lev_y, lev_z, tv.body4);
    launch_moment_prefix(tv, n, lev_x, lev_y, lev_z, st);
    launches += 3;
  }

  ReplayArgs replay_args(int L) {
    ReplayArgs r{};
    r.body4 = tv.body4;
    r.ploc = tv.mom_ploc;
    r.tpre = moment_tile_prefix(tv, n);
    const int sl = slot(L);
    r.perm = perm[sl];
    r.groups = groups[sl];
    r.n_groups = ngroups + sl;
    r.group_tape = gtape[sl];
    r.tape = pool[pidx(L)];
    r.tape_next = pool_next[pidx(L)];
    r.eps2 = p.softening * p.softening;
    r.work = work_b;
    r.status = tw.status;
    return r;
  }

  void launch_replay(const ReplayArgs& r, bool adj, bool fp64 = false) {
    check(cudaMemsetAsync(r.work, 0, sizeof(int), st), "replay work reset");
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = std::max(1, std::min(sms * 8, div_up(n, kRW)));
    const bool soft = p.softening > 0.f;
    if (fp64) {
      k_replay64<<<grid, kRW * 32, 0, st>>>(r);
    } else if (adj) {
      if (soft) k_replay<true, true><<<grid, kRW * 32, 0, st>>>(r);
      else k_replay<false, true><<<grid, kRW * 32, 0, st>>>(r);
    } else {
      if (soft) k_replay<true, false><<<grid, kRW * 32, 0, st>>>(r);
      else k_replay<false, false><<<grid, kRW * 32, 0, st>>>(r);
    }
    check(cudaGetLastError(), "k_replay launch");
    launches += 1;
  }

  // Frozen-tape forward from new initial conditions and perturber
  // parameters; final state into out (device).  fp64: FP64 interactions.
  void replay(const double* const* x0, double mass_mj, double radius, double* const* out,
              bool fp64) {
    if (!recorded) throw ArgError("adjoint replay: no recorded forward", NBODY_ERR_STATE);
    if (mode == kModeCheckpoint)
      throw ArgError("adjoint replay: a checkpointed engine keeps no tape to replay (use a "
                     "tape-mode engine)", NBODY_ERR_STATE);
    if (mode == kModeDirect) fp64 = true;
    const size_t n3 = 3 * (size_t)n;
    upload_pert(pert_rep, mass_mj, radius);
    for (int k = 0; k < 3; ++k) {
      check(cudaMemcpyAsync(xw + (size_t)k * n, x0[k], sizeof(double) * n,
                            cudaMemcpyDeviceToDevice, st), "replay positions");
      check(cudaMemcpyAsync(vw + (size_t)k * n, x0[3 + k], sizeof(double) * n,
                            cudaMemcpyDeviceToDevice, st), "replay velocities");
    }
    const int f = fp64 ? 1 : 0;
    check(cudaEventRecord(e0, st), "event");
    run_graph(g_rep[f], [&] {
      check(cudaMemsetAsync(tw.status, 0, sizeof(int), st), "status reset");
      double* xa = xw;
      double* xb = xw + n3;
      for (int L = 0; L <= steps; ++L) {
        const bool end = L > 0, begin = L < steps;
        if (mode == kModeDirect) {  // the direct-sum dynamics from the new inputs
          const double eps2 = (double)p.softening * (double)p.softening;
          k_direct_acc<<<div_up(n, kDirTile), kDirTile, 0, st>>>(xa, mass, n, eps2, aw64);
          launches += 1;
          launch_step(end, begin, step_args<double>(xa, vw, aw64, nullptr, begin ? xb : nullptr,
                                                    pert_rep, L));
          if (begin) std::swap(xa, xb);
          continue;
        }
        level_bodies(L, xa);
        ReplayArgs r = replay_args(L);
        if (fp64) {
          r.dax = aw64; r.day = aw64 + n; r.daz = aw64 + 2 * (size_t)n;
          r.xs = lev_x; r.ys = lev_y; r.zs = lev_z;
          launch_replay(r, false, true);
          launch_step(end, begin, step_args<double>(xa, vw, aw64, nullptr, begin ? xb : nullptr,
                                                    pert_rep, L));
        } else {
          r.ax = aw; r.ay = aw + n; r.az = aw + 2 * (size_t)n;
          launch_replay(r, false);
          launch_step(end, begin, step_args<float>(xa, vw, aw, nullptr, begin ? xb : nullptr,
                                                   pert_rep, L));
        }
        if (begin) std::swap(xa, xb);
      }
      rep_final[f] = xa;
    });
    check(cudaEventRecord(e1, st), "event");
    for (int k = 0; k < 3; ++k) {
      check(cudaMemcpyAsync(out[k], rep_final[f] + (size_t)k * n, sizeof(double) * n,
                            cudaMemcpyDeviceToDevice, st), "replay out");
      check(cudaMemcpyAsync(out[3 + k], vw + (size_t)k * n, sizeof(double) * n,
                            cudaMemcpyDeviceToDevice, st), "replay out");
    }
    const int s = read_status();
    if (s) throw ArgError("adjoint replay: device status " + std::to_string(s), NBODY_ERR_OVERFLOW);
    check(cudaEventElapsedTime(&ms_replay, e0, e1), "event time");
  }

  // Force adjoint at level L: lam (caller order) -> added to gx; then, for
  // L > 0, the drift and first-kick adjoints of step L-1.
  void force_adjoint(int L, bool step) {
    const int sl = slot(L);
    if (mode == kModeDirect) {
      force_adjoint_direct(L, step);
      return;
    }
    level_bodies(L, X[sl]);
    check(cudaMemsetAsync(radd, 0, sizeof(double4) * (n + 1), st), "range add reset");
    ReplayArgs r = replay_args(L);
    r.lx = lam; r.ly = lam + n; r.lz = lam + 2 * (size_t)n;
    r.mux = mu; r.muy = mu + n; r.muz = mu + 2 * (size_t)n;
    r.radd = radd;
    launch_replay(r, true);
    const int ntiles = (n + 1) / kMomentTile + 1;
    double4* tpre = rtiles + (ntiles + 1);
    k_prefix4_tiles<<<ntiles, kThreads, 0, st>>>(radd, n + 1, rploc, rtiles);
    k_tiles_scan4<<<1, 32, 0, st>>>(rtiles, ntiles, tpre);
    ApplyArgs a = apply_args(L);
    a.perm = perm[sl]; a.body4 = tv.body4;
    a.rploc = rploc; a.rtpre = tpre;
    if (step) k_adj_apply<true><<<grid1(n), kThreads, 0, st>>>(a);
    else k_adj_apply<false><<<grid1(n), kThreads, 0, st>>>(a);
    check(cudaGetLastError(), "adjoint apply launch");
    launches += 4;
  }

  // The direct-sum engine's force adjoint at level L: the pairwise
  // vector-Jacobian product, then the per-body star, perturber, drift and
  // kick adjoints.
  void force_adjoint_direct(int L, bool step) {
    const double eps2 = (double)p.softening * (double)p.softening;
    k_direct_vjp<<<div_up(n, kDirTile), kDirTile, 0, st>>>(X[L], mass, lam, n, eps2, mu);
    ApplyArgs a = apply_args(L);
    if (step) k_adj_apply<true, true><<<grid1(n), kThreads, 0, st>>>(a);
    else k_adj_apply<false, true><<<grid1(n), kThreads, 0, st>>>(a);
    check(cudaGetLastError(), "adjoint apply launch");
    launches += 2;
  }

  ApplyArgs apply_args(int L) {
    const int sl = slot(L);
    ApplyArgs a{};
    a.mux = mu; a.muy = mu + n; a.muz = mu + 2 * (size_t)n;
    a.x = X[sl]; a.y = X[sl] + n; a.z = X[sl] + 2 * (size_t)n;
    a.lx = lam; a.ly = lam + n; a.lz = lam + 2 * (size_t)n;
    a.gx = gx; a.gy = gx + n; a.gz = gx + 2 * (size_t)n;
    a.gvx = gv; a.gvy = gv + n; a.gvz = gv + 2 * (size_t)n;
    a.plx = lam; a.ply = lam + n; a.plz = lam + 2 * (size_t)n;  // lam is consumed per body
    a.pert_tab = pert_fwd;
    a.level = L;
    a.eps = p.softening; a.star_mass = p.star_mass;
    a.dt = (double)p.dt; a.dth = (double)p.dt * 0.5;
    a.pgrad = pgrad + 4 * (size_t)L;
    a.n = n;
    return a;
  }

  // Adjoint of the final state (device, caller order) -> adjoint of the
  // initial state and of (perturber mass in M_J, perturber radius in AU).
  void backward(const double* const* g_final, double* const* g_init, double* g_par) {
    if (!recorded) throw ArgError("adjoint backward: no recorded forward", NBODY_ERR_STATE);
    for (int k = 0; k < 3; ++k) {
      check(cudaMemcpyAsync(gx + (size_t)k * n, g_final[k], sizeof(double) * n,
                            cudaMemcpyDeviceToDevice, st), "final adjoint");
      check(cudaMemcpyAsync(gv + (size_t)k * n, g_final[3 + k], sizeof(double) * n,
                            cudaMemcpyDeviceToDevice, st), "final adjoint");
    }
    check(cudaEventRecord(e0, st), "event");
    run_graph(g_bwd, [&] { backward_levels(); });
    check(cudaEventRecord(e1, st), "event");
    finish_backward(g_init, g_par);
  }

  // The drift, second-kick and drag adjoints of step L (levels L and L+1).
  template <typename TA>
  void drag_adjoint(int L, const TA* a0, const TA* a1) {
    const int s0 = slot(L), s1 = slot(L + 1);
    DragAdjArgsT<TA> d{};
    d.x0 = X[s0]; d.y0 = X[s0] + n; d.z0 = X[s0] + 2 * (size_t)n;
    d.v0x = V[s0]; d.v0y = V[s0] + n; d.v0z = V[s0] + 2 * (size_t)n;
    d.a0x = a0; d.a0y = a0 + n; d.a0z = a0 + 2 * (size_t)n;
    d.x1 = X[s1]; d.y1 = X[s1] + n; d.z1 = X[s1] + 2 * (size_t)n;
    d.a1x = a1; d.a1y = a1 + n; d.a1z = a1 + 2 * (size_t)n;
    d.pert_tab = pert_fwd;
    d.level = L;
    d.eps = p.softening; d.star_mass = p.star_mass; d.dth = (double)p.dt * 0.5;
    d.drag = p.gas_drag_rate > 0.f;
    d.decay = d.drag ? std::exp(-(double)p.gas_drag_rate * (double)p.dt) : 1.0;
    d.gx = gx; d.gy = gx + n; d.gz = gx + 2 * (size_t)n;
    d.gvx = gv; d.gvy = gv + n; d.gvz = gv + 2 * (size_t)n;
    d.plx = lam; d.ply = lam + n; d.plz = lam + 2 * (size_t)n;
    d.n = n;
    k_adj_drag<TA><<<grid1(n), kThreads, 0, st>>>(d);
    check(cudaGetLastError(), "k_adj_drag launch");
    launches += 1;
  }

  // Every level of the backward (captured as one graph).
  void backward_levels() {
    const size_t n3 = 3 * (size_t)n;
    check(cudaMemsetAsync(lam, 0, sizeof(double) * n3, st), "pending reset");
    check(cudaMemsetAsync(pgrad, 0, sizeof(double) * 4 * (steps + 1), st), "perturber reset");
    check(cudaMemsetAsync(tw.status, 0, sizeof(int), st), "status reset");
    if (mode == kModeCheckpoint) {
      backward_levels_reversed();
      return;
    }
    for (int L = steps - 1; L >= 0; --L) {
      if (mode == kModeDirect) drag_adjoint<double>(L, AD[L], AD[L + 1]);
      else drag_adjoint<float>(L, A[L], A[L + 1]);
      force_adjoint(L + 1, true);
    }
    force_adjoint(0, false);
  }

  // Checkpoint mode: level `steps` is still in its slot from the forward.
  // Each earlier level is rebuilt by running step L-1 backwards from level L
  // (k_dstep_rev), its tree and tape re-recorded (which also gives its
  // self-gravity, so the first kick is undone too, k_kick_rev); a level that
  // holds a checkpoint is copied back exactly instead.
  // The rebuilds form one chain R(L) (level L-1 from level L) on rev_st, the
  // differentiation another, D(L) (the drag and second-kick adjoints of step
  // L-1, then the force adjoint at level L), on the engine stream.  D(L)
  // waits for R(L); R(L) writes the slot and tape pool of level L-1, which
  // with three of each is level L+2's, so it waits for D(L+2) and runs beside
  // D(L+1).  The two chains use disjoint buffers (tw and xs..zs for the
  // rebuilds; tv, lev_x..z and work_b for the adjoints); the order of every
  // computation is that of the serial loop, so the gradients are the same.
  void backward_levels_reversed() {
    const size_t n3 = 3 * (size_t)n;
    const double dth = (double)p.dt * 0.5;
    if (!rev_st) check(cudaStreamCreateWithFlags(&rev_st, cudaStreamNonBlocking), "rebuild stream");
    if (bwd_events.empty()) {
      bwd_events.resize(2 * (size_t)(steps + 2) + 1);
      for (cudaEvent_t& e : bwd_events)
        check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "backward event");
    }
    cudaEvent_t* evR = bwd_events.data();              // R(L) done, L = 1..steps
    cudaEvent_t* evD = bwd_events.data() + steps + 2;  // D(L) done, L = 1..steps
    cudaEvent_t fork = bwd_events.back();
    cudaStream_t dst = st;
    check(cudaEventRecord(fork, dst), "backward fork");
    check(cudaStreamWaitEvent(rev_st, fork, 0), "backward fork");
    for (int L = steps; L >= 1; --L) {
      const int Lm = L - 1, s = slot(L), sm = slot(Lm);
      const bool ck = (Lm % every) == 0;
      // R(L) on the rebuild stream
      if (L + 2 <= steps) check(cudaStreamWaitEvent(rev_st, evD[L + 2], 0), "slot reuse");
      st = rev_st;
      if (ck) {
        const double* c = CK[Lm / every];
        check(cudaMemcpyAsync(X[sm], c, sizeof(double) * n3, cudaMemcpyDeviceToDevice, st),
              "checkpoint x");
        check(cudaMemcpyAsync(V[sm], c + n3, sizeof(double) * n3, cudaMemcpyDeviceToDevice, st),
              "checkpoint v");
      } else {
        RevArgs r{};
        r.x = X[s]; r.vx = V[s]; r.ax = A[s];
        r.pert_tab = pert_fwd; r.level = L;
        r.px = X[sm]; r.vh = vh;
        r.eps = p.softening; r.star_mass = p.star_mass;
        r.dt = (double)p.dt; r.dth = dth;
        r.drag = p.gas_drag_rate > 0.f;
        r.decay = r.drag ? std::exp(-(double)p.gas_drag_rate * (double)p.dt) : 1.0;
        r.n = n;
        k_dstep_rev<<<grid1(n), kThreads, 0, st>>>(r);
        check(cudaGetLastError(), "k_dstep_rev launch");
        launches += 1;
      }
      record_level(Lm);
      if (!ck) {
        k_kick_rev<<<grid1(n), kThreads, 0, st>>>(X[sm], vh, A[sm], pert_fwd, Lm, p.softening,
                                                   p.star_mass, dth, V[sm], n);
        check(cudaGetLastError(), "k_kick_rev launch");
        launches += 1;
      }
      check(cudaEventRecord(evR[L], st), "rebuild done");
      // D(L) on the engine stream
      st = dst;
      check(cudaStreamWaitEvent(st, evR[L], 0), "rebuild wait");
      drag_adjoint<float>(Lm, A[sm], A[s]);
      force_adjoint(L, true);
      check(cudaEventRecord(evD[L], st), "adjoint done");
    }
    force_adjoint(0, false);  // R(1), the last rebuild, was waited for by D(1)
  }

  void finish_backward(double* const* g_init, double* g_par) {
    for (int k = 0; k < 3; ++k) {
      check(cudaMemcpyAsync(g_init[k], gx + (size_t)k * n, sizeof(double) * n,
                            cudaMemcpyDeviceToDevice, st), "initial adjoint");
      check(cudaMemcpyAsync(g_init[3 + k], gv + (size_t)k * n, sizeof(double) * n,
                            cudaMemcpyDeviceToDevice, st), "initial adjoint");
    }
    std::vector<double> pg(4 * (size_t)(steps + 1));
    check(cudaMemcpyAsync(pg.data(), pgrad, sizeof(double) * pg.size(), cudaMemcpyDeviceToHost,
                          st), "perturber adjoints");
    const int s = read_status();
    if (s) throw ArgError("adjoint backward: device status " + std::to_string(s),
                          NBODY_ERR_OVERFLOW);
    check(cudaEventElapsedTime(&ms_backward, e0, e1), "event time");
    // chain: p(t) = r (cos phi, 0, sin phi), phi = phi0 + sqrt(M / r^3) t;
    // mass in M_sun = mass_mj * mjup
    double gm = 0.0, gr = 0.0;
    if (p.perturber_enabled) {
      const double r = pr;
      const double om = std::sqrt((double)p.star_mass / (r * r * r));
      for (int L = 0; L <= steps; ++L) {
        const double t = (double)L * (double)p.dt;
        const double phi = (double)p.perturber_phase0 + om * t;
        const double c = std::cos(phi), sn = std::sin(phi);
        const double k = -1.5 * om * t;  // r dphi/dr
        const double dpx = c - k * sn, dpz = sn + k * c;
        gr += pg[4 * L + 0] * dpx + pg[4 * L + 2] * dpz;
        gm += pg[4 * L + 3] * mjup;
      }
    }
    g_par[0] = gm;
    g_par[1] = gr;
  }

  // Device memory that holds the forward for the backward: the tape (chunk
  // pools and per-level permutation and groups) and the level states
  // (checkpoints included).
  size_t tape_bytes() const {
    const size_t pools = n_pools();
    return pools * (size_t)pool_cap * (kTapeChunk * sizeof(int2) + sizeof(int)) +
           perm.size() * n * (sizeof(uint32_t) + 2 * sizeof(int2));
  }
  size_t state_bytes() const {
    const size_t lv = X.size() * n * 6 * sizeof(double) + A.size() * n * 3 * sizeof(float) +
                      AD.size() * n * 3 * sizeof(double);
    return lv + CK.size() * n * 6 * sizeof(double) + (vh ? n * 3 * sizeof(double) : 0);
  }
};

}  // namespace nb

struct nbody_adjoint {
  nb::AdjointImpl* impl;
};

extern "C" {

int nbody_adjoint_create_mode(const nbody_sim_params* p, int n, int n_steps, int mode,
                              int checkpoint_every, nbody_adjoint** out) {
  NBODY_API_BODY({
    NBODY_REQUIRE(p && out, "nbody_adjoint_create: null argument");
    *out = nullptr;
    NBODY_REQUIRE(n >= 2 && n < (1 << 26), "nbody_adjoint_create: n must be in [2, 2^26)");
    NBODY_REQUIRE(n_steps >= 1, "nbody_adjoint_create: n_steps must be >= 1");
    NBODY_REQUIRE(p->dt > 0.f, "nbody_adjoint_create: dt must be positive");
    NBODY_REQUIRE(p->r_coll <= 0.f,
                  "nbody_adjoint_create: collisions are not differentiable (r_coll must be 0)");
    NBODY_REQUIRE(mode == NBODY_ADJOINT_TAPE || mode == NBODY_ADJOINT_CHECKPOINT ||
                      mode == NBODY_ADJOINT_DIRECT,
                  "nbody_adjoint_create: unknown mode");
    NBODY_REQUIRE(mode != NBODY_ADJOINT_CHECKPOINT || checkpoint_every >= 1,
                  "nbody_adjoint_create: checkpoint_every must be >= 1");
    NBODY_REQUIRE(mode != NBODY_ADJOINT_DIRECT || n <= (1 << 20),
                  "nbody_adjoint_create: the direct-sum engine is O(N^2) per step; n <= 2^20");
    *out = new nbody_adjoint{new nb::AdjointImpl(*p, n, n_steps, mode, checkpoint_every)};
  })
}

int nbody_adjoint_create(const nbody_sim_params* p, int n, int n_steps, nbody_adjoint** out) {
  return nbody_adjoint_create_mode(p, n, n_steps, NBODY_ADJOINT_TAPE, 0, out);
}

int nbody_adjoint_destroy(nbody_adjoint* a) {
  NBODY_API_BODY({
    if (a) {
      delete a->impl;
      delete a;
    }
  })
}

int nbody_adjoint_set_stream(nbody_adjoint* a, void* stream) {
  NBODY_API_BODY({
    NBODY_REQUIRE(a, "nbody_adjoint_set_stream: null handle");
    a->impl->set_stream((cudaStream_t)stream);
  })
}

int nbody_adjoint_forward(nbody_adjoint* a, const double* x0, const double* y0, const double* z0,
                          const double* vx0, const double* vy0, const double* vz0,
                          const float* mass, double perturber_mass_mjup,
                          double perturber_radius_au, double* x, double* y, double* z,
                          double* vx, double* vy, double* vz) {
  NBODY_API_BODY({
    NBODY_REQUIRE(a && x0 && y0 && z0 && vx0 && vy0 && vz0 && mass,
                  "nbody_adjoint_forward: null input");
    NBODY_REQUIRE(perturber_radius_au > 0.0, "nbody_adjoint_forward: radius must be positive");
    const double* in[6] = {x0, y0, z0, vx0, vy0, vz0};
    nb::AdjointImpl* m = a->impl;
    m->forward(in, mass, perturber_mass_mjup, perturber_radius_au);
    double* out[6] = {x, y, z, vx, vy, vz};
    const size_t n = m->n;
    for (int k = 0; k < 6; ++k)
      if (out[k]) {
        const int sl = m->slot(m->steps);
        const double* src = (k < 3 ? m->X[sl] : m->V[sl]) + (k % 3) * n;
        nb::check(cudaMemcpyAsync(out[k], src, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                  m->st), "forward out");
      }
    nb::check(cudaStreamSynchronize(m->st), "forward sync");
  })
}

int nbody_adjoint_replay(nbody_adjoint* a, const double* x0, const double* y0, const double* z0,
                         const double* vx0, const double* vy0, const double* vz0,
                         double perturber_mass_mjup, double perturber_radius_au, int fp64,
                         double* x, double* y, double* z, double* vx, double* vy, double* vz) {
  NBODY_API_BODY({
    NBODY_REQUIRE(a && x0 && y0 && z0 && vx0 && vy0 && vz0 && x && y && z && vx && vy && vz,
                  "nbody_adjoint_replay: null array");
    NBODY_REQUIRE(perturber_radius_au > 0.0, "nbody_adjoint_replay: radius must be positive");
    const double* in[6] = {x0, y0, z0, vx0, vy0, vz0};
    double* out[6] = {x, y, z, vx, vy, vz};
    a->impl->replay(in, perturber_mass_mjup, perturber_radius_au, out, fp64 != 0);
  })
}

int nbody_adjoint_backward(nbody_adjoint* a, const double* gx, const double* gy, const double* gz,
                           const double* gvx, const double* gvy, const double* gvz,
                           double* gx0, double* gy0, double* gz0, double* gvx0, double* gvy0,
                           double* gvz0, double* g_perturber) {
  NBODY_API_BODY({
    NBODY_REQUIRE(a && gx && gy && gz && gvx && gvy && gvz && gx0 && gy0 && gz0 && gvx0 &&
                      gvy0 && gvz0 && g_perturber,
                  "nbody_adjoint_backward: null array");
    const double* gin[6] = {gx, gy, gz, gvx, gvy, gvz};
    double* gout[6] = {gx0, gy0, gz0, gvx0, gvy0, gvz0};
    a->impl->backward(gin, gout, g_perturber);
  })
}

int nbody_adjoint_stats_get(nbody_adjoint* a, nbody_adjoint_stats* out) {
  NBODY_API_BODY({
    NBODY_REQUIRE(a && out, "nbody_adjoint_stats_get: null argument");
    nb::AdjointImpl* m = a->impl;
    out->n = m->n;
    out->n_steps = m->steps;
    out->ms_forward = m->ms_forward;
    out->ms_backward = m->ms_backward;
    out->ms_replay = m->ms_replay;
    out->tape_bytes = m->tape_bytes();
    out->state_bytes = m->state_bytes();
    out->launches = m->launches;
  })
}

}  // extern "C"
