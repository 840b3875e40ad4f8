// walk.cu -- warp-cooperative Barnes-Hut force walk (FP32 SIMT).
//
// Replaces bhtree_forceKernel (BHTree.cu:530-598; one thread per body, a
// 256-entry local-memory stack) and fuses perturber_forceKernel
// (Perturber.cu:13-35) into its epilogue.
//
// A warp owns a group of 32 targets that are consecutive in Morton order.
// Traversal is shared: the warp pops up to 32 nodes from a per-warp stack in
// shared memory and each lane tests one node against the group's bounding
// box.  A node is accepted when half^2 < theta^2 d^2 with d the distance from
// the group box to the node's centre of mass: every target in the group is
// at least d away, so each target's own reference test half/|x - com| <
// theta (BHTree.cu:577) would accept it too.  Accepted nodes (and single
// bodies) are appended to a shared-memory source list; nodes that must be
// opened either push their contiguous children or, when they hold at most
// leaf_max bodies, append those bodies.  Each full batch of 32 sources is
// evaluated by all 32 lanes for their own target, reading the source from
// shared memory as a broadcast: 12 FP32 instructions + 1 MUFU.RSQ per
// interaction.  The softened self term is exactly zero (d = 0), so no
// self-skip test is needed when softening > 0.
//
// The stack spills to a per-warp global area when it would overflow; a
// spill area that runs out raises kStatusStackOverflow instead of hanging.
#include "common.cuh"
#include "kernels.cuh"

namespace nb {
namespace {

constexpr int kWalkWarps = 4;
constexpr int kStk = 384;
constexpr int kList = 64;

struct WarpSmem {
  float4 lst[kList];
  int stk[kStk];
  int sc[32];
  int slo[32];
};

template <bool kSoft>
__device__ __forceinline__ void interact(const float4 s, float px, float py, float pz,
                                         float eps2, float& ax, float& ay, float& az) {
  float dx = s.x - px, dy = s.y - py, dz = s.z - pz;
  float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
  float inv = rsqrtf(r2);
  if (!kSoft) inv = (r2 > 0.f) ? inv : 0.f;
  float f = s.w * (inv * inv * inv);
  ax = fmaf(f, dx, ax);
  ay = fmaf(f, dy, ay);
  az = fmaf(f, dz, az);
}

template <bool kSoft>
__device__ __forceinline__ void eval32(const float4* lst, float px, float py, float pz,
                                       float eps2, float& ax, float& ay, float& az) {
#pragma unroll
  for (int j = 0; j < 32; ++j) interact<kSoft>(lst[j], px, py, pz, eps2, ax, ay, az);
}

// Drops the first 32 entries of the list (caller guarantees nlist >= 32).
__device__ __forceinline__ void list_shift(float4* lst, int nlist, int lane) {
  const int rem = nlist - 32;
  float4 t;
  if (lane < rem) t = lst[32 + lane];
  __syncwarp();
  if (lane < rem) lst[lane] = t;
  __syncwarp();
}

template <bool kSoft>
__global__ void __launch_bounds__(kWalkWarps * 32) k_walk(const WalkArgs a) {
  __shared__ WarpSmem smem[kWalkWarps];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  WarpSmem& w = smem[wib];
  int* spill = a.spill + (size_t)(blockIdx.x * kWalkWarps + wib) * (size_t)a.spill_cap;
  const int n_groups = *a.n_groups;
  const float eps2 = a.eps * a.eps;

  while (true) {
    int g = 0;
    if (lane == 0) g = atomicAdd(a.work, 1);
    g = __shfl_sync(kFull, g, 0);
    if (g >= n_groups) break;
    const int2 gr = a.groups[g];
    const int s = gr.x + lane;
    const bool valid = lane < gr.y;
    const float4 me = a.body[valid ? s : gr.x];
    const float gx0 = warp_min(me.x), gx1 = warp_max(me.x);
    const float gy0 = warp_min(me.y), gy1 = warp_max(me.y);
    const float gz0 = warp_min(me.z), gz1 = warp_max(me.z);

    // The tree sum starts from zero: adding ~10^3 terms into an accumulator
    // that already holds the star pull (10^3-10^5 times larger) would round
    // every term at the star's ulp.  Star and perturber are added at the end.
    float ax = 0.f, ay = 0.f, az = 0.f;
    unsigned long long visited = 0, spills = 0;

    int top = 1, spilled = 0, nlist = 0;
    unsigned long long evaluated = 0;
    bool overflow = false;
    if (lane == 0) w.stk[0] = 0;
    __syncwarp();

    while (true) {
      if (top == 0) {
        if (spilled == 0) break;
        const int cnt = min(spilled, kStk / 2);
        for (int k = lane; k < cnt; k += 32) w.stk[k] = __ldcg(spill + (spilled - cnt) + k);
        spilled -= cnt;
        top = cnt;
        __syncwarp();
      }
      const int take = min(top, 32);
      top -= take;
      visited += take;
      const int node = (lane < take) ? w.stk[top + lane] : -1;
      __syncwarp();

      int act = 0;  // 1: source, 2: bodies of a leaf, 3: open children
      float4 c = make_float4(0.f, 0.f, 0.f, 0.f);
      int first = 0, cnt = 0;
      if (node >= 0) {
        c = __ldg(a.com + node);
        const int4 inf = __ldg(a.info + node);
        cnt = inf.z >> 4;
        const int nch = inf.z & 15;
        const float half = __int_as_float(inf.w);
        if (cnt == 1) {
          act = 1;
        } else {
          const float dx = fmaxf(fmaxf(gx0 - c.x, c.x - gx1), 0.f);
          const float dy = fmaxf(fmaxf(gy0 - c.y, c.y - gy1), 0.f);
          const float dz = fmaxf(fmaxf(gz0 - c.z, c.z - gz1), 0.f);
          const float d2 = dx * dx + dy * dy + dz * dz;
          if (half * half < a.theta2 * d2) {
            act = 1;
          } else if (nch == 0 || cnt <= a.leaf_max) {
            act = 2;
            first = inf.y;
          } else {
            act = 3;
            first = inf.x;
            cnt = nch;
          }
        }
      }

      // accepted sources -> list
      const unsigned m1 = __ballot_sync(kFull, act == 1);
      if (act == 1) w.lst[nlist + __popc(m1 & lanemask_lt())] = c;
      nlist += __popc(m1);
      __syncwarp();
      if (nlist >= 32) {
        eval32<kSoft>(w.lst, me.x, me.y, me.z, eps2, ax, ay, az);
        evaluated += 32;
        list_shift(w.lst, nlist, lane);
        nlist -= 32;
      }

      // opened nodes -> children on the stack
      const int pc = (act == 3) ? cnt : 0;
      const int pincl = warp_incl_scan(pc, lane);
      const int ptotal = __shfl_sync(kFull, pincl, 31);
      if (ptotal > 0) {
        if (top + ptotal > kStk) {
          if (spilled + top > a.spill_cap) { overflow = true; break; }
          ++spills;
          for (int k = lane; k < top; k += 32) __stcg(spill + spilled + k, w.stk[k]);
          spilled += top;
          top = 0;
          __syncwarp();
        }
        const int base = top + pincl - pc;
        for (int k = 0; k < pc; ++k) w.stk[base + k] = first + k;
        top += ptotal;
        __syncwarp();
      }

      // leaves to open -> their bodies into the list, 32 at a time
      const int bc = (act == 2) ? cnt : 0;
      const int bincl = warp_incl_scan(bc, lane);
      const int btotal = __shfl_sync(kFull, bincl, 31);
      if (btotal > 0) {
        w.sc[lane] = bincl;
        w.slo[lane] = first;
        __syncwarp();
        for (int base = 0; base < btotal; base += 32) {
          const int gi = base + lane;
          if (gi < btotal) {
            int o = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1)
              if (w.sc[o + step - 1] <= gi) o += step;
            const int prev = (o > 0) ? w.sc[o - 1] : 0;
            w.lst[nlist + lane] = __ldg(a.body + w.slo[o] + (gi - prev));
          }
          nlist += min(32, btotal - base);
          __syncwarp();
          if (nlist >= 32) {
            eval32<kSoft>(w.lst, me.x, me.y, me.z, eps2, ax, ay, az);
            evaluated += 32;
            list_shift(w.lst, nlist, lane);
            nlist -= 32;
          }
        }
      }
    }

    for (int j = 0; j < nlist; ++j) interact<kSoft>(w.lst[j], me.x, me.y, me.z, eps2, ax, ay, az);
    evaluated += nlist;
    __syncwarp();

    if (a.star_in_walk) {  // softened star term, BHTree.cu:547-553
      float dx = -me.x, dy = -me.y, dz = -me.z;
      float r2 = dx * dx + dy * dy + dz * dz + a.eps * a.eps;
      float r = sqrtf(r2);
      float f = a.star_mass / (r2 * r);
      ax += f * dx; ay += f * dy; az += f * dz;
    }
    if (a.pert) {  // perturber_forceKernel, Perturber.cu:20-34 (adds)
      const float4 p = *a.pert;
      float dx = p.x - me.x, dy = p.y - me.y, dz = p.z - me.z;
      float r2 = dx * dx + dy * dy + dz * dz + a.eps * a.eps;
      float r = sqrtf(r2);
      float f = p.w / (r2 * r);
      ax += f * dx; ay += f * dy; az += f * dz;
    }
    if (valid) {
      const uint32_t o = a.scatter ? a.scatter[s] : (uint32_t)s;
      a.ax[o] = ax;
      a.ay[o] = ay;
      a.az[o] = az;
    }
    const int nvalid = __popc(__ballot_sync(kFull, valid));
    if (lane == 0) {
      if (overflow) atomicOr(a.status, kStatusStackOverflow);
      atomicAdd(a.inter, evaluated * (unsigned long long)nvalid);
      if (a.counters) {
        atomicAdd(a.counters + 0, visited);
        atomicAdd(a.counters + 1, spills);
        atomicAdd(a.counters + 2, 1ull);
      }
    }
  }
}

int g_walk_blocks_per_sm[2] = {0, 0};

int walk_blocks_per_sm(bool soft) {
  int& b = g_walk_blocks_per_sm[soft ? 1 : 0];
  if (b == 0) {
    if (soft)
      check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_walk<true>, kWalkWarps * 32, 0),
            "walk occupancy");
    else
      check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_walk<false>, kWalkWarps * 32, 0),
            "walk occupancy");
    if (b < 1) b = 1;
  }
  return b;
}

int num_sms() {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
  }
  return sms;
}

}  // namespace

int walk_spill_slots(int) {
  return num_sms() * std::max(walk_blocks_per_sm(true), walk_blocks_per_sm(false)) * kWalkWarps;
}

void launch_walk(const WalkArgs& a, cudaStream_t s) {
  if (a.n <= 0) return;
  const bool soft = a.eps > 0.f;
  const int groups = a.n;  // upper bound on the group count
  int grid = num_sms() * walk_blocks_per_sm(soft);
  grid = std::min(grid, (groups + kWalkWarps - 1) / kWalkWarps);
  if (grid < 1) grid = 1;
  check(cudaMemsetAsync(a.work, 0, sizeof(int), s), "walk work reset");
  if (soft)
    k_walk<true><<<grid, kWalkWarps * 32, 0, s>>>(a);
  else
    k_walk<false><<<grid, kWalkWarps * 32, 0, s>>>(a);
  check(cudaGetLastError(), "k_walk launch");
}

}  // namespace nb
