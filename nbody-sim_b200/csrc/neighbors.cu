// neighbors.cu -- fixed-radius neighbour search over the octree: the
// two-pass collision impulse and the FoF links + union-find.
//
// Collision replaces bhtree_collisionKernel (BHTree.cu:620-673).  The
// reference prunes a cell when |x - com| - 1.732 half >= r_coll, which can
// skip pairs whose cell COM is off-centre; here a warp group of 32 targets
// descends every node whose tight AABB overlaps the group box grown by the
// radius, so every pair with dist2 < r_coll^2 is found.  The per-pair
// impulse is the reference's (BHTree.cu:650-660): dv_i -= J n with
// J = -(1+e) dvn / 2 for approaching pairs, computed from pre-collision
// velocities (two-pass semantics).
//
// FoF links use the exact test of detectAggregates (Aggregate.cpp:36-42),
// ((dx*dx + dy*dy) + dz*dz) < ll*ll in FP32 without contraction, so the
// linked pair set, the components and their smallest-index labels are
// bit-identical to the host O(N^2) loop.  Union-find always hooks the larger
// root under the smaller one, so every root is its component's smallest
// original index; every loop is bounded and reports kStatusUnionFindLimit.
#include "collide_math.cuh"
#include "common.cuh"
#include "kernels.cuh"

namespace nb {
namespace {

constexpr int kNbWarps = 4;
constexpr int kStk = 384;

struct NbSmem {
  float4 pos[64];
  int idx[64];
  int stk[kStk];
  int sc[32];
  int slo[32];
};

__device__ __forceinline__ int uf_find(int* parent, int x) {
  for (int guard = 0; guard < (1 << 26); ++guard) {
    int p = __ldcg(parent + x);
    if (p == x) return x;
    int gp = __ldcg(parent + p);
    if (gp != p) atomicCAS(parent + x, p, gp);  // path halving; parents only decrease
    x = p;
  }
  return -1;
}

__device__ void uf_union(int* parent, int a, int b, int* status) {
  for (int guard = 0; guard < (1 << 20); ++guard) {
    a = uf_find(parent, a);
    b = uf_find(parent, b);
    if (a < 0 || b < 0) break;
    if (a == b) return;
    if (a > b) { int t = a; a = b; b = t; }
    int old = atomicCAS(parent + b, b, a);
    if (old == b) return;
    b = old;
  }
  atomicOr(status, kStatusUnionFindLimit);
}

struct CollideOut {
  const void* vx;   // velocities in the state's storage type (vtype)
  const void* vy;
  const void* vz;
  int vtype;        // 0 float, 1 double, 2 hi/lo float pairs
  const uint32_t* vmap;
  float rc2;
  float e;
  float* dvx;
  float* dvy;
  float* dvz;
  // report mode: the octree's centres of mass, r_coll and the two counters
  // (pairs, pairs the reference's cell prune would skip)
  const float4* com;
  unsigned long long* report;
};

// Whether bhtree_collisionKernel would skip the pair (target at xi, sorted
// body j): descending the octree cells that contain j, the first whose
// |com - x_i| - 1.732 half is not below r_coll is pruned (BHTree.cu:663-665;
// the same float operations, without contraction).  A chain of single-child
// cells shares one centre of mass, so testing its smallest cell, the one the
// compressed octree keeps, decides the whole chain.  Cells below the tenth
// level (inside a bucket of equal keys) are not modelled.
__device__ bool ref_prunes(const float4* __restrict__ com, const int4* __restrict__ info,
                           float4 xi, int j, float r) {
  int node = 0;
  for (int depth = 0; depth < 64; ++depth) {
    const int4 inf = __ldg(info + node);
    const int nch = inf.z & 15;
    if (nch == 0) return false;  // a leaf: the reference tests the bodies themselves
    const float4 c = __ldg(com + node);
    const float dx = c.x - xi.x, dy = c.y - xi.y, dz = c.z - xi.z;
    const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    const float half = __int_as_float(inf.w);
    if (!(__fsub_rn(sqrtf(d2), __fmul_rn(half, 1.732f)) < r)) return true;
    int next = -1;
    for (int k = 0; k < nch; ++k) {
      const int4 ci = __ldg(info + inf.x + k);
      if (j >= ci.y && j < ci.y + (ci.z >> 4)) {
        next = inf.x + k;
        break;
      }
    }
    if (next < 0) return false;
    node = next;
  }
  return false;
}

struct FofOut {
  const uint32_t* ids;
  float ll2;
  int* parent;
};

template <int kMode>  // 0: collision impulse, 1: FoF links, 2: collision pair report
__global__ void __launch_bounds__(kNbWarps * 32)
k_neighbors(const NeighborArgs a, float radius, CollideOut co, FofOut fo) {
  __shared__ NbSmem smem[kNbWarps];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  NbSmem& w = smem[wib];
  int* spill = a.spill + (size_t)(blockIdx.x * kNbWarps + wib) * (size_t)a.spill_cap;
  const int n_groups = *a.n_groups;
  // conservative per-axis reach: a pair that passes the FP32 test is closer
  // than radius (1 + 2^-20) on every axis
  const float reach = radius * 1.00001f + 1e-30f;

  while (true) {
    int g = 0;
    if (lane == 0) g = atomicAdd(a.work, 1);
    g = __shfl_sync(kFull, g, 0);
    if (g >= n_groups) break;
    const int2 grp = a.groups[g];
    const int disk = a.group_disk ? a.group_disk[g] : 0;
    // groups hold up to 64 bodies; search them 32 (one per lane) at a time
    for (int c0 = 0; c0 < grp.y; c0 += 32) {
    const int2 gr = make_int2(grp.x + c0, min(32, grp.y - c0));
    const int s = gr.x + lane;
    const bool valid = lane < gr.y;
    const float4 me = a.body[valid ? s : gr.x];
    const float gx0 = warp_min(me.x) - reach, gx1 = warp_max(me.x) + reach;
    const float gy0 = warp_min(me.y) - reach, gy1 = warp_max(me.y) + reach;
    const float gz0 = warp_min(me.z) - reach, gz1 = warp_max(me.z) + reach;

    float vix = 0.f, viy = 0.f, viz = 0.f;
    if (kMode == 0 && valid) {
      const uint32_t vi = co.vmap ? co.vmap[s] : (uint32_t)s;
      vix = coll_vel(co.vx, co.vtype, vi);
      viy = coll_vel(co.vy, co.vtype, vi);
      viz = coll_vel(co.vz, co.vtype, vi);
    }
    float dvx = 0.f, dvy = 0.f, dvz = 0.f;
    unsigned long long npairs = 0, nmissed = 0;
    const int my_id = (kMode == 1 && valid) ? (int)fo.ids[s] : 0;

    int top = 1, spilled = 0;
    bool overflow = false;
    if (lane == 0) w.stk[0] = disk;  // root slot of the group's disk
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
      const int node = (lane < take) ? w.stk[top + lane] : -1;
      __syncwarp();
      int act = 0, first = 0, cnt = 0;
      if (node >= 0) {
        const float4 lo = __ldg(a.box_lo + node), hi = __ldg(a.box_hi + node);
        const bool overlap = lo.x <= gx1 && hi.x >= gx0 && lo.y <= gy1 && hi.y >= gy0 &&
                             lo.z <= gz1 && hi.z >= gz0;
        if (overlap) {
          const int4 inf = __ldg(a.info + node);
          cnt = inf.z >> 4;
          const int nch = inf.z & 15;
          if (nch == 0 || cnt <= a.leaf_max) {
            act = 2;
            first = inf.y;
          } else {
            act = 3;
            first = inf.x;
            cnt = nch;
          }
        }
      }
      const int pc = (act == 3) ? cnt : 0;
      const int pincl = warp_incl_scan(pc, lane);
      const int ptotal = __shfl_sync(kFull, pincl, 31);
      if (ptotal > 0) {
        if (top + ptotal > kStk) {
          if (spilled + top > a.spill_cap) { overflow = true; break; }
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
      const int bc = (act == 2) ? cnt : 0;
      const int bincl = warp_incl_scan(bc, lane);
      const int btotal = __shfl_sync(kFull, bincl, 31);
      if (btotal == 0) continue;
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
          const int j = w.slo[o] + (gi - prev);
          w.pos[lane] = __ldg(a.body + j);
          w.idx[lane] = j;
        }
        const int chunk = min(32, btotal - base);
        __syncwarp();
        if (valid) {
          for (int k = 0; k < chunk; ++k) {
            const float4 q = w.pos[k];
            const int j = w.idx[k];
            if (kMode == 0) {
              // BHTree.cu:642-660 (leaf branch), j != i
              const float dx = q.x - me.x, dy = q.y - me.y, dz = q.z - me.z;
              const float dist2 = coll_dist2(dx, dy, dz);
              if (j != s && dist2 < co.rc2) {
                const uint32_t vj = co.vmap ? co.vmap[j] : (uint32_t)j;
                coll_impulse(dx, dy, dz, dist2, coll_vel(co.vx, co.vtype, vj) - vix,
                             coll_vel(co.vy, co.vtype, vj) - viy,
                             coll_vel(co.vz, co.vtype, vj) - viz, co.e, dvx, dvy, dvz);
              }
            } else if (kMode == 2) {
              const float dx = q.x - me.x, dy = q.y - me.y, dz = q.z - me.z;
              if (j != s && coll_dist2(dx, dy, dz) < co.rc2) {
                ++npairs;
                if (ref_prunes(co.com, a.info, me, j, radius)) ++nmissed;
              }
            } else if (j > s) {
              // Aggregate.cpp:38-40, no FMA contraction
              float dx = __fsub_rn(me.x, q.x), dy = __fsub_rn(me.y, q.y),
                    dz = __fsub_rn(me.z, q.z);
              float d2 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)),
                                   __fmul_rn(dz, dz));
              if (d2 < fo.ll2) uf_union(fo.parent, my_id, (int)fo.ids[j], a.status);
            }
          }
        }
        __syncwarp();
      }
    }
    if (kMode == 0 && valid) {
      co.dvx[s] = dvx;
      co.dvy[s] = dvy;
      co.dvz[s] = dvz;
    }
    if (kMode == 2) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        npairs += __shfl_xor_sync(kFull, npairs, o);
        nmissed += __shfl_xor_sync(kFull, nmissed, o);
      }
      if (lane == 0 && npairs) atomicAdd(co.report, npairs);
      if (lane == 0 && nmissed) atomicAdd(co.report + 1, nmissed);
    }
    if (lane == 0 && overflow) atomicOr(a.status, kStatusStackOverflow);
    }  // chunks of the group
  }
}

__global__ void k_fof_init(int* parent, int n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    parent[i] = (int)i;
}

__global__ void k_fof_labels(int* parent, int n, int* labels, int* sizes, int* status) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    int r = uf_find(parent, (int)i);
    if (r < 0) { atomicOr(status, kStatusUnionFindLimit); r = (int)i; }
    labels[i] = r;
    atomicAdd(sizes + r, 1);
  }
}

__global__ void k_fof_sizes(const int* labels, const int* sizes, int n, uint16_t* agg_size,
                            int* n_groups) {
  int local = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    int c = sizes[labels[i]];
    agg_size[i] = (uint16_t)(c >= 2 ? (c < 65535 ? c : 65535) : 1);
    if (labels[i] == (int)i && c >= 2) ++local;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(kFull, local, o);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(n_groups, local);
}

int g_nb_blocks_per_sm[3] = {0, 0, 0};

template <int kMode>
int nb_blocks_per_sm() {
  int& b = g_nb_blocks_per_sm[kMode];
  if (b == 0) {
    check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_neighbors<kMode>, kNbWarps * 32, 0),
          "neighbors occupancy");
    if (b < 1) b = 1;
  }
  return b;
}

int sm_count() {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
  }
  return sms;
}

template <int kMode>
void launch_nb(const NeighborArgs& a, float radius, const CollideOut& co, const FofOut& fo,
               cudaStream_t s) {
  if (a.n <= 0) return;
  const int groups = a.n;  // upper bound on the group count
  int grid = sm_count() * nb_blocks_per_sm<kMode>();
  // the spill area is sized for the walk's slot count; never exceed it
  grid = std::min(grid, walk_spill_slots(0) / kNbWarps);
  grid = std::min(grid, (groups + kNbWarps - 1) / kNbWarps);
  if (grid < 1) grid = 1;
  check(cudaMemsetAsync(a.work, 0, sizeof(int), s), "neighbors work reset");
  k_neighbors<kMode><<<grid, kNbWarps * 32, 0, s>>>(a, radius, co, fo);
  check(cudaGetLastError(), "k_neighbors launch");
}

}  // namespace

void launch_collide_v(const NeighborArgs& a, const void* vx, const void* vy, const void* vz,
                      int vtype, const uint32_t* vmap, float r_coll, float restitution,
                      float* dvx, float* dvy, float* dvz, cudaStream_t s) {
  CollideOut co{vx, vy, vz, vtype, vmap, r_coll * r_coll, restitution, dvx, dvy, dvz, nullptr,
                nullptr};
  FofOut fo{nullptr, 0.f, nullptr};
  launch_nb<0>(a, r_coll, co, fo, s);
}

void launch_collide(const NeighborArgs& a, const float* vx, const float* vy, const float* vz,
                    const uint32_t* vmap, float r_coll, float restitution, float* dvx,
                    float* dvy, float* dvz, cudaStream_t s) {
  launch_collide_v(a, vx, vy, vz, 0, vmap, r_coll, restitution, dvx, dvy, dvz, s);
}

void launch_collision_report(const NeighborArgs& a, const float4* com, float r_coll,
                             unsigned long long* report, cudaStream_t s) {
  check(cudaMemsetAsync(report, 0, 2 * sizeof(unsigned long long), s), "report reset");
  CollideOut co{nullptr, nullptr, nullptr, 0, nullptr, r_coll * r_coll, 0.f,
                nullptr, nullptr, nullptr, com, report};
  FofOut fo{nullptr, 0.f, nullptr};
  launch_nb<2>(a, r_coll, co, fo, s);
}

void launch_fof_link(const NeighborArgs& a, const uint32_t* ids, float link_length, int* parent,
                     cudaStream_t s) {
  if (a.n <= 0) return;
  k_fof_init<<<div_up(a.n, 256), 256, 0, s>>>(parent, a.n);
  CollideOut co{nullptr, nullptr, nullptr, 0, nullptr, 0.f, 0.f, nullptr, nullptr, nullptr, nullptr, nullptr};
  const float ll2 = link_length * link_length;  // Aggregate.cpp:30
  FofOut fo{ids, ll2, parent};
  launch_nb<1>(a, link_length, co, fo, s);
}

void launch_fof_finish(int* parent, int n, int* labels, int* sizes, uint16_t* agg_size,
                       int* n_groups, int* status, cudaStream_t s) {
  if (n <= 0) return;
  check(cudaMemsetAsync(sizes, 0, sizeof(int) * (size_t)n, s), "fof sizes reset");
  check(cudaMemsetAsync(n_groups, 0, sizeof(int), s), "fof groups reset");
  const int g = std::min(div_up(n, 256), 148 * 16);
  k_fof_labels<<<g, 256, 0, s>>>(parent, n, labels, sizes, status);
  k_fof_sizes<<<g, 256, 0, s>>>(labels, sizes, n, agg_size, n_groups);
  check(cudaGetLastError(), "fof finish launch");
}

// FoF links with the warp count capped at max_warps, for a caller whose stack
// spill area holds max_warps slots of a.spill_cap entries (the allocation-free
// FoF entry point sizes its static area this way).
void launch_fof_link_capped(const NeighborArgs& a, const uint32_t* ids, float link_length,
                            int* parent, int max_warps, cudaStream_t s) {
  if (a.n <= 0) return;
  k_fof_init<<<div_up(a.n, 256), 256, 0, s>>>(parent, a.n);
  CollideOut co{nullptr, nullptr, nullptr, 0, nullptr, 0.f, 0.f, nullptr, nullptr, nullptr, nullptr, nullptr};
  const float ll2 = link_length * link_length;  // Aggregate.cpp:30
  FofOut fo{ids, ll2, parent};
  int grid = sm_count() * nb_blocks_per_sm<1>();
  grid = std::min(grid, max_warps / kNbWarps);
  grid = std::min(grid, (a.n + kNbWarps - 1) / kNbWarps);
  if (grid < 1) grid = 1;
  check(cudaMemsetAsync(a.work, 0, sizeof(int), s), "neighbors work reset");
  k_neighbors<1><<<grid, kNbWarps * 32, 0, s>>>(a, link_length, co, fo);
  check(cudaGetLastError(), "k_neighbors launch");
}

}  // namespace nb
