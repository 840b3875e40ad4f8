// tree.cu -- on-device octree build: bbox, Morton keys, Karras radix tree,
// FP64 bottom-up moments, compressed octree with contiguous children.
//
// Replaces resetOctree / launchBBoxKernel / launchBuildKernel /
// launchSummarizeKernel of the reference (BHTree.cu:42-317,397-516): no 9N
// node reset, no host round trips for the bbox and the root, no CAS
// insertion, one bottom-up pass instead of 20 summarize launches.
//
// Geometry follows the reference: the bbox is padded x1.001 about its middle
// (BHTree.cu:440-446) and the root half-size pads the largest extent x1.001
// again (BHTree.cu:484-485).  A node at octree level L is the cube of side
// 2*rhs/2^L that the first 3L key bits select; its half-size rhs/2^L is the
// `cell_size` of the reference's opening test (BHTree.cu:577).
#include "common.cuh"
#include "digit_hist.cuh"
#include "kernels.cuh"
#include "moments.cuh"

namespace nb {
namespace {

constexpr int kThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kThreads)
k_bbox(const T* __restrict__ x, const T* __restrict__ y, const T* __restrict__ z, int n,
       unsigned long long* __restrict__ enc) {
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double p[3] = {(double)x[i], (double)y[i], (double)z[i]};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      lo[k] = fmin(lo[k], p[k]);
      hi[k] = fmax(hi[k], p[k]);
    }
  }
  __shared__ double s[6][kThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double a = warp_min(lo[k]), b = warp_max(hi[k]);
    if (lane == 0) { s[k][warp] = a; s[3 + k][warp] = b; }
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    int k = threadIdx.x;
    double v = s[k][0];
    for (int w = 1; w < kThreads / 32; ++w) v = (k < 3) ? fmin(v, s[k][w]) : fmax(v, s[k][w]);
    if (v == v && fabs(v) != INFINITY) {
      if (k < 3) atomicMin(&enc[k], ordered_bits(v));
      else atomicMax(&enc[k], ordered_bits(v));
    }
  }
}

__global__ void k_bbox_reset(unsigned long long* enc) {
  int k = threadIdx.x;
  if (k < 6) enc[k] = (k < 3) ? ~0ull : 0ull;
}

// Root geometry from the encoded bbox, float arithmetic as the reference host
// code (BHTree.cu:440-446 then :481-485).
__device__ void compute_geom(const unsigned long long* enc, TreeGeom& g) {
  float bmin[3], bmax[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double lo = from_ordered_bits(enc[k]), hi = from_ordered_bits(enc[3 + k]);
    if (!(lo <= hi)) { lo = 0.0; hi = 0.0; }
    // round outward so the float box still holds every FP64 position
    float flo = __double2float_rd(lo), fhi = __double2float_ru(hi);
    float mid = __fmul_rn(__fadd_rn(flo, fhi), 0.5f);
    float half = __fmul_rn(__fmul_rn(__fsub_rn(fhi, flo), 0.5f), 1.001f);
    bmin[k] = __fsub_rn(mid, half);
    bmax[k] = __fadd_rn(mid, half);
    g.bmin[k] = bmin[k];
    g.bmax[k] = bmax[k];
    g.rc[k] = __fmul_rn(__fadd_rn(bmin[k], bmax[k]), 0.5f);
  }
  float ext = fmaxf(fmaxf(__fsub_rn(bmax[0], bmin[0]), __fsub_rn(bmax[1], bmin[1])),
                    __fsub_rn(bmax[2], bmin[2]));
  g.rhs = __fmul_rn(__fmul_rn(ext, 0.5f), 1.001f);
  double rhs = (double)g.rhs;
#pragma unroll
  for (int k = 0; k < 3; ++k) g.lo[k] = (double)g.rc[k] - rhs;
  g.scale = (rhs > 0.0) ? 512.0 / rhs : 0.0;
}

// The key kernels give each block one contiguous run of keys (a multiple of
// the block size, so every warp's keys are 32 consecutive ones): the keys
// arrive nearly sorted, so a run's high digits take few values, and the
// block adds far fewer non-zero bins to the global histograms than a
// grid-strided block, whose keys span the whole key range, would.
__device__ __forceinline__ long long key_block_span(long long end) {
  const long long per = (end + gridDim.x - 1) / gridDim.x;
  return (per + blockDim.x - 1) / blockDim.x * blockDim.x;
}

// Keys of n positions; hist (optional, 4 x 256 words, cleared) receives the
// digit counts of the four 8-bit passes of the radix sort that follows.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_keys(const T* __restrict__ x, const T* __restrict__ y, const T* __restrict__ z, int n,
       const unsigned long long* __restrict__ enc, TreeGeom* __restrict__ geom_out,
       uint32_t* __restrict__ keys, uint32_t* __restrict__ perm, int* __restrict__ status,
       uint32_t* __restrict__ hist) {
  __shared__ TreeGeom g;
  __shared__ uint32_t s_h[4][kHistBins];
  if (threadIdx.x == 0) {
    compute_geom(enc, g);
    if (blockIdx.x == 0) *geom_out = g;
  }
  if (hist)
    for (int i = threadIdx.x; i < 4 * kHistBins; i += blockDim.x) (&s_h[0][0])[i] = 0;
  __syncthreads();
  const long long end = hist ? (n + 31) / 32 * 32 : n;  // whole warps count digits (hist_add)
  const long long span = key_block_span(end);
  const long long stop = min(end, ((long long)blockIdx.x + 1) * span);
  for (long long i = (long long)blockIdx.x * span + threadIdx.x; i < stop; i += blockDim.x) {
    const bool valid = i < n;
    uint32_t key = 0;
    if (valid) {
      double p[3] = {(double)x[i], (double)y[i], (double)z[i]};
      uint32_t c[3];
      bool finite = true;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        double q = (p[k] - g.lo[k]) * g.scale;
        finite &= (q == q);
        q = fmin(fmax(q, 0.0), 1023.0);
        c[k] = (q == q) ? (uint32_t)q : 0u;
      }
      if (!finite) atomicOr(status, kStatusNonFinite);
      key = morton30(c[0], c[1], c[2]);
      keys[i] = key;
      perm[i] = (uint32_t)i;
    }
    if (hist) hist_add(s_h, key, valid, 4);
  }
  if (hist) {
    __syncthreads();
    hist_flush(s_h, 4, hist);
  }
}

__global__ void k_geoms(const unsigned long long* __restrict__ enc, TreeGeom* __restrict__ geoms,
                        int n_disks) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= n_disks) return;
  TreeGeom g;
  compute_geom(enc + 6 * d, g);
  geoms[d] = g;
}

__global__ void k_bbox_reset_n(unsigned long long* enc, int n_disks) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 6 * n_disks) enc[i] = ((i % 6) < 3) ? ~0ull : 0ull;
}

// Ensemble keys: (disk << 30) | Morton key in the disk's own root cube.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_keys_multi(const T* __restrict__ x, const T* __restrict__ y, const T* __restrict__ z,
             const int* __restrict__ disk, int n, const TreeGeom* __restrict__ geoms,
             uint64_t* __restrict__ keys, uint32_t* __restrict__ perm, int* __restrict__ status,
             uint32_t* __restrict__ hist, int passes) {
  __shared__ uint32_t s_h[kHistMaxPasses][kHistBins];
  if (hist) {
    for (int i = threadIdx.x; i < passes * kHistBins; i += blockDim.x) (&s_h[0][0])[i] = 0;
    __syncthreads();
  }
  const long long end = hist ? (n + 31) / 32 * 32 : n;  // whole warps count digits (hist_add)
  const long long span = key_block_span(end);
  const long long stop = min(end, ((long long)blockIdx.x + 1) * span);
  for (long long i = (long long)blockIdx.x * span + threadIdx.x; i < stop; i += blockDim.x) {
    const bool valid = i < n;
    uint64_t key = 0;
    if (valid) {
      const int d = disk[i];
      const TreeGeom& g = geoms[d];
      double p[3] = {(double)x[i], (double)y[i], (double)z[i]};
      uint32_t c[3];
      bool finite = true;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        double q = (p[k] - g.lo[k]) * g.scale;
        finite &= (q == q);
        q = fmin(fmax(q, 0.0), 1023.0);
        c[k] = (q == q) ? (uint32_t)q : 0u;
      }
      if (!finite) atomicOr(status, kStatusNonFinite);
      key = ((uint64_t)d << 30) | (uint64_t)morton30(c[0], c[1], c[2]);
      keys[i] = key;
      perm[i] = (uint32_t)i;
    }
    if (hist) hist_add(s_h, key, valid, passes);
  }
  if (hist) {
    __syncthreads();
    hist_flush(s_h, passes, hist);
  }
}

__global__ void __launch_bounds__(kThreads)
k_gather_body4(const uint32_t* __restrict__ perm, const float* __restrict__ x,
               const float* __restrict__ y, const float* __restrict__ z,
               const float* __restrict__ m, int n, float4* __restrict__ body4) {
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
       s += (long long)gridDim.x * blockDim.x) {
    uint32_t o = perm[s];
    body4[s] = make_float4(x[o], y[o], z[o], m ? m[o] : 1.f);
  }
}

// ---------------------------------------------------------------- Karras
// delta(i, j): common prefix of keys i and j, with the index as tie-break so
// equal keys still form a valid binary radix tree (Karras 2012, sec. 4).
__device__ __forceinline__ int clz_key(uint32_t v) { return __clz(v); }
__device__ __forceinline__ int clz_key(uint64_t v) { return __clzll((long long)v); }

// ki = keys[i], loaded once by the caller.
template <typename K>
__device__ __forceinline__ int delta(const K* __restrict__ keys, int n, K ki, int i, int j) {
  if (j < 0 || j >= n) return -1;
  const K kj = __ldg(keys + j);
  if (ki != kj) return clz_key(ki ^ kj);
  return 8 * (int)sizeof(K) + __clz((uint32_t)i ^ (uint32_t)j);
}

// key_bits: the low bits of K the keys use (30 Morton bits, plus the disk
// index above them for an ensemble).  prefix[] stores the common prefix in
// those bits, key_bits for runs of equal keys.  Tried and slower at N = 2^20:
// staging the block's keys and a halo in shared memory (35 -> 39 us), and a
// bottom-up agglomerative build (Apetrei 2014; 130 us: the last climbers'
// chains of atomics and fences run the depth of the tree), and range and
// split searches over byte arrays of adjacent-key prefixes and their block
// minima (the tree phase 0.123 -> 0.189 ms: the scans walk ~20 bytes per node
// one dependent load at a time).
// Each internal node also tells both of its children what the octree passes
// need to know about their parent, so that they never chase it: one word of
// the parent's body count (saturated at 2^27 - 1, far above any group span)
// << 5 | its octree level + 1 (0: it spans several disks).  Node 0 has no
// parent and no word.
constexpr uint32_t kNoParent = 0xffffffffu;
__device__ __forceinline__ uint32_t pack_pinfo(int count, int level) {
  return ((uint32_t)min(count, (1 << 27) - 1) << 5) | (uint32_t)(level + 1);
}

// Writes internal node i: range end j, split offset s along direction d, and
// dnode = delta(i, j).
template <typename K>
__device__ __forceinline__ void karras_write(int i, int j, int d, int s, int dnode, int n,
                                             int key_bits, int* __restrict__ left,
                                             int* __restrict__ right, uint32_t* __restrict__ pinfo,
                                             int* __restrict__ lo_out, int* __restrict__ hi_out,
                                             uint8_t* __restrict__ prefix) {
  const int gamma = i + s * d + min(d, 0);
  const int lo = min(i, j), hi = max(i, j);
  const int lc = (lo == gamma) ? (n - 1) + gamma : gamma;
  const int rc = (hi == gamma + 1) ? (n - 1) + gamma + 1 : gamma + 1;
  left[i] = lc;
  right[i] = rc;
  lo_out[i] = lo;
  hi_out[i] = hi;
  constexpr int kW = 8 * (int)sizeof(K);
  const int pre = dnode >= kW ? key_bits : dnode - (kW - key_bits);
  prefix[i] = (uint8_t)pre;
  // octree level as bin_level gives it (the disk index sits above 30 Morton bits)
  const int disk_bits = key_bits > 30 ? key_bits - 30 : 0;
  const uint32_t pi = pack_pinfo(hi - lo + 1, pre < disk_bits ? -1 : (pre - disk_bits) / 3);
  pinfo[lc] = pi;
  pinfo[rc] = pi;
}

// The whole warp narrows [lo, hi) to the last m with delta(i, i + m d) > thr
// (true at lo, false at hi; the predicate only turns false once as m grows,
// Karras 2012 sec. 3): each round every lane tests one of 31 evenly spaced
// points and a ballot keeps the step after the last true one.
template <typename K>
__device__ __forceinline__ long long warp_last_above(const K* __restrict__ keys, int n, K ki,
                                                     int i, int d, int thr, long long lo,
                                                     long long hi, int lane) {
  while (hi - lo > 1) {
    const long long step = (hi - lo + 31) / 32;
    const long long m = lo + (long long)(lane + 1) * step;
    const bool q = m < hi && delta(keys, n, ki, i, i + (int)m * d) > thr;
    const long long nlo = lo + (long long)__popc(__ballot_sync(kFull, q)) * step;
    hi = min(hi, nlo + step);
    lo = nlo;
  }
  return lo;
}

// One thread per internal node (Karras 2012, Fig. 4): direction, range end
// by an exponential then a binary search, split by a binary search.  A warp
// runs each search as many steps as its widest node needs, so a node whose
// range reaches kKarrasCap bodies is handed to the whole warp instead, which
// searches 32 points a step: the lanes' own searches stop at kKarrasCap.
constexpr int kKarrasCap = 1024;

template <typename K>
__global__ void __launch_bounds__(kThreads)
k_karras(const K* __restrict__ keys, int n, int key_bits, int* __restrict__ left,
         int* __restrict__ right, uint32_t* __restrict__ pinfo, int* __restrict__ lo_out,
         int* __restrict__ hi_out, uint8_t* __restrict__ prefix) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool act = i < n - 1;  // every lane stays for the warp's ballots
  K ki = 0;
  int d = 1, dmin = 0;
  bool wide = false;
  if (act) {
    ki = __ldg(keys + i);
    d = (delta(keys, n, ki, i, i + 1) - delta(keys, n, ki, i, i - 1)) > 0 ? 1 : -1;
    dmin = delta(keys, n, ki, i, i - d);
    int lmax = 2;
    while (lmax <= kKarrasCap && delta(keys, n, ki, i, i + lmax * d) > dmin) lmax <<= 1;
    wide = lmax > kKarrasCap;
    if (!wide) {
      int l = 0;
      for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(keys, n, ki, i, i + (l + t) * d) > dmin) l += t;
      const int j = i + l * d;
      const int dnode = delta(keys, n, ki, i, j);
      int s = 0, t = l;
      do {
        t = (t + 1) >> 1;
        if (delta(keys, n, ki, i, i + (s + t) * d) > dnode) s += t;
      } while (t > 1);
      karras_write<K>(i, j, d, s, dnode, n, key_bits, left, right, pinfo, lo_out, hi_out,
                      prefix);
    }
  }
  // wide nodes, one at a time: delta(i, i + kKarrasCap d) > dmin holds, and
  // nothing lies beyond n - 1 steps
  unsigned todo = __ballot_sync(kFull, wide);
  while (todo) {
    const int b = __ffs(todo) - 1;
    todo &= todo - 1;
    const int bi = __shfl_sync(kFull, i, b), bd = __shfl_sync(kFull, d, b);
    const int bmin = __shfl_sync(kFull, dmin, b);
    const K bk = __shfl_sync(kFull, ki, b);
    // the power of two the range end lies below: lane k tests kKarrasCap << k
    const long long mk = (long long)kKarrasCap << lane;
    const bool p = mk < n && delta(keys, n, bk, bi, bi + (int)mk * bd) > bmin;
    const int top = 31 - __clz(__ballot_sync(kFull, p) | 1u);
    const long long lo = (long long)kKarrasCap << top;
    const int l = (int)warp_last_above(keys, n, bk, bi, bd, bmin, lo, min(2 * lo, (long long)n),
                                       lane);
    const int j = bi + l * bd;
    const int dnode = delta(keys, n, bk, bi, j);
    const int s = (int)warp_last_above(keys, n, bk, bi, bd, dnode, 0ll, (long long)l, lane);
    if (lane == b)
      karras_write<K>(bi, j, bd, s, dnode, n, key_bits, left, right, pinfo, lo_out, hi_out,
                      prefix);
  }
}

// ------------------------------------------------------------- moments
// FP64 prefix sums of (m, m x, m y, m z) over the bodies in key order, kept
// tile-local: ploc[k] sums the bodies of k's tile before k, tpre[t] sums the
// tiles before t.  A node's moments over [lo, end) are then
//   (ploc[end] - ploc[lo]) + (tpre[tile(end)] - tpre[tile(lo)]),
// two differences of partial sums no larger than the node's own tiles, so
// cancellation stays at the level of a tile (~1e-13 relative) rather than of
// the whole disk.  Fixed tiling: the sums are the same on every run.
constexpr int kMomThreads = kMomentThreads;
constexpr int kTileM = kMomentTile;  // 1024 threads x 2 bodies

// Large blocks with two bodies per thread keep the registers low and the
// loads and stores nearly contiguous (8 bodies per thread needed 93
// registers and ran 513 blocks of 256 threads at 21% warp occupancy).
__global__ void __launch_bounds__(kMomThreads)
k_moment_tiles(const float4* __restrict__ body4, const double* __restrict__ xd,
               const double* __restrict__ yd, const double* __restrict__ zd, int n,
               double4* __restrict__ ploc, double4* __restrict__ tile_sum) {
  const long long base = (long long)blockIdx.x * kTileM + 2ll * threadIdx.x;
  double4 v[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const long long i = base + k;
    v[k] = make_double4(0, 0, 0, 0);
    if (i < n) {
      const float4 b = body4[i];
      v[k] = body_moment((double)b.w, xd ? xd[i] : (double)b.x, yd ? yd[i] : (double)b.y,
                         zd ? zd[i] : (double)b.z);
    }
  }
  moment_tile_scan(v[0], v[1], base, n, ploc, tile_sum);
}

// Exclusive scan of the tile sums into tpre[0..ntiles] (one block of 1024
// threads, chunks of 1024 tiles, a fixed order of additions).
__global__ void __launch_bounds__(1024) k_tile_scan(const double4* __restrict__ tile_sum,
                                                    int ntiles, double4* __restrict__ tpre) {
  __shared__ double4 s_w[32];
  __shared__ double4 s_carry;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_carry = make_double4(0, 0, 0, 0);
  for (int c0 = 0; c0 < ntiles; c0 += 1024) {
    const int t = c0 + tid;
    const double4 x = (t < ntiles) ? tile_sum[t] : make_double4(0, 0, 0, 0);
    double4 inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const double4 q = d4shfl_up(inc, o);
      if (lane >= o) inc = d4add(inc, q);
    }
    if (lane == 31) s_w[warp] = inc;
    __syncthreads();
    double4 run = s_carry;
    for (int w = 0; w < warp; ++w) run = d4add(run, s_w[w]);
    run = d4add(run, d4sub(inc, x));
    if (t < ntiles) tpre[t] = run;
    if (t == ntiles - 1) tpre[ntiles] = d4add(run, x);
    __syncthreads();
    if (tid == 0) {
      double4 c = s_carry;
      for (int w = 0; w < 32; ++w) c = d4add(c, s_w[w]);
      s_carry = c;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------- octree layout
// Octree level of binary node b: leaves and equal-key runs are level 10;
// nodes whose prefix does not cover the disk bits span several disks (-1).
__device__ __forceinline__ int bin_level(const uint8_t* prefix, int n, int b, int disk_bits) {
  if (b >= n - 1) return 10;
  const int p = (int)prefix[b];
  return (p < disk_bits) ? -1 : (p - disk_bits) / 3;
}

__device__ __forceinline__ int bin_count(const int* lo, const int* hi, int n, int b) {
  return (b >= n - 1) ? 1 : hi[b] - lo[b] + 1;
}

// Visits the octree children of top node b (binary descendants that start a
// deeper octree level, or leaves) in key order.
template <typename F>
__device__ __forceinline__ int for_each_oct_child(const int* __restrict__ left,
                                                  const int* __restrict__ right,
                                                  const uint8_t* __restrict__ prefix, int n,
                                                  int disk_bits, int b, int lb, F f) {
  // Binary nodes of b's own octree level have common prefixes 3 lb .. 3 lb + 2
  // bits (above the disk bits) and every binary child adds at least one, so
  // the octree children lie within three binary levels of b: a depth-first
  // search unrolled to that depth, left first (no stack in local memory).
  auto is_child = [&](int c) { return c >= n - 1 || bin_level(prefix, n, c, disk_bits) > lb; };
  int k = 0;
  const int c1[2] = {left[b], right[b]};
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int a = c1[i];
    if (is_child(a)) {
      f(a, k++);
      continue;
    }
    const int c2[2] = {left[a], right[a]};
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int e = c2[j];
      if (is_child(e)) {
        f(e, k++);
        continue;
      }
      f(left[e], k++);  // three levels down: a deeper octree level
      f(right[e], k++);
    }
  }
  return k;
}

// Per binary node: its octree child count (tops only) and how many target
// groups it holds -- a maximal node with <= gspan bodies is cut into the
// fewest equal runs of <= gmax.  Groups partition the bodies into contiguous
// key ranges inside one node's cell, so a group never straddles a jump of
// the space-filling curve (a fixed run of 32 consecutive bodies can: its box
// then spans most of the domain and its walk degenerates to O(N) work on one
// warp).  gspan = gmax gives the maximal nodes of <= gmax bodies themselves;
// gspan = 2 gmax fills the warps better (a node of 40 bodies is two runs of
// 20, not a binary split such as 5 + 30 + 5) at the price of larger boxes.
// A node is an octree node ("top") when it starts a deeper level than its
// parent; a disk's root is a top whose parent spans several disks (or node 0
// of a single disk).  Groups never span disks.
// lp: the parent's octree level (-1: it spans several disks, or b is node 0,
// which has no parent); pc: the parent's body count (INT_MAX when lp < 0).
__device__ __forceinline__ void classify(int n, int disk_bits, const uint32_t* __restrict__ pinfo,
                                         const uint8_t* __restrict__ prefix, int b, int& lb,
                                         int& lp, bool& top, int& pc) {
  lb = bin_level(prefix, n, b, disk_bits);
  const uint32_t pi = (b == 0) ? kNoParent : pinfo[b];
  lp = (pi == kNoParent) ? -1 : (int)(pi & 31u) - 1;
  top = lb >= 0 && lb > lp;
  pc = (lp < 0) ? 0x7fffffff : (int)(pi >> 5);
}

// ------------------------------------------------- octree slots + groups
// Three passes over the binary nodes, none of which waits on another block:
//   k_mark   counts each octree node's children (tops with more than `prune`
//            bodies) and each group node's runs, and reduces both counts per
//            tile;
//   k_tiles  scans the tile sums (one block);
//   k_apply  scans the counts within each tile, adds the tile prefix, stores
//            each node's first child slot and writes the group runs.
// k_apply also lists which binary node each slot holds: an octree node's
// children at n_roots + off[node] + index (index: the children in key order)
// and each disk's root at the disk index.  k_emit then writes one record per
// slot, one thread each.  No per-child parent or sibling-index array is
// needed (2 N words the slot passes wrote and the record pass read back).
// The two counts travel packed in one 64-bit word: children << 31 | runs.
constexpr int kMarkTile = kThreads;
constexpr uint8_t kNchTop = 0x80;   // nch[b]: b is an octree node
constexpr uint8_t kNchRoot = 0x40;  // nch[b]: b is a disk's root
constexpr uint8_t kNchCount = 0x0f; // nch[b]: its child records (<= 8)

__device__ __forceinline__ unsigned long long pack_counts(uint32_t children, uint32_t runs) {
  return ((unsigned long long)children << 31) | runs;
}

template <typename K>
struct MarkArgs {
  int n, gmax, gspan, prune, disk_bits;
  const int *left, *right;
  const uint32_t* pinfo;
  const int *lo, *hi;
  const uint8_t* prefix;
  uint8_t* nch;                // child count | kNchTop | kNchRoot
  uint32_t* off;               // k_mark: children | runs << 4; k_apply: first child slot - n_roots
  unsigned long long* tile_sum;
};

__device__ __forceinline__ unsigned long long block_sum_u64(unsigned long long v,
                                                            unsigned long long* s_w) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  if (lane == 0) s_w[warp] = v;
  __syncthreads();
  unsigned long long t = 0;
#pragma unroll
  for (int w = 0; w < kThreads / 32; ++w) t += s_w[w];
  return t;
}

template <typename K>
__global__ void __launch_bounds__(kThreads) k_mark(const MarkArgs<K> a) {
  __shared__ unsigned long long s_w[kThreads / 32];
  const int n = a.n, nb = 2 * n - 1;
  const int b = blockIdx.x * kMarkTile + threadIdx.x;
  uint32_t nchild = 0, runs = 0;
  if (b < nb) {
    int lb, lp, pc;
    bool top;
    classify(n, a.disk_bits, a.pinfo, a.prefix, b, lb, lp, top, pc);
    const int c = bin_count(a.lo, a.hi, n, b);
    if (top && b < n - 1 && lb < 10 && c > a.prune)
      nchild = (uint32_t)for_each_oct_child(a.left, a.right, a.prefix, n, a.disk_bits, b, lb,
                                            [](int, int) {});
    if (lb >= 0 && c <= a.gspan && pc > a.gspan) runs = (uint32_t)((c + a.gmax - 1) / a.gmax);
    const bool root = top && lp < 0;
    a.nch[b] = (uint8_t)nchild | (top ? kNchTop : 0) | (root ? kNchRoot : 0);
    a.off[b] = nchild | (runs << 4);
  }
  const unsigned long long t = block_sum_u64(pack_counts(nchild, runs), s_w);
  if (threadIdx.x == 0) a.tile_sum[blockIdx.x] = t;
}

__device__ __forceinline__ unsigned long long warp_incl_scan_u64(unsigned long long v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long q = __shfl_up_sync(kFull, v, o);
    if (lane >= o) v += q;
  }
  return v;
}

// Exclusive scan of the tile sums in place (one block; integer sums).  Warp
// w scans 256 consecutive sums of a chunk as 8 rows of 32 with coalesced
// loads and stores (a thread's own run of 8 consecutive sums made every load
// touch 16 lines, and the L1 wavefronts took 8 us at 8192 sums).
__global__ void __launch_bounds__(1024) k_tiles(unsigned long long* __restrict__ v, int m) {
  constexpr int kRows = 8, kChunk = 1024 * kRows;
  __shared__ unsigned long long s_w[32];
  __shared__ unsigned long long s_carry;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_carry = 0;
  __syncthreads();
  for (int c0 = 0; c0 < m; c0 += kChunk) {
    const int base = c0 + warp * (32 * kRows) + lane;
    unsigned long long x[kRows], ex[kRows], run = 0;
#pragma unroll
    for (int k = 0; k < kRows; ++k) x[k] = (base + 32 * k < m) ? v[base + 32 * k] : 0ull;
#pragma unroll
    for (int k = 0; k < kRows; ++k) {
      const unsigned long long inc = warp_incl_scan_u64(x[k], lane);
      ex[k] = run + inc - x[k];
      run += __shfl_sync(kFull, inc, 31);
    }
    if (lane == 0) s_w[warp] = run;  // the warp's total
    __syncthreads();
    // exclusive prefix of the warps' totals, by every warp for itself
    const unsigned long long t = s_w[lane];
    const unsigned long long ti = warp_incl_scan_u64(t, lane);
    const unsigned long long wpre = s_carry + __shfl_sync(kFull, ti - t, warp);
    const unsigned long long total = __shfl_sync(kFull, ti, 31);
#pragma unroll
    for (int k = 0; k < kRows; ++k)
      if (base + 32 * k < m) v[base + 32 * k] = wpre + ex[k];
    __syncthreads();
    if (tid == 0) s_carry += total;
    __syncthreads();
  }
}

// Disk index of a key (the bits above the 30 Morton bits).
template <typename K>
__device__ __forceinline__ int key_disk(K k) { return (int)(k >> 30); }

template <typename K>
struct ApplyArgs {
  int n, n_roots, disk_bits;
  const int *left, *right, *lo, *hi;
  const uint8_t* prefix;
  const uint8_t* nch;
  const K* keys;
  uint32_t* off;
  int* node_of;  // octree slot -> binary node of its record
  const unsigned long long* tile_pre;
  int2* groups;
  int* group_disk;  // optional: disk of each group
  int* n_nodes;
  int* n_groups;
  int2* group_span;  // optional: (first group of the span node, its bodies)
};

template <typename K>
__global__ void __launch_bounds__(kThreads) k_apply(const ApplyArgs<K> a) {
  __shared__ unsigned long long s_w[kThreads / 32];
  const int n = a.n, nb = 2 * n - 1;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int b = blockIdx.x * kMarkTile + tid;
  const uint32_t v = (b < nb) ? a.off[b] : 0u;
  const uint32_t nchild = v & 15u, runs = v >> 4;
  const unsigned long long mine = pack_counts(nchild, runs);
  unsigned long long inc = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long q = __shfl_up_sync(kFull, inc, o);
    if (lane >= o) inc += q;
  }
  if (lane == 31) s_w[warp] = inc;
  __syncthreads();
  unsigned long long ex = a.tile_pre[blockIdx.x] + inc - mine;
  for (int w = 0; w < warp; ++w) ex += s_w[w];
  if (b >= nb) return;
  const uint32_t first = (uint32_t)(ex >> 31);
  const uint32_t goff = (uint32_t)(ex & 0x7fffffffull);
  a.off[b] = first;
  if (nchild > 0) {  // which binary node each child slot holds, in key order
    const int base = a.n_roots + (int)first;
    for_each_oct_child(a.left, a.right, a.prefix, n, a.disk_bits, b,
                       bin_level(a.prefix, n, b, a.disk_bits),
                       [&](int ch, int i) { a.node_of[base + i] = ch; });
  }
  if (a.nch[b] & kNchRoot) {  // a disk's root: slot = the disk index
    const int lo = (b >= n - 1) ? b - (n - 1) : a.lo[b];
    a.node_of[sizeof(K) == 4 ? 0 : key_disk(a.keys[lo])] = b;
  }
  if (runs > 0) {  // runs of c / runs or c / runs + 1 consecutive bodies
    const int lo = (b >= n - 1) ? b - (n - 1) : a.lo[b];
    const int c = (b >= n - 1) ? 1 : a.hi[b] - lo + 1;
    const int ng = (int)runs, q = c / ng, r = c % ng;
    const int disk = a.group_disk ? key_disk(a.keys[lo]) : 0;
    for (int j = 0, s = lo; j < ng; ++j) {
      const int sz = q + (j < r ? 1 : 0);
      a.groups[goff + j] = make_int2(s, sz);
      if (a.group_disk) a.group_disk[goff + j] = disk;
      if (a.group_span) a.group_span[goff + j] = make_int2((int)goff, c);
      s += sz;
    }
  }
  if (b == nb - 1) {
    *a.n_nodes = a.n_roots + (int)(first + nchild);
    *a.n_groups = (int)(goff + runs);
  }
}

__device__ __forceinline__ uint32_t compact3(uint32_t v) {
  v &= 0x09249249u;
  v = (v ^ (v >> 2)) & 0x030c30c3u;
  v = (v ^ (v >> 4)) & 0x0300f00fu;
  v = (v ^ (v >> 8)) & 0x030000ffu;
  v = (v ^ (v >> 16)) & 0x000003ffu;
  return v;
}

template <typename K>
struct EmitArgs {
  int n, disk_bits, n_roots;
  const int *lo, *hi;
  const uint8_t* prefix;
  const K* keys;
  const uint8_t* nch;
  const uint32_t* off;
  const float4* body4;
  const double4* ploc;
  const double4* tpre;
  const TreeGeom* geom;
  OctNodes oct;
  bool boxes;  // also the records' boxes (the neighbour search reads them)
};

// Writes the octree record of binary node c into slot f.
template <typename K>
__device__ void write_node(const EmitArgs<K>& a, int c, int f) {
  const int first = (c >= a.n - 1) ? c - (a.n - 1) : a.lo[c];
  // 30-bit keys carry no disk: the geometry needs no key load then
  const TreeGeom* geom = a.geom + (sizeof(K) == 4 ? 0 : key_disk(a.keys[first]));
  const float rhs = geom->rhs;
  if (c >= a.n - 1) {  // single-body leaf
    const int j = c - (a.n - 1);
    const float4 p = a.body4[j];
    a.oct.com[f] = p;
    a.oct.info[f] = make_int4(-1, j, (1 << 4), __float_as_int(ldexpf(rhs, -10)));
    if (a.boxes) {
      a.oct.box_lo[f] = make_float4(p.x, p.y, p.z, 0.f);
      a.oct.box_hi[f] = make_float4(p.x, p.y, p.z, 0.f);
    }
    return;
  }
  const int L = ((int)a.prefix[c] - a.disk_bits) / 3;
  const int lo = a.lo[c], hi = a.hi[c];
  // loaded before the record's stores (the arrays carry no restrict)
  const int k = a.nch[c] & kNchCount;
  const int first_child = k > 0 ? a.n_roots + (int)a.off[c] : -1;
  const double4 s = range_moments(a.ploc, a.tpre, lo, hi + 1);
  // the node's cube: level L cell of its key prefix (side 2 rhs / 2^L, exact
  // power-of-two scaling), grown by a margin for float positions that sit an
  // ulp outside their FP64-quantised cell
  const uint32_t kl = (uint32_t)(a.keys[lo] & (K)0x3fffffffu) >> (3 * (10 - L));
  const uint32_t cc[3] = {compact3(kl), compact3(kl >> 1), compact3(kl >> 2)};
  const double side = (double)rhs * (double)(2.0f / (float)(1u << L));
  float blo[3], bhi[3], ctr[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double l0 = geom->lo[k] + (double)cc[k] * side;
    const float fl = (float)l0, fs = (float)side;
    const float margin = 1e-6f * (fabsf(fl) + fs) + 1e-30f;
    blo[k] = fl - margin;
    bhi[k] = fl + fs + margin;
    ctr[k] = fl + 0.5f * fs;
  }
  const float4 com = com_of(s, ctr[0], ctr[1], ctr[2]);
  a.oct.com[f] = com;
  a.oct.info[f] = make_int4(first_child, lo, ((hi - lo + 1) << 4) | k,
                            __float_as_int(ldexpf(rhs, -L)));
  if (a.boxes) {
    a.oct.box_lo[f] = make_float4(blo[0], blo[1], blo[2], 0.f);
    a.oct.box_hi[f] = make_float4(bhi[0], bhi[1], bhi[2], 0.f);
  }
}

// One thread per record: slot f holds binary node node_of[f] (written by
// k_apply); consecutive slots are siblings, so the record stores coalesce.
// The record count is read on the device (a grid-stride loop over it).
template <typename K>
__global__ void __launch_bounds__(kThreads) k_emit(const EmitArgs<K> a,
                                                   const int* __restrict__ node_of,
                                                   const int* __restrict__ n_nodes) {
  const int total = *n_nodes;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < total; f += gridDim.x * blockDim.x)
    write_node(a, node_of[f], f);
}

// N == 1: the root is the single body and the only group.
__global__ void k_single(const float4* __restrict__ body4, const TreeGeom* __restrict__ geom,
                         OctNodes oct, int* __restrict__ n_nodes, int2* __restrict__ groups,
                         int* __restrict__ n_groups) {
  float4 p = body4[0];
  oct.com[0] = p;
  oct.info[0] = make_int4(-1, 0, (1 << 4), __float_as_int(geom->rhs));
  oct.box_lo[0] = make_float4(p.x, p.y, p.z, 0.f);
  oct.box_hi[0] = make_float4(p.x, p.y, p.z, 0.f);
  *n_nodes = 1;
  groups[0] = make_int2(0, 1);
  *n_groups = 1;
}

template <typename T>
T* dalloc(size_t count, const char* what) {
  T* p = nullptr;
  check(cudaMalloc(&p, sizeof(T) * (count ? count : 1)), what);
  return p;
}

int grid_for(long long n) { return (int)((n + kThreads - 1) / kThreads); }

}  // namespace

void tree_alloc(TreeWork& w, int cap) {
  tree_free(w);
  if (cap < 1) cap = 1;
  w.cap = cap;
  const size_t n = (size_t)cap, nb = 2 * n;
  w.keys = dalloc<uint32_t>(n, "keys");
  w.perm = dalloc<uint32_t>(n, "perm");
  w.keys_alt = dalloc<uint32_t>(n, "keys_alt");
  w.perm_alt = dalloc<uint32_t>(n, "perm_alt");
  w.counts = dalloc<uint32_t>(radix_sort_count_words(cap), "sort counts");
  w.body4 = dalloc<float4>(n, "body4");
  w.bin_left = dalloc<int>(n, "bin_left");
  w.bin_right = dalloc<int>(n, "bin_right");
  w.bin_pinfo = dalloc<uint32_t>(nb, "bin_pinfo");
  w.bin_lo = dalloc<int>(n, "bin_lo");
  w.bin_hi = dalloc<int>(n, "bin_hi");
  w.bin_prefix = dalloc<uint8_t>(n, "bin_prefix");
  w.mom_ploc = dalloc<double4>(n + 1, "moment prefix");
  w.mom_tiles = dalloc<double4>(2 * ((n + 1) / kTileM + 2), "moment tiles");
  w.oct_nch = dalloc<uint8_t>(nb, "oct_nch");
  w.oct_off = dalloc<uint32_t>(nb, "oct_off");
  w.oct_node = dalloc<int>(nb, "oct_node");
  w.scan_tmp = dalloc<uint32_t>(octree_scan_words((int)nb), "octree tile sums");
  w.oct.com = dalloc<float4>(nb, "oct com");
  w.oct.info = dalloc<int4>(nb, "oct info");
  w.oct.box_lo = dalloc<float4>(nb, "oct box_lo");
  w.oct.box_hi = dalloc<float4>(nb, "oct box_hi");
  w.bbox_enc = dalloc<unsigned long long>(6, "bbox");
  w.geom = dalloc<TreeGeom>(1, "geom");
  w.n_nodes = dalloc<int>(1, "n_nodes");
  w.groups = dalloc<int2>(n, "groups");
  w.n_groups = dalloc<int>(1, "n_groups");
  w.status = dalloc<int>(1, "status");
  check(cudaMemset(w.status, 0, sizeof(int)), "status init");
  check(cudaMemset(w.n_nodes, 0, sizeof(int)), "n_nodes init");
}

void tree_free(TreeWork& w) {
  void* ptrs[] = {w.keys, w.perm, w.keys_alt, w.perm_alt, w.counts, w.body4, w.bin_left,
                  w.bin_right, w.bin_pinfo, w.bin_lo, w.bin_hi, w.bin_prefix, w.mom_ploc,
                  w.mom_tiles, w.oct_nch, w.oct_off, w.oct_node, w.scan_tmp, w.oct.com, w.oct.info, w.oct.box_lo, w.oct.box_hi, w.bbox_enc,
                  w.geom, w.n_nodes, w.status, w.groups, w.n_groups};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (w.side) cudaStreamDestroy(w.side);
  if (w.ev_fork) cudaEventDestroy(w.ev_fork);
  if (w.ev_join) cudaEventDestroy(w.ev_join);
  w = TreeWork();
}

void tree_enable_overlap(TreeWork& w) {
  if (w.side) return;
  check(cudaStreamCreateWithFlags(&w.side, cudaStreamNonBlocking), "tree side stream");
  check(cudaEventCreateWithFlags(&w.ev_fork, cudaEventDisableTiming), "tree fork event");
  check(cudaEventCreateWithFlags(&w.ev_join, cudaEventDisableTiming), "tree join event");
}

void launch_bbox_reset(TreeWork& w, cudaStream_t s) {
  k_bbox_reset<<<1, 32, 0, s>>>(w.bbox_enc);
}

template <typename T>
void launch_bbox(TreeWork& w, const T* x, const T* y, const T* z, int n, cudaStream_t s) {
  launch_bbox_reset(w, s);
  int g = std::min(grid_for(n), 148 * 8);
  if (g < 1) g = 1;
  k_bbox<T><<<g, kThreads, 0, s>>>(x, y, z, n, w.bbox_enc);
  check(cudaGetLastError(), "k_bbox launch");
}

template <typename T>
void launch_keys(TreeWork& w, const T* x, const T* y, const T* z, int n, cudaStream_t s,
                 uint32_t* hist) {
  // with histograms: fewer blocks, so fewer block histograms to add up
  int g = hist ? std::min(div_up(n, kThreads * 8), 148 * 4) : std::min(grid_for(n), 148 * 16);
  if (g < 1) g = 1;
  k_keys<T><<<g, kThreads, 0, s>>>(x, y, z, n, w.bbox_enc, w.geom, w.keys, w.perm, w.status,
                                   hist);
  check(cudaGetLastError(), "k_keys launch");
}

template void launch_bbox<float>(TreeWork&, const float*, const float*, const float*, int,
                                 cudaStream_t);
template void launch_bbox<double>(TreeWork&, const double*, const double*, const double*, int,
                                  cudaStream_t);
template void launch_keys<float>(TreeWork&, const float*, const float*, const float*, int,
                                 cudaStream_t, uint32_t*);
template void launch_keys<double>(TreeWork&, const double*, const double*, const double*, int,
                                  cudaStream_t, uint32_t*);
template void launch_bbox<HiLo>(TreeWork&, const HiLo*, const HiLo*, const HiLo*, int,
                                cudaStream_t);
template void launch_keys<HiLo>(TreeWork&, const HiLo*, const HiLo*, const HiLo*, int,
                                cudaStream_t, uint32_t*);

void launch_gather_body4(TreeWork& w, const float* x, const float* y, const float* z,
                         const float* m, int n, cudaStream_t s) {
  int g = std::min(grid_for(n), 148 * 16);
  if (g < 1) g = 1;
  k_gather_body4<<<g, kThreads, 0, s>>>(w.perm, x, y, z, m, n, w.body4);
  check(cudaGetLastError(), "k_gather_body4 launch");
}

void launch_geoms(const unsigned long long* enc, TreeGeom* geoms, int n_disks, cudaStream_t s) {
  k_geoms<<<div_up(n_disks, 64), 64, 0, s>>>(enc, geoms, n_disks);
  check(cudaGetLastError(), "k_geoms launch");
}

void launch_bbox_reset_n(unsigned long long* enc, int n_disks, cudaStream_t s) {
  k_bbox_reset_n<<<div_up(6 * n_disks, 256), 256, 0, s>>>(enc, n_disks);
  check(cudaGetLastError(), "k_bbox_reset_n launch");
}

template <typename T>
void launch_keys_multi(const T* x, const T* y, const T* z, const int* disk, int n,
                       const TreeGeom* geoms, uint64_t* keys, uint32_t* perm, int* status,
                       cudaStream_t s, uint32_t* hist, int key_bits) {
  int g = hist ? std::min(div_up(n, kThreads * 8), 148 * 4) : std::min(grid_for(n), 148 * 16);
  if (g < 1) g = 1;
  k_keys_multi<T><<<g, kThreads, 0, s>>>(x, y, z, disk, n, geoms, keys, perm, status, hist,
                                         (key_bits + 7) / 8);
  check(cudaGetLastError(), "k_keys_multi launch");
}

template void launch_keys_multi<float>(const float*, const float*, const float*, const int*, int,
                                       const TreeGeom*, uint64_t*, uint32_t*, int*, cudaStream_t,
                                       uint32_t*, int);
template void launch_keys_multi<double>(const double*, const double*, const double*, const int*,
                                        int, const TreeGeom*, uint64_t*, uint32_t*, int*,
                                        cudaStream_t, uint32_t*, int);
template void launch_keys_multi<HiLo>(const HiLo*, const HiLo*, const HiLo*, const int*, int,
                                      const TreeGeom*, uint64_t*, uint32_t*, int*, cudaStream_t,
                                      uint32_t*, int);

template <typename K>
void launch_karras(TreeWork& w, const K* keys, int n, int key_bits, cudaStream_t s) {
  if (n < 2) return;
  k_karras<K><<<grid_for(n - 1), kThreads, 0, s>>>(keys, n, key_bits, w.bin_left, w.bin_right,
                                                   w.bin_pinfo, w.bin_lo, w.bin_hi,
                                                   w.bin_prefix);
  check(cudaGetLastError(), "k_karras launch");
}

template <typename K>
void launch_octree(TreeWork& w, const K* keys, int n, int disk_bits, int n_roots,
                   const TreeGeom* geoms, int* group_disk, const double* xd, const double* yd,
                   const double* zd, cudaStream_t s, bool moments_ready) {
  if (n < 1) return;
  if (n == 1) {
    k_single<<<1, 1, 0, s>>>(w.body4, geoms, w.oct, w.n_nodes, w.groups, w.n_groups);
    if (group_disk) check(cudaMemsetAsync(group_disk, 0, sizeof(int), s), "group disk");
    check(cudaGetLastError(), "k_single launch");
    return;
  }
  const int nb = 2 * n - 1;
  const int gmax = w.group_max;
  const int gspan = gmax * std::max(1, w.group_span);
  const int ntiles = n / kTileM + 1;
  double4* tile_sum = w.mom_tiles;
  double4* tpre = w.mom_tiles + (ntiles + 1);
  if (!moments_ready) {
    k_moment_tiles<<<ntiles, kMomThreads, 0, s>>>(w.body4, xd, yd, zd, n, w.mom_ploc, tile_sum);
    k_tile_scan<<<1, 1024, 0, s>>>(tile_sum, ntiles, tpre);
  }
  unsigned long long* tsum = (unsigned long long*)w.scan_tmp;
  const int mtiles = div_up(nb, kMarkTile);
  MarkArgs<K> m{n, gmax, gspan, w.prune_max, disk_bits, w.bin_left, w.bin_right, w.bin_pinfo,
                w.bin_lo, w.bin_hi, w.bin_prefix, w.oct_nch, w.oct_off, tsum};
  k_mark<K><<<mtiles, kMarkTile, 0, s>>>(m);
  k_tiles<<<1, 1024, 0, s>>>(tsum, mtiles);
  ApplyArgs<K> ap{n,         n_roots,  disk_bits, w.bin_left, w.bin_right, w.bin_lo,
                  w.bin_hi,  w.bin_prefix, w.oct_nch, keys,   w.oct_off,   w.oct_node,
                  tsum,      w.groups, group_disk, w.n_nodes, w.n_groups,  w.group_spans};
  k_apply<K><<<mtiles, kMarkTile, 0, s>>>(ap);
  EmitArgs<K> a{n, disk_bits, n_roots, w.bin_lo, w.bin_hi, w.bin_prefix, keys, w.oct_nch,
                w.oct_off, w.body4, w.mom_ploc, tpre, geoms, w.oct, w.boxes};
  if (moments_ready && w.moments_on_side) check(cudaStreamWaitEvent(s, w.ev_join, 0), "moment join");
  // one thread per record for up to n / 2 records (about 0.35 n with leaves of
  // eight bodies); the loop covers any more
  k_emit<K><<<std::max(1, div_up(n, 2 * kThreads)), kThreads, 0, s>>>(
      a, w.oct_node, w.n_nodes);
  check(cudaGetLastError(), "octree launch");
}

template <typename K>
void launch_tree(TreeWork& w, const K* keys, int n, int key_bits, int disk_bits, int n_roots,
                 const TreeGeom* geoms, int* group_disk, const double* xd, const double* yd,
                 const double* zd, cudaStream_t s, bool tiles_done) {
  if (tiles_done && n >= 1) {  // the caller's permute wrote the tile-local prefix and tile sums
    w.moments_on_side = false;
    const int ntiles = moment_tiles(n);
    k_tile_scan<<<1, 1024, 0, s>>>(w.mom_tiles, ntiles, moment_tile_prefix(w, n));
    launch_karras<K>(w, keys, n, key_bits, s);
    launch_octree<K>(w, keys, n, disk_bits, n_roots, geoms, group_disk, xd, yd, zd, s, true);
    return;
  }
  const bool fork = w.side && n >= 2;
  w.moments_on_side = fork;
  if (fork) {
    check(cudaEventRecord(w.ev_fork, s), "tree fork");
    check(cudaStreamWaitEvent(w.side, w.ev_fork, 0), "tree fork");
    launch_moment_prefix(w, n, xd, yd, zd, w.side);
    check(cudaEventRecord(w.ev_join, w.side), "tree join");
  }
  launch_karras<K>(w, keys, n, key_bits, s);
  launch_octree<K>(w, keys, n, disk_bits, n_roots, geoms, group_disk, xd, yd, zd, s, fork);
}

template void launch_karras<uint64_t>(TreeWork&, const uint64_t*, int, int, cudaStream_t);

void radix_tree_u32(const uint32_t* keys, int n, int key_bits, int* left, int* right, int* lo,
                    int* hi, uint8_t* prefix) {
  TreeWork w;
  tree_alloc(w, n);
  try {
    launch_karras<uint32_t>(w, keys, n, key_bits, 0);
    const size_t m = (size_t)std::max(n - 1, 0);
    check(cudaMemcpy(left, w.bin_left, sizeof(int) * m, cudaMemcpyDeviceToDevice), "tree out");
    check(cudaMemcpy(right, w.bin_right, sizeof(int) * m, cudaMemcpyDeviceToDevice), "tree out");
    check(cudaMemcpy(lo, w.bin_lo, sizeof(int) * m, cudaMemcpyDeviceToDevice), "tree out");
    check(cudaMemcpy(hi, w.bin_hi, sizeof(int) * m, cudaMemcpyDeviceToDevice), "tree out");
    check(cudaMemcpy(prefix, w.bin_prefix, m, cudaMemcpyDeviceToDevice), "tree out");
    check(cudaDeviceSynchronize(), "radix tree");
  } catch (...) {
    tree_free(w);
    throw;
  }
  tree_free(w);
}
template void launch_octree<uint64_t>(TreeWork&, const uint64_t*, int, int, int,
                                      const TreeGeom*, int*, const double*, const double*,
                                      const double*, cudaStream_t, bool);
template void launch_tree<uint32_t>(TreeWork&, const uint32_t*, int, int, int, int,
                                    const TreeGeom*, int*, const double*, const double*,
                                    const double*, cudaStream_t, bool);
template void launch_tree<uint64_t>(TreeWork&, const uint64_t*, int, int, int, int,
                                    const TreeGeom*, int*, const double*, const double*,
                                    const double*, cudaStream_t, bool);

void launch_moment_prefix(TreeWork& w, int n, const double* xd, const double* yd,
                          const double* zd, cudaStream_t s) {
  if (n < 1) return;
  const int ntiles = n / kTileM + 1;
  k_moment_tiles<<<ntiles, kMomThreads, 0, s>>>(w.body4, xd, yd, zd, n, w.mom_ploc, w.mom_tiles);
  k_tile_scan<<<1, 1024, 0, s>>>(w.mom_tiles, ntiles, moment_tile_prefix(w, n));
  check(cudaGetLastError(), "moment prefix launch");
}

size_t octree_scan_words(int nb) { return 2 * (size_t)div_up(nb, kMarkTile); }

double4* moment_tile_prefix(TreeWork& w, int n) { return w.mom_tiles + (n / kTileM + 2); }

void launch_build_topology(TreeWork& w, int n, cudaStream_t s) {
  launch_karras<uint32_t>(w, w.keys, n, 30, s);
}

void launch_build_moments(TreeWork& w, int n, const double* xd, const double* yd,
                          const double* zd, cudaStream_t s) {
  launch_octree<uint32_t>(w, w.keys, n, 0, 1, w.geom, nullptr, xd, yd, zd, s);
}

}  // namespace nb
