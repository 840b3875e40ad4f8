// sort.cu -- stable LSD radix sort of (uint32 / uint64 key, uint32 value)
// pairs, one-sweep form.
//
// Replaces the reference's serial DFS ordering (bhtree_sortKernel,
// BHTree.cu:322-352, a <<<1,1>>> launch) by a Morton-order sort: the body
// order of the octree IS the sorted key order.  Digits are 8 bits.
//   * the digits of every pass are counted in a single read of the keys (a
//     digit's count does not depend on the key order), by a histogram kernel
//     or by the kernel that wrote the keys; every tile of a pass scans its
//     pass's 256 counts into the global digit offsets;
//   * one kernel per pass: a block takes the next tile (atomic ticket, so
//     tiles start in order), ranks its keys with __match_any_sync, publishes
//     its per-digit counts, and finds the counts of all earlier tiles by
//     decoupled look-back over their published words (aggregate or inclusive
//     prefix, a 2-bit flag over a 30-bit count); then it stages the tile in
//     shared memory by digit and writes runs of consecutive addresses.
// HBM traffic per pass: 8 B read + 8 B write per pair (+ 4 B once for the
// histograms).  Every look-back wait is bounded: a wait that gives up raises
// kStatusSortWait instead of hanging (the result is then unusable).
#include <algorithm>

#include "common.cuh"
#include "digit_hist.cuh"
#include "kernels.cuh"

namespace nb {
namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / kWarp;
// keys per thread: at most 16 (uint32 keys, 4096-key tiles) or 8 (uint64,
// 2048) so the staged tile stays within 48 KB of static shared memory; fewer
// (down to 2) when there would be fewer tiles than half the SMs.  Measured
// step times (CUDA graphs): N = 2^20 is fastest with 16 (0.745 ms; 8: 0.748,
// 4: 0.761, 2: 0.797), N = 131072 with 8 or 4 (0.221 ms; 16: 0.225).
template <typename K>
constexpr int sort_items() { return sizeof(K) == 8 ? 8 : 16; }
constexpr int kMinItems = 2;
constexpr int kMinTile = kSortThreads * kMinItems;
constexpr int kBins = kHistBins;

// Exclusive scan of `total` uint32 in place, one block of 1024 threads.
__global__ void __launch_bounds__(1024) k_scan_inplace(uint32_t* __restrict__ data, int total) {
  __shared__ uint32_t s_warp[32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int per = (total + 1023) / 1024;
  const long long lo = (long long)tid * per;
  const long long hi = min((long long)total, lo + per);
  uint32_t sum = 0;
  for (long long i = lo; i < hi; ++i) sum += data[i];
  // block exclusive scan of per-thread sums
  uint32_t v = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(kFull, v, o);
    if (lane >= o) v += t;
  }
  if (lane == 31) s_warp[warp] = v;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = s_warp[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(kFull, w, o);
      if (lane >= o) w += t;
    }
    s_warp[lane] = w;
  }
  __syncthreads();
  uint32_t run = v - sum + (warp > 0 ? s_warp[warp - 1] : 0u);
  for (long long i = lo; i < hi; ++i) {
    uint32_t c = data[i];
    data[i] = run;
    run += c;
  }
}

// ------------------------------------------------------------- one sweep
constexpr uint32_t kFlagA = 1u << 30;  // tile aggregate published
constexpr uint32_t kFlagP = 2u << 30;  // inclusive prefix published
constexpr uint32_t kValMask = (1u << 30) - 1u;
constexpr uint32_t kFlagMask = ~kValMask;
constexpr int kSpinLimit = 1 << 20;
constexpr int kLookAhead = 8;  // look-back words read per round
constexpr int kMaxPasses = kHistMaxPasses;

// Digit counts of every pass in one read: hist[p * 256 + d] (zeroed first).
template <typename K>
__global__ void __launch_bounds__(kSortThreads)
k_digit_hist(const K* __restrict__ keys, int n, int passes, uint32_t* __restrict__ hist) {
  __shared__ uint32_t s_h[kMaxPasses][kBins];
  const int tid = threadIdx.x;
  for (int i = tid; i < kMaxPasses * kBins; i += kSortThreads) (&s_h[0][0])[i] = 0;
  __syncthreads();
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long end = (n + 31) / 32 * 32;  // whole warps count digits (hist_add)
  for (long long i = (long long)blockIdx.x * blockDim.x + tid; i < end; i += stride) {
    const bool valid = i < n;
    hist_add(s_h, valid ? __ldg(keys + i) : (K)0, valid, passes);
  }
  __syncthreads();
  hist_flush(s_h, passes, hist);
}


// Decoupled look-back of tile t > 0 for digit d: the sum of the counts of
// tiles 0 .. t-1.  kLookAhead predecessors are loaded per round (tiles below
// 0 read as an inclusive prefix of 0), so a walk back over aggregates takes
// that many times fewer dependent L2 round trips; it stops at the first
// inclusive prefix.  A round whose nearest predecessor has published nothing
// waits; after kSpinLimit such rounds (about a second) the wait gives up,
// raises kStatusSortWait and returns the partial sum.  That sum is no larger
// than the true one, so the caller's scatter stays inside the output.
__device__ __forceinline__ uint32_t lookback_prefix(const uint32_t* status, int t, int d,
                                                    int* err) {
  uint32_t excl = 0;
  int j = t - 1, spins = 0;
  while (j >= 0) {
    uint32_t w[kLookAhead];
#pragma unroll
    for (int q = 0; q < kLookAhead; ++q)
      w[q] = (j - q >= 0) ? __ldcv(status + (size_t)(j - q) * kBins + d) : kFlagP;
    int used = 0;
    bool done = false;
#pragma unroll
    for (int q = 0; q < kLookAhead; ++q) {
      if (done || used < q) break;  // stop at the first unpublished word
      const uint32_t f = w[q] & kFlagMask;
      if (f == 0u) break;
      excl += w[q] & kValMask;
      used = q + 1;
      if (f == kFlagP) done = true;
    }
    if (done) break;
    if (used == 0) {
      if (++spins > kSpinLimit) {
        atomicOr(err, kStatusSortWait);
        break;
      }
      continue;
    }
    j -= used;
  }
  return excl;
}

// Self-test of the look-back's bound: the wait of tile t over status words
// that no tile publishes (the caller passes them zeroed) must give up and
// raise kStatusSortWait in *err.  One block of kBins threads, one per digit.
__global__ void __launch_bounds__(kBins)
k_lookback_probe(const uint32_t* status, int t, int* err, uint32_t* out) {
  out[threadIdx.x] = lookback_prefix(status, t, threadIdx.x, err);
}

// Shared memory of one tile of a one-sweep pass.
template <typename K, int kItems>
struct SweepSmem {
  uint32_t cnt[kSortWarps][kBins];
  K keys[kSortThreads * kItems];
  uint32_t vals[kSortThreads * kItems];
  uint32_t base[kBins];
  uint32_t glob[kBins];
  uint32_t wsum[kSortWarps];
  uint32_t hsum[kSortWarps];
  int tile;
};

// One tile t of a pass: rank its keys, publish, look back, scatter.  The
// caller has zeroed sm.cnt and synchronised; status (ntiles x 256 words)
// starts at zero.  clear_next: the status words of tile t for the pass after
// next (double buffering), or null.
template <typename K, int kItems>
__device__ __forceinline__ void sweep_tile(SweepSmem<K, kItems>& sm, int t,
                                           const K* __restrict__ keys_in,
                                           const uint32_t* __restrict__ vals_in,
                                           K* __restrict__ keys_out,
                                           uint32_t* __restrict__ vals_out, int n, int shift,
                                           const uint32_t* __restrict__ digit_count,
                                           uint32_t* __restrict__ status, int* __restrict__ err,
                                           uint32_t* __restrict__ clear_next) {
  constexpr int kTile = kSortThreads * kItems;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // the next pass's status words of this tile (the pass before last used
  // them, and it has finished)
  if (clear_next) clear_next[(size_t)t * kBins + tid] = 0u;
  // the pass's global digit offsets: an exclusive scan of its digit counts,
  // redone by every tile (256 words) instead of a kernel of its own
  const uint32_t hcount = __ldg(digit_count + tid);
  uint32_t hincl = hcount;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t q = __shfl_up_sync(kFull, hincl, o);
    if (lane >= o) hincl += q;
  }
  if (lane == 31) sm.hsum[warp] = hincl;  // read after the ranking's barrier

  const long long tile0 = (long long)t * kTile;
  const long long wbase = tile0 + (long long)warp * (kWarp * kItems);
  K k_reg[kItems];
  uint32_t v_reg[kItems], r_reg[kItems];
  // all loads in flight before the ranking starts
#pragma unroll
  for (int r = 0; r < kItems; ++r) {
    const long long idx = wbase + r * kWarp + lane;
    k_reg[r] = (idx < n) ? __ldg(keys_in + idx) : (K)0;
    v_reg[r] = (idx < n) ? __ldg(vals_in + idx) : 0u;
  }
#pragma unroll
  for (int r = 0; r < kItems; ++r) {
    const long long idx = wbase + r * kWarp + lane;
    const bool valid = idx < n;
    const K key = k_reg[r];
    const uint32_t d = valid ? (uint32_t)(key >> shift) & 0xffu : kBins;
    const unsigned peers = __match_any_sync(kFull, d);
    const int leader = __ffs(peers) - 1;
    uint32_t old = 0;
    if (valid && lane == leader) {
      old = sm.cnt[warp][d];
      sm.cnt[warp][d] = old + __popc(peers);
    }
    old = __shfl_sync(kFull, old, leader);
    __syncwarp();
    r_reg[r] = old + __popc(peers & lanemask_lt());
  }
  __syncthreads();

  {
    const int d = tid;  // kSortThreads == kBins
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
      const uint32_t c = sm.cnt[w][d];
      sm.cnt[w][d] = run;
      run += c;
    }
    // run = this tile's count of digit d: publish it, then look back
    uint32_t* mine = status + (size_t)t * kBins + d;
    atomicExch(mine, (t == 0 ? kFlagP : kFlagA) | run);
    uint32_t excl = 0;
    if (t > 0) {
      excl = lookback_prefix(status, t, d, err);
      atomicExch(mine, kFlagP | ((excl + run) & kValMask));
    }
    uint32_t gbase = hincl - hcount;
    for (int w = 0; w < warp; ++w) gbase += sm.hsum[w];
    sm.glob[d] = gbase + excl;
    // tile-local base of digit d: exclusive prefix over digits
    uint32_t v = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t q = __shfl_up_sync(kFull, v, o);
      if (lane >= o) v += q;
    }
    if (lane == 31) sm.wsum[warp] = v;
    __syncthreads();
    uint32_t add = 0;
    for (int w = 0; w < warp; ++w) add += sm.wsum[w];
    sm.base[d] = v - run + add;
  }
  __syncthreads();

#pragma unroll
  for (int r = 0; r < kItems; ++r) {
    const long long idx = wbase + r * kWarp + lane;
    if (idx < n) {
      const uint32_t d = (uint32_t)(k_reg[r] >> shift) & 0xffu;
      const uint32_t lp = sm.base[d] + sm.cnt[warp][d] + r_reg[r];
      sm.keys[lp] = k_reg[r];
      sm.vals[lp] = v_reg[r];
    }
  }
  __syncthreads();

  const int tile_n = (int)min((long long)kTile, (long long)n - tile0);
  for (int i = tid; i < tile_n; i += kSortThreads) {
    const K key = sm.keys[i];
    const uint32_t d = (uint32_t)(key >> shift) & 0xffu;
    const uint32_t g = sm.glob[d] + (uint32_t)i - sm.base[d];
    keys_out[g] = key;
    vals_out[g] = sm.vals[i];
  }
}

// One pass, one tile per block.  ticket and status (ntiles x 256 words)
// start at zero.
template <typename K, int kItems>
__global__ void __launch_bounds__(kSortThreads)
k_onesweep(const K* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
           K* __restrict__ keys_out, uint32_t* __restrict__ vals_out, int n, int shift,
           const uint32_t* __restrict__ digit_count, int* __restrict__ ticket,
           uint32_t* __restrict__ status, int* __restrict__ err,
           uint32_t* __restrict__ clear_next) {
  __shared__ SweepSmem<K, kItems> sm;
  const int tid = threadIdx.x;
  for (int i = tid; i < kSortWarps * kBins; i += kSortThreads) (&sm.cnt[0][0])[i] = 0;
  // the ticket words were cleared before the sort's first pass
  if (tid == 0) sm.tile = atomicAdd(ticket, 1);
  // Launched as a programmatic dependent of the previous pass, the tile may
  // start while that pass still runs: everything below reads or clears what
  // it writes, so wait for it to finish here, then let the next pass launch.
  grid_dependency_wait();
  grid_dependents_launch();
  __syncthreads();
  sweep_tile<K, kItems>(sm, sm.tile, keys_in, vals_in, keys_out, vals_out, n, shift,
                        digit_count, status, err, clear_next);
}

// ---------------------------------------------------------------- scan
constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

__global__ void __launch_bounds__(kScanThreads)
k_scan_reduce(const uint32_t* __restrict__ data, int n, uint32_t* __restrict__ sums) {
  __shared__ uint32_t s_w[kScanThreads / 32];
  const long long base = (long long)blockIdx.x * kScanTile;
  uint32_t acc = 0;
  for (int r = 0; r < kScanItems; ++r) {
    long long i = base + (long long)r * kScanThreads + threadIdx.x;
    if (i < n) acc += data[i];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
  if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < kScanThreads / 32; ++w) t += s_w[w];
    sums[blockIdx.x] = t;
  }
}

// Shared-memory index with one pad word per 32: thread t's run of
// kScanItems consecutive words then spreads over all 32 banks.
__device__ __forceinline__ int pad32(int i) { return i + (i >> 5); }

__global__ void __launch_bounds__(kScanThreads)
k_scan_down(uint32_t* __restrict__ data, int n, const uint32_t* __restrict__ sums) {
  __shared__ uint32_t s_tile[kScanTile + kScanTile / 32];
  __shared__ uint32_t s_w[kScanThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long base = (long long)blockIdx.x * kScanTile;
  for (int r = 0; r < kScanItems; ++r) {
    long long i = base + (long long)r * kScanThreads + tid;
    s_tile[pad32(r * kScanThreads + tid)] = (i < n) ? data[i] : 0u;
  }
  __syncthreads();
  uint32_t loc[kScanItems];
  uint32_t sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    loc[k] = s_tile[pad32(tid * kScanItems + k)];
    sum += loc[k];
  }
  uint32_t v = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(kFull, v, o);
    if (lane >= o) v += t;
  }
  if (lane == 31) s_w[warp] = v;
  __syncthreads();
  uint32_t add = sums[blockIdx.x];
  for (int w = 0; w < warp; ++w) add += s_w[w];
  uint32_t run = add + v - sum;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    s_tile[pad32(tid * kScanItems + k)] = run;
    run += loc[k];
  }
  __syncthreads();
  for (int r = 0; r < kScanItems; ++r) {
    long long i = base + (long long)r * kScanThreads + tid;
    if (i < n) data[i] = s_tile[pad32(r * kScanThreads + tid)];
  }
}

int sort_sm_count() {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
  }
  return sms;
}

// Keys per thread for n keys: the largest that still gives half as many
// tiles as SMs.
template <typename K>
int pick_items(int n) {
  const int target = sort_sm_count() / 2;
  int it = sort_items<K>();
  while (it > kMinItems && div_up(n, kSortThreads * it) < target) it >>= 1;
  return it;
}

// dependent: launched as a programmatic dependent of the kernel ahead of it
// on s (the previous pass), so that its launch overlaps that pass's tail.
template <typename K, int kItems>
void launch_onesweep(int ntiles, const K* ki, const uint32_t* vi, K* ko, uint32_t* vo, int n,
                     int shift, const uint32_t* base, int* ticket, uint32_t* st, int* err,
                     uint32_t* clear_next, cudaStream_t s, bool dependent) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)ntiles);
  cfg.blockDim = dim3(kSortThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = dependent ? 1 : 0;
  check(cudaLaunchKernelEx(&cfg, k_onesweep<K, kItems>, ki, vi, ko, vo, n, shift, base, ticket,
                           st, err, clear_next),
        "k_onesweep launch");
}

template <typename K>
void launch_onesweep_items(int items, int ntiles, const K* ki, const uint32_t* vi, K* ko,
                           uint32_t* vo, int n, int shift, const uint32_t* base, int* ticket,
                           uint32_t* st, int* err, uint32_t* clear_next, cudaStream_t s,
                           bool dependent) {
  if constexpr (sizeof(K) == 4) {
    if (items == 16)
      return launch_onesweep<K, 16>(ntiles, ki, vi, ko, vo, n, shift, base, ticket, st, err,
                                    clear_next, s, dependent);
  }
  if (items == 8)
    return launch_onesweep<K, 8>(ntiles, ki, vi, ko, vo, n, shift, base, ticket, st, err,
                                 clear_next, s, dependent);
  if (items == 4)
    return launch_onesweep<K, 4>(ntiles, ki, vi, ko, vo, n, shift, base, ticket, st, err,
                                 clear_next, s, dependent);
  launch_onesweep<K, 2>(ntiles, ki, vi, ko, vo, n, shift, base, ticket, st, err, clear_next, s,
                        dependent);
}

}  // namespace

size_t scan_tmp_words(int n);

// Scratch of the sort: per-pass digit counts (passes x 256), per-pass tile
// tickets (passes), one word for give-up reports when the caller passes no
// status word, then the tile status words of one or two passes (ntiles x 256
// each).  Sized for the smallest tiles.
size_t radix_sort_count_words(int n) {
  return (size_t)kMaxPasses * kBins + kMaxPasses + 1 + (size_t)kBins * div_up(n, kMinTile);
}

uint32_t* radix_sort_prepare(uint32_t* counts, int bits, cudaStream_t s) {
  const int passes = (bits + 7) / 8;
  check(cudaMemsetAsync(counts, 0, sizeof(uint32_t) * ((size_t)passes * kBins + passes + 1), s),
        "radix sort histogram reset");
  return counts;
}

template <typename K>
void radix_sort_pairs(K* keys, uint32_t* vals, K* keys_alt, uint32_t* vals_alt,
                      uint32_t* counts, int n, int bits, cudaStream_t s, int* status,
                      bool hist_ready) {
  if (n <= 1) return;
  const int items = pick_items<K>(n);
  const int ntiles = div_up(n, kSortThreads * items);
  const int passes = (bits + 7) / 8;
  if (passes > kMaxPasses) throw CudaError("radix_sort_pairs: too many key bits");
  uint32_t* hist = counts;                      // passes x 256
  int* tickets = (int*)(counts + (size_t)passes * kBins);
  int* err = status ? status : tickets + passes;
  uint32_t* st = counts + (size_t)passes * kBins + passes + 1;
  if (!hist_ready) {
    radix_sort_prepare(counts, bits, s);
    const int hgrid = std::max(1, std::min(div_up(n, kSortThreads * 8), 148 * 4));
    k_digit_hist<K><<<hgrid, kSortThreads, 0, s>>>(keys, n, passes, hist);
  }

  K *ki = keys, *ko = keys_alt;
  uint32_t *vi = vals, *vo = vals_alt;
  // Two status buffers when the scratch holds them (it is sized for the
  // smallest tiles): each pass clears the other buffer's words of its own
  // tiles for the pass after it, so only the first needs a memset.
  const size_t tile_words = (size_t)ntiles * kBins;
  const bool two = 2 * (size_t)ntiles <= (size_t)div_up(n, kMinTile);
  for (int p = 0; p < passes; ++p) {
    uint32_t* cur = (two && (p & 1)) ? st + tile_words : st;
    uint32_t* next = (two && p + 1 < passes) ? ((p & 1) ? st : st + tile_words) : nullptr;
    const bool reset = p == 0 || !two;
    if (reset)
      check(cudaMemsetAsync(cur, 0, sizeof(uint32_t) * tile_words, s), "radix sort status reset");
    // a pass right behind the previous one launches as its programmatic dependent
    launch_onesweep_items<K>(items, ntiles, ki, vi, ko, vo, n, 8 * p, hist + (size_t)p * kBins,
                             tickets + p, cur, err, next, s, !reset);
    K* t = ki; ki = ko; ko = t;
    uint32_t* u = vi; vi = vo; vo = u;
  }
  if (ki != keys) {
    check(cudaMemcpyAsync(keys, ki, sizeof(K) * n, cudaMemcpyDeviceToDevice, s),
          "radix sort copy-back keys");
    check(cudaMemcpyAsync(vals, vi, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s),
          "radix sort copy-back vals");
  }
  check(cudaGetLastError(), "radix_sort_pairs launch");
}

int sort_wait_selftest() {
  constexpr int kTiles = 4;
  uint32_t *status = nullptr, *out = nullptr;
  int* err = nullptr;
  auto release = [&]() {
    cudaFree(status);
    cudaFree(out);
    cudaFree(err);
  };
  int bits = 0;
  try {
    check(cudaMalloc(&status, sizeof(uint32_t) * kTiles * kBins), "probe status");
    check(cudaMalloc(&out, sizeof(uint32_t) * kBins), "probe out");
    check(cudaMalloc(&err, sizeof(int)), "probe err");
    check(cudaMemset(status, 0, sizeof(uint32_t) * kTiles * kBins), "probe status clear");
    check(cudaMemset(err, 0, sizeof(int)), "probe err clear");
    k_lookback_probe<<<1, kBins>>>(status, kTiles - 1, err, out);
    check(cudaGetLastError(), "k_lookback_probe launch");
    check(cudaDeviceSynchronize(), "k_lookback_probe");
    check(cudaMemcpy(&bits, err, sizeof(int), cudaMemcpyDeviceToHost), "probe err read");
  } catch (...) {
    release();
    throw;
  }
  release();
  return bits;
}

template void radix_sort_pairs<uint32_t>(uint32_t*, uint32_t*, uint32_t*, uint32_t*, uint32_t*,
                                         int, int, cudaStream_t, int*, bool);
template void radix_sort_pairs<uint64_t>(uint64_t*, uint32_t*, uint64_t*, uint32_t*, uint32_t*,
                                         int, int, cudaStream_t, int*, bool);

}  // namespace nb

namespace nb {

size_t scan_tmp_words(int n) { return (size_t)div_up(n, kScanTile) + 1; }

// Exclusive prefix sum of n uint32 in place (tmp: scan_tmp_words(n) words).
void scan_exclusive_u32(uint32_t* data, int n, uint32_t* tmp, cudaStream_t s) {
  if (n <= 0) return;
  const int nb = div_up(n, kScanTile);
  k_scan_reduce<<<nb, kScanThreads, 0, s>>>(data, n, tmp);
  k_scan_inplace<<<1, 1024, 0, s>>>(tmp, nb);
  k_scan_down<<<nb, kScanThreads, 0, s>>>(data, n, tmp);
  check(cudaGetLastError(), "scan_exclusive_u32 launch");
}

}  // namespace nb
