// sort.cu -- stable LSD radix sort of (uint32 key, uint32 value) pairs.
//
// Replaces the reference's serial DFS ordering (bhtree_sortKernel,
// BHTree.cu:322-352, a <<<1,1>>> launch) by a Morton-order sort: the body
// order of the octree IS the sorted key order.  Per 8-bit digit: an upsweep
// (per-block digit counts, warp-aggregated shared atomics so runs of equal
// digits in nearly sorted input do not serialise), one scan of the
// digit-major count table, and a stable scatter that ranks keys with
// __match_any_sync and stages the tile in shared memory so global writes are
// runs of consecutive addresses.  HBM traffic per pass: 4 B (upsweep) +
// 8 B read + 8 B write (scatter) per pair.
#include "common.cuh"
#include "kernels.cuh"

namespace nb {
namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / kWarp;
// keys per thread: 16 (uint32 keys, 4096-key tiles) or 8 (uint64, 2048) so
// the staged tile stays within 48 KB of static shared memory
template <typename K>
constexpr int sort_items() { return sizeof(K) == 8 ? 8 : 16; }
template <typename K>
constexpr int sort_tile() { return kSortThreads * sort_items<K>(); }
constexpr int kMinTile = kSortThreads * 8;
constexpr int kBins = 256;

template <typename K>
__global__ void __launch_bounds__(kSortThreads)
k_sort_upsweep(const K* __restrict__ keys, uint32_t* __restrict__ counts, int n,
               int shift, int nblocks) {
  __shared__ uint32_t s_hist[kBins];
  const int tid = threadIdx.x, lane = tid & 31;
  s_hist[tid] = 0;
  __syncthreads();
  constexpr int kItems = sort_items<K>();
  const long long base = (long long)blockIdx.x * sort_tile<K>();
#pragma unroll 4
  for (int r = 0; r < kItems; ++r) {
    long long idx = base + (long long)r * kSortThreads + tid;
    bool valid = idx < n;
    uint32_t d = valid ? (uint32_t)(__ldg(keys + idx) >> shift) & 0xffu : kBins;
    unsigned peers = __match_any_sync(kFull, d);
    int leader = __ffs(peers) - 1;
    if (valid && lane == leader) atomicAdd(&s_hist[d], (uint32_t)__popc(peers));
  }
  __syncthreads();
  counts[(long long)tid * nblocks + blockIdx.x] = s_hist[tid];
}

// Exclusive scan of `total` uint32 in place, one block of 1024 threads.
__global__ void __launch_bounds__(1024) k_scan_inplace(uint32_t* __restrict__ data, int total) {
  __shared__ uint32_t s_part[1024];
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
  s_part[tid] = run;
  for (long long i = lo; i < hi; ++i) {
    uint32_t c = data[i];
    data[i] = run;
    run += c;
  }
}

template <typename K>
__global__ void __launch_bounds__(kSortThreads)
k_sort_scatter(const K* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
               K* __restrict__ keys_out, uint32_t* __restrict__ vals_out,
               const uint32_t* __restrict__ offsets, int n, int shift, int nblocks) {
  constexpr int kItems = sort_items<K>();
  constexpr int kTile = sort_tile<K>();
  __shared__ uint32_t s_cnt[kSortWarps][kBins];
  __shared__ K s_keys[kTile];
  __shared__ uint32_t s_vals[kTile];
  __shared__ uint32_t s_base[kBins];
  __shared__ uint32_t s_glob[kBins];
  __shared__ uint32_t s_wsum[kSortWarps];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < kSortWarps * kBins; i += kSortThreads) (&s_cnt[0][0])[i] = 0;
  __syncthreads();

  const long long tile0 = (long long)blockIdx.x * kTile;
  const long long wbase = tile0 + (long long)warp * (kWarp * kItems);
  K k_reg[kItems];
  uint32_t v_reg[kItems], r_reg[kItems];
#pragma unroll
  for (int r = 0; r < kItems; ++r) {
    long long idx = wbase + r * kWarp + lane;
    bool valid = idx < n;
    K key = valid ? __ldg(keys_in + idx) : (K)0;
    uint32_t val = valid ? __ldg(vals_in + idx) : 0u;
    uint32_t d = valid ? (uint32_t)(key >> shift) & 0xffu : kBins;
    unsigned peers = __match_any_sync(kFull, d);
    int leader = __ffs(peers) - 1;
    uint32_t old = 0;
    if (valid && lane == leader) {
      old = s_cnt[warp][d];
      s_cnt[warp][d] = old + __popc(peers);
    }
    old = __shfl_sync(kFull, old, leader);
    __syncwarp();
    k_reg[r] = key;
    v_reg[r] = val;
    r_reg[r] = old + __popc(peers & lanemask_lt());
  }
  __syncthreads();

  // per digit: exclusive prefix over warps; tile-local digit bases
  {
    const int d = tid;  // kSortThreads == kBins
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
      uint32_t c = s_cnt[w][d];
      s_cnt[w][d] = run;
      run += c;
    }
    uint32_t v = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(kFull, v, o);
      if (lane >= o) v += t;
    }
    if (lane == 31) s_wsum[warp] = v;
    __syncthreads();
    uint32_t add = 0;
    for (int w = 0; w < warp; ++w) add += s_wsum[w];
    s_base[d] = v - run + add;
    s_glob[d] = offsets[(long long)d * nblocks + blockIdx.x];
  }
  __syncthreads();

#pragma unroll
  for (int r = 0; r < kItems; ++r) {
    long long idx = wbase + r * kWarp + lane;
    if (idx < n) {
      uint32_t d = (uint32_t)(k_reg[r] >> shift) & 0xffu;
      uint32_t lp = s_base[d] + s_cnt[warp][d] + r_reg[r];
      s_keys[lp] = k_reg[r];
      s_vals[lp] = v_reg[r];
    }
  }
  __syncthreads();

  const int tile_n = (int)min((long long)kTile, (long long)n - tile0);
  for (int i = tid; i < tile_n; i += kSortThreads) {
    K key = s_keys[i];
    uint32_t d = (uint32_t)(key >> shift) & 0xffu;
    uint32_t g = s_glob[d] + (uint32_t)i - s_base[d];
    keys_out[g] = key;
    vals_out[g] = s_vals[i];
  }
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

__global__ void __launch_bounds__(kScanThreads)
k_scan_down(uint32_t* __restrict__ data, int n, const uint32_t* __restrict__ sums) {
  __shared__ uint32_t s_tile[kScanTile];
  __shared__ uint32_t s_w[kScanThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long base = (long long)blockIdx.x * kScanTile;
  for (int r = 0; r < kScanItems; ++r) {
    long long i = base + (long long)r * kScanThreads + tid;
    s_tile[r * kScanThreads + tid] = (i < n) ? data[i] : 0u;
  }
  __syncthreads();
  uint32_t loc[kScanItems];
  uint32_t sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    loc[k] = s_tile[tid * kScanItems + k];
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
    s_tile[tid * kScanItems + k] = run;
    run += loc[k];
  }
  __syncthreads();
  for (int r = 0; r < kScanItems; ++r) {
    long long i = base + (long long)r * kScanThreads + tid;
    if (i < n) data[i] = s_tile[r * kScanThreads + tid];
  }
}

}  // namespace

size_t scan_tmp_words(int n);

size_t radix_sort_count_words(int n) {
  const size_t table = (size_t)kBins * (size_t)div_up(n, kMinTile);
  return table + scan_tmp_words((int)table);
}

template <typename K>
void radix_sort_pairs(K* keys, uint32_t* vals, K* keys_alt, uint32_t* vals_alt,
                      uint32_t* counts, int n, int bits, cudaStream_t s) {
  if (n <= 1) return;
  const int nb = div_up(n, sort_tile<K>());
  const int passes = (bits + 7) / 8;
  // the count table is followed by room for the multi-block scan's partials
  uint32_t* scan_tmp = counts + (size_t)kBins * nb;
  K *ki = keys, *ko = keys_alt;
  uint32_t *vi = vals, *vo = vals_alt;
  for (int p = 0; p < passes; ++p) {
    const int shift = 8 * p;
    k_sort_upsweep<K><<<nb, kSortThreads, 0, s>>>(ki, counts, n, shift, nb);
    scan_exclusive_u32(counts, kBins * nb, scan_tmp, s);
    k_sort_scatter<K><<<nb, kSortThreads, 0, s>>>(ki, vi, ko, vo, counts, n, shift, nb);
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

template void radix_sort_pairs<uint32_t>(uint32_t*, uint32_t*, uint32_t*, uint32_t*, uint32_t*,
                                         int, int, cudaStream_t);
template void radix_sort_pairs<uint64_t>(uint64_t*, uint32_t*, uint64_t*, uint32_t*, uint32_t*,
                                         int, int, cudaStream_t);

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
