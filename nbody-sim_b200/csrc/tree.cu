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
#include "kernels.cuh"

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

template <typename T>
__global__ void __launch_bounds__(kThreads)
k_keys(const T* __restrict__ x, const T* __restrict__ y, const T* __restrict__ z, int n,
       const unsigned long long* __restrict__ enc, TreeGeom* __restrict__ geom_out,
       uint32_t* __restrict__ keys, uint32_t* __restrict__ perm, int* __restrict__ status) {
  __shared__ TreeGeom g;
  if (threadIdx.x == 0) {
    compute_geom(enc, g);
    if (blockIdx.x == 0) *geom_out = g;
  }
  __syncthreads();
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
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
    keys[i] = morton30(c[0], c[1], c[2]);
    perm[i] = (uint32_t)i;
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
__device__ __forceinline__ int delta(const uint32_t* __restrict__ keys, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  uint32_t a = keys[i], b = keys[j];
  if (a != b) return __clz(a ^ b);
  return 32 + __clz((uint32_t)i ^ (uint32_t)j);
}

__global__ void __launch_bounds__(kThreads)
k_karras(const uint32_t* __restrict__ keys, int n, int* __restrict__ left,
         int* __restrict__ right, int* __restrict__ parent, int* __restrict__ lo_out,
         int* __restrict__ hi_out, uint8_t* __restrict__ prefix, int* __restrict__ visit) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) > 0 ? 1 : -1;
  const int dmin = delta(keys, n, i, i - d);
  int lmax = 2;
  while (delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dnode = delta(keys, n, i, j);
  int s = 0, t = l;
  do {
    t = (t + 1) >> 1;
    if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
  } while (t > 1);
  const int gamma = i + s * d + min(d, 0);
  const int lo = min(i, j), hi = max(i, j);
  const int lc = (lo == gamma) ? (n - 1) + gamma : gamma;
  const int rc = (hi == gamma + 1) ? (n - 1) + gamma + 1 : gamma + 1;
  left[i] = lc;
  right[i] = rc;
  parent[lc] = i;
  parent[rc] = i;
  lo_out[i] = lo;
  hi_out[i] = hi;
  prefix[i] = (uint8_t)(dnode >= 32 ? 30 : dnode - 2);
  visit[i] = 0;
  if (i == 0) parent[0] = -1;
}

// ------------------------------------------------------------- moments
struct Moments {
  double m, x, y, z;
  float lx, ly, lz, hx, hy, hz;
};

__device__ __forceinline__ Moments leaf_moments(const float4* __restrict__ body4,
                                                const double* xd, const double* yd,
                                                const double* zd, int j) {
  float4 b = body4[j];
  Moments r;
  double px = xd ? xd[j] : (double)b.x, py = yd ? yd[j] : (double)b.y,
         pz = zd ? zd[j] : (double)b.z;
  r.m = (double)b.w;
  r.x = r.m * px; r.y = r.m * py; r.z = r.m * pz;
  r.lx = r.hx = b.x; r.ly = r.hy = b.y; r.lz = r.hz = b.z;
  return r;
}

__device__ __forceinline__ Moments node_moments(const double4* sum, const float4* blo,
                                                const float4* bhi, int i) {
  const double2* s2 = reinterpret_cast<const double2*>(sum + i);
  const double2 s0 = __ldcg(s2), s1 = __ldcg(s2 + 1);
  float4 a = __ldcg(blo + i), b = __ldcg(bhi + i);
  Moments r;
  r.m = s0.x; r.x = s0.y; r.y = s1.x; r.z = s1.y;
  r.lx = a.x; r.ly = a.y; r.lz = a.z; r.hx = b.x; r.hy = b.y; r.hz = b.z;
  return r;
}

// One thread per leaf climbs while it is the second child to arrive; the
// node is then the sum left + right (fixed order, so the FP64 sums do not
// depend on arrival order).  No thread ever waits on another.
__global__ void __launch_bounds__(kThreads)
k_bottom_up(const float4* __restrict__ body4, const double* __restrict__ xd,
            const double* __restrict__ yd, const double* __restrict__ zd, int n,
            const int* __restrict__ left, const int* __restrict__ right,
            const int* __restrict__ parent, int* __restrict__ visit, double4* __restrict__ sum,
            float4* __restrict__ blo, float4* __restrict__ bhi, int* __restrict__ status) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n || n < 2) return;
  int p = parent[(n - 1) + j];
  for (int guard = 0; p >= 0; ++guard) {
    if (guard > 4096) { atomicOr(status, kStatusTreeLimit); return; }
    __threadfence();
    if (atomicAdd(&visit[p], 1) == 0) return;
    __threadfence();
    const int l = left[p], r = right[p];
    Moments a = (l >= n - 1) ? leaf_moments(body4, xd, yd, zd, l - (n - 1))
                             : node_moments(sum, blo, bhi, l);
    Moments b = (r >= n - 1) ? leaf_moments(body4, xd, yd, zd, r - (n - 1))
                             : node_moments(sum, blo, bhi, r);
    double2* d2 = reinterpret_cast<double2*>(sum + p);
    __stcg(d2, make_double2(a.m + b.m, a.x + b.x));
    __stcg(d2 + 1, make_double2(a.y + b.y, a.z + b.z));
    __stcg(blo + p, make_float4(fminf(a.lx, b.lx), fminf(a.ly, b.ly), fminf(a.lz, b.lz), 0.f));
    __stcg(bhi + p, make_float4(fmaxf(a.hx, b.hx), fmaxf(a.hy, b.hy), fmaxf(a.hz, b.hz), 0.f));
    p = parent[p];
  }
}

// ---------------------------------------------------------- octree layout
__device__ __forceinline__ int bin_level(const uint8_t* prefix, int n, int b) {
  return (b >= n - 1) ? 10 : (int)prefix[b] / 3;
}

// Visits the octree children of top node b (binary descendants that start a
// deeper octree level, or leaves) in key order.
template <typename F>
__device__ __forceinline__ int for_each_oct_child(const int* __restrict__ left,
                                                  const int* __restrict__ right,
                                                  const uint8_t* __restrict__ prefix, int n,
                                                  int b, int lb, F f) {
  int stack[8];
  int top = 0, k = 0;
  stack[top++] = right[b];
  stack[top++] = left[b];
  while (top > 0) {
    int c = stack[--top];
    if (c >= n - 1 || bin_level(prefix, n, c) > lb) {
      f(c, k++);
    } else if (top + 2 <= 8) {
      stack[top++] = right[c];
      stack[top++] = left[c];
    }
  }
  return k;
}

__global__ void __launch_bounds__(kThreads)
k_oct_mark(int n, const int* __restrict__ left, const int* __restrict__ right,
           const int* __restrict__ parent, const uint8_t* __restrict__ prefix,
           uint8_t* __restrict__ nch, uint32_t* __restrict__ off, int* __restrict__ fin) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int nb = 2 * n - 1;
  if (b >= nb) return;
  const int lb = bin_level(prefix, n, b);
  const bool top = (b == 0) || lb > bin_level(prefix, n, parent[b]);
  int cnt = 0;
  if (top && b < n - 1 && lb < 10)
    cnt = for_each_oct_child(left, right, prefix, n, b, lb, [](int, int) {});
  nch[b] = (uint8_t)cnt;
  off[b] = (uint32_t)cnt;
  fin[b] = top ? 0 : -1;
}

__global__ void __launch_bounds__(kThreads)
k_oct_assign(int n, const int* __restrict__ left, const int* __restrict__ right,
             const uint8_t* __restrict__ prefix, const uint8_t* __restrict__ nch,
             const uint32_t* __restrict__ off, int* __restrict__ fin, int* __restrict__ n_nodes) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int nb = 2 * n - 1;
  if (b >= nb) return;
  if (b == nb - 1) *n_nodes = 1 + (int)(off[b] + nch[b]);
  if (nch[b] == 0) return;
  const int lb = bin_level(prefix, n, b);
  const int base = 1 + (int)off[b];
  for_each_oct_child(left, right, prefix, n, b, lb, [&](int c, int k) { fin[c] = base + k; });
}

__global__ void __launch_bounds__(kThreads)
k_oct_write(int n, const int* __restrict__ lo, const int* __restrict__ hi,
            const uint8_t* __restrict__ prefix, const uint8_t* __restrict__ nch,
            const uint32_t* __restrict__ off, const int* __restrict__ fin,
            const double4* __restrict__ sum, const float4* __restrict__ blo,
            const float4* __restrict__ bhi, const float4* __restrict__ body4,
            const TreeGeom* __restrict__ geom, OctNodes oct) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int nb = 2 * n - 1;
  if (b >= nb) return;
  const int f = (b == 0) ? 0 : fin[b];
  if (f < 0) return;
  const float rhs = geom->rhs;
  if (b >= n - 1) {  // single-body leaf
    const int j = b - (n - 1);
    float4 p = body4[j];
    oct.com[f] = p;
    oct.info[f] = make_int4(-1, j, (1 << 4), __float_as_int(ldexpf(rhs, -10)));
    oct.box_lo[f] = make_float4(p.x, p.y, p.z, 0.f);
    oct.box_hi[f] = make_float4(p.x, p.y, p.z, 0.f);
    return;
  }
  const int L = (int)prefix[b] / 3;
  const double4 s = sum[b];
  float4 lo4 = blo[b], hi4 = bhi[b];
  float4 c;
  if (s.x > 0.0) {
    c = make_float4((float)(s.y / s.x), (float)(s.z / s.x), (float)(s.w / s.x), (float)s.x);
  } else {
    c = make_float4(0.5f * (lo4.x + hi4.x), 0.5f * (lo4.y + hi4.y), 0.5f * (lo4.z + hi4.z), 0.f);
  }
  const int k = nch[b];
  const int count = hi[b] - lo[b] + 1;
  oct.com[f] = c;
  oct.info[f] = make_int4(k > 0 ? 1 + (int)off[b] : -1, lo[b], (count << 4) | k,
                          __float_as_int(ldexpf(rhs, -L)));
  oct.box_lo[f] = lo4;
  oct.box_hi[f] = hi4;
}

// Target groups for the warp walks: the maximal nodes of the binary radix
// tree holding <= gmax bodies.  They partition the bodies into contiguous
// key ranges whose bodies share a Morton prefix, so a group never straddles
// a jump of the space-filling curve (a fixed run of 32 consecutive bodies
// can: its box then spans most of the domain and its walk degenerates to
// O(N) work on one warp).
__global__ void __launch_bounds__(kThreads)
k_group_mark(int n, int gmax, const int* __restrict__ lo, const int* __restrict__ hi,
             const int* __restrict__ parent, uint32_t* __restrict__ flag) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int nb = 2 * n - 1;
  if (b >= nb) return;
  const int cnt = (b >= n - 1) ? 1 : hi[b] - lo[b] + 1;
  int pc = 0x7fffffff;
  if (b != 0) {
    const int p = parent[b];
    pc = hi[p] - lo[p] + 1;
  }
  flag[b] = (cnt <= gmax && pc > gmax) ? 1u : 0u;
}

__global__ void __launch_bounds__(kThreads)
k_group_write(int n, int gmax, const int* __restrict__ lo, const int* __restrict__ hi,
              const int* __restrict__ parent, const uint32_t* __restrict__ off,
              int2* __restrict__ groups, int* __restrict__ n_groups) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int nb = 2 * n - 1;
  if (b >= nb) return;
  const bool leaf = b >= n - 1;
  const int cnt = leaf ? 1 : hi[b] - lo[b] + 1;
  int pc = 0x7fffffff;
  if (b != 0) {
    const int p = parent[b];
    pc = hi[p] - lo[p] + 1;
  }
  const bool is_group = cnt <= gmax && pc > gmax;
  if (is_group) groups[off[b]] = make_int2(leaf ? b - (n - 1) : lo[b], cnt);
  if (b == nb - 1) *n_groups = (int)off[b] + (is_group ? 1 : 0);
}

__global__ void k_group_single(int2* groups, int* n_groups) {
  groups[0] = make_int2(0, 1);
  *n_groups = 1;
}

// N == 1: the root is the single body.
__global__ void k_oct_single(const float4* __restrict__ body4, const TreeGeom* __restrict__ geom,
                             OctNodes oct, int* __restrict__ n_nodes) {
  float4 p = body4[0];
  oct.com[0] = p;
  oct.info[0] = make_int4(-1, 0, (1 << 4), __float_as_int(geom->rhs));
  oct.box_lo[0] = make_float4(p.x, p.y, p.z, 0.f);
  oct.box_hi[0] = make_float4(p.x, p.y, p.z, 0.f);
  *n_nodes = 1;
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
  w.bin_parent = dalloc<int>(nb, "bin_parent");
  w.bin_lo = dalloc<int>(n, "bin_lo");
  w.bin_hi = dalloc<int>(n, "bin_hi");
  w.bin_prefix = dalloc<uint8_t>(n, "bin_prefix");
  w.bin_visit = dalloc<int>(n, "bin_visit");
  w.bin_sum = dalloc<double4>(n, "bin_sum");
  w.bin_box_lo = dalloc<float4>(n, "bin_box_lo");
  w.bin_box_hi = dalloc<float4>(n, "bin_box_hi");
  w.oct_nch = dalloc<uint8_t>(nb, "oct_nch");
  w.oct_off = dalloc<uint32_t>(nb, "oct_off");
  w.oct_final = dalloc<int>(nb, "oct_final");
  w.scan_tmp = dalloc<uint32_t>(scan_tmp_words((int)nb), "scan_tmp");
  w.oct.com = dalloc<float4>(nb, "oct com");
  w.oct.info = dalloc<int4>(nb, "oct info");
  w.oct.box_lo = dalloc<float4>(nb, "oct box_lo");
  w.oct.box_hi = dalloc<float4>(nb, "oct box_hi");
  w.bbox_enc = dalloc<unsigned long long>(6, "bbox");
  w.geom = dalloc<TreeGeom>(1, "geom");
  w.n_nodes = dalloc<int>(1, "n_nodes");
  w.groups = dalloc<int2>(n, "groups");
  w.group_flag = dalloc<uint32_t>(nb, "group flags");
  w.n_groups = dalloc<int>(1, "n_groups");
  w.status = dalloc<int>(1, "status");
  check(cudaMemset(w.status, 0, sizeof(int)), "status init");
  check(cudaMemset(w.n_nodes, 0, sizeof(int)), "n_nodes init");
}

void tree_free(TreeWork& w) {
  void* ptrs[] = {w.keys, w.perm, w.keys_alt, w.perm_alt, w.counts, w.body4, w.bin_left,
                  w.bin_right, w.bin_parent, w.bin_lo, w.bin_hi, w.bin_prefix, w.bin_visit,
                  w.bin_sum, w.bin_box_lo, w.bin_box_hi, w.oct_nch, w.oct_off, w.oct_final,
                  w.scan_tmp, w.oct.com, w.oct.info, w.oct.box_lo, w.oct.box_hi, w.bbox_enc,
                  w.geom, w.n_nodes, w.status, w.groups, w.group_flag, w.n_groups};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  w = TreeWork();
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
void launch_keys(TreeWork& w, const T* x, const T* y, const T* z, int n, cudaStream_t s) {
  int g = std::min(grid_for(n), 148 * 16);
  if (g < 1) g = 1;
  k_keys<T><<<g, kThreads, 0, s>>>(x, y, z, n, w.bbox_enc, w.geom, w.keys, w.perm, w.status);
  check(cudaGetLastError(), "k_keys launch");
}

template void launch_bbox<float>(TreeWork&, const float*, const float*, const float*, int,
                                 cudaStream_t);
template void launch_bbox<double>(TreeWork&, const double*, const double*, const double*, int,
                                  cudaStream_t);
template void launch_keys<float>(TreeWork&, const float*, const float*, const float*, int,
                                 cudaStream_t);
template void launch_keys<double>(TreeWork&, const double*, const double*, const double*, int,
                                  cudaStream_t);

void launch_gather_body4(TreeWork& w, const float* x, const float* y, const float* z,
                         const float* m, int n, cudaStream_t s) {
  int g = std::min(grid_for(n), 148 * 16);
  if (g < 1) g = 1;
  k_gather_body4<<<g, kThreads, 0, s>>>(w.perm, x, y, z, m, n, w.body4);
  check(cudaGetLastError(), "k_gather_body4 launch");
}

void launch_build_topology(TreeWork& w, int n, cudaStream_t s) {
  if (n < 2) return;
  k_karras<<<grid_for(n - 1), kThreads, 0, s>>>(w.keys, n, w.bin_left, w.bin_right,
                                                w.bin_parent, w.bin_lo, w.bin_hi, w.bin_prefix,
                                                w.bin_visit);
  check(cudaGetLastError(), "k_karras launch");
}

void launch_build_groups(TreeWork& w, int n, int gmax, cudaStream_t s) {
  if (n < 1) return;
  if (n == 1) {
    k_group_single<<<1, 1, 0, s>>>(w.groups, w.n_groups);
    check(cudaGetLastError(), "k_group_single launch");
    return;
  }
  const int nb = 2 * n - 1;
  k_group_mark<<<grid_for(nb), kThreads, 0, s>>>(n, gmax, w.bin_lo, w.bin_hi, w.bin_parent,
                                                 w.group_flag);
  scan_exclusive_u32(w.group_flag, nb, w.scan_tmp, s);
  k_group_write<<<grid_for(nb), kThreads, 0, s>>>(n, gmax, w.bin_lo, w.bin_hi, w.bin_parent,
                                                  w.group_flag, w.groups, w.n_groups);
  check(cudaGetLastError(), "group launch");
}

void launch_build_moments(TreeWork& w, int n, const double* xd, const double* yd,
                          const double* zd, cudaStream_t s) {
  if (n < 1) return;
  if (n == 1) {
    k_oct_single<<<1, 1, 0, s>>>(w.body4, w.geom, w.oct, w.n_nodes);
    check(cudaGetLastError(), "k_oct_single launch");
    return;
  }
  const int nb = 2 * n - 1;
  k_bottom_up<<<grid_for(n), kThreads, 0, s>>>(w.body4, xd, yd, zd, n, w.bin_left, w.bin_right,
                                               w.bin_parent, w.bin_visit, w.bin_sum,
                                               w.bin_box_lo, w.bin_box_hi, w.status);
  k_oct_mark<<<grid_for(nb), kThreads, 0, s>>>(n, w.bin_left, w.bin_right, w.bin_parent,
                                               w.bin_prefix, w.oct_nch, w.oct_off, w.oct_final);
  scan_exclusive_u32(w.oct_off, nb, w.scan_tmp, s);
  k_oct_assign<<<grid_for(nb), kThreads, 0, s>>>(n, w.bin_left, w.bin_right, w.bin_prefix,
                                                 w.oct_nch, w.oct_off, w.oct_final, w.n_nodes);
  k_oct_write<<<grid_for(nb), kThreads, 0, s>>>(n, w.bin_lo, w.bin_hi, w.bin_prefix, w.oct_nch,
                                                w.oct_off, w.oct_final, w.bin_sum, w.bin_box_lo,
                                                w.bin_box_hi, w.body4, w.geom, w.oct);
  check(cudaGetLastError(), "octree launch");
}

}  // namespace nb
