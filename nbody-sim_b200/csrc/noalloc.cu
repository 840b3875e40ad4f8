// noalloc.cu -- nbody_fof_noalloc: the device FoF of nbody_fof for callers
// that may not allocate device memory.
//
// Every buffer the FoF needs (Morton keys and radix-sort buffers, the Karras
// tree, FP64 moments, the octree, warp groups, union-find arrays and a
// bounded stack-spill area) is carved out of one file-scope __device__ array
// sized for kMaxN bodies; a tail of the same array holds a set-up input.
// Host code never uses the array's name as a pointer: the device address
// comes from cudaGetSymbolAddress, looked up once per device with that device
// current, on the first call made there.
//
// Under CUDA's lazy module loading (the default since CUDA 12.2) the runtime
// backs a __device__ array with device memory, and loads a kernel's code,
// only when they are first used.  The first call on a device therefore does
// both on purpose: it looks the array up and runs the whole FoF once on a
// set-up input of kMaxN bodies kept in the array's tail, so that every kernel
// the call launches (one variant each for n <= kMaxN) is loaded and the
// local-memory reservation has grown to what they need.  Later calls on that
// device then need no device memory at all.
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "capi_util.h"
#include "common.cuh"
#include "kernels.cuh"

namespace nb {
namespace {

constexpr int kMaxN = NBODY_FOF_NOALLOC_MAX_N;
constexpr int kSpillCap = 1024;     // stack entries per warp slot
constexpr int kSpillWarps = 1184;   // warp slots: 148 SMs x 2 blocks x 4 warps
constexpr size_t kAlign = 256;

constexpr size_t al(size_t b) { return (b + kAlign - 1) / kAlign * kAlign; }
constexpr size_t kNb = 2 * (size_t)kMaxN;
constexpr size_t kCountWords = 20480;  // >= 18441 words the 32-bit-key sort of kMaxN uses
constexpr size_t kScanWords = 4096;   // >= octree_scan_words(2 kMaxN - 1) = 512
constexpr size_t kMomTiles = 2 * ((size_t)kMaxN / kMomentTile + 2) + 8;

constexpr size_t kWorkBytes =
    4 * al(sizeof(uint32_t) * kMaxN) +          // keys, perm, keys_alt, perm_alt
    al(sizeof(uint32_t) * kCountWords) +        // radix-sort counts + scan partials
    al(sizeof(float4) * kMaxN) +                // body4
    4 * al(sizeof(int) * kMaxN) +               // bin_left, bin_right, bin_lo, bin_hi
    al(sizeof(uint32_t) * kNb) +                // bin_pinfo
    al(sizeof(uint8_t) * kMaxN) +               // bin_prefix
    al(sizeof(double4) * (kMaxN + 1)) +         // moment prefix sums
    al(sizeof(double4) * kMomTiles) +           // moment tile sums / prefixes
    al(sizeof(uint8_t) * kNb) +                 // oct_nch
    al(sizeof(uint32_t) * kNb) +                // oct_off
    al(sizeof(int) * kNb) +                     // oct_node
    al(sizeof(uint32_t) * kScanWords) +         // octree tile sums
    4 * al(sizeof(float4) * kNb) +              // octree com, info, box_lo, box_hi
    al(sizeof(unsigned long long) * 6) +        // bbox
    al(sizeof(TreeGeom)) +                      // root geometry
    5 * al(sizeof(int)) +                       // n_nodes, status, n_groups, fof groups, work
    al(sizeof(int2) * kMaxN) +                  // warp groups
    2 * al(sizeof(int) * kMaxN) +               // union-find parent, group sizes
    al(sizeof(int) * (size_t)kSpillWarps * kSpillCap);  // stack spill
// the set-up input and outputs: x, y, z, labels, agg_size of kMaxN bodies
constexpr size_t kSetupBytes = 4 * al(sizeof(float) * kMaxN) + al(sizeof(uint16_t) * kMaxN);
constexpr size_t kScratchBytes = kWorkBytes + kSetupBytes;

static_assert(kScratchBytes == NBODY_FOF_NOALLOC_SCRATCH_BYTES,
              "header's stated scratch size must match the array");

static __device__ __align__(256) unsigned char g_fof_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_addr[kMaxDevices] = {nullptr};

struct Carve {
  unsigned char* base;
  size_t off = 0;
  template <typename T>
  T* take(size_t count) {
    T* p = reinterpret_cast<T*>(base + off);
    off += al(sizeof(T) * count);
    if (off > kScratchBytes) throw ArgError("nbody_fof_noalloc: scratch layout overflow");
    return p;
  }
};


// The FoF of n <= kMaxN bodies on the legacy default stream, all scratch
// from the array at `base`; returns the number of groups (>= 2 members).
int fof_in_scratch(unsigned char* base, const float* x, const float* y, const float* z, int n,
                   float link_length, int* labels, uint16_t* agg_size) {
  if (n == 0) return 0;
  if (radix_sort_count_words(n) > kCountWords)
    throw CudaError("nbody_fof_noalloc: sort scratch too small");
  if (octree_scan_words(2 * n - 1) > kScanWords)
    throw CudaError("nbody_fof_noalloc: octree tile-sum scratch too small");
  Carve c{base};
  TreeWork w;
  w.cap = kMaxN;
  w.keys = c.take<uint32_t>(kMaxN);
  w.perm = c.take<uint32_t>(kMaxN);
  w.keys_alt = c.take<uint32_t>(kMaxN);
  w.perm_alt = c.take<uint32_t>(kMaxN);
  w.counts = c.take<uint32_t>(kCountWords);
  w.body4 = c.take<float4>(kMaxN);
  w.bin_left = c.take<int>(kMaxN);
  w.bin_right = c.take<int>(kMaxN);
  w.bin_lo = c.take<int>(kMaxN);
  w.bin_hi = c.take<int>(kMaxN);
  w.bin_pinfo = c.take<uint32_t>(kNb);
  w.bin_prefix = c.take<uint8_t>(kMaxN);
  w.mom_ploc = c.take<double4>(kMaxN + 1);
  w.mom_tiles = c.take<double4>(kMomTiles);
  w.oct_nch = c.take<uint8_t>(kNb);
  w.oct_off = c.take<uint32_t>(kNb);
  w.oct_node = c.take<int>(kNb);
  w.scan_tmp = c.take<uint32_t>(kScanWords);
  w.oct.com = c.take<float4>(kNb);
  w.oct.info = c.take<int4>(kNb);
  w.oct.box_lo = c.take<float4>(kNb);
  w.oct.box_hi = c.take<float4>(kNb);
  w.bbox_enc = c.take<unsigned long long>(6);
  w.geom = c.take<TreeGeom>(1);
  w.n_nodes = c.take<int>(1);
  w.status = c.take<int>(1);
  w.n_groups = c.take<int>(1);
  int* fof_groups = c.take<int>(1);
  int* work = c.take<int>(1);
  w.groups = c.take<int2>(kMaxN);
  int* parent = c.take<int>(kMaxN);
  int* sizes = c.take<int>(kMaxN);
  int* spill = c.take<int>((size_t)kSpillWarps * kSpillCap);
  if (c.off > kWorkBytes) throw CudaError("nbody_fof_noalloc: scratch layout overflow");
  w.group_max = 32;
  // the array keeps the previous call's contents: clear what is read before written
  check(cudaMemsetAsync(w.status, 0, sizeof(int), 0), "status clear");
  launch_bbox<float>(w, x, y, z, n, 0);
  launch_keys<float>(w, x, y, z, n, 0);
  radix_sort_pairs(w.keys, w.perm, w.keys_alt, w.perm_alt, w.counts, n, 30, 0, w.status);
  launch_gather_body4(w, x, y, z, nullptr, n, 0);
  launch_build_topology(w, n, 0);
  launch_build_moments(w, n, nullptr, nullptr, nullptr, 0);
  NeighborArgs na{w.oct.info, w.oct.box_lo, w.oct.box_hi, w.body4, n, w.groups,
                  w.n_groups, 8, spill, kSpillCap, work, w.status};
  launch_fof_link_capped(na, w.perm, link_length, parent, kSpillWarps, 0);
  launch_fof_finish(parent, n, labels, sizes, agg_size, fof_groups, w.status, 0);
  check(cudaGetLastError(), "nbody_fof_noalloc launch");
  check(cudaStreamSynchronize(0), "nbody_fof_noalloc sync");
  int st = 0;
  check(cudaMemcpy(&st, w.status, sizeof(int), cudaMemcpyDeviceToHost), "status read");
  if (st)
    throw ArgError("nbody_fof_noalloc: device status " + std::to_string(st), NBODY_ERR_OVERFLOW);
  int groups = 0;
  check(cudaMemcpy(&groups, fof_groups, sizeof(int), cudaMemcpyDeviceToHost), "groups read");
  return groups;
}

// The array's address on the current device.  The first call on a device
// also runs the FoF once on the set-up input (a unit lattice of kMaxN bodies
// with a 0.5 linking length, copied from host memory into the array's tail),
// which makes the runtime back the array and load every kernel the FoF uses.
unsigned char* scratch_for_current_device() {
  int dev = 0;
  check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) throw ArgError("nbody_fof_noalloc: device ordinal too large");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    check(cudaGetSymbolAddress(&p, g_fof_scratch), "cudaGetSymbolAddress(FoF scratch)");
    unsigned char* base = static_cast<unsigned char*>(p);
    unsigned char* in = base + kWorkBytes;
    const size_t f = al(sizeof(float) * kMaxN);
    std::vector<float> lattice(3 * (size_t)kMaxN);
    for (int i = 0; i < kMaxN; ++i) {
      lattice[i] = (float)(i & 31);
      lattice[kMaxN + i] = (float)((i >> 5) & 31);
      lattice[2 * (size_t)kMaxN + i] = (float)(i >> 10);
    }
    for (int k = 0; k < 3; ++k)
      check(cudaMemcpy(in + k * f, lattice.data() + (size_t)k * kMaxN, sizeof(float) * kMaxN,
                       cudaMemcpyHostToDevice), "set-up input copy");
    const float* sx = reinterpret_cast<const float*>(in);
    const float* sy = reinterpret_cast<const float*>(in + f);
    const float* sz = reinterpret_cast<const float*>(in + 2 * f);
    int* sl = reinterpret_cast<int*>(in + 3 * f);
    uint16_t* sa = reinterpret_cast<uint16_t*>(in + 4 * f);
    if (fof_in_scratch(base, sx, sy, sz, kMaxN, 0.5f, sl, sa) != 0)
      throw CudaError("nbody_fof_noalloc: set-up run found links in the unit lattice");
    g_addr[dev] = base;
  }
  return g_addr[dev];
}

}  // namespace
}  // namespace nb

extern "C" int nbody_fof_noalloc(const float* x, const float* y, const float* z, int n,
                                 float link_length, int* labels, uint16_t* agg_size,
                                 int* n_groups) {
  NBODY_API_BODY({
    NBODY_REQUIRE(n_groups && (n == 0 || (x && y && z && labels && agg_size)),
                  "nbody_fof_noalloc: null argument");
    NBODY_REQUIRE(n >= 0, "nbody_fof_noalloc: negative body count");
    if (n > nb::kMaxN)
      throw nb::ArgError("nbody_fof_noalloc: n = " + std::to_string(n) + " exceeds the static "
                         "scratch limit NBODY_FOF_NOALLOC_MAX_N = " + std::to_string(nb::kMaxN) +
                         "; use nbody_fof");
    *n_groups = 0;
    unsigned char* base = nb::scratch_for_current_device();  // the device's set-up, once
    *n_groups = nb::fof_in_scratch(base, x, y, z, n, link_length, labels, agg_size);
  })
}
