// kernels.cuh -- internal launch interface of the nbody-b200 CUDA library.
//
// Data layout in HBM (all SoA, Morton order unless noted):
//   body4[s]      float4 (x, y, z, m) of the s-th body in key order (16 B)
//   keys/perm     uint32 Morton key and source index per body
//   binary tree   Karras radix tree over the sorted keys: left/right/parent,
//                 [lo,hi] body range, prefix length (bits)
//   moments       FP64 tile-local prefix sums of (m, m x, m y, m z)
//   octree        compressed octree over the same keys; the children of a
//                 node are contiguous: com4 (x,y,z,m float, from FP64 sums),
//                 info int4 (first_child, body_lo, count<<4|nchild,
//                 bits of half-size), box_lo/box_hi float4 (the node's
//                 cell cube, grown by a float-rounding margin)
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace nb {

// Bodies per tile of the FP64 moment prefix sums.
constexpr int kMomentTile = 2048;

// Root cube and key quantisation, computed on the device from the bbox.
struct TreeGeom {
  float bmin[3], bmax[3];  // padded bbox: launchBBoxKernel semantics (BHTree.cu:440-446)
  float rc[3];             // root centre (BHTree.cu:481-483)
  float rhs;               // root half size (BHTree.cu:484-485)
  double lo[3];            // lower corner of the root cube
  double scale;            // 1024 / (2 rhs): cells per unit length at level 10
};

struct OctNodes {
  float4* com = nullptr;
  int4* info = nullptr;
  float4* box_lo = nullptr;
  float4* box_hi = nullptr;
};

// Scratch + outputs of one tree build for up to `cap` bodies.
struct TreeWork {
  int cap = 0;
  // sort
  uint32_t *keys = nullptr, *perm = nullptr, *keys_alt = nullptr, *perm_alt = nullptr;
  uint32_t* counts = nullptr;
  // bodies in key order
  float4* body4 = nullptr;
  // binary radix tree (internal nodes 0..n-2, leaves encoded n-1+j)
  int *bin_left = nullptr, *bin_right = nullptr;
  uint32_t* bin_pinfo = nullptr;  // per node: its parent's body count << 5 | level + 1
  int *bin_lo = nullptr, *bin_hi = nullptr;
  uint8_t* bin_prefix = nullptr;
  // FP64 moments: tile-local prefix sums of (m, m x, m y, m z), tile prefixes
  double4* mom_ploc = nullptr;
  double4* mom_tiles = nullptr;
  // octree layout
  uint8_t* oct_nch = nullptr;
  uint32_t* oct_off = nullptr;
  int* oct_node = nullptr;  // octree slot -> the binary node whose record it holds
  uint32_t* scan_tmp = nullptr;
  OctNodes oct;
  // device words
  unsigned long long* bbox_enc = nullptr;  // 6: min xyz, max xyz (ordered bits)
  TreeGeom* geom = nullptr;
  int* n_nodes = nullptr;
  int* status = nullptr;
  // warp target groups: (first body, count), maximal binary nodes <= 32 bodies
  int2* groups = nullptr;
  int* n_groups = nullptr;
  // optional (set by the caller): per group, (index of the first group cut
  // from the same span node, bodies in that node) -- the shared walk's spans
  int2* group_spans = nullptr;
  int group_max = 32;     // bodies per target group (32 x targets per lane)
  // Octree nodes with <= prune_max bodies get no child records (0: every
  // node down to single bodies).  The walk and the neighbour search open a
  // node of <= leaf_max bodies straight into its bodies, so a tree built with
  // prune_max = leaf_max gives them the same results with fewer records.
  int prune_max = 0;
  // Target groups come from maximal nodes of <= group_span x group_max
  // bodies, each cut into the fewest equal runs of <= group_max (1: the
  // maximal nodes of <= group_max bodies themselves).
  int group_span = 1;
  // Optional overlap (launch_tree): the FP64 moment prefix runs on `side`
  // while the Karras tree and the slot passes run on the caller's stream,
  // forked and joined by the two events (graph capture turns them into
  // parallel branches).  Created by tree_enable_overlap; null: one stream.
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // Host-side flag: the moment prefix of the octree build in flight runs on
  // `side` (joined through ev_join before the records are written).
  bool moments_on_side = false;
  // the emit pass writes the records' boxes (oct.box_lo / box_hi): the
  // neighbour search and the fused-collision walk read them, the plain walk
  // does not
  bool boxes = true;
};

void tree_alloc(TreeWork& w, int cap);
void tree_free(TreeWork& w);
// Creates w.side and its events (freed by tree_free).
void tree_enable_overlap(TreeWork& w);

// bbox of n positions of type T (float or double) into w.bbox_enc (reset first).
template <typename T>
void launch_bbox(TreeWork& w, const T* x, const T* y, const T* z, int n, cudaStream_t s);
void launch_bbox_reset(TreeWork& w, cudaStream_t s);
// Morton keys of n positions using w.bbox_enc; writes w.geom, keys, perm = 0..n-1.
template <typename T>
void launch_keys(TreeWork& w, const T* x, const T* y, const T* z, int n, cudaStream_t s,
                 uint32_t* hist = nullptr);
// body4[s] = (x,y,z,m)[perm[s]] for float inputs in caller order.
void launch_gather_body4(TreeWork& w, const float* x, const float* y, const float* z,
                         const float* m, int n, cudaStream_t s);
// Karras radix tree over sorted keys that use their low key_bits bits.
template <typename K>
void launch_karras(TreeWork& w, const K* keys, int n, int key_bits, cudaStream_t s);
// The binary radix tree of n sorted 32-bit keys into caller device arrays of
// n - 1 internal nodes (synchronous, allocates its own work space).
void radix_tree_u32(const uint32_t* keys, int n, int key_bits, int* left, int* right, int* lo,
                    int* hi, uint8_t* prefix);
// Octree, FP64 moments and target groups over a Karras tree whose keys carry
// a disk index in the disk_bits above the 30 Morton bits: one root slot per
// disk (slots 0..n_roots-1), geoms[d] the root cube of disk d, group_disk
// (optional) receives each group's disk.
// moments_ready: the moment prefix is already launched (on w.side when
// w.moments_on_side, joined through w.ev_join before the records are
// written; else earlier on s).
template <typename K>
void launch_octree(TreeWork& w, const K* keys, int n, int disk_bits, int n_roots,
                   const TreeGeom* geoms, int* group_disk, const double* xd, const double* yd,
                   const double* zd, cudaStream_t s, bool moments_ready = false);
// launch_karras + launch_octree, with the moment prefix on w.side when set.
// tiles_done: the caller has already written the tile-local moment prefix
// (w.mom_ploc) and the tile sums (w.mom_tiles) on s, as the engine's permute
// does; only the scan of the tile sums is left.
template <typename K>
void launch_tree(TreeWork& w, const K* keys, int n, int key_bits, int disk_bits, int n_roots,
                 const TreeGeom* geoms, int* group_disk, const double* xd, const double* yd,
                 const double* zd, cudaStream_t s, bool tiles_done = false);
// Ensembles: root cube of every disk from its encoded bbox (6 words per
// disk); bbox accumulators reset for n_disks; composite keys
// (disk << 30 | Morton) with disk[i] the body's disk.
void launch_geoms(const unsigned long long* enc, TreeGeom* geoms, int n_disks, cudaStream_t s);
void launch_bbox_reset_n(unsigned long long* enc, int n_disks, cudaStream_t s);
template <typename T>
// hist (optional, from radix_sort_prepare): the digit counts of the sort of
// the key_bits-bit keys that follows.
void launch_keys_multi(const T* x, const T* y, const T* z, const int* disk, int n,
                       const TreeGeom* geoms, uint64_t* keys, uint32_t* perm, int* status,
                       cudaStream_t s, uint32_t* hist = nullptr, int key_bits = 0);
// Single disk: Karras radix tree over w.keys.
void launch_build_topology(TreeWork& w, int n, cudaStream_t s);
// FP64 moments, compressed octree (contiguous children) and the target
// groups.  xd/yd/zd (optional, key order) give FP64 positions for the
// moments; otherwise body4 is used.
void launch_build_moments(TreeWork& w, int n, const double* xd, const double* yd,
                          const double* zd, cudaStream_t s);

// FP64 moment prefix sums only (k_moment_tiles + tile scan) over w.body4 and
// the optional key-order FP64 positions; moment_tile_prefix is where the
// tile prefixes land (the tpre argument of range_moments).
void launch_moment_prefix(TreeWork& w, int n, const double* xd, const double* yd,
                          const double* zd, cudaStream_t s);
double4* moment_tile_prefix(TreeWork& w, int n);
// Moment tiles over n bodies (blocks of the tile-local scan).
inline int moment_tiles(int n) { return n / kMomentTile + 1; }

size_t radix_sort_count_words(int n);
// Runs the sort's look-back wait against tile-status words that nothing
// publishes; returns the status bits it raised (kStatusSortWait expected).
int sort_wait_selftest();
// Stable LSD sort of (key, value) by the low `bits` bits of the keys; K is
// uint32_t (single disk, 30-bit Morton keys) or uint64_t (ensemble: disk
// index above the 30 Morton bits).
// counts: radix_sort_count_words(n) words of scratch; status (optional)
// receives kStatusSortWait if a look-back wait gave up.  hist_ready: the
// digit histograms at the start of counts were cleared by radix_sort_prepare
// and filled by the kernel that wrote the keys (launch_keys with hist).
template <typename K>
void radix_sort_pairs(K* keys, uint32_t* vals, K* keys_alt, uint32_t* vals_alt,
                      uint32_t* counts, int n, int bits, cudaStream_t s, int* status = nullptr,
                      bool hist_ready = false);
// Clears the histograms and tickets at the start of counts; returns the
// histograms (passes x 256 words) for a key kernel to fill.
uint32_t* radix_sort_prepare(uint32_t* counts, int bits, cudaStream_t s);
size_t scan_tmp_words(int n);
void scan_exclusive_u32(uint32_t* data, int n, uint32_t* tmp, cudaStream_t s);
// Words of TreeWork::scan_tmp the octree build uses for nb binary nodes
// (one 64-bit count sum per tile of 256 nodes).
size_t octree_scan_words(int nb);

// ------------------------------------------------------------------ walk
// Walk variant used unless a caller picks one (walk.cu lists the variants).
constexpr int kDefaultWalkMode = 1;
// Target groups cut from maximal nodes of <= 8 x 32 bodies (TreeWork::
// group_span): at N = 2^20 warps hold 29 targets on average instead of 22
// and the walk takes 0.49 ms instead of 0.55 ms.  Below ~2^19 bodies the
// fewer groups no longer fill the GPU's warp slots (N = 65536: walk 0.074 ->
// 0.093 ms, collisions 0.033 -> 0.060 ms), so the automatic choice keeps
// span 1 there.
constexpr int kDefaultGroupSpan = 8;
constexpr int kGroupSpanMinBodies = 1 << 19;
// Default leaf size (bodies a walk takes directly instead of opening the
// node): 12 from 2^19 bodies on (the step at N = 2^20 takes 0.602 ms against
// 0.608 ms with 8: fewer nodes to build and visit outweigh 3% more
// interactions), else 8.
constexpr int kLeafMaxLarge = 12;
constexpr int kLeafMaxSmall = 8;
inline int default_leaf_max(int n) {
  return n >= kGroupSpanMinBodies ? kLeafMaxLarge : kLeafMaxSmall;
}

struct WalkArgs {
  const float4* com;
  const int4* info;
  const float4* body;
  int n;
  const int2* groups;     // target groups (first body, count <= 32)
  const int* n_groups;    // device count of groups
  float theta2;           // theta^2
  float eps;              // softening
  float star_mass;
  int star_in_walk;       // 1: add the softened star pull in FP32 (reference form)
  int leaf_max;           // nodes with <= leaf_max bodies are opened into bodies
  const float4* pert;     // (px, py, pz, m) of the perturber, or nullptr
  float* ax;
  float* ay;
  float* az;
  const uint32_t* scatter;  // output index map (caller order), or nullptr
  int* spill;
  int spill_cap;
  unsigned long long* inter;  // accepted interactions (sources x targets)
  unsigned long long* counters;  // optional: nodes visited, stack spills, groups
  int* work;
  int* status;
  int targets_per_lane;   // 1 or 2: groups of up to 32 or 64 bodies
  int walk_mode;          // 0, 1, 2: see walk.cu (targets_per_lane 1 only)
  bool counters_zeroed;   // work, inter and counters already zero (no reset launch)
  // ensembles: a group's walk starts at its disk's root slot, and pert holds
  // n_disks perturbers per force evaluation, the current one at *pert_step
  const int* group_disk;  // nullptr: one disk
  int n_disks;
  const int* pert_step;   // nullptr: pert points at the current entries
  // recording walks (tape != nullptr; targets_per_lane must be 1): every
  // group's source list as (first body, count) entries in evaluation order,
  // in chains of 32-entry chunks: tape[c*32 ..], tape_next[c] the next chunk
  // (-1 ends), group_tape[g] = (first chunk, entries) or (-1, 0)
  int2* tape;
  int* tape_next;
  int* tape_used;         // chunks taken (reset to 0 before the walk)
  int tape_cap;           // chunks in the pool
  int2* group_tape;
  // fused collisions (coll_dv[0] != nullptr; targets_per_lane 1, no tape):
  // every target also gets the two-pass collision impulse of the bodies
  // closer than coll_r, found in its own source list (walk.cu).  dv is in
  // the bodies' (key) order; velocities in the state's storage type.
  const void* coll_v[3];
  int coll_vtype;         // 0 float, 1 double, 2 hi/lo float pairs
  float coll_r;
  float coll_e;
  float* coll_dv[3];
  const float4* box_lo;   // node boxes (the octree's), for the reach test
  const float4* box_hi;
  // shared walk (span_lists != nullptr; single disk, targets_per_lane 1, no
  // tape, no fused collisions): each group starts from its span's shared
  // sources and frontier (launch_span_walk) instead of the root
  const int2* group_span;
  const int4* span_lists;  // at a span's first group: (shared head, shared
                           // count, frontier head, frontier count); count -1:
                           // no lists, walk from the root
  const int* span_pool;    // chunks of 32 entries
  const int* span_next;    // next chunk (-1 ends)
};
int walk_spill_slots(int device);  // warps resident at once (spill area slots)
void launch_walk(const WalkArgs& a, cudaStream_t s);

// The first, shared traversal of the shared walk: one warp per span node.
struct SpanArgs {
  const float4* com;
  const int4* info;
  const float4* body;
  const int2* groups;
  const int2* group_span;
  const int* n_groups;
  float theta2;
  int leaf_max;
  int4* span_lists;
  int* pool;
  int* next;
  int* used;               // chunks taken (reset to 0 before the launch)
  int cap;                 // chunks in the pool
  int* work;               // span counter (reset to 0 before the launch)
  unsigned long long* counters;  // optional: shared entries, frontier entries, spans
};
void launch_span_walk(const SpanArgs& a, int n, cudaStream_t s);

// ------------------------------------------------------------ collisions
struct NeighborArgs {
  const int4* info;
  const float4* box_lo;
  const float4* box_hi;
  const float4* body;
  int n;
  const int2* groups;
  const int* n_groups;
  int leaf_max;
  int* spill;
  int spill_cap;
  int* work;
  int* status;
  const int* group_disk;  // nullptr: one disk (root slot 0)
};
// Two-pass impulse (BHTree.cu:620-686): dv[s] for body s in key order.
// v* are velocities in key order, or in caller order when vmap != nullptr
// (v[vmap[j]] is body j's velocity).
void launch_collide(const NeighborArgs& a, const float* vx, const float* vy, const float* vz,
                    const uint32_t* vmap, float r_coll, float restitution, float* dvx,
                    float* dvy, float* dvz, cudaStream_t s);
// Collision pairs of the octree's bodies (report[0], ordered pairs i, j != i
// closer than r_coll) and how many of them the reference's cell prune would
// skip (report[1]); the tree must hold every node (prune_max 0).
void launch_collision_report(const NeighborArgs& a, const float4* com, float r_coll,
                             unsigned long long* report, cudaStream_t s);
// The same with velocities in the state's storage type: vtype 0 float,
// 1 double, 2 hi/lo float pairs (converted to float as they are read).
void launch_collide_v(const NeighborArgs& a, const void* vx, const void* vy, const void* vz,
                      int vtype, const uint32_t* vmap, float r_coll, float restitution,
                      float* dvx, float* dvy, float* dvz, cudaStream_t s);
// FoF links (Aggregate.cpp:36-42 test) -> union-find over original ids.
void launch_fof_link(const NeighborArgs& a, const uint32_t* ids, float link_length,
                     int* parent, cudaStream_t s);
void launch_fof_finish(int* parent, int n, int* labels, int* sizes, uint16_t* agg_size,
                       int* n_groups, int* status, cudaStream_t s);
// launch_fof_link with at most max_warps warps (spill slots) in flight.
void launch_fof_link_capped(const NeighborArgs& a, const uint32_t* ids, float link_length,
                            int* parent, int max_warps, cudaStream_t s);

// -------------------------------------------------------- streaming (compat)
void launch_half_kick(float* vx, float* vy, float* vz, const float* ax, const float* ay,
                      const float* az, float dt_half, int n, cudaStream_t s);
void launch_drift(float* x, float* y, float* z, const float* vx, const float* vy,
                  const float* vz, float dt, int n, cudaStream_t s);
void launch_reset_acc(float* ax, float* ay, float* az, int n, cudaStream_t s);
void launch_gas_drag(const float* x, const float* y, const float* z, float* vx, float* vy,
                     float* vz, float decay, float star_mass, int n, cudaStream_t s);
void launch_perturber_force(float* ax, float* ay, float* az, const float* x, const float* y,
                            const float* z, float px, float py, float pz, float pmass,
                            float eps, int n, cudaStream_t s);
void launch_apply_dv(float* vx, float* vy, float* vz, const float* dvx, const float* dvy,
                     const float* dvz, const uint32_t* map, int n, cudaStream_t s);
void launch_copy_perm(int* dst, const uint32_t* perm, int n, cudaStream_t s);

}  // namespace nb
