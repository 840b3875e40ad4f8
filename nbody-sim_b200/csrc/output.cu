// output.cu -- the output step of src/main.cu:143-181 on the GPU, overlapped
// with the steps that follow it.
//
// The reference stops the loop every output_every steps, copies all eleven
// arrays to the host (main.cu:144), runs detectAggregates (an O(N^2) host
// loop, Aggregate.cpp:26-76), fills agg_size (main.cu:153-161) and writes.
// Here an output is:
//   engine stream : snapshot of x..vz in caller order (float) -> event
//   side stream   : octree of the snapshot, FoF (the Aggregate.cpp:36-42 pair
//                   test, union-find with smallest-index roots), agg_size,
//                   aggregate records, D2H of x, y, z, agg_size and the
//                   record count into pinned host memory -> event
//   host (wait)   : the records themselves (count known by then)
// The engine keeps stepping while the side stream works.  Two slots, so one
// frame can be in flight while the host writes the previous one.
//
// Aggregate records match Aggregate.cpp:54-74 bit for bit: groups of >= 2
// ordered by smallest member, mass = n * particle mass, FP32 position and
// velocity sums in ascending member index, times 1/n, dist_center =
// sqrt(cx^2 + cy^2 + cz^2) without contraction.  The members of each group
// come out of a stable sort of (label, index), so one thread per group sums
// them in index order.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "capi_util.h"
#include "common.cuh"
#include "kernels.cuh"
#include "output.h"

namespace nb {
namespace {

constexpr int kThreads = 256;

int grid1(long long n) { return std::max(1, std::min(div_up(n, kThreads), 148 * 8)); }

template <typename T>
T* dalloc(size_t count, const char* what) {
  T* p = nullptr;
  check(cudaMalloc(&p, sizeof(T) * (count ? count : 1)), what);
  return p;
}

__global__ void k_label_pairs(const int* __restrict__ labels, int n, uint32_t* __restrict__ keys,
                              uint32_t* __restrict__ vals) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    keys[i] = (uint32_t)labels[i];
    vals[i] = (uint32_t)i;
  }
}

// flag[s] = 1 where a group of >= 2 members starts in the sorted order.
__global__ void k_group_heads(const uint32_t* __restrict__ keys, const int* __restrict__ sizes,
                              int n, uint32_t* __restrict__ flag) {
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
       s += (long long)gridDim.x * blockDim.x) {
    const uint32_t k = keys[s];
    const bool head = (s == 0) || keys[s - 1] != k;
    flag[s] = (head && sizes[k] >= 2) ? 1u : 0u;
  }
}

__global__ void k_group_records(const uint32_t* __restrict__ keys,
                                const uint32_t* __restrict__ vals,
                                const int* __restrict__ sizes, const uint32_t* __restrict__ flag,
                                const uint32_t* __restrict__ slot, int n,
                                const float* __restrict__ x, const float* __restrict__ y,
                                const float* __restrict__ z, const float* __restrict__ vx,
                                const float* __restrict__ vy, const float* __restrict__ vz,
                                float particle_mass, nbody_aggregate* __restrict__ out,
                                int* __restrict__ count) {
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n;
       s += (long long)gridDim.x * blockDim.x) {
    if (s == n - 1) *count = (int)(slot[s] + flag[s]);
    if (!flag[s]) continue;
    const uint32_t label = keys[s];
    const int cnt = sizes[label];
    float cx = 0.f, cy = 0.f, cz = 0.f, ux = 0.f, uy = 0.f, uz = 0.f;
    for (int k = 0; k < cnt; ++k) {  // ascending member index (stable sort)
      const uint32_t i = vals[s + k];
      cx = __fadd_rn(cx, x[i]); cy = __fadd_rn(cy, y[i]); cz = __fadd_rn(cz, z[i]);
      ux = __fadd_rn(ux, vx[i]); uy = __fadd_rn(uy, vy[i]); uz = __fadd_rn(uz, vz[i]);
    }
    const float inv = 1.0f / (float)cnt;
    nbody_aggregate a;
    a.id = (int)slot[s];
    a.n_particles = cnt;
    a.mass_msun = __fmul_rn((float)cnt, particle_mass);
    a.cx = __fmul_rn(cx, inv); a.cy = __fmul_rn(cy, inv); a.cz = __fmul_rn(cz, inv);
    a.vx = __fmul_rn(ux, inv); a.vy = __fmul_rn(uy, inv); a.vz = __fmul_rn(uz, inv);
    a.dist_center = sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(a.cx, a.cx), __fmul_rn(a.cy, a.cy)),
                                    __fmul_rn(a.cz, a.cz)));
    a.first_member = (int)label;
    out[slot[s]] = a;
  }
}

int bits_for(int n) {
  int b = 1;
  while (b < 32 && (1ll << b) < (long long)n) ++b;
  return b;
}

}  // namespace

OutputPipe::OutputPipe(int nn, int leaf_max_) : n(nn), leaf_max(leaf_max_) {
  check(cudaStreamCreateWithFlags(&os, cudaStreamNonBlocking), "output stream");
  tree_alloc(tw, n);
  tw.group_max = 32;
  tw.prune_max = leaf_max;
  parent = dalloc<int>(n, "output parent");
  labels = dalloc<int>(n, "output labels");
  sizes = dalloc<int>(n, "output sizes");
  agg = dalloc<uint16_t>(n, "output agg_size");
  ngroups = dalloc<int>(1, "output groups");
  spill = dalloc<int>((size_t)walk_spill_slots(0) * spill_cap, "output spill");
  work = dalloc<int>(1, "output work");
  keys = dalloc<uint32_t>(n, "aggregate keys");
  vals = dalloc<uint32_t>(n, "aggregate vals");
  keys_alt = dalloc<uint32_t>(n, "aggregate keys alt");
  vals_alt = dalloc<uint32_t>(n, "aggregate vals alt");
  flag = dalloc<uint32_t>(n, "aggregate heads");
  slotix = dalloc<uint32_t>(n, "aggregate slots");
  scan_tmp = dalloc<uint32_t>(scan_tmp_words(n), "aggregate scan");
  const size_t max_aggs = (size_t)n / 2 + 1;
  for (auto& sl : slot) {
    for (int k = 0; k < 6; ++k) sl.snap[k] = dalloc<float>(n, "snapshot");
    sl.drec = dalloc<nbody_aggregate>(max_aggs, "aggregate records");
    sl.dcount = dalloc<int>(1, "aggregate count");
    check(cudaMallocHost(&sl.hx, sizeof(float) * 3 * (size_t)n), "pinned frame");
    check(cudaMallocHost(&sl.hagg, sizeof(uint16_t) * (size_t)n), "pinned agg_size");
    check(cudaMallocHost(&sl.hrec, sizeof(nbody_aggregate) * max_aggs), "pinned aggregates");
    check(cudaMallocHost(&sl.hcount, sizeof(int)), "pinned count");
    check(cudaMallocHost(&sl.hstatus, sizeof(int)), "pinned status");
    check(cudaEventCreateWithFlags(&sl.snap_ready, cudaEventDisableTiming), "event");
    check(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming), "event");
  }
}

OutputPipe::~OutputPipe() {
  if (os) cudaStreamSynchronize(os);
  void* ptrs[] = {parent, labels, sizes, agg, ngroups, spill, work, keys, vals, keys_alt,
                  vals_alt, flag, slotix, scan_tmp};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  for (auto& sl : slot) {
    for (int k = 0; k < 6; ++k) cudaFree(sl.snap[k]);
    cudaFree(sl.drec);
    cudaFree(sl.dcount);
    cudaFreeHost(sl.hx);
    cudaFreeHost(sl.hagg);
    cudaFreeHost(sl.hrec);
    cudaFreeHost(sl.hcount);
    cudaFreeHost(sl.hstatus);
    cudaEventDestroy(sl.snap_ready);
    cudaEventDestroy(sl.done);
  }
  tree_free(tw);
  if (os) cudaStreamDestroy(os);
}

// Side-stream work of one frame whose snapshot is (or will be) in sl.snap.
void OutputPipe::enqueue(Slot& sl, float link_length, float particle_mass) {
  const float *x = sl.snap[0], *y = sl.snap[1], *z = sl.snap[2];
  check(cudaMemsetAsync(tw.status, 0, sizeof(int), os), "output status reset");
  // octree of the snapshot
  launch_bbox<float>(tw, x, y, z, n, os);
  launch_keys<float>(tw, x, y, z, n, os);
  radix_sort_pairs(tw.keys, tw.perm, tw.keys_alt, tw.perm_alt, tw.counts, n, 30, os,
                   tw.status);
  launch_gather_body4(tw, x, y, z, nullptr, n, os);
  launch_build_topology(tw, n, os);
  launch_build_moments(tw, n, nullptr, nullptr, nullptr, os);
  // FoF: labels (smallest member index) and agg_size by caller index
  NeighborArgs na{tw.oct.info, tw.oct.box_lo, tw.oct.box_hi, tw.body4, n, tw.groups,
                  tw.n_groups, leaf_max, spill, spill_cap, work, tw.status, nullptr};
  launch_fof_link(na, tw.perm, link_length, parent, os);
  launch_fof_finish(parent, n, labels, sizes, agg, ngroups, tw.status, os);
  // aggregate records
  k_label_pairs<<<grid1(n), kThreads, 0, os>>>(labels, n, keys, vals);
  radix_sort_pairs(keys, vals, keys_alt, vals_alt, tw.counts, n, bits_for(n), os, tw.status);
  k_group_heads<<<grid1(n), kThreads, 0, os>>>(keys, sizes, n, flag);
  check(cudaMemcpyAsync(slotix, flag, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, os),
        "aggregate slots");
  scan_exclusive_u32(slotix, n, scan_tmp, os);
  k_group_records<<<grid1(n), kThreads, 0, os>>>(keys, vals, sizes, flag, slotix, n, x, y, z,
                                                 sl.snap[3], sl.snap[4], sl.snap[5],
                                                 particle_mass, sl.drec, sl.dcount);
  check(cudaGetLastError(), "aggregate launch");
  // to the host
  for (int k = 0; k < 3; ++k)
    check(cudaMemcpyAsync(sl.hx + (size_t)k * n, sl.snap[k], sizeof(float) * n,
                          cudaMemcpyDeviceToHost, os), "frame D2H");
  check(cudaMemcpyAsync(sl.hagg, agg, sizeof(uint16_t) * n, cudaMemcpyDeviceToHost, os),
        "agg_size D2H");
  check(cudaMemcpyAsync(sl.hcount, sl.dcount, sizeof(int), cudaMemcpyDeviceToHost, os),
        "aggregate count D2H");
  check(cudaMemcpyAsync(sl.hstatus, tw.status, sizeof(int), cudaMemcpyDeviceToHost, os),
        "output status D2H");
  check(cudaEventRecord(sl.done, os), "output done");
}

int OutputPipe::begin_slot() {
  Slot& sl = slot[next];
  if (sl.pending)
    throw ArgError("nbody_sim_output_begin: both frames are in flight; call nbody_sim_output_wait",
                   NBODY_ERR_STATE);
  return next;
}

void OutputPipe::launch(int k, cudaStream_t engine, float link_length, float particle_mass,
                        float sim_time, int frame_index) {
  Slot& sl = slot[k];
  check(cudaEventRecord(sl.snap_ready, engine), "snapshot ready");
  check(cudaStreamWaitEvent(os, sl.snap_ready, 0), "output wait");
  enqueue(sl, link_length, particle_mass);
  sl.pending = true;
  sl.time = sim_time;
  sl.frame = frame_index;
  sl.seq = seq++;
  next ^= 1;
}

void OutputPipe::wait(nbody_frame* out) {
  int k = -1;
  for (int i = 0; i < 2; ++i)
    if (slot[i].pending && (k < 0 || slot[i].seq < slot[k].seq)) k = i;
  if (k < 0) throw ArgError("nbody_sim_output_wait: no frame in flight", NBODY_ERR_STATE);
  Slot& sl = slot[k];
  check(cudaEventSynchronize(sl.done), "output sync");
  const int s = *sl.hstatus;
  sl.pending = false;
  if (s)
    throw ArgError("nbody_sim_output_wait: device status " + std::to_string(s),
                   NBODY_ERR_OVERFLOW);
  out->n = n;
  out->frame_index = sl.frame;
  out->sim_time = sl.time;
  out->x = sl.hx;
  out->y = sl.hx + n;
  out->z = sl.hx + 2 * (size_t)n;
  out->agg_size = sl.hagg;
  const int na = *sl.hcount;
  if (na > 0)  // the slot's device records stay put until the slot is reused
    check(cudaMemcpy(sl.hrec, sl.drec, sizeof(nbody_aggregate) * (size_t)na,
                     cudaMemcpyDeviceToHost), "aggregates D2H");
  out->aggregates = sl.hrec;
  out->n_aggregates = na;
}

}  // namespace nb
