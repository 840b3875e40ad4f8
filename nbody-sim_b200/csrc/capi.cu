// capi.cu -- extern "C" phase API: the reference's BHTree.cuh, Integrator.cuh
// and Perturber.h launchers (and a device FoF) over the nbody-b200 kernels.
// Each call runs on the legacy default stream and synchronises it before
// returning, as every reference launcher does (cudaDeviceSynchronize after
// each launch, e.g. BHTree.cu:407-408, Integrator.cu:83-84).
#include <cmath>
#include <cstring>
#include <string>

#include "capi_util.h"
#include "common.cuh"
#include "kernels.cuh"

namespace nb {

thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }

namespace {
template <typename T>
T* dalloc(size_t count, const char* what) {
  T* p = nullptr;
  check(cudaMalloc(&p, sizeof(T) * (count ? count : 1)), what);
  return p;
}

void finish(const char* what) {
  check(cudaGetLastError(), what);
  check(cudaStreamSynchronize(0), what);
}

void check_particles(const nbody_particles* p, int n, bool need_v, bool need_a) {
  NBODY_REQUIRE(p, "null particle struct");
  NBODY_REQUIRE(p->n == n, "particle count " + std::to_string(p->n) +
                               " does not match the tree's " + std::to_string(n));
  NBODY_REQUIRE(p->x && p->y && p->z, "null position array");
  if (need_v) NBODY_REQUIRE(p->vx && p->vy && p->vz, "null velocity array");
  if (need_a) NBODY_REQUIRE(p->ax && p->ay && p->az, "null acceleration array");
}
}  // namespace
}  // namespace nb

struct nbody_tree {
  int n = 0;
  int leaf_max = 8;
  nb::TreeWork tw;
  int* sort_idx = nullptr;
  float *dvx = nullptr, *dvy = nullptr, *dvz = nullptr;
  int* spill = nullptr;
  int spill_cap = 4096;
  int* work = nullptr;
  unsigned long long* inter = nullptr;
  unsigned long long* counters = nullptr;
  int* parent = nullptr;
  int* sizes = nullptr;
  int* ngroups = nullptr;
  bool have_bbox = false, built = false, summarized = false;

  void throw_status(const char* what) {
    int st = 0;
    nb::check(cudaMemcpy(&st, tw.status, sizeof(int), cudaMemcpyDeviceToHost), "status read");
    if (st) {
      nb::check(cudaMemset(tw.status, 0, sizeof(int)), "status reset");
      throw nb::ArgError(std::string(what) + ": device status " + std::to_string(st) +
                             " (1 walk stack, 2 union-find, 4 tree, 8 non-finite position)",
                         NBODY_ERR_OVERFLOW);
    }
  }
};

extern "C" {

const char* nbody_last_error(void) { return nb::g_last_error.c_str(); }
int nbody_abi_version(void) { return NBODY_ABI_VERSION; }

int nbody_tree_create(int n_bodies, nbody_tree** out) {
  NBODY_API_BODY({
    NBODY_REQUIRE(out, "nbody_tree_create: null out");
    NBODY_REQUIRE(n_bodies > 0 && n_bodies < (1 << 27), "nbody_tree_create: n must be in [1, 2^27)");
    *out = nullptr;
    nbody_tree* t = new nbody_tree();
    try {
      t->n = n_bodies;
      nb::tree_alloc(t->tw, n_bodies);
      t->tw.group_max = 32;
      t->sort_idx = nb::dalloc<int>(n_bodies, "sort_idx");
      nb::check(cudaMemset(t->sort_idx, 0, sizeof(int) * n_bodies), "sort_idx init");
      t->dvx = nb::dalloc<float>(n_bodies, "dvx");
      t->dvy = nb::dalloc<float>(n_bodies, "dvy");
      t->dvz = nb::dalloc<float>(n_bodies, "dvz");
      t->spill = nb::dalloc<int>((size_t)nb::walk_spill_slots(0) * t->spill_cap, "spill");
      t->work = nb::dalloc<int>(1, "work");
      t->inter = nb::dalloc<unsigned long long>(1, "inter");
      t->counters = nb::dalloc<unsigned long long>(3, "walk counters");
      t->parent = nb::dalloc<int>(n_bodies, "fof parent");
      t->sizes = nb::dalloc<int>(n_bodies, "fof sizes");
      t->ngroups = nb::dalloc<int>(1, "fof groups");
      nb::check(cudaMemset(t->inter, 0, sizeof(unsigned long long)), "inter init");
    } catch (...) {
      nbody_tree_destroy(t);
      throw;
    }
    *out = t;
  })
}

void nbody_tree_destroy(nbody_tree* t) {
  if (!t) return;
  cudaStreamSynchronize(0);
  nb::tree_free(t->tw);
  void* ptrs[] = {t->sort_idx, t->dvx, t->dvy, t->dvz, t->spill, t->work,
                  t->inter, t->counters, t->parent, t->sizes, t->ngroups};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  delete t;
}

int nbody_tree_reset(nbody_tree* t) {
  NBODY_API_BODY({
    NBODY_REQUIRE(t, "nbody_tree_reset: null tree");
    nb::check(cudaMemset(t->tw.status, 0, sizeof(int)), "status reset");
    t->have_bbox = t->built = t->summarized = false;
  })
}

int nbody_tree_set_leaf_max(nbody_tree* t, int leaf_max) {
  NBODY_API_BODY({
    NBODY_REQUIRE(t && leaf_max >= 1 && leaf_max <= (1 << 20), "nbody_tree_set_leaf_max: bad value");
    t->leaf_max = leaf_max;
  })
}

int nbody_tree_set_targets_per_lane(nbody_tree* t, int k) {
  NBODY_API_BODY({
    NBODY_REQUIRE(t && (k == 1 || k == 2), "nbody_tree_set_targets_per_lane: 1 or 2");
    t->tw.group_max = 32 * k;
  })
}

int nbody_tree_bbox(nbody_tree* t, const nbody_particles* p) {
  NBODY_API_BODY({
    NBODY_REQUIRE(t, "nbody_tree_bbox: null tree");
    nb::check_particles(p, t->n, false, false);
    nb::launch_bbox<float>(t->tw, p->x, p->y, p->z, t->n, 0);
    nb::finish("launchBBoxKernel");
    t->have_bbox = true;
    t->built = t->summarized = false;
  })
}

int nbody_tree_build(nbody_tree* t, const nbody_particles* p) {
  NBODY_API_BODY({
    NBODY_REQUIRE(t, "nbody_tree_build: null tree");
    nb::check_particles(p, t->n, false, false);
    NBODY_REQUIRE(p->mass, "nbody_tree_build: null mass array");
    if (!t->have_bbox) nb::launch_bbox<float>(t->tw, p->x, p->y, p->z, t->n, 0);
    nb::launch_keys<float>(t->tw, p->x, p->y, p->z, t->n, 0);
    nb::radix_sort_pairs(t->tw.keys, t->tw.perm, t->tw.keys_alt, t->tw.perm_alt, t->tw.counts,
                         t->n, 30, 0, t->tw.status);
    nb::launch_gather_body4(t->tw, p->x, p->y, p->z, p->mass, t->n, 0);
    nb::launch_build_topology(t->tw, t->n, 0);
    nb::finish("launchBuildKernel");
    t->have_bbox = false;
    t->built = true;
    t->summarized = false;
    t->throw_status("launchBuildKernel");
  })
}

int nbody_tree_summarize(nbody_tree* t) {
  NBODY_API_BODY({
    NBODY_REQUIRE(t, "nbody_tree_summarize: null tree");
    if (!t->built) throw nb::ArgError("nbody_tree_summarize: tree not built", NBODY_ERR_STATE);
    nb::launch_build_moments(t->tw, t->n, nullptr, nullptr, nullptr, 0);
    nb::finish("launchSummarizeKernel");
    t->summarized = true;
    t->throw_status("launchSummarizeKernel");
  })
}

int nbody_tree_sort(nbody_tree* t) {
  NBODY_API_BODY({
    NBODY_REQUIRE(t, "nbody_tree_sort: null tree");
    if (!t->built) throw nb::ArgError("nbody_tree_sort: tree not built", NBODY_ERR_STATE);
    nb::launch_copy_perm(t->sort_idx, t->tw.perm, t->n, 0);
    nb::finish("launchSortKernel");
  })
}

int* nbody_tree_sort_idx(nbody_tree* t) { return t ? t->sort_idx : nullptr; }

int nbody_tree_sort_idx_copy(nbody_tree* t, int* dst, int dst_on_device) {
  NBODY_API_BODY({
    NBODY_REQUIRE(t && dst, "nbody_tree_sort_idx_copy: null argument");
    nb::check(cudaMemcpy(dst, t->sort_idx, sizeof(int) * t->n,
                         dst_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost),
              "sort_idx copy");
  })
}

int nbody_tree_force(nbody_tree* t, nbody_particles* p, float theta, float softening,
                     float star_mass) {
  NBODY_API_BODY({
    NBODY_REQUIRE(t, "nbody_tree_force: null tree");
    nb::check_particles(p, t->n, false, true);
    if (!t->summarized) throw nb::ArgError("nbody_tree_force: tree not summarized", NBODY_ERR_STATE);
    nb::check(cudaMemset(t->inter, 0, sizeof(unsigned long long)), "inter reset");
    nb::check(cudaMemset(t->counters, 0, 3 * sizeof(unsigned long long)), "counters reset");
    nb::WalkArgs w{};
    w.com = t->tw.oct.com; w.info = t->tw.oct.info; w.body = t->tw.body4; w.n = t->n;
    w.groups = t->tw.groups; w.n_groups = t->tw.n_groups;
    w.theta2 = theta * theta; w.eps = softening; w.star_mass = star_mass; w.star_in_walk = 1;
    w.leaf_max = t->leaf_max; w.pert = nullptr;
    w.ax = p->ax; w.ay = p->ay; w.az = p->az; w.scatter = t->tw.perm;
    w.spill = t->spill; w.spill_cap = t->spill_cap; w.inter = t->inter; w.work = t->work;
    w.counters = t->counters;
    w.status = t->tw.status; w.targets_per_lane = t->tw.group_max / 32;
    w.walk_mode = nb::kDefaultWalkMode;
    nb::launch_walk(w, 0);
    nb::finish("launchForceKernel");
    t->throw_status("launchForceKernel");
  })
}

int nbody_tree_collide(nbody_tree* t, nbody_particles* p, float r_coll, float restitution) {
  NBODY_API_BODY({
    NBODY_REQUIRE(t, "nbody_tree_collide: null tree");
    nb::check_particles(p, t->n, true, false);
    if (!t->summarized) throw nb::ArgError("nbody_tree_collide: tree not summarized", NBODY_ERR_STATE);
    nb::NeighborArgs na{t->tw.oct.info, t->tw.oct.box_lo, t->tw.oct.box_hi, t->tw.body4, t->n,
                        t->tw.groups, t->tw.n_groups, t->leaf_max, t->spill, t->spill_cap, t->work, t->tw.status};
    nb::launch_collide(na, p->vx, p->vy, p->vz, t->tw.perm, r_coll, restitution, t->dvx, t->dvy,
                       t->dvz, 0);
    nb::launch_apply_dv(p->vx, p->vy, p->vz, t->dvx, t->dvy, t->dvz, t->tw.perm, t->n, 0);
    nb::finish("launchCollisionKernel");
    t->throw_status("launchCollisionKernel");
  })
}

int nbody_tree_collision_report(nbody_tree* t, float r_coll, unsigned long long* pairs,
                                unsigned long long* missed) {
  NBODY_API_BODY({
    NBODY_REQUIRE(t && pairs && missed, "nbody_tree_collision_report: null argument");
    NBODY_REQUIRE(r_coll >= 0.f, "nbody_tree_collision_report: negative radius");
    if (!t->summarized)
      throw nb::ArgError("nbody_tree_collision_report: tree not summarized", NBODY_ERR_STATE);
    *pairs = 0;
    *missed = 0;
    if (t->n < 2 || r_coll == 0.f) return NBODY_OK;
    unsigned long long* rep = nullptr;
    nb::check(cudaMalloc(&rep, 2 * sizeof(unsigned long long)), "report counters");
    unsigned long long h[2] = {0, 0};
    try {
      nb::NeighborArgs na{t->tw.oct.info, t->tw.oct.box_lo, t->tw.oct.box_hi, t->tw.body4, t->n,
                          t->tw.groups, t->tw.n_groups, t->leaf_max, t->spill, t->spill_cap,
                          t->work, t->tw.status};
      nb::launch_collision_report(na, t->tw.oct.com, r_coll, rep, 0);
      nb::check(cudaMemcpy(h, rep, sizeof(h), cudaMemcpyDeviceToHost), "report read");
    } catch (...) {
      cudaFree(rep);
      throw;
    }
    cudaFree(rep);
    t->throw_status("nbody_tree_collision_report");
    *pairs = h[0];
    *missed = h[1];
  })
}

int nbody_tree_stats_get(nbody_tree* t, nbody_tree_stats* out) {
  NBODY_API_BODY({
    NBODY_REQUIRE(t && out, "nbody_tree_stats_get: null argument");
    std::memset(out, 0, sizeof(*out));
    nb::check(cudaStreamSynchronize(0), "stats sync");
    out->n_bodies = t->n;
    unsigned long long enc[6];
    nb::check(cudaMemcpy(enc, t->tw.bbox_enc, sizeof(enc), cudaMemcpyDeviceToHost), "bbox read");
    // padding of launchBBoxKernel (BHTree.cu:440-446) and root of :481-485
    float bmin[3], bmax[3];
    for (int k = 0; k < 3; ++k) {
      double lo = nb::from_ordered_bits(enc[k]), hi = nb::from_ordered_bits(enc[3 + k]);
      if (!(lo <= hi)) lo = hi = 0.0;
      float flo = (float)lo, fhi = (float)hi;
      if ((double)flo > lo) flo = std::nextafter(flo, -INFINITY);
      if ((double)fhi < hi) fhi = std::nextafter(fhi, INFINITY);
      volatile float mid = (flo + fhi) * 0.5f;
      volatile float half = (fhi - flo) * 0.5f;
      half = half * 1.001f;
      bmin[k] = mid - half;
      bmax[k] = mid + half;
      out->bbox_min[k] = bmin[k];
      out->bbox_max[k] = bmax[k];
      out->root_center[k] = (bmin[k] + bmax[k]) * 0.5f;
    }
    volatile float ext = std::fmax(std::fmax(bmax[0] - bmin[0], bmax[1] - bmin[1]), bmax[2] - bmin[2]);
    volatile float h = ext * 0.5f;
    out->root_half = h * 1.001f;
    nb::check(cudaMemcpy(&out->n_nodes, t->tw.n_nodes, sizeof(int), cudaMemcpyDeviceToHost),
              "n_nodes read");
    if (t->n >= 2) {
      // total of the FP64 moment prefix sums (tile prefixes, last entry)
      const int ntiles = t->n / nb::kMomentTile + 1;
      double4 s;
      nb::check(cudaMemcpy(&s, t->tw.mom_tiles + (ntiles + 1) + ntiles, sizeof(double4),
                           cudaMemcpyDeviceToHost), "root read");
      out->root_mass = s.x;
      if (s.x > 0) {
        out->root_com[0] = s.y / s.x; out->root_com[1] = s.z / s.x; out->root_com[2] = s.w / s.x;
      }
    } else {
      float4 b;
      nb::check(cudaMemcpy(&b, t->tw.body4, sizeof(float4), cudaMemcpyDeviceToHost), "root read");
      out->root_mass = b.w;
      out->root_com[0] = b.x; out->root_com[1] = b.y; out->root_com[2] = b.z;
    }
    nb::check(cudaMemcpy(&out->interactions, t->inter, sizeof(unsigned long long),
                         cudaMemcpyDeviceToHost), "interactions read");
    nb::check(cudaMemcpy(&out->status, t->tw.status, sizeof(int), cudaMemcpyDeviceToHost),
              "status read");
    unsigned long long c[3];
    nb::check(cudaMemcpy(c, t->counters, sizeof(c), cudaMemcpyDeviceToHost), "counters read");
    out->walk_nodes_visited = c[0];
    out->walk_stack_spills = c[1];
  })
}

int nbody_half_kick(nbody_particles* p, float dt_half) {
  NBODY_API_BODY({
    NBODY_REQUIRE(p && p->n >= 0 && p->vx && p->vy && p->vz && p->ax && p->ay && p->az,
                  "nbody_half_kick: null array");
    nb::launch_half_kick(p->vx, p->vy, p->vz, p->ax, p->ay, p->az, dt_half, p->n, 0);
    nb::finish("integrator_halfKickKernel");
  })
}

int nbody_drift(nbody_particles* p, float dt) {
  NBODY_API_BODY({
    NBODY_REQUIRE(p && p->n >= 0 && p->x && p->y && p->z && p->vx && p->vy && p->vz,
                  "nbody_drift: null array");
    nb::launch_drift(p->x, p->y, p->z, p->vx, p->vy, p->vz, dt, p->n, 0);
    nb::finish("integrator_driftKernel");
  })
}

int nbody_reset_acc(nbody_particles* p) {
  NBODY_API_BODY({
    NBODY_REQUIRE(p && p->n >= 0 && p->ax && p->ay && p->az, "nbody_reset_acc: null array");
    nb::launch_reset_acc(p->ax, p->ay, p->az, p->n, 0);
    nb::finish("integrator_resetAccKernel");
  })
}

int nbody_gas_drag(nbody_particles* p, float drag_rate, float dt, float star_mass) {
  NBODY_API_BODY({
    NBODY_REQUIRE(p && p->n >= 0, "nbody_gas_drag: null particles");
    if (drag_rate <= 0.0f) return NBODY_OK;  // Integrator.cu:102
    NBODY_REQUIRE(p->x && p->z && p->vx && p->vy && p->vz, "nbody_gas_drag: null array");
    float decay = expf(-drag_rate * dt);    // Integrator.cu:103, host expf
    nb::launch_gas_drag(p->x, p->y, p->z, p->vx, p->vy, p->vz, decay, star_mass, p->n, 0);
    nb::finish("integrator_gasDragKernel");
  })
}

int nbody_perturber_force(nbody_particles* p, float px, float py, float pz, float pmass,
                          float softening) {
  NBODY_API_BODY({
    NBODY_REQUIRE(p && p->n >= 0 && p->x && p->y && p->z && p->ax && p->ay && p->az,
                  "nbody_perturber_force: null array");
    nb::launch_perturber_force(p->ax, p->ay, p->az, p->x, p->y, p->z, px, py, pz, pmass,
                               softening, p->n, 0);
    nb::finish("perturber_forceKernel");
  })
}

int nbody_fof(nbody_tree* t, const float* x, const float* y, const float* z, int n,
              float link_length, int* labels, uint16_t* agg_size, int* n_groups) {
  NBODY_API_BODY({
    NBODY_REQUIRE(t && x && y && z && labels && agg_size && n_groups, "nbody_fof: null argument");
    NBODY_REQUIRE(n >= 0 && n <= t->n, "nbody_fof: n exceeds the tree's capacity");
    *n_groups = 0;
    if (n == 0) return NBODY_OK;
    nb::TreeWork& w = t->tw;
    nb::launch_bbox<float>(w, x, y, z, n, 0);
    nb::launch_keys<float>(w, x, y, z, n, 0);
    nb::radix_sort_pairs(w.keys, w.perm, w.keys_alt, w.perm_alt, w.counts, n, 30, 0, w.status);
    nb::launch_gather_body4(w, x, y, z, nullptr, n, 0);
    nb::launch_build_topology(w, n, 0);
    nb::launch_build_moments(w, n, nullptr, nullptr, nullptr, 0);
    nb::NeighborArgs na{w.oct.info, w.oct.box_lo, w.oct.box_hi, w.body4, n,
                        w.groups, w.n_groups, t->leaf_max, t->spill, t->spill_cap, t->work, w.status};
    nb::launch_fof_link(na, w.perm, link_length, t->parent, 0);
    nb::launch_fof_finish(t->parent, n, labels, t->sizes, agg_size, t->ngroups, w.status, 0);
    nb::finish("nbody_fof");
    nb::check(cudaMemcpy(n_groups, t->ngroups, sizeof(int), cudaMemcpyDeviceToHost), "groups read");
    t->have_bbox = t->built = t->summarized = false;  // buffers now hold the FoF tree
    t->throw_status("nbody_fof");
  })
}

}  // extern "C"
