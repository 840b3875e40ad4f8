// BHTree.cuh -- drop-in for the reference's include/BHTree.cuh: the same
// launcher names and signatures (:38-50), each synchronous like the
// reference's, over the nbody-b200 octree (Morton keys, radix sort, Karras
// tree, FP64 moments, warp-group walk).  OctreeData keeps the fields callers
// read (sort_idx, n_bodies, n_total); the node arrays live in the library.
#pragma once

#include "ParticleData.h"

static constexpr int MAX_NODES_MULT = 8;

struct OctreeData {
  int* sort_idx = nullptr;  // device [n_bodies]: body order of the octree
  int n_bodies = 0;
  int n_total = 0;          // node capacity of the library's octree (2 n_bodies)
  nbody_tree* impl = nullptr;
};

inline OctreeData allocateOctree(int n_bodies) {
  OctreeData t;
  nbody_check(nbody_tree_create(n_bodies, &t.impl));
  t.n_bodies = n_bodies;
  t.n_total = 2 * n_bodies;
  t.sort_idx = nbody_tree_sort_idx(t.impl);
  return t;
}

inline void freeOctree(OctreeData& t) {
  nbody_tree_destroy(t.impl);
  t = OctreeData();
}

inline void resetOctree(OctreeData& t) { nbody_check(nbody_tree_reset(t.impl)); }

inline void launchBBoxKernel(OctreeData& t, const ParticleData& p) {
  nbody_check(nbody_tree_bbox(t.impl, nbody_view(p)));
}

inline void launchBuildKernel(OctreeData& t, const ParticleData& p) {
  nbody_check(nbody_tree_build(t.impl, nbody_view(p)));
}

inline void launchSummarizeKernel(OctreeData& t) { nbody_check(nbody_tree_summarize(t.impl)); }

inline void launchSortKernel(OctreeData& t) { nbody_check(nbody_tree_sort(t.impl)); }

inline void launchForceKernel(OctreeData& t, ParticleData& p, float theta, float softening,
                              float star_mass) {
  nbody_check(nbody_tree_force(t.impl, nbody_view(p), theta, softening, star_mass));
}

inline void launchCollisionKernel(OctreeData& t, ParticleData& p, float r_coll,
                                  float restitution) {
  nbody_check(nbody_tree_collide(t.impl, nbody_view(p), r_coll, restitution));
}
