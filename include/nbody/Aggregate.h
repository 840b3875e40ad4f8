// Aggregate.h -- drop-in for the reference's include/Aggregate.h:
// detectAggregates(host particles, link length, cfg) (:17-18).  Links and
// union-find run on the GPU (nbody_fof), the records on the host
// (nbody_aggregates).  Groups come out ordered by their smallest member; the
// reference's order is its unordered_map's iteration order.
#pragma once

#include <vector>

#include "Config.h"
#include "ParticleData.h"

struct Aggregate {
  int id;
  int n_particles;
  float mass_msun;
  float cx, cy, cz;
  float vx, vy, vz;
  float dist_center;
  std::vector<int> particle_ids;
};

inline std::vector<Aggregate> detectAggregates(const ParticleData& p, float link_length,
                                               const Config& cfg) {
  const int n = p.n;
  std::vector<Aggregate> out;
  if (n <= 0) return out;
  nbody_tree* t = nullptr;
  float* d[3] = {nullptr, nullptr, nullptr};
  int* d_lab = nullptr;
  uint16_t* d_agg = nullptr;
  std::vector<int> labels(n);
  int groups = 0;
  try {
    nbody_check(nbody_tree_create(n, &t));
    const float* h[3] = {p.x, p.y, p.z};
    for (int k = 0; k < 3; ++k) {
      nbody_check_cuda(cudaMalloc((void**)&d[k], n * sizeof(float)), "cudaMalloc fof");
      nbody_check_cuda(cudaMemcpy(d[k], h[k], n * sizeof(float), cudaMemcpyHostToDevice), "fof H2D");
    }
    nbody_check_cuda(cudaMalloc((void**)&d_lab, n * sizeof(int)), "cudaMalloc fof");
    nbody_check_cuda(cudaMalloc((void**)&d_agg, n * sizeof(uint16_t)), "cudaMalloc fof");
    nbody_check(nbody_fof(t, d[0], d[1], d[2], n, link_length, d_lab, d_agg, &groups));
    nbody_check_cuda(cudaMemcpy(labels.data(), d_lab, n * sizeof(int), cudaMemcpyDeviceToHost),
                     "fof D2H");
  } catch (...) {
    for (float* q : d) cudaFree(q);
    cudaFree(d_lab);
    cudaFree(d_agg);
    nbody_tree_destroy(t);
    throw;
  }
  for (float* q : d) cudaFree(q);
  cudaFree(d_lab);
  cudaFree(d_agg);
  nbody_tree_destroy(t);
  std::vector<nbody_aggregate> recs((size_t)groups);
  int ng = 0;
  nbody_check(nbody_aggregates(p.x, p.y, p.z, p.vx, p.vy, p.vz, labels.data(), n,
                               cfg.particle_mass_msun, recs.data(), groups, &ng));
  std::vector<int> slot(n, -1);
  out.resize((size_t)ng);
  for (int g = 0; g < ng; ++g) {
    const nbody_aggregate& r = recs[g];
    Aggregate& a = out[g];
    a.id = r.id;
    a.n_particles = r.n_particles;
    a.mass_msun = r.mass_msun;
    a.cx = r.cx; a.cy = r.cy; a.cz = r.cz;
    a.vx = r.vx; a.vy = r.vy; a.vz = r.vz;
    a.dist_center = r.dist_center;
    a.particle_ids.reserve(r.n_particles);
    slot[r.first_member] = g;
  }
  for (int i = 0; i < n; ++i) {
    int g = slot[labels[i]];
    if (g >= 0) out[g].particle_ids.push_back(i);
  }
  return out;
}
