// Perturber.h -- drop-in for the reference's include/Perturber.h: the
// analytic circular orbit in the XZ plane (:39-66) and the pull launcher
// (:73-75), over the nbody-b200 library.
#pragma once

#include <cmath>

#include "Config.h"
#include "ParticleData.h"

constexpr float MJUP_TO_MSUN = 9.5479e-4f;

struct Perturber {
  bool enabled = false;
  float r = 0.f;
  float mass_msun = 0.f;
  float phase0 = 0.f;
  float omega = 0.f;
  float x = 0.f, y = 0.f, z = 0.f;
};

inline Perturber makePerturber(const Config& cfg) {
  nbody_config c = nbody_to_c(cfg);
  nbody_perturber q;
  nbody_perturber_make(&c, &q);
  Perturber p;
  p.enabled = q.enabled != 0;
  p.r = q.r;
  p.mass_msun = q.mass_msun;
  p.phase0 = q.phase0;
  p.omega = q.omega;
  p.x = q.x;
  p.y = q.y;
  p.z = q.z;
  return p;
}

inline void updatePerturber(Perturber& p, float sim_time) {
  nbody_perturber q{p.enabled ? 1 : 0, p.r, p.mass_msun, p.phase0, p.omega, p.x, p.y, p.z};
  nbody_perturber_update(&q, sim_time);
  p.x = q.x;
  p.y = q.y;
  p.z = q.z;
}

inline void launchPerturberForceKernel(ParticleData& gpu, float px, float py, float pz,
                                       float pmass, float softening) {
  nbody_check(nbody_perturber_force(nbody_view(gpu), px, py, pz, pmass, softening));
}
