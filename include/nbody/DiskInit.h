// DiskInit.h -- drop-in for the reference's include/DiskInit.h (:10-14):
// particlePhysicalRadius over the C ABI and initDisk, the reference's
// Gaussian-thickness disk (src/disk/DiskInit.cpp:18-69): r by inverse CDF of
// Sigma ~ r^-1.5, uniform phi, y ~ N(0, h r), circular speed plus 1% noise,
// drawn from std::mt19937 in the same order, so the same standard library
// reproduces the same disk.
#pragma once

#include <cmath>
#include <random>
#include <stdexcept>

#include "Config.h"
#include "ParticleData.h"

inline float particlePhysicalRadius(const Config& cfg) {
  return nbody_particle_radius(cfg.particle_mass_msun);
}

inline ParticleData initDisk(const Config& cfg, unsigned int seed = 42) {
  if (cfg.n_particles <= 0) throw std::invalid_argument("initDisk: n_particles must be positive");
  if (cfg.disk_r_min <= 0.0f) throw std::invalid_argument("initDisk: disk_r_min must be positive");
  if (cfg.disk_r_min >= cfg.disk_r_max)
    throw std::invalid_argument("initDisk: disk_r_min must be less than disk_r_max");
  const float pi = 3.14159265358979f;
  ParticleData p = allocateParticlesCPU(cfg.n_particles);
  std::mt19937 gen(seed);
  std::uniform_real_distribution<float> uniform(0.0f, 1.0f);
  std::normal_distribution<float> gauss(0.0f, 1.0f);
  const float lo = std::sqrt(cfg.disk_r_min), hi = std::sqrt(cfg.disk_r_max);
  for (int i = 0; i < cfg.n_particles; ++i) {
    const float s = uniform(gen) * (hi - lo) + lo;
    const float r = s * s;
    const float phi = uniform(gen) * 2.0f * pi;
    const float c = std::cos(phi), sn = std::sin(phi);
    p.x[i] = r * c;
    p.z[i] = r * sn;
    p.y[i] = gauss(gen) * (cfg.disk_h_factor * r);
    const float v = std::sqrt(cfg.star_mass_msun / r);
    const float noise = 0.01f * v;
    p.vx[i] = -v * sn + gauss(gen) * noise;
    p.vz[i] = v * c + gauss(gen) * noise;
    p.vy[i] = gauss(gen) * noise;
    p.ax[i] = p.ay[i] = p.az[i] = 0.0f;
    p.mass[i] = cfg.particle_mass_msun;
    p.id[i] = i;
  }
  return p;
}
