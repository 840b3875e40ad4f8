// Config.h -- drop-in for the reference's include/Config.h: the same struct,
// field defaults and loadConfig(path) (src/config/Config.cpp:6-55), which
// throws std::runtime_error with the reference's messages.
#pragma once

#include <cstdio>
#include <stdexcept>
#include <string>

#include "../nbody_b200.h"

struct Config {
  int n_particles = 100000;
  float disk_r_min = 0.5f;
  float disk_r_max = 5.0f;
  float disk_h_factor = 0.05f;
  float particle_mass_msun = 3.003e-7f;
  float star_mass_msun = 1.0f;
  float softening_AU = 0.01f;
  float theta = 0.5f;
  float collision_radius_factor = 100.0f;
  float restitution = 0.3f;
  float gas_drag_rate = 0.0f;
  float dt = 0.01f;
  float total_time = 2000.0f;
  int output_every_n_steps = 200;
  std::string output_dir = "data";
  bool perturber_enabled = false;
  float perturber_mass_mjup = 1.0f;
  float perturber_radius_AU = 20.0f;
  float perturber_phase0 = 0.0f;
};

inline nbody_config nbody_to_c(const Config& c) {
  nbody_config o;
  nbody_config_defaults(&o);
  o.n_particles = c.n_particles;
  o.disk_r_min = c.disk_r_min;
  o.disk_r_max = c.disk_r_max;
  o.disk_h_factor = c.disk_h_factor;
  o.particle_mass_msun = c.particle_mass_msun;
  o.star_mass_msun = c.star_mass_msun;
  o.softening_AU = c.softening_AU;
  o.theta = c.theta;
  o.collision_radius_factor = c.collision_radius_factor;
  o.restitution = c.restitution;
  o.gas_drag_rate = c.gas_drag_rate;
  o.dt = c.dt;
  o.total_time = c.total_time;
  o.output_every_n_steps = c.output_every_n_steps;
  std::snprintf(o.output_dir, sizeof(o.output_dir), "%s", c.output_dir.c_str());
  o.perturber_enabled = c.perturber_enabled ? 1 : 0;
  o.perturber_mass_mjup = c.perturber_mass_mjup;
  o.perturber_radius_AU = c.perturber_radius_AU;
  o.perturber_phase0 = c.perturber_phase0;
  return o;
}

inline Config nbody_from_c(const nbody_config& o) {
  Config c;
  c.n_particles = o.n_particles;
  c.disk_r_min = o.disk_r_min;
  c.disk_r_max = o.disk_r_max;
  c.disk_h_factor = o.disk_h_factor;
  c.particle_mass_msun = o.particle_mass_msun;
  c.star_mass_msun = o.star_mass_msun;
  c.softening_AU = o.softening_AU;
  c.theta = o.theta;
  c.collision_radius_factor = o.collision_radius_factor;
  c.restitution = o.restitution;
  c.gas_drag_rate = o.gas_drag_rate;
  c.dt = o.dt;
  c.total_time = o.total_time;
  c.output_every_n_steps = o.output_every_n_steps;
  c.output_dir = o.output_dir;
  c.perturber_enabled = o.perturber_enabled != 0;
  c.perturber_mass_mjup = o.perturber_mass_mjup;
  c.perturber_radius_AU = o.perturber_radius_AU;
  c.perturber_phase0 = o.perturber_phase0;
  return c;
}

inline Config loadConfig(const std::string& path) {
  nbody_config o;
  if (nbody_config_load(path.c_str(), &o) != NBODY_OK) throw std::runtime_error(nbody_last_error());
  return nbody_from_c(o);
}
