// OutputWriter.h -- drop-in for the reference's include/OutputWriter.h
// (:15-51): frames.bin v2 and stats.csv, byte-compatible, over nbody_writer.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "Aggregate.h"
#include "Config.h"
#include "ParticleData.h"

constexpr float T0_TO_YEARS = 1.0f / (2.0f * 3.14159265f);
constexpr float MSUN_TO_MEARTH = 332946.0f;

class OutputWriter {
 public:
  OutputWriter(const std::string& output_dir, const Config& cfg) {
    nbody_config c = nbody_to_c(cfg);
    nbody_check(nbody_writer_open(output_dir.c_str(), &c, &w_));
  }
  ~OutputWriter() { nbody_writer_close(w_); }
  OutputWriter(const OutputWriter&) = delete;
  OutputWriter& operator=(const OutputWriter&) = delete;

  void writeFrame(const ParticleData& cpu_particles, float sim_time_T0,
                  const std::vector<uint16_t>& agg_sizes_per_particle) {
    if ((int)agg_sizes_per_particle.size() != cpu_particles.n)
      throw std::runtime_error("OutputWriter::writeFrame: agg_sizes_per_particle size mismatch");
    nbody_check(nbody_writer_frame(w_, cpu_particles.x, cpu_particles.y, cpu_particles.z,
                                   cpu_particles.n, sim_time_T0, agg_sizes_per_particle.data()));
  }

  void writeStats(const std::vector<Aggregate>& aggregates, int frame_idx, float sim_time_T0) {
    std::vector<nbody_aggregate> r(aggregates.size());
    for (size_t k = 0; k < aggregates.size(); ++k) {
      const Aggregate& a = aggregates[k];
      r[k] = nbody_aggregate{a.id, a.n_particles, a.mass_msun, a.cx, a.cy, a.cz,
                             a.vx, a.vy, a.vz, a.dist_center, 0};
    }
    nbody_check(nbody_writer_stats(w_, r.data(), (int)r.size(), frame_idx, sim_time_T0));
  }

  void writePerturberStats(int frame_idx, float sim_time_T0, int n_aggregates, float px,
                           float py, float pz, float mass_msun, float omega) {
    nbody_check(nbody_writer_perturber(w_, frame_idx, sim_time_T0, n_aggregates, px, py, pz,
                                       mass_msun, omega));
  }

  void finalize(int total_frames_written) {
    nbody_check(nbody_writer_finalize(w_, total_frames_written));
  }

 private:
  nbody_writer* w_ = nullptr;
};
