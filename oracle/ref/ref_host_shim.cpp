// oracle/ref/ref_host_shim.cpp -- extern "C" entry points over the reference's
// own host code (src/config/Config.cpp, src/analysis/Aggregate.cpp,
// src/io/OutputWriter.cpp, src/disk/DiskInit.cpp), compiled from the files
// where they lie in the reference checkout into oracle/_ref/libref_host.so.
//
// TEST INFRASTRUCTURE ONLY: used to pin the oracle and to generate the golden
// fixtures under tests/golden/, and as the timed CPU FoF baseline.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "Aggregate.h"
#include "Config.h"
#include "DiskInit.h"
#include "OutputWriter.h"
#include "ParticleData.h"

namespace {
void copy_err(const std::exception& e, char* err, int errlen) {
    if (err && errlen > 0) {
        std::strncpy(err, e.what(), (size_t)errlen - 1);
        err[errlen - 1] = 0;
    }
}

ParticleData wrap(const float* x, const float* y, const float* z, const float* vx,
                  const float* vy, const float* vz, int n) {
    ParticleData p;
    p.n = n;
    p.x = const_cast<float*>(x); p.y = const_cast<float*>(y); p.z = const_cast<float*>(z);
    p.vx = const_cast<float*>(vx); p.vy = const_cast<float*>(vy); p.vz = const_cast<float*>(vz);
    return p;
}
}  // namespace

extern "C" {

// Config fields in declaration order (include/Config.h:5-35):
// f[0..11] = disk_r_min, disk_r_max, disk_h_factor, particle_mass_msun,
//            star_mass_msun, softening_AU, theta, collision_radius_factor,
//            restitution, gas_drag_rate, dt, total_time
// f[12..14] = perturber_mass_mjup, perturber_radius_AU, perturber_phase0
// i[0] = n_particles, i[1] = output_every_n_steps, i[2] = perturber_enabled
int ref_load_config(const char* path, float* f, int* i, char* out_dir, int dir_len,
                    char* err, int errlen) {
    try {
        Config c = loadConfig(path);
        float vals[15] = {c.disk_r_min, c.disk_r_max, c.disk_h_factor, c.particle_mass_msun,
                          c.star_mass_msun, c.softening_AU, c.theta,
                          c.collision_radius_factor, c.restitution, c.gas_drag_rate, c.dt,
                          c.total_time, c.perturber_mass_mjup, c.perturber_radius_AU,
                          c.perturber_phase0};
        std::memcpy(f, vals, sizeof(vals));
        i[0] = c.n_particles;
        i[1] = c.output_every_n_steps;
        i[2] = c.perturber_enabled ? 1 : 0;
        std::strncpy(out_dir, c.output_dir.c_str(), (size_t)dir_len - 1);
        out_dir[dir_len - 1] = 0;
        return 0;
    } catch (const std::exception& e) {
        copy_err(e, err, errlen);
        return 1;
    }
}

// initDisk (src/disk/DiskInit.cpp:18-69) into caller arrays (n = cfg size).
int ref_init_disk(int n, unsigned seed, float* x, float* y, float* z, float* vx, float* vy,
                  float* vz) {
  try {
    Config c;
    c.n_particles = n;
    ParticleData p = initDisk(c, seed);
    size_t b = (size_t)n * sizeof(float);
    std::memcpy(x, p.x, b); std::memcpy(y, p.y, b); std::memcpy(z, p.z, b);
    std::memcpy(vx, p.vx, b); std::memcpy(vy, p.vy, b); std::memcpy(vz, p.vz, b);
    freeParticlesCPU(p);
    return 0;
  } catch (...) {
    return 1;
  }
}

float ref_particle_radius(float particle_mass_msun) {
    Config c;
    c.particle_mass_msun = particle_mass_msun;
    return particlePhysicalRadius(c);
}

// detectAggregates on host arrays.  Output per particle: labels[i] = the
// smallest member index of i's aggregate (i itself for singletons) and the
// uint16 size of src/main.cu:153-161.  Aggregates are returned ordered by
// their smallest member index (the reference's own order is unordered_map
// iteration order, so it is canonicalised here).  Returns the group count or
// -1 on error; at most max_groups are written.
int ref_detect_aggregates(const float* x, const float* y, const float* z, const float* vx,
                          const float* vy, const float* vz, int n, float link_length,
                          float particle_mass, int* labels, uint16_t* agg_size,
                          int max_groups, int* g_n, float* g_mass, float* g_c, float* g_v,
                          float* g_dist, int* g_label) {
    try {
        ParticleData p = wrap(x, y, z, vx, vy, vz, n);
        Config cfg;
        cfg.particle_mass_msun = particle_mass;
        std::vector<Aggregate> aggs = detectAggregates(p, link_length, cfg);
        for (int k = 0; k < n; ++k) { labels[k] = k; agg_size[k] = 1; }
        std::map<int, const Aggregate*> order;
        for (const Aggregate& a : aggs) {
            int lo = *std::min_element(a.particle_ids.begin(), a.particle_ids.end());
            order[lo] = &a;
            uint16_t s = (uint16_t)std::min(a.n_particles, 65535);
            for (int pid : a.particle_ids) { labels[pid] = lo; agg_size[pid] = s; }
        }
        int g = 0;
        for (auto& kv : order) {
            if (g >= max_groups) break;
            const Aggregate& a = *kv.second;
            g_label[g] = kv.first; g_n[g] = a.n_particles; g_mass[g] = a.mass_msun;
            g_c[3 * g] = a.cx; g_c[3 * g + 1] = a.cy; g_c[3 * g + 2] = a.cz;
            g_v[3 * g] = a.vx; g_v[3 * g + 1] = a.vy; g_v[3 * g + 2] = a.vz;
            g_dist[g] = a.dist_center;
            ++g;
        }
        return (int)aggs.size();
    } catch (...) {
        return -1;
    }
}

// Times detectAggregates alone (no output conversion) for the CPU baseline.
int ref_detect_aggregates_count(const float* x, const float* y, const float* z, int n,
                                float link_length) {
    ParticleData p = wrap(x, y, z, x, y, z, n);
    Config cfg;
    return (int)detectAggregates(p, link_length, cfg).size();
}

// Drives OutputWriter through a scripted run: n_frames frames of the given
// positions (frame k at time t[k]) with per-particle sizes, the aggregates of
// ref_detect_aggregates for each frame (same aggregates every frame), an
// optional perturber row, then finalize.  Used to produce golden output bytes.
int ref_write_run(const char* dir, int n, float dt, int output_every, const float* x,
                  const float* y, const float* z, const uint16_t* agg_size, int n_frames,
                  const float* t, int n_aggs, const int* g_n, const float* g_mass,
                  const float* g_c, const float* g_v, const float* g_dist, int pert_enabled,
                  const float* pert /* x,y,z,mass,omega per frame: 5*n_frames */, char* err,
                  int errlen) {
    try {
        Config cfg;
        cfg.n_particles = n;
        cfg.dt = dt;
        cfg.output_every_n_steps = output_every;
        ParticleData p = wrap(x, y, z, x, y, z, n);
        std::vector<uint16_t> sizes(agg_size, agg_size + n);
        std::vector<Aggregate> aggs;
        for (int g = 0; g < n_aggs; ++g) {
            Aggregate a;
            a.id = g; a.n_particles = g_n[g]; a.mass_msun = g_mass[g];
            a.cx = g_c[3 * g]; a.cy = g_c[3 * g + 1]; a.cz = g_c[3 * g + 2];
            a.vx = g_v[3 * g]; a.vy = g_v[3 * g + 1]; a.vz = g_v[3 * g + 2];
            a.dist_center = g_dist[g];
            aggs.push_back(a);
        }
        OutputWriter w(dir, cfg);
        for (int f = 0; f < n_frames; ++f) {
            w.writeFrame(p, t[f], sizes);
            w.writeStats(aggs, f, t[f]);
            if (pert_enabled)
                w.writePerturberStats(f, t[f], n_aggs, pert[5 * f], pert[5 * f + 1],
                                      pert[5 * f + 2], pert[5 * f + 3], pert[5 * f + 4]);
        }
        w.finalize(n_frames);
        return 0;
    } catch (const std::exception& e) {
        copy_err(e, err, errlen);
        return 1;
    }
}

}  // extern "C"
