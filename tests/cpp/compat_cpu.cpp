// Compiles the drop-in headers (include/nbody/) as a reference caller would
// and exercises their host-only parts: loadConfig, initDisk,
// particlePhysicalRadius, makePerturber/updatePerturber, OutputWriter.
// Prints one line per check; the pytest wrapper compares them with the
// reference's own host code.
#include <cstdio>
#include <cstring>
#include <string>

#include "Aggregate.h"
#include "BHTree.cuh"
#include "Config.h"
#include "DiskInit.h"
#include "Integrator.cuh"
#include "OutputWriter.h"
#include "ParticleData.h"
#include "Perturber.h"

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  Config cfg = loadConfig(argv[1]);
  std::printf("config %d %.9g %.9g %d %s %d\n", cfg.n_particles, cfg.dt, cfg.theta,
              cfg.output_every_n_steps, cfg.output_dir.c_str(), cfg.perturber_enabled ? 1 : 0);
  try {
    loadConfig("/nonexistent/path.json");
    std::printf("missing-file no-throw\n");
  } catch (const std::runtime_error& e) {
    std::printf("missing-file %s\n", e.what());
  }
  Config dc;
  dc.n_particles = 1000;
  ParticleData p = initDisk(dc, 42);
  double h = 0;
  for (int i = 0; i < p.n; ++i) {
    unsigned u;
    float f[6] = {p.x[i], p.y[i], p.z[i], p.vx[i], p.vy[i], p.vz[i]};
    for (float q : f) {
      std::memcpy(&u, &q, 4);
      h = h * 1.0000001 + (double)(u % 100003);
    }
  }
  std::printf("disk %.17g %.9g %.9g\n", h, p.x[0], p.vz[999]);
  std::printf("radius %.9g\n", particlePhysicalRadius(dc));
  Config pc;
  pc.perturber_enabled = true;
  pc.perturber_radius_AU = 10.0f;
  Perturber pert = makePerturber(pc);
  updatePerturber(pert, 12.5f);
  std::printf("perturber %.9g %.9g %.9g\n", pert.omega, pert.x, pert.z);
  Config wc;
  wc.n_particles = p.n;
  {
    OutputWriter w(argv[2], wc);
    std::vector<uint16_t> agg(p.n, 1);
    w.writeFrame(p, 0.5f, agg);
    w.writeStats({}, 0, 0.5f);
    w.writePerturberStats(0, 0.5f, 0, pert.x, pert.y, pert.z, pert.mass_msun, pert.omega);
    w.finalize(1);
  }
  std::printf("writer ok\n");
  freeParticlesCPU(p);
  return 0;
}
