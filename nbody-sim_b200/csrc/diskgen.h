// diskgen.h -- the synthetic Keplerian disk, one body at a time, shared by
// the host generator (nbody_make_disk) and the GPU one
// (nbody_make_disks_device) so both run the same arithmetic; they differ only
// in the last-ulp rounding of the sin/cos/log1p of their math libraries.
//
// Body i of a disk with seed s: semi-major axis from Sigma ~ r^-1.5 by the
// inverse CDF of src/disk/DiskInit.cpp:42-44; Rayleigh eccentricity and
// inclination (capped at e = 0.9); node, periapsis and mean anomaly uniform;
// Kepler's equation by Newton; perifocal -> frame with the +Z pole, then the
// reference's disk plane XZ with +Y up: (X, Y, Z) -> (X, -Z, Y) (the sense of
// rotation of DiskInit.cpp:47-49).  Draw k of body i is splitmix64 (Vigna) of
// splitmix64(seed) ^ (16 i + k): any body is reproducible on its own.
#pragma once
#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define NB_HD __host__ __device__ __forceinline__
#else
#define NB_HD inline
#endif

namespace nb {

NB_HD uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Uniform draw in [0, 1) with 53 random bits.
NB_HD double disk_unit(uint64_t seed, uint64_t i, uint64_t k) {
  const uint64_t h = splitmix64(splitmix64(seed) ^ (i * 16u + k));
  return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

// out = x, y, z, vx, vy, vz of body i (G = 1, star mass mu).
NB_HD void disk_body(uint64_t seed, uint64_t i, double r_min, double r_max, double sigma_e,
                     double sigma_i, double mu, double* out) {
  const double two_pi = 6.283185307179586476925287;
  const double sa = sqrt(r_min), sb = sqrt(r_max);
  const double u = disk_unit(seed, i, 0);
  const double sr = u * (sb - sa) + sa;
  const double a = sr * sr;
  double e = sigma_e * sqrt(-2.0 * log1p(-disk_unit(seed, i, 1)));
  const double inc = sigma_i * sqrt(-2.0 * log1p(-disk_unit(seed, i, 2)));
  if (e > 0.9) e = 0.9;
  const double Om = two_pi * disk_unit(seed, i, 3);
  const double om = two_pi * disk_unit(seed, i, 4);
  const double M = two_pi * disk_unit(seed, i, 5);
  double E = (e < 0.8) ? M : 3.141592653589793;
  for (int it = 0; it < 60; ++it) {
    const double f = E - e * sin(E) - M;
    const double d = f / (1.0 - e * cos(E));
    E -= d;
    if (fabs(d) < 1e-15) break;
  }
  const double cE = cos(E), sE = sin(E);
  const double q = sqrt(1.0 - e * e);
  const double nmot = sqrt(mu / (a * a * a));
  const double den = 1.0 - e * cE;
  const double xp = a * (cE - e), yp = a * q * sE;
  const double vxp = -a * nmot * sE / den, vyp = a * nmot * q * cE / den;
  const double cO = cos(Om), sO = sin(Om), co = cos(om), so = sin(om);
  const double ci = cos(inc), si = sin(inc);
  const double r11 = cO * co - sO * so * ci, r12 = -cO * so - sO * co * ci;
  const double r21 = sO * co + cO * so * ci, r22 = -sO * so + cO * co * ci;
  const double r31 = so * si, r32 = co * si;
  const double X = r11 * xp + r12 * yp, Y = r21 * xp + r22 * yp, Z = r31 * xp + r32 * yp;
  const double VX = r11 * vxp + r12 * vyp, VY = r21 * vxp + r22 * vyp,
               VZ = r31 * vxp + r32 * vyp;
  out[0] = X; out[1] = -Z; out[2] = Y;
  out[3] = VX; out[4] = -VZ; out[5] = VY;
}

}  // namespace nb
