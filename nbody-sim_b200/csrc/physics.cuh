// physics.cuh -- per-particle formulas shared by the phase kernels and the
// fused step kernel, so both round identically.
#pragma once
#include <cuda_runtime.h>

namespace nb {

// Gas drag about the XZ-plane circular orbit (Integrator.cu:47-75): damps
// v_r, v_y and (v_phi - v_K) by `decay`, keeping the sign of v_phi.  Same
// expression order as the reference so default contraction matches.
template <typename R>
__device__ __forceinline__ void gas_drag(R xi, R zi, R& vx, R& vy, R& vz, R decay, R star_mass) {
  R r_xz2 = xi * xi + zi * zi;
  if (r_xz2 < R(1e-12f)) return;
  R r_xz = sqrt(r_xz2);
  R inv_r = R(1) / r_xz;
  R vxi = vx, vyi = vy, vzi = vz;
  R v_r = (vxi * xi + vzi * zi) * inv_r;
  R v_phi = (vxi * (-zi) + vzi * xi) * inv_r;
  R v_kep_mag = sqrt(star_mass * inv_r);
  R v_kep = (v_phi >= R(0)) ? v_kep_mag : -v_kep_mag;
  R v_r_new = v_r * decay;
  R v_phi_new = v_kep + (v_phi - v_kep) * decay;
  R v_y_new = vyi * decay;
  vx = v_r_new * (xi * inv_r) + v_phi_new * (-zi * inv_r);
  vz = v_r_new * (zi * inv_r) + v_phi_new * (xi * inv_r);
  vy = v_y_new;
}

// FP64 state (the engine's own precision mode, no reference kernel to match):
// every multiply-add is an explicit fma or a separately rounded product, so
// each kernel that inlines it rounds the same way whatever the compiler's
// contraction choices (the fused kick of a step boundary and the split
// closing/opening kicks of two calls then agree bit for bit).
template <>
__device__ __forceinline__ void gas_drag<double>(double xi, double zi, double& vx, double& vy,
                                                 double& vz, double decay, double star_mass) {
  const double r_xz2 = fma(xi, xi, __dmul_rn(zi, zi));
  if (r_xz2 < 1e-12) return;
  const double inv_r = 1.0 / sqrt(r_xz2);
  const double vxi = vx, vyi = vy, vzi = vz;
  const double v_r = __dmul_rn(fma(vxi, xi, __dmul_rn(vzi, zi)), inv_r);
  const double v_phi = __dmul_rn(fma(vxi, -zi, __dmul_rn(vzi, xi)), inv_r);
  const double v_kep_mag = sqrt(__dmul_rn(star_mass, inv_r));
  const double v_kep = (v_phi >= 0.0) ? v_kep_mag : -v_kep_mag;
  const double v_r_new = __dmul_rn(v_r, decay);
  const double v_phi_new = fma(v_phi - v_kep, decay, v_kep);
  const double ux = __dmul_rn(xi, inv_r), uz = __dmul_rn(zi, inv_r);
  vx = fma(v_r_new, ux, __dmul_rn(v_phi_new, -uz));
  vz = fma(v_r_new, uz, __dmul_rn(v_phi_new, ux));
  vy = __dmul_rn(vyi, decay);
}

// Softened star pull -M x / (|x|^2 + eps^2)^(3/2) (BHTree.cu:547-553 form).
template <typename R>
__device__ __forceinline__ void star_accel(R x, R y, R z, R eps, R star_mass, R& ax, R& ay,
                                           R& az) {
  R dx = -x, dy = -y, dz = -z;
  R r2 = dx * dx + dy * dy + dz * dz + eps * eps;
  R r = sqrt(r2);
  R f = star_mass / (r2 * r);
  ax = f * dx;
  ay = f * dy;
  az = f * dz;
}

template <>
__device__ __forceinline__ void star_accel<double>(double x, double y, double z, double eps,
                                                   double star_mass, double& ax, double& ay,
                                                   double& az) {
  const double r2 = fma(x, x, fma(y, y, fma(z, z, __dmul_rn(eps, eps))));
  const double r = sqrt(r2);
  const double f = star_mass / __dmul_rn(r2, r);
  ax = __dmul_rn(f, -x);
  ay = __dmul_rn(f, -y);
  az = __dmul_rn(f, -z);
}

}  // namespace nb
