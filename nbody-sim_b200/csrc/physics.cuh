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

}  // namespace nb
