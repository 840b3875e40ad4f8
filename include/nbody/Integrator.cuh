// Integrator.cuh -- drop-in for the reference's include/Integrator.cuh
// (:9-22); synchronous launchers over the nbody-b200 streaming kernels.
#pragma once

#include "ParticleData.h"

inline void launchHalfKickKernel(ParticleData& gpu, float dt_half) {
  nbody_check(nbody_half_kick(nbody_view(gpu), dt_half));
}

inline void launchDriftKernel(ParticleData& gpu, float dt) {
  nbody_check(nbody_drift(nbody_view(gpu), dt));
}

inline void launchResetAccelerationKernel(ParticleData& gpu) {
  nbody_check(nbody_reset_acc(nbody_view(gpu)));
}

inline void launchGasDragKernel(ParticleData& gpu, float drag_rate, float dt,
                                float star_mass_msun) {
  nbody_check(nbody_gas_drag(nbody_view(gpu), drag_rate, dt, star_mass_msun));
}
