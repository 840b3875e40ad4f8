// ParticleData.h -- drop-in for the reference's include/ParticleData.h
// (struct and helpers at :9-123): the same SoA struct, allocation and copy
// helpers, over the nbody-b200 library.  The struct has the field order of
// nbody_particles (include/nbody_b200.h), so a ParticleData* can be passed to
// the C ABI as an nbody_particles*.
#pragma once

#include <stdexcept>
#include <string>

#include "../nbody_b200.h"

#ifdef __CUDACC__
#include <cuda_runtime.h>
#else
#include <cuda_runtime_api.h>
#endif

inline void nbody_check_cuda(cudaError_t err, const char* op) {
  if (err != cudaSuccess)
    throw std::runtime_error(std::string("CUDA error in ") + op + ": " + cudaGetErrorString(err));
}

// Throws std::runtime_error for a failed C ABI call (the reference throws
// from nbody_check_cuda and from loadConfig; callers see the same type).
inline void nbody_check(int rc) {
  if (rc != NBODY_OK) throw std::runtime_error(nbody_last_error());
}

struct ParticleData {
  float* x = nullptr;
  float* y = nullptr;
  float* z = nullptr;
  float* vx = nullptr;
  float* vy = nullptr;
  float* vz = nullptr;
  float* ax = nullptr;
  float* ay = nullptr;
  float* az = nullptr;
  float* mass = nullptr;
  int* id = nullptr;
  int n = 0;
};

static_assert(sizeof(ParticleData) == sizeof(nbody_particles), "layout must match the C ABI");

inline nbody_particles* nbody_view(ParticleData& p) {
  return reinterpret_cast<nbody_particles*>(&p);
}
inline const nbody_particles* nbody_view(const ParticleData& p) {
  return reinterpret_cast<const nbody_particles*>(&p);
}

inline ParticleData allocateParticlesCPU(int n) {
  ParticleData p;
  p.n = n;
  float** f[] = {&p.x, &p.y, &p.z, &p.vx, &p.vy, &p.vz, &p.ax, &p.ay, &p.az, &p.mass};
  for (float** a : f) *a = new float[n]();
  p.id = new int[n]();
  return p;
}

inline void freeParticlesCPU(ParticleData& p) {
  float** f[] = {&p.x, &p.y, &p.z, &p.vx, &p.vy, &p.vz, &p.ax, &p.ay, &p.az, &p.mass};
  for (float** a : f) {
    delete[] *a;
    *a = nullptr;
  }
  delete[] p.id;
  p.id = nullptr;
  p.n = 0;
}

inline ParticleData allocateParticlesGPU(int n) {
  ParticleData p;
  p.n = n;
  float** f[] = {&p.x, &p.y, &p.z, &p.vx, &p.vy, &p.vz, &p.ax, &p.ay, &p.az, &p.mass};
  for (float** a : f) nbody_check_cuda(cudaMalloc((void**)a, n * sizeof(float)), "cudaMalloc");
  nbody_check_cuda(cudaMalloc((void**)&p.id, n * sizeof(int)), "cudaMalloc id");
  return p;
}

inline void freeParticlesGPU(ParticleData& p) {
  float** f[] = {&p.x, &p.y, &p.z, &p.vx, &p.vy, &p.vz, &p.ax, &p.ay, &p.az, &p.mass};
  for (float** a : f) {
    cudaFree(*a);
    *a = nullptr;
  }
  cudaFree(p.id);
  p.id = nullptr;
  p.n = 0;
}

namespace nbody_detail {
inline void copy_all(const ParticleData& src, ParticleData& dst, cudaMemcpyKind kind,
                     const char* what) {
  if (src.n != dst.n)
    throw std::runtime_error(std::string(what) + ": n=" + std::to_string(src.n) +
                             " != n=" + std::to_string(dst.n));
  const size_t b = (size_t)src.n * sizeof(float);
  const float* s[] = {src.x, src.y, src.z, src.vx, src.vy, src.vz, src.ax, src.ay, src.az,
                      src.mass};
  float* d[] = {dst.x, dst.y, dst.z, dst.vx, dst.vy, dst.vz, dst.ax, dst.ay, dst.az, dst.mass};
  for (int k = 0; k < 10; ++k) nbody_check_cuda(cudaMemcpy(d[k], s[k], b, kind), what);
  nbody_check_cuda(cudaMemcpy(dst.id, src.id, (size_t)src.n * sizeof(int), kind), what);
}
}  // namespace nbody_detail

inline void copyToGPU(const ParticleData& cpu, ParticleData& gpu) {
  nbody_detail::copy_all(cpu, gpu, cudaMemcpyHostToDevice, "copyToGPU");
}

inline void copyToCPU(const ParticleData& gpu, ParticleData& cpu) {
  nbody_detail::copy_all(gpu, cpu, cudaMemcpyDeviceToHost, "copyToCPU");
}
