// stream.cu -- element-wise kernels behind the reference's Integrator.cuh and
// Perturber.h launchers (drop-in phase API, caller order, FP32).
//
// Each kernel keeps the reference's per-element arithmetic (Integrator.cu:7-76,
// Perturber.cu:13-35, BHTree.cu:676-686) so that, compiled with the same
// default contraction, results are bit-identical to the reference kernels.
// They differ in launch shape: a grid-stride loop over 148 x 8 blocks of 256
// threads instead of ceil(n/256) blocks, no per-launch device sync.
#include "common.cuh"
#include "kernels.cuh"
#include "physics.cuh"

namespace nb {
namespace {

constexpr int kThreads = 256;

int grid_for(int n) {
  int g = div_up(n, kThreads);
  return std::max(1, std::min(g, 148 * 8));
}

#define GRID_STRIDE(i, n)                                                        \
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (n); \
       i += (long long)gridDim.x * blockDim.x)

__global__ void k_half_kick(float* __restrict__ vx, float* __restrict__ vy,
                            float* __restrict__ vz, const float* __restrict__ ax,
                            const float* __restrict__ ay, const float* __restrict__ az,
                            float dt_half, int n) {
  GRID_STRIDE(i, n) {
    vx[i] += ax[i] * dt_half;
    vy[i] += ay[i] * dt_half;
    vz[i] += az[i] * dt_half;
  }
}

__global__ void k_drift(float* __restrict__ x, float* __restrict__ y, float* __restrict__ z,
                        const float* __restrict__ vx, const float* __restrict__ vy,
                        const float* __restrict__ vz, float dt, int n) {
  GRID_STRIDE(i, n) {
    x[i] += vx[i] * dt;
    y[i] += vy[i] * dt;
    z[i] += vz[i] * dt;
  }
}

__global__ void k_reset_acc(float* __restrict__ ax, float* __restrict__ ay,
                            float* __restrict__ az, int n) {
  GRID_STRIDE(i, n) {
    ax[i] = 0.f;
    ay[i] = 0.f;
    az[i] = 0.f;
  }
}

// Gas drag (Integrator.cu:40-76), formula shared with the fused step kernel.
__global__ void k_gas_drag(const float* __restrict__ x, const float* __restrict__ z,
                           float* __restrict__ vx, float* __restrict__ vy,
                           float* __restrict__ vz, float decay, float star_mass, int n) {
  GRID_STRIDE(i, n) {
    float a = vx[i], b = vy[i], c = vz[i];
    gas_drag<float>(x[i], z[i], a, b, c, decay, star_mass);
    vx[i] = a;
    vy[i] = b;
    vz[i] = c;
  }
}

__global__ void k_perturber(float* __restrict__ ax, float* __restrict__ ay,
                            float* __restrict__ az, const float* __restrict__ x,
                            const float* __restrict__ y, const float* __restrict__ z, float px,
                            float py, float pz, float pm, float eps, int n) {
  GRID_STRIDE(i, n) {
    float dx = px - x[i];
    float dy = py - y[i];
    float dz = pz - z[i];
    float r2 = dx * dx + dy * dy + dz * dz + eps * eps;
    float r = sqrtf(r2);
    float f = pm / (r2 * r);
    ax[i] += f * dx;
    ay[i] += f * dy;
    az[i] += f * dz;
  }
}

__global__ void k_apply_dv(float* __restrict__ vx, float* __restrict__ vy,
                           float* __restrict__ vz, const float* __restrict__ dvx,
                           const float* __restrict__ dvy, const float* __restrict__ dvz,
                           const uint32_t* __restrict__ map, int n) {
  GRID_STRIDE(s, n) {
    const uint32_t i = map ? map[s] : (uint32_t)s;
    vx[i] += dvx[s];
    vy[i] += dvy[s];
    vz[i] += dvz[s];
  }
}

__global__ void k_copy_perm(int* __restrict__ dst, const uint32_t* __restrict__ perm, int n) {
  GRID_STRIDE(i, n) dst[i] = (int)perm[i];
}

}  // namespace

void launch_half_kick(float* vx, float* vy, float* vz, const float* ax, const float* ay,
                      const float* az, float dt_half, int n, cudaStream_t s) {
  if (n <= 0) return;
  k_half_kick<<<grid_for(n), kThreads, 0, s>>>(vx, vy, vz, ax, ay, az, dt_half, n);
  check(cudaGetLastError(), "k_half_kick launch");
}

void launch_drift(float* x, float* y, float* z, const float* vx, const float* vy,
                  const float* vz, float dt, int n, cudaStream_t s) {
  if (n <= 0) return;
  k_drift<<<grid_for(n), kThreads, 0, s>>>(x, y, z, vx, vy, vz, dt, n);
  check(cudaGetLastError(), "k_drift launch");
}

void launch_reset_acc(float* ax, float* ay, float* az, int n, cudaStream_t s) {
  if (n <= 0) return;
  k_reset_acc<<<grid_for(n), kThreads, 0, s>>>(ax, ay, az, n);
  check(cudaGetLastError(), "k_reset_acc launch");
}

void launch_gas_drag(const float* x, const float*, const float* z, float* vx, float* vy,
                     float* vz, float decay, float star_mass, int n, cudaStream_t s) {
  if (n <= 0) return;
  k_gas_drag<<<grid_for(n), kThreads, 0, s>>>(x, z, vx, vy, vz, decay, star_mass, n);
  check(cudaGetLastError(), "k_gas_drag launch");
}

void launch_perturber_force(float* ax, float* ay, float* az, const float* x, const float* y,
                            const float* z, float px, float py, float pz, float pmass,
                            float eps, int n, cudaStream_t s) {
  if (n <= 0) return;
  k_perturber<<<grid_for(n), kThreads, 0, s>>>(ax, ay, az, x, y, z, px, py, pz, pmass, eps, n);
  check(cudaGetLastError(), "k_perturber launch");
}

void launch_apply_dv(float* vx, float* vy, float* vz, const float* dvx, const float* dvy,
                     const float* dvz, const uint32_t* map, int n, cudaStream_t s) {
  if (n <= 0) return;
  k_apply_dv<<<grid_for(n), kThreads, 0, s>>>(vx, vy, vz, dvx, dvy, dvz, map, n);
  check(cudaGetLastError(), "k_apply_dv launch");
}

void launch_copy_perm(int* dst, const uint32_t* perm, int n, cudaStream_t s) {
  if (n <= 0) return;
  k_copy_perm<<<grid_for(n), kThreads, 0, s>>>(dst, perm, n);
  check(cudaGetLastError(), "k_copy_perm launch");
}

}  // namespace nb
