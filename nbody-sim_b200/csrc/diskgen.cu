// diskgen.cu -- synthetic Keplerian disks generated on the GPU, many disks in
// one launch (the initial conditions of an ensemble), body for body the same
// arithmetic as the host generator (diskgen.h).
#include <algorithm>
#include <vector>

#include "capi_util.h"
#include "common.cuh"
#include "diskgen.h"

namespace nb {
namespace {

struct DiskGenArgs {
  const int* offsets;        // n_disks + 1 prefix of the disk sizes
  const uint64_t* seeds;
  int n_disks;
  long long total;
  double r_min, r_max, sigma_e, sigma_i, mu;
  double *x, *y, *z, *vx, *vy, *vz;
};

__global__ void k_make_disks(const DiskGenArgs a) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.total;
       i += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = a.n_disks - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (a.offsets[mid] <= i) lo = mid;
      else hi = mid - 1;
    }
    double st[6];
    disk_body(a.seeds[lo], (uint64_t)(i - a.offsets[lo]), a.r_min, a.r_max, a.sigma_e,
              a.sigma_i, a.mu, st);
    a.x[i] = st[0]; a.y[i] = st[1]; a.z[i] = st[2];
    a.vx[i] = st[3]; a.vy[i] = st[4]; a.vz[i] = st[5];
  }
}

}  // namespace
}  // namespace nb

extern "C" int nbody_make_disks_device(const int* counts, const uint64_t* seeds, int n_disks,
                                       double r_min, double r_max, double sigma_e,
                                       double sigma_i, double star_mass, double* x, double* y,
                                       double* z, double* vx, double* vy, double* vz,
                                       void* stream) {
  NBODY_API_BODY({
    NBODY_REQUIRE(counts && seeds && n_disks >= 1, "nbody_make_disks_device: bad disk table");
    NBODY_REQUIRE(x && y && z && vx && vy && vz, "nbody_make_disks_device: null output");
    NBODY_REQUIRE(r_min > 0.0 && r_max > r_min && star_mass > 0.0,
                  "nbody_make_disks_device: bad radii or star mass");
    std::vector<int> off(n_disks + 1, 0);
    for (int d = 0; d < n_disks; ++d) {
      NBODY_REQUIRE(counts[d] >= 0, "nbody_make_disks_device: negative disk size");
      NBODY_REQUIRE((long long)off[d] + counts[d] < (1ll << 31),
                    "nbody_make_disks_device: too many bodies");
      off[d + 1] = off[d] + counts[d];
    }
    if (off[n_disks] == 0) return NBODY_OK;
    cudaStream_t st = (cudaStream_t)stream;
    int* d_off = nullptr;
    uint64_t* d_seed = nullptr;
    nb::check(cudaMallocAsync(&d_off, sizeof(int) * (n_disks + 1), st), "disk offsets");
    nb::check(cudaMallocAsync(&d_seed, sizeof(uint64_t) * n_disks, st), "disk seeds");
    nb::check(cudaMemcpyAsync(d_off, off.data(), sizeof(int) * (n_disks + 1),
                              cudaMemcpyHostToDevice, st), "offsets H2D");
    nb::check(cudaMemcpyAsync(d_seed, seeds, sizeof(uint64_t) * n_disks, cudaMemcpyHostToDevice,
                              st), "seeds H2D");
    nb::DiskGenArgs a{d_off, d_seed, n_disks, off[n_disks], r_min, r_max, sigma_e, sigma_i,
                      star_mass, x, y, z, vx, vy, vz};
    const int grid = std::max(1, std::min(nb::div_up(a.total, 256), 148 * 16));
    nb::k_make_disks<<<grid, 256, 0, st>>>(a);
    nb::check(cudaGetLastError(), "k_make_disks launch");
    nb::check(cudaFreeAsync(d_off, st), "offsets free");
    nb::check(cudaFreeAsync(d_seed, st), "seeds free");
    nb::check(cudaStreamSynchronize(st), "disk generation");
  })
}
