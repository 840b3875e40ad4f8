// oracle/ref/ref_engine_shim.cu -- extern "C" driver for the reference's own
// CUDA engine (src/physics/BHTree.cu, Integrator.cu, Perturber.cu compiled
// unchanged for sm_100a into oracle/_ref/libref_engine*.so).  It replays the
// launcher sequence of src/main.cu:85-139 without file I/O.
//
// TEST INFRASTRUCTURE ONLY: pins the CPU oracle bit-for-bit (-fmad=false
// build) and measures the reference engine's step rate on the same GPU.
//
// Memory safety: the reference's launchSortKernel writes sort_idx only for
// bodies that made it into the tree; tree.sort_idx is zeroed once here so a
// body lost by the build (coincident bodies, 128-level limit) can never send
// the force kernel to an out-of-range index.  Callers also reject inputs the
// CPU oracle flags (lost bodies, unsummarized nodes) before calling in.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <vector>

#include "BHTree.cuh"
#include "Config.h"
#include "Integrator.cuh"
#include "ParticleData.h"
#include "Perturber.h"

namespace {
struct RefEngine {
    ParticleData gpu;
    OctreeData tree;
    int n;
};
char g_err[512];
}  // namespace

#define REF_TRY(...)                                          \
    try {                                                     \
        __VA_ARGS__;                                          \
        return 0;                                             \
    } catch (const std::exception& e) {                       \
        std::snprintf(g_err, sizeof(g_err), "%s", e.what());  \
        return 1;                                             \
    }

extern "C" {

const char* ref_eng_error() { return g_err; }

void* ref_eng_create(int n) {
    try {
        RefEngine* e = new RefEngine();
        e->n = n;
        e->gpu = allocateParticlesGPU(n);
        e->tree = allocateOctree(n);
        nbody_check_cuda(cudaMemset(e->tree.sort_idx, 0, n * sizeof(int)), "zero sort_idx");
        return e;
    } catch (const std::exception& ex) {
        std::snprintf(g_err, sizeof(g_err), "%s", ex.what());
        return nullptr;
    }
}

void ref_eng_destroy(void* h) {
    RefEngine* e = (RefEngine*)h;
    if (!e) return;
    freeOctree(e->tree);
    freeParticlesGPU(e->gpu);
    delete e;
}

int ref_eng_set_state(void* h, const float* x, const float* y, const float* z,
                      const float* vx, const float* vy, const float* vz, const float* ax,
                      const float* ay, const float* az, const float* m) {
    RefEngine* e = (RefEngine*)h;
    REF_TRY({
        ParticleData c = allocateParticlesCPU(e->n);
        size_t b = e->n * sizeof(float);
        std::memcpy(c.x, x, b); std::memcpy(c.y, y, b); std::memcpy(c.z, z, b);
        std::memcpy(c.vx, vx, b); std::memcpy(c.vy, vy, b); std::memcpy(c.vz, vz, b);
        std::memcpy(c.ax, ax, b); std::memcpy(c.ay, ay, b); std::memcpy(c.az, az, b);
        std::memcpy(c.mass, m, b);
        for (int i = 0; i < e->n; ++i) c.id[i] = i;
        copyToGPU(c, e->gpu);
        freeParticlesCPU(c);
    })
}

int ref_eng_get_state(void* h, float* x, float* y, float* z, float* vx, float* vy, float* vz,
                      float* ax, float* ay, float* az) {
    RefEngine* e = (RefEngine*)h;
    REF_TRY({
        ParticleData c = allocateParticlesCPU(e->n);
        copyToCPU(e->gpu, c);
        size_t b = e->n * sizeof(float);
        std::memcpy(x, c.x, b); std::memcpy(y, c.y, b); std::memcpy(z, c.z, b);
        std::memcpy(vx, c.vx, b); std::memcpy(vy, c.vy, b); std::memcpy(vz, c.vz, b);
        std::memcpy(ax, c.ax, b); std::memcpy(ay, c.ay, b); std::memcpy(az, c.az, b);
        freeParticlesCPU(c);
    })
}

// resetOctree .. launchSortKernel (src/main.cu:113-117)
int ref_eng_build(void* h) {
    RefEngine* e = (RefEngine*)h;
    REF_TRY({
        resetOctree(e->tree);
        launchBBoxKernel(e->tree, e->gpu);
        launchBuildKernel(e->tree, e->gpu);
        launchSummarizeKernel(e->tree);
        launchSortKernel(e->tree);
    })
}

// Reads back sort_idx and the root's mass/count after ref_eng_build.
int ref_eng_tree_info(void* h, int* sort_idx, float* root_mass, int* root_count,
                      int* next_node) {
    RefEngine* e = (RefEngine*)h;
    REF_TRY({
        int root = e->tree.n_total - 1;
        nbody_check_cuda(cudaMemcpy(sort_idx, e->tree.sort_idx, e->n * sizeof(int),
                                    cudaMemcpyDeviceToHost), "sort_idx");
        nbody_check_cuda(cudaMemcpy(root_mass, e->tree.mass + root, sizeof(float),
                                    cudaMemcpyDeviceToHost), "root mass");
        nbody_check_cuda(cudaMemcpy(root_count, e->tree.count + root, sizeof(int),
                                    cudaMemcpyDeviceToHost), "root count");
        nbody_check_cuda(cudaMemcpy(next_node, e->tree.next_node, sizeof(int),
                                    cudaMemcpyDeviceToHost), "next_node");
    })
}

// launchResetAccelerationKernel + launchForceKernel (+ perturber) on the built tree.
int ref_eng_force(void* h, float theta, float softening, float star_mass, int pert_on,
                  float px, float py, float pz, float pmass) {
    RefEngine* e = (RefEngine*)h;
    REF_TRY({
        launchResetAccelerationKernel(e->gpu);
        launchForceKernel(e->tree, e->gpu, theta, softening, star_mass);
        if (pert_on) launchPerturberForceKernel(e->gpu, px, py, pz, pmass, softening);
    })
}

int ref_eng_collide(void* h, float r_coll, float restitution) {
    RefEngine* e = (RefEngine*)h;
    REF_TRY(launchCollisionKernel(e->tree, e->gpu, r_coll, restitution))
}

int ref_eng_kick(void* h, float dt_half) {
    RefEngine* e = (RefEngine*)h;
    REF_TRY(launchHalfKickKernel(e->gpu, dt_half))
}

int ref_eng_drift(void* h, float dt) {
    RefEngine* e = (RefEngine*)h;
    REF_TRY(launchDriftKernel(e->gpu, dt))
}

int ref_eng_drag(void* h, float rate, float dt, float star_mass) {
    RefEngine* e = (RefEngine*)h;
    REF_TRY(launchGasDragKernel(e->gpu, rate, dt, star_mass))
}

int ref_eng_perturber_force(void* h, float px, float py, float pz, float pmass, float eps) {
    RefEngine* e = (RefEngine*)h;
    REF_TRY(launchPerturberForceKernel(e->gpu, px, py, pz, pmass, eps))
}

// The step loop of src/main.cu:101-139, steps [step0, step0+nsteps), with the
// perturber built by makePerturber from these fields.  *ms = wall time of the
// loop (every launcher synchronizes, so this is device time plus host gaps).
int ref_eng_steps(void* h, int step0, int nsteps, float dt, float theta, float softening,
                  float star_mass, float r_coll, float restitution, float drag_rate,
                  int pert_on, float pert_mjup, float pert_r, float pert_phase0, double* ms) {
    RefEngine* e = (RefEngine*)h;
    REF_TRY({
        Config cfg;
        cfg.star_mass_msun = star_mass;
        cfg.perturber_enabled = pert_on != 0;
        cfg.perturber_mass_mjup = pert_mjup;
        cfg.perturber_radius_AU = pert_r;
        cfg.perturber_phase0 = pert_phase0;
        Perturber pert = makePerturber(cfg);
        nbody_check_cuda(cudaDeviceSynchronize(), "pre-loop sync");
        auto t0 = std::chrono::steady_clock::now();
        for (int step = step0; step < step0 + nsteps; ++step) {
            launchHalfKickKernel(e->gpu, dt * 0.5f);
            launchDriftKernel(e->gpu, dt);
            float sim_time_now = static_cast<float>(step + 1) * dt;
            resetOctree(e->tree);
            launchBBoxKernel(e->tree, e->gpu);
            launchBuildKernel(e->tree, e->gpu);
            launchSummarizeKernel(e->tree);
            launchSortKernel(e->tree);
            launchResetAccelerationKernel(e->gpu);
            launchForceKernel(e->tree, e->gpu, theta, softening, star_mass);
            if (pert.enabled) {
                updatePerturber(pert, sim_time_now);
                launchPerturberForceKernel(e->gpu, pert.x, pert.y, pert.z, pert.mass_msun,
                                           softening);
            }
            launchCollisionKernel(e->tree, e->gpu, r_coll, restitution);
            launchHalfKickKernel(e->gpu, dt * 0.5f);
            launchGasDragKernel(e->gpu, drag_rate, dt, star_mass);
        }
        nbody_check_cuda(cudaDeviceSynchronize(), "post-loop sync");
        auto t1 = std::chrono::steady_clock::now();
        *ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    })
}

}  // extern "C"
