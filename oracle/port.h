/*
 * oracle/port.h -- CPU restatement of the reference engine's per-step path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the nbody-sim_b200
 * package, its CUDA library or the C++ drop-in headers) may include, link or
 * call this code.  It is imported by tests/, by __graft_entry__.smoke() as the
 * checker, and by bench.py's cpu_baseline / --impl reference leg as the timed
 * CPU baseline.
 *
 * Parity pins: the restatement is checked bit-for-bit against the reference's
 * own CUDA engine compiled from src/physics/*.cu with -fmad=false
 * (oracle/_ref, GPU tests), and against the known-answer tests of the
 * reference's tests/*.cu|cpp (CPU tests).  All float arithmetic here is FP32
 * with contraction disabled (-ffp-contract=off), which is what the reference's
 * kernels compute under -fmad=false, since sqrtf and '/' are IEEE on both.
 */
#ifndef NBODY_ORACLE_PORT_H
#define NBODY_ORACLE_PORT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Octree in the reference layout (include/BHTree.cuh:13-36): slots
 * [0, n_bodies) are one-body leaves, internal nodes are allocated upward from
 * n_bodies, the root is slot n_total-1, child[node*8+k] = -1 when empty. */
typedef struct {
    int    n_bodies;
    int    n_total;
    float *pos_x, *pos_y, *pos_z, *mass, *cell_size;
    int   *child, *count, *start, *sort_idx;
    int    next_node;
    float  bbox_min[3], bbox_max[3];
    int    lost_bodies;      /* bodies dropped by the 128-iteration / overflow limits */
    int    unsummarized;     /* internal nodes left with count 0 by summarize        */
} orc_tree;

int  orc_tree_alloc(orc_tree* t, int n_bodies);
void orc_tree_free(orc_tree* t);
/* resetOctree + launchBBoxKernel + launchBuildKernel (BHTree.cu:397-499). */
void orc_tree_build(orc_tree* t, const float* x, const float* y, const float* z,
                    const float* m, int n);
/* launchSummarizeKernel run to convergence (BHTree.cu:282-317,501-516). */
void orc_tree_summarize(orc_tree* t);
/* launchSortKernel (BHTree.cu:322-352,518-525). */
void orc_tree_sort(orc_tree* t);
/* launchForceKernel (BHTree.cu:530-609): OVERWRITES a. nthreads<=0: all cores. */
void orc_force(const orc_tree* t, const float* x, const float* y, const float* z,
               float* ax, float* ay, float* az,
               float theta, float softening, float star_mass, int nthreads);
/* Same walk, counting accepted interactions per body (opening tests excluded). */
long long orc_force_count(const orc_tree* t, const float* x, const float* y,
                          const float* z, float theta, int nthreads);
/* launchCollisionKernel (BHTree.cu:611-708): both passes, v updated in place. */
void orc_collision(const orc_tree* t, const float* x, const float* y, const float* z,
                   float* vx, float* vy, float* vz, float r_coll, float restitution,
                   int nthreads);
long long orc_collision_pairs(const orc_tree* t, const float* x, const float* y, const float* z,
                              float r_coll, int nthreads);

/* Integrator.cu:7-76 and the launchers' host-side arithmetic (:80-109). */
void orc_half_kick(float* vx, float* vy, float* vz, const float* ax, const float* ay,
                   const float* az, float dt_half, int n);
void orc_drift(float* x, float* y, float* z, const float* vx, const float* vy,
               const float* vz, float dt, int n);
void orc_reset_acc(float* ax, float* ay, float* az, int n);
void orc_gas_drag(const float* x, const float* y, const float* z, float* vx, float* vy,
                  float* vz, float drag_rate, float dt, float star_mass, int n);

/* Perturber.h:39-66 (host analytic orbit) and Perturber.cu:13-51 (pull). */
typedef struct { int enabled; float r, mass_msun, phase0, omega, x, y, z; } orc_perturber;
void orc_perturber_make(orc_perturber* p, int enabled, float mass_mjup, float radius_au,
                        float phase0, float star_mass);
void orc_perturber_update(orc_perturber* p, float sim_time);
void orc_perturber_force(float* ax, float* ay, float* az, const float* x, const float* y,
                         const float* z, float px, float py, float pz, float pmass,
                         float softening, int n);

/* One full step of src/main.cu:101-139 on host arrays (FP32 state). The tree
 * is rebuilt inside; a must hold the forces of the current positions. */
typedef struct {
    float dt, theta, softening, star_mass, r_coll, restitution, gas_drag_rate;
    int   collisions;        /* launchCollisionKernel is called every step in main.cu */
    orc_perturber pert;
} orc_step_params;
void orc_compute_forces(orc_tree* t, const float* x, const float* y, const float* z,
                        const float* m, float* ax, float* ay, float* az, int n,
                        const orc_step_params* sp, float sim_time, int nthreads);
void orc_step(orc_tree* t, float* x, float* y, float* z, float* vx, float* vy, float* vz,
              float* ax, float* ay, float* az, const float* m, int n,
              orc_step_params* sp, int step_index, int nthreads);

/* detectAggregates (src/analysis/Aggregate.cpp:26-76), O(N^2) union-find.
 * labels[i] = smallest member index of i's group; agg_size[i] = group size
 * clamped to 65535, or 1 for singletons (src/main.cu:153-161).  Returns the
 * number of groups with >= 2 members. */
int orc_fof(const float* x, const float* y, const float* z, int n, float link_length,
            int* labels, unsigned short* agg_size);
/* Aggregates of orc_fof's labels, ordered by smallest member index: n, mass
 * (n * particle_mass), mean position and velocity summed in ascending member
 * index, distance from the origin (Aggregate.cpp:54-74). Arrays of n_groups. */
void orc_fof_aggregates(const float* x, const float* y, const float* z, const float* vx,
                        const float* vy, const float* vz, int n, const int* labels,
                        float particle_mass, int n_groups, int* g_n, float* g_mass,
                        float* g_c /*3*n_groups*/, float* g_v /*3*n_groups*/,
                        float* g_dist, int* g_label);

/* FP64 direct summation (softened, star included) on a subset of targets. */
void orc_direct_f64(const double* x, const double* y, const double* z, const double* m,
                    int n, const int* targets, int n_targets, double softening,
                    double star_mass, int include_star, double* ax, double* ay,
                    double* az, int nthreads);
/* Softened total energy and vertical angular momentum L_y in FP64. */
void orc_energy_f64(const double* x, const double* y, const double* z, const double* vx,
                    const double* vy, const double* vz, const double* m, int n,
                    double softening, double star_mass, double* energy, double* ly,
                    int nthreads);

/* The fixed-pass summarize of the reference (launchSummarizeKernel,
 * BHTree.cu:501-516).  orc_set_summarize_passes(20) makes every later
 * orc_compute_forces / orc_step use it instead of the converged sweep (0
 * restores the sweep); used to time the reference's own summarize work. */
void orc_tree_summarize_passes(orc_tree* t, int passes, int nthreads);
void orc_set_summarize_passes(int passes);

/* The synthetic Keplerian disk recipe of the product's nbody_make_disk,
 * restated for callers that must not load the product (FP64 SoA out). */
void orc_make_disk(int n, double r_min, double r_max, double sigma_e, double sigma_i,
                   double mu, uint64_t seed, double* x, double* y, double* z, double* vx,
                   double* vy, double* vz);

#ifdef __cplusplus
}
#endif
#endif
