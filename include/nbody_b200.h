/*
 * nbody_b200.h -- C ABI of libnbody_b200.so, the B200 (sm_100a) engine for the
 * per-step path of ualiberik/nbody-sim: octree build, Barnes-Hut force walk,
 * perturber, two-pass collision impulse, KDK leapfrog + gas drag, FoF
 * aggregates and the frames.bin / stats.csv writers.
 *
 * Plain pointers and sizes only.  Every entry point returns NBODY_OK (0) or an
 * NBODY_ERR_* code; nbody_last_error() then gives a message (thread-local).
 * Each function below names the reference interface it replaces
 * (path:line within the reference project).
 *
 * Threading and synchronisation: the phase functions (nbody_tree_*,
 * nbody_half_kick, ...) mirror the reference launchers, which all return
 * after cudaDeviceSynchronize (include/Integrator.cuh:6, BHTree.cuh:42); they
 * run on the legacy default stream and synchronise it before returning.  The
 * engine functions (nbody_sim_*) are asynchronous on the engine's stream
 * until nbody_sim_sync().
 */
#ifndef NBODY_B200_H
#define NBODY_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NBODY_OK 0
#define NBODY_ERR_CUDA 1      /* a CUDA runtime call failed                         */
#define NBODY_ERR_ARG 2       /* bad argument (size mismatch, null pointer, range)  */
#define NBODY_ERR_OVERFLOW 3  /* a bounded device loop gave up (stack, union-find)  */
#define NBODY_ERR_TIMEOUT 4   /* reserved: a bounded wait expired                  */
#define NBODY_ERR_IO 5        /* file could not be opened / written                 */
#define NBODY_ERR_CONFIG 6    /* configuration rejected (loadConfig's checks)       */
#define NBODY_ERR_STATE 7     /* call out of order (e.g. force before build)        */

#define NBODY_ABI_VERSION 1

const char* nbody_last_error(void);
int nbody_abi_version(void);

/* ---------------------------------------------------------------- data --- */

/* SoA particle arrays; same fields, order and types as ParticleData
 * (include/ParticleData.h:19-32).  Pointers are device pointers for the phase
 * API, host or device (as stated) elsewhere. */
typedef struct nbody_particles {
  float* x;
  float* y;
  float* z;
  float* vx;
  float* vy;
  float* vz;
  float* ax;
  float* ay;
  float* az;
  float* mass;
  int* id;
  int n;
} nbody_particles;

/* Config (include/Config.h:4-36): same fields and defaults. */
typedef struct nbody_config {
  int n_particles;
  float disk_r_min;
  float disk_r_max;
  float disk_h_factor;
  float particle_mass_msun;
  float star_mass_msun;
  float softening_AU;
  float theta;
  float collision_radius_factor;
  float restitution;
  float gas_drag_rate;
  float dt;
  float total_time;
  int output_every_n_steps;
  char output_dir[1024];
  int perturber_enabled;
  float perturber_mass_mjup;
  float perturber_radius_AU;
  float perturber_phase0;
} nbody_config;

/* Config member initialisers (include/Config.h:5-35). */
void nbody_config_defaults(nbody_config* cfg);
/* loadConfig (src/config/Config.cpp:6-55): same keys, defaults, checks and
 * messages; NBODY_ERR_IO for an unreadable file, NBODY_ERR_CONFIG otherwise. */
int nbody_config_load(const char* path, nbody_config* cfg);
/* particlePhysicalRadius (src/disk/DiskInit.cpp:10-16), AU at 3000 kg/m^3. */
float nbody_particle_radius(float particle_mass_msun);

/* Perturber (include/Perturber.h:28-37). */
typedef struct nbody_perturber {
  int enabled;
  float r;
  float mass_msun;
  float phase0;
  float omega;
  float x, y, z;
} nbody_perturber;
/* makePerturber (include/Perturber.h:39-57). */
void nbody_perturber_make(const nbody_config* cfg, nbody_perturber* p);
/* updatePerturber (include/Perturber.h:60-66). */
void nbody_perturber_update(nbody_perturber* p, float sim_time);

/* ------------------------------------------------- octree phase API --- */

typedef struct nbody_tree nbody_tree;

/* allocateOctree (src/physics/BHTree.cu:358-381). */
int nbody_tree_create(int n_bodies, nbody_tree** out);
/* freeOctree (src/physics/BHTree.cu:383-395). */
void nbody_tree_destroy(nbody_tree* t);
/* resetOctree (src/physics/BHTree.cu:397-420): nothing to clear here (the
 * build overwrites every node it uses); resets the device status word. */
int nbody_tree_reset(nbody_tree* t);
/* launchBBoxKernel (src/physics/BHTree.cu:422-452): bbox of p->x,y,z padded
 * x1.001 about its middle, computed and padded on the device. */
int nbody_tree_bbox(nbody_tree* t, const nbody_particles* p);
/* launchBuildKernel (src/physics/BHTree.cu:454-499): Morton keys, radix sort,
 * Karras radix tree.  Runs the bbox itself if nbody_tree_bbox was not called. */
int nbody_tree_build(nbody_tree* t, const nbody_particles* p);
/* launchSummarizeKernel (src/physics/BHTree.cu:501-516): FP64 centre of mass
 * and mass of every node in one bottom-up pass, and the octree layout. */
int nbody_tree_summarize(nbody_tree* t);
/* launchSortKernel (src/physics/BHTree.cu:518-525): fills the tree's sort_idx
 * (nbody_tree_sort_idx) with the body order of the octree (Morton order). */
int nbody_tree_sort(nbody_tree* t);
/* tree.sort_idx (include/BHTree.cuh:20): device array of n_bodies ints. */
int* nbody_tree_sort_idx(nbody_tree* t);
/* Copies tree.sort_idx into dst (device if dst_on_device, else host), the
 * cudaMemcpy of tests/test_bhtree.cu:14. */
int nbody_tree_sort_idx_copy(nbody_tree* t, int* dst, int dst_on_device);
/* launchForceKernel (src/physics/BHTree.cu:600-609): OVERWRITES p->ax,ay,az
 * with the softened star pull plus the Barnes-Hut sum (theta = half-size over
 * distance to the centre of mass, BHTree.cu:577). */
int nbody_tree_force(nbody_tree* t, nbody_particles* p, float theta, float softening,
                     float star_mass);
/* launchCollisionKernel (src/physics/BHTree.cu:688-708): two-pass inelastic
 * impulse for pairs closer than r_coll; updates p->vx,vy,vz in place. */
int nbody_tree_collide(nbody_tree* t, nbody_particles* p, float r_coll, float restitution);
/* Collision miss report for the summarized tree (its own copy of the
 * positions): *pairs = ordered pairs (i, j != i) closer than r_coll, all of
 * which nbody_tree_collide applies; *missed = how many of them the
 * reference's traversal would skip, because its cell prune
 * |x_i - com| - 1.732 half >= r_coll (src/physics/BHTree.cu:663-665) drops a
 * cell whose centre of mass lies away from the body.  Cells below the tenth
 * octree level (inside buckets of equal 30-bit keys) are not modelled.
 * Synchronous. */
int nbody_tree_collision_report(nbody_tree* t, float r_coll, unsigned long long* pairs,
                                unsigned long long* missed);
/* Bodies opened directly instead of subdivided further (default 8). */
int nbody_tree_set_leaf_max(nbody_tree* t, int leaf_max);
/* Targets per lane of the force walk: 1 (warp groups of <= 32 bodies, the
 * default) or 2 (<= 64); takes effect at the next summarize. */
int nbody_tree_set_targets_per_lane(nbody_tree* t, int targets_per_lane);

typedef struct nbody_tree_stats {
  int n_bodies;
  int n_nodes;
  float bbox_min[3];   /* padded, as tree.bbox_min after launchBBoxKernel */
  float bbox_max[3];
  float root_center[3];
  float root_half;     /* cell_size of the root (BHTree.cu:484-485)      */
  double root_mass;
  double root_com[3];
  unsigned long long interactions; /* accepted interactions of the last force */
  int status;          /* device status bits of the last calls                */
  unsigned long long walk_nodes_visited;  /* node tests of the last force walk */
  unsigned long long walk_stack_spills;   /* stack spills of the last force walk */
} nbody_tree_stats;
int nbody_tree_stats_get(nbody_tree* t, nbody_tree_stats* out);

/* ---------------------------------------------- integrator / perturber --- */

/* launchHalfKickKernel (include/Integrator.cuh:9, Integrator.cu:80-85). */
int nbody_half_kick(nbody_particles* p, float dt_half);
/* launchDriftKernel (include/Integrator.cuh:12, Integrator.cu:87-92). */
int nbody_drift(nbody_particles* p, float dt);
/* launchResetAccelerationKernel (include/Integrator.cuh:15). */
int nbody_reset_acc(nbody_particles* p);
/* launchGasDragKernel (include/Integrator.cuh:21-22, Integrator.cu:100-109):
 * no-op when drag_rate <= 0; decay = expf(-drag_rate * dt) on the host. */
int nbody_gas_drag(nbody_particles* p, float drag_rate, float dt, float star_mass);
/* launchPerturberForceKernel (include/Perturber.h:73-75): ADDS the pull. */
int nbody_perturber_force(nbody_particles* p, float px, float py, float pz, float pmass,
                          float softening);

/* ------------------------------------------------------------- FoF --- */

/* GPU friends-of-friends over device positions x,y,z (n bodies), linking
 * pairs with ((dx*dx + dy*dy) + dz*dz) < link_length^2 in FP32 exactly as
 * detectAggregates (src/analysis/Aggregate.cpp:26-52).  Outputs (device):
 * labels[i] = smallest index in i's group, agg_size[i] = group size clamped
 * to 65535 or 1 for singletons (src/main.cu:153-161).  *n_groups (host) =
 * groups with >= 2 members.  Uses t's buffers (t must hold >= n bodies). */
int nbody_fof(nbody_tree* t, const float* x, const float* y, const float* z, int n,
              float link_length, int* labels, uint16_t* agg_size, int* n_groups);

/* Friends-of-friends without any device allocation.  No counterpart in the
 * reference: it is nbody_fof for callers that may not allocate device memory
 * when they need aggregates -- an analysis or visualisation process that
 * polls a running simulation's snapshots while the simulation has reserved
 * the rest of the GPU's memory; code whose device memory belongs to another
 * allocator (a framework's caching allocator, a pool sized at start-up); and
 * loops that must not stall, since cudaFree waits for the whole device and
 * cudaMalloc can block behind work in flight.  nbody_fof, by contrast, needs
 * an nbody_tree, which allocates.
 *
 * All scratch (sort buffers, tree, union-find arrays, a bounded stack-spill
 * area, and a set-up input) lives in one statically sized device array inside
 * libnbody_b200.so, NBODY_FOF_NOALLOC_SCRATCH_BYTES bytes (13.1 MiB).  n is
 * limited to NBODY_FOF_NOALLOC_MAX_N bodies; larger n returns NBODY_ERR_ARG
 * with a message naming the limit.  Inputs and outputs are as for nbody_fof
 * (device x, y, z, labels, agg_size; host *n_groups), bit-identical results.
 *
 * Set-up.  The first call on each device sets that device up, with the
 * device current: it looks up the device's address of the array
 * (cudaGetSymbolAddress) and runs the FoF once on a set-up input of
 * NBODY_FOF_NOALLOC_MAX_N bodies held in the array.  Under CUDA's lazy module
 * loading (the default) that first use is when the runtime backs the array
 * with device memory and loads the code of every kernel the call launches, so
 * the first call DOES take device memory (the array, about 13 MiB, plus
 * kernel code) and holds it until the process exits; later calls take none.
 * Make that first call at start-up, before the rest of the GPU's memory is
 * reserved and before any stream capture; a call with n = 0 (pointers other
 * than n_groups may then be NULL) does only the set-up.
 *
 * All calls on a device share the one array and each call overwrites it: the
 * function runs on the legacy default stream and synchronises before it
 * returns, so calls from one host thread never overlap, but calls that could
 * overlap on the GPU (other host threads, or the default stream in
 * per-thread mode) race on the scratch and must be serialised by the caller.
 * The function calls no cudaMalloc, cudaFree or allocating library routine. */
#define NBODY_FOF_NOALLOC_MAX_N 32768
#define NBODY_FOF_NOALLOC_SCRATCH_BYTES 13766144
int nbody_fof_noalloc(const float* x, const float* y, const float* z, int n, float link_length,
                      int* labels, uint16_t* agg_size, int* n_groups);

/* Aggregate (include/Aggregate.h:4-12) without the member list. */
typedef struct nbody_aggregate {
  int id;
  int n_particles;
  float mass_msun;
  float cx, cy, cz;
  float vx, vy, vz;
  float dist_center;
  int first_member;   /* smallest member index (the group's label) */
} nbody_aggregate;

/* Aggregate records of detectAggregates (Aggregate.cpp:54-74) from host
 * labels: groups of >= 2 ordered by smallest member, mass = n * particle
 * mass, mean position / velocity summed in ascending member index.
 * Writes at most max_aggs records; returns the group count in *n_aggs. */
int nbody_aggregates(const float* x, const float* y, const float* z, const float* vx,
                     const float* vy, const float* vz, const int* labels, int n,
                     float particle_mass, nbody_aggregate* out, int max_aggs, int* n_aggs);

/* --------------------------------------------------------- writers --- */

typedef struct nbody_writer nbody_writer;
/* OutputWriter::OutputWriter (src/io/OutputWriter.cpp:16-34): creates
 * dir/frames.bin (32-byte v2 header) and dir/stats.csv (15-column header). */
int nbody_writer_open(const char* dir, const nbody_config* cfg, nbody_writer** out);
/* OutputWriter::writeFrame (OutputWriter.cpp:96-115); host arrays. */
int nbody_writer_frame(nbody_writer* w, const float* x, const float* y, const float* z, int n,
                       float sim_time, const uint16_t* agg_size);
/* OutputWriter::writeStats (OutputWriter.cpp:124-148). */
int nbody_writer_stats(nbody_writer* w, const nbody_aggregate* aggs, int n_aggs, int frame_idx,
                       float sim_time);
/* OutputWriter::writePerturberStats (OutputWriter.cpp:161-186). */
int nbody_writer_perturber(nbody_writer* w, int frame_idx, float sim_time, int n_aggregates,
                           float px, float py, float pz, float mass_msun, float omega);
/* OutputWriter::finalize (OutputWriter.cpp:191-197). */
int nbody_writer_finalize(nbody_writer* w, int total_frames);
/* OutputWriter::~OutputWriter (OutputWriter.cpp:39-42). */
void nbody_writer_close(nbody_writer* w);

/* ------------------------------------------------------------ engine --- */
/* The whole step of src/main.cu:101-139 with the state resident on the GPU
 * in Morton order: one fused stream kernel (dv + K2 + drag + K1 + drift +
 * bbox), keys, sort, tree, walk (+ star, + perturber), collision. */

#define NBODY_STATE_F32 0    /* positions/velocities float (reference)     */
#define NBODY_STATE_F64 1    /* positions/velocities double                */
#define NBODY_STATE_F32X2 2  /* hi/lo float pairs (~48 bits), FP64 kicks   */

typedef struct nbody_sim_params {
  float dt;
  float theta;
  float softening;
  float star_mass;
  float r_coll;              /* <= 0: no collision pass                    */
  float restitution;
  float gas_drag_rate;       /* <= 0: no drag                              */
  int perturber_enabled;
  float perturber_mass_mjup;
  float perturber_radius_au;
  float perturber_phase0;
  int state_precision;       /* NBODY_STATE_*                              */
  int leaf_max;              /* <= 0: default (12 from 2^19 bodies, else 8;
                                an ensemble: 8)                             */
  int targets_per_lane;      /* walk: 1 (groups <= 32) or 2 (<= 64); 0: 1  */
  int walk_mode;             /* walk kernel variant (1 target per lane):
                                0 acceptance vote, 96 registers; 1
                                (default) vote, 64 registers; 2 no vote,
                                64 registers.  Same forces to the walk's
                                approximation level; speed depends on the
                                disk (2 suits many small compact disks). */
  int group_span;            /* walk target groups: maximal tree nodes of
                                <= group_span x 32 x targets_per_lane
                                bodies cut into equal runs of <= 32 x
                                targets_per_lane; 1 .. 64.  Larger spans
                                fill the warps better and give each group
                                a larger box.  <= 0: automatic (8 for a
                                simulation of >= 2^19 bodies, else 1; 1
                                for an ensemble).                          */
  int fuse_collisions;       /* 0 (default): the collision impulse comes from
                                a neighbour search over the step's tree
                                (launchCollisionKernel's pairs), run on a
                                second stream beside the force walk; 1: it
                                is found inside the force walk, among each
                                group's own sources (no second tree walk).
                                Same pairs; a body's impulses are summed in
                                another order.                            */
  int span_walk;             /* shared walk: 1 on when the target groups
                                come from span nodes of more than one group
                                (group_span > 1, unfused collisions, one
                                target per lane); 0 (default) or 2 off.  The
                                groups of one span node
                                share a first traversal with the node's box,
                                which decides what every group would decide
                                alike; each group then starts from the
                                shared sources and the frontier left.  Same
                                interactions as a walk from the root, summed
                                in another order.                          */
  int spill_cap;             /* walk / neighbour-search stack entries per
                                warp kept in HBM when the shared-memory
                                stack is full; <= 0: default (4096).  A
                                walk that needs more stops, and the step
                                reports NBODY_ERR_OVERFLOW (status bit 1). */
} nbody_sim_params;

/* Parameters of src/main.cu:58-73 from a Config (r_coll = factor * radius). */
void nbody_sim_params_from_config(const nbody_config* cfg, nbody_sim_params* out);

typedef struct nbody_sim nbody_sim;
int nbody_sim_create(const nbody_sim_params* p, int n, nbody_sim** out);
void nbody_sim_destroy(nbody_sim* s);
/* Runs on this CUDA stream (a cudaStream_t); 0 = the legacy default stream. */
int nbody_sim_set_stream(nbody_sim* s, void* cuda_stream);
/* State in the caller's particle order (index i = particle id i).  on_device:
 * pointers are device (1) or host (0).  Mass is float.  Setting the state
 * resets the step counter and computes the forces at t = 0 (main.cu:85-96). */
int nbody_sim_set_state(nbody_sim* s, const float* x, const float* y, const float* z,
                        const float* vx, const float* vy, const float* vz, const float* mass,
                        int on_device);
int nbody_sim_set_state_f64(nbody_sim* s, const double* x, const double* y, const double* z,
                            const double* vx, const double* vy, const double* vz,
                            const float* mass, int on_device);
/* Advances nsteps steps (asynchronous). */
int nbody_sim_step(nbody_sim* s, int nsteps);
/* Advances nsteps steps and leaves the last one open: its second kick and
 * drag (src/main.cu:133-138) stay pending, so the next step's first kernel
 * does them together with that step's first kick and drift, as every step
 * inside one nbody_sim_step call does.  The engine closes a pending step
 * itself before any read of the state (get_state, fof, output_begin,
 * autotune) and nbody_sim_step finishes one; nbody_sim_close does only
 * that.  For callers that advance one step per call in a loop. */
int nbody_sim_step_open(nbody_sim* s, int nsteps);
int nbody_sim_close(nbody_sim* s);
/* Waits for the engine's stream and reports device status bits as errors. */
int nbody_sim_sync(nbody_sim* s);
/* State after the last step, in the caller's order (acceleration pointers may
 * be null).  Synchronises. */
int nbody_sim_get_state(nbody_sim* s, float* x, float* y, float* z, float* vx, float* vy,
                        float* vz, float* ax, float* ay, float* az, int on_device);
int nbody_sim_get_state_f64(nbody_sim* s, double* x, double* y, double* z, double* vx,
                            double* vy, double* vz, int on_device);
/* FoF of the current positions (FP32 snapshot), outputs in caller order. */
int nbody_sim_fof(nbody_sim* s, float link_length, int* labels, uint16_t* agg_size,
                  int* n_groups, int on_device);

typedef struct nbody_sim_stats {
  int n;
  int steps_done;
  int n_nodes;
  unsigned long long interactions;  /* accepted interactions of the last walk */
  int status;
  unsigned long long walk_nodes_visited;  /* node tests of the last walk */
  unsigned long long walk_stack_spills;   /* stack spills of the last walk */
  unsigned long long walk_groups;         /* warp groups of the last walk */
  unsigned long long launches;            /* kernels launched so far (graph nodes included) */
  unsigned long long graph_launches;      /* steps replayed as one CUDA graph */
  int targets_per_lane;                   /* the walk settings in use (after */
  int leaf_max;                           /* nbody_sim_autotune, the kept    */
  int walk_mode;                          /* candidate)                      */
  int group_span;
  int span_walk;                          /* 1: the last walk was shared     */
  unsigned long long span_shared;         /* shared-walk entries of the last */
  unsigned long long span_frontier;       /* walk (span-decided sources and  */
  unsigned long long spans;               /* frontier nodes) and its spans   */
} nbody_sim_stats;
int nbody_sim_stats_get(nbody_sim* s, nbody_sim_stats* out);
/* 1 (default): each step is replayed as one CUDA graph (captured on first
 * use, four variants); 0: its kernels are launched one by one.  Steps run
 * while profiling is on are always launched one by one. */
/* Walk autotuner (as nbody_ensemble_autotune; no reference counterpart):
 * times two force evaluations of the current state for each candidate
 * (targets_per_lane, leaf_max, walk_mode, group_span) in candidates[4k ..
 * 4k+3] (NULL: a built-in list of 6; group_span <= 0: automatic) and keeps
 * the fastest.  The best variant depends on the disk, and the choice holds
 * for the state it was timed on: on the C2 disk (N = 131072, collisions)
 * mode 2 is the faster at t = 0 but 20% slower over a 2000-step run, as
 * the disk evolves; re-tune along a run.  The forces of the current time are
 * recomputed with the kept setting (state unchanged; the next step's
 * collision pass is not affected).  Synchronous; ms_out (optional) receives
 * each candidate's time. */
int nbody_sim_autotune(nbody_sim* s, const int* candidates, int n_candidates, float* ms_out);
int nbody_sim_set_graphs(nbody_sim* s, int on);

/* Per-phase device time of the steps run while profiling is on: CUDA events
 * at the phase boundaries of every step, on the engine's stream.  Phase k of
 * a step runs from its boundary k to boundary k+1; the stream phase also
 * holds the closing dv + K2 + drag of the call's last step.  With graphs on
 * (the default) each profiled step is captured with the events as nodes of
 * its graph, so the phases are timed as the step graphs run them. */
#define NBODY_PHASE_STREAM 0   /* dv + K2 + drag + K1 + drift + bbox          */
#define NBODY_PHASE_SORT 1     /* Morton keys + radix sort                    */
#define NBODY_PHASE_PERMUTE 2  /* state gathered into key order               */
#define NBODY_PHASE_TREE 3     /* Karras tree, FP64 moments, octree layout    */
#define NBODY_PHASE_WALK 4     /* Barnes-Hut walk (+ star, + perturber)       */
#define NBODY_PHASE_COLLIDE 5  /* collision neighbour search                  */
#define NBODY_PHASES 6
typedef struct nbody_sim_profile {
  double ms[NBODY_PHASES];   /* summed over the profiled steps */
  int steps;
  unsigned long long launches;  /* kernels launched by nbody_sim_step */
} nbody_sim_profile;
int nbody_sim_set_profiling(nbody_sim* s, int on);
/* Synchronises, then returns the sums since the last reset. */
int nbody_sim_profile_get(nbody_sim* s, nbody_sim_profile* out, int reset);

/* Host-buffer round trip, the per-call work of a caller that keeps its
 * ParticleData on the host (copyToGPU, nsteps of src/main.cu:101-139,
 * copyToCPU; include/ParticleData.h:90-123): copies x..az and mass in,
 * advances nsteps with the given accelerations as the current forces, copies
 * x..az back out.  The step counter (simulation time) continues across calls.
 * NBODY_STATE_F32 only.  Synchronous. */
int nbody_sim_step_host(nbody_sim* s, float* x, float* y, float* z, float* vx, float* vy,
                        float* vz, float* ax, float* ay, float* az, const float* mass,
                        int nsteps);

/* Output step of src/main.cu:143-181 on the GPU, overlapped with the steps
 * that follow.  nbody_sim_output_begin enqueues, behind the steps issued so
 * far: a snapshot of the state (caller order), FoF of the snapshot with the
 * Aggregate.cpp:36-42 pair test, agg_size (main.cu:153-161), the aggregate
 * records of detectAggregates (Aggregate.cpp:54-74, bit for bit, ordered by
 * smallest member), and their copy into pinned host memory.  It returns at
 * once; the engine may keep stepping.  nbody_sim_output_wait blocks for the
 * oldest frame in flight and points *out at the engine's pinned buffers.
 * Two frames can be in flight; a frame's buffers stay valid until the second
 * output_begin after its wait (the slot it used comes round again). */
typedef struct nbody_frame {
  int n;
  int frame_index;
  float sim_time;
  const float* x;                     /* host, caller order */
  const float* y;
  const float* z;
  const uint16_t* agg_size;           /* main.cu:153-161 */
  const nbody_aggregate* aggregates;  /* ordered by smallest member */
  int n_aggregates;
} nbody_frame;
int nbody_sim_output_begin(nbody_sim* s, float link_length, float particle_mass,
                           float sim_time, int frame_index);
int nbody_sim_output_wait(nbody_sim* s, nbody_frame* out);

/* ----------------------------------------------------------- ensemble --- */

/* Many independent disks advanced together.  The reference runs one disk per
 * process (src/main.cu:101-139); an ensemble runs every disk's step order
 * (main.cu:101-139 per disk) with each phase one launch over all disks, and a
 * whole step replayed as one CUDA graph.  Disks share dt, theta, softening,
 * star mass, collision radius, restitution, drag and precision (the
 * nbody_sim_params); each has its own body count and perturber
 * (src/physics/Perturber.h:39-58).  A body feels only its own disk, its star
 * and its perturber: results equal those of separate nbody_sim runs up to the
 * float summation order of the tree walk. */
typedef struct nbody_disk_spec {
  int n;                      /* bodies, >= 2 */
  int perturber_enabled;
  float perturber_mass_mjup;
  float perturber_radius_au;
  float perturber_phase0;
} nbody_disk_spec;

typedef struct nbody_ensemble nbody_ensemble;

int nbody_ensemble_create(const nbody_sim_params* p, const nbody_disk_spec* disks, int n_disks,
                          nbody_ensemble** out);
int nbody_ensemble_destroy(nbody_ensemble* e);
int nbody_ensemble_set_stream(nbody_ensemble* e, void* cuda_stream);
/* State of all disks concatenated in disk order (disk 0's bodies first),
 * host or device SoA; computes the forces at t = 0. */
int nbody_ensemble_set_state(nbody_ensemble* e, const float* x, const float* y, const float* z,
                             const float* vx, const float* vy, const float* vz,
                             const float* mass, int on_device);
int nbody_ensemble_set_state_f64(nbody_ensemble* e, const double* x, const double* y,
                                 const double* z, const double* vx, const double* vy,
                                 const double* vz, const float* mass, int on_device);
/* nsteps steps of every disk; asynchronous on the ensemble's stream. */
int nbody_ensemble_step(nbody_ensemble* e, int nsteps);
int nbody_ensemble_sync(nbody_ensemble* e);
int nbody_ensemble_get_state(nbody_ensemble* e, float* x, float* y, float* z, float* vx,
                             float* vy, float* vz, float* ax, float* ay, float* az,
                             int on_device);
int nbody_ensemble_get_state_f64(nbody_ensemble* e, double* x, double* y, double* z,
                                 double* vx, double* vy, double* vz, float* ax, float* ay,
                                 float* az, int on_device);
/* Host round trip, as nbody_sim_step_host: loads x..vz (double) and the
 * accelerations of that state, advances nsteps without recomputing the
 * starting forces, writes x..az back.  The step counter continues across
 * calls.  Synchronous. */
int nbody_ensemble_step_host(nbody_ensemble* e, double* x, double* y, double* z, double* vx,
                             double* vy, double* vz, float* ax, float* ay, float* az,
                             const float* mass, int nsteps);
/* Force-evaluation autotuner: times force evaluations of the current state
 * for each (targets_per_lane, leaf_max, walk_mode) candidate
 * (candidates[3k .. 3k+2]; NULL = the built-in list of 6) and keeps the
 * fastest (best of two timings each).  The
 * forces are recomputed with the kept setting, so the state is unchanged.
 * Needs set_state first.  ms_out (optional) receives each candidate's time. */
int nbody_ensemble_autotune(nbody_ensemble* e, const int* candidates, int n_candidates,
                            float* ms_out);
/* 0: launch the step's kernels one by one; 1 (default): replay CUDA graphs. */
int nbody_ensemble_set_graphs(nbody_ensemble* e, int on);
typedef struct nbody_ensemble_stats {
  int n_disks;
  int n_total;
  int steps_done;
  int targets_per_lane;
  int leaf_max;
  int status;
  unsigned long long interactions;  /* accepted interactions of the last walk */
  unsigned long long launches;      /* kernels launched so far (graph nodes included) */
  unsigned long long graph_launches;
  int walk_mode;
} nbody_ensemble_stats;
int nbody_ensemble_stats_get(nbody_ensemble* e, nbody_ensemble_stats* out);

/* ------------------------------------------------------------ adjoint --- */

/* Reverse-mode derivatives of one disk's trajectory.  The step is the
 * reference's order (src/main.cu:101-139: K1, drift, tree + force, perturber,
 * K2, gas drag; collisions are not differentiable and must be off) with FP64
 * state, FP32 tree-walk self-gravity, and FP64 star, perturber and drag; the
 * perturber moves on the orbit of updatePerturber (Perturber.h:60-66)
 * evaluated in FP64.  The forward records a tape in device memory -- every
 * level's state, sort permutation, warp groups and source lists -- and the
 * backward is the exact adjoint of that computation with the tree frozen.
 * nbody_adjoint_replay runs the same frozen-tree forward from other initial
 * conditions or perturber parameters (the function the backward
 * differentiates; for finite-difference checks).  No reference counterpart:
 * the reference has no derivatives.  All arrays are device arrays in caller
 * order; calls are synchronous. */
typedef struct nbody_adjoint nbody_adjoint;
int nbody_adjoint_create(const nbody_sim_params* p, int n, int n_steps, nbody_adjoint** out);
/* How the backward gets at the forward's levels:
 *  NBODY_ADJOINT_TAPE        (nbody_adjoint_create) every level's FP64 state
 *                            and tape stay in HBM; the backward recomputes
 *                            nothing.
 *  NBODY_ADJOINT_CHECKPOINT  only FP64 states every checkpoint_every levels are
 *                            kept; the backward rebuilds each level by running
 *                            the step backwards in time (time-reversed
 *                            leapfrog, drag inverted in closed form) from the
 *                            level after it, re-records its tree and tape, and
 *                            restarts each segment from its exact checkpoint;
 *                            two levels of state and tape are held.  No replay.
 *  NBODY_ADJOINT_DIRECT      self-gravity by FP64 direct summation over every
 *                            pair instead of the tree (O(N^2) per step, every
 *                            level kept): the reference gradient of the same
 *                            loss; replay runs the direct-sum dynamics. */
#define NBODY_ADJOINT_TAPE 0
#define NBODY_ADJOINT_CHECKPOINT 1
#define NBODY_ADJOINT_DIRECT 2
int nbody_adjoint_create_mode(const nbody_sim_params* p, int n, int n_steps, int mode,
                              int checkpoint_every, nbody_adjoint** out);
int nbody_adjoint_destroy(nbody_adjoint* a);
int nbody_adjoint_set_stream(nbody_adjoint* a, void* cuda_stream);
/* Records n_steps steps from (x0..vz0, mass) with the perturber at
 * perturber_radius_au (M_J mass perturber_mass_mjup; params' phase and
 * enable flag); writes the final state (outputs may be NULL). */
int nbody_adjoint_forward(nbody_adjoint* a, const double* x0, const double* y0, const double* z0,
                          const double* vx0, const double* vy0, const double* vz0,
                          const float* mass, double perturber_mass_mjup,
                          double perturber_radius_au, double* x, double* y, double* z,
                          double* vx, double* vy, double* vz);
/* fp64 = 1: the interactions in FP64 (sources at their FP64 positions and
 * centres of mass) -- the finite-difference reference, free of the FP32
 * rounding that a perturbed body's own terms add to a difference quotient. */
int nbody_adjoint_replay(nbody_adjoint* a, const double* x0, const double* y0, const double* z0,
                         const double* vx0, const double* vy0, const double* vz0,
                         double perturber_mass_mjup, double perturber_radius_au, int fp64,
                         double* x, double* y, double* z, double* vx, double* vy, double* vz);
/* Adjoint (dL/d final state) -> dL/d initial state and
 * g_perturber[0] = dL/d mass (per M_J), g_perturber[1] = dL/d radius (per AU). */
int nbody_adjoint_backward(nbody_adjoint* a, const double* gx, const double* gy, const double* gz,
                           const double* gvx, const double* gvy, const double* gvz,
                           double* gx0, double* gy0, double* gz0, double* gvx0, double* gvy0,
                           double* gvz0, double* g_perturber);
typedef struct nbody_adjoint_stats {
  int n;
  int n_steps;
  float ms_forward;    /* device time of the last recorded forward  */
  float ms_backward;   /* device time of the last backward           */
  float ms_replay;     /* device time of the last replay             */
  unsigned long long tape_bytes;
  unsigned long long state_bytes;
  unsigned long long launches;
} nbody_adjoint_stats;
int nbody_adjoint_stats_get(nbody_adjoint* a, nbody_adjoint_stats* out);

/* -------------------------------------------------------- diagnostics --- */

/* FP64 direct sum of the softened self-gravity (no star term) for a list of
 * targets: a_t = sum_{j != i} m_j d / (|d|^2 + eps^2)^{3/2} and
 * phi_t = -sum_{j != i} m_j / (|d|^2 + eps^2)^{1/2}, i = targets[t] (targets
 * NULL: every body, n_targets ignored).  The yardstick for the walk's force
 * error and the pair term of the softened energy.  No reference counterpart
 * (the reference has no accuracy diagnostics).  Device arrays; any output may
 * be NULL; synchronous. */
int nbody_direct_f64(const double* x, const double* y, const double* z, const float* mass, int n,
                     const int* targets, int n_targets, double eps, double* ax, double* ay,
                     double* az, double* phi);

/* Stable LSD radix sort of (key, value) pairs in place on device arrays, by
 * the low `bits` key bits (1..32 for 32-bit keys, 1..64 for 64-bit): the sort
 * behind the body order of every octree (launchSortKernel's sort_idx,
 * src/physics/BHTree.cu:518-525, comes out of it).  Scratch is allocated and
 * freed per call; synchronous on the legacy stream.  Returns NBODY_ERR_CUDA
 * if a tile's look-back wait gave up. */
int nbody_radix_sort_u32(uint32_t* keys, uint32_t* values, int n, int bits);
int nbody_radix_sort_u64(uint64_t* keys, uint32_t* values, int n, int bits);
/* The binary radix tree (Karras 2012) of n sorted keys, the structure the
 * octree build starts from (it replaces the CAS insertion of
 * bhtree_buildKernel, src/physics/BHTree.cu:175-277).  Device arrays of n - 1
 * internal nodes: children left/right (internal node i, or leaf j encoded as
 * n - 1 + j), key range lo..hi, and the common prefix within the low
 * key_bits.  Equal keys are split by their index.  Synchronous; allocates
 * its own work space. */
int nbody_radix_tree_u32(const uint32_t* keys, int n, int key_bits, int* left, int* right,
                         int* lo, int* hi, uint8_t* prefix);
/* Self-test of the radix sort's one bounded wait (no counterpart in the
 * reference, whose DFS sort is one serial thread, BHTree.cu:322-352): the
 * look-back of a tile over predecessor status words that no tile publishes.
 * The wait must give up after its bound (about a second) instead of hanging;
 * *status_bits receives the device status bits it raised (32, the bit a real
 * sort reports as NBODY_ERR_OVERFLOW / NBODY_ERR_CUDA).  Synchronous. */
int nbody_selftest_sort_wait(int* status_bits);

/* ------------------------------------------------------ initial disks --- */

/* Synthetic disk of n bodies: star mass at the origin, disk in XZ, +Y pole;
 * r from Sigma ~ r^-1.5 (inverse CDF as src/disk/DiskInit.cpp:42-44), Rayleigh
 * eccentricity/inclination (sigma_e, sigma_i), uniform node / periapsis /
 * mean anomaly, Keplerian state (G = 1), FP64 then rounded.  Counter-based
 * RNG (splitmix64 of seed, index, draw), so any subset is reproducible.
 * Host arrays; x..vz double. */
int nbody_make_disk(int n, double r_min, double r_max, double sigma_e, double sigma_i,
                    double star_mass, uint64_t seed, double* x, double* y, double* z,
                    double* vx, double* vy, double* vz);

/* The same disks generated on the GPU, many at once (an ensemble's initial
 * conditions): disk d has counts[d] bodies and seed seeds[d] (host arrays);
 * outputs are device arrays with the disks concatenated in order.  Body for
 * body the arithmetic of nbody_make_disk; the two differ only in the last-ulp
 * rounding of the device and host math libraries.  Synchronous on stream
 * (NULL: the legacy stream). */
int nbody_make_disks_device(const int* counts, const uint64_t* seeds, int n_disks,
                            double r_min, double r_max, double sigma_e, double sigma_i,
                            double star_mass, double* x, double* y, double* z, double* vx,
                            double* vy, double* vz, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* NBODY_B200_H */
