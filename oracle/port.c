/*
 * oracle/port.c -- CPU restatement of the reference engine (see port.h).
 *
 * TEST INFRASTRUCTURE ONLY: the checker and the timed CPU baseline, never the
 * product.  Every function names the reference file:line it restates.  Built
 * with -O2 -ffp-contract=off so that each FP32 expression rounds exactly like
 * the reference kernels compiled with -fmad=false (IEEE sqrtf and '/').
 */
#include "port.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static void set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
    else omp_set_num_threads(omp_get_num_procs());
#else
    (void)nthreads;
#endif
}

/* ------------------------------------------------------------------ tree */

int orc_tree_alloc(orc_tree* t, int n) {
    memset(t, 0, sizeof(*t));
    t->n_bodies = n;
    t->n_total = n + 8 * n; /* BHTree.cuh:4 MAX_NODES_MULT, BHTree.cu:361 */
    size_t nt = (size_t)t->n_total;
    t->pos_x = (float*)malloc(nt * sizeof(float));
    t->pos_y = (float*)malloc(nt * sizeof(float));
    t->pos_z = (float*)malloc(nt * sizeof(float));
    t->mass = (float*)malloc(nt * sizeof(float));
    t->cell_size = (float*)malloc(nt * sizeof(float));
    t->child = (int*)malloc(nt * 8 * sizeof(int));
    t->count = (int*)malloc(nt * sizeof(int));
    t->start = (int*)malloc(nt * sizeof(int));
    t->sort_idx = (int*)malloc((size_t)n * sizeof(int));
    if (!t->pos_x || !t->pos_y || !t->pos_z || !t->mass || !t->cell_size || !t->child ||
        !t->count || !t->start || !t->sort_idx) {
        orc_tree_free(t);
        return -1;
    }
    return 0;
}

void orc_tree_free(orc_tree* t) {
    free(t->pos_x); free(t->pos_y); free(t->pos_z); free(t->mass); free(t->cell_size);
    free(t->child); free(t->count); free(t->start); free(t->sort_idx);
    memset(t, 0, sizeof(*t));
}

/* bhtree_getOctant, BHTree.cu:164-170 */
static int octant(float cx, float cy, float cz, float px, float py, float pz) {
    return ((px > cx) ? 1 : 0) | ((py > cy) ? 2 : 0) | ((pz > cz) ? 4 : 0);
}

void orc_tree_build(orc_tree* t, const float* x, const float* y, const float* z,
                    const float* m, int n) {
    const int nt = t->n_total;
    /* bhtree_resetKernel, BHTree.cu:42-71 */
    for (int i = 0; i < nt; ++i) {
        t->count[i] = 0; t->start[i] = -1; t->mass[i] = 0.f;
        t->pos_x[i] = 0.f; t->pos_y[i] = 0.f; t->pos_z[i] = 0.f; t->cell_size[i] = 0.f;
    }
    for (long i = 0; i < 8L * nt; ++i) t->child[i] = -1;
    for (int i = 0; i < n; ++i) t->sort_idx[i] = -1;
    t->lost_bodies = 0;
    t->unsummarized = 0;

    /* bhtree_bboxKernel, BHTree.cu:76-134: exact min/max (fminf/fmaxf). */
    float bmin[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, bmax[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = 0; i < n; ++i) {
        bmin[0] = fminf(bmin[0], x[i]); bmax[0] = fmaxf(bmax[0], x[i]);
        bmin[1] = fminf(bmin[1], y[i]); bmax[1] = fmaxf(bmax[1], y[i]);
        bmin[2] = fminf(bmin[2], z[i]); bmax[2] = fmaxf(bmax[2], z[i]);
    }
    /* host padding, launchBBoxKernel BHTree.cu:440-446 */
    for (int i = 0; i < 3; ++i) {
        float mid = (bmin[i] + bmax[i]) * 0.5f;
        float half = (bmax[i] - bmin[i]) * 0.5f * 1.001f;
        bmin[i] = mid - half;
        bmax[i] = mid + half;
    }
    memcpy(t->bbox_min, bmin, sizeof(bmin));
    memcpy(t->bbox_max, bmax, sizeof(bmax));

    /* bhtree_copyLeafDataKernel / setLeafCount, BHTree.cu:139-159 */
    for (int i = 0; i < n; ++i) {
        t->pos_x[i] = x[i]; t->pos_y[i] = y[i]; t->pos_z[i] = z[i];
        t->mass[i] = m[i]; t->count[i] = 1;
    }
    /* root geometry, launchBuildKernel BHTree.cu:481-490 (and :187-191) */
    const float rcx = (bmin[0] + bmax[0]) * 0.5f;
    const float rcy = (bmin[1] + bmax[1]) * 0.5f;
    const float rcz = (bmin[2] + bmax[2]) * 0.5f;
    const float rhs = fmaxf(fmaxf(bmax[0] - bmin[0], bmax[1] - bmin[1]), bmax[2] - bmin[2]) *
                      0.5f * 1.001f;
    const int root = nt - 1;
    t->pos_x[root] = rcx; t->pos_y[root] = rcy; t->pos_z[root] = rcz;
    t->cell_size[root] = rhs;
    t->next_node = n; /* resetOctree BHTree.cu:411 */

    /* bhtree_buildKernel, BHTree.cu:175-277, one body at a time.  The shape of
     * a one-body-per-leaf octree does not depend on insertion order, so the
     * serial loop builds the tree the concurrent CAS kernel builds (node
     * numbers differ; child slots and geometry do not). */
    for (int body = 0; body < n; ++body) {
        const float px = x[body], py = y[body], pz = z[body];
        int node = root;
        float ncx = rcx, ncy = rcy, ncz = rcz, nhs = rhs;
        int max_iter = 128;
        int placed = 0;
        while (max_iter-- > 0) {
            int oct = octant(ncx, ncy, ncz, px, py, pz);
            int* slot = &t->child[(long)node * 8 + oct];
            int old = *slot;
            if (old == -1) { *slot = body; placed = 1; break; }
            if (old >= n) {
                node = old;
                ncx = t->pos_x[node]; ncy = t->pos_y[node]; ncz = t->pos_z[node];
                nhs = t->cell_size[node];
                continue;
            }
            int new_node = t->next_node++;
            if (new_node >= nt) { break; } /* overflow: body lost (:246-250) */
            float child_hs = nhs * 0.5f;
            float new_cx = ncx + ((px > ncx) ? child_hs : -child_hs);
            float new_cy = ncy + ((py > ncy) ? child_hs : -child_hs);
            float new_cz = ncz + ((pz > ncz) ? child_hs : -child_hs);
            t->pos_x[new_node] = new_cx; t->pos_y[new_node] = new_cy;
            t->pos_z[new_node] = new_cz; t->cell_size[new_node] = child_hs;
            int disp = octant(new_cx, new_cy, new_cz, t->pos_x[old], t->pos_y[old], t->pos_z[old]);
            t->child[(long)new_node * 8 + disp] = old;
            *slot = new_node;
            node = new_node; ncx = new_cx; ncy = new_cy; ncz = new_cz; nhs = child_hs;
        }
        if (!placed) t->lost_bodies++;
    }
}

/* bhtree_summarizeKernel, BHTree.cu:282-317, run until nothing changes.
 * Children of an internal node are always allocated after it, so decreasing
 * slot order (root last) visits every child before its parent.  A node stays
 * unsummarized (count 0) when a child is unsummarized or its mass is 0, as in
 * the kernel's early return and `if (m > 0)` guard. */
void orc_tree_summarize(orc_tree* t) {
    const int n = t->n_bodies, root = t->n_total - 1;
    int last = t->next_node < t->n_total ? t->next_node : t->n_total;
    int unsum = 0;
    for (int pass = 0; pass < 2; ++pass) {
        int lo = (pass == 0) ? last - 1 : root;
        int hi = (pass == 0) ? n : root;
        for (int node = lo; node >= hi; --node) {
            if (pass == 0 && node == root) continue;
            float mm = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
            int cnt = 0, ready = 1;
            for (int k = 0; k < 8; ++k) {
                int c = t->child[(long)node * 8 + k];
                if (c < 0) continue;
                if (t->count[c] == 0) { ready = 0; break; }
                float cm = t->mass[c];
                mm += cm;
                cx += t->pos_x[c] * cm;
                cy += t->pos_y[c] * cm;
                cz += t->pos_z[c] * cm;
                cnt += t->count[c];
            }
            if (ready && mm > 0.f) {
                t->pos_x[node] = cx / mm; t->pos_y[node] = cy / mm; t->pos_z[node] = cz / mm;
                t->mass[node] = mm; t->count[node] = cnt;
            } else {
                unsum++;
            }
        }
    }
    t->unsummarized = unsum;
}

/* launchSummarizeKernel, BHTree.cu:501-516: `passes` parallel launches of
 * bhtree_summarizeKernel (:282-317), each over every internal slot.  A pass
 * here reads the previous pass's children and writes its own copy (a Jacobi
 * sweep: the kernel's in-place passes can finish sooner, never later), so
 * every node of height <= passes ends summarized, as in the reference.  This
 * is the reference's amount of summarize work, for the timed CPU baseline;
 * its values equal orc_tree_summarize's whenever the tree's height is at
 * most `passes`. */
static int g_summarize_passes = 0;

void orc_set_summarize_passes(int passes) { g_summarize_passes = passes > 0 ? passes : 0; }

void orc_tree_summarize_passes(orc_tree* t, int passes, int nthreads) {
    const int n = t->n_bodies, root = t->n_total - 1;
    int last = t->next_node < t->n_total ? t->next_node : t->n_total;
    if (last > root) last = root;
    const int slots = last - n + 1; /* [n, last) and the root */
    float* nm = (float*)malloc((size_t)slots * 4 * sizeof(float));
    int* nc = (int*)malloc((size_t)slots * sizeof(int));
    set_threads(nthreads);
    for (int pass = 0; pass < passes; ++pass) {
#pragma omp parallel for schedule(static, 1024)
        for (int j = 0; j < slots; ++j) {
            const int node = (j == slots - 1) ? root : n + j;
            float mm = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
            int cnt = 0, ready = 1;
            for (int k = 0; k < 8; ++k) {
                int c = t->child[(long)node * 8 + k];
                if (c < 0) continue;
                if (t->count[c] == 0) { ready = 0; break; }
                float cm = t->mass[c];
                mm += cm;
                cx += t->pos_x[c] * cm;
                cy += t->pos_y[c] * cm;
                cz += t->pos_z[c] * cm;
                cnt += t->count[c];
            }
            if (ready && mm > 0.f) {
                nm[4 * j] = cx / mm; nm[4 * j + 1] = cy / mm; nm[4 * j + 2] = cz / mm;
                nm[4 * j + 3] = mm; nc[j] = cnt;
            } else {
                nm[4 * j] = t->pos_x[node]; nm[4 * j + 1] = t->pos_y[node];
                nm[4 * j + 2] = t->pos_z[node]; nm[4 * j + 3] = t->mass[node];
                nc[j] = t->count[node];
            }
        }
#pragma omp parallel for schedule(static, 1024)
        for (int j = 0; j < slots; ++j) {
            const int node = (j == slots - 1) ? root : n + j;
            t->pos_x[node] = nm[4 * j]; t->pos_y[node] = nm[4 * j + 1];
            t->pos_z[node] = nm[4 * j + 2]; t->mass[node] = nm[4 * j + 3];
            t->count[node] = nc[j];
        }
    }
    int unsum = 0;
    for (int j = 0; j < slots; ++j) {
        const int node = (j == slots - 1) ? root : n + j;
        if (t->count[node] == 0) unsum++;
    }
    t->unsummarized = unsum;
    free(nm);
    free(nc);
}

/* bhtree_sortKernel, BHTree.cu:322-352 */
void orc_tree_sort(orc_tree* t) {
    int stack[2048];
    int top = 0, out = 0;
    const int n = t->n_bodies;
    stack[top++] = t->n_total - 1;
    while (top > 0) {
        int node = stack[--top];
        if (node < 0) continue;
        if (node < n) { t->sort_idx[out++] = node; continue; }
        t->start[node] = out;
        for (int k = 7; k >= 0; --k) {
            int c = t->child[(long)node * 8 + k];
            if (c >= 0 && top < 2047) stack[top++] = c;
        }
    }
}

/* bhtree_forceKernel body for one target, BHTree.cu:539-597 */
static void force_one(const orc_tree* t, int body, const float* px, const float* py,
                      const float* pz, float theta, float softening, float star_mass,
                      float* oax, float* oay, float* oaz, long long* n_inter) {
    const int n = t->n_bodies;
    float bx = px[body], by = py[body], bz = pz[body];
    float fx = 0.f, fy = 0.f, fz = 0.f;
    {
        float dx = -bx, dy = -by, dz = -bz;
        float r2 = dx * dx + dy * dy + dz * dz + softening * softening;
        float r = sqrtf(r2);
        float f = star_mass / (r2 * r);
        fx += f * dx; fy += f * dy; fz += f * dz;
    }
    int stack[256];
    int top = 0;
    long long cnt = 0;
    stack[top++] = t->n_total - 1;
    while (top > 0) {
        int node = stack[--top];
        if (node < 0) continue;
        float dx = t->pos_x[node] - bx;
        float dy = t->pos_y[node] - by;
        float dz = t->pos_z[node] - bz;
        float r_geom2 = dx * dx + dy * dy + dz * dz;
        float r_geom = sqrtf(r_geom2);
        float r2 = r_geom2 + softening * softening;
        float r = sqrtf(r2);
        int is_leaf = (node < n);
        int accept = is_leaf || (t->cell_size[node] / r_geom < theta);
        if (accept) {
            if (node == body) continue;
            float mm = t->mass[node];
            float f = mm / (r2 * r);
            fx += f * dx; fy += f * dy; fz += f * dz;
            cnt++;
        } else {
            for (int k = 0; k < 8; ++k) {
                int c = t->child[(long)node * 8 + k];
                if (c >= 0) {
                    if (top < 255) stack[top++] = c;
                }
            }
        }
    }
    if (oax) { *oax = fx; *oay = fy; *oaz = fz; }
    if (n_inter) *n_inter = cnt;
}

void orc_force(const orc_tree* t, const float* x, const float* y, const float* z,
               float* ax, float* ay, float* az, float theta, float softening,
               float star_mass, int nthreads) {
    const int n = t->n_bodies;
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
    for (int idx = 0; idx < n; ++idx) {
        int body = t->sort_idx[idx];
        if (body < 0) continue; /* lost body: the reference would read garbage here */
        force_one(t, body, x, y, z, theta, softening, star_mass, &ax[body], &ay[body],
                  &az[body], 0);
    }
}

long long orc_force_count(const orc_tree* t, const float* x, const float* y, const float* z,
                          float theta, int nthreads) {
    const int n = t->n_bodies;
    long long total = 0;
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : total)
    for (int idx = 0; idx < n; ++idx) {
        int body = t->sort_idx[idx];
        if (body < 0) continue;
        long long c = 0;
        force_one(t, body, x, y, z, theta, 0.01f, 1.0f, 0, 0, 0, &c);
        total += c;
    }
    return total;
}

/* bhtree_collisionKernel + bhtree_applyCollisionDeltaKernel, BHTree.cu:620-708 */
void orc_collision(const orc_tree* t, const float* px, const float* py, const float* pz,
                   float* vx, float* vy, float* vz, float r_coll, float e, int nthreads) {
    const int n = t->n_bodies;
    float* dv = (float*)calloc((size_t)3 * n, sizeof(float));
    if (!dv) return;
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
    for (int idx = 0; idx < n; ++idx) {
        int i = t->sort_idx[idx];
        if (i < 0) continue;
        float ix = px[i], iy = py[i], iz = pz[i];
        float vi_x = vx[i], vi_y = vy[i], vi_z = vz[i];
        float dvx = 0.f, dvy = 0.f, dvz = 0.f;
        int stack[256];
        int top = 0;
        stack[top++] = t->n_total - 1;
        while (top > 0) {
            int node = stack[--top];
            if (node < 0) continue;
            float dx = t->pos_x[node] - ix, dy = t->pos_y[node] - iy, dz = t->pos_z[node] - iz;
            float dist2 = dx * dx + dy * dy + dz * dz;
            if (node < n) {
                int j = node;
                if (j == i) continue;
                if (dist2 < r_coll * r_coll) {
                    float dist = sqrtf(dist2) + 1e-10f;
                    float nx = dx / dist, ny = dy / dist, nz = dz / dist;
                    float dvn = (vx[j] - vi_x) * nx + (vy[j] - vi_y) * ny + (vz[j] - vi_z) * nz;
                    if (dvn < 0.f) {
                        float J = -(1.f + e) * dvn * 0.5f;
                        dvx += -J * nx; dvy += -J * ny; dvz += -J * nz;
                    }
                }
            } else {
                float cell_half = t->cell_size[node];
                float cell_dist = sqrtf(dist2) - cell_half * 1.732f;
                if (cell_dist < r_coll) {
                    for (int k = 0; k < 8; ++k) {
                        int c = t->child[(long)node * 8 + k];
                        if (c >= 0 && top < 255) stack[top++] = c;
                    }
                }
            }
        }
        dv[3 * i] = dvx; dv[3 * i + 1] = dvy; dv[3 * i + 2] = dvz;
    }
    for (int i = 0; i < n; ++i) {
        vx[i] += dv[3 * i]; vy[i] += dv[3 * i + 1]; vz[i] += dv[3 * i + 2];
    }
    free(dv);
}

/* The ordered pairs (i, j != i) closer than r_coll that the traversal of
 * bhtree_collisionKernel (BHTree.cu:620-673) reaches: its cell prune
 * |x_i - com| - 1.732 half >= r_coll can skip some (BHTree.cu:663-665). */
long long orc_collision_pairs(const orc_tree* t, const float* px, const float* py,
                              const float* pz, float r_coll, int nthreads) {
    const int n = t->n_bodies;
    long long total = 0;
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : total)
    for (int idx = 0; idx < n; ++idx) {
        int i = t->sort_idx[idx];
        if (i < 0) continue;
        float ix = px[i], iy = py[i], iz = pz[i];
        int stack[256];
        int top = 0;
        stack[top++] = t->n_total - 1;
        while (top > 0) {
            int node = stack[--top];
            if (node < 0) continue;
            float dx = t->pos_x[node] - ix, dy = t->pos_y[node] - iy, dz = t->pos_z[node] - iz;
            float dist2 = dx * dx + dy * dy + dz * dz;
            if (node < n) {
                if (node != i && dist2 < r_coll * r_coll) ++total;
            } else {
                float cell_half = t->cell_size[node];
                float cell_dist = sqrtf(dist2) - cell_half * 1.732f;
                if (cell_dist < r_coll) {
                    for (int k = 0; k < 8; ++k) {
                        int c = t->child[(long)node * 8 + k];
                        if (c >= 0 && top < 255) stack[top++] = c;
                    }
                }
            }
        }
    }
    return total;
}

/* ------------------------------------------------------------ integrator */

/* integrator_halfKickKernel, Integrator.cu:7-15 */
void orc_half_kick(float* vx, float* vy, float* vz, const float* ax, const float* ay,
                   const float* az, float dt_half, int n) {
    for (int i = 0; i < n; ++i) {
        vx[i] += ax[i] * dt_half; vy[i] += ay[i] * dt_half; vz[i] += az[i] * dt_half;
    }
}

/* integrator_driftKernel, Integrator.cu:17-25 */
void orc_drift(float* x, float* y, float* z, const float* vx, const float* vy,
               const float* vz, float dt, int n) {
    for (int i = 0; i < n; ++i) {
        x[i] += vx[i] * dt; y[i] += vy[i] * dt; z[i] += vz[i] * dt;
    }
}

/* integrator_resetAccKernel, Integrator.cu:27-33 */
void orc_reset_acc(float* ax, float* ay, float* az, int n) {
    for (int i = 0; i < n; ++i) { ax[i] = 0.f; ay[i] = 0.f; az[i] = 0.f; }
}

/* launchGasDragKernel + integrator_gasDragKernel, Integrator.cu:40-76,100-109 */
void orc_gas_drag(const float* x, const float* y, const float* z, float* vx, float* vy,
                  float* vz, float drag_rate, float dt, float star_mass, int n) {
    (void)y;
    if (drag_rate <= 0.0f) return;
    float decay = expf(-drag_rate * dt);
    for (int i = 0; i < n; ++i) {
        float xi = x[i], zi = z[i];
        float r_xz2 = xi * xi + zi * zi;
        if (r_xz2 < 1e-12f) continue;
        float r_xz = sqrtf(r_xz2);
        float inv_r = 1.0f / r_xz;
        float vxi = vx[i], vyi = vy[i], vzi = vz[i];
        float v_r = (vxi * xi + vzi * zi) * inv_r;
        float v_phi = (vxi * (-zi) + vzi * xi) * inv_r;
        float v_kep_mag = sqrtf(star_mass * inv_r);
        float v_kep = (v_phi >= 0.0f) ? v_kep_mag : -v_kep_mag;
        float v_r_new = v_r * decay;
        float v_phi_new = v_kep + (v_phi - v_kep) * decay;
        float v_y_new = vyi * decay;
        vx[i] = v_r_new * (xi * inv_r) + v_phi_new * (-zi * inv_r);
        vz[i] = v_r_new * (zi * inv_r) + v_phi_new * (xi * inv_r);
        vy[i] = v_y_new;
    }
}

/* ------------------------------------------------------------- perturber */

/* makePerturber, Perturber.h:39-57 (MJUP_TO_MSUN = 9.5479e-4f, :25) */
void orc_perturber_make(orc_perturber* p, int enabled, float mass_mjup, float radius_au,
                        float phase0, float star_mass) {
    memset(p, 0, sizeof(*p));
    p->enabled = enabled;
    if (!enabled) return;
    p->r = radius_au;
    p->mass_msun = mass_mjup * 9.5479e-4f;
    p->phase0 = phase0;
    p->omega = sqrtf(star_mass / (p->r * p->r * p->r));
    p->x = p->r * cosf(p->phase0);
    p->z = p->r * sinf(p->phase0);
    p->y = 0.f;
}

/* updatePerturber, Perturber.h:60-66 */
void orc_perturber_update(orc_perturber* p, float sim_time) {
    if (!p->enabled) return;
    float phi = p->phase0 + p->omega * sim_time;
    p->x = p->r * cosf(phi);
    p->z = p->r * sinf(phi);
    p->y = 0.f;
}

/* perturber_forceKernel, Perturber.cu:13-35 (adds to a) */
void orc_perturber_force(float* ax, float* ay, float* az, const float* x, const float* y,
                         const float* z, float px, float py, float pz, float pmass,
                         float softening, int n) {
    for (int i = 0; i < n; ++i) {
        float dx = px - x[i], dy = py - y[i], dz = pz - z[i];
        float r2 = dx * dx + dy * dy + dz * dz + softening * softening;
        float r = sqrtf(r2);
        float f = pmass / (r2 * r);
        ax[i] += f * dx; ay[i] += f * dy; az[i] += f * dz;
    }
}

/* ------------------------------------------------------------ main loop */

/* src/main.cu:113-127: rebuild, reset a, walk, add the perturber. */
void orc_compute_forces(orc_tree* t, const float* x, const float* y, const float* z,
                        const float* m, float* ax, float* ay, float* az, int n,
                        const orc_step_params* sp, float sim_time, int nthreads) {
    orc_tree_build(t, x, y, z, m, n);
    if (g_summarize_passes > 0) orc_tree_summarize_passes(t, g_summarize_passes, nthreads);
    else orc_tree_summarize(t);
    orc_tree_sort(t);
    orc_reset_acc(ax, ay, az, n);
    orc_force(t, x, y, z, ax, ay, az, sp->theta, sp->softening, sp->star_mass, nthreads);
    if (sp->pert.enabled) {
        orc_perturber p = sp->pert;
        orc_perturber_update(&p, sim_time);
        orc_perturber_force(ax, ay, az, x, y, z, p.x, p.y, p.z, p.mass_msun, sp->softening, n);
    }
}

/* src/main.cu:101-139 (one iteration of the step loop). */
void orc_step(orc_tree* t, float* x, float* y, float* z, float* vx, float* vy, float* vz,
              float* ax, float* ay, float* az, const float* m, int n, orc_step_params* sp,
              int step, int nthreads) {
    orc_half_kick(vx, vy, vz, ax, ay, az, sp->dt * 0.5f, n);
    orc_drift(x, y, z, vx, vy, vz, sp->dt, n);
    float sim_time_now = (float)(step + 1) * sp->dt;
    orc_compute_forces(t, x, y, z, m, ax, ay, az, n, sp, sim_time_now, nthreads);
    if (sp->collisions) orc_collision(t, x, y, z, vx, vy, vz, sp->r_coll, sp->restitution, nthreads);
    orc_half_kick(vx, vy, vz, ax, ay, az, sp->dt * 0.5f, n);
    orc_gas_drag(x, y, z, vx, vy, vz, sp->gas_drag_rate, sp->dt, sp->star_mass, n);
}

/* ------------------------------------------------------------------ FoF */

/* find / unite, Aggregate.cpp:9-24 (path halving, union by rank) */
static int uf_find(int* parent, int i) {
    while (parent[i] != i) {
        parent[i] = parent[parent[i]];
        i = parent[i];
    }
    return i;
}

static void uf_unite(int* parent, int* rank, int a, int b) {
    a = uf_find(parent, a);
    b = uf_find(parent, b);
    if (a == b) return;
    if (rank[a] < rank[b]) { int tmp = a; a = b; b = tmp; }
    parent[b] = a;
    if (rank[a] == rank[b]) ++rank[a];
}

/* detectAggregates, Aggregate.cpp:26-52, plus the per-particle size of
 * src/main.cu:153-161. */
int orc_fof(const float* x, const float* y, const float* z, int n, float link_length,
            int* labels, unsigned short* agg_size) {
    float ll2 = link_length * link_length;
    int* parent = (int*)malloc((size_t)n * sizeof(int));
    int* rank = (int*)calloc((size_t)n, sizeof(int));
    int* minidx = (int*)malloc((size_t)n * sizeof(int));
    int* gsize = (int*)calloc((size_t)n, sizeof(int));
    for (int i = 0; i < n; ++i) { parent[i] = i; minidx[i] = n; }
    for (int i = 0; i < n - 1; ++i) {
        for (int j = i + 1; j < n; ++j) {
            float dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
            if (dx * dx + dy * dy + dz * dz < ll2) uf_unite(parent, rank, i, j);
        }
    }
    for (int i = 0; i < n; ++i) {
        int r = uf_find(parent, i);
        if (i < minidx[r]) minidx[r] = i;
        gsize[r]++;
    }
    int groups = 0;
    for (int i = 0; i < n; ++i) {
        int r = uf_find(parent, i);
        labels[i] = minidx[r];
        int s = gsize[r];
        agg_size[i] = (unsigned short)(s >= 2 ? (s < 65535 ? s : 65535) : 1);
        if (s >= 2 && minidx[r] == i) groups++;
    }
    free(parent); free(rank); free(minidx); free(gsize);
    return groups;
}

/* Aggregate.cpp:54-74, groups ordered by smallest member index. */
void orc_fof_aggregates(const float* x, const float* y, const float* z, const float* vx,
                        const float* vy, const float* vz, int n, const int* labels,
                        float particle_mass, int n_groups, int* g_n, float* g_mass,
                        float* g_c, float* g_v, float* g_dist, int* g_label) {
    int* slot = (int*)malloc((size_t)n * sizeof(int));
    int* cnt = (int*)calloc((size_t)n, sizeof(int));
    for (int i = 0; i < n; ++i) cnt[labels[i]]++;
    int g = 0;
    for (int i = 0; i < n; ++i) {
        slot[i] = -1;
        if (labels[i] == i && cnt[i] >= 2 && g < n_groups) {
            slot[i] = g;
            g_label[g] = i; g_n[g] = cnt[i];
            g_c[3 * g] = g_c[3 * g + 1] = g_c[3 * g + 2] = 0.f;
            g_v[3 * g] = g_v[3 * g + 1] = g_v[3 * g + 2] = 0.f;
            g++;
        }
    }
    for (int i = 0; i < n; ++i) {
        int s = slot[labels[i]];
        if (s < 0) continue;
        g_c[3 * s] += x[i]; g_c[3 * s + 1] += y[i]; g_c[3 * s + 2] += z[i];
        g_v[3 * s] += vx[i]; g_v[3 * s + 1] += vy[i]; g_v[3 * s + 2] += vz[i];
    }
    for (int s = 0; s < g; ++s) {
        g_mass[s] = (float)g_n[s] * particle_mass;
        float inv = 1.0f / (float)g_n[s];
        for (int k = 0; k < 3; ++k) { g_c[3 * s + k] *= inv; g_v[3 * s + k] *= inv; }
        float cx = g_c[3 * s], cy = g_c[3 * s + 1], cz = g_c[3 * s + 2];
        g_dist[s] = sqrtf(cx * cx + cy * cy + cz * cz);
    }
    free(slot); free(cnt);
}

/* ----------------------------------------------------------- FP64 tools */

void orc_direct_f64(const double* x, const double* y, const double* z, const double* m,
                    int n, const int* targets, int n_targets, double eps, double star_mass,
                    int include_star, double* ax, double* ay, double* az, int nthreads) {
    double e2 = eps * eps;
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
    for (int k = 0; k < n_targets; ++k) {
        int i = targets ? targets[k] : k;
        double xi = x[i], yi = y[i], zi = z[i];
        double fx = 0, fy = 0, fz = 0;
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            double dx = x[j] - xi, dy = y[j] - yi, dz = z[j] - zi;
            double r2 = dx * dx + dy * dy + dz * dz + e2;
            double inv = 1.0 / sqrt(r2);
            double f = m[j] * inv * inv * inv;
            fx += f * dx; fy += f * dy; fz += f * dz;
        }
        if (include_star) {
            double r2 = xi * xi + yi * yi + zi * zi + e2;
            double inv = 1.0 / sqrt(r2);
            double f = star_mass * inv * inv * inv;
            fx -= f * xi; fy -= f * yi; fz -= f * zi;
        }
        ax[k] = fx; ay[k] = fy; az[k] = fz;
    }
}

void orc_energy_f64(const double* x, const double* y, const double* z, const double* vx,
                    const double* vy, const double* vz, const double* m, int n, double eps,
                    double star_mass, double* energy, double* ly, int nthreads) {
    double e2 = eps * eps, kin = 0, star = 0, pair = 0, l = 0;
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : kin, star, pair, l)
    for (int i = 0; i < n; ++i) {
        kin += 0.5 * m[i] * (vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i]);
        star -= star_mass * m[i] / sqrt(x[i] * x[i] + y[i] * y[i] + z[i] * z[i] + e2);
        /* L_y = m (z vx - x vz) for the XZ disk with +Y pole */
        l += m[i] * (z[i] * vx[i] - x[i] * vz[i]);
        double p = 0;
        for (int j = i + 1; j < n; ++j) {
            double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
            p -= m[i] * m[j] / sqrt(dx * dx + dy * dy + dz * dz + e2);
        }
        pair += p;
    }
    *energy = kin + star + pair;
    *ly = l;
}

/* ---------------------------------------------------------- disk recipe */

/* The synthetic Keplerian disk that the product's nbody_make_disk writes,
 * restated so that CPU-only callers (the reference arm of the benchmark) can
 * build the same initial conditions without loading the product library.
 * Semi-major axis by the inverse CDF of Sigma ~ r^-1.5
 * (src/disk/DiskInit.cpp:42-44), Rayleigh e (capped at 0.9) and inclination,
 * uniform node, periapsis and mean anomaly, Kepler's equation by Newton,
 * perifocal -> +Z-pole frame -> disk plane XZ with +Y up.  Draw k of body i is
 * splitmix64 (Vigna's published mixer) of splitmix64(seed) ^ (16 i + k). */
static uint64_t orc_splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

static double orc_unit(uint64_t seed_mix, uint64_t i, uint64_t k) {
    return (double)(orc_splitmix64(seed_mix ^ (i * 16u + k)) >> 11) * (1.0 / 9007199254740992.0);
}

void orc_make_disk(int n, double r_min, double r_max, double sigma_e, double sigma_i,
                   double mu, uint64_t seed, double* x, double* y, double* z, double* vx,
                   double* vy, double* vz) {
    const double two_pi = 6.283185307179586476925287;
    const uint64_t sm = orc_splitmix64(seed);
    const double sa = sqrt(r_min), sb = sqrt(r_max);
#pragma omp parallel for schedule(static, 4096)
    for (int i = 0; i < n; ++i) {
        const double sr = orc_unit(sm, i, 0) * (sb - sa) + sa;
        const double a = sr * sr;
        double e = sigma_e * sqrt(-2.0 * log1p(-orc_unit(sm, i, 1)));
        const double inc = sigma_i * sqrt(-2.0 * log1p(-orc_unit(sm, i, 2)));
        if (e > 0.9) e = 0.9;
        const double node = two_pi * orc_unit(sm, i, 3);
        const double peri = two_pi * orc_unit(sm, i, 4);
        const double mean = two_pi * orc_unit(sm, i, 5);
        double ea = (e < 0.8) ? mean : 3.141592653589793;
        for (int it = 0; it < 60; ++it) {
            const double step = (ea - e * sin(ea) - mean) / (1.0 - e * cos(ea));
            ea -= step;
            if (fabs(step) < 1e-15) break;
        }
        const double ce = cos(ea), se = sin(ea), q = sqrt(1.0 - e * e);
        const double nmot = sqrt(mu / (a * a * a)), den = 1.0 - e * ce;
        const double px = a * (ce - e), py = a * q * se;
        const double pvx = -a * nmot * se / den, pvy = a * nmot * q * ce / den;
        const double cn = cos(node), sn = sin(node), cp = cos(peri), sp = sin(peri);
        const double ci = cos(inc), si = sin(inc);
        const double m11 = cn * cp - sn * sp * ci, m12 = -cn * sp - sn * cp * ci;
        const double m21 = sn * cp + cn * sp * ci, m22 = -sn * sp + cn * cp * ci;
        const double m31 = sp * si, m32 = cp * si;
        x[i] = m11 * px + m12 * py;
        y[i] = -(m31 * px + m32 * py);
        z[i] = m21 * px + m22 * py;
        vx[i] = m11 * pvx + m12 * pvy;
        vy[i] = -(m31 * pvx + m32 * pvy);
        vz[i] = m21 * pvx + m22 * pvy;
    }
}
