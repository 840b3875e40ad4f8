"""ctypes front end for the oracle libraries.

TEST INFRASTRUCTURE ONLY.  ``tests/``, ``__graft_entry__.smoke()`` (as the
checker) and ``bench.py``'s CPU-baseline / ``--impl reference`` leg import this
module; the product package never does.

* ``Port`` wraps ``oracle/liboracle_port.so``: the CPU restatement of the
  reference's octree build, summarize, DFS sort, Barnes-Hut walk, collision,
  KDK, gas drag, perturber and FoF (``oracle/port.c``), plus FP64 direct-sum
  and energy tools.
* ``RefHost`` wraps ``oracle/_ref/libref_host.so``: the reference's own
  Config.cpp / Aggregate.cpp / OutputWriter.cpp / DiskInit.cpp.
* ``RefEngine`` wraps ``oracle/_ref/libref_engine[_nofma].so``: the reference's
  own BHTree.cu / Integrator.cu / Perturber.cu compiled for sm_100a (GPU).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_F = C.POINTER(C.c_float)
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_U16 = C.POINTER(C.c_uint16)


def _f32(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(_F)


def _ptr(a, t):
    return a.ctypes.data_as(t)


class _Tree(C.Structure):
    _fields_ = [
        ("n_bodies", C.c_int), ("n_total", C.c_int),
        ("pos_x", _F), ("pos_y", _F), ("pos_z", _F), ("mass", _F), ("cell_size", _F),
        ("child", _I), ("count", _I), ("start", _I), ("sort_idx", _I),
        ("next_node", C.c_int),
        ("bbox_min", C.c_float * 3), ("bbox_max", C.c_float * 3),
        ("lost_bodies", C.c_int), ("unsummarized", C.c_int),
    ]


class _Pert(C.Structure):
    _fields_ = [("enabled", C.c_int), ("r", C.c_float), ("mass_msun", C.c_float),
                ("phase0", C.c_float), ("omega", C.c_float),
                ("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class _StepParams(C.Structure):
    _fields_ = [("dt", C.c_float), ("theta", C.c_float), ("softening", C.c_float),
                ("star_mass", C.c_float), ("r_coll", C.c_float), ("restitution", C.c_float),
                ("gas_drag_rate", C.c_float), ("collisions", C.c_int), ("pert", _Pert)]


def build_port():
    """Compile oracle/liboracle_port.so (gcc, no GPU needed)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)


@dataclass
class TreeInfo:
    sort_idx: np.ndarray
    root_mass: float
    root_count: int
    next_node: int
    lost_bodies: int
    unsummarized: int
    height: int


class Port:
    """The CPU restatement (oracle/port.c)."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "liboracle_port.so")
        if not os.path.exists(path):
            build_port()
        L = self.lib = C.CDLL(path)
        L.orc_tree_alloc.argtypes = [C.POINTER(_Tree), C.c_int]
        L.orc_tree_free.argtypes = [C.POINTER(_Tree)]
        L.orc_tree_build.argtypes = [C.POINTER(_Tree), _F, _F, _F, _F, C.c_int]
        L.orc_tree_summarize.argtypes = [C.POINTER(_Tree)]
        L.orc_tree_sort.argtypes = [C.POINTER(_Tree)]
        L.orc_force.argtypes = [C.POINTER(_Tree), _F, _F, _F, _F, _F, _F, C.c_float,
                                C.c_float, C.c_float, C.c_int]
        L.orc_force_count.argtypes = [C.POINTER(_Tree), _F, _F, _F, C.c_float, C.c_int]
        L.orc_force_count.restype = C.c_longlong
        L.orc_collision.argtypes = [C.POINTER(_Tree), _F, _F, _F, _F, _F, _F, C.c_float,
                                    C.c_float, C.c_int]
        L.orc_collision_pairs.argtypes = [C.POINTER(_Tree), _F, _F, _F, C.c_float, C.c_int]
        L.orc_collision_pairs.restype = C.c_longlong
        for name in ("orc_half_kick", "orc_drift"):
            getattr(L, name).argtypes = [_F, _F, _F, _F, _F, _F, C.c_float, C.c_int]
        L.orc_gas_drag.argtypes = [_F, _F, _F, _F, _F, _F, C.c_float, C.c_float, C.c_float,
                                   C.c_int]
        L.orc_perturber_make.argtypes = [C.POINTER(_Pert), C.c_int, C.c_float, C.c_float,
                                         C.c_float, C.c_float]
        L.orc_perturber_update.argtypes = [C.POINTER(_Pert), C.c_float]
        L.orc_perturber_force.argtypes = [_F, _F, _F, _F, _F, _F, C.c_float, C.c_float,
                                          C.c_float, C.c_float, C.c_float, C.c_int]
        L.orc_compute_forces.argtypes = [C.POINTER(_Tree), _F, _F, _F, _F, _F, _F, _F, C.c_int,
                                         C.POINTER(_StepParams), C.c_float, C.c_int]
        L.orc_step.argtypes = [C.POINTER(_Tree), _F, _F, _F, _F, _F, _F, _F, _F, _F, _F,
                               C.c_int, C.POINTER(_StepParams), C.c_int, C.c_int]
        L.orc_fof.argtypes = [_F, _F, _F, C.c_int, C.c_float, _I, _U16]
        L.orc_fof.restype = C.c_int
        L.orc_fof_aggregates.argtypes = [_F, _F, _F, _F, _F, _F, C.c_int, _I, C.c_float,
                                         C.c_int, _I, _F, _F, _F, _F, _I]
        L.orc_direct_f64.argtypes = [_D, _D, _D, _D, C.c_int, _I, C.c_int, C.c_double,
                                     C.c_double, C.c_int, _D, _D, _D, C.c_int]
        L.orc_energy_f64.argtypes = [_D, _D, _D, _D, _D, _D, _D, C.c_int, C.c_double,
                                     C.c_double, _D, _D, C.c_int]
        L.orc_set_summarize_passes.argtypes = [C.c_int]
        L.orc_make_disk.argtypes = [C.c_int] + [C.c_double] * 5 + [C.c_uint64] + [_D] * 6

    # -- tree -------------------------------------------------------------
    def build_tree(self, x, y, z, m):
        n = len(x)
        t = _Tree()
        if self.lib.orc_tree_alloc(C.byref(t), n) != 0:
            raise MemoryError("orc_tree_alloc")
        arrs = [_f32(a) for a in (x, y, z, m)]
        self.lib.orc_tree_build(C.byref(t), *[p for _, p in arrs], n)
        self.lib.orc_tree_summarize(C.byref(t))
        self.lib.orc_tree_sort(C.byref(t))
        t._keep = arrs
        return t

    def free_tree(self, t):
        self.lib.orc_tree_free(C.byref(t))

    def tree_info(self, t) -> TreeInfo:
        n = t.n_bodies
        root = t.n_total - 1
        sort_idx = np.ctypeslib.as_array(t.sort_idx, shape=(n,)).copy()
        # height (levels of internal nodes) of the tree, iterative DFS
        child = np.ctypeslib.as_array(t.child, shape=(t.n_total * 8,))
        height, stack = 0, [(root, 1)]
        while stack:
            node, d = stack.pop()
            height = max(height, d)
            for k in range(8):
                c = int(child[node * 8 + k])
                if c >= n:
                    stack.append((c, d + 1))
        return TreeInfo(sort_idx, float(t.mass[root]), int(t.count[root]), int(t.next_node),
                        int(t.lost_bodies), int(t.unsummarized), height)

    def forces(self, x, y, z, m, theta, softening, star_mass, nthreads=0, pert=None,
               sim_time=0.0):
        """launchForceKernel (+ launchPerturberForceKernel) on a fresh tree."""
        n = len(x)
        t = self.build_tree(x, y, z, m)
        try:
            ax = np.zeros(n, np.float32); ay = np.zeros(n, np.float32); az = np.zeros(n, np.float32)
            xs = [np.ascontiguousarray(a, np.float32) for a in (x, y, z)]
            self.lib.orc_force(C.byref(t), *[_ptr(a, _F) for a in xs], _ptr(ax, _F),
                               _ptr(ay, _F), _ptr(az, _F), theta, softening, star_mass, nthreads)
            if pert is not None and pert.enabled:
                p = _Pert.from_buffer_copy(pert)
                self.lib.orc_perturber_update(C.byref(p), sim_time)
                self.lib.orc_perturber_force(_ptr(ax, _F), _ptr(ay, _F), _ptr(az, _F),
                                             *[_ptr(a, _F) for a in xs], p.x, p.y, p.z,
                                             p.mass_msun, softening, n)
            return ax, ay, az, self.tree_info(t)
        finally:
            self.free_tree(t)

    def interaction_count(self, x, y, z, m, theta, nthreads=0):
        t = self.build_tree(x, y, z, m)
        try:
            xs = [np.ascontiguousarray(a, np.float32) for a in (x, y, z)]
            return int(self.lib.orc_force_count(C.byref(t), *[_ptr(a, _F) for a in xs],
                                                theta, nthreads))
        finally:
            self.free_tree(t)

    def collision(self, x, y, z, m, vx, vy, vz, r_coll, restitution, nthreads=0):
        t = self.build_tree(x, y, z, m)
        try:
            xs = [np.ascontiguousarray(a, np.float32) for a in (x, y, z)]
            vs = [np.array(a, np.float32) for a in (vx, vy, vz)]
            self.lib.orc_collision(C.byref(t), *[_ptr(a, _F) for a in xs],
                                   *[_ptr(a, _F) for a in vs], r_coll, restitution, nthreads)
            return vs
        finally:
            self.free_tree(t)

    def collision_pairs(self, x, y, z, m, r_coll, nthreads=0):
        """Ordered pairs closer than r_coll that the reference's collision
        traversal reaches (port.c orc_collision_pairs)."""
        t = self.build_tree(x, y, z, m)
        try:
            xs = [np.ascontiguousarray(a, np.float32) for a in (x, y, z)]
            return int(self.lib.orc_collision_pairs(C.byref(t), *[_ptr(a, _F) for a in xs],
                                                    r_coll, nthreads))
        finally:
            self.free_tree(t)

    # -- perturber / step --------------------------------------------------
    def perturber(self, enabled, mass_mjup, radius_au, phase0, star_mass):
        p = _Pert()
        self.lib.orc_perturber_make(C.byref(p), int(enabled), mass_mjup, radius_au, phase0,
                                    star_mass)
        return p

    def perturber_at(self, pert, t):
        p = _Pert.from_buffer_copy(pert)
        self.lib.orc_perturber_update(C.byref(p), t)
        return p

    def step_params(self, dt, theta, softening, star_mass, r_coll=0.0, restitution=0.0,
                    gas_drag_rate=0.0, collisions=True, pert=None):
        sp = _StepParams(dt, theta, softening, star_mass, r_coll, restitution, gas_drag_rate,
                         int(collisions))
        if pert is not None:
            sp.pert = pert
        return sp

    def run(self, state, sp, steps, step0=0, nthreads=0, initial_forces=True):
        """src/main.cu:85-139 on host FP32 arrays (dict with x..az, m). In place."""
        n = len(state["x"])
        for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m"):
            state[k] = np.ascontiguousarray(state.get(k, np.zeros(n)), np.float32)
        P = {k: _ptr(state[k], _F) for k in state}
        t = _Tree()
        if self.lib.orc_tree_alloc(C.byref(t), n) != 0:
            raise MemoryError("orc_tree_alloc")
        try:
            if initial_forces:
                self.lib.orc_compute_forces(C.byref(t), P["x"], P["y"], P["z"], P["m"], P["ax"],
                                            P["ay"], P["az"], n, C.byref(sp),
                                            C.c_float(step0 * sp.dt), nthreads)
            for s in range(step0, step0 + steps):
                self.lib.orc_step(C.byref(t), P["x"], P["y"], P["z"], P["vx"], P["vy"], P["vz"],
                                  P["ax"], P["ay"], P["az"], P["m"], n, C.byref(sp), s, nthreads)
        finally:
            self.lib.orc_tree_free(C.byref(t))
        return state

    def half_kick(self, v, a, dt_half):
        v = [np.array(q, np.float32) for q in v]
        a = [np.ascontiguousarray(q, np.float32) for q in a]
        self.lib.orc_half_kick(*[_ptr(q, _F) for q in v + a], dt_half, len(v[0]))
        return v

    def drift(self, x, v, dt):
        x = [np.array(q, np.float32) for q in x]
        v = [np.ascontiguousarray(q, np.float32) for q in v]
        self.lib.orc_drift(*[_ptr(q, _F) for q in x + v], dt, len(x[0]))
        return x

    def gas_drag(self, x, v, rate, dt, star_mass):
        x = [np.ascontiguousarray(q, np.float32) for q in x]
        v = [np.array(q, np.float32) for q in v]
        self.lib.orc_gas_drag(*[_ptr(q, _F) for q in x + v], rate, dt, star_mass, len(x[0]))
        return v

    def perturber_force(self, a, x, p, softening):
        a = [np.array(q, np.float32) for q in a]
        x = [np.ascontiguousarray(q, np.float32) for q in x]
        self.lib.orc_perturber_force(*[_ptr(q, _F) for q in a + x], p.x, p.y, p.z, p.mass_msun,
                                     softening, len(x[0]))
        return a

    def set_summarize_passes(self, passes: int):
        """passes > 0: every later step summarizes the tree with the
        reference's fixed number of parallel passes (BHTree.cu:501-516)
        instead of the converged sweep; 0 restores the sweep."""
        self.lib.orc_set_summarize_passes(int(passes))

    def make_disk(self, n, r_min, r_max, sigma_e=0.01, sigma_i=0.005, star_mass=1.0, seed=0):
        """The product's synthetic-disk recipe (nbody_make_disk), restated in
        oracle/port.c: dict of float64 arrays x..vz."""
        out = {k: np.zeros(n, np.float64) for k in ("x", "y", "z", "vx", "vy", "vz")}
        self.lib.orc_make_disk(n, r_min, r_max, sigma_e, sigma_i, star_mass, seed,
                               *[_ptr(out[k], _D) for k in ("x", "y", "z", "vx", "vy", "vz")])
        return out

    # -- FoF -----------------------------------------------------------------
    def fof(self, x, y, z, link_length):
        n = len(x)
        labels = np.zeros(n, np.int32)
        size = np.zeros(n, np.uint16)
        xs = [np.ascontiguousarray(a, np.float32) for a in (x, y, z)]
        g = self.lib.orc_fof(*[_ptr(a, _F) for a in xs], n, link_length, _ptr(labels, _I),
                             _ptr(size, _U16))
        return labels, size, g

    def aggregates(self, x, y, z, vx, vy, vz, labels, particle_mass, n_groups):
        n = len(x)
        arrs = [np.ascontiguousarray(a, np.float32) for a in (x, y, z, vx, vy, vz)]
        labels = np.ascontiguousarray(labels, np.int32)
        g = max(n_groups, 1)
        out = dict(n=np.zeros(g, np.int32), mass=np.zeros(g, np.float32),
                   c=np.zeros(3 * g, np.float32), v=np.zeros(3 * g, np.float32),
                   dist=np.zeros(g, np.float32), label=np.zeros(g, np.int32))
        self.lib.orc_fof_aggregates(*[_ptr(a, _F) for a in arrs], n, _ptr(labels, _I),
                                    particle_mass, n_groups, _ptr(out["n"], _I),
                                    _ptr(out["mass"], _F), _ptr(out["c"], _F),
                                    _ptr(out["v"], _F), _ptr(out["dist"], _F),
                                    _ptr(out["label"], _I))
        return {k: v[: n_groups * (3 if k in ("c", "v") else 1)] for k, v in out.items()}

    # -- FP64 tools ------------------------------------------------------------
    def direct_f64(self, x, y, z, m, targets, softening, star_mass, include_star=True,
                   nthreads=0):
        xs = [np.ascontiguousarray(a, np.float64) for a in (x, y, z, m)]
        tg = np.ascontiguousarray(targets, np.int32)
        k = len(tg)
        out = [np.zeros(k, np.float64) for _ in range(3)]
        self.lib.orc_direct_f64(*[_ptr(a, _D) for a in xs], len(xs[0]), _ptr(tg, _I), k,
                                softening, star_mass, int(include_star),
                                *[_ptr(a, _D) for a in out], nthreads)
        return out

    def energy_f64(self, x, y, z, vx, vy, vz, m, softening, star_mass, nthreads=0):
        xs = [np.ascontiguousarray(a, np.float64) for a in (x, y, z, vx, vy, vz, m)]
        e = C.c_double(); l = C.c_double()
        self.lib.orc_energy_f64(*[_ptr(a, _D) for a in xs], len(xs[0]), softening, star_mass,
                                C.byref(e), C.byref(l), nthreads)
        return e.value, l.value


class RefHost:
    """The reference's own host code (oracle/_ref/libref_host.so)."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "_ref", "libref_host.so")
        L = self.lib = C.CDLL(path)
        L.ref_load_config.argtypes = [C.c_char_p, _F, _I, C.c_char_p, C.c_int, C.c_char_p, C.c_int]
        L.ref_particle_radius.argtypes = [C.c_float]
        L.ref_particle_radius.restype = C.c_float
        L.ref_detect_aggregates.argtypes = [_F, _F, _F, _F, _F, _F, C.c_int, C.c_float, C.c_float,
                                            _I, _U16, C.c_int, _I, _F, _F, _F, _F, _I]
        L.ref_detect_aggregates_count.argtypes = [_F, _F, _F, C.c_int, C.c_float]
        L.ref_write_run.argtypes = [C.c_char_p, C.c_int, C.c_float, C.c_int, _F, _F, _F, _U16,
                                    C.c_int, _F, C.c_int, _I, _F, _F, _F, _F, C.c_int, _F,
                                    C.c_char_p, C.c_int]

    FIELDS = ["disk_r_min", "disk_r_max", "disk_h_factor", "particle_mass_msun",
              "star_mass_msun", "softening_AU", "theta", "collision_radius_factor",
              "restitution", "gas_drag_rate", "dt", "total_time", "perturber_mass_mjup",
              "perturber_radius_AU", "perturber_phase0"]

    def load_config(self, path):
        f = (C.c_float * 15)(); i = (C.c_int * 3)()
        d = C.create_string_buffer(1024); err = C.create_string_buffer(1024)
        rc = self.lib.ref_load_config(path.encode(), f, i, d, 1024, err, 1024)
        if rc:
            raise RuntimeError(err.value.decode())
        cfg = {k: f[j] for j, k in enumerate(self.FIELDS)}
        cfg.update(n_particles=i[0], output_every_n_steps=i[1], perturber_enabled=bool(i[2]),
                   output_dir=d.value.decode())
        return cfg

    def particle_radius(self, m):
        return self.lib.ref_particle_radius(m)

    def detect_aggregates(self, x, y, z, vx, vy, vz, link_length, particle_mass):
        n = len(x)
        arrs = [np.ascontiguousarray(a, np.float32) for a in (x, y, z, vx, vy, vz)]
        labels = np.zeros(n, np.int32); size = np.zeros(n, np.uint16)
        g = max(n // 2, 1)
        out = dict(n=np.zeros(g, np.int32), mass=np.zeros(g, np.float32),
                   c=np.zeros(3 * g, np.float32), v=np.zeros(3 * g, np.float32),
                   dist=np.zeros(g, np.float32), label=np.zeros(g, np.int32))
        ng = self.lib.ref_detect_aggregates(*[_ptr(a, _F) for a in arrs], n, link_length,
                                            particle_mass, _ptr(labels, _I), _ptr(size, _U16), g,
                                            _ptr(out["n"], _I), _ptr(out["mass"], _F),
                                            _ptr(out["c"], _F), _ptr(out["v"], _F),
                                            _ptr(out["dist"], _F), _ptr(out["label"], _I))
        if ng < 0:
            raise RuntimeError("detectAggregates failed")
        aggs = {k: v[: ng * (3 if k in ("c", "v") else 1)] for k, v in out.items()}
        return labels, size, ng, aggs

    def detect_aggregates_count(self, x, y, z, link_length):
        xs = [np.ascontiguousarray(a, np.float32) for a in (x, y, z)]
        return self.lib.ref_detect_aggregates_count(*[_ptr(a, _F) for a in xs], len(xs[0]),
                                                    link_length)


class RefEngine:
    """The reference's own CUDA engine compiled for sm_100a (needs a GPU)."""

    def __init__(self, n, nofma=False, path=None):
        name = "libref_engine_nofma.so" if nofma else "libref_engine.so"
        path = path or os.path.join(HERE, "_ref", name)
        L = self.lib = C.CDLL(path)
        L.ref_eng_error.restype = C.c_char_p
        L.ref_eng_create.restype = C.c_void_p
        L.ref_eng_create.argtypes = [C.c_int]
        L.ref_eng_destroy.argtypes = [C.c_void_p]
        L.ref_eng_set_state.argtypes = [C.c_void_p] + [_F] * 10
        L.ref_eng_get_state.argtypes = [C.c_void_p] + [_F] * 9
        L.ref_eng_build.argtypes = [C.c_void_p]
        L.ref_eng_tree_info.argtypes = [C.c_void_p, _I, _F, _I, _I]
        L.ref_eng_force.argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_float, C.c_int,
                                    C.c_float, C.c_float, C.c_float, C.c_float]
        L.ref_eng_collide.argtypes = [C.c_void_p, C.c_float, C.c_float]
        L.ref_eng_kick.argtypes = [C.c_void_p, C.c_float]
        L.ref_eng_drift.argtypes = [C.c_void_p, C.c_float]
        L.ref_eng_drag.argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_float]
        L.ref_eng_perturber_force.argtypes = [C.c_void_p] + [C.c_float] * 5
        L.ref_eng_steps.argtypes = [C.c_void_p, C.c_int, C.c_int] + [C.c_float] * 7 + [
            C.c_int, C.c_float, C.c_float, C.c_float, _D]
        self.n = n
        self.h = L.ref_eng_create(n)
        if not self.h:
            raise RuntimeError(L.ref_eng_error().decode())

    def _chk(self, rc):
        if rc:
            raise RuntimeError(self.lib.ref_eng_error().decode())

    def close(self):
        if self.h:
            self.lib.ref_eng_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, s):
        n = self.n
        arrs = [np.ascontiguousarray(s.get(k, np.zeros(n)), np.float32)
                for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m")]
        self._chk(self.lib.ref_eng_set_state(self.h, *[_ptr(a, _F) for a in arrs]))

    def get_state(self):
        out = {k: np.zeros(self.n, np.float32) for k in ("x", "y", "z", "vx", "vy", "vz",
                                                         "ax", "ay", "az")}
        self._chk(self.lib.ref_eng_get_state(self.h, *[_ptr(out[k], _F) for k in out]))
        return out

    def build(self):
        self._chk(self.lib.ref_eng_build(self.h))
        si = np.zeros(self.n, np.int32); rm = C.c_float(); rc = C.c_int(); nn = C.c_int()
        self._chk(self.lib.ref_eng_tree_info(self.h, _ptr(si, _I), C.byref(rm), C.byref(rc),
                                             C.byref(nn)))
        return si, rm.value, rc.value, nn.value

    def force(self, theta, softening, star_mass, pert=None):
        if pert is not None and pert.enabled:
            self._chk(self.lib.ref_eng_force(self.h, theta, softening, star_mass, 1, pert.x,
                                             pert.y, pert.z, pert.mass_msun))
        else:
            self._chk(self.lib.ref_eng_force(self.h, theta, softening, star_mass, 0, 0, 0, 0, 0))

    def collide(self, r_coll, e):
        self._chk(self.lib.ref_eng_collide(self.h, r_coll, e))

    def kick(self, dth):
        self._chk(self.lib.ref_eng_kick(self.h, dth))

    def drift(self, dt):
        self._chk(self.lib.ref_eng_drift(self.h, dt))

    def drag(self, rate, dt, star_mass):
        self._chk(self.lib.ref_eng_drag(self.h, rate, dt, star_mass))

    def steps(self, step0, nsteps, dt, theta, softening, star_mass, r_coll, restitution,
              drag_rate, pert_on=False, pert_mjup=1.0, pert_r=20.0, pert_phase0=0.0):
        ms = C.c_double()
        self._chk(self.lib.ref_eng_steps(self.h, step0, nsteps, dt, theta, softening, star_mass,
                                         r_coll, restitution, drag_rate, int(pert_on), pert_mjup,
                                         pert_r, pert_phase0, C.byref(ms)))
        return ms.value
