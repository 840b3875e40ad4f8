"""nbody-b200: Python binding of libnbody_b200.so (the C ABI in include/nbody_b200.h).

The package directory is named ``nbody-sim_b200``; import it with
``importlib.import_module("nbody-sim_b200")``.

Everything computational runs in the CUDA library; this module only declares
the C signatures, moves buffers (torch CUDA tensors for device memory, numpy
for host memory) and turns NBODY_ERR_* codes into exceptions.  There is no CPU
fallback: if the shared library is missing or fails to load, importing the
package raises.

Python-side names mirror the reference API they wrap:

* :class:`ParticleData`, :func:`allocate_particles_gpu`, :func:`copy_to_gpu`,
  :func:`copy_to_cpu` -- include/ParticleData.h:19-123
* :class:`Octree` (``reset``, ``bbox``, ``build``, ``summarize``, ``sort``,
  ``force``, ``collide``) -- include/BHTree.cuh:38-50
* :func:`half_kick`, :func:`drift`, :func:`reset_acceleration`,
  :func:`gas_drag`, :func:`perturber_force` -- include/Integrator.cuh:9-22,
  include/Perturber.h:73-75
* :func:`make_perturber`, :func:`update_perturber` -- include/Perturber.h:39-66
* :func:`load_config`, :func:`particle_physical_radius` -- include/Config.h:38,
  include/DiskInit.h:14
* :func:`detect_aggregates` -- include/Aggregate.h:17-18
* :class:`OutputWriter` -- include/OutputWriter.h:15-51
* :class:`Sim` -- the step loop of src/main.cu:85-139 resident on the GPU
* :class:`Ensemble` -- many independent disks, each with main.cu's step loop,
  stepped together (one launch per phase over all disks, CUDA graphs)
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnbody_b200.so")

NBODY_OK = 0
NBODY_ERR_CUDA = 1
NBODY_ERR_ARG = 2
NBODY_ERR_OVERFLOW = 3
NBODY_ERR_TIMEOUT = 4
NBODY_ERR_IO = 5
NBODY_ERR_CONFIG = 6
NBODY_ERR_STATE = 7
NBODY_STATE_F32 = 0
NBODY_STATE_F64 = 1
NBODY_STATE_F32X2 = 2
FOF_NOALLOC_MAX_N = 32768
STATE_F32 = 0
STATE_F64 = 1
STATE_F32X2 = 2


class NBodyError(RuntimeError):
    """An NBODY_ERR_* status from the C ABI (``code`` holds the value)."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


_F = C.POINTER(C.c_float)
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_U16 = C.POINTER(C.c_uint16)
_VP = C.c_void_p


class nbody_particles(C.Structure):
    _fields_ = [(k, _F) for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "mass")] + [
        ("id", _I), ("n", C.c_int)]


class nbody_config(C.Structure):
    _fields_ = [
        ("n_particles", C.c_int), ("disk_r_min", C.c_float), ("disk_r_max", C.c_float),
        ("disk_h_factor", C.c_float), ("particle_mass_msun", C.c_float),
        ("star_mass_msun", C.c_float), ("softening_AU", C.c_float), ("theta", C.c_float),
        ("collision_radius_factor", C.c_float), ("restitution", C.c_float),
        ("gas_drag_rate", C.c_float), ("dt", C.c_float), ("total_time", C.c_float),
        ("output_every_n_steps", C.c_int), ("output_dir", C.c_char * 1024),
        ("perturber_enabled", C.c_int), ("perturber_mass_mjup", C.c_float),
        ("perturber_radius_AU", C.c_float), ("perturber_phase0", C.c_float)]

    def to_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["output_dir"] = self.output_dir.decode()
        d["perturber_enabled"] = bool(self.perturber_enabled)
        return d


class nbody_perturber(C.Structure):
    _fields_ = [("enabled", C.c_int), ("r", C.c_float), ("mass_msun", C.c_float),
                ("phase0", C.c_float), ("omega", C.c_float),
                ("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class nbody_tree_stats(C.Structure):
    _fields_ = [("n_bodies", C.c_int), ("n_nodes", C.c_int), ("bbox_min", C.c_float * 3),
                ("bbox_max", C.c_float * 3), ("root_center", C.c_float * 3),
                ("root_half", C.c_float), ("root_mass", C.c_double),
                ("root_com", C.c_double * 3), ("interactions", C.c_ulonglong),
                ("status", C.c_int), ("walk_nodes_visited", C.c_ulonglong),
                ("walk_stack_spills", C.c_ulonglong)]


class nbody_aggregate(C.Structure):
    _fields_ = [("id", C.c_int), ("n_particles", C.c_int), ("mass_msun", C.c_float),
                ("cx", C.c_float), ("cy", C.c_float), ("cz", C.c_float),
                ("vx", C.c_float), ("vy", C.c_float), ("vz", C.c_float),
                ("dist_center", C.c_float), ("first_member", C.c_int)]


class nbody_sim_params(C.Structure):
    _fields_ = [("dt", C.c_float), ("theta", C.c_float), ("softening", C.c_float),
                ("star_mass", C.c_float), ("r_coll", C.c_float), ("restitution", C.c_float),
                ("gas_drag_rate", C.c_float), ("perturber_enabled", C.c_int),
                ("perturber_mass_mjup", C.c_float), ("perturber_radius_au", C.c_float),
                ("perturber_phase0", C.c_float), ("state_precision", C.c_int),
                ("leaf_max", C.c_int), ("targets_per_lane", C.c_int), ("walk_mode", C.c_int),
                ("group_span", C.c_int), ("fuse_collisions", C.c_int), ("span_walk", C.c_int),
                ("spill_cap", C.c_int)]


NBODY_PHASES = 6
PHASE_NAMES = ("stream", "sort", "permute", "tree", "walk", "collide")


class nbody_sim_profile(C.Structure):
    _fields_ = [("ms", C.c_double * NBODY_PHASES), ("steps", C.c_int),
                ("launches", C.c_ulonglong)]


class nbody_sim_stats(C.Structure):
    _fields_ = [("n", C.c_int), ("steps_done", C.c_int), ("n_nodes", C.c_int),
                ("interactions", C.c_ulonglong), ("status", C.c_int),
                ("walk_nodes_visited", C.c_ulonglong), ("walk_stack_spills", C.c_ulonglong),
                ("walk_groups", C.c_ulonglong), ("launches", C.c_ulonglong),
                ("graph_launches", C.c_ulonglong), ("targets_per_lane", C.c_int),
                ("leaf_max", C.c_int), ("walk_mode", C.c_int), ("group_span", C.c_int),
                ("span_walk", C.c_int), ("span_shared", C.c_ulonglong),
                ("span_frontier", C.c_ulonglong), ("spans", C.c_ulonglong)]


class nbody_frame(C.Structure):
    _fields_ = [("n", C.c_int), ("frame_index", C.c_int), ("sim_time", C.c_float),
                ("x", _F), ("y", _F), ("z", _F), ("agg_size", _U16),
                ("aggregates", C.POINTER(nbody_aggregate)), ("n_aggregates", C.c_int)]


class nbody_disk_spec(C.Structure):
    _fields_ = [("n", C.c_int), ("perturber_enabled", C.c_int),
                ("perturber_mass_mjup", C.c_float), ("perturber_radius_au", C.c_float),
                ("perturber_phase0", C.c_float)]


class nbody_ensemble_stats(C.Structure):
    _fields_ = [("n_disks", C.c_int), ("n_total", C.c_int), ("steps_done", C.c_int),
                ("targets_per_lane", C.c_int), ("leaf_max", C.c_int), ("status", C.c_int),
                ("interactions", C.c_ulonglong), ("launches", C.c_ulonglong),
                ("graph_launches", C.c_ulonglong), ("walk_mode", C.c_int)]


class nbody_adjoint_stats(C.Structure):
    _fields_ = [("n", C.c_int), ("n_steps", C.c_int), ("ms_forward", C.c_float),
                ("ms_backward", C.c_float), ("ms_replay", C.c_float),
                ("tape_bytes", C.c_ulonglong), ("state_bytes", C.c_ulonglong),
                ("launches", C.c_ulonglong)]


# (name, restype, argtypes): every symbol include/nbody_b200.h declares
SIGNATURES = [
    ("nbody_last_error", C.c_char_p, []),
    ("nbody_abi_version", C.c_int, []),
    ("nbody_config_defaults", None, [C.POINTER(nbody_config)]),
    ("nbody_config_load", C.c_int, [C.c_char_p, C.POINTER(nbody_config)]),
    ("nbody_particle_radius", C.c_float, [C.c_float]),
    ("nbody_perturber_make", None, [C.POINTER(nbody_config), C.POINTER(nbody_perturber)]),
    ("nbody_perturber_update", None, [C.POINTER(nbody_perturber), C.c_float]),
    ("nbody_tree_create", C.c_int, [C.c_int, C.POINTER(_VP)]),
    ("nbody_tree_destroy", None, [_VP]),
    ("nbody_tree_reset", C.c_int, [_VP]),
    ("nbody_tree_bbox", C.c_int, [_VP, C.POINTER(nbody_particles)]),
    ("nbody_tree_build", C.c_int, [_VP, C.POINTER(nbody_particles)]),
    ("nbody_tree_summarize", C.c_int, [_VP]),
    ("nbody_tree_sort", C.c_int, [_VP]),
    ("nbody_tree_sort_idx", _I, [_VP]),
    ("nbody_tree_sort_idx_copy", C.c_int, [_VP, _I, C.c_int]),
    ("nbody_tree_force", C.c_int, [_VP, C.POINTER(nbody_particles), C.c_float, C.c_float,
                                   C.c_float]),
    ("nbody_tree_collide", C.c_int, [_VP, C.POINTER(nbody_particles), C.c_float, C.c_float]),
    ("nbody_tree_set_leaf_max", C.c_int, [_VP, C.c_int]),
    ("nbody_tree_collision_report", C.c_int, [_VP, C.c_float, C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)]),
    ("nbody_tree_set_targets_per_lane", C.c_int, [_VP, C.c_int]),
    ("nbody_tree_stats_get", C.c_int, [_VP, C.POINTER(nbody_tree_stats)]),
    ("nbody_half_kick", C.c_int, [C.POINTER(nbody_particles), C.c_float]),
    ("nbody_drift", C.c_int, [C.POINTER(nbody_particles), C.c_float]),
    ("nbody_reset_acc", C.c_int, [C.POINTER(nbody_particles)]),
    ("nbody_gas_drag", C.c_int, [C.POINTER(nbody_particles), C.c_float, C.c_float, C.c_float]),
    ("nbody_perturber_force", C.c_int, [C.POINTER(nbody_particles), C.c_float, C.c_float,
                                        C.c_float, C.c_float, C.c_float]),
    ("nbody_fof", C.c_int, [_VP, _VP, _VP, _VP, C.c_int, C.c_float, _VP, _VP, _I]),
    ("nbody_fof_noalloc", C.c_int, [_VP, _VP, _VP, C.c_int, C.c_float, _VP, _VP, _I]),
    ("nbody_aggregates", C.c_int, [_F, _F, _F, _F, _F, _F, _I, C.c_int, C.c_float,
                                   C.POINTER(nbody_aggregate), C.c_int, _I]),
    ("nbody_writer_open", C.c_int, [C.c_char_p, C.POINTER(nbody_config), C.POINTER(_VP)]),
    ("nbody_writer_frame", C.c_int, [_VP, _F, _F, _F, C.c_int, C.c_float, _U16]),
    ("nbody_writer_stats", C.c_int, [_VP, C.POINTER(nbody_aggregate), C.c_int, C.c_int,
                                     C.c_float]),
    ("nbody_writer_perturber", C.c_int, [_VP, C.c_int, C.c_float, C.c_int, C.c_float, C.c_float,
                                         C.c_float, C.c_float, C.c_float]),
    ("nbody_writer_finalize", C.c_int, [_VP, C.c_int]),
    ("nbody_writer_close", None, [_VP]),
    ("nbody_sim_params_from_config", None, [C.POINTER(nbody_config),
                                            C.POINTER(nbody_sim_params)]),
    ("nbody_sim_create", C.c_int, [C.POINTER(nbody_sim_params), C.c_int, C.POINTER(_VP)]),
    ("nbody_sim_destroy", None, [_VP]),
    ("nbody_sim_set_stream", C.c_int, [_VP, _VP]),
    ("nbody_sim_set_state", C.c_int, [_VP] + [_VP] * 7 + [C.c_int]),
    ("nbody_sim_set_state_f64", C.c_int, [_VP] + [_VP] * 7 + [C.c_int]),
    ("nbody_sim_step", C.c_int, [_VP, C.c_int]),
    ("nbody_sim_step_open", C.c_int, [_VP, C.c_int]),
    ("nbody_sim_close", C.c_int, [_VP]),
    ("nbody_sim_sync", C.c_int, [_VP]),
    ("nbody_sim_get_state", C.c_int, [_VP] + [_VP] * 9 + [C.c_int]),
    ("nbody_sim_get_state_f64", C.c_int, [_VP] + [_VP] * 6 + [C.c_int]),
    ("nbody_sim_fof", C.c_int, [_VP, C.c_float, _VP, _VP, _I, C.c_int]),
    ("nbody_sim_stats_get", C.c_int, [_VP, C.POINTER(nbody_sim_stats)]),
    ("nbody_sim_set_profiling", C.c_int, [_VP, C.c_int]),
    ("nbody_sim_profile_get", C.c_int, [_VP, C.POINTER(nbody_sim_profile), C.c_int]),
    ("nbody_sim_step_host", C.c_int, [_VP] + [_VP] * 10 + [C.c_int]),
    ("nbody_sim_autotune", C.c_int, [_VP, _VP, C.c_int, _VP]),
    ("nbody_sim_set_graphs", C.c_int, [_VP, C.c_int]),
    ("nbody_sim_output_begin", C.c_int, [_VP, C.c_float, C.c_float, C.c_float, C.c_int]),
    ("nbody_sim_output_wait", C.c_int, [_VP, C.POINTER(nbody_frame)]),
    ("nbody_ensemble_create", C.c_int, [C.POINTER(nbody_sim_params), C.POINTER(nbody_disk_spec),
                                        C.c_int, C.POINTER(_VP)]),
    ("nbody_ensemble_destroy", C.c_int, [_VP]),
    ("nbody_ensemble_set_stream", C.c_int, [_VP, _VP]),
    ("nbody_ensemble_set_state", C.c_int, [_VP] + [_VP] * 7 + [C.c_int]),
    ("nbody_ensemble_set_state_f64", C.c_int, [_VP] + [_VP] * 7 + [C.c_int]),
    ("nbody_ensemble_step", C.c_int, [_VP, C.c_int]),
    ("nbody_ensemble_sync", C.c_int, [_VP]),
    ("nbody_ensemble_get_state", C.c_int, [_VP] + [_VP] * 9 + [C.c_int]),
    ("nbody_ensemble_get_state_f64", C.c_int, [_VP] + [_VP] * 9 + [C.c_int]),
    ("nbody_ensemble_step_host", C.c_int, [_VP] + [_VP] * 10 + [C.c_int]),
    ("nbody_ensemble_autotune", C.c_int, [_VP, _VP, C.c_int, _VP]),
    ("nbody_ensemble_set_graphs", C.c_int, [_VP, C.c_int]),
    ("nbody_ensemble_stats_get", C.c_int, [_VP, C.POINTER(nbody_ensemble_stats)]),
    ("nbody_adjoint_create", C.c_int, [C.POINTER(nbody_sim_params), C.c_int, C.c_int,
                                       C.POINTER(_VP)]),
    ("nbody_adjoint_create_mode", C.c_int, [C.POINTER(nbody_sim_params), C.c_int, C.c_int,
                                            C.c_int, C.c_int, C.POINTER(_VP)]),
    ("nbody_adjoint_destroy", C.c_int, [_VP]),
    ("nbody_adjoint_set_stream", C.c_int, [_VP, _VP]),
    ("nbody_adjoint_forward", C.c_int, [_VP] + [_VP] * 7 + [C.c_double, C.c_double] + [_VP] * 6),
    ("nbody_adjoint_replay", C.c_int, [_VP] + [_VP] * 6 + [C.c_double, C.c_double, C.c_int]
     + [_VP] * 6),
    ("nbody_adjoint_backward", C.c_int, [_VP] + [_VP] * 13),
    ("nbody_adjoint_stats_get", C.c_int, [_VP, C.POINTER(nbody_adjoint_stats)]),
    ("nbody_make_disks_device", C.c_int, [_VP, _VP, C.c_int] + [C.c_double] * 5 + [_VP] * 7),
    ("nbody_direct_f64", C.c_int, [_VP] * 4 + [C.c_int, _VP, C.c_int, C.c_double] + [_VP] * 4),
    ("nbody_radix_sort_u32", C.c_int, [_VP, _VP, C.c_int, C.c_int]),
    ("nbody_radix_sort_u64", C.c_int, [_VP, _VP, C.c_int, C.c_int]),
    ("nbody_selftest_sort_wait", C.c_int, [_I]),
    ("nbody_radix_tree_u32", C.c_int, [_VP, C.c_int, C.c_int] + [_VP] * 5),
    ("nbody_make_disk", C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                  C.c_double, C.c_uint64, _D, _D, _D, _D, _D, _D]),
]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python nbody-sim_b200/build.py` "
            "(there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def _check(rc: int):
    if rc != NBODY_OK:
        raise NBodyError(rc, lib.nbody_last_error().decode())


# ------------------------------------------------------------------ config
def default_config() -> nbody_config:
    c = nbody_config()
    lib.nbody_config_defaults(C.byref(c))
    return c


def load_config(path: str) -> nbody_config:
    """loadConfig (src/config/Config.cpp:6-55); raises NBodyError."""
    c = nbody_config()
    _check(lib.nbody_config_load(os.fsencode(path), C.byref(c)))
    return c


def particle_physical_radius(particle_mass_msun: float) -> float:
    return float(lib.nbody_particle_radius(particle_mass_msun))


def make_perturber(cfg: nbody_config) -> nbody_perturber:
    p = nbody_perturber()
    lib.nbody_perturber_make(C.byref(cfg), C.byref(p))
    return p


def update_perturber(p: nbody_perturber, sim_time: float) -> None:
    lib.nbody_perturber_update(C.byref(p), sim_time)


# --------------------------------------------------------------- particles
FIELDS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "mass")


@dataclass
class ParticleData:
    """SoA particles (include/ParticleData.h:19-32): torch CUDA float tensors
    (device) or numpy float32 arrays (host), plus int ids."""

    n: int
    arrays: dict = field(default_factory=dict)

    def __getattr__(self, k):
        a = self.__dict__.get("arrays", {})
        if k in a:
            return a[k]
        raise AttributeError(k)

    def struct(self) -> nbody_particles:
        s = nbody_particles()
        s.n = self.n
        for k in FIELDS:
            a = self.arrays.get(k)
            if a is not None:
                setattr(s, k, C.cast(_data_ptr(a), _F))
        if self.arrays.get("id") is not None:
            s.id = C.cast(_data_ptr(self.arrays["id"]), _I)
        return s


def _data_ptr(a):
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


def allocate_particles_cpu(n: int) -> ParticleData:
    arr = {k: np.zeros(n, np.float32) for k in FIELDS}
    arr["id"] = np.zeros(n, np.int32)
    return ParticleData(n, arr)


def allocate_particles_gpu(n: int, device="cuda") -> ParticleData:
    import torch
    arr = {k: torch.zeros(n, dtype=torch.float32, device=device) for k in FIELDS}
    arr["id"] = torch.zeros(n, dtype=torch.int32, device=device)
    return ParticleData(n, arr)


def copy_to_gpu(cpu: ParticleData, gpu: ParticleData) -> None:
    """copyToGPU (include/ParticleData.h:90-105), same size check."""
    import torch
    if cpu.n != gpu.n:
        raise RuntimeError(f"copyToGPU: CPU n={cpu.n} != GPU n={gpu.n}")
    for k in FIELDS + ("id",):
        gpu.arrays[k].copy_(torch.from_numpy(np.ascontiguousarray(cpu.arrays[k])))


def copy_to_cpu(gpu: ParticleData, cpu: ParticleData) -> None:
    """copyToCPU (include/ParticleData.h:108-123)."""
    if cpu.n != gpu.n:
        raise RuntimeError(f"copyToCPU: GPU n={gpu.n} != CPU n={cpu.n}")
    for k in FIELDS + ("id",):
        cpu.arrays[k][:] = gpu.arrays[k].cpu().numpy()


# ------------------------------------------------------------ phase API
class Octree:
    """OctreeData + its launchers (include/BHTree.cuh:38-50); each call
    synchronises before returning, as the reference launchers do."""

    def __init__(self, n_bodies: int, leaf_max: int | None = None,
                 targets_per_lane: int | None = None):
        h = _VP()
        _check(lib.nbody_tree_create(n_bodies, C.byref(h)))
        self.h = h
        self.n_bodies = n_bodies
        if leaf_max is not None:
            _check(lib.nbody_tree_set_leaf_max(self.h, leaf_max))
        if targets_per_lane is not None:
            _check(lib.nbody_tree_set_targets_per_lane(self.h, targets_per_lane))

    def close(self):
        if getattr(self, "h", None):
            lib.nbody_tree_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reset(self):
        _check(lib.nbody_tree_reset(self.h))

    def bbox(self, p: ParticleData):
        s = p.struct()
        _check(lib.nbody_tree_bbox(self.h, C.byref(s)))

    def build(self, p: ParticleData):
        s = p.struct()
        _check(lib.nbody_tree_build(self.h, C.byref(s)))

    def summarize(self):
        _check(lib.nbody_tree_summarize(self.h))

    def collision_report(self, r_coll: float):
        """(pairs, missed): ordered pairs closer than r_coll, and how many of
        them the reference's collision cell prune would skip
        (nbody_tree_collision_report)."""
        pairs, missed = C.c_ulonglong(), C.c_ulonglong()
        _check(lib.nbody_tree_collision_report(self.h, r_coll, C.byref(pairs), C.byref(missed)))
        return pairs.value, missed.value

    def sort(self):
        _check(lib.nbody_tree_sort(self.h))

    def sort_idx(self) -> np.ndarray:
        """tree.sort_idx (include/BHTree.cuh:20) copied to the host."""
        out = np.zeros(self.n_bodies, np.int32)
        _check(lib.nbody_tree_sort_idx_copy(self.h, out.ctypes.data_as(_I), 0))
        return out

    def force(self, p: ParticleData, theta: float, softening: float, star_mass: float):
        s = p.struct()
        _check(lib.nbody_tree_force(self.h, C.byref(s), theta, softening, star_mass))

    def collide(self, p: ParticleData, r_coll: float, restitution: float):
        s = p.struct()
        _check(lib.nbody_tree_collide(self.h, C.byref(s), r_coll, restitution))

    def stats(self) -> nbody_tree_stats:
        st = nbody_tree_stats()
        _check(lib.nbody_tree_stats_get(self.h, C.byref(st)))
        return st

    def fof(self, x, y, z, link_length: float):
        """Device FoF over torch CUDA float tensors -> (labels, agg_size, n_groups)."""
        import torch
        n = x.numel()
        labels = torch.empty(n, dtype=torch.int32, device=x.device)
        agg = torch.empty(n, dtype=torch.int16, device=x.device)
        ng = C.c_int()
        _check(lib.nbody_fof(self.h, x.data_ptr(), y.data_ptr(), z.data_ptr(), n, link_length,
                             labels.data_ptr(), agg.data_ptr(), C.byref(ng)))
        return labels, agg, ng.value  # agg: int16 tensor holding uint16 sizes


def half_kick(p: ParticleData, dt_half: float):
    s = p.struct(); _check(lib.nbody_half_kick(C.byref(s), dt_half))


def drift(p: ParticleData, dt: float):
    s = p.struct(); _check(lib.nbody_drift(C.byref(s), dt))


def reset_acceleration(p: ParticleData):
    s = p.struct(); _check(lib.nbody_reset_acc(C.byref(s)))


def gas_drag(p: ParticleData, drag_rate: float, dt: float, star_mass: float):
    s = p.struct(); _check(lib.nbody_gas_drag(C.byref(s), drag_rate, dt, star_mass))


def perturber_force(p: ParticleData, px, py, pz, pmass, softening):
    s = p.struct(); _check(lib.nbody_perturber_force(C.byref(s), px, py, pz, pmass, softening))


# --------------------------------------------------------------- FoF
def fof_noalloc(x, y, z, link_length: float):
    """nbody_fof_noalloc on torch CUDA float tensors: the device FoF with its
    scratch in the library's static device array (no allocation by the
    library; n <= FOF_NOALLOC_MAX_N).  Returns (labels, agg_size as int16
    holding uint16 sizes, n_groups)."""
    import torch
    n = x.numel()
    labels = torch.empty(n, dtype=torch.int32, device=x.device)
    agg = torch.empty(n, dtype=torch.int16, device=x.device)
    ng = C.c_int()
    _check(lib.nbody_fof_noalloc(x.data_ptr(), y.data_ptr(), z.data_ptr(), n, link_length,
                                 labels.data_ptr(), agg.data_ptr(), C.byref(ng)))
    return labels, agg, ng.value


def fof_noalloc_setup():
    """nbody_fof_noalloc with n = 0 on the current device: the device's
    one-time set-up (the static scratch and the FoF kernels take their device
    memory now, under lazy module loading), so that later calls take none."""
    ng = C.c_int()
    _check(lib.nbody_fof_noalloc(None, None, None, 0, 0.0, None, None, C.byref(ng)))


@dataclass
class Aggregate:
    """include/Aggregate.h:4-12."""
    id: int
    n_particles: int
    mass_msun: float
    cx: float
    cy: float
    cz: float
    vx: float
    vy: float
    vz: float
    dist_center: float
    particle_ids: list


def aggregates_from_labels(x, y, z, vx, vy, vz, labels, particle_mass: float):
    """Aggregate records (Aggregate.cpp:54-74) from host labels, ordered by
    smallest member index; returns the raw nbody_aggregate array."""
    arrs = [np.ascontiguousarray(a, np.float32) for a in (x, y, z, vx, vy, vz)]
    lab = np.ascontiguousarray(labels, np.int32)
    n = len(lab)
    cnt = C.c_int()
    _check(lib.nbody_aggregates(*[a.ctypes.data_as(_F) for a in arrs], lab.ctypes.data_as(_I), n,
                                particle_mass, None, 0, C.byref(cnt)))
    out = (nbody_aggregate * max(cnt.value, 1))()
    _check(lib.nbody_aggregates(*[a.ctypes.data_as(_F) for a in arrs], lab.ctypes.data_as(_I), n,
                                particle_mass, out, cnt.value, C.byref(cnt)))
    return out, cnt.value


def detect_aggregates(p: ParticleData, link_length: float, cfg: nbody_config, tree=None):
    """detectAggregates (include/Aggregate.h:17-18) on host particles: the
    links and union-find run on the GPU, the records on the host."""
    import torch
    n = p.n
    own = tree is None
    tree = tree or Octree(max(n, 1))
    try:
        xs = [torch.from_numpy(np.ascontiguousarray(p.arrays[k], np.float32)).cuda()
              for k in ("x", "y", "z")]
        labels, _, _ = tree.fof(*xs, link_length)
        lab = labels.cpu().numpy()
    finally:
        if own:
            tree.close()
    recs, g = aggregates_from_labels(p.x, p.y, p.z, p.vx, p.vy, p.vz, lab, cfg.particle_mass_msun)
    members = {}
    for i, l in enumerate(lab):
        members.setdefault(int(l), []).append(i)
    out = []
    for k in range(g):
        r = recs[k]
        out.append(Aggregate(r.id, r.n_particles, r.mass_msun, r.cx, r.cy, r.cz, r.vx, r.vy,
                             r.vz, r.dist_center, members[r.first_member]))
    return out


# ------------------------------------------------------------- writer
class OutputWriter:
    """frames.bin + stats.csv writer (include/OutputWriter.h:15-51)."""

    def __init__(self, output_dir: str, cfg: nbody_config):
        h = _VP()
        _check(lib.nbody_writer_open(os.fsencode(output_dir), C.byref(cfg), C.byref(h)))
        self.h = h

    def write_frame(self, p: ParticleData, sim_time: float, agg_sizes):
        agg = np.ascontiguousarray(agg_sizes, np.uint16)
        if len(agg) != p.n:
            raise RuntimeError("OutputWriter::writeFrame: agg_sizes_per_particle size mismatch")
        xs = [np.ascontiguousarray(p.arrays[k], np.float32) for k in ("x", "y", "z")]
        _check(lib.nbody_writer_frame(self.h, *[a.ctypes.data_as(_F) for a in xs], p.n, sim_time,
                                      agg.ctypes.data_as(_U16)))

    def write_stats(self, aggs, frame_idx: int, sim_time: float, count: int | None = None):
        """aggs: Aggregate-like objects, or (with count) a ctypes array / pointer
        of nbody_aggregate records passed to the writer as they are."""
        if count is not None:
            _check(lib.nbody_writer_stats(self.h, C.cast(aggs, C.POINTER(nbody_aggregate)),
                                          count, frame_idx, sim_time))
            return
        arr = (nbody_aggregate * max(len(aggs), 1))()
        for k, a in enumerate(aggs):
            r = arr[k]
            r.id, r.n_particles, r.mass_msun = a.id, a.n_particles, a.mass_msun
            r.cx, r.cy, r.cz, r.vx, r.vy, r.vz = a.cx, a.cy, a.cz, a.vx, a.vy, a.vz
            r.dist_center = a.dist_center
        _check(lib.nbody_writer_stats(self.h, arr, len(aggs), frame_idx, sim_time))

    def write_perturber_stats(self, frame_idx, sim_time, n_aggregates, px, py, pz, mass, omega):
        _check(lib.nbody_writer_perturber(self.h, frame_idx, sim_time, n_aggregates, px, py, pz,
                                          mass, omega))

    def finalize(self, total_frames: int):
        _check(lib.nbody_writer_finalize(self.h, total_frames))

    def close(self):
        if getattr(self, "h", None):
            lib.nbody_writer_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------- engine
# the engine's default walk variant (nbody_sim_params.walk_mode; vote, 64 registers)
WALK_MODE_DEFAULT = 1
# walk target groups (nbody_sim_params.group_span): 0 lets the engine choose
GROUP_SPAN_DEFAULT = 0


def sim_params(cfg: nbody_config | None = None, **kw) -> nbody_sim_params:
    p = nbody_sim_params()
    if cfg is not None:
        lib.nbody_sim_params_from_config(C.byref(cfg), C.byref(p))
    else:
        p.dt, p.theta, p.softening, p.star_mass, p.leaf_max = 0.01, 0.5, 0.01, 1.0, 0
        p.targets_per_lane = 1
        p.walk_mode = WALK_MODE_DEFAULT
        p.group_span = GROUP_SPAN_DEFAULT
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class Sim:
    """The GPU-resident step engine (nbody_sim_* in include/nbody_b200.h)."""

    def __init__(self, params: nbody_sim_params, n: int):
        h = _VP()
        _check(lib.nbody_sim_create(C.byref(params), n, C.byref(h)))
        self.h, self.n, self.params = h, n, params

    def close(self):
        if getattr(self, "h", None):
            lib.nbody_sim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int):
        _check(lib.nbody_sim_set_stream(self.h, stream_ptr))

    def set_state(self, x, y, z, vx, vy, vz, mass):
        """Host numpy (float32 or float64) or CUDA torch tensors, caller order."""
        arrs = [x, y, z, vx, vy, vz]
        on_dev = hasattr(x, "data_ptr")
        if on_dev:
            dbl = str(x.dtype) == "torch.float64"
            ptrs = [a.data_ptr() for a in arrs]
            mptr = mass.data_ptr()
            keep = None
        else:
            dbl = np.asarray(x).dtype == np.float64
            keep = [np.ascontiguousarray(a, np.float64 if dbl else np.float32) for a in arrs]
            km = np.ascontiguousarray(mass, np.float32)
            ptrs = [a.ctypes.data for a in keep]
            mptr = km.ctypes.data
        fn = lib.nbody_sim_set_state_f64 if dbl else lib.nbody_sim_set_state
        _check(fn(self.h, *ptrs, mptr, int(on_dev)))
        del keep

    def step(self, nsteps: int = 1):
        _check(lib.nbody_sim_step(self.h, nsteps))

    def step_open(self, nsteps: int = 1):
        """nsteps steps, the last left open (nbody_sim_step_open): a loop of
        one-step calls then runs every step in its fused form."""
        _check(lib.nbody_sim_step_open(self.h, nsteps))

    def close_steps(self):
        """Finishes an open step (nbody_sim_close)."""
        _check(lib.nbody_sim_close(self.h))

    def sync(self):
        _check(lib.nbody_sim_sync(self.h))

    def get_state(self, double: bool = False, accel: bool = True):
        """Host numpy state in caller order: dict x..vz (+ ax..az)."""
        n = self.n
        dt = np.float64 if double else np.float32
        out = {k: np.zeros(n, dt) for k in ("x", "y", "z", "vx", "vy", "vz")}
        if double:
            _check(lib.nbody_sim_get_state_f64(self.h, *[out[k].ctypes.data for k in out], 0))
        else:
            acc = {k: np.zeros(n, np.float32) for k in ("ax", "ay", "az")} if accel else None
            aptr = [acc[k].ctypes.data for k in ("ax", "ay", "az")] if accel else [None] * 3
            _check(lib.nbody_sim_get_state(self.h, *[out[k].ctypes.data for k in out], *aptr, 0))
            if accel:
                out.update(acc)
        return out

    def fof(self, link_length: float):
        labels = np.zeros(self.n, np.int32)
        agg = np.zeros(self.n, np.uint16)
        ng = C.c_int()
        _check(lib.nbody_sim_fof(self.h, link_length, labels.ctypes.data, agg.ctypes.data,
                                 C.byref(ng), 0))
        return labels, agg, ng.value

    def stats(self) -> nbody_sim_stats:
        st = nbody_sim_stats()
        _check(lib.nbody_sim_stats_get(self.h, C.byref(st)))
        return st

    def set_profiling(self, on: bool = True):
        _check(lib.nbody_sim_set_profiling(self.h, int(on)))

    def autotune(self, candidates=None):
        """Times force evaluations per (targets_per_lane, leaf_max, walk_mode,
        group_span) and keeps the fastest (nbody_sim_autotune).  Returns
        [(tpl, leaf_max, walk_mode, group_span, ms), ...]."""
        if candidates is None:
            candidates = [(1, 8, 1, 0), (1, 8, 0, 0), (1, 8, 2, 0), (1, 16, 1, 0), (1, 16, 2, 0),
                          (1, 4, 2, 0)]
        flat = np.ascontiguousarray(np.array(candidates, np.int32).reshape(-1))
        ms = np.zeros(len(candidates), np.float32)
        _check(lib.nbody_sim_autotune(self.h, flat.ctypes.data, len(candidates), ms.ctypes.data))
        return [(*map(int, c), float(t)) for c, t in zip(candidates, ms)]

    def set_graphs(self, on: bool = True):
        _check(lib.nbody_sim_set_graphs(self.h, int(on)))

    def profile(self, reset: bool = True) -> dict:
        pr = nbody_sim_profile()
        _check(lib.nbody_sim_profile_get(self.h, C.byref(pr), int(reset)))
        d = {name: pr.ms[k] for k, name in enumerate(PHASE_NAMES)}
        d["steps"] = pr.steps
        d["launches"] = pr.launches
        return d

    def output_begin(self, link_length: float, particle_mass: float, sim_time: float,
                     frame_index: int):
        """Enqueue one output step (snapshot, FoF, agg_size, aggregates) on the GPU."""
        _check(lib.nbody_sim_output_begin(self.h, link_length, particle_mass, sim_time,
                                          frame_index))

    def output_wait(self, copy: bool = True) -> dict:
        """Oldest frame in flight: x, y, z, agg_size (numpy) and the aggregate
        records.  copy=False returns views of the engine's pinned buffers
        (valid until the slot is reused) and the records as a raw pointer
        ("aggregates_ptr"), without per-record Python objects."""
        f = nbody_frame()
        _check(lib.nbody_sim_output_wait(self.h, C.byref(f)))
        n = f.n
        grab = (lambda a: np.array(a)) if copy else (lambda a: a)
        out = {"frame_index": f.frame_index, "sim_time": f.sim_time,
               "x": grab(np.ctypeslib.as_array(f.x, (n,))),
               "y": grab(np.ctypeslib.as_array(f.y, (n,))),
               "z": grab(np.ctypeslib.as_array(f.z, (n,))),
               "agg_size": grab(np.ctypeslib.as_array(f.agg_size, (n,))),
               "n_aggregates": f.n_aggregates, "aggregates_ptr": f.aggregates}
        if copy:
            out["aggregates"] = [nbody_aggregate.from_buffer_copy(f.aggregates[i])
                                 for i in range(f.n_aggregates)]
        return out

    def step_host(self, st: dict, mass, nsteps: int = 1):
        """Host round trip (copyToGPU, nsteps, copyToCPU) on float32 arrays in place."""
        keys = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")
        _check(lib.nbody_sim_step_host(self.h, *[st[k].ctypes.data for k in keys],
                                       mass.ctypes.data, nsteps))


class Ensemble:
    """Many independent disks stepped together (nbody_ensemble_* in include/nbody_b200.h).

    ``disks`` is a list of dicts with keys n, perturber_enabled,
    perturber_mass_mjup, perturber_radius_au, perturber_phase0.  State arrays
    hold every disk's bodies concatenated in disk order.
    """

    def __init__(self, params: nbody_sim_params, disks):
        specs = (nbody_disk_spec * len(disks))()
        for k, d in enumerate(disks):
            specs[k].n = int(d["n"])
            specs[k].perturber_enabled = int(d.get("perturber_enabled", 0))
            specs[k].perturber_mass_mjup = float(d.get("perturber_mass_mjup", 1.0))
            specs[k].perturber_radius_au = float(d.get("perturber_radius_au", 5.2))
            specs[k].perturber_phase0 = float(d.get("perturber_phase0", 0.0))
        h = _VP()
        _check(lib.nbody_ensemble_create(C.byref(params), specs, len(disks), C.byref(h)))
        self.h, self.params = h, params
        self.sizes = [int(d["n"]) for d in disks]
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)]).astype(np.int64)
        self.n = int(self.offsets[-1])

    def close(self):
        if getattr(self, "h", None):
            lib.nbody_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int):
        _check(lib.nbody_ensemble_set_stream(self.h, stream_ptr))

    def set_state(self, x, y, z, vx, vy, vz, mass):
        """Host numpy (float32 or float64) or CUDA torch tensors, disk order."""
        arrs = [x, y, z, vx, vy, vz]
        on_dev = hasattr(x, "data_ptr")
        if on_dev:
            dbl = str(x.dtype) == "torch.float64"
            ptrs = [a.data_ptr() for a in arrs]
            mptr = mass.data_ptr()
            keep = None
        else:
            dbl = np.asarray(x).dtype == np.float64
            keep = [np.ascontiguousarray(a, np.float64 if dbl else np.float32) for a in arrs]
            km = np.ascontiguousarray(mass, np.float32)
            ptrs = [a.ctypes.data for a in keep]
            mptr = km.ctypes.data
        fn = lib.nbody_ensemble_set_state_f64 if dbl else lib.nbody_ensemble_set_state
        _check(fn(self.h, *ptrs, mptr, int(on_dev)))
        del keep

    def step(self, nsteps: int = 1):
        _check(lib.nbody_ensemble_step(self.h, nsteps))

    def sync(self):
        _check(lib.nbody_ensemble_sync(self.h))

    def get_state(self, double: bool = False, accel: bool = True):
        """Host numpy state in disk order: dict x..vz (+ ax..az)."""
        n = self.n
        dt = np.float64 if double else np.float32
        out = {k: np.zeros(n, dt) for k in ("x", "y", "z", "vx", "vy", "vz")}
        acc = {k: np.zeros(n, np.float32) for k in ("ax", "ay", "az")} if accel else None
        aptr = [acc[k].ctypes.data for k in ("ax", "ay", "az")] if accel else [None] * 3
        fn = lib.nbody_ensemble_get_state_f64 if double else lib.nbody_ensemble_get_state
        _check(fn(self.h, *[out[k].ctypes.data for k in out], *aptr, 0))
        if accel:
            out.update(acc)
        return out

    def step_host(self, st: dict, mass, nsteps: int = 1):
        """Host round trip on float64 x..vz and float32 ax..az arrays, in place."""
        keys = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")
        _check(lib.nbody_ensemble_step_host(self.h, *[st[k].ctypes.data for k in keys],
                                            mass.ctypes.data, nsteps))

    def autotune(self, candidates=None):
        """Times force evaluations per (targets_per_lane, leaf_max, walk_mode);
        keeps the fastest.  Returns [(tpl, leaf_max, walk_mode, ms), ...]."""
        if candidates is None:
            candidates = [(1, 8, 0), (1, 8, 1), (1, 8, 2), (1, 4, 2), (1, 16, 2), (2, 8, 0)]
        flat = np.ascontiguousarray(np.array(candidates, np.int32).reshape(-1))
        ms = np.zeros(len(candidates), np.float32)
        _check(lib.nbody_ensemble_autotune(self.h, flat.ctypes.data, len(candidates),
                                           ms.ctypes.data))
        return [(int(a), int(b), int(c), float(t)) for (a, b, c), t in zip(candidates, ms)]

    def set_graphs(self, on: bool = True):
        _check(lib.nbody_ensemble_set_graphs(self.h, int(on)))

    def stats(self) -> nbody_ensemble_stats:
        st = nbody_ensemble_stats()
        _check(lib.nbody_ensemble_stats_get(self.h, C.byref(st)))
        return st


class Adjoint:
    """Differentiable trajectory of one disk (nbody_adjoint_* in include/nbody_b200.h).

    States are (3, n) float64 CUDA tensors (rows x, y, z) in caller order;
    ``mass`` a float32 CUDA tensor.  ``forward`` records the tape,
    ``backward`` returns the adjoints of the initial state and of the
    perturber's (mass in M_J, radius in AU), ``replay`` reruns the frozen-tree
    forward with other inputs."""

    MODES = {"tape": 0, "checkpoint": 1, "direct": 2}

    def __init__(self, params: nbody_sim_params, n: int, n_steps: int, mode: str = "tape",
                 checkpoint_every: int = 50):
        """mode: "tape" (every level in HBM), "checkpoint" (FP64 checkpoints
        every ``checkpoint_every`` levels, levels rebuilt by time-reversed
        leapfrog in the backward) or "direct" (FP64 direct-sum self-gravity:
        the reference gradient)."""
        h = _VP()
        _check(lib.nbody_adjoint_create_mode(C.byref(params), n, n_steps, self.MODES[mode],
                                             int(checkpoint_every), C.byref(h)))
        self.h, self.n, self.n_steps, self.params, self.mode = h, n, n_steps, params, mode

    def close(self):
        if getattr(self, "h", None):
            lib.nbody_adjoint_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int):
        _check(lib.nbody_adjoint_set_stream(self.h, stream_ptr))

    @staticmethod
    def _rows(t):
        t = t.contiguous()
        return t, [t[k].data_ptr() for k in range(3)]

    def forward(self, x0, v0, mass, perturber_mass_mjup: float, perturber_radius_au: float):
        import torch
        x0, px = self._rows(x0)
        v0, pv = self._rows(v0)
        x = torch.empty_like(x0)
        v = torch.empty_like(v0)
        _check(lib.nbody_adjoint_forward(self.h, *px, *pv, mass.data_ptr(),
                                         float(perturber_mass_mjup), float(perturber_radius_au),
                                         *[x[k].data_ptr() for k in range(3)],
                                         *[v[k].data_ptr() for k in range(3)]))
        return x, v

    def replay(self, x0, v0, perturber_mass_mjup: float, perturber_radius_au: float,
               fp64: bool = False):
        import torch
        x0, px = self._rows(x0)
        v0, pv = self._rows(v0)
        x = torch.empty_like(x0)
        v = torch.empty_like(v0)
        _check(lib.nbody_adjoint_replay(self.h, *px, *pv, float(perturber_mass_mjup),
                                        float(perturber_radius_au), int(fp64),
                                        *[x[k].data_ptr() for k in range(3)],
                                        *[v[k].data_ptr() for k in range(3)]))
        return x, v

    def backward(self, gx, gv):
        import torch
        gx, pgx = self._rows(gx)
        gv, pgv = self._rows(gv)
        gx0 = torch.empty_like(gx)
        gv0 = torch.empty_like(gv)
        gp = (C.c_double * 2)()
        _check(lib.nbody_adjoint_backward(self.h, *pgx, *pgv,
                                          *[gx0[k].data_ptr() for k in range(3)],
                                          *[gv0[k].data_ptr() for k in range(3)], gp))
        return gx0, gv0, gp[0], gp[1]

    def stats(self) -> nbody_adjoint_stats:
        st = nbody_adjoint_stats()
        _check(lib.nbody_adjoint_stats_get(self.h, C.byref(st)))
        return st


def _trajectory_function():
    import torch

    class DiskTrajectory(torch.autograd.Function):
        """(x0, v0, perturber mass M_J, perturber radius AU) -> (x_N, v_N)
        through an Adjoint engine; backward is the engine's reverse mode."""

        @staticmethod
        def forward(ctx, x0, v0, pmass, pradius, engine, mass):
            x, v = engine.forward(x0, v0, mass, float(pmass), float(pradius))
            ctx.engine = engine
            return x, v

        @staticmethod
        def backward(ctx, gx, gv):
            gx0, gv0, gm, gr = ctx.engine.backward(gx.to(torch.float64), gv.to(torch.float64))
            dev = gx0.device
            return (gx0, gv0, torch.tensor(gm, dtype=torch.float64, device=dev),
                    torch.tensor(gr, dtype=torch.float64, device=dev), None, None)

    return DiskTrajectory


def disk_trajectory(engine: "Adjoint", x0, v0, pmass, pradius, mass):
    """Autograd entry: differentiable final state of ``engine``'s trajectory."""
    return _trajectory_function().apply(x0, v0, pmass, pradius, engine, mass)


def eccentricity2(x, v, star_mass: float = 1.0):
    """Per-body e^2 (torch, FP64): e = ((|v|^2 - mu/r) x - (x . v) v) / mu."""
    import torch
    r = torch.sqrt((x * x).sum(0))
    v2 = (v * v).sum(0)
    xv = (x * v).sum(0)
    mu = float(star_mass)
    e = ((v2 - mu / r) * x - xv * v) / mu
    return (e * e).sum(0)


def eccentricity_loss(x, v, mass, star_mass: float = 1.0, r_max: float = 2.0):
    """Mass-weighted mean e^2 over bodies with final r < r_max (torch, FP64):
    e = ((|v|^2 - mu/r) x - (x . v) v) / mu with mu = star_mass (G = 1)."""
    import torch
    r = torch.sqrt((x * x).sum(0))
    v2 = (v * v).sum(0)
    xv = (x * v).sum(0)
    mu = float(star_mass)
    e = ((v2 - mu / r) * x - xv * v) / mu
    e2 = (e * e).sum(0)
    w = mass.to(torch.float64) * (r < r_max).to(torch.float64)
    return (w * e2).sum() / w.sum()


def direct_f64(x, y, z, mass, eps: float, targets=None, want_acc=True, want_phi=False):
    """FP64 direct-sum self-gravity (nbody_direct_f64) on CUDA tensors.

    x, y, z: float64 CUDA tensors; mass: float32; targets: int32 CUDA tensor
    or None (every body).  Returns (ax, ay, az, phi) float64 tensors (None
    where not wanted)."""
    import torch
    n = x.numel()
    nt = n if targets is None else targets.numel()
    mk = lambda on: torch.empty(nt, dtype=torch.float64, device=x.device) if on else None
    ax, ay, az, phi = mk(want_acc), mk(want_acc), mk(want_acc), mk(want_phi)
    p = lambda t: None if t is None else t.data_ptr()
    _check(lib.nbody_direct_f64(p(x), p(y), p(z), p(mass), n, p(targets), nt, eps,
                                p(ax), p(ay), p(az), p(phi)))
    return ax, ay, az, phi


def radix_sort(keys, values, bits: int):
    """Stable radix sort of (key, value) pairs in place (nbody_radix_sort_u32 /
    _u64) on CUDA tensors: keys int32 or int64 (read as unsigned), values
    int32."""
    import torch
    n = keys.numel()
    if values.numel() != n or values.dtype != torch.int32:
        raise ValueError("radix_sort: values must be int32 and as long as keys")
    fn = {torch.int32: lib.nbody_radix_sort_u32, torch.int64: lib.nbody_radix_sort_u64}.get(keys.dtype)
    if fn is None:
        raise ValueError("radix_sort: keys must be int32 or int64")
    _check(fn(keys.data_ptr(), values.data_ptr(), n, bits))


# --------------------------------------------------------- initial disks
def make_disk(n: int, r_min: float, r_max: float, sigma_e=0.01, sigma_i=0.005, star_mass=1.0,
              seed: int = 0):
    """Synthetic Keplerian disk (nbody_make_disk): dict of float64 numpy arrays."""
    out = {k: np.zeros(n, np.float64) for k in ("x", "y", "z", "vx", "vy", "vz")}
    _check(lib.nbody_make_disk(n, r_min, r_max, sigma_e, sigma_i, star_mass, seed,
                               *[out[k].ctypes.data_as(_D) for k in ("x", "y", "z", "vx", "vy",
                                                                       "vz")]))
    return out


def make_disks_device(counts, seeds, r_min: float, r_max: float, sigma_e=0.01, sigma_i=0.005,
                      star_mass=1.0, stream_ptr: int = 0):
    """Disks generated on the GPU (nbody_make_disks_device): (x, v) as (3, N)
    float64 CUDA tensors, the disks concatenated in order."""
    import torch
    cnt = np.ascontiguousarray(counts, np.int32)
    sd = np.ascontiguousarray(seeds, np.uint64)
    total = int(cnt.sum())
    x = torch.empty((3, total), dtype=torch.float64, device="cuda")
    v = torch.empty((3, total), dtype=torch.float64, device="cuda")
    _check(lib.nbody_make_disks_device(cnt.ctypes.data, sd.ctypes.data, len(cnt), r_min, r_max,
                                       sigma_e, sigma_i, star_mass,
                                       *[x[k].data_ptr() for k in range(3)],
                                       *[v[k].data_ptr() for k in range(3)], stream_ptr))
    return x, v
