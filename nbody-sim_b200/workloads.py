"""Synthetic workloads: disk sizes, perturbers and initial states of the
benchmark configurations.

The reference generates one disk per run with src/disk/DiskInit.cpp:18-69 and
a fixed seed (src/main.cu:46).  These workloads use the package's Keplerian
disk generator (``make_disk``, counter-based RNG keyed by seed) so every disk
of an ensemble is reproducible on its own.

Configurations:

* C1: N=4096, m=1e-8, r in [0.5, 5], eps=1e-3, theta=0.5, collisions
  (factor 1), dt=0.01.
* C2: N=131072, m=1e-8, r in [0.5, 5], collisions (factor 5), drag 1e-3,
  perturber 1 M_J at 5.2 AU, dt=0.005, FP64 state.
* C3: N=1,048,576, m=1e-9, r in [0.3, 30], eps=5e-4, dt=0.002, gravity only.
* C4: 64 disks with N log-uniform in [2048, 65536], perturber mass
  log-uniform in [0.3, 10] M_J at a radius uniform in [5, 30] AU, collisions
  (factor 5), drag 1e-3, theta=0.5, dt=0.005, FP64 state.
"""
from __future__ import annotations

import numpy as np

C4_DISKS = 64
C4_N_RANGE = (2048, 65536)
C4_MASS_MJ = (0.3, 10.0)
C4_RADIUS_AU = (5.0, 30.0)
DISK_R = (0.5, 5.0)
PARTICLE_MASS = 1e-8
SOFTENING = 1e-3


def c4_disks(n_disks: int = C4_DISKS, seed: int = 0, n_range=C4_N_RANGE):
    """Disk specs of the ensemble workload: list of dicts (n, seed, perturber_*).

    Disk k uses initial-condition seed k; sizes and perturbers are drawn from
    one numpy Generator seeded with ``seed``."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(n_range[0]), np.log(n_range[1])
    out = []
    for k in range(n_disks):
        n = int(round(np.exp(rng.uniform(lo, hi))))
        mass = float(np.exp(rng.uniform(np.log(C4_MASS_MJ[0]), np.log(C4_MASS_MJ[1]))))
        radius = float(rng.uniform(*C4_RADIUS_AU))
        phase = float(rng.uniform(0.0, 2.0 * np.pi))
        out.append({"n": n, "seed": k, "perturber_enabled": 1, "perturber_mass_mjup": mass,
                    "perturber_radius_au": radius, "perturber_phase0": phase})
    return out


def c4_params(nb, precision=None):
    """nbody_sim_params of the ensemble workload (shared by every disk)."""
    return nb.sim_params(dt=0.005, theta=0.5, softening=SOFTENING, star_mass=1.0,
                         r_coll=5.0 * nb.particle_physical_radius(PARTICLE_MASS),
                         restitution=0.0, gas_drag_rate=1e-3,
                         state_precision=nb.NBODY_STATE_F64 if precision is None else precision)


def disk_state(nb, spec, r=DISK_R, m=PARTICLE_MASS):
    """One disk's float64 initial state (dict x..vz) and float32 masses."""
    d = nb.make_disk(spec["n"], r[0], r[1], 0.01, 0.005, 1.0, spec["seed"])
    return d, np.full(spec["n"], m, np.float32)


def ensemble_state(nb, specs, r=DISK_R, m=PARTICLE_MASS):
    """Every disk's initial state concatenated in disk order."""
    parts = [disk_state(nb, s, r, m) for s in specs]
    keys = ("x", "y", "z", "vx", "vy", "vz")
    st = {k: np.concatenate([p[0][k] for p in parts]) for k in keys}
    return st, np.concatenate([p[1] for p in parts])


def partition_disks(sizes, n_ranks: int):
    """Greedy balance of sum(N log N) over ranks: list of disk indices per rank.

    Disks go largest first to the rank with the least work so far; each rank
    gets its disks in ascending index order."""
    work = [(n * np.log(max(n, 2)), k) for k, n in enumerate(sizes)]
    work.sort(key=lambda t: (-t[0], t[1]))
    load = [0.0] * n_ranks
    parts = [[] for _ in range(n_ranks)]
    for w, k in work:
        r = min(range(n_ranks), key=lambda i: (load[i], i))
        load[r] += w
        parts[r].append(k)
    return [sorted(p) for p in parts]
