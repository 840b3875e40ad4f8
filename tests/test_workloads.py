"""Host logic of the ensemble workload: disk specs, the partition of disks
over ranks, and the two-rank gather of per-disk results (gloo, CPU)."""
from __future__ import annotations

import importlib
import os
import socket

import numpy as np
import pytest

wl = importlib.import_module("nbody-sim_b200.workloads")


def test_c4_disks_reproducible_and_in_range():
    a = wl.c4_disks()
    b = wl.c4_disks()
    assert a == b and len(a) == 64
    ns = np.array([d["n"] for d in a])
    assert ns.min() >= 2048 and ns.max() <= 65536
    assert [d["seed"] for d in a] == list(range(64))
    for d in a:
        assert 0.3 <= d["perturber_mass_mjup"] <= 10.0
        assert 5.0 <= d["perturber_radius_au"] <= 30.0
    # log-uniform sizes: E[N] = (65536 - 2048) / ln 32 ~ 18318; 64 draws
    assert 0.6e6 < ns.sum() < 1.8e6


@pytest.mark.parametrize("ranks", [1, 2, 3, 8])
def test_partition_covers_every_disk_once_and_balances(ranks):
    sizes = [d["n"] for d in wl.c4_disks()]
    parts = wl.partition_disks(sizes, ranks)
    flat = sorted(k for p in parts for k in p)
    assert flat == list(range(len(sizes)))
    work = [sum(sizes[k] * np.log(sizes[k]) for k in p) for p in parts]
    biggest = max(n * np.log(n) for n in sizes)
    # greedy largest-first: no rank exceeds the mean by more than one disk
    assert max(work) - np.mean(work) <= biggest + 1e-6


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


# a small ensemble of the C4 recipe for the CPU: 12 disks of 256..2048 bodies
SMALL = dict(n_disks=12, n_range=(256, 2048))


def disk_result(port, spec, steps=2):
    """One disk of the ensemble advanced on the CPU restatement of the
    reference step (collisions, drag and its perturber), as the SHA-256 of its
    final FP32 state: the per-disk record a rank sends back."""
    import hashlib
    d = port.make_disk(spec["n"], wl.DISK_R[0], wl.DISK_R[1], 0.01, 0.005, 1.0, spec["seed"])
    st = {k: v.astype(np.float32) for k, v in d.items()}
    st["m"] = np.full(spec["n"], wl.PARTICLE_MASS, np.float32)
    pert = port.perturber(True, spec["perturber_mass_mjup"], spec["perturber_radius_au"],
                          spec["perturber_phase0"], 1.0)
    r_coll = 5.0 * 2.416e-5 * (wl.PARTICLE_MASS / 3.003e-7) ** (1.0 / 3.0)
    sp = port.step_params(0.005, 0.5, wl.SOFTENING, 1.0, r_coll=r_coll, restitution=0.0,
                          gas_drag_rate=1e-3, collisions=True, pert=pert)
    port.run(st, sp, steps, nthreads=1)
    h = hashlib.sha256()
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        h.update(np.ascontiguousarray(st[k]).tobytes())
    return h.hexdigest()


def _rank_main(rank, world, port, q):
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(
        __file__))), "oracle"))
    import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        specs = wl.c4_disks(**SMALL)
        mine = wl.partition_disks([d["n"] for d in specs], world)[rank]
        orc = oracle.Port()
        rows = [(k, specs[k]["n"], disk_result(orc, specs[k])) for k in mine]
        got = [None] * world
        dist.all_gather_object(got, rows)
        if rank == 0:
            q.put(got)
    finally:
        dist.destroy_process_group()


def test_two_rank_partition_gathers_every_disk_result(port):
    """Two gloo ranks each advance their share of the disks (partition by
    N log N) and gather the per-disk results: every disk comes back once,
    from the rank the partition gave it to, with the result a single process
    computes for it."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    pnum = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, pnum, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    specs = wl.c4_disks(**SMALL)
    parts = wl.partition_disks([d["n"] for d in specs], 2)
    assert [sorted(r[0] for r in got[k]) for k in range(2)] == parts
    rows = sorted(r for part in got for r in part)
    assert [r[0] for r in rows] == list(range(len(specs)))
    for k, n, digest in rows:
        assert n == specs[k]["n"]
        assert digest == disk_result(port, specs[k]), k
