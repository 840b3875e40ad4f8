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


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        specs = wl.c4_disks()
        mine = wl.partition_disks([d["n"] for d in specs], world)[rank]
        # per-disk result stand-in: the disk's size and seed
        rows = [(k, specs[k]["n"], specs[k]["seed"]) for k in mine]
        got = [None] * world
        dist.all_gather_object(got, rows)
        if rank == 0:
            q.put(got)
    finally:
        dist.destroy_process_group()


def test_two_rank_partition_gathers_every_disk():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    rows = sorted(r for part in got for r in part)
    specs = wl.c4_disks()
    assert [r[0] for r in rows] == list(range(64))
    assert all(r[1] == specs[r[0]]["n"] for r in rows)
