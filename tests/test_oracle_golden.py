"""The CPU oracle (oracle/port.c) pinned to the reference (CPU suite).

* FoF: the restated union-find against golden vectors made by the reference's
  own detectAggregates (tests/golden/fof_*.npz, tests/golden/make_golden.py).
* Engine: the restated build/walk against golden vectors made by the
  reference's own CUDA engine compiled with -fmad=false
  (tests/golden/ref_engine_*.npz) -- bit-for-bit.
* The known-answer tests of the reference's tests/*.cu|cpp, on the oracle.
"""
from __future__ import annotations

import glob
import math
import os

import numpy as np
import pytest

from conftest import golden


def _npz(name):
    path = golden(name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not generated")
    return np.load(path)


@pytest.mark.parametrize("name", ["fof_a.npz", "fof_b.npz", "fof_c.npz"])
def test_oracle_fof_matches_reference_golden(port, name):
    g = _npz(name)
    labels, size, ng = port.fof(g["x"], g["y"], g["z"], float(g["link_length"]))
    assert ng == int(g["n_groups"])
    np.testing.assert_array_equal(labels, g["labels"])
    np.testing.assert_array_equal(size, g["agg_size"])
    ag = port.aggregates(g["x"], g["y"], g["z"], g["vx"], g["vy"], g["vz"], labels,
                         float(g["particle_mass"]), ng)
    for k in ("n", "mass", "c", "v", "dist", "label"):
        np.testing.assert_array_equal(ag[k], g["g_" + k], err_msg=k)


@pytest.mark.parametrize("path", sorted(glob.glob(golden("ref_engine_*.npz"))) or ["missing"])
def test_oracle_walk_matches_reference_engine_golden(port, path):
    if path == "missing":
        pytest.skip("reference-engine fixtures not generated (make_golden.py --gpu)")
    g = np.load(path)
    ax, ay, az, info = port.forces(g["x"], g["y"], g["z"], g["m"], 0.5, 1e-3, 1.0)
    assert info.lost_bodies == 0
    np.testing.assert_array_equal(info.sort_idx, g["sort_idx"])
    np.testing.assert_array_equal(ax, g["ax"])
    np.testing.assert_array_equal(ay, g["ay"])
    np.testing.assert_array_equal(az, g["az"])


@pytest.mark.parametrize("path", sorted(glob.glob(golden("ref_engine_*.npz"))) or ["missing"])
def test_oracle_step_loop_matches_reference_engine_golden(port, path):
    if path == "missing":
        pytest.skip("reference-engine fixtures not generated (make_golden.py --gpu)")
    g = np.load(path)
    st = {k: g[k].copy() for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
    pert = port.perturber(True, 1.0, 5.2, 0.0, 1.0)
    sp = port.step_params(0.01, 0.5, 1e-3, 1.0, r_coll=float(g["r_coll"]), restitution=0.0,
                          gas_drag_rate=1e-2, collisions=True, pert=pert)
    port.run(st, sp, 3)
    for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az"):
        np.testing.assert_array_equal(st[k], g["s3_" + k], err_msg=k)


# ------------------------------------------- reference known-answer tests
def test_kat_star_force(port):
    # tests/test_bhtree.cu:104-134
    ax, ay, az, _ = port.forces([1.0], [0.0], [0.0], [1e-6], 0.5, 0.001, 1.0)
    assert abs(ax[0] + 1.0) <= 0.05
    assert abs(ay[0]) <= 0.05 and abs(az[0]) <= 0.05


def test_kat_sort_idx_permutation(port):
    # tests/test_bhtree.cu:29-99
    n = 1000
    i = np.arange(n)
    r = 0.5 + 4.5 * i / (n - 1)
    phi = 2 * np.pi * i / n
    t = port.build_tree(r * np.cos(phi), 0.01 * (i % 10 - 5), r * np.sin(phi), np.full(n, 3.003e-7))
    info = port.tree_info(t)
    port.free_tree(t)
    assert sorted(info.sort_idx.tolist()) == list(range(n))


def test_kat_collision_head_on(port):
    # tests/test_collision.cu:7-48
    vx, vy, vz = port.collision([-0.001, 0.001], [0, 0], [0, 0], [3.003e-7] * 2, [0.1, -0.1],
                                [0, 0], [0, 0], 0.005, 0.3)
    assert vx[0] < 0 < vx[1]
    assert abs(vx[0] + vx[1]) < 1e-5


def test_kat_perturber(port):
    # tests/test_perturber.cu:17-116
    p = port.perturber(True, 1.0, 10.0, 0.0, 1.0)
    assert abs(p.x - 10.0) < 1e-5 and abs(p.z) < 1e-5
    assert abs(p.mass_msun - 9.5479e-4) <= 1e-4 * 9.5479e-4
    assert abs(p.omega - math.sqrt(1.0 / 1000.0)) <= 1e-5 * math.sqrt(1.0 / 1000.0)
    T = np.float32(2.0) * np.float32(3.14159265358979) / np.float32(p.omega)
    q = port.perturber_at(p, float(T * np.float32(0.25)))
    assert abs(q.x) < 1e-2 and abs(q.z - 10.0) < 1e-2
    a = port.perturber_force([np.float32([1e-3]), np.zeros(1), np.zeros(1)],
                             [np.zeros(1)] * 3, port.perturber_at(
                                 port.perturber(True, 1e-3 / 9.5479e-4, 10.0, 0.0, 1.0), 0.0),
                             0.01)
    r2 = 100.0 + 1e-4
    expect = 1e-3 + 1e-3 / (r2 * math.sqrt(r2)) * 10.0
    assert abs(a[0][0] - expect) <= 1e-4 * expect


def test_kat_leapfrog_energy_one_orbit(port):
    # tests/test_integrator.cu:10-59: KDK with the star pull, one period
    x = [np.float32([1.0]), np.float32([0.0]), np.float32([0.0])]
    v = [np.float32([0.0]), np.float32([0.0]), np.float32([1.0])]
    dt, soft = np.float32(0.01), np.float32(0.001)

    def acc(x):
        r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2] + soft * soft
        r3 = r2 * np.sqrt(r2)
        return [-xx / r3 for xx in x]

    a = acc(x)
    for _ in range(int(np.float32(6.28318530) / dt)):
        v = port.half_kick(v, a, float(dt * np.float32(0.5)))
        x = port.drift(x, v, float(dt))
        a = acc(x)
        v = port.half_kick(v, a, float(dt * np.float32(0.5)))
    r = math.sqrt(sum(float(q[0]) ** 2 for q in x))
    e = 0.5 * sum(float(q[0]) ** 2 for q in v) - 1.0 / r
    assert abs(e - (-0.5)) <= 0.01 * 0.5


def test_kat_fof_cases(port):
    # tests/test_aggregate.cpp:20-119
    x = [0, 1e-4, 0, 1e-4, 0, 3.0, -4.0]; y = [0, 0, 1e-4, 1e-4, 0, 0, 0]; z = [0, 0, 0, 0, 1e-4, 0, 0]
    lab, size, g = port.fof(x, y, z, 0.002)
    assert g == 1 and sorted(size.tolist()) == [1, 1, 5, 5, 5, 5, 5]
    assert port.fof([0, 10, 20], [0] * 3, [0] * 3, 0.01)[2] == 0
    x = [0, 0.001, 0, 10, 10.001, 10]; y = [0, 0, 0.001, 0, 0, 0.001]
    lab, size, g = port.fof(x, y, [0] * 6, 0.01)
    assert g == 2 and (size == 3).all()
    lab, size, g = port.fof([1.0, 3.0], [0, 0], [0, 0], 5.0)
    ag = port.aggregates([1.0, 3.0], [0, 0], [0, 0], [0.5, 1.5], [0, 0], [0, 0], lab, 3.003e-7, g)
    assert abs(ag["c"][0] - 2.0) < 1e-5 and abs(ag["v"][0] - 1.0) < 1e-5
    assert abs(ag["dist"][0] - 2.0) < 1e-5
    assert abs(ag["mass"][0] - 2 * 3.003e-7) <= 1e-4 * 2 * 3.003e-7


def test_oracle_fof_vs_reference_host_live(port, refhost):
    """The restated FoF against the reference's Aggregate.cpp, fresh inputs."""
    rng = np.random.default_rng(99)
    n = 1500
    p = (rng.random((n, 3)) * 0.05).astype(np.float32)
    v = rng.standard_normal((n, 3)).astype(np.float32)
    l1, s1, g1 = port.fof(p[:, 0], p[:, 1], p[:, 2], 0.0015)
    l2, s2, g2, _ = refhost.detect_aggregates(*p.T, *v.T, 0.0015, 1e-8)
    assert g1 == g2
    np.testing.assert_array_equal(l1, l2)
    np.testing.assert_array_equal(s1, s2)


def test_oracle_direct_sum_symmetry(port):
    """FP64 direct sum: momentum of the pair forces cancels (sum m a = 0)."""
    rng = np.random.default_rng(1)
    n = 400
    p = rng.random((n, 3))
    m = rng.random(n) * 1e-6
    ax, ay, az = port.direct_f64(p[:, 0], p[:, 1], p[:, 2], m, np.arange(n), 1e-3, 1.0, False)
    tot = np.array([np.dot(m, ax), np.dot(m, ay), np.dot(m, az)])
    assert np.abs(tot).max() < 1e-12 * np.abs(m).sum() ** 2 / 1e-6 + 1e-18


def test_oracle_collision_pairs_against_brute_force(port):
    """orc_collision_pairs (the reference's collision traversal, counted): it
    never reports more pairs than exist, finds them all on a uniform cloud,
    and skips some on clustered data, where a cell's centre of mass can lie
    away from a body that touches one of its members (BHTree.cu:663-665)."""
    def brute(x, y, z, r):
        n = len(x)
        total = 0
        for i0 in range(0, n, 500):
            i1 = min(n, i0 + 500)
            dx = x[None, :] - x[i0:i1, None]
            dy = y[None, :] - y[i0:i1, None]
            dz = z[None, :] - z[i0:i1, None]
            close = (dx * dx + dy * dy + dz * dz) < r * r
            close[np.arange(i1 - i0), np.arange(i0, i1)] = False
            total += int(close.sum())
        return total

    rng = np.random.default_rng(3)
    n, r = 2000, np.float32(0.01)
    pos = rng.random((n, 3)).astype(np.float32) * np.float32(0.2)
    x, y, z = [np.ascontiguousarray(pos[:, k]) for k in range(3)]
    m = np.full(n, 1e-9, np.float32)
    b = brute(x, y, z, r)
    assert b > 100
    assert port.collision_pairs(x, y, z, m, r) == b
    centers = rng.random((40, 3)) * 0.05
    pos = (centers[rng.integers(0, 40, 4000)] + rng.standard_normal((4000, 3)) * 0.002)
    pos = pos.astype(np.float32)
    x, y, z = [np.ascontiguousarray(pos[:, k]) for k in range(3)]
    m = np.full(4000, 1e-9, np.float32)
    b = brute(x, y, z, np.float32(0.002))
    found = port.collision_pairs(x, y, z, m, np.float32(0.002))
    assert 0 < b - found < b // 100
