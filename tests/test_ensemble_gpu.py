"""Batched ensemble (nbody_ensemble_*) against separate nbody_sim runs.

Every disk of an ensemble is an independent simulation: its own octree, star,
perturber and collisions.  The ensemble's per-disk trees have the same cells
and moments as a separate run's tree; only the binary split of bodies that
share a 30-bit Morton key (and therefore, rarely, a warp group's box) can
differ, which changes which nodes a group opens.  The bar is therefore the
walk's approximation level: accelerations agree to 1e-5 relative, and after
a few steps positions agree to 1e-7 AU and velocities to 1e-6 AU/yr-unit.
Graph replay against plain launches, and the autotuner's round trip, are
deterministic and compared bit for bit.
"""
from __future__ import annotations

import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

wl = importlib.import_module("nbody-sim_b200.workloads")

SPECS = [
    {"n": 2048, "seed": 0, "perturber_enabled": 1, "perturber_mass_mjup": 3.0,
     "perturber_radius_au": 6.0, "perturber_phase0": 0.3},
    {"n": 5003, "seed": 1, "perturber_enabled": 0},
    {"n": 9000, "seed": 2, "perturber_enabled": 1, "perturber_mass_mjup": 0.5,
     "perturber_radius_au": 12.0, "perturber_phase0": 2.0},
    {"n": 3333, "seed": 3, "perturber_enabled": 1, "perturber_mass_mjup": 9.0,
     "perturber_radius_au": 5.0, "perturber_phase0": 4.0},
]


def params(nb, precision):
    return wl.c4_params(nb, precision)


def separate(nb, prm, spec, steps):
    d, m = wl.disk_state(nb, spec)
    p = nb.sim_params(**{f: getattr(prm, f) for f, _ in prm._fields_})
    p.perturber_enabled = spec.get("perturber_enabled", 0)
    p.perturber_mass_mjup = spec.get("perturber_mass_mjup", 1.0)
    p.perturber_radius_au = spec.get("perturber_radius_au", 5.2)
    p.perturber_phase0 = spec.get("perturber_phase0", 0.0)
    sim = nb.Sim(p, spec["n"])
    dbl = prm.state_precision == nb.NBODY_STATE_F64
    st = {k: (v if dbl else v.astype(np.float32)) for k, v in d.items()}
    sim.set_state(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], m)
    out0 = sim.get_state(double=False, accel=True)
    sim.step(steps)
    sim.sync()
    out = sim.get_state(double=dbl, accel=False)
    sim.close()
    return out0, out


def ensemble(nb, prm, specs, steps, graphs=True, tune=False):
    st, m = wl.ensemble_state(nb, specs)
    e = nb.Ensemble(prm, specs)
    e.set_graphs(graphs)
    dbl = prm.state_precision == nb.NBODY_STATE_F64
    if not dbl:
        st = {k: v.astype(np.float32) for k, v in st.items()}
    e.set_state(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], m)
    tuned = e.autotune() if tune else None
    out0 = e.get_state(double=False, accel=True)
    e.step(steps)
    e.sync()
    out = e.get_state(double=dbl, accel=False)
    stats = e.stats()
    e.close()
    return out0, out, stats, tuned


def rel_acc_err(a, b):
    na = np.sqrt(a["ax"].astype(np.float64) ** 2 + a["ay"] ** 2 + a["az"] ** 2)
    d = np.sqrt((a["ax"].astype(np.float64) - b["ax"]) ** 2 + (a["ay"].astype(np.float64) - b["ay"]) ** 2
                + (a["az"].astype(np.float64) - b["az"]) ** 2)
    return d / na


@pytest.mark.parametrize("precision", [1, 0], ids=["f64", "f32"])
def test_ensemble_matches_separate_runs(nb, cuda, precision):
    prm = params(nb, precision)
    steps = 6
    e0, e1, stats, _ = ensemble(nb, prm, SPECS, steps)
    assert stats.status == 0
    assert stats.steps_done == steps and stats.n_disks == len(SPECS)
    assert stats.graph_launches == steps
    off = 0
    for spec in SPECS:
        s0, s1 = separate(nb, prm, spec, steps)
        sl = slice(off, off + spec["n"])
        a0 = {k: v[sl] for k, v in e0.items()}
        err = rel_acc_err(s0, a0)
        assert np.max(err) < 1e-5, (spec, np.max(err))
        for k in ("x", "y", "z"):
            assert np.max(np.abs(e1[k][sl] - s1[k])) < 1e-7, (spec, k)
        for k in ("vx", "vy", "vz"):
            assert np.max(np.abs(e1[k][sl] - s1[k])) < 1e-6, (spec, k)
        off += spec["n"]


TINY = [{"n": 2, "seed": 5}, {"n": 3, "seed": 6}, {"n": 2, "seed": 7},
        {"n": 700, "seed": 8}, {"n": 3, "seed": 9}]


def test_ensemble_with_disks_of_two_or_three_bodies(nb, cuda):
    """The smallest disks an ensemble takes (two bodies each at least): their
    roots sit right under binary nodes that span several disks and have only
    leaves below them; each disk still matches the same disk run on its own."""
    prm = params(nb, 1)
    steps = 4
    e0, e1, stats, _ = ensemble(nb, prm, TINY, steps)
    assert stats.status == 0
    off = 0
    for spec in TINY:
        s0, s1 = separate(nb, prm, spec, steps)
        sl = slice(off, off + spec["n"])
        a0 = {k: v[sl] for k, v in e0.items()}
        assert np.max(rel_acc_err(s0, a0)) < 1e-5, spec
        for k in ("x", "y", "z"):
            assert np.max(np.abs(e1[k][sl] - s1[k])) < 1e-7, (spec, k)
        off += spec["n"]


def test_ensemble_graphs_equal_plain_launches(nb, cuda):
    prm = params(nb, 1)
    _, g, sg, _ = ensemble(nb, prm, SPECS, 5, graphs=True)
    _, p, sp, _ = ensemble(nb, prm, SPECS, 5, graphs=False)
    assert sg.graph_launches == 5 and sp.graph_launches == 0
    assert sg.launches == sp.launches
    for k in g:
        assert np.array_equal(g[k], p[k]), k


def test_ensemble_two_calls_equal_one(nb, cuda):
    """step(3); step(4) is step(7): the closing kick and perturber rows line up."""
    prm = params(nb, 1)
    st, m = wl.ensemble_state(nb, SPECS)
    res = []
    for split in ((7,), (3, 4)):
        e = nb.Ensemble(prm, SPECS)
        e.set_state(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], m)
        for k in split:
            e.step(k)
        e.sync()
        res.append(e.get_state(double=True, accel=True))
        e.close()
    for k in res[0]:
        assert np.array_equal(res[0][k], res[1][k]), (k, np.max(np.abs(res[0][k] - res[1][k])))


def test_ensemble_autotune_keeps_state(nb, cuda):
    prm = params(nb, 1)
    st, m = wl.ensemble_state(nb, SPECS)
    e = nb.Ensemble(prm, SPECS)
    e.set_state(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], m)
    before = e.get_state(double=True, accel=True)
    tuned = e.autotune()
    after = e.get_state(double=True, accel=True)
    stats = e.stats()
    e.close()
    assert len(tuned) == 6 and all(t[3] > 0 for t in tuned)
    best = min(tuned, key=lambda t: t[3])
    assert (stats.targets_per_lane, stats.leaf_max, stats.walk_mode) == best[:3]
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.array_equal(before[k], after[k]), k
    # the kept setting may group targets and open leaves differently: its
    # forces differ by the walk's approximation error, a few 1e-5 of the total
    # acceleration here (self-gravity is ~1e-3 of the star's pull)
    assert np.max(rel_acc_err(before, after)) < 1e-4


def test_ensemble_rejects_bad_input(nb, cuda):
    prm = params(nb, 1)
    with pytest.raises(nb.NBodyError) as e:
        nb.Ensemble(prm, [{"n": 100}, {"n": 1}])
    assert e.value.code == nb.NBODY_ERR_ARG
    ens = nb.Ensemble(prm, [{"n": 100}, {"n": 200}])
    with pytest.raises(nb.NBodyError) as e:
        ens.step(1)
    assert e.value.code == nb.NBODY_ERR_ARG
    ens.close()


def test_device_disk_generator_matches_host(nb, cuda):
    """nbody_make_disks_device against nbody_make_disk disk by disk: the same
    arithmetic, differing only in the math libraries' last-ulp rounding."""
    counts = [2048, 5003, 1, 0, 9000]
    seeds = [0, 1, 2, 3, 2 ** 40 + 5]
    x, v = nb.make_disks_device(counts, seeds, 0.5, 5.0)
    x, v = x.cpu().numpy(), v.cpu().numpy()
    off = 0
    for n, s in zip(counts, seeds):
        d = nb.make_disk(n, 0.5, 5.0, 0.01, 0.005, 1.0, s)
        for k, key in enumerate(("x", "y", "z")):
            assert np.allclose(x[k, off:off + n], d[key], rtol=1e-12, atol=1e-13), (s, key)
        for k, key in enumerate(("vx", "vy", "vz")):
            assert np.allclose(v[k, off:off + n], d[key], rtol=1e-12, atol=1e-13), (s, key)
        off += n
    assert off == x.shape[1]


def test_ensemble_fused_collisions_match_the_separate_pass(nb, cuda):
    """The ensemble's collisions found inside its force walk (fuse_collisions)
    against its neighbour pass beside the walk: the same pairs per disk, so
    the states after a few steps agree to the rounding of the impulse sums."""
    specs = [dict(s) for s in SPECS]
    out = []
    for fuse in (0, 1):
        prm = params(nb, 1)
        prm.fuse_collisions = fuse
        prm.r_coll = 1e-2  # many touching pairs in these disks
        prm.walk_mode = 1  # the vote walk (the autotuner is not run)
        st, m = wl.ensemble_state(nb, specs)
        e = nb.Ensemble(prm, specs)
        e.set_state(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], m)
        e.step(3)
        e.sync()
        out.append(e.get_state(double=True, accel=False))
        assert e.stats().status == 0
        e.close()
    for k in ("vx", "vy", "vz"):
        assert np.abs(out[0][k] - out[1][k]).max() < 1e-5, k
    for k in ("x", "y", "z"):
        assert np.abs(out[0][k] - out[1][k]).max() < 1e-7, k


def test_ensemble_step_host_read_back_equals_get_state(nb, cuda):
    """nbody_ensemble_step_host reads the positions back on a second stream
    while the steps finish; what it returns must be the final state, as
    get_state reads it afterwards, bit for bit, over two calls in a row."""
    prm = params(nb, 1)
    st, m = wl.ensemble_state(nb, SPECS)
    e = nb.Ensemble(prm, SPECS)
    e.set_state(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], m)
    g = e.get_state(double=False, accel=True)
    host = {k: np.ascontiguousarray(st[k], np.float64) for k in ("x", "y", "z", "vx", "vy", "vz")}
    for k in ("ax", "ay", "az"):
        host[k] = np.ascontiguousarray(g[k], np.float32)
    for nsteps in (1, 3):
        before = host["x"].copy()
        e.step_host(host, m, nsteps)
        got = e.get_state(double=True, accel=False)
        acc = e.get_state(double=False, accel=True)
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            assert np.array_equal(host[k], got[k]), (nsteps, k)
        for k in ("ax", "ay", "az"):
            assert np.array_equal(host[k], acc[k]), (nsteps, k)
        assert not np.array_equal(host["x"], before)
    assert e.stats().status == 0
    e.close()
