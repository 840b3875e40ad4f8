"""The engine's CUDA-graph steps against the same steps launched kernel by
kernel: bit for bit, in every precision, with collisions, drag and the
perturber (whose table row the graph advances on the device), across calls
of different lengths."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import disk

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1, 2], ids=["f32", "f64", "f32x2"])
def test_graph_steps_equal_plain_launches(nb, cuda, precision):
    n = 6000
    st = disk(nb, n, 0.5, 5.0, seed=9, m=1e-8)
    prm = nb.sim_params(dt=0.005, theta=0.5, softening=1e-3, star_mass=1.0,
                        r_coll=5.0 * nb.particle_physical_radius(1e-8), restitution=0.0,
                        gas_drag_rate=1e-3, perturber_enabled=1, perturber_mass_mjup=3.0,
                        perturber_radius_au=6.0, perturber_phase0=0.5,
                        state_precision=precision)
    out = []
    for graphs in (True, False):
        sim = nb.Sim(prm, n)
        sim.set_graphs(graphs)
        sim.set_state(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], st["m"])
        for k in (3, 1, 5):
            sim.step(k)
        sim.sync()
        stats = sim.stats()
        out.append((sim.get_state(double=True, accel=False), stats))
        sim.close()
    (g, sg), (p, sp) = out
    assert sg.graph_launches == 9 and sp.graph_launches == 0
    assert sg.launches == sp.launches
    for k in g:
        assert np.array_equal(g[k], p[k]), k


def test_walk_modes_agree(nb, cuda):
    """The three walk variants: modes 0 and 1 differ only in register budget
    (bit-identical forces); mode 2 skips the acceptance vote, so it opens more
    nodes and agrees to the walk's approximation level."""
    n = 20000
    st = disk(nb, n, 0.3, 30.0, seed=3, m=1e-9)
    acc = {}
    for mode in (0, 1, 2):
        prm = nb.sim_params(dt=0.002, theta=0.5, softening=5e-4, star_mass=0.0, r_coll=0.0,
                            gas_drag_rate=0.0, walk_mode=mode)
        sim = nb.Sim(prm, n)
        sim.set_state(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], st["m"])
        g = sim.get_state(accel=True)
        acc[mode] = np.stack([g["ax"], g["ay"], g["az"]], 1).astype(np.float64)
        inter = sim.stats().interactions
        acc[f"i{mode}"] = inter
        sim.close()
    assert np.array_equal(acc[0], acc[1])
    assert acc["i0"] == acc["i1"] and acc["i2"] > acc["i0"]
    rel = np.linalg.norm(acc[0] - acc[2], axis=1) / np.linalg.norm(acc[2], axis=1)
    assert np.median(rel) < 5e-2


def test_group_span_keeps_the_error_and_fills_the_warps(nb, cuda):
    """Target groups cut from larger nodes (group_span 8) against the maximal
    nodes of <= 32 bodies (group_span 1): fewer, fuller groups; the walk's
    self-gravity error against the FP64 direct sum stays at the same level
    (a larger group box only makes the acceptance test stricter)."""
    import torch
    n = 30000
    st = disk(nb, n, 0.3, 30.0, seed=4, m=1e-9)
    tg = np.sort(np.random.default_rng(1).choice(n, 512, replace=False))
    x64 = [torch.from_numpy(st[k].astype(np.float32).astype(np.float64)).cuda()
           for k in ("x", "y", "z")]
    m32 = torch.from_numpy(np.asarray(st["m"], np.float32)).cuda()
    dx, dy, dz, _ = nb.direct_f64(*x64, m32, 5e-4, targets=torch.from_numpy(tg.astype(np.int32)).cuda())
    ref = np.stack([dx.cpu().numpy(), dy.cpu().numpy(), dz.cpu().numpy()], 1)
    res = {}
    for span in (1, 8):
        prm = nb.sim_params(dt=0.002, theta=0.5, softening=5e-4, star_mass=0.0, r_coll=0.0,
                            gas_drag_rate=0.0, group_span=span)
        sim = nb.Sim(prm, n)
        sim.set_state(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], st["m"])
        g = sim.get_state(accel=True)
        a = np.stack([g["ax"][tg], g["ay"][tg], g["az"][tg]], 1).astype(np.float64)
        s = sim.stats()
        sim.close()
        assert s.status == 0
        err = np.linalg.norm(a - ref, axis=1) / np.linalg.norm(ref, axis=1)
        res[span] = (np.median(err), s.walk_groups)
    assert res[8][1] < 0.9 * res[1][1], res
    assert n / res[8][1] <= 32
    assert res[8][0] < 1.05 * res[1][0], res


@pytest.mark.parametrize("graphs", [True, False], ids=["graphs", "plain"])
def test_step_host_read_back_equals_get_state(nb, cuda, graphs):
    """nbody_sim_step_host reads the positions back on a second stream while
    the step finishes; what it returns must be the engine's final state, as
    get_state reads it afterwards, bit for bit, over two calls in a row (a
    read-back that did not wait for the step would return old positions)."""
    n = 7000
    st = disk(nb, n, 0.5, 5.0, seed=11, m=1e-8)
    prm = nb.sim_params(dt=0.005, theta=0.5, softening=1e-3, star_mass=1.0,
                        r_coll=5.0 * nb.particle_physical_radius(1e-8), restitution=0.0,
                        gas_drag_rate=1e-3, perturber_enabled=1, perturber_mass_mjup=1.0,
                        perturber_radius_au=5.2)
    keys = ("x", "y", "z", "vx", "vy", "vz")
    host = {k: np.ascontiguousarray(st[k], np.float32) for k in keys}
    m = np.ascontiguousarray(st["m"], np.float32)
    sim = nb.Sim(prm, n)
    sim.set_graphs(graphs)
    sim.set_state(*[host[k] for k in keys], m)
    g = sim.get_state(accel=True)
    for k in ("ax", "ay", "az"):
        host[k] = g[k].copy()
    for nsteps in (1, 3):
        before = {k: v.copy() for k, v in host.items()}
        sim.step_host(host, m, nsteps)
        got = sim.get_state(accel=True)
        for k in got:
            assert np.array_equal(host[k], got[k]), (nsteps, k)
        assert not np.array_equal(host["x"], before["x"])
    assert sim.stats().status == 0
    sim.close()


@pytest.mark.parametrize("precision", [0, 1, 2], ids=["f32", "f64", "f32x2"])
def test_fused_collisions_match_the_separate_pass(nb, cuda, precision):
    """Collisions found inside the force walk (fuse_collisions = 1) against
    the stand-alone neighbour search on a crowded disk where many pairs touch: the same pairs, so the velocities after the step agree to
    the rounding of the impulse sums and of the few extra nodes the fused
    walk opens near each group."""
    n = 12000
    st = disk(nb, n, 0.5, 1.0, seed=21, m=1e-8)
    out = {}
    for sep in (0, 1):
        prm = nb.sim_params(dt=0.005, theta=0.5, softening=1e-3, star_mass=1.0, r_coll=2e-3,
                            restitution=0.2, gas_drag_rate=1e-3, state_precision=precision,
                            fuse_collisions=1 - sep)
        sim = nb.Sim(prm, n)
        sim.set_state(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], st["m"])
        sim.step(2)
        sim.sync()
        out[sep] = sim.get_state(double=True, accel=False)
        assert sim.stats().status == 0
        sim.close()
    # positions after two steps carry the first step's impulses
    for k in ("vx", "vy", "vz"):
        d = np.abs(out[0][k] - out[1][k])
        assert d.max() < 1e-5, (k, d.max())
    for k in ("x", "y", "z"):
        assert np.abs(out[0][k] - out[1][k]).max() < 1e-7, k
    # the case exercises real collisions: the impulses are far above the tolerance
    ref = nb.sim_params(dt=0.005, theta=0.5, softening=1e-3, star_mass=1.0, r_coll=0.0,
                        restitution=0.2, gas_drag_rate=1e-3, state_precision=precision)
    sim = nb.Sim(ref, n)
    sim.set_state(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], st["m"])
    sim.step(2)
    sim.sync()
    free = sim.get_state(double=True, accel=False)
    sim.close()
    assert np.abs(free["vx"] - out[1]["vx"]).max() > 1e-3


def test_sim_autotune_keeps_the_state_and_the_fastest_setting(nb, cuda):
    """nbody_sim_autotune mid-run: positions and velocities untouched, the
    kept setting is the fastest candidate, the recomputed forces agree with
    the step's own to the walk's approximation level, and stepping goes on."""
    n = 20000
    st = disk(nb, n, 0.5, 5.0, seed=5, m=1e-8)
    prm = nb.sim_params(dt=0.005, theta=0.5, softening=1e-3, star_mass=1.0,
                        r_coll=5.0 * nb.particle_physical_radius(1e-8), gas_drag_rate=1e-3,
                        perturber_enabled=1, perturber_mass_mjup=1.0, perturber_radius_au=5.2,
                        state_precision=1)
    sim = nb.Sim(prm, n)
    sim.set_state(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], st["m"])
    sim.step(3)
    before = sim.get_state(double=True, accel=False)
    acc0 = sim.get_state(double=False, accel=True)
    tuned = sim.autotune()
    after = sim.get_state(double=True, accel=False)
    acc1 = sim.get_state(double=False, accel=True)
    s = sim.stats()
    assert len(tuned) == 6 and all(t[4] > 0 for t in tuned)
    best = min(tuned, key=lambda t: t[4])
    assert (s.targets_per_lane, s.leaf_max, s.walk_mode) == best[:3]
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.array_equal(before[k], after[k]), k
    a0 = np.stack([acc0[k] for k in ("ax", "ay", "az")], 1).astype(np.float64)
    a1 = np.stack([acc1[k] for k in ("ax", "ay", "az")], 1).astype(np.float64)
    rel = np.linalg.norm(a0 - a1, axis=1) / np.linalg.norm(a0, axis=1)
    assert rel.max() < 1e-4, rel.max()
    sim.step(2)
    sim.sync()
    assert sim.stats().status == 0 and sim.stats().steps_done == 5
    sim.close()


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_shared_walk_gives_the_same_interactions(nb, cuda, mode):
    """The shared walk (span_walk): the groups of one span node start from
    the shared sources and frontier of one traversal with the span's box.
    Every target must get exactly the interactions of a walk from the root
    (the interaction count is equal), summed in another order (forces agree
    to FP32 rounding)."""
    n = 200_000
    st = disk(nb, n, 0.3, 30.0, seed=8, m=1e-9)
    out = {}
    for sw in (2, 1):
        prm = nb.sim_params(dt=0.002, theta=0.5, softening=5e-4, star_mass=0.0, r_coll=0.0,
                            walk_mode=mode, group_span=8, span_walk=sw)
        sim = nb.Sim(prm, n)
        sim.set_state(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], st["m"])
        g = sim.get_state(accel=True)
        s = sim.stats()
        out[sw] = (np.stack([g["ax"], g["ay"], g["az"]], 1).astype(np.float64), s)
        sim.close()
    (a0, s0), (a1, s1) = out[2], out[1]
    assert s0.span_walk == 0 and s1.span_walk == 1 and s1.spans > 0
    assert s1.status == 0 and s0.status == 0
    assert s1.interactions == s0.interactions
    scale = np.sqrt(np.mean((a0 * a0).sum(1)))
    d = np.linalg.norm(a1 - a0, axis=1) / scale
    print(f"mode {mode}: spans {s1.spans} shared {s1.span_shared} frontier {s1.span_frontier} "
          f"visited {s0.walk_nodes_visited} -> {s1.walk_nodes_visited}; "
          f"diff max {d.max():.2e} median {np.median(d):.2e}")
    assert d.max() < 5e-5


@pytest.mark.parametrize("precision", [0, 1], ids=["f32", "f64"])
def test_open_steps_equal_one_call(nb, cuda, precision):
    """Steps taken one call at a time and left open (nbody_sim_step_open)
    run every step in its fused form; with the final second kick done by
    nbody_sim_close they must equal one nbody_sim_step call of as many
    steps, bit for bit (drag and perturber on)."""
    n = 6000
    st = disk(nb, n, 0.5, 5.0, seed=12, m=1e-8)
    prm = nb.sim_params(dt=0.005, theta=0.5, softening=1e-3, star_mass=1.0, r_coll=0.0,
                        gas_drag_rate=1e-3, perturber_enabled=1, perturber_mass_mjup=2.0,
                        perturber_radius_au=7.0, state_precision=precision)
    out = []
    for mode in ("one call", "open"):
        sim = nb.Sim(prm, n)
        sim.set_state(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], st["m"])
        if mode == "one call":
            sim.step(7)
        else:
            for _ in range(7):
                sim.step_open(1)
            sim.close_steps()
        sim.sync()
        out.append(sim.get_state(double=True, accel=False))
        assert sim.stats().steps_done == 7
        sim.close()
    for k in out[0]:
        assert np.array_equal(out[0][k], out[1][k]), k
    # a read of the state closes a pending step by itself
    sim = nb.Sim(prm, n)
    sim.set_state(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], st["m"])
    for _ in range(7):
        sim.step_open(1)
    g = sim.get_state(double=True, accel=False)
    sim.close()
    for k in g:
        assert np.array_equal(g[k], out[0][k]), k
