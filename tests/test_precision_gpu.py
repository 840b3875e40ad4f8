"""Precision modes and accuracy diagnostics.

* nbody_direct_f64 (the FP64 yardstick) against the oracle's FP64 direct sum.
* The softened energy and L_y of the diagnostics module against the oracle's.
* Hi/lo float-pair state (NBODY_STATE_F32X2): keeps about 48 significant
  bits through set/get, and its trajectory tracks the FP64 engine far more
  closely than the FP32 engine does.
* The walk's force error at the headline theta stays under the 1e-3 median
  bar against the FP64 direct sum (GPU yardstick, N = 65536), and its
  self-gravity error is no larger than the reference walk's.
"""
from __future__ import annotations

import importlib

import numpy as np
import pytest

from conftest import disk

pytestmark = pytest.mark.gpu

dg = importlib.import_module("nbody-sim_b200.diagnostics")


def test_direct_f64_matches_oracle(nb, cuda, port):
    n = 3000
    st = disk(nb, n, 0.5, 5.0, seed=4, m=1e-8)
    eps = 1e-3
    tg = np.arange(0, n, 7).astype(np.int32)
    x64 = [cuda.from_numpy(st[k].astype(np.float64)).cuda() for k in ("x", "y", "z")]
    m = cuda.from_numpy(st["m"]).cuda()
    ax, ay, az, phi = nb.direct_f64(*x64, m, eps, targets=cuda.from_numpy(tg).cuda(),
                                    want_phi=True)
    rx, ry, rz = port.direct_f64(st["x"], st["y"], st["z"], st["m"], tg, eps, 1.0, False)
    for got, ref in ((ax, rx), (ay, ry), (az, rz)):
        g = got.cpu().numpy()
        assert np.max(np.abs(g - ref)) <= 1e-12 * np.max(np.abs(ref))
    # potential: every body, against the pair sum of the oracle's energy
    _, _, _, phi_all = nb.direct_f64(*x64, m, eps, want_acc=False, want_phi=True)
    w = 0.5 * np.sum(st["m"].astype(np.float64) * phi_all.cpu().numpy())
    z = np.zeros(n)
    e_pair, _ = port.energy_f64(st["x"], st["y"], st["z"], z, z, z, st["m"], eps, 0.0)
    assert abs(w - e_pair) <= 1e-12 * abs(e_pair)


def test_conserved_matches_oracle(nb, cuda, port):
    n = 2500
    st = disk(nb, n, 0.5, 5.0, seed=5, m=1e-8)
    c = dg.conserved(st, st["m"], 1e-3, 1.0)
    e, ly = port.energy_f64(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], st["m"],
                            1e-3, 1.0)
    assert abs(c["E"] - e) <= 1e-12 * abs(e)
    assert abs(c["L_y"] - ly) <= 1e-12 * abs(ly)


def _sim(nb, prec, n, st, steps):
    prm = nb.sim_params(dt=0.002, theta=0.5, softening=5e-4, star_mass=1.0, r_coll=0.0,
                        gas_drag_rate=0.0, state_precision=prec)
    sim = nb.Sim(prm, n)
    dt = np.float32 if prec == nb.STATE_F32 else np.float64
    sim.set_state(*[st[k].astype(dt) for k in ("x", "y", "z", "vx", "vy", "vz")], st["m"])
    s0 = sim.get_state(double=True)
    sim.step(steps)
    sim.sync()
    s1 = sim.get_state(double=True)
    sim.close()
    return s0, s1


def test_hilo_state_keeps_48_bits_and_tracks_f64(nb, cuda):
    n = 20000
    d = nb.make_disk(n, 0.3, 30.0, 0.01, 0.005, 1.0, 7)
    st = dict(d)
    st["m"] = np.full(n, 1e-9, np.float32)
    h0, h1 = _sim(nb, nb.STATE_F32X2, n, st, 30)
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        rel = np.abs(h0[k] - d[k]) / np.maximum(np.abs(d[k]), 1e-300)
        assert np.max(rel) <= 2.0 ** -47, k
    _, f1 = _sim(nb, nb.STATE_F64, n, st, 30)
    _, s1 = _sim(nb, nb.STATE_F32, n, st, 30)
    err_hilo = max(np.max(np.abs(h1[k] - f1[k])) for k in ("x", "y", "z"))
    err_f32 = max(np.max(np.abs(s1[k] - f1[k])) for k in ("x", "y", "z"))
    # both walks see float positions, so the hi/lo run differs from FP64 only
    # by the state's rounding: orders of magnitude below FP32 state's
    assert err_hilo < 1e-3 * err_f32, (err_hilo, err_f32)


def test_walk_force_error_vs_fp64_direct(nb, cuda, port):
    """Headline bar on the total acceleration; the self-gravity part of an
    extended thin disk is a near-cancelling sum, so its relative error is far
    larger for any monopole walk: it must not exceed the reference walk's
    (the CPU restatement of BHTree.cu:530-598) on the same bodies."""
    n = 65536
    d = nb.make_disk(n, 0.3, 30.0, 0.01, 0.005, 1.0, 0)
    st = {k: d[k].astype(np.float32) for k in ("x", "y", "z")}
    st["m"] = np.full(n, 1e-9, np.float32)
    tg = np.sort(np.random.default_rng(0).choice(n, 4096, replace=False))
    r = dg.force_errors(st, 0.5, 5e-4, 1.0, tg, keep=True)
    assert r["status"] == 0
    assert r["total"]["median"] <= 1e-3
    rx, ry, rz, _ = port.forces(st["x"], st["y"], st["z"], st["m"], 0.5, 5e-4, 0.0)
    ref = np.stack([rx[tg], ry[tg], rz[tg]], 1).astype(np.float64)
    e_ref = np.linalg.norm(ref - r["direct_self"], axis=1) / np.linalg.norm(r["direct_self"],
                                                                             axis=1)
    assert r["self"]["median"] <= np.median(e_ref)
    assert r["self"]["p99"] <= np.percentile(e_ref, 99)
    r3 = dg.force_errors(st, 0.3, 5e-4, 1.0, tg)
    assert r3["self"]["median"] < r["self"]["median"]
