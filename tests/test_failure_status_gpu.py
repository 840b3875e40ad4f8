"""The engine's failure statuses, raised without a GPU fault.

The reference loses work silently where its loops run out: its build drops a
body after 128 retries or when the node pool is full (BHTree.cu:246-250,276)
and its walk drops stack entries beyond 255 (BHTree.cu:589).  Every bounded
loop here instead raises a device status bit that the host turns into
NBODY_ERR_OVERFLOW.  These tests make three of them fire on purpose:

* a non-finite position reaching key generation (bit 8): the bbox ignores or
  collapses on it, the body gets key 0, and every later loop is bounded by
  integer tree sizes, so the step finishes and reports;
* a walk whose stack spill area is too small (bit 1): theta = 0 opens every
  node, so a warp's stack overflows its shared-memory part; with a spill
  capacity of one entry per warp the walk stops and reports;
* the radix sort's decoupled look-back wait (bit 32), run against tile
  status words that nothing publishes: it gives up after its bound.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import disk

pytestmark = pytest.mark.gpu
STATE = ("x", "y", "z", "vx", "vy", "vz")


@pytest.mark.parametrize("precision", [0, 1], ids=["f32", "f64"])
@pytest.mark.parametrize("bad", [np.nan, np.inf], ids=["nan", "inf"])
def test_non_finite_position_reports_overflow(nb, cuda, precision, bad):
    n = 4096
    st = disk(nb, n, 0.5, 5.0, seed=5, m=1e-8)
    st["x"] = st["x"].copy()
    st["x"][17] = bad
    prm = nb.sim_params(dt=0.01, theta=0.5, softening=1e-3, star_mass=1.0,
                        r_coll=nb.particle_physical_radius(1e-8), restitution=0.0,
                        state_precision=precision)
    sim = nb.Sim(prm, n)
    sim.set_state(*[st[k] for k in STATE], st["m"])
    sim.step(2)
    with pytest.raises(nb.NBodyError) as e:
        sim.sync()
    assert e.value.code == nb.NBODY_ERR_OVERFLOW
    assert "device status 8" in str(e.value)
    # the status was reported once and cleared; the context still works
    sim.close()
    ok = disk(nb, n, 0.5, 5.0, seed=5, m=1e-8)
    sim = nb.Sim(prm, n)
    sim.set_state(*[ok[k] for k in STATE], ok["m"])
    sim.step(2)
    sim.sync()
    assert sim.stats().status == 0
    sim.close()


def test_phase_api_reports_a_non_finite_position(nb, cuda):
    from test_gpu_core import to_gpu
    n = 1000
    st = disk(nb, n, 0.5, 5.0, seed=6, m=1e-8)
    st["z"] = st["z"].copy()
    st["z"][999] = np.nan
    p = to_gpu(nb, cuda, st)
    t = nb.Octree(n)
    t.reset()
    t.bbox(p)
    with pytest.raises(nb.NBodyError) as e:
        t.build(p)
        t.summarize()
        t.sort()
    assert e.value.code == nb.NBODY_ERR_OVERFLOW
    t.close()


def test_walk_stack_spill_capacity_reports_overflow(nb, cuda):
    n = 200_000
    st = disk(nb, n, 0.5, 5.0, seed=7, m=1e-8)

    def run(spill_cap):
        # theta 0 and single-body leaves: every node is opened and pushed, so
        # a warp's stack outgrows its shared-memory part
        prm = nb.sim_params(dt=0.01, theta=0.0, softening=1e-3, star_mass=1.0, r_coll=0.0,
                            leaf_max=1, spill_cap=spill_cap)
        sim = nb.Sim(prm, n)
        sim.set_state(*[st[k] for k in STATE], st["m"])
        return sim

    sim = run(0)  # the default capacity: the walk spills and finishes
    sim.sync()
    s = sim.stats()
    assert s.status == 0 and s.walk_stack_spills > 0
    assert s.interactions >= n * (n - 1)  # theta 0: every pair directly
    sim.close()
    sim = run(1)
    with pytest.raises(nb.NBodyError) as e:
        sim.sync()
    assert e.value.code == nb.NBODY_ERR_OVERFLOW
    assert "device status 1" in str(e.value)
    sim.close()


def test_sort_look_back_wait_gives_up(nb, cuda):
    import ctypes as C
    bits = C.c_int(-1)
    rc = nb.lib.nbody_selftest_sort_wait(C.byref(bits))
    assert rc == 0, nb.lib.nbody_last_error()
    assert bits.value == 32
