"""Per-phase profiling (nbody_sim_set_profiling): profiled steps run the same
kernels as plain ones, with graphs on (events captured as nodes of the step
graphs) and off (kernels launched one by one), so the state after them is
bit-identical; every phase of a collisional step but the closing one gets a
positive time, the step counts match, and the phase sum stays within a sane
bound of the plain step's own device time."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import disk

pytestmark = pytest.mark.gpu


def _params(nb):
    return nb.sim_params(dt=0.005, theta=0.5, softening=1e-3, star_mass=1.0,
                         r_coll=5.0 * nb.particle_physical_radius(1e-8), restitution=0.0,
                         gas_drag_rate=1e-3, fuse_collisions=0)


@pytest.mark.parametrize("graphs", [True, False], ids=["graphs", "eager"])
def test_profiled_steps_equal_plain_steps(nb, cuda, graphs):
    n = 20000
    st = disk(nb, n, 0.5, 5.0, seed=4, m=1e-8)
    prm = _params(nb)
    out = []
    for profiled in (True, False):
        sim = nb.Sim(prm, n)
        sim.set_graphs(graphs)
        sim.set_state(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], st["m"])
        sim.set_profiling(profiled)
        for _ in range(4):
            sim.step_open(1)
        sim.close_steps()
        prof = sim.profile(reset=True)
        out.append((sim.get_state(double=True, accel=True), prof))
        sim.close()
    (a, pa), (b, pb) = out
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert pa["steps"] == 4 and pb["steps"] == 0
    for name in nb.PHASE_NAMES:  # the collide boundary only closes the step
        assert pa[name] > 0.0 or (name == "collide" and pa[name] >= 0.0), name


def test_profiled_phase_sum_matches_the_step(nb, cuda):
    """The phases of a profiled graph step add up to about the step's own
    device time (events inside the graph cost a little; a factor of two
    either way would mean the boundaries are misplaced)."""
    n = 100000
    st = disk(nb, n, 0.3, 30.0, seed=5, m=1e-9)
    prm = nb.sim_params(dt=0.002, theta=0.5, softening=5e-4, star_mass=1.0, r_coll=0.0,
                        gas_drag_rate=0.0)
    sim = nb.Sim(prm, n)
    stream = torch.cuda.current_stream()
    sim.set_stream(stream.cuda_stream)
    sim.set_state(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], st["m"])
    for _ in range(3):
        sim.step_open(1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sim.sync()
    e0.record(stream)
    for _ in range(5):
        sim.step_open(1)
    sim.sync()
    e1.record(stream)
    torch.cuda.synchronize()
    plain_ms = e0.elapsed_time(e1) / 5
    sim.set_profiling(True)
    sim.profile(reset=True)
    for _ in range(5):
        sim.step_open(1)
    prof = sim.profile(reset=True)
    sim.set_profiling(False)
    sim.close_steps()
    sim.close()
    phase_ms = sum(prof[k] for k in nb.PHASE_NAMES) / prof["steps"]
    assert prof["steps"] == 5
    assert 0.5 * plain_ms < phase_ms < 2.0 * plain_ms, (phase_ms, plain_ms)
