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
