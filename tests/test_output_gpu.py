"""GPU output pipeline (nbody_sim_output_begin / _wait) against the host path.

The reference's output step (src/main.cu:143-181) copies the state to the
host, runs detectAggregates and fills agg_size.  The pipeline does the same
on a side stream while the engine keeps stepping.  Its frame must equal the
engine's state at the moment output_begin was called (bit for bit), its
agg_size must equal the FoF of that snapshot, and its aggregate records must
equal the host reconstruction of Aggregate.cpp:54-74 (nbody_aggregates) and,
where the reference host build is present, detectAggregates itself.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("id", "n_particles", "mass_msun", "cx", "cy", "cz", "vx", "vy", "vz", "dist_center",
          "first_member")


def clumpy_state(n, seed):
    rng = np.random.default_rng(seed)
    centers = rng.uniform(-3, 3, (n // 40, 3))
    centers[:, 1] *= 0.05
    pos = centers[rng.integers(0, len(centers), n)] + rng.standard_normal((n, 3)) * 2e-4
    r = np.linalg.norm(pos[:, [0, 2]], axis=1) + 0.5
    pos[:, [0, 2]] *= (r / np.linalg.norm(pos[:, [0, 2]], axis=1))[:, None]
    vk = 1.0 / np.sqrt(r)
    phi = np.arctan2(pos[:, 2], pos[:, 0])
    vel = np.stack([-vk * np.sin(phi), np.zeros(n), vk * np.cos(phi)], 1)
    st = {k: np.ascontiguousarray(pos[:, i], np.float32) for i, k in enumerate(("x", "y", "z"))}
    st.update({k: np.ascontiguousarray(vel[:, i], np.float32)
               for i, k in enumerate(("vx", "vy", "vz"))})
    st["m"] = np.full(n, 1e-10, np.float32)
    return st


def make_sim(nb, n, st):
    prm = nb.sim_params(dt=1e-4, theta=0.5, softening=1e-4, star_mass=1.0, r_coll=0.0,
                        gas_drag_rate=0.0)
    sim = nb.Sim(prm, n)
    sim.set_state(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], st["m"])
    return sim


def records(arr, count):
    return [tuple(getattr(arr[i], f) for f in FIELDS) for i in range(count)]


def test_frame_matches_engine_state_fof_and_host_aggregates(nb, cuda, refhost):
    n, ll, pm = 20000, 8e-4, 1e-10
    st = clumpy_state(n, 1)
    sim = make_sim(nb, n, st)
    sim.step(3)
    ref = sim.get_state(accel=False)
    sim.output_begin(ll, pm, 0.5, 7)
    sim.step(4)  # the engine keeps going while the frame is produced
    fr = sim.output_wait()
    assert fr["frame_index"] == 7 and fr["sim_time"] == 0.5
    for k in ("x", "y", "z"):
        assert np.array_equal(fr[k], ref[k]), k
    # FoF of the same snapshot through the tree API
    x, y, z = [cuda.from_numpy(ref[k]).cuda() for k in ("x", "y", "z")]
    tree = nb.Octree(n)
    labels, agg, ng = tree.fof(x, y, z, ll)
    tree.close()
    assert np.array_equal(fr["agg_size"], agg.cpu().numpy().view(np.uint16))
    host, cnt = nb.aggregates_from_labels(ref["x"], ref["y"], ref["z"], ref["vx"], ref["vy"],
                                          ref["vz"], labels.cpu().numpy(), pm)
    assert fr["n_aggregates"] == cnt and cnt > 50
    assert records(fr["aggregates"], cnt) == records(host, cnt)
    # the reference's own detectAggregates on the snapshot
    rl, rsize, rng_, ra = refhost.detect_aggregates(ref["x"], ref["y"], ref["z"], ref["vx"],
                                                    ref["vy"], ref["vz"], ll, pm)
    assert rng_ == cnt
    assert np.array_equal(fr["agg_size"], rsize)
    got = fr["aggregates"]
    assert [a.n_particles for a in got] == list(ra["n"])
    assert np.array_equal(np.array([a.mass_msun for a in got], np.float32), ra["mass"])
    c = np.array([[a.cx, a.cy, a.cz] for a in got], np.float32).reshape(-1)
    v = np.array([[a.vx, a.vy, a.vz] for a in got], np.float32).reshape(-1)
    assert np.array_equal(c, ra["c"]) and np.array_equal(v, ra["v"])
    assert np.array_equal(np.array([a.dist_center for a in got], np.float32), ra["dist"])
    sim.close()


def test_two_frames_in_flight_and_order(nb, cuda):
    n = 8000
    st = clumpy_state(n, 2)
    sim = make_sim(nb, n, st)
    refs = []
    for f in range(2):
        sim.step(2)
        refs.append(sim.get_state(accel=False))
        sim.output_begin(8e-4, 1e-10, float(f), f)
    with pytest.raises(nb.NBodyError) as e:
        sim.output_begin(8e-4, 1e-10, 2.0, 2)
    assert e.value.code == nb.NBODY_ERR_STATE
    for f in range(2):
        fr = sim.output_wait()
        assert fr["frame_index"] == f
        assert np.array_equal(fr["x"], refs[f]["x"])
    with pytest.raises(nb.NBodyError):
        sim.output_wait()
    sim.close()


def test_pipelined_run_writes_the_same_files_as_the_synchronous_run(nb, cuda, tmp_path):
    """run_simulation with the GPU pipeline against the reference's stop-copy-
    detect-write order: frames.bin and stats.csv byte for byte (C1-sized run
    with collisions, drag and a perturber)."""
    run = __import__("importlib").import_module("nbody-sim_b200.run")
    cfg = nb.default_config()
    cfg.n_particles = 4096
    cfg.disk_r_min, cfg.disk_r_max = 0.5, 5.0
    cfg.particle_mass_msun = 1e-8
    cfg.softening_AU = 1e-3
    cfg.collision_radius_factor = 5.0
    cfg.gas_drag_rate = 1e-3
    cfg.dt = 0.01
    cfg.total_time = 0.6
    cfg.output_every_n_steps = 10
    cfg.perturber_enabled = 1
    cfg.perturber_mass_mjup = 1.0
    cfg.perturber_radius_AU = 5.2
    outs = []
    for pipelined in (True, False):
        d = tmp_path / ("pipe" if pipelined else "sync")
        d.mkdir()
        r = run.run_simulation(cfg, str(d), pipelined=pipelined, precision=nb.STATE_F64)
        assert r["frames"] == 6 and r["steps"] == 60
        outs.append({f: (d / f).read_bytes() for f in ("frames.bin", "stats.csv")})
    assert outs[0]["frames.bin"] == outs[1]["frames.bin"]
    assert outs[0]["stats.csv"] == outs[1]["stats.csv"]
    assert len(outs[0]["frames.bin"]) == 32 + 6 * (8 + 14 * 4096)
