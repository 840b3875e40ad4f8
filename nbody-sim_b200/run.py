"""The reference's simulation driver (src/main.cu:85-190) on the B200 engine.

Same loop and outputs: forces at t = 0, ``int(total_time / dt)`` KDK steps,
and every ``output_every_n_steps`` steps a frame (positions + agg_size), the
aggregate statistics and, with a perturber, its row, written by the same
frames.bin / stats.csv writer.  The link length of the aggregates is the
collision radius (main.cu:58-59, :151).

Two output schedules:

* ``pipelined`` (default): the output step runs on the GPU's side stream
  (nbody_sim_output_begin) while the engine already steps towards the next
  frame; the host writes frame k while the GPU produces frame k+1.
* synchronous: the reference's order -- stop, copy the state to the host,
  aggregates, write -- with the aggregates from the GPU FoF.
"""
from __future__ import annotations

import importlib
import os
import time

import numpy as np


def _nb():
    return importlib.import_module("nbody-sim_b200")


class _Host:
    """Host arrays in the shape the writer binding expects (ParticleData)."""

    def __init__(self, n, x, y, z):
        self.n = n
        self.arrays = {"x": x, "y": y, "z": z}


def run_simulation(cfg, out_dir: str, state=None, precision=None, pipelined: bool = True,
                   total_steps: int | None = None, seed: int = 0, params=None):
    """Runs cfg (an nbody_config) and writes out_dir/frames.bin and stats.csv.

    ``state``: dict x..vz (float32 or float64 host arrays) and m; default a
    Keplerian disk from make_disk(seed).  ``params``: optional overrides of
    nbody_sim_params fields (e.g. the walk settings an autotune kept).
    Returns timings and counts."""
    nb = _nb()
    n = cfg.n_particles
    if state is None:
        d = nb.make_disk(n, cfg.disk_r_min, cfg.disk_r_max, 0.01, 0.005, cfg.star_mass_msun, seed)
        state = dict(d)
        state["m"] = np.full(n, cfg.particle_mass_msun, np.float32)
    prm = nb.sim_params(cfg)
    if precision is not None:
        prm.state_precision = precision
    for k, v in (params or {}).items():
        setattr(prm, k, v)
    r_coll = prm.r_coll
    pm = cfg.particle_mass_msun
    every = cfg.output_every_n_steps
    total = int(np.float32(cfg.total_time) / np.float32(cfg.dt)) if total_steps is None \
        else total_steps
    dt = np.float32(cfg.dt)
    pert = nb.make_perturber(cfg)

    sim = nb.Sim(prm, n)
    dbl = prm.state_precision != nb.STATE_F32
    ty = np.float64 if dbl else np.float32
    sim.set_state(*[np.asarray(state[k], ty) for k in ("x", "y", "z", "vx", "vy", "vz")],
                  state["m"])
    os.makedirs(out_dir, exist_ok=True)  # main.cu creates the run directory (:30-41)
    writer = nb.OutputWriter(out_dir, cfg)
    frames = 0
    n_out = total // every

    host = {"wait": 0.0, "write": 0.0, "enqueue": 0.0}

    def write(fr_x, fr_y, fr_z, agg, aggs, n_aggs, t, idx):
        t_w = time.perf_counter()
        writer.write_frame(_Host(n, fr_x, fr_y, fr_z), t, agg)
        writer.write_stats(aggs, idx, t, count=n_aggs)
        if pert.enabled:
            q = nb.nbody_perturber.from_buffer_copy(pert)
            nb.update_perturber(q, t)
            writer.write_perturber_stats(idx, t, n_aggs, q.x, q.y, q.z, q.mass_msun, q.omega)
        host["write"] += time.perf_counter() - t_w

    t0 = time.perf_counter()
    if pipelined:
        pending = 0
        for k in range(n_out):
            t_e = time.perf_counter()
            sim.step(every)
            t = np.float32((k + 1) * every) * dt
            sim.output_begin(r_coll, pm, float(t), k)
            host["enqueue"] += time.perf_counter() - t_e
            pending += 1
            if pending == 2:  # the older frame is ready or nearly so: write it
                t_q = time.perf_counter()
                fr = sim.output_wait(copy=False)
                host["wait"] += time.perf_counter() - t_q
                write(fr["x"], fr["y"], fr["z"], fr["agg_size"], fr["aggregates_ptr"],
                      fr["n_aggregates"], fr["sim_time"], fr["frame_index"])
                frames += 1
                pending -= 1
        while pending:
            fr = sim.output_wait(copy=False)
            write(fr["x"], fr["y"], fr["z"], fr["agg_size"], fr["aggregates_ptr"],
                  fr["n_aggregates"], fr["sim_time"], fr["frame_index"])
            frames += 1
            pending -= 1
    else:
        for k in range(n_out):
            t_e = time.perf_counter()
            sim.step(every)
            host["enqueue"] += time.perf_counter() - t_e
            t = float(np.float32((k + 1) * every) * dt)
            t_q = time.perf_counter()
            s = sim.get_state(accel=False)
            labels, agg, _ = sim.fof(r_coll)
            host["wait"] += time.perf_counter() - t_q
            aggs, cnt = nb.aggregates_from_labels(s["x"], s["y"], s["z"], s["vx"], s["vy"],
                                                  s["vz"], labels, pm)
            write(s["x"], s["y"], s["z"], agg, aggs, cnt, t, k)
            frames += 1
    rest = total - n_out * every
    if rest:
        sim.step(rest)
    sim.sync()
    secs = time.perf_counter() - t0
    writer.finalize(frames)
    writer.close()
    sim.close()
    return {"steps": total, "frames": frames, "seconds": secs,
            "particle_steps_per_s": n * total / secs, "host_seconds": host}
