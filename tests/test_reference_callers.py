"""The reference's own callers, built unmodified against the drop-in headers.

``make -C oracle dropin`` compiles, from the reference checkout where it lies
and without changing a line of it:

* ``src/main.cu`` (the reference's simulation driver; MSVC's localtime_s is
  mapped to glibc's localtime_r by a force-included shim) -> oracle/_ref/ref_main;
* ``tests/test_{bhtree,collision,integrator,perturber}.cu`` -> ref_tests_gpu;
* ``tests/test_{aggregate,config,disk_init,output}.cpp`` -> ref_tests_cpu;

all against include/nbody and libnbody_b200.so, behind a small Catch2 stand-in
(tests/cpp/catch2_shim; Catch2 v3.8.1 itself is not in this image).  The CPU
tests are also built against the reference's own host sources
(ref_tests_cpu_own) so both builds' outcomes can be compared case by case.
The binaries land in oracle/_ref/ and travel with the repository, so the GPU
tests below run them where the reference checkout is absent.
"""
from __future__ import annotations

import glob
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

OUT = os.path.join(ROOT, "oracle", "_ref")


def outcomes(binary, cwd, *args):
    r = subprocess.run([binary, *args], capture_output=True, text=True, cwd=cwd, timeout=600)
    res = {}
    for line in r.stdout.splitlines():
        f = line.split("\t")
        if f[0] in ("PASS", "FAIL"):
            res[f[1]] = (f[0], f[2] if len(f) > 2 else "")
    assert res, (r.stdout[-2000:], r.stderr[-2000:])
    return res, r.returncode


def binary(name):
    path = os.path.join(OUT, name)
    if not os.path.exists(path):
        pytest.skip(f"oracle/_ref/{name} not built (make -C oracle dropin, needs the reference)")
    return path


# -------------------------------------------------------------- CPU suite
@pytest.fixture(scope="module")
def built(nb, reference_root):
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "dropin"],
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-4000:]
    return reference_root


def test_reference_callers_compile_unmodified(built):
    for name in ("ref_main", "ref_tests_gpu", "ref_tests_cpu", "ref_tests_cpu_own"):
        assert os.access(os.path.join(OUT, name), os.X_OK), name


def test_reference_cpu_tests_same_outcomes_as_the_reference_build(built, tmp_path):
    """Case by case against the reference's own host code.  The FoF cases
    of the drop-in build run detectAggregates on the GPU, so without a
    device they are left to the GPU test below."""
    own, _ = outcomes(os.path.join(OUT, "ref_tests_cpu_own"), str(tmp_path))
    ours, _ = outcomes(os.path.join(OUT, "ref_tests_cpu"), str(tmp_path))
    assert set(own) == set(ours)
    for name, (res, msg) in own.items():
        if name.startswith("detectAggregates"):
            continue
        assert ours[name][0] == res, (name, ours[name], res, msg)
    # every case but the config-file one passes in the reference build
    assert [n for n, (r, _) in own.items() if r == "FAIL"] == \
        ["loadConfig reads simulation.json correctly"]


def test_reference_config_test_fails_the_same_way(built):
    """test_config.cpp:5-21 against the shipped config/simulation.json: the
    reference's own loadConfig fails it (the file no longer holds the values
    the test expects), and the drop-in loadConfig fails it at the same
    REQUIRE."""
    name = "loadConfig reads simulation.json correctly"
    own, _ = outcomes(os.path.join(OUT, "ref_tests_cpu_own"), built, name)
    ours, _ = outcomes(os.path.join(OUT, "ref_tests_cpu"), built, name)
    assert own[name][0] == "FAIL" and ours[name] == own[name]


# -------------------------------------------------------------- GPU suite
@pytest.mark.gpu
def test_reference_gpu_tests_pass(cuda, tmp_path):
    """tests/test_bhtree.cu, test_collision.cu, test_integrator.cu and
    test_perturber.cu of the reference, unmodified, on the drop-in engine."""
    res, rc = outcomes(binary("ref_tests_gpu"), str(tmp_path))
    failed = {k: v for k, v in res.items() if v[0] != "PASS"}
    assert not failed and rc == 0, failed
    assert len(res) == 9


@pytest.mark.gpu
def test_reference_cpu_tests_pass_with_the_gpu_fof(cuda, tmp_path):
    """tests/test_aggregate.cpp, test_config.cpp, test_disk_init.cpp and
    test_output.cpp, unmodified; detectAggregates runs on the GPU.  The one
    case that reads the shipped config/simulation.json fails in the
    reference's own build too (see the CPU test above); here the file is
    absent."""
    res, _ = outcomes(binary("ref_tests_cpu"), str(tmp_path))
    failed = {k: v for k, v in res.items() if v[0] != "PASS"}
    assert set(failed) == {"loadConfig reads simulation.json correctly"}, failed
    assert len(res) == 12


@pytest.mark.gpu
def test_reference_main_runs_on_the_drop_in_engine(nb, cuda, port, refhost, tmp_path):
    """src/main.cu, unmodified, on a small disk with collisions, gas drag and a
    perturber: 50 steps, a frame every 10.  frames.bin and stats.csv are
    read back; every frame's agg_size is bit-exact against the reference's
    own detectAggregates of that frame's positions; the last frame tracks the
    oracle's restatement of the same loop from the same initDisk disk."""
    import importlib
    frames = importlib.import_module("nbody-sim_b200.frames")
    cfg = {"n_particles": 2048, "total_time": 0.5, "dt": 0.01, "output_every_n_steps": 10,
           "output_dir": str(tmp_path / "data"), "gas_drag_rate": 0.01,
           "perturber_enabled": True, "perturber_mass_mjup": 1.0, "perturber_radius_AU": 20.0,
           "perturber_phase0": 0.0}
    cpath = tmp_path / "run.json"
    cpath.write_text(json.dumps(cfg))
    r = subprocess.run([binary("ref_main"), str(cpath)], capture_output=True, text=True,
                       cwd=str(tmp_path), timeout=600)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    runs = glob.glob(str(tmp_path / "data" / "*" / "frames.bin"))
    assert len(runs) == 1
    run_dir = os.path.dirname(runs[0])
    steps = int(np.float32(cfg["total_time"]) / np.float32(cfg["dt"]))
    n_frames = steps // cfg["output_every_n_steps"]
    rd = frames.FramesReader(runs[0])
    assert rd.header.n_particles == 2048 and rd.header.n_frames == n_frames
    assert os.path.getsize(runs[0]) == 32 + n_frames * (8 + 2048 * 14)
    with open(os.path.join(run_dir, "stats.csv")) as f:
        head = f.readline().strip()
        rows = f.read().strip().splitlines()
    assert head.startswith("frame,")
    # the perturber's rows: agg_id -1 (OutputWriter.cpp:161-186), one per frame
    assert sum(1 for row in rows if row.split(",")[4] == "-1") == n_frames
    m = np.float32(3.003e-7)
    r_coll = np.float32(100.0) * np.float32(refhost.particle_radius(m))
    zeros = np.zeros(2048, np.float32)
    for k in range(n_frames):
        _, x, y, z, agg = rd.read_frame(k)
        _, rsize, _, _ = refhost.detect_aggregates(x, y, z, zeros, zeros, zeros, r_coll, m)
        assert np.array_equal(agg, rsize), k
    # the same loop on the CPU restatement, from initDisk(cfg, 42)
    st = {k: np.zeros(2048, np.float32) for k in ("x", "y", "z", "vx", "vy", "vz")}
    import ctypes as C
    refhost.lib.ref_init_disk.argtypes = [C.c_int, C.c_uint] + [C.c_void_p] * 6
    assert refhost.lib.ref_init_disk(2048, 42, *[st[k].ctypes.data for k in
                                                 ("x", "y", "z", "vx", "vy", "vz")]) == 0
    st["m"] = np.full(2048, m, np.float32)
    pert = port.perturber(True, 1.0, 20.0, 0.0, 1.0)
    sp = port.step_params(0.01, 0.5, 0.01, 1.0, r_coll=float(r_coll), restitution=0.3,
                          gas_drag_rate=0.01, collisions=True, pert=pert)
    port.run(st, sp, steps)
    last = dict(zip(("t", "x", "y", "z", "agg"), rd.read_frame(n_frames - 1)))
    for k in ("x", "y", "z"):
        d = np.abs(last[k].astype(np.float64) - st[k])
        print(f"ref_main vs oracle {k}: median {np.median(d):.3e} max {d.max():.3e}")
        assert np.median(d) < 1e-5, (k, np.median(d))
