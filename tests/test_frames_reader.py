"""frames.bin reader / validator (nbody-sim_b200/frames.py) on the golden file
the reference's own OutputWriter wrote, and on round trips through the
writer.  CPU only."""
from __future__ import annotations

import importlib
import os
import struct

import numpy as np
import pytest

from conftest import GOLDEN

fr = importlib.import_module("nbody-sim_b200.frames")


def test_reads_the_reference_writer_golden_file():
    d = np.load(os.path.join(GOLDEN, "writer_run", "inputs.npz"))
    path = os.path.join(GOLDEN, "writer_run", "frames.bin")
    r = fr.FramesReader(path)
    n = int(d["n"])
    assert r.header.version == 2 and r.header.n_particles == n and len(r) == 3
    assert r.header.dt == pytest.approx(float(d["dt"]), rel=1e-7)
    assert r.header.output_dt == pytest.approx(float(d["dt"]) * int(d["output_every"]), rel=1e-7)
    for k in range(3):
        t, x, y, z, agg = r.read_frame(k)
        assert t == float(np.float32(d["t"][k]))
        assert np.array_equal(x, d["x"]) and np.array_equal(y, d["y"])
        assert np.array_equal(z, d["z"]) and np.array_equal(agg, d["agg"])
    v = fr.validate(path)
    assert v["size_ok"] and v["expected_bytes"] == 32 + 3 * (8 + n * 14)


def test_round_trip_through_the_writer(nb, tmp_path):
    n = 1000
    rng = np.random.default_rng(5)
    c = nb.default_config()
    c.n_particles, c.dt, c.output_every_n_steps = n, 0.005, 50
    w = nb.OutputWriter(str(tmp_path), c)
    p = nb.allocate_particles_cpu(n)
    frames = []
    for k in range(4):
        for key in ("x", "y", "z"):
            p.arrays[key][:] = rng.standard_normal(n).astype(np.float32)
        agg = rng.integers(1, 9, n).astype(np.uint16)
        t = float(np.float32((k + 1) * 50) * np.float32(0.005))
        w.write_frame(p, t, agg)
        frames.append((t, p.arrays["x"].copy(), p.arrays["y"].copy(), p.arrays["z"].copy(), agg))
    w.finalize(4)
    w.close()
    r = fr.FramesReader(str(tmp_path / "frames.bin"))
    assert len(r) == 4
    for k, want in enumerate(frames):
        got = r.read_frame(k)
        assert got[0] == pytest.approx(want[0], rel=1e-7)
        for a, b in zip(got[1:], want[1:]):
            assert np.array_equal(a, b)
    assert fr.validate(str(tmp_path / "frames.bin"))["size_ok"]
    with pytest.raises(IndexError):
        r.read_frame(4)


def test_rejects_bad_files(tmp_path):
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"XXXX" + bytes(28))
    with pytest.raises(ValueError, match="expected magic 'NBOD'"):
        fr.FramesReader(str(bad))
    v3 = tmp_path / "v3.bin"
    v3.write_bytes(b"NBOD" + struct.pack("<IIIdd", 3, 1, 0, 0.01, 0.1))
    with pytest.raises(ValueError, match="Unsupported frames.bin version 3"):
        fr.FramesReader(str(v3))
    with pytest.raises(FileNotFoundError):
        fr.FramesReader(str(tmp_path / "missing.bin"))


def test_version_1_files_have_unit_aggregate_sizes(tmp_path):
    n = 3
    path = tmp_path / "v1.bin"
    body = struct.pack("<d", 0.5) + np.arange(3 * n, dtype=np.float32).tobytes()
    path.write_bytes(b"NBOD" + struct.pack("<IIIdd", 1, n, 1, 0.01, 0.1) + body)
    r = fr.FramesReader(str(path))
    t, x, y, z, agg = r.read_frame(0)
    assert t == 0.5 and np.array_equal(agg, np.ones(n, np.uint16))
    assert np.array_equal(z, np.arange(6, 9, dtype=np.float32))
