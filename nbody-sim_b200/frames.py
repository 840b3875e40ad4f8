"""frames.bin reader and validator.

Reads the file OutputWriter writes (src/io/OutputWriter.cpp:56-79 header,
:96-115 frames) the way the reference's visualiser reads it
(unity-visualizer/Assets/Scripts/NBodyReader.cs): a 32-byte header -- magic
"NBOD", uint32 version (1 or 2), uint32 particle count, uint32 frame count,
float64 dt, float64 output dt -- then per frame a float64 time, the x, y and
z float32 arrays and, from version 2 on, a uint16 aggregate size per
particle (1 when the file has none).  ``validate`` applies the size check of
test_frames_validator.cs:39: 32 + frames * (8 + n * (3 * 4 + 2)).
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass

import numpy as np

HEADER_BYTES = 32


@dataclass
class Header:
    version: int
    n_particles: int
    n_frames: int
    dt: float
    output_dt: float


class FramesReader:
    """Random access to the frames of a frames.bin (memory-mapped)."""

    def __init__(self, path: str):
        if not os.path.exists(path):
            raise FileNotFoundError(f"frames.bin not found: {path}")
        with open(path, "rb") as f:
            head = f.read(HEADER_BYTES)
        if len(head) < HEADER_BYTES or head[:4] != b"NBOD":
            got = head[:4].decode("latin-1", "replace")
            raise ValueError(f"Invalid file (expected magic 'NBOD', got '{got}'). "
                             "Is this a frames.bin produced by nbody-sim?")
        version, n, frames = struct.unpack_from("<III", head, 4)
        if version not in (1, 2):
            raise ValueError(f"Unsupported frames.bin version {version}. Supported: 1, 2.")
        dt, output_dt = struct.unpack_from("<dd", head, 16)
        self.header = Header(version, n, frames, dt, output_dt)
        self.has_aggregate_sizes = version >= 2
        self.frame_bytes = 8 + n * 12 + (n * 2 if self.has_aggregate_sizes else 0)
        self._mm = np.memmap(path, dtype=np.uint8, mode="r")

    def __len__(self):
        return self.header.n_frames

    def read_frame(self, index: int):
        """(time, x, y, z, agg_size) of frame ``index``; agg_size is all ones
        for version 1 files."""
        h = self.header
        if index < 0 or index >= h.n_frames:
            raise IndexError(f"Frame {index} out of range [0, {h.n_frames - 1}].")
        off = HEADER_BYTES + index * self.frame_bytes
        n = h.n_particles
        buf = self._mm[off:off + self.frame_bytes]
        if len(buf) < self.frame_bytes:
            raise ValueError(f"Frame {index} is truncated")
        t = struct.unpack_from("<d", buf, 0)[0]
        xyz = np.frombuffer(buf, dtype="<f4", count=3 * n, offset=8).reshape(3, n)
        if self.has_aggregate_sizes:
            agg = np.frombuffer(buf, dtype="<u2", count=n, offset=8 + 12 * n)
        else:
            agg = np.ones(n, np.uint16)
        return t, xyz[0], xyz[1], xyz[2], agg


def validate(path: str) -> dict:
    """Header fields and the file-size check of test_frames_validator.cs:39."""
    r = FramesReader(path)
    h = r.header
    expected = HEADER_BYTES + h.n_frames * (8 + h.n_particles * (3 * 4 + 2))
    actual = os.path.getsize(path)
    out = {"magic": "NBOD", "version": h.version, "n_particles": h.n_particles,
           "n_frames": h.n_frames, "dt": h.dt, "output_dt": h.output_dt,
           "total_time": h.n_frames * h.output_dt, "expected_bytes": expected,
           "actual_bytes": actual, "size_ok": expected == actual}
    if h.n_frames > 0 and actual >= HEADER_BYTES + r.frame_bytes:
        t, x, _, _, _ = r.read_frame(0)
        out["first_time"] = t
        out["first_x0"] = float(x[0]) if h.n_particles else None
    return out
