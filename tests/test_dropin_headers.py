"""The C++ drop-in headers (include/nbody/) compile as a reference caller
would use them, and their host-only parts agree with the reference's own
host code (CPU suite): loadConfig, initDisk (bit-for-bit with the reference's
DiskInit.cpp under the same standard library), particlePhysicalRadius,
makePerturber/updatePerturber, OutputWriter."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT


@pytest.fixture(scope="module")
def compat_bin(tmp_path_factory, nb):
    out = tmp_path_factory.mktemp("compat") / "compat_cpu"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", f"-I{ROOT}/include/nbody",
           "-I/usr/local/cuda/include", os.path.join(ROOT, "tests", "cpp", "compat_cpu.cpp"),
           "-o", str(out), f"-L{os.path.dirname(nb.LIB_PATH)}", "-lnbody_b200",
           "-L/usr/local/cuda/lib64", "-lcudart",
           f"-Wl,-rpath,{os.path.dirname(nb.LIB_PATH)}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def run(compat_bin, tmp_path, cfg="full.json"):
    r = subprocess.run([str(compat_bin), os.path.join(GOLDEN, "configs", cfg), str(tmp_path)],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    return {ln.split()[0]: ln.split()[1:] for ln in r.stdout.splitlines()}


def test_headers_compile_and_load_config(compat_bin, tmp_path):
    out = run(compat_bin, tmp_path)
    assert out["config"] == ["131072", "0.00499999989", "0.5", "50", "runs/full", "1"]
    assert " ".join(out["missing-file"]) == "Cannot open config: /nonexistent/path.json"
    assert out["writer"] == ["ok"]
    assert (tmp_path / "frames.bin").stat().st_size == 32 + 8 + 1000 * 14


def test_init_disk_bit_exact_with_reference(compat_bin, tmp_path, refhost):
    out = run(compat_bin, tmp_path)
    n = 1000
    arr = [np.zeros(n, np.float32) for _ in range(6)]
    refhost.lib.ref_init_disk.argtypes = [C.c_int, C.c_uint] + [C.c_void_p] * 6
    assert refhost.lib.ref_init_disk(n, 42, *[a.ctypes.data for a in arr]) == 0
    h = 0.0
    bits = [a.view(np.uint32) for a in arr]
    for i in range(n):
        for k in range(6):
            h = h * 1.0000001 + float(int(bits[k][i]) % 100003)
    assert float(out["disk"][0]) == pytest.approx(h, rel=1e-15)
    assert np.float32(out["disk"][1]) == arr[0][0]
    assert np.float32(out["disk"][2]) == arr[5][999]


def test_radius_and_perturber(compat_bin, tmp_path, refhost):
    out = run(compat_bin, tmp_path)
    assert np.float32(out["radius"][0]) == np.float32(refhost.particle_radius(3.003e-7))
    import oracle
    p = oracle.Port().perturber(True, 1.0, 10.0, 0.0, 1.0)
    q = oracle.Port().perturber_at(p, 12.5)
    assert np.float32(out["perturber"][0]) == np.float32(p.omega)
    assert np.float32(out["perturber"][1]) == np.float32(q.x)
    assert np.float32(out["perturber"][2]) == np.float32(q.z)
