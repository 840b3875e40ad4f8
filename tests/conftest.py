"""Shared fixtures for the nbody-b200 test suite.

Markers: ``gpu`` tests need a CUDA device and call the library through its C
ABI; everything else runs on CPU (oracle against golden vectors, host-side C
ABI pieces, multi-process host logic over gloo).
"""
from __future__ import annotations

import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def nb():
    """The product package (CUDA library through ctypes)."""
    return importlib.import_module("nbody-sim_b200")


@pytest.fixture(scope="session")
def port():
    import oracle
    return oracle.Port()


@pytest.fixture(scope="session")
def refhost():
    path = os.path.join(ROOT, "oracle", "_ref", "libref_host.so")
    if not os.path.exists(path):
        pytest.skip("oracle/_ref/libref_host.so not built (needs the reference checkout)")
    import oracle
    return oracle.RefHost(path)


@pytest.fixture(scope="session")
def reference_root():
    """The reference checkout, where oracle/Makefile looks for it
    (NBODY_REFERENCE_ROOT overrides); tests that read it skip without it."""
    import subprocess
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "print-ref"],
                       capture_output=True, text=True)
    path = r.stdout.strip()
    if not path or not os.path.isdir(os.path.join(path, "src")):
        pytest.skip("the reference checkout is absent (set NBODY_REFERENCE_ROOT)")
    return path


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def golden(name):
    return os.path.join(GOLDEN, name)


def disk(nb, n, r_min=0.5, r_max=5.0, seed=0, m=1e-8):
    d = nb.make_disk(n, r_min, r_max, 0.01, 0.005, 1.0, seed)
    out = {k: v.astype(np.float32) for k, v in d.items()}
    out["m"] = np.full(n, m, np.float32)
    return out
