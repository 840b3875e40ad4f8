"""The allocation-free FoF entry point, nbody_fof_noalloc, against nbody_fof.

Some callers cannot allocate device memory at the moment they need
aggregates: a process that polls a running simulation's snapshots while the
simulation holds the rest of the GPU's memory, code whose device memory
belongs to another allocator, or a loop that must not stall in cudaMalloc or
cudaFree.  nbody_fof_noalloc keeps all of its scratch in one static device
array inside the library.  These tests call it through the C ABI, twice in a
row on different inputs, and check every result against the allocating
nbody_fof on the same inputs.  Labels and sizes are integers, so the bar is
bit-for-bit equality, as for the other FoF tests.  One test runs in a fresh
process on a GPU whose memory is full once the device has been set up (the
first call, which under lazy module loading is when the library's array and
kernels take their device memory).

The file name sorts last, so a stop-at-first-failure run has run every other
test before it; it also passes run alone in a fresh process.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def clustered(seed, n, spread=0.003):
    rng = np.random.default_rng(seed)
    centers = rng.random((max(n // 100, 2), 3)).astype(np.float32)
    pts = centers[rng.integers(0, len(centers), n)] + \
        rng.standard_normal((n, 3)).astype(np.float32) * spread
    return [np.ascontiguousarray(pts[:, k], np.float32) for k in range(3)]


def check_against_fof(nb, cuda, seed, n, ll):
    x, y, z = [cuda.from_numpy(a).cuda() for a in clustered(seed, n)]
    tree = nb.Octree(n)
    l_ref, a_ref, g_ref = tree.fof(x, y, z, ll)
    tree.close()
    labels, agg, g = nb.fof_noalloc(x, y, z, ll)
    assert g == g_ref and g > 0
    assert cuda.equal(labels, l_ref)
    assert cuda.equal(agg, a_ref)


def test_noalloc_fof_matches_fof_on_consecutive_calls(nb, cuda):
    # the second call is smaller than the first: whatever the first left in
    # the shared scratch must not leak into the second's result
    check_against_fof(nb, cuda, 31, 20000, 0.0015)
    check_against_fof(nb, cuda, 32, 5000, 0.004)


def test_noalloc_fof_at_the_size_limit(nb, cuda):
    check_against_fof(nb, cuda, 33, nb.FOF_NOALLOC_MAX_N, 0.002)


def test_noalloc_fof_rejects_sizes_beyond_the_limit(nb, cuda):
    n = nb.FOF_NOALLOC_MAX_N + 1
    x = cuda.zeros(n, dtype=cuda.float32, device="cuda")
    with pytest.raises(nb.NBodyError) as e:
        nb.fof_noalloc(x, x, x, 0.01)
    assert e.value.code == nb.NBODY_ERR_ARG
    assert "NBODY_FOF_NOALLOC_MAX_N" in str(e.value)


_FULL_GPU_CHILD = r"""
import ctypes as C, importlib, json, sys
import numpy as np, torch
sys.path.insert(0, sys.argv[1])
nb = importlib.import_module("nbody-sim_b200")
torch.cuda.set_device(0)
n, ll = 20000, 0.0015
rng = np.random.default_rng(41)
centers = rng.random((200, 3)).astype(np.float32)
pts = centers[rng.integers(0, 200, n)] + rng.standard_normal((n, 3)).astype(np.float32) * 0.003
x, y, z = [torch.from_numpy(np.ascontiguousarray(pts[:, k])).cuda() for k in range(3)]
labels = torch.empty(n, dtype=torch.int32, device="cuda")
agg = torch.empty(n, dtype=torch.int16, device="cuda")
torch.cuda.synchronize()
nb.fof_noalloc_setup()                      # the device's one-time set-up
free_after_setup = torch.cuda.mem_get_info()[0]
fill, chunk = [], 1 << 30                   # take every byte the GPU has left
while True:
    try:
        fill.append(torch.empty(chunk, dtype=torch.uint8, device="cuda"))
    except torch.OutOfMemoryError:
        if chunk <= (2 << 20):
            break
        chunk //= 2
free_before = torch.cuda.mem_get_info()[0]
alloc_before = torch.cuda.memory_allocated()
ng = C.c_int()
rcs = []
for _ in range(2):
    rcs.append(nb.lib.nbody_fof_noalloc(x.data_ptr(), y.data_ptr(), z.data_ptr(), n, ll,
                                        labels.data_ptr(), agg.data_ptr(), C.byref(ng)))
torch.cuda.synchronize()
free_after = torch.cuda.mem_get_info()[0]
alloc_after = torch.cuda.memory_allocated()
err = nb.lib.nbody_last_error().decode() if any(rcs) else ""
del fill
torch.cuda.empty_cache()
tree = nb.Octree(n)
l_ref, a_ref, g_ref = tree.fof(x, y, z, ll)
print(json.dumps({"rcs": rcs, "error": err, "groups": ng.value, "groups_ref": g_ref,
                  "labels_equal": bool(torch.equal(labels, l_ref)),
                  "agg_equal": bool(torch.equal(agg, a_ref)),
                  "free_after_setup": free_after_setup, "free_before": free_before,
                  "free_after": free_after, "alloc_before": alloc_before,
                  "alloc_after": alloc_after}))
"""


def test_noalloc_fof_runs_on_a_full_gpu_after_setup(nb, cuda):
    """The property the entry point exists for.  In a fresh process (so the
    set-up has not happened yet): inputs and outputs are allocated, the
    device is set up with an n = 0 call, then every byte of free device
    memory is taken.  Two calls in a row must still succeed, leave the free
    memory and torch's allocation count unchanged, and give nbody_fof's
    results."""
    import json
    import subprocess
    import sys
    from conftest import ROOT
    r = subprocess.run([sys.executable, "-c", _FULL_GPU_CHILD, ROOT], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["rcs"] == [0, 0], out
    assert out["free_before"] < (64 << 20), out  # the GPU really was full
    assert out["free_after"] == out["free_before"], out
    assert out["alloc_after"] == out["alloc_before"], out
    assert out["groups"] == out["groups_ref"] and out["groups"] > 0
    assert out["labels_equal"] and out["agg_equal"]
