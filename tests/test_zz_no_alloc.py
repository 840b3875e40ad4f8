"""The allocation-free FoF entry point, nbody_fof_noalloc, against nbody_fof.

Some callers cannot allocate device memory at the moment they need
aggregates: a process that polls a running simulation's snapshots while the
simulation holds the rest of the GPU's memory, code whose device memory
belongs to another allocator, or a loop that must not stall in cudaMalloc or
cudaFree.  nbody_fof_noalloc keeps all of its scratch in one static device
array inside the library.  These tests call it through the C ABI, twice in a
row on different inputs, and check every result against the allocating
nbody_fof on the same inputs.  Labels and sizes are integers, so the bar is
bit-for-bit equality, as for the other FoF tests.

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
