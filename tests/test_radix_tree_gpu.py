"""The binary radix tree of the octree build (nbody_radix_tree_u32) against a
restatement of Karras's published construction (Karras 2012, "Maximizing
parallelism in the construction of BVHs, octrees, and k-d trees", Fig. 4),
in Python on the CPU: the library's tree must be exactly the restatement's
(integer arrays, bit for bit), including long runs of equal keys (split by
index) and tiny inputs."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def karras_numpy(keys):
    """Internal nodes 0 .. n-2: (left, right, lo, hi, delta) with leaves
    encoded n - 1 + j.  delta(i, j) is the common prefix of the 64-bit
    (key, index) strings; -1 outside [0, n)."""
    n = len(keys)
    k = keys.astype(np.uint64)

    def delta(i, j):
        if j < 0 or j >= n:
            return -1
        a, b = int(k[i]), int(k[j])
        if a != b:
            return 32 - (a ^ b).bit_length()
        return 32 + 32 - (i ^ j).bit_length()

    left = np.zeros(n - 1, np.int64)
    right = np.zeros(n - 1, np.int64)
    lo_a = np.zeros(n - 1, np.int64)
    hi_a = np.zeros(n - 1, np.int64)
    dn = np.zeros(n - 1, np.int64)
    for i in range(n - 1):
        d = 1 if delta(i, i + 1) - delta(i, i - 1) > 0 else -1
        dmin = delta(i, i - d)
        lmax = 2
        while delta(i, i + lmax * d) > dmin:
            lmax *= 2
        l = 0
        t = lmax // 2
        while t >= 1:
            if delta(i, i + (l + t) * d) > dmin:
                l += t
            t //= 2
        j = i + l * d
        dnode = delta(i, j)
        s = 0
        t = l
        while True:
            t = (t + 1) // 2
            if delta(i, i + (s + t) * d) > dnode:
                s += t
            if t <= 1:
                break
        gamma = i + s * d + min(d, 0)
        lo, hi = min(i, j), max(i, j)
        left[i] = (n - 1) + gamma if lo == gamma else gamma
        right[i] = (n - 1) + gamma + 1 if hi == gamma + 1 else gamma + 1
        lo_a[i], hi_a[i], dn[i] = lo, hi, dnode
    return left, right, lo_a, hi_a, dn


def tree_gpu(nb, cuda, keys, bits):
    n = len(keys)
    kt = cuda.from_numpy(keys.view(np.int32)).cuda()
    out = [cuda.empty(max(n - 1, 1), dtype=cuda.int32, device="cuda") for _ in range(4)]
    pre = cuda.empty(max(n - 1, 1), dtype=cuda.uint8, device="cuda")
    rc = nb.lib.nbody_radix_tree_u32(kt.data_ptr(), n, bits, *[o.data_ptr() for o in out],
                                     pre.data_ptr())
    assert rc == 0, nb.lib.nbody_last_error()
    return [o.cpu().numpy()[: n - 1] for o in out] + [pre.cpu().numpy()[: n - 1]]


@pytest.mark.parametrize("n,dup", [(2, 0), (3, 0), (33, 0), (1000, 0), (5000, 1), (20000, 2)])
def test_radix_tree_matches_the_restatement(nb, cuda, n, dup):
    rng = np.random.default_rng(n + dup)
    bits = 30
    keys = rng.integers(0, 1 << bits, n, dtype=np.uint32)
    if dup == 1:   # long runs of one key
        keys[rng.integers(0, n, n // 3)] = keys[0]
    if dup == 2:   # few distinct keys: deep index splits everywhere
        keys = rng.integers(0, 64, n, dtype=np.uint32) << np.uint32(20)
    keys = np.sort(keys)
    left, right, lo, hi, dn = karras_numpy(keys)
    g = tree_gpu(nb, cuda, keys, bits)
    assert np.array_equal(g[0], left) and np.array_equal(g[1], right)
    assert np.array_equal(g[2], lo) and np.array_equal(g[3], hi)
    pref = np.where(dn >= 32, bits, dn - (32 - bits))
    assert np.array_equal(g[4].astype(np.int64), pref)
