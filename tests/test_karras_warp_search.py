"""The Karras pass's two searches (csrc/tree.cu k_karras), restated on the CPU.

A lane searches its own node's range end and split by the published
exponential and binary searches (Karras 2012, Fig. 4) while the range stays
below a cap; a node whose range reaches the cap is searched by the whole warp,
which tests 32 powers of two and then narrows [lo, hi) 32 points at a time.
This restatement of both paths must give every node the tree of the plain
restatement in tests/test_radix_tree_gpu.py (which the GPU kernel is checked
against bit for bit); small caps send most nodes down the warp path."""
from __future__ import annotations

import numpy as np
import pytest

from test_radix_tree_gpu import karras_numpy


def karras_two_path(keys, cap):
    n = len(keys)
    k = keys.astype(np.uint64)

    def delta(i, j):
        if j < 0 or j >= n:
            return -1
        a, b = int(k[i]), int(k[j])
        if a != b:
            return 32 - (a ^ b).bit_length()
        return 64 - (i ^ j).bit_length()

    def warp_last_above(i, d, thr, lo, hi):
        # 31 evenly spaced points a round; the ballot's count keeps the step after the last true one
        while hi - lo > 1:
            step = (hi - lo + 31) // 32
            c = sum(1 for lane in range(32)
                    if lo + (lane + 1) * step < hi
                    and delta(i, i + (lo + (lane + 1) * step) * d) > thr)
            nlo = lo + c * step
            hi = min(hi, nlo + step)
            lo = nlo
        return lo

    out = []
    for i in range(n - 1):
        d = 1 if delta(i, i + 1) - delta(i, i - 1) > 0 else -1
        dmin = delta(i, i - d)
        lmax = 2
        while lmax <= cap and delta(i, i + lmax * d) > dmin:
            lmax *= 2
        if lmax <= cap:  # the lane's own searches
            l, t = 0, lmax // 2
            while t >= 1:
                if delta(i, i + (l + t) * d) > dmin:
                    l += t
                t //= 2
            j = i + l * d
            dnode = delta(i, j)
            s, t = 0, l
            while True:
                t = (t + 1) // 2
                if delta(i, i + (s + t) * d) > dnode:
                    s += t
                if t <= 1:
                    break
        else:  # the warp's: lane k tests cap << k, then two narrowings
            ps = [(cap << lane) < n and delta(i, i + (cap << lane) * d) > dmin for lane in range(32)]
            top = max(lane for lane in range(32) if ps[lane])
            lo = cap << top
            l = warp_last_above(i, d, dmin, lo, min(2 * lo, n))
            j = i + l * d
            dnode = delta(i, j)
            s = warp_last_above(i, d, dnode, 0, l)
        gamma = i + s * d + min(d, 0)
        lo_, hi_ = min(i, j), max(i, j)
        left = (n - 1) + gamma if lo_ == gamma else gamma
        right = (n - 1) + gamma + 1 if hi_ == gamma + 1 else gamma + 1
        out.append((left, right, lo_, hi_, dnode))
    return [np.array(c, np.int64) for c in zip(*out)]


@pytest.mark.parametrize("cap", [2, 8, 1024])
@pytest.mark.parametrize("kind", ["random", "runs", "equal", "coarse"])
def test_warp_search_gives_the_restated_tree(cap, kind):
    rng = np.random.default_rng(cap + len(kind))
    n = 3000
    keys = {"random": rng.integers(0, 1 << 30, n),
            "runs": rng.integers(0, 16, n),
            "equal": np.zeros(n, np.int64),
            "coarse": rng.integers(0, 1 << 10, n) << 20}[kind]
    keys = np.sort(keys).astype(np.uint32)
    want = karras_numpy(keys)
    got = karras_two_path(keys, cap)
    for a, b in zip(got, want):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("n", [2, 3, 33])
def test_warp_search_tiny_inputs(n):
    keys = np.sort(np.random.default_rng(n).integers(0, 1 << 30, n)).astype(np.uint32)
    for a, b in zip(karras_two_path(keys, 2), karras_numpy(keys)):
        assert np.array_equal(a, b)
