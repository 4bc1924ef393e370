"""The kNN kernels' fixed networks, checked on the host from the CUDA source.

A lane's top-k set (KMAX = 10, 15 or 16 slots) is sorted by Batcher's
odd-even merge sort network on 16 inputs, with the comparators that touch a
slot at or above KMAX left out (those slots count as +infinity).  The network
is a table in dwg_b200/csrc/knn.cu; here it is read back and run on seeded
inputs with repeated values, and its comparator count and depth are checked
against the construction.  The tournament that finds a full set's maximum
must return the lowest slot among equal keys, as a scan from slot 0 with a
strict comparison does; its recursion is restated and compared.
"""
import os
import re

import numpy as np

SRC = os.path.join(os.path.dirname(__file__), "..", "dwg_b200", "csrc", "knn.cu")


def _table(name):
    s = open(SRC).read()
    m = re.search(r"constexpr unsigned char %s\[kSortNet\] = \{([^}]*)\};" % name, s)
    assert m, name
    return [int(v) for v in m.group(1).split(",")]


def _batcher(n):
    """the iterative odd-even merge sort construction"""
    out = []
    p = 1
    while p < n:
        d = p
        while d >= 1:
            j = d % p
            while j + d < n:
                for i in range(d):
                    if i + j + d < n and (i + j) // (2 * p) == (i + j + d) // (2 * p):
                        out.append((i + j, i + j + d))
                j += 2 * d
            d //= 2
        p *= 2
    return out


def test_sort_table_is_the_batcher_network():
    lo, hi = _table("kSortLo"), _table("kSortHi")
    assert list(zip(lo, hi)) == _batcher(16)
    assert len(lo) == 63 and all(a < b for a, b in zip(lo, hi))
    # depth 10: comparators placed greedily in layers
    layer = [0] * 16
    for a, b in zip(lo, hi):
        layer[a] = layer[b] = max(layer[a], layer[b]) + 1
    assert max(layer) == 10


def test_sort_network_sorts_every_slot_count():
    net = list(zip(_table("kSortLo"), _table("kSortHi")))
    rng = np.random.default_rng(21)
    for kmax, expect in ((10, 32), (15, 59), (16, 63)):
        kept = [(a, b) for a, b in net if b < kmax]
        assert len(kept) == expect
        for _ in range(3000):
            v = list(rng.integers(0, 12, kmax))  # many repeats
            for a, b in kept:
                if v[b] < v[a]:
                    v[a], v[b] = v[b], v[a]
            assert v == sorted(v)
        # every 0/1 input (the 0-1 principle: a network that sorts all 0/1
        # inputs sorts every input)
        for bits in range(1 << kmax) if kmax <= 10 else rng.integers(0, 1 << kmax, 20000):
            v = [(int(bits) >> t) & 1 for t in range(kmax)]
            for a, b in kept:
                if v[b] < v[a]:
                    v[a], v[b] = v[b], v[a]
            assert v == sorted(v)


def _tour_max(v, lo, n):
    """tour_max<LO, N> of knn.cu: halves of N // 2 and N - N // 2, the right
    one taken only when strictly larger"""
    if n == 1:
        return v[lo], lo
    m1, p1 = _tour_max(v, lo, n // 2)
    m2, p2 = _tour_max(v, lo + n // 2, n - n // 2)
    return (m2, p2) if m2 > m1 else (m1, p1)


def test_tournament_maximum_takes_the_scan_slot():
    assert "const bool r = m2 > m1;" in open(SRC).read()
    rng = np.random.default_rng(22)
    for n in (10, 15, 16):
        for _ in range(5000):
            v = list(rng.integers(0, 6, n))
            m, p = _tour_max(v, 0, n)
            assert m == max(v) and p == v.index(max(v))
