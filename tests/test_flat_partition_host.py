"""A host model of the spread-probe walk of flat_count (dfs_device.cuh): 32
lanes each own a run of probes (an exclusive scan of their counts); the warp
walks the concatenation 32 probes at a time, every lane finds the owner of
its probe by a five-step search over the scan, and each owner adds the hits
of the ballot that fall in its own range.  The model follows the kernel's
arithmetic step for step (owner search, range masks) and must hand every
probe to exactly its owner for any distribution of counts, the empty and
lopsided ones included."""
from __future__ import annotations

import numpy as np
import pytest

FULL = 0xFFFFFFFF


def _walk(counts, hits):
    """Per-owner hit totals as the kernel computes them; hits[i] is the
    outcome of the i-th probe of the concatenation."""
    n = list(counts)
    incl, acc = [], 0
    for c in n:
        acc += c
        incl.append(acc)
    off = [incl[i] - n[i] for i in range(32)]
    total = incl[31]
    tot = [0] * 32
    for t0 in range(0, total, 32):
        ballot = 0
        for lane in range(32):
            item = t0 + lane
            c = 0
            for step in (16, 8, 4, 2, 1):  # the kernel's owner search
                if off[c + step] <= item:
                    c += step
            k = item - off[c]
            if item < total:
                assert 0 <= k < n[c], (item, c, k)  # the probe lies in its owner's run
                if hits[item]:
                    ballot |= 1 << lane
        for lane in range(32):  # each owner keeps the hits in its range
            lo, hi = max(off[lane] - t0, 0), min(off[lane] + n[lane] - t0, 32)
            if lo < hi:
                rm = ((FULL if hi == 32 else (1 << hi) - 1) & ~((1 << lo) - 1)) & FULL
                tot[lane] += bin(ballot & rm).count("1")
    return tot


@pytest.mark.parametrize("seed", range(40))
def test_every_probe_reaches_its_owner(seed):
    rng = np.random.default_rng(seed)
    kind = seed % 4
    if kind == 0:
        counts = rng.integers(0, 5, 32)
    elif kind == 1:
        counts = rng.integers(0, 200, 32)
    elif kind == 2:  # one heavy owner among idle lanes
        counts = np.zeros(32, int)
        counts[rng.integers(0, 32)] = rng.integers(1, 500)
    else:  # zeros interleaved with runs that end exactly on a 32-probe step
        counts = rng.choice([0, 32, 64, 1, 31], 32)
    counts = [int(c) for c in counts]
    total = sum(counts)
    hits = rng.random(total) < 0.37
    want, pos = [], 0
    for c in counts:
        want.append(int(hits[pos:pos + c].sum()))
        pos += c
    assert _walk(counts, hits) == want


def test_no_probes():
    assert _walk([0] * 32, np.zeros(0, bool)) == [0] * 32
