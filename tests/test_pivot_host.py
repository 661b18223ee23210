"""The clique-tree pivoting search of the GPU kernel (csrc/pivot.cuh), built
for the host as one lane, over bitmaps laid out as the k-clique bitmap
kernels (csrc/kclique.cu) lay them out, against the host oracle's
independent pivoting counter, its enumerating counter and C(n, k)."""
from __future__ import annotations

import ctypes as C
import subprocess
from math import comb
from pathlib import Path

import numpy as np
import pytest

from graphindor_b200 import gen

HERE = Path(__file__).resolve().parent


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    so = tmp_path_factory.mktemp("pivot") / "libpivot_host.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-Wall", "-o", str(so),
                    str(HERE / "pivot_host_harness.cpp")], check=True)
    L = C.CDLL(str(so))
    L.pivot_host_counts.restype = C.c_int
    L.pivot_host_counts.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    return L


def _dag_bitmaps(g):
    """Degree-oriented DAG (arc u -> v when (deg u, u) < (deg v, v)), out-lists
    in id order, and per-vertex bitmaps: ceil(d / 32) words a row, row i bit j
    when out-neighbour j is an out-neighbour of out-neighbour i."""
    deg = np.diff(g.vertex)
    outs = []
    for u in range(g.v_cnt):
        nb = g.edge[g.vertex[u]:g.vertex[u + 1]]
        keep = (deg[nb] > deg[u]) | ((deg[nb] == deg[u]) & (nb > u))
        outs.append(np.sort(nb[keep]).astype(np.int64))
    dvertex = np.zeros(g.v_cnt + 1, dtype=np.int64)
    dvertex[1:] = np.cumsum([len(o) for o in outs])
    words = np.array([len(o) * ((len(o) + 31) // 32) if len(o) >= 2 else 0 for o in outs], dtype=np.int64)
    off = np.zeros(g.v_cnt + 1, dtype=np.int64)
    off[1:] = np.cumsum(words)
    bitmap = np.zeros(max(int(off[-1]), 1), dtype=np.uint32)
    weights = (np.uint64(1) << np.arange(32, dtype=np.uint64))
    for u, o in enumerate(outs):
        d = len(o)
        if d < 2:
            continue
        W = (d + 31) // 32
        for i, v in enumerate(o):
            hit = np.zeros(W * 32, dtype=np.uint64)
            hit[:d] = np.isin(o, outs[int(v)])
            words = (hit.reshape(W, 32) * weights).sum(axis=1).astype(np.uint32)
            bitmap[off[u] + i * W: off[u] + (i + 1) * W] = words
    return dvertex, off, bitmap


def _counts(L, g, kmax, levels=256):
    dvertex, off, bitmap = _dag_bitmaps(g)
    out = np.zeros(kmax + 1, dtype=np.uint64)
    rc = L.pivot_host_counts(dvertex.ctypes.data, g.v_cnt, off.ctypes.data, bitmap.ctypes.data, kmax, levels,
                             out.ctypes.data)
    return rc, [int(x) for x in out]


def test_host_build_matches_the_oracles(harness, oracle):
    # The last graph has out-degrees above 64 (rows of three or more words).
    for g in (gen.erdos_renyi(300, 4000, 1), gen.rmat(9, 8.0, 11), gen.chung_lu(1500, 12000, 2.2, 150.0, 14),
              gen.chung_lu(3000, 90000, 1.9, 900.0, 17)):
        want = oracle.clique_counts_pivot(7, g.vertex, g.edge)
        for kmax in (1, 2, 3, 4, 5, 7):
            rc, got = _counts(harness, g, kmax)
            assert rc == 0
            assert got[1:] == want[1:kmax + 1], (kmax, got, want)
        assert want[3:6] == [oracle.cliques(k, g.vertex, g.edge) for k in range(3, 6)]


def test_host_build_on_complete_graphs_and_stack_limit(harness):
    # 70 vertices: rows of three 32-bit words; a pendant path hangs off it.
    k70 = gen.from_edges(73, [(i, j) for i in range(70) for j in range(i + 1, 70)] + [(69, 70), (70, 71), (71, 72)])
    rc, got = _counts(harness, k70, 7)
    want = [comb(70, k) for k in range(1, 8)]
    want[0] += 3
    want[1] += 3
    assert rc == 0 and got[1:] == want
    # A stack shallower than the search reports it instead of counting.
    rc, _ = _counts(harness, k70, 7, levels=2)
    assert rc == -1
