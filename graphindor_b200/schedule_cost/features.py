"""Features of the learned schedule cost model: a fixed-length float32
vector per (candidate schedule, graph).  The same layout is computed in C++
by the engine (csrc/schedule_cost.cpp) when it ranks candidates."""
from __future__ import annotations

import math

import numpy as np

MAXN = 7
PAIRS = [(i, j) for i in range(MAXN) for j in range(i + 1, MAXN)]  # 21 position pairs
DEG_BINS = 16
GRAPH_DIM = 3 + DEG_BINS
PLAN_DIM = 2 * len(PAIRS) + 6
DIM = PLAN_DIM + GRAPH_DIM


def graph_features(vertex: np.ndarray, tri_cnt: int) -> np.ndarray:
    """log10 of v_cnt, edges and triangles, then the share of vertices whose
    degree falls in each power-of-two bin [2^b, 2^(b+1)) (bin 0 also holds 0)."""
    deg = np.diff(np.asarray(vertex, dtype=np.int64))
    v = len(deg)
    e = int(deg.sum()) // 2
    b = np.zeros(DEG_BINS, dtype=np.float64)
    bins = np.minimum(np.floor(np.log2(np.maximum(deg, 1))).astype(np.int64), DEG_BINS - 1)
    np.add.at(b, bins, 1.0)
    return np.concatenate([[math.log10(max(v, 1)), math.log10(max(e, 1)), math.log10(max(tri_cnt, 1))],
                           b / max(v, 1)]).astype(np.float32)


def plan_features(n: int, adj: str, order, restricts, model_cost: float, iep_k: int) -> np.ndarray:
    """Adjacency in schedule order (21 position pairs), the restriction
    pairs by position, n, edges, restriction count, IEP depth, log10 of the
    analytic model's cost and its square."""
    a = np.zeros(len(PAIRS), dtype=np.float32)
    r = np.zeros(len(PAIRS), dtype=np.float32)
    idx = {p: k for k, p in enumerate(PAIRS)}
    edges = 0
    for i in range(n):
        for j in range(i + 1, n):
            if adj[order[i] * n + order[j]] == "1":
                a[idx[(i, j)]] = 1.0
                edges += 1
    for x, y in restricts:
        i, j = min(x, y), max(x, y)
        r[idx[(i, j)]] = 1.0
    lc = math.log10(max(model_cost, 1.0))
    return np.concatenate([a, r, [n / 7.0, edges / 21.0, len(restricts) / 21.0, iep_k / 5.0, lc / 10.0,
                                  (lc / 10.0) ** 2]]).astype(np.float32)
