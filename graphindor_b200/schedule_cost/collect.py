"""Times candidate schedules on the GPU: the training data of the learned
schedule cost model (train.py).

For three seeded graphs (R-MAT, Chung-Lu, Erdos-Renyi) and a seeded set of
connected 5-, 6- and 7-vertex patterns (MotifGenerator order), the valid
candidates of each pattern (order + restriction set that counts every
subgraph equally often, analytic cost from the reference model) are ranked by
analytic cost; up to eight are timed with gi_count (CUDA events, device time
of the work split and the counting kernel) under a device budget.  Every
valid candidate of a pattern must return the same count: the collector
records any disagreement.

    python -m graphindor_b200.schedule_cost.collect --out runs.json [--budget-ms 400] [--max-s 420]
        [--light] [--graphs name,name]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import random
import time

import numpy as np

from .. import Graph, Pattern, Schedule_IEP, lib, motif_patterns
from .. import _native as N
from .. import gen
from .features import graph_features

GRAPHS = {
    "rmat_s15_ef16": lambda: gen.rmat(15, 16.0, 7),
    "chunglu_50k": lambda: gen.chung_lu(50000, 600000, 2.1, 2000.0, 8),
    "er_50k": lambda: gen.erdos_renyi(50000, 800000, 9),
}
# Smaller graphs of the same three families: most candidates finish in budget.
LIGHT_GRAPHS = {
    "rmat_s12_ef12": lambda: gen.rmat(12, 12.0, 7),
    "chunglu_20k": lambda: gen.chung_lu(20000, 160000, 2.1, 600.0, 8),
    "er_20k": lambda: gen.erdos_renyi(20000, 200000, 9),
}


def random_connected(n: int, density: float, rng: random.Random) -> str:
    """A seeded random connected n-vertex pattern (edge probability `density`)."""
    while True:
        adj = [[0] * n for _ in range(n)]
        for i in range(n):
            for j in range(i + 1, n):
                if rng.random() < density:
                    adj[i][j] = adj[j][i] = 1
        seen, todo = {0}, [0]
        while todo:
            u = todo.pop()
            for v in range(n):
                if adj[u][v] and v not in seen:
                    seen.add(v)
                    todo.append(v)
        if len(seen) == n:
            return "".join(str(adj[i][j]) for i in range(n) for j in range(n))


def pattern_set(seed: int = 5):
    """All 21 connected 5-vertex patterns, 40 of the 112 6-vertex ones and
    20 random connected 7-vertex patterns (density 0.4 - 0.8)."""
    rng = random.Random(seed)
    pats = [(5, a) for a in motif_patterns(5)]
    pats += [(6, a) for a in rng.sample(motif_patterns(6), 40)]
    pats += [(7, random_connected(7, rng.uniform(0.4, 0.8), rng)) for _ in range(20)]
    return pats


def pick(cands, k: int = 8):
    valid = sorted([c for c in cands if c[3] > 0], key=lambda c: c[2])
    out, seen = [], set()
    head = valid[: k // 2]
    rest = valid[k // 2:]
    step = max(1, len(rest) // max(1, k - len(head)))
    for c in head + rest[::step]:
        key = (tuple(c[0]), tuple(map(tuple, c[1])))
        if key not in seen and len(out) < k:
            seen.add(key)
            out.append(c)
    return out


def time_plan(g: Graph, s: Schedule_IEP, budget_ms: float):
    st = N.Stats()
    st.budget_ms = budget_ms
    out = C.c_uint64()
    rc = lib().gi_count(g.handle, s.handle, None, C.byref(out), C.byref(st))
    if rc == N.GI_ETIMEOUT:
        return None, None
    N.check(rc, "gi_count")
    return st.kernel_ms + st.prep_ms, out.value


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--budget-ms", type=float, default=400.0)
    ap.add_argument("--max-s", type=float, default=420.0)
    ap.add_argument("--light", action="store_true", help="the smaller graph set")
    ap.add_argument("--graphs", default="", help="comma-separated graph names to time (default: all of the set)")
    a = ap.parse_args()
    t_start = time.time()
    pats = pattern_set()
    runs = {"budget_ms": a.budget_ms, "graphs": {}, "rows": []}
    chosen = set(filter(None, a.graphs.split(",")))
    for gname, make in (LIGHT_GRAPHS if a.light else GRAPHS).items():
        if chosen and gname not in chosen:
            continue
        g = make()
        dg = Graph.from_csr(g.vertex, g.edge)
        from .. import clique_count
        tri = clique_count(dg, 3, 1).count
        dg = Graph.from_csr(g.vertex, g.edge, tri_cnt=tri)
        runs["graphs"][gname] = {"v_cnt": g.v_cnt, "e_cnt": g.e_cnt, "tri_cnt": tri,
                                 "features": graph_features(g.vertex, tri).tolist()}
        for n, adj in pats:
            if time.time() - t_start > a.max_s:
                break
            p = Pattern(n, adj)
            cands = pick(Schedule_IEP.candidates(p, g.v_cnt, g.e_cnt, tri))
            counts = set()
            for i, (order, rs, cost, div) in enumerate(cands):
                s = Schedule_IEP(p, order=order, restricts=rs)
                if i == 0:
                    time_plan(dg, s, a.budget_ms)  # warm-up of the pattern's first plan
                ms, cnt = time_plan(dg, s, a.budget_ms)
                if cnt is not None:
                    counts.add(cnt)
                runs["rows"].append({"graph": gname, "n": n, "adj": adj, "order": order, "restricts": rs,
                                     "model_cost": cost, "divisor": div, "iep_k": s.export()["in_exclusion_optimize_num"],
                                     "ms": ms, "count": cnt})
                if ms is None and i == 0:
                    break  # the cheapest-by-model candidate already exceeds the budget
            if len(counts) > 1:
                runs.setdefault("count_mismatch", []).append({"graph": gname, "adj": adj, "counts": sorted(counts)})
            print(gname, n, adj, len(cands), f"{time.time() - t_start:.0f}s", flush=True)
            with open(a.out, "w") as f:  # after every pattern: a cut-short run keeps what it measured
                json.dump(runs, f)
    with open(a.out, "w") as f:
        json.dump(runs, f)


if __name__ == "__main__":
    main()
