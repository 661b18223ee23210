"""The edge-triangle path's evaluation on the host: for plans that end at
depth 2 in an IEP tail over N(v0), N(v1) and N(v0) ∩ N(v1), the raw sum is a
function of (d(v0), d(v1), t = |N(v0) ∩ N(v1)|) per first-level edge.  This
restates tri_edge.cu's per-edge evaluation (the chain-1 break-size prunes,
the sets' sizes and embedded counts, the IEP formula) in Python and checks
it against the oracle's DFS count (a restatement of the reference CPU path)
on seeded graphs, so the formula the kernel evaluates is pinned on CPU."""
from __future__ import annotations

import numpy as np
import pytest

import graphindor_b200 as gi
from graphindor_b200 import gen
from conftest import plan_desc

M64 = (1 << 64) - 1


def _adj(n, edges):
    m = [[0] * n for _ in range(n)]
    for a, b in edges:
        m[a][b] = m[b][a] = 1
    return "".join(str(m[i][j]) for i in range(n) for j in range(n))


PATTERNS = [(4, "0111101111001100"),  # diamond
            (5, _adj(5, [(0, 1), (0, 2), (1, 2), (0, 3), (1, 3), (0, 4), (1, 4)])),  # 3-book
            (6, _adj(6, [(0, 1)] + [(0, k) for k in range(2, 6)] + [(1, k) for k in range(2, 6)])),  # 4-book
            (4, _adj(4, [(0, 1), (1, 2), (0, 2), (0, 3)]))]  # tailed triangle


def _eligible(e):
    """The plan qualifies for the edge-triangle path (capi_plan.cpp)."""
    n, k = e["size"], e["in_exclusion_optimize_num"]
    if k == 0 or n - k != 2 or e["is_vertex_induced"]:
        return False
    father, depth = e["father_prefix_id"], [p[-1] for p in e["prefix_data"]]
    for p in range(e["total_prefix_num"]):
        f = father[p]
        if depth[p] == 0 and f != -1:
            return False
        if depth[p] == 1 and f != -1 and (depth[f] != 0 or father[f] != -1):
            return False
    return True


def _iep_combine(e, ans):
    acc, val, last_pos = 0, 0, -1
    for pos, (coef, flag, ap) in enumerate(zip(e["iep_coef"], e["iep_flag"], e["iep_ans_pos_eff"])):
        a = ans[ap] & M64
        if pos == last_pos + 1:
            val = a
        elif val != 0:
            val = (val * a) & M64
        if flag:
            last_pos = pos
            acc = (acc + val * (coef & M64)) & M64
    return acc


def _edge_triangle_raw(e, g):
    father, depth = e["father_prefix_id"], [p[-1] for p in e["prefix_data"]]
    restricted = e["restrict_last"][1] != -1
    chain1, p = [], e["last"][1]
    while p != -1:
        chain1.append(p)
        p = e["next"][p]
    loop2 = e["loop_set_prefix_id"][2]
    nbr = [g.edge[g.vertex[v]:g.vertex[v + 1]] for v in range(g.v_cnt)]
    raw = 0
    for v0 in range(g.v_cnt):
        for v1 in nbr[v0]:
            v1 = int(v1)
            if restricted and v0 <= v1:
                continue
            d0, d1 = len(nbr[v0]), len(nbr[v1])
            t = len(np.intersect1d(nbr[v0], nbr[v1], assume_unique=True))
            size = lambda q: d0 if depth[q] == 0 else d1 if father[q] == -1 else t  # noqa: E731
            if any(size(q) == e["break_size"][q] for q in chain1):
                continue
            if size(loop2) <= 0:
                continue
            ans = []
            for q, flag, coef in zip(e["iep_vertex_id"], e["iep_vertex_flag_eff"], e["iep_vertex_coef_eff"]):
                emb = 1 if depth[q] == 0 or father[q] == -1 else 0
                ans.append(size(q) - coef if flag else size(q) - emb)
            raw = (raw + _iep_combine(e, ans)) & M64
    return raw


@pytest.mark.parametrize("which", range(4))
def test_edge_triangle_evaluation_equals_the_oracle_count(oracle, which):
    n, adj = PATTERNS[which]
    for g in (gen.erdos_renyi(120, 900, 51 + which), gen.rmat(8, 8.0, 61 + which)):
        s = gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, 0)
        e = s.export()
        assert _eligible(e), adj
        want, _ = oracle.count(plan_desc(s), g.vertex, g.edge)
        assert _edge_triangle_raw(e, g) == want, adj


def test_eligibility_matches_the_engine():
    # The variant reads back as set exactly when the plan qualifies.
    for n, adj in PATTERNS + [(4, "0110100110010110"), (3, "011101110"), (5, "0111110111110111110111110")]:
        s = gi.Schedule_IEP(gi.Pattern(n, adj), 1 << 12, 1 << 16, 1 << 14)
        s.variant = {"edge_triangles": 1}
        assert bool(s.variant["edge_triangles"]) == _eligible(s.export()), adj
