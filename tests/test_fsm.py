"""FSM on the CPU: the engine's FSM plans and labeled loader against the
reference planner's FSM schedules and the oracle's loader restatement; the
oracle's FSM count (oracle/oracle.c, oracle_fsm_support) pinned against the
reference fsm_test results in tests/golden/fsm.json."""
from __future__ import annotations

import numpy as np
import pytest

import graphindor_b200 as gi
from graphindor_b200 import gen


def test_fsm_plans_match_reference_planner(golden_fsm):
    for name, meta in golden_fsm["graphs"].items():
        max_me = max(r["max_edge"] for r in meta["runs"])
        ours = gi.fsm_plan(max_me, meta["v_cnt"], meta["e_cnt"], golden_fsm["tri_cnt"])
        ref = meta["plans"]
        assert len(ours) == len(ref), name
        for o, r in zip(ours, ref):
            assert (o["n"], o["edges"], o["adj"]) == (r["n"], r["edges"], r["adj"]), name
            assert [list(x) for x in o["restricts"]] == r["restricts"], (name, r["adj"])


def test_oracle_fsm_matches_reference_fsm_test(golden_fsm, fsm_graphs, oracle):
    for name, meta in golden_fsm["graphs"].items():
        g, labels, _ = fsm_graphs[name]
        G = oracle.fsm_load(g.vertex, g.edge, labels)
        for run in meta["runs"]:
            if run["max_edge"] > 3 and G["v_cnt"] > 1000:
                continue
            got = oracle.fsm_count(G, meta["plans"], run["max_edge"], run["min_support"])
            assert got == run["fsm_cnt"], (name, run)


def test_labeled_loader_matches_oracle_restatement(golden_fsm, fsm_graphs, oracle):
    for name, (g, labels, path) in fsm_graphs.items():
        G = oracle.fsm_load(g.vertex, g.edge, labels)
        for LG in (gi.LabeledGraph.from_csr(g.vertex, g.edge, labels), gi.LabeledGraph.load_adj(str(path))):
            assert (LG.v_cnt, LG.e_cnt, LG.l_cnt) == (G["v_cnt"], G["e_cnt"], G["l_cnt"])
            ex = LG.export()
            if G["l_cnt"] <= 16:  # the reference's std::sort is an insertion sort, stable, up to 16 labels
                for k in ("new_id", "v_label", "label_value", "label_start", "bucket", "edge"):
                    assert np.array_equal(ex[k].astype(np.int64), G[k].astype(np.int64)), (name, k)
            # Structure that holds whatever the tie order: label ranges are
            # contiguous and by descending max degree, buckets partition the
            # neighbour lists and each bucket is sorted.
            v_label, ls, bucket, edge = ex["v_label"], ex["label_start"], ex["bucket"], ex["edge"]
            assert np.all(np.diff(v_label) >= 0)
            assert np.array_equal(np.bincount(v_label, minlength=LG.l_cnt), np.diff(ls.astype(np.int64)))
            assert bucket[-1] == LG.e_cnt and np.all(np.diff(bucket.astype(np.int64)) >= 0)
            L = LG.l_cnt
            for v in range(0, LG.v_cnt, 97):
                for l in range(L):
                    seg = edge[bucket[v * L + l]:bucket[v * L + l + 1]]
                    assert np.all(np.diff(seg.astype(np.int64)) > 0)
                    assert np.all(v_label[seg] == l)


def test_loader_rejects_bad_input(native):
    vertex = np.array([0, 1, 1], dtype=np.int64)
    edge = np.array([1], dtype=np.int32)  # 0 -> 1 without 1 -> 0
    with pytest.raises(gi.GIError):
        gi.LabeledGraph.from_csr(vertex, edge, np.array([0, 1], dtype=np.uint32))
    edge = np.array([5], dtype=np.int32)
    with pytest.raises(gi.GIError):
        gi.LabeledGraph.from_csr(vertex, edge, np.array([0, 1], dtype=np.uint32))


def test_loader_skips_self_loops_and_uses_line_order(tmp_path, native, oracle):
    # Vertex lines out of id order: labels are first seen in line order.
    text = "4\n2 9 1 3 2\n0 7 1\n1 9 0 2\n3 7 2\n"
    p = tmp_path / "x.adj"
    p.write_text(text)
    LG = gi.LabeledGraph.load_adj(str(p))
    assert (LG.v_cnt, LG.e_cnt, LG.l_cnt) == (4, 6, 2)
    vertex = np.array([0, 1, 3, 6, 7], dtype=np.int64)
    edge = np.array([1, 0, 2, 1, 3, 2, 2], dtype=np.int32)
    labels = np.array([7, 9, 9, 7], dtype=np.uint32)
    G = oracle.fsm_load(vertex, edge, labels, order=[2, 0, 1, 3])
    ex = LG.export()
    for k in ("new_id", "v_label", "label_value", "label_start", "bucket", "edge"):
        assert np.array_equal(ex[k].astype(np.int64), G[k].astype(np.int64)), k


def test_fsm_plan_counts_patterns():
    # Connected patterns with at most e edges and at least one edge.
    assert [len(gi.fsm_plan(e, 1000, 8000)) for e in (1, 2, 3, 4)] == [1, 2, 5, 10]
    with pytest.raises(gi.GIError):
        gi.fsm_plan(7, 1000, 8000)


def _canon(n, adj):
    import itertools
    best = None
    for p in itertools.permutations(range(n)):
        key = tuple(adj[p[i] * n + p[j]] for i in range(n) for j in range(i + 1, n))
        if best is None or key > best:
            best = key
    return best


def test_fsm_pattern_list_for_six_edges_matches_the_filtered_motif_lists():
    """FSM enumerates motifs with an edge cap; the kept patterns, in order,
    must be those of the full MotifGenerator lists filtered by edge count."""
    plans = gi.fsm_plan(6, 50000, 1000000)
    want = [(2, "0110")]
    for k in range(3, 8):
        for a in (gi.motif_patterns(k) if k < 7 else []):
            if sum(a[i * k + j] == "1" for i in range(k) for j in range(i + 1, k)) <= 6:
                want.append((k, a))
    got7 = [p for p in plans if p["n"] == 7]
    assert len(got7) == 11  # the trees on 7 vertices
    got = [p for p in plans if p["n"] < 7]
    want_e = sorted(want, key=lambda t: sum(t[1][i * t[0] + j] == "1" for i in range(t[0]) for j in range(i + 1, t[0])))
    assert [(p["n"], _canon(p["n"], p["adj"])) for p in got] == [(n, _canon(n, a)) for n, a in want_e]
