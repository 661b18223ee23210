"""FSM on the GPU: gi_fsm (through the C ABI) against the reference fsm_test
results (tests/golden/fsm.json) and against the oracle's FSM count on more
seeded labeled graphs.  Counts are integers and must be identical."""
from __future__ import annotations

import numpy as np
import pytest

import graphindor_b200 as gi
from graphindor_b200 import gen

pytestmark = pytest.mark.gpu


def test_fsm_matches_reference_fsm_test(golden_fsm, fsm_graphs):
    for name, meta in golden_fsm["graphs"].items():
        _, _, path = fsm_graphs[name]
        LG = gi.LabeledGraph.load_adj(str(path))
        for run in meta["runs"]:
            r = gi.fsm(LG, run["max_edge"], run["min_support"], golden_fsm["tri_cnt"])
            assert r.count == run["fsm_cnt"], (name, run)
            assert r.kernel_launches >= 1 or r.jobs == 0


def test_per_pattern_frequent_counts_match_oracle(golden_fsm, fsm_graphs, oracle):
    name = "lrmat_s11_l12"
    g, labels, _ = fsm_graphs[name]
    LG = gi.LabeledGraph.from_csr(g.vertex, g.edge, labels)
    G = oracle.fsm_load(g.vertex, g.edge, labels)
    for ms in (10, 40):
        r = gi.fsm(LG, 3, ms, gi.YOUTUBE_TRI_CNT)
        plans = gi.fsm_plan(3, LG.v_cnt, LG.e_cnt, gi.YOUTUBE_TRI_CNT)
        want = oracle.fsm_frequent_per_pattern(G, plans, ms)
        assert [p["frequent"] for p in r.patterns] == want
        assert r.count == sum(w for w, p in zip(want, plans) if p["edges"] == 3)


@pytest.mark.parametrize("case", range(6))
def test_fsm_matches_oracle_on_seeded_graphs(oracle, case):
    rng = np.random.default_rng(100 + case)
    scale = int(rng.integers(9, 12))
    keep = int((1 << scale) * rng.uniform(0.6, 1.0))
    n_labels = int(rng.integers(2, 9))
    g, labels = gen.labeled_rmat(scale, float(rng.uniform(4, 12)), 200 + case, keep, n_labels,
                                 float(rng.uniform(0.2, 1.5)), 300 + case)
    LG = gi.LabeledGraph.from_csr(g.vertex, g.edge, labels)
    G = oracle.fsm_load(g.vertex, g.edge, labels)
    tri = [gi.YOUTUBE_TRI_CNT, gi.PATENTS_TRI_CNT, 0][case % 3]
    max_edge = 3 if case < 5 else 4
    plans = gi.fsm_plan(max_edge, LG.v_cnt, LG.e_cnt, tri)
    for ms in (int(rng.integers(2, 30)), int(rng.integers(30, 200))):
        want = oracle.fsm_count(G, plans, max_edge, ms)
        assert gi.fsm(LG, max_edge, ms, tri).count == want, (case, ms)


def test_fsm_edge_cases(oracle):
    # Single-label graph, star, isolated pairs; max_edge 0; a support no
    # label reaches; repeated calls.
    star = gen.from_edges(33, [(0, i) for i in range(1, 33)])
    pairs = gen.from_edges(10, [(0, 1), (2, 3), (4, 5)])
    ring = gen.from_edges(12, [(i, (i + 1) % 12) for i in range(12)])
    for g in (star, pairs, ring):
        for labels in (np.zeros(g.v_cnt, np.uint32), (np.arange(g.v_cnt) % 3).astype(np.uint32)):
            LG = gi.LabeledGraph.from_csr(g.vertex, g.edge, labels)
            G = oracle.fsm_load(g.vertex, g.edge, labels)
            for me in (0, 1, 2, 3):
                plans = gi.fsm_plan(me, LG.v_cnt, LG.e_cnt, gi.YOUTUBE_TRI_CNT)
                for ms in (1, 2, 5, 1000):
                    want = oracle.fsm_count(G, plans, me, ms)
                    a = gi.fsm(LG, me, ms).count
                    assert a == want, (me, ms)
                    assert gi.fsm(LG, me, ms).count == a
    with pytest.raises(gi.GIError):
        gi.fsm(LG, 2, 0)


def test_gpu_fsm_cli_prints_the_reference_lines(fsm_graphs):
    import re
    import subprocess
    from pathlib import Path
    _, _, path = fsm_graphs["lrmat_s11_l12"]
    tool = Path(gi.__file__).resolve().parent / "bin" / "gpu_fsm"
    out = subprocess.run([str(tool), str(path), "3", "40"], capture_output=True, text=True, check=True).stdout
    want = gi.fsm(gi.LabeledGraph.load_adj(str(path)), 3, 40, gi.YOUTUBE_TRI_CNT).count
    assert int(re.search(r"fsm cnt = (\d+)", out).group(1)) == want
    assert re.search(r"Counting time cost: [\d.]+ s", out)
