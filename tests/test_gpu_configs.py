"""GPU parity at the workloads' stated sizes: the engine through the C ABI
against the reference's own outputs recorded in tests/golden/configs.json
(written by tests/golden/make_configs.py from the reference binaries, or, for
5- and 6-cliques of the 3.07M-vertex graph, from the oracle's clique-tree
pivoting counter).  Every graph is regenerated from its seeded parameters
and checked against its recorded sha1 first.  Counts are integers and must
be bit-identical."""
from __future__ import annotations

import hashlib
import json

import pytest

import graphindor_b200 as gi
from graphindor_b200 import gen
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

WORKLOAD = {"diamond": (4, "0111101111001100"), "4-cycle": (4, "0110100110010110"),
            "house": (5, "0101110101010101010011000"), "5-clique": (5, "0111110111110111110111110"),
            "prism": (6, "011100101010110001100011010101001110"),
            "6-cycle+chord": (6, "010101101000010100101010000101100010")}


@pytest.fixture(scope="module")
def configs():
    path = GOLDEN / "configs.json"
    return json.loads(path.read_text()) if path.exists() else {}


def _section(configs, name):
    if name not in configs:
        pytest.skip(f"configs.json has no {name} section")
    return configs[name]


def _sha1(g) -> str:
    h = hashlib.sha1()
    h.update(g.vertex.tobytes())
    h.update(g.edge.tobytes())
    return h.hexdigest()


def _check_subsets(dg, tri, rows_by_pattern):
    """Raw sums of the reference's per-edge task over edge subsets, and the
    reference's redundancy, against the engine's edge-subset counts."""
    for name, rows in rows_by_pattern.items():
        n, adj = WORKLOAD[name]
        s = gi.Schedule_IEP(gi.Pattern(n, adj), dg.v_cnt, dg.e_cnt, tri)
        assert s.export()["redundancy"] == rows[0]["redundancy"], name
        for r in rows:
            st = gi.count_edges(dg, s, r["step"], r["offset"])
            assert st.raw_sum == r["raw"], (name, r)


def test_config1_triangles_and_4_cliques(configs):
    c = _section(configs, "c1")
    g = gen.rmat(**c["params"])
    assert _sha1(g) == c["sha1"]
    dg = gi.Graph.from_csr(g.vertex, g.edge)
    for k, want in c["cliques"].items():
        k = int(k)
        assert gi.clique_count(dg, k, 0).count == want, k  # gpu_clique: id orientation
        assert gi.clique_count(dg, k, 1).count == want, k  # gpu_kclique: degree orientation
        s = gi.Schedule_IEP(gi.Pattern.clique(k), g.v_cnt, g.e_cnt, 0)
        assert gi.pattern_matching(dg, s).count == want, k  # gpu_graph with the clique's adjacency
        assert gi.clique_counts_pivot(dg, k)[k] == want, k


def test_config2_patterns_on_edge_subsets_of_a_moderate_graph(configs):
    c = _section(configs, "c2")["moderate"]
    g = gen.rmat(**c["params"])
    assert _sha1(g) == c["sha1"]
    dg = gi.Graph.from_csr(g.vertex, g.edge, tri_cnt=c["tri_cnt"])
    _check_subsets(dg, c["tri_cnt"], c["subsets"])
    # The subsets of one step add up (mod 2^64) to the whole count.
    n, adj = WORKLOAD["house"]
    s = gi.Schedule_IEP(gi.Pattern(n, adj), dg.v_cnt, dg.e_cnt, c["tri_cnt"])
    total = sum(gi.count_edges(dg, s, 7, off).raw_sum for off in range(7)) % (1 << 64)
    assert total == gi.pattern_matching(dg, s).raw_sum


@pytest.fixture(scope="module")
def s22(configs):
    c = _section(configs, "c2")["s22"]
    g = gen.rmat(**c["params"])
    assert _sha1(g) == c["sha1"]
    return c, gi.Graph.from_csr(g.vertex, g.edge, tri_cnt=c["tri_cnt"])


def test_config2_whole_diamond_count_at_scale_22(s22):
    c, dg = s22
    w = c["diamond_whole"]
    n, adj = WORKLOAD["diamond"]
    s = gi.Schedule_IEP(gi.Pattern(n, adj), dg.v_cnt, dg.e_cnt, c["tri_cnt"])
    r = gi.pattern_matching(dg, s)
    assert r.raw_sum == w["raw"]
    assert r.count == w["raw"] // w["redundancy"]


def test_config2_bench_sample_at_scale_22(configs, s22):
    """The six patterns over exactly the edge subsets bench.py times."""
    c = _section(configs, "c2_sample")
    c22, dg = s22
    assert c["sha1"] == c22["sha1"]
    _check_subsets(dg, c["tri_cnt"], c["subsets"])


def test_config3_cliques_on_the_chung_lu_graph(configs):
    c = _section(configs, "c3_cliques")
    g = gen.chung_lu(**c["params"])
    assert _sha1(g) == c["sha1"]
    dg = gi.Graph.from_csr(g.vertex, g.edge)
    del g
    want = {int(k): v for k, v in c["cliques"].items()}
    for k in (3, 4, 5):
        assert gi.clique_count(dg, k, 1).count == want[k], k
    piv = gi.clique_counts_pivot(dg, max(want))
    for k, v in want.items():
        assert piv[k] == v, k


def test_config3_fsm(configs, tmp_path):
    c = _section(configs, "c3_fsm")
    g, labels = gen.labeled_rmat(**c["params"])
    path = tmp_path / "fsm.adj"
    gen.write_adj(str(path), g, labels)
    assert hashlib.sha1(path.read_bytes()).hexdigest() == c["adj_sha1"]
    lg = gi.LabeledGraph.from_csr(g.vertex, g.edge, labels)
    for r in c["runs"]:
        # fsm_test plans with the Patents triangle count (reference src/fsm_test.cpp:27).
        assert gi.fsm(lg, r["max_edge"], r["min_support"], tri_cnt=7515023).count == r["fsm_cnt"], r
