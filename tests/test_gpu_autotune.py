"""The autotuner (gi_autotune) and kernel variants on the GPU: every
variant of a plan counts exactly what the default does (the raw sums are
integers and must be identical), the tuner keeps one of the variants it
timed and caches it per class of (plan, graph), and a batch built after
tuning applies the cached variants and still counts what single counts do."""
from __future__ import annotations

import pytest

import graphindor_b200 as gi
from graphindor_b200 import gen

pytestmark = pytest.mark.gpu

PATTERNS = [(4, "0111101111001100"), (4, "0110100110010110"), (5, "0101110101010101010011000"),
            (5, "0111110111110111110111110"), (6, "011100101010110001100011010101001110"), (3, "011101110")]


def test_every_variant_counts_the_same():
    g = gen.rmat(12, 12.0, 31)
    dg = gi.Graph.from_csr(g.vertex, g.edge)
    for n, adj in PATTERNS:
        s = gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, 0)
        want = gi.pattern_matching(dg, s).raw_sum
        for flat in (0, 1):
            for budget in (64, 256, 2048):
                for occ in (0, 1, 16):
                    s.variant = {"leaf_flat": flat, "lane_budget": budget, "occupancy": occ}
                    assert gi.pattern_matching(dg, s).raw_sum == want, (adj, flat, budget, occ)
        for split, lh, mh in ((1, 1, 1), (8, 16, 2), (1024, 256, 64)):
            s.variant = {"split": split, "leaf_handoff": lh, "mid_handoff": mh}
            assert gi.pattern_matching(dg, s).raw_sum == want, (adj, split, lh, mh)
        # Edge subsets too (the tuner's sample).
        s.variant = {"leaf_flat": 1, "occupancy": 16}
        tot = sum(gi.count_edges(dg, s, 5, off).raw_sum for off in range(5)) % (1 << 64)
        assert tot == want


def test_tuner_picks_a_timed_variant_and_caches_it():
    gi.autotune_clear()
    g = gen.rmat(13, 10.0, 32)
    dg = gi.Graph.from_csr(g.vertex, g.edge)
    for n, adj in PATTERNS[:4]:
        s = gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, 0)
        want = gi.pattern_matching(dg, s).raw_sum
        info = gi.autotune(dg, s, sample_edges=4096)
        assert not info["cached"] and 6 <= info["candidates"] <= 10
        assert info["best_ms"] > 0 and info["best_ms"] <= info["default_ms"] + 1e-9
        assert s.variant == info["chosen"]
        assert gi.pattern_matching(dg, s).raw_sum == want
        s2 = gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, 0)
        again = gi.autotune(dg, s2)
        assert again["cached"] and again["chosen"] == info["chosen"]


def test_batch_applies_tuned_variants():
    gi.autotune_clear()
    graphs = [gen.rmat(11, 8.0, 40), gen.rmat(12, 14.0, 41)]
    dgs = [gi.Graph.from_csr(g.vertex, g.edge) for g in graphs]
    jobs, want = [], []
    for dg, g in zip(dgs, graphs):
        for n, adj in PATTERNS:
            s = gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, 0)
            want.append(gi.pattern_matching(dg, s).count)
            gi.autotune(dg, s, sample_edges=2048)
            jobs.append((dg, s))
    b = gi.Batch(jobs)
    for _ in range(2):  # capture, then replay
        counts, lat, _ = b.run()
        assert counts == want
        assert all(x >= 0 for x in lat)


def test_membership_structures_do_not_change_counts(monkeypatch):
    # The same graph with neither hub bitmaps nor hash sets, with hash sets
    # only, and with both (a low hub threshold): every count and every
    # variant gives the same raw sum.
    g = gen.rmat(12, 16.0, 33)
    graphs = []
    for hub_mb, hash_mb in ((0, 0), (0, 4096), (64, 4096)):
        monkeypatch.setenv("GI_HUB_BITMAP_MB", str(hub_mb))
        monkeypatch.setenv("GI_HUB_MIN_DEGREE", "16")
        monkeypatch.setenv("GI_HASH_MB", str(hash_mb))
        dg = gi.Graph.from_csr(g.vertex, g.edge)
        graphs.append(dg)
    assert graphs[0].n_hubs == 0 and graphs[0].hash_slots == 0
    assert graphs[1].n_hubs == 0 and graphs[1].hash_slots > 0 and graphs[1].hash_min_degree == 32
    assert graphs[2].n_hubs > 0 and graphs[2].hash_slots > 0
    for n, adj in PATTERNS:
        s = gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, 0)
        want = gi.pattern_matching(graphs[0], s).raw_sum
        for flat in (0, 1):
            s.variant = {"leaf_flat": flat}
            for dg in graphs:
                assert gi.pattern_matching(dg, s).raw_sum == want, (adj, flat)


def _adj(n, edges):
    m = [[0] * n for _ in range(n)]
    for a, b in edges:
        m[a][b] = m[b][a] = 1
    return "".join(str(m[i][j]) for i in range(n) for j in range(n))


# Plans that end at depth 2 in an IEP tail over N(v0), N(v1), N(v0) ∩ N(v1).
EDGE_TRIANGLE_PATTERNS = [(4, "0111101111001100"),  # diamond
                          (5, _adj(5, [(0, 1), (0, 2), (1, 2), (0, 3), (1, 3), (0, 4), (1, 4)])),  # 3-book
                          (6, _adj(6, [(0, 1)] + [(0, k) for k in range(2, 6)] + [(1, k) for k in range(2, 6)])),
                          (4, _adj(4, [(0, 1), (1, 2), (0, 2), (0, 3)]))]  # tailed triangle


def test_edge_triangle_path_counts_like_the_dfs():
    for g in (gen.rmat(12, 16.0, 34), gen.chung_lu(3000, 60000, 2.0, 800.0, 35), gen.erdos_renyi(500, 9000, 36)):
        dg = gi.Graph.from_csr(g.vertex, g.edge)
        for n, adj in EDGE_TRIANGLE_PATTERNS:
            s = gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, 0)
            want = gi.pattern_matching(dg, s)
            subsets = [gi.count_edges(dg, s, 7, off).raw_sum for off in (0, 3, 6)]
            shards = [gi.count_edges(dg, s, 3, 1, shard=k, num_shards=2).raw_sum for k in (0, 1)]
            s.variant = {"edge_triangles": 1}
            assert s.variant["edge_triangles"] == 1
            got = gi.pattern_matching(dg, s)
            assert (got.raw_sum, got.count, got.tasks) == (want.raw_sum, want.count, want.tasks), adj
            assert [gi.count_edges(dg, s, 7, off).raw_sum for off in (0, 3, 6)] == subsets, adj
            assert [gi.count_edges(dg, s, 3, 1, shard=k, num_shards=2).raw_sum for k in (0, 1)] == shards, adj
    # A plan that does not qualify keeps the general kernel.
    s = gi.Schedule_IEP(gi.Pattern(4, "0110100110010110"), 100, 1000, 0)
    s.variant = {"edge_triangles": 1}
    assert s.variant["edge_triangles"] == 0
