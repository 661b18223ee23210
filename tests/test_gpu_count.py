"""GPU parity: the CUDA engine (through the C ABI) against the reference's
own outputs (golden counts from the reference binaries) and the oracle
(oracle/oracle.c) on the same seeded inputs.  Counts are integers and must
be bit-identical."""
from __future__ import annotations

import ctypes as C
import random

import numpy as np
import pytest

import graphindor_b200 as gi
from graphindor_b200 import _native as N
from graphindor_b200 import gen
from conftest import plan_desc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev_graphs(golden_graphs):
    return {name: gi.Graph.from_csr(g.vertex, g.edge) for name, g in golden_graphs.items()}


def test_counts_match_reference_binaries(golden_counts, golden_graphs, dev_graphs):
    checked = 0
    for name, rows in golden_counts["patterns"].items():
        g, dg = golden_graphs[name], dev_graphs[name]
        for adj, want in rows.items():
            n = int(round(len(adj) ** 0.5))
            # pm_test plans without a triangle count (reference src/pm_test.cpp:22).
            s = gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, 0)
            if s.export()["iep_tables_rebuilt"]:
                continue
            assert gi.pattern_matching(dg, s).count == want, (name, adj)
            checked += 1
    assert checked > 100


@pytest.mark.parametrize("iep", [True, False])
def test_raw_sum_and_bytes_match_oracle(oracle, golden_graphs, dev_graphs, iep):
    g, dg = golden_graphs["rmat_s10_ef12"], dev_graphs["rmat_s10_ef12"]
    pats = [(3, "011101110"), (4, "0111101111001100"), (4, "0110100110010110"), (5, "0101110101010101010011000"),
            (5, "0111110111110111110111110"), (6, "011100101010110001100011010101001110"),
            (6, "010101101000010100101010000101100010"), (7, "0111111101111111011101110100111100011100001100000")]
    for n, adj in pats:
        s = gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, 0, enable_iep=iep)
        raw, nbytes = oracle.count(plan_desc(s), g.vertex, g.edge, threads=8, want_bytes=True)
        r = gi.pattern_matching(dg, s, count_bytes=True)
        assert r.raw_sum == raw, adj
        assert r.alg_bytes == nbytes, adj
        plain = gi.pattern_matching(dg, s)
        assert plain.raw_sum == raw and plain.count == r.count


def test_validated_plans_are_exact(oracle):
    graphs = [gen.erdos_renyi(40, 160, 21), gen.rmat(6, 6.0, 22)]
    pats = [(k, a) for k in (3, 4, 5) for a in gi.motif_patterns(k)]
    pats += random.Random(3).sample([(6, a) for a in gi.motif_patterns(6)], 20)
    for g in graphs:
        dg = gi.Graph.from_csr(g.vertex, g.edge)
        for n, adj in pats:
            want = oracle.brute(n, adj, g.vertex, g.edge)
            for iep in (True, False):
                s = gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, 0, model=2, enable_iep=iep)
                assert gi.pattern_matching(dg, s).count == want, (n, adj, iep)


def _shard(dg, s, shard, num, budget_ms=0.0, partial=False):
    st = N.Stats()
    st.budget_ms = budget_ms
    st.allow_partial = 1 if partial else 0
    raw = C.c_uint64()
    N.check(gi.lib().gi_count_shard(dg.handle, s.handle, shard, num, None, C.byref(raw), C.byref(st)),
            "gi_count_shard")
    return raw.value, st


@pytest.mark.parametrize("adj", ["0110100110010110", "011100101010110001100011010101001110"])
def test_shards_add_up_to_the_whole_count(golden_graphs, dev_graphs, adj):
    g, dg = golden_graphs["rmat_s10_ef12"], dev_graphs["rmat_s10_ef12"]
    n = int(round(len(adj) ** 0.5))
    s = gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, 0)
    full = gi.pattern_matching(dg, s).raw_sum
    for partial in (False, True):  # plain interleave, and the sampled (permuted) order with a roomy budget
        total, done = 0, 0
        for shard in range(5):
            raw, st = _shard(dg, s, shard, 5, budget_ms=60000.0 if partial else 0.0, partial=partial)
            assert st.chunks_done == st.chunks_total
            total, done = (total + raw) % (1 << 64), done + st.chunks_done
        assert total == full


def test_time_budgeted_sample_returns_a_partial_count():
    g = gen.rmat(14, 16.0, 9)
    dg = gi.Graph.from_csr(g.vertex, g.edge)
    s = gi.Schedule_IEP(gi.Pattern(6, "011100101010110001100011010101001110"), g.v_cnt, g.e_cnt, 0)
    raw, st = _shard(dg, s, 0, 1, budget_ms=0.05, partial=True)
    assert 0 <= st.chunks_done < st.chunks_total
    assert st.prep_ms >= 0.0 and st.kernel_ms > 0.0


def test_vertex_induced_plans(oracle):
    g = gen.erdos_renyi(60, 300, 5)
    dg = gi.Graph.from_csr(g.vertex, g.edge)
    for n, adj in [(3, "011101110"), (4, "0111101111011110"), (4, "0111101111001100")]:
        s = gi.Schedule_IEP(gi.Pattern(n, adj), vertex_induced=True)
        raw, _ = oracle.count(plan_desc(s), g.vertex, g.edge)
        assert gi.pattern_matching(dg, s).raw_sum == raw


@pytest.mark.parametrize("orientation", [0, 1])
def test_cliques_match_reference(golden_counts, dev_graphs, orientation):
    for name, cl in golden_counts["cliques"].items():
        for k, want in cl.items():
            assert gi.clique_count(dev_graphs[name], int(k), orientation).count == want, (name, k)


def test_motifs_match_reference(golden_counts, golden_graphs, dev_graphs):
    for name, mo in golden_counts["motifs"].items():
        counts4, _ = gi.motif_counting(dev_graphs[name], 4)
        assert counts4 == mo["4"], name
        tri, open_wedges = mo["3"]
        counts3, _ = gi.motif_counting(dev_graphs[name], 3)
        # MotifGenerator(3) = [triangle, wedge]; edge-induced wedges include
        # the closed ones (the reference's motif_counting_3 prints open ones).
        assert counts3 == [tri, open_wedges + 3 * tri], name


def test_larger_graph_invariants(oracle):
    """R-MAT scale 16: triangles four ways, 4-cliques two ways."""
    g = gen.rmat(16, 16.0, 7)
    dg = gi.Graph.from_csr(g.vertex, g.edge)
    tri = oracle.triangles(g.vertex, g.edge)
    s3 = gi.Schedule_IEP(gi.Pattern(3, "011101110"), g.v_cnt, g.e_cnt, tri)
    assert gi.pattern_matching(dg, s3).count == tri
    assert gi.clique_count(dg, 3, 0).count == tri
    assert gi.clique_count(dg, 3, 1).count == tri
    s4 = gi.Schedule_IEP(gi.Pattern.clique(4), g.v_cnt, g.e_cnt, tri)
    assert gi.pattern_matching(dg, s4).count == gi.clique_count(dg, 4, 1).count == gi.clique_count(dg, 4, 0).count


def test_hub_bitmaps_keep_counts_exact(oracle):
    """A graph with hubs (vertices whose lists the kernels test through a
    bitmap): edge subsets of the workload patterns and a 7-vertex pattern,
    whole counts of the cheaper ones, and the algorithmic bytes, against the
    oracle.  Both sides of every bitmap path run: hub lists as the father set
    and hubs as candidates, in the warp-built prefixes and the leaf level."""
    g = gen.rmat(14, 12.0, 2)
    dg = gi.Graph.from_csr(g.vertex, g.edge)
    assert dg.n_hubs > 0 and dg.hub_min_degree >= 256
    deg = np.diff(g.vertex)
    assert dg.n_hubs == int((deg >= dg.hub_min_degree).sum())
    pats = [(4, "0111101111001100"), (4, "0110100110010110"), (5, "0101110101010101010011000"),
            (5, "0111110111110111110111110"), (6, "011100101010110001100011010101001110"),
            (6, "010101101000010100101010000101100010"), (7, "0111111101111111011101110100111100011100001100000")]
    for n, adj in pats:
        for iep in (True, False):
            s = gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, 0, enable_iep=iep)
            d = plan_desc(s)
            want, _ = oracle.count_edges_timed(d, g.vertex, g.edge, 211, offset=17)
            assert gi.count_edges(dg, s, 211, 17).raw_sum == want, (adj, iep)
            if n <= 5:
                raw, nbytes = oracle.count(d, g.vertex, g.edge, want_bytes=True)
                r = gi.pattern_matching(dg, s, count_bytes=True)
                assert r.raw_sum == raw and r.alg_bytes == nbytes, (adj, iep)
                assert gi.pattern_matching(dg, s).raw_sum == raw


def test_budget_expiry_returns_timeout_and_device_stays_usable():
    g = gen.rmat(15, 16.0, 9)
    dg = gi.Graph.from_csr(g.vertex, g.edge)
    s = gi.Schedule_IEP(gi.Pattern(6, "011100101010110001100011010101001110"), g.v_cnt, g.e_cnt, 0)
    with pytest.raises(gi.GIError) as ei:
        gi.pattern_matching(dg, s, budget_ms=0.001)
    assert ei.value.status == N.GI_ETIMEOUT
    s3 = gi.Schedule_IEP(gi.Pattern(3, "011101110"), g.v_cnt, g.e_cnt, 0)
    assert gi.pattern_matching(dg, s3).count == gi.clique_count(dg, 3, 1).count


def test_cli_tools_print_the_reference_lines(tmp_path, golden_counts, golden_graphs):
    """gpu_graph / gpu_clique / gpu_kclique / gpu_mc with the reference's argv
    print the reference's result lines with the reference's counts."""
    import re
    import subprocess
    from pathlib import Path
    bindir = Path(gi.__file__).resolve().parent / "bin"
    name = "rmat_s9_ef8"
    g = golden_graphs[name]
    path = tmp_path / "g.g"
    gi.write_g(str(path), g.vertex, g.edge, g.max_intersection_size, 0)
    adj = "0101110101010101010011000"
    out = subprocess.run([str(bindir / "gpu_graph"), str(path), "5", adj], capture_output=True, text=True,
                         check=True).stdout
    assert int(re.search(r"Pattern count: (\d+)", out).group(1)) == golden_counts["patterns"][name][adj]
    assert re.search(r"Counting time cost: [\d.]+ s", out)
    out = subprocess.run([str(bindir / "gpu_clique"), str(path), "4"], capture_output=True, text=True,
                         check=True).stdout
    assert int(re.search(r"count (\d+)", out).group(1)) == golden_counts["cliques"][name]["4"]
    out = subprocess.run([str(bindir / "gpu_kclique"), str(path), "5"], capture_output=True, text=True,
                         check=True).stdout
    assert int(re.search(r"Answer: (\d+)", out).group(1)) == golden_counts["cliques"][name]["5"]
    out = subprocess.run([str(bindir / "gpu_mc"), str(path), "4"], capture_output=True, text=True, check=True).stdout
    assert [int(x) for x in re.findall(r"Pattern count: (\d+)", out)] == golden_counts["motifs"][name]["4"]


def test_rejects_malformed_graphs(native):
    vertex = np.array([0, 2, 3, 4], dtype=np.int64)
    edge = np.array([2, 1, 0, 0], dtype=np.int32)  # unsorted list of vertex 0
    with pytest.raises(gi.GIError) as ei:
        gi.Graph.from_csr(vertex, edge)
    assert ei.value.status == N.GI_EINVAL
    edge = np.array([1, 7, 0, 0], dtype=np.int32)  # id out of range
    with pytest.raises(gi.GIError):
        gi.Graph.from_csr(vertex, edge)
    vertex = np.array([0, 1, 2, 4], dtype=np.int64)
    edge = np.array([1, 0, 2, 1], dtype=np.int32)  # self-loop on vertex 2
    with pytest.raises(gi.GIError):
        gi.Graph.from_csr(vertex, edge)


def test_edge_cases(oracle):
    # A star (no triangles), a path, and a graph whose edges are all isolated pairs.
    star = gen.from_edges(33, [(0, i) for i in range(1, 33)])
    path = gen.from_edges(20, [(i, i + 1) for i in range(19)])
    pairs = gen.from_edges(10, [(0, 1), (2, 3), (4, 5)])
    for g in (star, path, pairs):
        dg = gi.Graph.from_csr(g.vertex, g.edge)
        for n, adj in [(3, "011101110"), (3, "011100100"), (4, "0110100110010110"), (4, "0111100010001000")]:
            s = gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, 0, model=2)
            assert gi.pattern_matching(dg, s).count == oracle.brute(n, adj, g.vertex, g.edge)
        assert gi.clique_count(dg, 3, 0).count == 0 or g is not star


def test_distributed_count_over_nccl_matches_the_single_gpu_count(golden_graphs, dev_graphs):
    """World size 1 over NCCL: the shard count plus the 2^64 all-reduce, and a
    batch whose jobs are spread over the ranks."""
    import datetime
    import os
    import socket
    import torch
    import torch.distributed as dist
    from graphindor_b200 import distributed as gd
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        g, dg = golden_graphs["rmat_s10_ef12"], dev_graphs["rmat_s10_ef12"]
        for n, adj in [(4, "0110100110010110"), (5, "0101110101010101010011000")]:
            s = gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, 0)
            assert gd.count(dg, s) == gi.pattern_matching(dg, s).count
        assert gd.allreduce_u64([(1 << 64) - 1]) == [(1 << 64) - 1]
        # Jobs of a batch spread over the ranks (here one) and exchanged.
        jobs = [(dg, gi.Schedule_IEP(gi.Pattern(n, a), g.v_cnt, g.e_cnt, 0))
                for n, a in [(3, "011101110"), (4, "0110100110010110"), (4, "0111101111001100")]]
        assert gd.batch_counts(jobs) == [gi.pattern_matching(d, s).count for d, s in jobs]
    finally:
        dist.destroy_process_group()


def _complete(n):
    return gen.from_edges(n, [(i, j) for i in range(n) for j in range(i + 1, n)])


def test_kclique_bitmaps_match_the_dfs_path_and_closed_forms(oracle):
    """Degree orientation runs the bitmap kernels (kclique.cu): rows of up to
    four words one per lane, longer rows (out-degree > 128) one per warp, lists
    over 1024 entries searched in global memory.  They must equal the general
    kernel on the same DAG and on the id DAG, the oracle's triangles, and
    C(n, k) on complete graphs."""
    from math import comb
    g = gen.chung_lu(10000, 800000, 1.9, 3000.0, 17)  # out-degrees up to 208
    deg = np.diff(g.vertex)
    src = np.repeat(np.arange(g.v_cnt), deg)
    dst = g.edge.astype(np.int64)
    keep = (deg[src] < deg[dst]) | ((deg[src] == deg[dst]) & (src < dst))
    assert np.bincount(src[keep], minlength=g.v_cnt).max() > 128  # both tiers run
    dg = gi.Graph.from_csr(g.vertex, g.edge)
    assert gi.clique_count(dg, 3, 1).count == oracle.triangles(g.vertex, g.edge)
    for k in (3, 4, 5):
        bitmap = gi.clique_count(dg, k, 1)
        dfs = gi.clique_count(dg, k, 1, count_bytes=True)  # byte accounting forces the general kernel
        assert bitmap.count == dfs.count == gi.clique_count(dg, k, 0).count, k
    for n, ks in ((40, (3, 4, 5, 6, 7)), (300, (3, 4, 5)), (1100, (3, 4))):
        dg = gi.Graph.from_csr(*(lambda c: (c.vertex, c.edge))(_complete(n)))
        for k in ks:
            assert gi.clique_count(dg, k, 1).count == comb(n, k) % (1 << 64), (n, k)


def test_fixed_samples_repeat_exactly_and_grow_to_the_whole_shard(golden_graphs, dev_graphs):
    """gi_stats.sample_chunks: the first M chunks of the shard's pseudo-random
    order, each counted to completion — the same raw sum on every call, and,
    when M covers every shard, shards that add up to the whole count."""
    g, dg = golden_graphs["rmat_s10_ef12"], dev_graphs["rmat_s10_ef12"]
    s = gi.Schedule_IEP(gi.Pattern(5, "0101110101010101010011000"), g.v_cnt, g.e_cnt, 0)

    def run(shard, m):
        st = N.Stats()
        st.sample_chunks = m
        raw = C.c_uint64()
        N.check(gi.lib().gi_count_shard(dg.handle, s.handle, shard, 3, None, C.byref(raw), C.byref(st)), "shard")
        return raw.value, st

    a, sa = run(1, 7)
    b, sb = run(1, 7)
    assert a == b and sa.chunks_done == sb.chunks_done == 7 < sa.chunks_total
    total = 0
    for shard in range(3):
        raw, st = run(shard, 1 << 40)
        assert st.chunks_done == st.chunks_total
        total = (total + raw) % (1 << 64)
    assert total == gi.pattern_matching(dg, s).raw_sum


def test_learned_schedules_count_exactly(golden_graphs, dev_graphs, oracle):
    """The learned cost model picks among valid candidates only, so its plans
    count exactly: equal to the validated analytic plan (model 2)."""
    g, dg = golden_graphs["rmat_s9_ef8"], dev_graphs["rmat_s9_ef8"]
    for n, adj in [(4, "0110100110010110"), (5, "0101110101010101010011000"),
                   (6, "011100101010110001100011010101001110"), (6, "010101101000010100101010000101100010")]:
        p = gi.Pattern(n, adj)
        learned = gi.Schedule_IEP.learned(p, dg)
        assert learned.export()["exact"] == 1
        exact = gi.Schedule_IEP(p, g.v_cnt, g.e_cnt, 0, model=2)
        assert gi.pattern_matching(dg, learned).count == gi.pattern_matching(dg, exact).count, adj


def test_batch_counts_match_single_counts(golden_graphs, dev_graphs):
    """One launch for (pattern, graph) jobs across four graphs, a graph with
    no edges among them; the first run captures the CUDA graph, the second
    replays it."""
    empty = gi.Graph.from_csr(np.array([0, 0, 0], dtype=np.int64), np.zeros(0, dtype=np.int32))
    pats = [(3, "011101110"), (4, "0111101111001100"), (4, "0110100110010110"), (5, "0101110101010101010011000"),
            (5, "0111110111110111110111110")]
    jobs, want = [], []
    for name, g in golden_graphs.items():
        for n, adj in pats:
            s = gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, 0)
            jobs.append((dev_graphs[name], s))
            want.append(gi.pattern_matching(dev_graphs[name], s).count)
    s0 = gi.Schedule_IEP(gi.Pattern(4, "0110100110010110"), 2, 1, 0, model=0)
    jobs.insert(3, (empty, s0))
    want.insert(3, 0)
    b = gi.Batch(jobs)
    for _ in range(2):
        counts, ms, kernel_ms = b.run()
        assert counts == want
        assert kernel_ms > 0 and all(m >= 0 for m in ms) and ms[3] == 0.0
