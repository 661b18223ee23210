"""The oracle (a C restatement of the reference CPU path, oracle/oracle.c)
against the reference's own outputs: golden counts from the reference
binaries on seeded graphs, the independent brute-force counter, and — when
the reference checkout is present — the Wiki-Vote vectors."""
from __future__ import annotations

import os
from pathlib import Path

import pytest

import graphindor_b200 as gi
from conftest import plan_desc

# The reference checkout ($GI_REFERENCE, else "reference" beside this
# repository); its one shipped dataset, when present.
REFERENCE = Path(os.environ.get("GI_REFERENCE", str(Path(__file__).resolve().parents[2] / "reference")))
WIKI = REFERENCE / "dataset" / "wiki-vote.g"


def _oracle_count(oracle, g, n, adj, enable_iep=True, tri=0, model=1):
    s = gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, tri, enable_iep=enable_iep, model=model)
    d = plan_desc(s)
    raw, _ = oracle.count(d, g.vertex, g.edge, threads=4)
    return raw // d.count_divisor, d


def test_oracle_matches_reference_binaries(oracle, golden_counts, golden_graphs):
    checked = 0
    for name, rows in golden_counts["patterns"].items():
        g = golden_graphs[name]
        for adj, want in rows.items():
            n = int(round(len(adj) ** 0.5))
            got, d = _oracle_count(oracle, g, n, adj)
            if d.iep_tables_rebuilt:
                continue  # reference count undefined for this plan (out-of-bounds read)
            assert got == want, (name, adj)
            checked += 1
    assert checked > 100


@pytest.mark.parametrize("model", [1, 2])
def test_oracle_iep_off_equals_iep_on(oracle, golden_graphs, model):
    """IEP is an exact shortcut: with it or without it the count is the same,
    for every plan whose restriction set is valid."""
    g = golden_graphs["rmat_s9_ef8"]
    for n, adj in [(4, "0111101111001100"), (5, "0101110101010101010011000"),
                   (6, "011100101010110001100011010101001110")]:
        a, da = _oracle_count(oracle, g, n, adj, enable_iep=True, model=model)
        b, db = _oracle_count(oracle, g, n, adj, enable_iep=False, model=model)
        if da.exact == 1 and db.exact == 1:
            assert a == b




def _brute_cases():
    from graphindor_b200 import gen
    graphs = [gen.erdos_renyi(40, 160, 21), gen.rmat(6, 6.0, 22)]
    pats = [(k, a) for k in (3, 4, 5) for a in gi.motif_patterns(k)]
    pats += [(6, "011100101010110001100011010101001110"), (6, "010101101000010100101010000101100010"),
             (6, "011011101110110101011000110000101000")]
    return graphs, pats


def test_reference_plans_are_exact_exactly_when_their_restrictions_are_valid(oracle, native):
    """The reference's restriction generator validates candidate sets on a
    complete graph in vertex-induced mode (reference src/schedule_IEP.cpp:
    1737-1760), which accepts any set for a non-clique pattern, so some of its
    plans over- or under-count.  Its count (= the oracle's on its plan) equals
    exhaustive search exactly when the plan's applied restrictions count every
    subgraph equally (gi_plan_desc.exact)."""
    graphs, pats = _brute_cases()
    wrong = 0
    for g in graphs:
        for n, adj in pats:
            want = oracle.brute(n, adj, g.vertex, g.edge)
            got, d = _oracle_count(oracle, g, n, adj)
            if d.exact == 1:
                assert got == want, (n, adj)
            elif got != want:
                wrong += 1
    # The prism and the chorded 6-cycle are among the reference's miscounts.
    assert wrong >= 4


def test_validated_plans_match_brute_force(oracle, native):
    graphs, pats = _brute_cases()
    for g in graphs:
        for n, adj in pats:
            want = oracle.brute(n, adj, g.vertex, g.edge)
            for iep in (True, False):
                got, d = _oracle_count(oracle, g, n, adj, enable_iep=iep, model=2)
                assert d.exact == 1
                assert got == want, (n, adj, iep)


def test_edge_sampled_counts_partition_the_whole(oracle, golden_graphs):
    """Counting per directed edge (the CPU baseline's sampling unit) sums to
    the per-start-vertex count, and the strided slices partition it."""
    g = golden_graphs["rmat_s10_ef12"]
    for n, adj in [(4, "0110100110010110"), (5, "0101110101010101010011000"),
                   (6, "011100101010110001100011010101001110")]:
        s = gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, 0)
        d = plan_desc(s)
        whole, _ = oracle.count(d, g.vertex, g.edge, threads=4)
        raw, done = oracle.count_edges_timed(d, g.vertex, g.edge, 1, threads=4)
        assert raw == whole and done == g.e_cnt
    s = gi.Schedule_IEP(gi.Pattern(3, "011101110"), vertex_induced=True)
    d = plan_desc(s)
    whole, _ = oracle.count(d, g.vertex, g.edge, threads=4)
    assert oracle.count_edges_timed(d, g.vertex, g.edge, 1, threads=4)[0] == whole


def test_oracle_cliques_and_triangles(oracle, golden_counts, golden_graphs):
    for name, cl in golden_counts["cliques"].items():
        g = golden_graphs[name]
        assert oracle.triangles(g.vertex, g.edge) == cl["3"]
        for k in ("3", "4", "5"):
            assert oracle.cliques(int(k), g.vertex, g.edge) == cl[k], (name, k)


@pytest.mark.skipif(not WIKI.exists(), reason="reference checkout not present")
def test_oracle_wiki_vote_vectors(oracle):
    """Known answers on the reference's Wiki-Vote file: the published triangle
    count (reference include/dataloader.h:32) and the counts the reference's
    CPU binaries print for the same patterns."""
    vertex, edge, _, _ = gi.read_g(str(WIKI))
    from graphindor_b200.gen import CSR
    g = CSR(vertex, edge, 0, 0)
    assert oracle.triangles(vertex, edge) == 608389
    for n, adj, want in [(3, "011101110", 608389), (4, "0111101111001100", 40544543),
                         (4, "0110100110010110", 57654491), (5, "0111110111110111110111110", 4514137)]:
        got, _ = _oracle_count(oracle, g, n, adj)
        assert got == want


def test_pivoting_clique_counts_match_enumeration(oracle):
    """The clique-tree pivoting oracle (exact counts for large k) against the
    enumerating one and against C(n, k) on a complete graph."""
    from math import comb
    from graphindor_b200 import gen
    for g in (gen.erdos_renyi(200, 3000, 1), gen.rmat(9, 8.0, 11), gen.chung_lu(2000, 12000, 2.2, 200.0, 14)):
        piv = oracle.clique_counts_pivot(7, g.vertex, g.edge)
        assert piv[3:7] == [oracle.cliques(k, g.vertex, g.edge) for k in range(3, 7)]
        for kmax in (3, 5):  # a smaller kmax closes the search earlier; the lower counts stay the same
            assert oracle.clique_counts_pivot(kmax, g.vertex, g.edge) == piv[:kmax + 1]
    k40 = gen.from_edges(40, [(i, j) for i in range(40) for j in range(i + 1, 40)])
    assert oracle.clique_counts_pivot(7, k40.vertex, k40.edge)[1:] == [comb(40, k) for k in range(1, 8)]
    # Cliques longer than one 64-bit row word, with a pendant path attached.
    k70 = gen.from_edges(73, [(i, j) for i in range(70) for j in range(i + 1, 70)] + [(69, 70), (70, 71), (71, 72)])
    want = [comb(70, k) for k in range(1, 8)]
    want[0] += 3
    want[1] += 3
    assert oracle.clique_counts_pivot(7, k70.vertex, k70.edge)[1:] == want


REF_SAMPLER = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "ref_edge_sample"


@pytest.mark.skipif(not os.access(REF_SAMPLER, os.X_OK), reason="reference sources not compiled here")
def test_reference_edge_tasks_sum_to_the_oracle_count(oracle, native, tmp_path):
    """The reference's own per-edge task (oracle/_ref/ref_edge_sample, the CPU
    baseline's sampler) summed over every directed edge, with the plans the
    reference makes from the .g header, equals the oracle's whole count, and
    its redundancy equals this planner's divisor."""
    import subprocess
    import graphindor_b200 as gi
    from graphindor_b200 import gen
    from conftest import plan_desc
    pats = [(4, "0111101111001100"), (4, "0110100110010110"), (5, "0101110101010101010011000"),
            (6, "011100101010110001100011010101001110")]
    for g in (gen.rmat(10, 12.0, 12), gen.erdos_renyi(500, 4000, 3)):
        tri = oracle.triangles(g.vertex, g.edge)
        path = tmp_path / "g.g"
        gi.write_g(str(path), g.vertex, g.edge, g.max_intersection_size, tri)
        for iep in (1, 0):
            # A target far above the sample's time drives the stride down to 1.
            args = [str(REF_SAMPLER), str(path), str(iep), "1000", "4"] + [x for n, a in pats for x in (str(n), a)]
            out = subprocess.run(args, capture_output=True, text=True, check=True, timeout=300).stdout
            rows = {f[0]: f for f in (line.split() for line in out.splitlines() if " raw " in line)}
            for n, a in pats:
                f = rows[a]
                d = plan_desc(gi.Schedule_IEP(gi.Pattern(n, a), g.v_cnt, g.e_cnt, tri, enable_iep=bool(iep)))
                raw, _ = oracle.count(d, g.vertex, g.edge)
                assert (int(f[2]), int(f[4]), int(f[6])) == (raw, g.e_cnt, 1), (iep, a)
                assert int(f[10]) == d.count_divisor, (iep, a)
