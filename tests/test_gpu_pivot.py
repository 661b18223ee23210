"""GPU parity of clique-tree pivoting (gi_clique_counts_pivot, kc_pivot_kernel):
the counts of every clique size at once against the oracle's own pivoting
counter, the enumerating bitmap kernel (gi_clique_count, degree orientation)
and C(n, k) on complete graphs.  Counts are integers and must be equal."""
from __future__ import annotations

from math import comb

import pytest

import graphindor_b200 as gi
from graphindor_b200 import gen

pytestmark = pytest.mark.gpu


def _graphs():
    # The Chung-Lu graphs have out-degrees above 64 and 128: rows of three
    # and more words, and the warp-wide row search of the bitmap kernels.
    return [("er_300", gen.erdos_renyi(300, 4000, 1)), ("rmat_s9", gen.rmat(9, 8.0, 11)),
            ("rmat_s12", gen.rmat(12, 16.0, 3)), ("cl_3000", gen.chung_lu(3000, 90000, 1.9, 900.0, 17)),
            ("cl_10000", gen.chung_lu(10000, 800000, 1.9, 3000.0, 17))]


def test_pivot_counts_match_the_oracle_and_the_enumerating_kernel(oracle):
    for name, g in _graphs():
        dg = gi.Graph.from_csr(g.vertex, g.edge)
        want = oracle.clique_counts_pivot(7, g.vertex, g.edge)
        assert want[1] == g.v_cnt and want[2] == g.e_cnt // 2
        for kmax in (1, 2, 3, 4, 5, 6, 7):
            got = gi.clique_counts_pivot(dg, kmax)
            assert got[0] == 0 and got[1:] == want[1:kmax + 1], (name, kmax, got, want)
        for k in (3, 4, 5):
            assert gi.clique_count(dg, k, 1).count == want[k], (name, k)


def test_pivot_on_complete_graphs_and_a_search_deeper_than_the_first_stack():
    # K40: every root's search is a chain of its out-degree.  K70 plus a
    # pendant path: the root of out-degree 69 needs more than the 64 stack
    # levels the first launch gets, so the count retries with a deeper stack.
    k40 = gen.from_edges(40, [(i, j) for i in range(40) for j in range(i + 1, 40)])
    dg = gi.Graph.from_csr(k40.vertex, k40.edge)
    assert gi.clique_counts_pivot(dg, 7)[1:] == [comb(40, k) for k in range(1, 8)]
    k70 = gen.from_edges(73, [(i, j) for i in range(70) for j in range(i + 1, 70)] + [(69, 70), (70, 71), (71, 72)])
    dg = gi.Graph.from_csr(k70.vertex, k70.edge)
    want = [comb(70, k) for k in range(1, 8)]
    want[0] += 3
    want[1] += 3
    assert gi.clique_counts_pivot(dg, 7)[1:] == want
    for k in (3, 4, 5):
        assert gi.clique_count(dg, k, 1).count == want[k - 1]


def test_pivot_repeats_and_handles_graphs_without_edges():
    g = gen.rmat(11, 12.0, 5)
    dg = gi.Graph.from_csr(g.vertex, g.edge)
    a = gi.clique_counts_pivot(dg, 6)
    assert gi.clique_counts_pivot(dg, 6) == a
    assert gi.clique_counts_pivot(dg, 4) == a[:5]
    empty = gen.from_edges(5, [])
    de = gi.Graph.from_csr(empty.vertex, empty.edge)
    assert gi.clique_counts_pivot(de, 7) == [0, 5, 0, 0, 0, 0, 0, 0]
