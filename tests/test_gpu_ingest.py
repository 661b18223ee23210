"""GPU ingest of labeled graphs: gi_labeled_graph_create_device (renaming,
renumbering and label bucketing by kernels and device sorts) against the
host loader gi_labeled_graph_create, which is pinned to the reference's
fsm_test through the FSM fixtures.  Every exported array must be identical,
and so must the FSM counts of the two structures."""
from __future__ import annotations

import numpy as np
import pytest

import graphindor_b200 as gi
from graphindor_b200 import gen

pytestmark = pytest.mark.gpu


def _same(a: gi.LabeledGraph, b: gi.LabeledGraph):
    assert (a.v_cnt, a.e_cnt, a.l_cnt) == (b.v_cnt, b.e_cnt, b.l_cnt)
    ea, eb = a.export(), b.export()
    assert ea.keys() == eb.keys()
    for k in ea:
        assert np.array_equal(ea[k], eb[k]), k


@pytest.mark.parametrize("case", range(5))
def test_device_ingest_equals_host_loader(case):
    rng = np.random.default_rng(40 + case)
    scale = int(rng.integers(9, 14))
    keep = int((1 << scale) * rng.uniform(0.5, 1.0))
    n_labels = int(rng.integers(1, 40))
    g, labels = gen.labeled_rmat(scale, float(rng.uniform(4, 16)), 500 + case, keep, n_labels,
                                 float(rng.uniform(0.3, 1.6)), 600 + case)
    # Original label values far from 0..l-1, and a shuffled line order
    # (it fixes the first-seen label order).
    labels = (labels.astype(np.uint64) * 7919 + 13).astype(np.uint32)
    order = rng.permutation(g.v_cnt).astype(np.int32) if case % 2 else None
    host = gi.LabeledGraph.from_csr(g.vertex, g.edge, labels, order)
    dev = gi.LabeledGraph.from_csr(g.vertex, g.edge, labels, order, device=True)
    _same(host, dev)
    for ms in (5, 50):
        assert gi.fsm(dev, 3, ms, gi.YOUTUBE_TRI_CNT).count == gi.fsm(host, 3, ms, gi.YOUTUBE_TRI_CNT).count


def test_device_ingest_self_loops_duplicates_and_ties():
    # Self-loops are dropped, duplicate entries kept, equal degrees and equal
    # label maxima resolved as the host loader resolves them.
    vertex = np.array([0, 3, 6, 8, 10, 12, 12], dtype=np.int64)
    # vertex 0: a self-loop and 1 twice; vertex 1: 0 twice and 2; vertex 4: a self-loop
    edge = np.array([0, 1, 1, 0, 0, 2, 1, 3, 2, 4, 3, 4], dtype=np.int32)
    labels = np.array([5, 5, 9, 9, 5, 7], dtype=np.uint32)
    host = gi.LabeledGraph.from_csr(vertex, edge, labels)
    dev = gi.LabeledGraph.from_csr(vertex, edge, labels, device=True)
    _same(host, dev)


def test_device_ingest_rejects_what_the_host_loader_rejects():
    g = gen.from_edges(6, [(0, 1), (1, 2), (2, 3)])
    labels = np.zeros(6, np.uint32)
    bad = g.edge.copy()
    bad[0] = 7  # out of range
    with pytest.raises(gi.GIError):
        gi.LabeledGraph.from_csr(g.vertex, bad, labels, device=True)
    one_way = gen.from_edges(6, [(0, 1), (1, 2), (2, 3)])
    e = one_way.edge.copy()
    e[e.tolist().index(0)] = 3  # vertex 1 lists 3, vertex 3 does not list 1
    with pytest.raises(gi.GIError):
        gi.LabeledGraph.from_csr(one_way.vertex, e, labels, device=True)
    many = np.arange(300, dtype=np.uint32)
    big = gen.from_edges(300, [(i, i + 1) for i in range(299)])
    with pytest.raises(gi.GIError):
        gi.LabeledGraph.from_csr(big.vertex, big.edge, many, device=True)


def test_device_ingest_of_the_config3_fsm_graph():
    # The 100,000-vertex, 29-label FSM input: same structure and same
    # frequent-pattern count as the host loader at min_support 1000.
    g, labels = gen.labeled_rmat(17, 16.65, 4, 100_000, 29, 1.1, 4)
    host = gi.LabeledGraph.from_csr(g.vertex, g.edge, labels)
    dev = gi.LabeledGraph.from_csr(g.vertex, g.edge, labels, device=True)
    _same(host, dev)
    assert gi.fsm(dev, 3, 1000, 7515023).count == gi.fsm(host, 3, 1000, 7515023).count
