"""gi_count_noalloc: the count for callers that cannot allocate device
memory (their GPU memory belongs to another framework's pool, or a serving
loop must not pay cudaMalloc's latency and implicit synchronisation).  The
caller's own device buffers go in; the result must equal gi_count's, call
after call, although every call reuses the same fixed scratch array.

Collected last on purpose (file name), so that a run stopping at the first
failure has already run every other test.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import graphindor_b200 as gi
from graphindor_b200 import _native as N
from graphindor_b200 import gen

pytestmark = pytest.mark.gpu


def _noalloc(L, dv, de, v_cnt, e_cnt, plan, result):
    return L.gi_count_noalloc(C.c_void_p(dv.data_ptr()), C.c_void_p(de.data_ptr()), v_cnt, e_cnt, plan.handle,
                              None, C.c_void_p(result.data_ptr()))


@pytest.fixture(scope="module")
def lib():
    L = gi.lib()
    L.gi_count_noalloc.restype = C.c_int
    L.gi_count_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p,
                                   C.c_void_p]
    return L


def test_noalloc_matches_gi_count_on_consecutive_calls(lib):
    import torch
    g = gen.rmat(12, 12.0, 31)
    dg = gi.Graph.from_csr(g.vertex, g.edge)
    dv = torch.from_numpy(g.vertex).cuda()
    de = torch.from_numpy(g.edge).cuda()
    result = torch.zeros(2, dtype=torch.int64, device="cuda")
    patterns = [(5, "0101110101010101010011000"), (4, "0110100110010110"), (6, "011100101010110001100011010101001110")]
    for n, adj in patterns:
        s = gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, 0)
        want = gi.pattern_matching(dg, s)
        for _ in range(2):  # two calls in a row share (and reuse) the scratch array
            result.fill_(-1)
            N.check(_noalloc(lib, dv, de, g.v_cnt, g.e_cnt, s, result), "gi_count_noalloc")
            count, raw = (int(x) & ((1 << 64) - 1) for x in result.tolist())
            assert count == want.count
            assert raw == want.raw_sum


def test_noalloc_rejects_malformed_and_oversized_inputs(lib):
    import torch
    result = torch.zeros(2, dtype=torch.int64, device="cuda")
    s = gi.Schedule_IEP(gi.Pattern(3, "011101110"), 4, 8, 0)
    vertex = torch.tensor([0, 2, 3, 4], dtype=torch.int64, device="cuda")
    edge = torch.tensor([2, 1, 0, 0], dtype=torch.int32, device="cuda")  # unsorted list of vertex 0
    assert _noalloc(lib, vertex, edge, 3, 4, s, result) == N.GI_EINVAL
    # Two hubs joined to 2M leaves: one block of a prism plan would need more
    # than the fixed scratch (materialised sets x the second-largest degree).
    m = 2_000_000
    leaves = np.arange(2, m + 2, dtype=np.int32)
    vertex_h = np.concatenate([[0, m, 2 * m], 2 * m + 2 * np.arange(1, m + 1)]).astype(np.int64)
    edge_h = np.concatenate([leaves, leaves, np.tile(np.array([0, 1], dtype=np.int32), m)]).astype(np.int32)
    prism = gi.Schedule_IEP(gi.Pattern(6, "011100101010110001100011010101001110"), m + 2, 4 * m, 0)
    rc = _noalloc(lib, torch.from_numpy(vertex_h).cuda(), torch.from_numpy(edge_h).cuda(), m + 2, 4 * m, prism, result)
    assert rc == N.GI_EOVERFLOW
