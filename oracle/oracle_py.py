"""ORACLE — test infrastructure only: ctypes access to oracle/liboracle.so.

Used by tests/, the smoke check and bench.py's CPU-baseline leg; the engine
never imports it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE), "liboracle.so"], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()  # incremental: rebuilds only when oracle.c changed
        L = C.CDLL(str(LIB))
        L.oracle_count.restype = C.c_int
        L.oracle_count.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int,
                                   C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.oracle_count_strided.restype = C.c_int
        L.oracle_count_strided.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                                           C.c_int32, C.c_int, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.oracle_count_timed.restype = C.c_int
        L.oracle_count_timed.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int,
                                         C.c_double, C.POINTER(C.c_uint64), C.POINTER(C.c_int64)]
        L.oracle_count_edges_timed.restype = C.c_int
        L.oracle_count_edges_timed.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_int64,
                                               C.c_int, C.c_double, C.POINTER(C.c_uint64), C.POINTER(C.c_int64)]
        L.oracle_brute_count.restype = C.c_uint64
        L.oracle_brute_count.argtypes = [C.c_int, C.c_char_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int32]
        L.oracle_clique_count.restype = C.c_uint64
        L.oracle_clique_count.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int32]
        L.oracle_triangles.restype = C.c_uint64
        L.oracle_triangles.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int]
        _lib = L
    return _lib


def _arrays(vertex, edge):
    vertex = np.ascontiguousarray(vertex, dtype=np.int64)
    edge = np.ascontiguousarray(edge, dtype=np.int32)
    if edge.size == 0:
        edge = np.zeros(1, dtype=np.int32)
    return vertex, edge


def count(plan_desc, vertex, edge, v_begin=0, v_end=None, threads=0, want_bytes=False):
    """(raw_sum mod 2^64, alg_bytes or None) over start vertices [v_begin, v_end).
    plan_desc is a graphindor_b200._native.PlanDesc (the exported Schedule_IEP)."""
    vertex, edge = _arrays(vertex, edge)
    n = len(vertex) - 1
    raw, nb = C.c_uint64(), C.c_uint64()
    rc = lib().oracle_count(C.byref(plan_desc), vertex.ctypes.data, edge.ctypes.data, n, v_begin,
                            n if v_end is None else v_end, threads, C.byref(raw),
                            C.byref(nb) if want_bytes else None)
    if rc != 0:
        raise ValueError("oracle_count rejected its input")
    return raw.value, (nb.value if want_bytes else None)


def count_strided(plan_desc, vertex, edge, stride, v_begin=0, threads=0):
    """Raw sum over the start vertices v_begin, v_begin + stride, ...: an
    unbiased 1/stride sample when vertex ids are randomly assigned."""
    vertex, edge = _arrays(vertex, edge)
    n = len(vertex) - 1
    raw = C.c_uint64()
    rc = lib().oracle_count_strided(C.byref(plan_desc), vertex.ctypes.data, edge.ctypes.data, n, v_begin, n,
                                    stride, threads, C.byref(raw), None)
    if rc != 0:
        raise ValueError("oracle_count_strided rejected its input")
    return raw.value


def count_timed(plan_desc, vertex, edge, stride, max_seconds, threads=0):
    """(raw sum, start vertices counted) over every stride-th start vertex,
    beginning no start vertex after max_seconds."""
    vertex, edge = _arrays(vertex, edge)
    raw, done = C.c_uint64(), C.c_int64()
    rc = lib().oracle_count_timed(C.byref(plan_desc), vertex.ctypes.data, edge.ctypes.data, len(vertex) - 1,
                                  stride, threads, max_seconds, C.byref(raw), C.byref(done))
    if rc != 0:
        raise ValueError("oracle_count_timed rejected its input")
    return raw.value, done.value


def count_edges_timed(plan_desc, vertex, edge, stride, max_seconds=0.0, threads=0, offset=0):
    """(raw sum, edges counted) over the directed edges offset, offset +
    stride, offset + 2 * stride, ..."""
    vertex, edge = _arrays(vertex, edge)
    raw, done = C.c_uint64(), C.c_int64()
    rc = lib().oracle_count_edges_timed(C.byref(plan_desc), vertex.ctypes.data, edge.ctypes.data, len(vertex) - 1,
                                        stride, offset, threads, max_seconds, C.byref(raw), C.byref(done))
    if rc != 0:
        raise ValueError("oracle_count_edges_timed rejected its input")
    return raw.value, done.value


def brute(n, adj, vertex, edge, induced=False):
    vertex, edge = _arrays(vertex, edge)
    return lib().oracle_brute_count(n, adj.encode(), int(induced), vertex.ctypes.data, edge.ctypes.data,
                                    len(vertex) - 1)


def cliques(k, vertex, edge):
    vertex, edge = _arrays(vertex, edge)
    return lib().oracle_clique_count(k, vertex.ctypes.data, edge.ctypes.data, len(vertex) - 1)


def clique_counts_pivot(kmax, vertex, edge, threads=0):
    """[count of k-cliques for k = 0 .. kmax] (index 0 unused) by clique-tree
    pivoting, modulo 2^64."""
    L_ = lib()
    if not hasattr(L_.oracle_clique_counts_pivot, "_typed"):
        L_.oracle_clique_counts_pivot.restype = C.c_int
        L_.oracle_clique_counts_pivot.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int32, C.c_int, C.c_void_p]
        L_.oracle_clique_counts_pivot._typed = True
    vertex, edge = _arrays(vertex, edge)
    out = np.zeros(kmax + 1, dtype=np.uint64)
    if L_.oracle_clique_counts_pivot(kmax, vertex.ctypes.data, edge.ctypes.data, len(vertex) - 1, threads,
                                     out.ctypes.data) != 0:
        raise ValueError("oracle_clique_counts_pivot failed")
    return [int(x) for x in out]


def triangles(vertex, edge, threads=0):
    vertex, edge = _arrays(vertex, edge)
    return lib().oracle_triangles(vertex.ctypes.data, edge.ctypes.data, len(vertex) - 1, threads)


# ------------------------------------------------------------------ FSM

def fsm_load(vertex, edge, labels, order=None):
    """Restatement of the reference's labeled loader (reference
    src/dataloader.cpp:440-620) for symmetric input: labels in first-seen
    order renamed by descending maximum degree, vertices renumbered by
    (label, -degree, id), neighbour lists sorted by (label, id) and bucketed.
    Ties in maximum degree keep first-seen order (a stable sort); the
    reference's std::sort agrees for up to 16 labels, where it is an
    insertion sort.  Returns a dict of numpy arrays."""
    vertex = np.asarray(vertex, dtype=np.int64)
    edge = np.asarray(edge, dtype=np.int64)
    labels = np.asarray(labels, dtype=np.uint64)
    n = len(vertex) - 1
    seq = np.arange(n) if order is None else np.asarray(order)
    first = {}
    for v in seq:
        first.setdefault(int(labels[v]), len(first))
    tmp = np.array([first[int(x)] for x in labels], dtype=np.int64)
    L = len(first)
    src = np.repeat(np.arange(n), np.diff(vertex))
    keep = edge != src
    src, dst = src[keep], edge[keep]
    degree = np.bincount(src, minlength=n)
    max_deg = np.zeros(L, dtype=np.int64)
    np.maximum.at(max_deg, tmp, degree)
    by = sorted(range(L), key=lambda l: -max_deg[l])  # stable
    rename = np.empty(L, dtype=np.int64)
    rename[by] = np.arange(L)
    lab = rename[tmp]
    rank = np.lexsort((np.arange(n), -degree, lab))
    new_id = np.empty(n, dtype=np.int64)
    new_id[rank] = np.arange(n)
    v_label = lab[rank]
    s2, d2 = new_id[src], new_id[dst]
    o = np.lexsort((d2, v_label[d2], s2))
    s2, d2 = s2[o], d2[o]
    key = s2 * L + v_label[d2]
    bucket = np.searchsorted(key, np.arange(n * L + 1), side="left").astype(np.uint32)
    freq = np.bincount(lab, minlength=L)
    label_start = np.concatenate([[0], np.cumsum(freq)]).astype(np.uint32)
    label_value = np.empty(L, dtype=np.uint64)
    for val, t in first.items():
        label_value[rename[t]] = val
    return {"v_cnt": n, "l_cnt": L, "e_cnt": len(d2), "new_id": new_id.astype(np.int32),
            "v_label": v_label.astype(np.int32), "label_value": label_value.astype(np.uint32),
            "label_start": label_start, "label_frequency": freq, "bucket": bucket,
            "edge": d2.astype(np.uint32)}


def fsm_support(G, adj, jobs, min_support, threads=0):
    """(support[j], frequent[j]) of labeled patterns by the reference's
    enumeration.  adj: n*n '0'/'1' string in schedule order; jobs: int array
    (n_jobs, n) of labels by position."""
    L_ = lib()
    if not hasattr(L_.oracle_fsm_support, "_typed"):
        L_.oracle_fsm_support.restype = C.c_int
        L_.oracle_fsm_support.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                          C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int, C.c_void_p,
                                          C.c_void_p]
        L_.oracle_fsm_support._typed = True
    jobs = np.ascontiguousarray(jobs, dtype=np.uint8)
    n_jobs, n = jobs.shape
    a = np.array([int(c) for c in adj], dtype=np.int32)
    bucket = np.ascontiguousarray(G["bucket"], dtype=np.uint32)
    edge = np.ascontiguousarray(G["edge"] if len(G["edge"]) else np.zeros(1), dtype=np.uint32)
    ls = np.ascontiguousarray(G["label_start"], dtype=np.uint32)
    sup = np.zeros(max(n_jobs, 1), dtype=np.int64)
    freq = np.zeros(max(n_jobs, 1), dtype=np.uint8)
    rc = L_.oracle_fsm_support(G["v_cnt"], G["l_cnt"], bucket.ctypes.data, edge.ctypes.data, ls.ctypes.data, n,
                               a.ctypes.data, n_jobs, jobs.ctypes.data, int(min_support), threads,
                               sup.ctypes.data, freq.ctypes.data)
    if rc != 0:
        raise ValueError("oracle_fsm_support rejected its input")
    return sup[:n_jobs], freq[:n_jobs].astype(bool)


def fsm_frequent_per_pattern(G, plans, min_support, threads=0):
    """For each plan, the number of restriction-satisfying labelings with MNI
    support >= min_support (the per-pattern terms of fsm_count)."""
    import itertools
    freq_labels = [l for l in range(G["l_cnt"]) if G["label_frequency"][l] >= min_support]
    out = []
    for p in plans:
        n = p["n"]
        jobs = [t for t in itertools.product(freq_labels, repeat=n)
                if all(t[d] <= t[r] for d, r in p["restricts"])]
        if not jobs:
            out.append(0)
            continue
        _, fr = fsm_support(G, p["adj"], np.array(jobs, dtype=np.uint8), min_support, threads)
        out.append(int(fr.sum()))
    return out


def fsm_count(G, plans, max_edge, min_support, threads=0):
    """The reference FSM result by its definition: over the patterns with
    exactly max_edge edges, the labelings (labels by schedule position) that
    satisfy the plan's restrictions (label[d] <= label[r]) and whose MNI
    support reaches min_support.  The reference reaches the same set through
    Apriori pruning (reference src/labeled_graph.cpp:393-433), which only
    drops labelings with an infrequent sub-pattern, hence infrequent ones.
    plans: dicts with n, edges, adj (schedule order), restricts [(d, r)].
    Labelings that use a label occurring fewer than min_support times are
    infrequent (the support of a position is at most its label's count) and
    are not run."""
    import itertools
    freq_labels = [l for l in range(G["l_cnt"]) if G["label_frequency"][l] >= min_support]
    if max_edge == 0:
        return len(freq_labels)
    total = 0
    for p in plans:
        if p["edges"] != max_edge:
            continue
        n = p["n"]
        jobs = [t for t in itertools.product(freq_labels, repeat=n)
                if all(t[d] <= t[r] for d, r in p["restricts"])]
        if not jobs:
            continue
        _, fr = fsm_support(G, p["adj"], np.array(jobs, dtype=np.uint8), min_support, threads)
        total += int(fr.sum())
    return total
