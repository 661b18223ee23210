"""Seeded synthetic graphs (include/gi_gen.h) as numpy CSR arrays."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._native import check, lib


class _HostCSR(C.Structure):
    _fields_ = [("v_cnt", C.c_int32), ("e_cnt", C.c_int64), ("vertex", C.POINTER(C.c_int64)),
                ("edge", C.POINTER(C.c_int32)), ("max_degree", C.c_int32), ("max_intersection_size", C.c_int32)]


@dataclass
class CSR:
    vertex: np.ndarray  # int64[v_cnt + 1]
    edge: np.ndarray    # int32[e_cnt]
    max_degree: int
    max_intersection_size: int

    @property
    def v_cnt(self) -> int:
        return len(self.vertex) - 1

    @property
    def e_cnt(self) -> int:
        return len(self.edge)


def _take(ptr: C.POINTER(_HostCSR)) -> CSR:
    L = lib()
    h = ptr.contents
    v = np.ctypeslib.as_array(h.vertex, shape=(h.v_cnt + 1,)).copy()
    e = np.ctypeslib.as_array(h.edge, shape=(max(1, h.e_cnt),))[: h.e_cnt].copy()
    out = CSR(v, e, h.max_degree, h.max_intersection_size)
    L.gi_host_csr_free(ptr)
    return out


def _call(name, *args) -> CSR:
    L = lib()
    fn = getattr(L, name)
    fn.restype = C.c_int
    L.gi_host_csr_free.argtypes = [C.POINTER(_HostCSR)]
    L.gi_host_csr_free.restype = None
    out = C.POINTER(_HostCSR)()
    check(fn(*args, C.byref(out)), name)
    return _take(out)


def rmat(scale: int, edge_factor: float, seed: int, a: float = 0.57, b: float = 0.19, c: float = 0.19) -> CSR:
    return _call("gi_gen_rmat", C.c_int(scale), C.c_double(edge_factor), C.c_double(a), C.c_double(b),
                 C.c_double(c), C.c_uint64(seed))


def chung_lu(n: int, m: int, gamma: float, max_degree: float, seed: int) -> CSR:
    return _call("gi_gen_chung_lu", C.c_int32(n), C.c_int64(m), C.c_double(gamma), C.c_double(max_degree),
                 C.c_uint64(seed))


def erdos_renyi(n: int, m: int, seed: int) -> CSR:
    return _call("gi_gen_er", C.c_int32(n), C.c_int64(m), C.c_uint64(seed))


def restrict(g: CSR, keep: int) -> CSR:
    L = lib()
    h = _HostCSR(g.v_cnt, g.e_cnt, g.vertex.ctypes.data_as(C.POINTER(C.c_int64)),
                 g.edge.ctypes.data_as(C.POINTER(C.c_int32)), g.max_degree, g.max_intersection_size)
    L.gi_csr_restrict.argtypes = [C.POINTER(_HostCSR), C.c_int32, C.POINTER(C.POINTER(_HostCSR))]
    L.gi_csr_restrict.restype = C.c_int
    L.gi_host_csr_free.argtypes = [C.POINTER(_HostCSR)]
    out = C.POINTER(_HostCSR)()
    check(L.gi_csr_restrict(C.byref(h), keep, C.byref(out)), "gi_csr_restrict")
    return _take(out)


def from_edges(n: int, edges) -> CSR:
    """CSR of a small explicit undirected edge list (tests)."""
    adj = [set() for _ in range(n)]
    for u, v in edges:
        if u != v:
            adj[u].add(v)
            adj[v].add(u)
    vertex = np.zeros(n + 1, dtype=np.int64)
    for i in range(n):
        vertex[i + 1] = vertex[i] + len(adj[i])
    edge = np.array([x for i in range(n) for x in sorted(adj[i])], dtype=np.int32)
    degs = sorted((len(a) for a in adj), reverse=True) + [0, 0]
    return CSR(vertex, edge, degs[0], degs[1])


def _splitmix64(x: np.ndarray) -> np.ndarray:
    """splitmix64 finaliser over a uint64 array (counter-based, so the labels
    of a graph do not depend on numpy's generator streams)."""
    with np.errstate(over="ignore"):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def zipf_labels(n: int, n_labels: int, s: float, seed: int) -> np.ndarray:
    """n labels drawn i.i.d. from Zipf(s) over 0..n_labels-1 (label k with
    weight (k+1)^-s)."""
    idx = np.arange(n, dtype=np.uint64) + np.uint64((seed * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF)
    u = (_splitmix64(idx) >> np.uint64(11)).astype(np.float64) / float(1 << 53)
    w = np.arange(1, n_labels + 1, dtype=np.float64) ** (-s)
    cdf = np.cumsum(w) / w.sum()
    cdf[-1] = 1.0
    return np.minimum(np.searchsorted(cdf, u, side="right"), n_labels - 1).astype(np.uint32)


def labeled_rmat(scale: int, edge_factor: float, seed: int, keep: int, n_labels: int, zipf_s: float,
                 label_seed: int) -> tuple[CSR, np.ndarray]:
    """R-MAT graph restricted to the vertex ids below ``keep``, with Zipf
    labels: the labeled FSM input (symmetric, duplicate-free)."""
    g = rmat(scale, edge_factor, seed)
    if keep < g.v_cnt:
        g = restrict(g, keep)
    return g, zipf_labels(g.v_cnt, n_labels, zipf_s, label_seed)


def write_adj(path: str, g: CSR, labels: np.ndarray) -> None:
    """The reference's labeled text format: first line v_cnt, then one line
    per vertex "id label nbr nbr ..."."""
    with open(path, "w") as f:
        f.write(f"{g.v_cnt}\n")
        for v in range(g.v_cnt):
            nb = g.edge[g.vertex[v]:g.vertex[v + 1]]
            f.write(f"{v} {int(labels[v])} " + " ".join(map(str, nb.tolist())) + "\n")
