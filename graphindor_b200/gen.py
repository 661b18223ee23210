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
