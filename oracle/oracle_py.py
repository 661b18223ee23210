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
        L.oracle_count_edges_timed.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_int,
                                               C.c_double, C.POINTER(C.c_uint64), C.POINTER(C.c_int64)]
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


def count_edges_timed(plan_desc, vertex, edge, stride, max_seconds=0.0, threads=0):
    """(raw sum, edges counted) over every stride-th directed edge."""
    vertex, edge = _arrays(vertex, edge)
    raw, done = C.c_uint64(), C.c_int64()
    rc = lib().oracle_count_edges_timed(C.byref(plan_desc), vertex.ctypes.data, edge.ctypes.data, len(vertex) - 1,
                                        stride, threads, max_seconds, C.byref(raw), C.byref(done))
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


def triangles(vertex, edge, threads=0):
    vertex, edge = _arrays(vertex, edge)
    return lib().oracle_triangles(vertex.ctypes.data, edge.ctypes.data, len(vertex) - 1, threads)
