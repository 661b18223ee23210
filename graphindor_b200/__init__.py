"""graphindor_b200: a B200-native graph pattern-counting engine.

Python mirror of the reference's host interface (Pattern, Schedule_IEP,
Graph and the pattern_matching / clique / motif entry points) over the C ABI
in include/gi.h.  Every count runs in the CUDA library; there is no CPU
fallback: if the library or a GPU is missing, the calls raise.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _native as N
from ._native import GIError, check, lib

__all__ = ["Pattern", "Schedule_IEP", "Graph", "pattern_matching", "clique_count", "motif_counting",
           "motif_patterns", "GIError", "lib", "write_g", "read_g", "LabeledGraph", "fsm", "fsm_plan",
           "FsmResult", "PATENTS_TRI_CNT", "YOUTUBE_TRI_CNT", "Batch", "load_cost_model", "autotune",
           "autotune_clear"]


class Pattern:
    """n-vertex pattern from the reference's n*n '0'/'1' string (reference
    src/pattern.cpp:22-31: any '1' at (i, j) adds the undirected edge)."""

    def __init__(self, size: int, adj: str):
        if len(adj) < size * size:
            raise ValueError("adjacency string shorter than size*size")
        self.size = size
        m = np.zeros((size, size), dtype=np.int32)
        for i in range(size):
            for j in range(size):
                if adj[i * size + j] == "1":
                    m[i, j] = m[j, i] = 1
        self.adj = m

    @property
    def adj_string(self) -> str:
        return "".join("1" if x else "0" for x in self.adj.reshape(-1))

    @classmethod
    def clique(cls, k: int) -> "Pattern":
        return cls(k, "".join("0" if i == j else "1" for i in range(k) for j in range(k)))


class Schedule_IEP:
    """Immutable plan (reference include/schedule_IEP.h).  model=1 picks the
    vertex order with the reference's analytic model from the graph's
    v_cnt / e_cnt / tri_cnt; ``order``/``restricts`` give a schedule
    explicitly; ``vertex_induced`` mirrors Schedule_IEP(adj_mat, size)."""

    def __init__(self, pattern: Pattern, v_cnt: int = 0, e_cnt: int = 0, tri_cnt: int = 0, *,
                 model: int = 1, enable_iep: bool = True, order: Optional[Sequence[int]] = None,
                 restricts: Optional[Sequence[Sequence[int]]] = None, vertex_induced: bool = False):
        L = lib()
        h = C.c_void_p()
        adj = pattern.adj_string.encode()
        if vertex_induced:
            check(L.gi_plan_create_induced(pattern.size, adj, C.byref(h)), "gi_plan_create_induced")
        elif order is not None:
            o = (C.c_int32 * pattern.size)(*order)
            rs = list(restricts or [])
            r = (C.c_int32 * max(1, 2 * len(rs)))(*[x for p in rs for x in p])
            check(L.gi_plan_create_explicit(pattern.size, adj, o, r, len(rs), int(enable_iep), C.byref(h)),
                  "gi_plan_create_explicit")
        else:
            check(L.gi_plan_create(pattern.size, adj, int(v_cnt), int(e_cnt), int(tri_cnt), int(model),
                                   int(enable_iep), C.byref(h)), "gi_plan_create")
        self._h = h
        self.pattern = pattern

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().gi_plan_destroy(h)
            self._h = None

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def export(self) -> dict:
        d = N.PlanDesc()
        check(lib().gi_plan_export(self._h, C.byref(d)), "gi_plan_export")
        n, tp = d.size, d.total_prefix_num
        nr = d.total_restrict_num
        out = {
            "size": n,
            "adj_mat": list(d.adj_mat[: n * n]),
            "order": list(d.order[:n]),
            "total_prefix_num": tp,
            "basic_prefix_num": d.basic_prefix_num,
            "father_prefix_id": list(d.father_prefix_id[:tp]),
            "last": list(d.last[:n]),
            "next": list(d.next[:tp]),
            "loop_set_prefix_id": list(d.loop_set_prefix_id[:n]),
            "break_size": list(d.break_size[:tp]),
            "only_need_size": list(d.only_need_size[:tp]),
            "prefix_data": [list(d.prefix_data[i][: d.prefix_len[i]]) for i in range(tp)],
            "total_restrict_num": nr,
            "restrict_last": list(d.restrict_last[:n]),
            "restrict_next": list(d.restrict_next[:nr]),
            "restrict_index": list(d.restrict_index[:nr]),
            "restrict_pair": [list(d.restrict_pairs[i]) for i in range(d.n_restrict_pairs)],
            "in_exclusion_optimize_num": d.in_exclusion_optimize_num,
            "iep_vertex_id": list(d.iep_vertex_id[: d.iep_vertex_id_size]),
            "iep_vertex_flag_eff": list(d.iep_vertex_flag[: d.iep_vertex_id_size]),
            "iep_vertex_coef_eff": list(d.iep_vertex_coef[: d.iep_vertex_id_size]),
            "iep_coef": list(d.iep_coef[: d.iep_term_count]),
            "iep_flag": list(d.iep_flag[: d.iep_term_count]),
            "iep_ans_pos_eff": list(d.iep_ans_pos[: d.iep_term_count]),
            "is_vertex_induced": d.is_vertex_induced,
            "redundancy": d.redundancy,
            "k_val": d.k_val,
            "multiplicity": d.multiplicity,
            "model_cost": d.model_cost,
            "iep_tables_rebuilt": d.iep_tables_rebuilt,
            "count_divisor": d.count_divisor,
            "exact": d.exact,
        }
        for which, key in ((0, "iep_vertex_flag"), (1, "iep_vertex_coef"), (2, "iep_ans_pos")):
            n_raw = C.c_int64()
            check(lib().gi_plan_export_raw(self._h, which, None, 0, C.byref(n_raw)), "gi_plan_export_raw")
            buf = (C.c_int32 * max(1, n_raw.value))()
            check(lib().gi_plan_export_raw(self._h, which, buf, n_raw.value, C.byref(n_raw)), "gi_plan_export_raw")
            out[key] = list(buf[: n_raw.value])
        return out

    @property
    def variant(self) -> dict:
        """The plan's kernel variant (speed only, never counts)."""
        v = N.Variant()
        check(lib().gi_plan_get_variant(self._h, C.byref(v)), "gi_plan_get_variant")
        return {k: getattr(v, k) for k, _ in N.Variant._fields_}

    @variant.setter
    def variant(self, v: dict) -> None:
        cur = self.variant
        cur.update(v)
        check(lib().gi_plan_set_variant(self._h, C.byref(N.Variant(**cur))), "gi_plan_set_variant")

    @classmethod
    def learned(cls, pattern: Pattern, graph: "Graph", enable_iep: bool = True,
                model_path: Optional[str] = None) -> "Schedule_IEP":
        """Of the analytic model's GI_LEARNED_CANDIDATES best valid candidate
        schedules, the one with the smallest device time the learned cost
        model predicts on `graph` (exact counts).  Loads the package's trained
        model on first use unless model_path is given."""
        L = lib()
        load_cost_model(model_path)
        feats = (C.c_float * N.GI_GRAPH_FEATURES)()
        check(L.gi_graph_features(graph.handle, feats, N.GI_GRAPH_FEATURES), "gi_graph_features")
        h = C.c_void_p()
        pred = C.c_double()
        check(L.gi_plan_create_learned(pattern.size, pattern.adj_string.encode(), graph.v_cnt, graph.e_cnt,
                                       graph.tri_cnt, feats, int(enable_iep), C.byref(h), C.byref(pred)),
              "gi_plan_create_learned")
        obj = cls.__new__(cls)
        obj._h = h
        obj.pattern = pattern
        obj.predicted_ms = pred.value
        return obj

    @staticmethod
    def candidates(pattern: Pattern, v_cnt: int, e_cnt: int, tri_cnt: int, enable_iep: bool = True):
        """(order, restricts, analytic cost, exact divisor or 0 if the
        restriction set is invalid) in the reference model's order."""
        L = lib()
        adj = pattern.adj_string.encode()
        cnt = C.c_int64()
        check(L.gi_plan_candidates(pattern.size, adj, v_cnt, e_cnt, tri_cnt, int(enable_iep), None, None, None,
                                   None, None, 0, C.byref(cnt)), "gi_plan_candidates")
        m, n = cnt.value, pattern.size
        orders = (C.c_int32 * max(1, m * n))()
        rs = (C.c_int32 * max(1, m * N.GI_MAX_PREFIX * 2))()
        nr = (C.c_int32 * max(1, m))()
        costs = (C.c_double * max(1, m))()
        divs = (C.c_int32 * max(1, m))()
        check(L.gi_plan_candidates(pattern.size, adj, v_cnt, e_cnt, tri_cnt, int(enable_iep), orders, rs, nr,
                                   costs, divs, m, C.byref(cnt)), "gi_plan_candidates")
        out = []
        for i in range(m):
            r = [(rs[(i * N.GI_MAX_PREFIX + j) * 2], rs[(i * N.GI_MAX_PREFIX + j) * 2 + 1]) for j in range(nr[i])]
            out.append((list(orders[i * n:(i + 1) * n]), r, costs[i], divs[i]))
        return out


def autotune(graph: "Graph", schedule: Schedule_IEP, *, sample_edges: int = 0, max_ms: float = 0.0, reps: int = 0,
             use_cache: bool = True, quick: bool = False, lookup_only: bool = False, stream: int = 0) -> dict:
    """Times the kernel variants of `schedule` on a sample of `graph` and
    keeps the fastest in the plan (gi_autotune); the choice is cached for the
    class of (plan, graph), and batches apply cached choices to their jobs."""
    o = N.TuneOptions(int(sample_edges), float(max_ms), int(reps), int(use_cache), int(quick), int(lookup_only))
    info = N.TuneInfo()
    check(lib().gi_autotune(graph.handle, schedule.handle, C.c_void_p(stream) if stream else None, C.byref(o),
                            C.byref(info)), "gi_autotune")
    c = info.chosen
    return {"chosen": {k: getattr(c, k) for k, _ in N.Variant._fields_},
            "cached": bool(info.cached), "candidates": info.candidates, "best_ms": info.best_ms,
            "default_ms": info.default_ms, "sample_edges": info.sample_edges}


def autotune_clear() -> None:
    check(lib().gi_autotune_clear(), "gi_autotune_clear")


COST_MODEL_PATH = __import__("pathlib").Path(__file__).resolve().parent / "schedule_cost" / "weights.bin"
_cost_model_loaded: Optional[str] = None


def load_cost_model(path: Optional[str] = None) -> None:
    """Loads the learned schedule cost model (default: the trained weights
    shipped in the package) once per process."""
    global _cost_model_loaded
    p = str(path or COST_MODEL_PATH)
    if _cost_model_loaded != p:
        check(lib().gi_cost_model_load(p.encode()), "gi_cost_model_load")
        _cost_model_loaded = p


@dataclass
class CountResult:
    count: int
    kernel_ms: float
    raw_sum: int
    tasks: int
    alg_bytes: int
    grid_blocks: int
    block_threads: int
    kernel_launches: int


def _stats(count_bytes: bool, budget_ms: float = 0.0) -> N.Stats:
    s = N.Stats()
    s.count_bytes = 1 if count_bytes else 0
    s.budget_ms = float(budget_ms)
    return s


def _result(count: int, s: N.Stats) -> CountResult:
    return CountResult(int(count), s.kernel_ms, int(s.raw_sum), int(s.tasks), int(s.alg_bytes), s.grid_blocks,
                       s.block_threads, s.kernel_launches)


class Graph:
    """CSR graph resident on the current CUDA device (reference
    include/graph.h:12-33).  ``vertex`` int64[v_cnt+1], ``edge`` int32[e_cnt]
    with sorted, duplicate-free adjacency lists and both directions present."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle
        info = N.GraphInfo()
        check(lib().gi_graph_get_info(handle, C.byref(info)), "gi_graph_get_info")
        self.v_cnt = info.v_cnt
        self.e_cnt = info.e_cnt
        self.tri_cnt = info.tri_cnt
        self.max_degree = info.max_degree
        self.max_intersection_size = info.max_intersection_size
        self.n_hubs = info.n_hubs
        self.hub_min_degree = info.hub_min_degree
        self.hash_min_degree = info.hash_min_degree
        self.hash_slots = info.hash_slots

    @classmethod
    def from_csr(cls, vertex: np.ndarray, edge: np.ndarray, tri_cnt: int = 0, stream: int = 0) -> "Graph":
        vertex = np.ascontiguousarray(vertex, dtype=np.int64)
        edge = np.ascontiguousarray(edge, dtype=np.int32)
        h = C.c_void_p()
        check(lib().gi_graph_create(vertex.ctypes.data, edge.ctypes.data if edge.size else None,
                                    len(vertex) - 1, len(edge), int(tri_cnt), C.c_void_p(stream) if stream else None,
                                    C.byref(h)), "gi_graph_create")
        return cls(h)

    @classmethod
    def load_g(cls, path: str) -> "Graph":
        h = C.c_void_p()
        check(lib().gi_graph_load_g(str(path).encode(), C.byref(h)), "gi_graph_load_g")
        return cls(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().gi_graph_destroy(h)
            self._h = None

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def plan(self, pattern: Pattern, enable_iep: bool = True, model: int = 1) -> Schedule_IEP:
        return Schedule_IEP(pattern, self.v_cnt, self.e_cnt, self.tri_cnt, model=model, enable_iep=enable_iep)


def pattern_matching(graph: Graph, schedule: Schedule_IEP, *, count_bytes: bool = False, budget_ms: float = 0.0,
                     stream: int = 0) -> CountResult:
    """Count of the schedule's pattern (gpu_graph semantics: raw sum modulo
    2^64 divided by the redundancy)."""
    out = C.c_uint64()
    s = _stats(count_bytes, budget_ms)
    check(lib().gi_count(graph.handle, schedule.handle, C.c_void_p(stream) if stream else None, C.byref(out),
                         C.byref(s)), "gi_count")
    return _result(out.value, s)


def count_edges(graph: Graph, schedule: Schedule_IEP, edge_step: int, edge_offset: int = 0, *, shard: int = 0,
                num_shards: int = 1, count_bytes: bool = False, stream: int = 0) -> N.Stats:
    """Raw sum (modulo 2^64, not divided) of the first-level tasks of the
    directed edges e with e % edge_step == edge_offset (gi_count_shard's edge
    subset): the reference's per-edge task summed over exactly those edges.
    Returns the gi_stats of the call (raw_sum, kernel_ms, chunks, ...)."""
    s = _stats(count_bytes)
    s.edge_step = int(edge_step)
    s.edge_offset = int(edge_offset)
    raw = C.c_uint64()
    check(lib().gi_count_shard(graph.handle, schedule.handle, int(shard), int(num_shards),
                               C.c_void_p(stream) if stream else None, C.byref(raw), C.byref(s)), "gi_count_shard")
    return s


def clique_count(graph: Graph, k: int, orientation: int = 0, *, count_bytes: bool = False,
                 stream: int = 0) -> CountResult:
    out = C.c_uint64()
    s = _stats(count_bytes)
    check(lib().gi_clique_count(graph.handle, k, orientation, C.c_void_p(stream) if stream else None,
                                C.byref(out), C.byref(s)), "gi_clique_count")
    return _result(out.value, s)


def clique_counts_pivot(graph: Graph, kmax: int, *, stream: int = 0, with_stats: bool = False):
    """k-clique counts for every k in [1, kmax] (index k; index 0 is 0) at
    once, by clique-tree pivoting on the degree-oriented DAG's bitmaps.  With
    with_stats, (counts, gi_stats)."""
    out = (C.c_uint64 * (kmax + 1))()
    s = N.Stats()
    check(lib().gi_clique_counts_pivot(graph.handle, kmax, C.c_void_p(stream) if stream else None, out,
                                       C.byref(s)), "gi_clique_counts_pivot")
    counts = [int(x) for x in out]
    return (counts, s) if with_stats else counts


def motif_patterns(k: int) -> list[str]:
    L = lib()
    m = L.gi_motif_num(k)
    if m < 0:
        raise ValueError("motif size must be between 3 and 7")
    buf = C.create_string_buffer(m * k * k)
    check(L.gi_motif_patterns(k, buf, m), "gi_motif_patterns")
    raw = buf.raw
    return [raw[i * k * k:(i + 1) * k * k].decode() for i in range(m)]


def motif_counting(graph: Graph, k: int, *, stream: int = 0, budget_ms: float = 0.0) -> tuple[list[int], CountResult]:
    L = lib()
    m = L.gi_motif_num(k)
    out = (C.c_uint64 * max(1, m))()
    s = _stats(False, budget_ms)
    check(L.gi_motif_count(graph.handle, k, C.c_void_p(stream) if stream else None, out, m, C.byref(s)),
          "gi_motif_count")
    return [int(x) for x in out[:m]], _result(0, s)


def write_g(path: str, vertex: np.ndarray, edge: np.ndarray, max_isect: int, tri_cnt: int) -> None:
    vertex = np.ascontiguousarray(vertex, dtype=np.int64)
    edge = np.ascontiguousarray(edge, dtype=np.int32)
    check(lib().gi_g_write(str(path).encode(), vertex.ctypes.data, edge.ctypes.data if edge.size else None,
                           len(vertex) - 1, len(edge), int(max_isect), int(tri_cnt)), "gi_g_write")


def read_g(path: str):
    L = lib()
    v, e, mi, tri = C.c_int32(), C.c_int64(), C.c_uint32(), C.c_int64()
    check(L.gi_g_read_header(str(path).encode(), C.byref(v), C.byref(e), C.byref(mi), C.byref(tri)),
          "gi_g_read_header")
    vertex = np.empty(v.value + 1, dtype=np.int64)
    edge = np.empty(max(1, e.value), dtype=np.int32)
    check(L.gi_g_read(str(path).encode(), vertex.ctypes.data, edge.ctypes.data, v.value, e.value), "gi_g_read")
    return vertex, edge[: e.value], int(mi.value), int(tri.value)


# ------------------------------------------------------------ labeled graphs + FSM

PATENTS_TRI_CNT = 7515023      # the constant fsm_test plans with (reference include/dataloader.h:28)
YOUTUBE_TRI_CNT = 103017122    # the constant gpu_fsm plans with (reference include/dataloader.h:35)


class LabeledGraph:
    """Labeled graph in the reference loader's numbering (reference
    include/labeled_graph.h, src/dataloader.cpp:381-625): labels renamed by
    descending maximum degree, vertices sorted by (label, -degree, id), each
    neighbour list bucketed by neighbour label.  Built on the host; copied to
    the current device by the first :func:`fsm`."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle
        info = N.LabeledGraphInfo()
        check(lib().gi_labeled_graph_get_info(handle, C.byref(info)), "gi_labeled_graph_get_info")
        self.v_cnt, self.e_cnt, self.l_cnt = info.v_cnt, info.e_cnt, info.l_cnt

    @classmethod
    def from_csr(cls, vertex: np.ndarray, edge: np.ndarray, labels: np.ndarray,
                 order: Optional[np.ndarray] = None, device: bool = False, stream=None) -> "LabeledGraph":
        """``vertex``/``edge``: symmetric CSR in original ids; ``labels``:
        original label value per vertex; ``order``: the order of the vertex
        lines (default ascending id).  ``device``: build the renumbered,
        bucketed structure on the current GPU (gi_labeled_graph_create_device)
        instead of on the host; the result is the same."""
        vertex = np.ascontiguousarray(vertex, dtype=np.int64)
        edge = np.ascontiguousarray(edge, dtype=np.int32)
        labels = np.ascontiguousarray(labels, dtype=np.uint32)
        if order is not None:
            order = np.ascontiguousarray(order, dtype=np.int32)
        h = C.c_void_p()
        args = (len(vertex) - 1, vertex.ctypes.data, edge.ctypes.data if edge.size else None, labels.ctypes.data,
                order.ctypes.data if order is not None else None)
        if device:
            check(lib().gi_labeled_graph_create_device(*args, stream, C.byref(h)), "gi_labeled_graph_create_device")
        else:
            check(lib().gi_labeled_graph_create(*args, C.byref(h)), "gi_labeled_graph_create")
        return cls(h)

    @classmethod
    def load_adj(cls, path: str) -> "LabeledGraph":
        h = C.c_void_p()
        check(lib().gi_labeled_graph_load_adj(str(path).encode(), C.byref(h)), "gi_labeled_graph_load_adj")
        return cls(h)

    def export(self) -> dict:
        """Host copies of the renumbered structure."""
        v, l, e = self.v_cnt, self.l_cnt, self.e_cnt
        out = {"new_id": np.empty(v, np.int32), "v_label": np.empty(v, np.int32),
               "label_value": np.empty(l, np.uint32), "label_start": np.empty(l + 1, np.uint32),
               "bucket": np.empty(v * l + 1, np.uint32), "edge": np.empty(max(e, 1), np.uint32)}
        check(lib().gi_labeled_graph_export(self._h, *[out[k].ctypes.data for k in
                                                       ("new_id", "v_label", "label_value", "label_start",
                                                        "bucket", "edge")]), "gi_labeled_graph_export")
        out["edge"] = out["edge"][:e]
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().gi_labeled_graph_destroy(h)
            self._h = None

    @property
    def handle(self) -> C.c_void_p:
        return self._h


def _fsm_pattern(p: N.FsmPattern) -> dict:
    n = p.n
    return {"n": n, "edges": p.edges, "adj": p.adj[: n * n].decode(),
            "restricts": [(p.restricts[i][0], p.restricts[i][1]) for i in range(p.n_restricts)],
            "automorphisms": p.n_automorphisms, "jobs": p.jobs, "frequent": p.frequent, "kernel_ms": p.kernel_ms}


@dataclass
class FsmResult:
    count: int
    kernel_ms: float
    total_ms: float
    jobs: int
    candidates: int
    kernel_launches: int
    patterns: list


def fsm(graph: LabeledGraph, max_edge: int, min_support: int, tri_cnt: int = YOUTUBE_TRI_CNT, *,
        stream: int = 0) -> FsmResult:
    """Number of frequent labeled patterns with exactly ``max_edge`` edges
    under MNI support (gpu_fsm / LabeledGraph::fsm semantics).  ``tri_cnt``
    is the triangle count the planner is given (gpu_fsm uses YouTube's
    constant, fsm_test Patents')."""
    pats = (N.FsmPattern * N.GI_FSM_MAX_PATTERNS)()
    st = N.FsmStats()
    st.patterns = C.cast(pats, C.POINTER(N.FsmPattern))
    out = C.c_int64()
    check(lib().gi_fsm(graph.handle, max_edge, int(min_support), int(tri_cnt), C.c_void_p(stream) if stream else None,
                       C.byref(out), C.byref(st)), "gi_fsm")
    return FsmResult(out.value, st.kernel_ms, st.total_ms, st.jobs, st.candidates, st.kernel_launches,
                     [_fsm_pattern(pats[i]) for i in range(st.n_patterns)])


def fsm_plan(max_edge: int, v_cnt: int, e_cnt: int, tri_cnt: int = YOUTUBE_TRI_CNT) -> list[dict]:
    """The unlabeled patterns of an FSM run with their plans (schedule-order
    adjacency, label restrictions (d, r): label[d] <= label[r])."""
    pats = (N.FsmPattern * N.GI_FSM_MAX_PATTERNS)()
    cnt = C.c_int()
    check(lib().gi_fsm_plan(max_edge, v_cnt, e_cnt, tri_cnt, pats, N.GI_FSM_MAX_PATTERNS, C.byref(cnt)),
          "gi_fsm_plan")
    return [_fsm_pattern(pats[i]) for i in range(min(cnt.value, N.GI_FSM_MAX_PATTERNS))]


# ------------------------------------------------------------------ batches

class Batch:
    """Many (graph, plan) jobs counted in one persistent launch, captured in a
    CUDA graph on the first run and replayed afterwards."""

    def __init__(self, jobs: Sequence[tuple["Graph", "Schedule_IEP"]]):
        self._keep = list(jobs)  # the handles must outlive the batch
        n = len(self._keep)
        graphs = (C.c_void_p * n)(*[g.handle for g, _ in self._keep])
        plans = (C.c_void_p * n)(*[p.handle for _, p in self._keep])
        h = C.c_void_p()
        check(lib().gi_batch_create(graphs, plans, n, C.byref(h)), "gi_batch_create")
        self._h = h
        self.n_jobs = n

    def run(self, stream: int = 0):
        """(counts, per-job device ms from launch start to job end, kernel ms)."""
        counts = (C.c_uint64 * self.n_jobs)()
        ms = (C.c_double * self.n_jobs)()
        st = N.Stats()
        check(lib().gi_batch_run(self._h, C.c_void_p(stream) if stream else None, counts, ms, C.byref(st)),
              "gi_batch_run")
        return [int(x) for x in counts], [float(x) for x in ms], st.kernel_ms

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().gi_batch_destroy(h)
            self._h = None
