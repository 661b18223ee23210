"""ctypes binding of include/gi.h (the engine's C ABI).

The library is the in-tree build ``graphindor_b200/lib/libgraphindor_b200.so``;
importing this module never falls back to anything else: if the library is
missing, :func:`lib` raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libgraphindor_b200.so"

GI_MAX_PATTERN = 7
GI_MAX_PREFIX = 22
GI_MAX_IEP_SETS = 32
GI_MAX_IEP_TERMS = 160

GI_OK, GI_EINVAL, GI_ENOMEM, GI_ECUDA, GI_ETIMEOUT, GI_EOVERFLOW, GI_EIO, GI_ENOTSUP, GI_EDISCONNECTED = range(9)


class GraphInfo(C.Structure):
    _fields_ = [("v_cnt", C.c_int32), ("e_cnt", C.c_int64), ("tri_cnt", C.c_int64),
                ("max_degree", C.c_int32), ("max_intersection_size", C.c_int32), ("n_hubs", C.c_int32),
                ("hub_min_degree", C.c_int32), ("hash_min_degree", C.c_int32), ("hash_slots", C.c_int64)]


class PlanDesc(C.Structure):
    P, X, S, T = GI_MAX_PATTERN, GI_MAX_PREFIX, GI_MAX_IEP_SETS, GI_MAX_IEP_TERMS
    _fields_ = [
        ("size", C.c_int32),
        ("adj_mat", C.c_int32 * (P * P)),
        ("order", C.c_int32 * P),
        ("total_prefix_num", C.c_int32),
        ("basic_prefix_num", C.c_int32),
        ("father_prefix_id", C.c_int32 * X),
        ("last", C.c_int32 * P),
        ("next", C.c_int32 * X),
        ("loop_set_prefix_id", C.c_int32 * P),
        ("break_size", C.c_int32 * X),
        ("only_need_size", C.c_int32 * X),
        ("prefix_len", C.c_int32 * X),
        ("prefix_data", (C.c_int32 * P) * X),
        ("total_restrict_num", C.c_int32),
        ("restrict_last", C.c_int32 * P),
        ("restrict_next", C.c_int32 * X),
        ("restrict_index", C.c_int32 * X),
        ("n_restrict_pairs", C.c_int32),
        ("restrict_pairs", (C.c_int32 * 2) * X),
        ("in_exclusion_optimize_num", C.c_int32),
        ("iep_vertex_id_size", C.c_int32),
        ("iep_vertex_id", C.c_int32 * S),
        ("iep_vertex_flag", C.c_int32 * S),
        ("iep_vertex_coef", C.c_int32 * S),
        ("iep_term_count", C.c_int32),
        ("iep_coef", C.c_int32 * T),
        ("iep_flag", C.c_int32 * T),
        ("iep_ans_pos", C.c_int32 * T),
        ("iep_vertex_flag_raw_len", C.c_int64),
        ("iep_ans_pos_raw_len", C.c_int64),
        ("is_vertex_induced", C.c_int32),
        ("redundancy", C.c_int64),
        ("k_val", C.c_int32),
        ("multiplicity", C.c_int32),
        ("model_cost", C.c_double),
        ("iep_tables_rebuilt", C.c_int32),
        ("count_divisor", C.c_int64),
        ("exact", C.c_int32),
    ]


class Stats(C.Structure):
    _fields_ = [("kernel_ms", C.c_double), ("raw_sum", C.c_uint64), ("tasks", C.c_uint64),
                ("alg_bytes", C.c_uint64), ("count_bytes", C.c_int32), ("budget_ms", C.c_double),
                ("grid_blocks", C.c_int32), ("block_threads", C.c_int32), ("kernel_launches", C.c_int32),
                ("allow_partial", C.c_int32), ("chunks_done", C.c_int64), ("chunks_total", C.c_int64),
                ("prep_ms", C.c_double), ("sample_chunks", C.c_int64), ("edge_step", C.c_int64),
                ("edge_offset", C.c_int64)]


class Variant(C.Structure):
    _fields_ = [("leaf_flat", C.c_int32), ("lane_budget", C.c_int32), ("occupancy", C.c_int32), ("split", C.c_int32),
                ("leaf_handoff", C.c_int32), ("mid_handoff", C.c_int32), ("edge_triangles", C.c_int32)]


class TuneOptions(C.Structure):
    _fields_ = [("sample_edges", C.c_int64), ("max_ms", C.c_double), ("reps", C.c_int32), ("use_cache", C.c_int32),
                ("quick", C.c_int32), ("lookup_only", C.c_int32)]


class TuneInfo(C.Structure):
    _fields_ = [("chosen", Variant), ("cached", C.c_int32), ("candidates", C.c_int32), ("best_ms", C.c_double),
                ("default_ms", C.c_double), ("sample_edges", C.c_int64)]


class LabeledGraphInfo(C.Structure):
    _fields_ = [("v_cnt", C.c_int32), ("e_cnt", C.c_int64), ("l_cnt", C.c_int32), ("device", C.c_int32)]


GI_FSM_MAX_PATTERNS = 64
GI_GRAPH_FEATURES = 19
GI_LEARNED_CANDIDATES = 16  # the analytic model's best valid candidates that the learned model re-ranks


class FsmPattern(C.Structure):
    _fields_ = [("n", C.c_int32), ("edges", C.c_int32), ("adj", C.c_char * (GI_MAX_PATTERN * GI_MAX_PATTERN)),
                ("n_restricts", C.c_int32), ("restricts", (C.c_int32 * 2) * 21), ("n_automorphisms", C.c_int32),
                ("jobs", C.c_int64), ("frequent", C.c_int64), ("kernel_ms", C.c_double)]


class FsmStats(C.Structure):
    _fields_ = [("kernel_ms", C.c_double), ("total_ms", C.c_double), ("jobs", C.c_int64),
                ("candidates", C.c_int64), ("kernel_launches", C.c_int32), ("n_patterns", C.c_int32),
                ("patterns", C.POINTER(FsmPattern))]


# name -> (restype, argtypes)
_SIGS = {
    "gi_status_string": (C.c_char_p, [C.c_int]),
    "gi_last_error": (C.c_char_p, []),
    "gi_version": (C.c_int, []),
    "gi_graph_create": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_int64, C.c_void_p,
                                  C.POINTER(C.c_void_p)]),
    "gi_graph_load_g": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "gi_graph_destroy": (C.c_int, [C.c_void_p]),
    "gi_graph_get_info": (C.c_int, [C.c_void_p, C.POINTER(GraphInfo)]),
    "gi_g_write": (C.c_int, [C.c_char_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_uint32, C.c_int64]),
    "gi_g_read_header": (C.c_int, [C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                                   C.POINTER(C.c_uint32), C.POINTER(C.c_int64)]),
    "gi_g_read": (C.c_int, [C.c_char_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int64]),
    "gi_plan_create": (C.c_int, [C.c_int, C.c_char_p, C.c_int32, C.c_int64, C.c_int64, C.c_int, C.c_int,
                                 C.POINTER(C.c_void_p)]),
    "gi_plan_create_explicit": (C.c_int, [C.c_int, C.c_char_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                          C.POINTER(C.c_void_p)]),
    "gi_plan_create_induced": (C.c_int, [C.c_int, C.c_char_p, C.POINTER(C.c_void_p)]),
    "gi_plan_destroy": (C.c_int, [C.c_void_p]),
    "gi_plan_export": (C.c_int, [C.c_void_p, C.POINTER(PlanDesc)]),
    "gi_plan_export_raw": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]),
    "gi_plan_candidates": (C.c_int, [C.c_int, C.c_char_p, C.c_int32, C.c_int64, C.c_int64, C.c_int,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                     C.POINTER(C.c_int64)]),
    "gi_count": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(Stats)]),
    "gi_count_shard": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.POINTER(C.c_uint64),
                                 C.POINTER(Stats)]),
    "gi_clique_count": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_uint64),
                                  C.POINTER(Stats)]),
    "gi_clique_counts_pivot": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(Stats)]),
    "gi_motif_num": (C.c_int, [C.c_int]),
    "gi_motif_patterns": (C.c_int, [C.c_int, C.c_char_p, C.c_int]),
    "gi_motif_count": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(Stats)]),
    "gi_labeled_graph_create": (C.c_int, [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.POINTER(C.c_void_p)]),
    "gi_labeled_graph_create_device": (C.c_int, [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                 C.c_void_p, C.POINTER(C.c_void_p)]),
    "gi_labeled_graph_load_adj": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "gi_plan_get_variant": (C.c_int, [C.c_void_p, C.POINTER(Variant)]),
    "gi_plan_set_variant": (C.c_int, [C.c_void_p, C.POINTER(Variant)]),
    "gi_autotune": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(TuneOptions), C.POINTER(TuneInfo)]),
    "gi_autotune_clear": (C.c_int, []),
    "gi_labeled_graph_destroy": (C.c_int, [C.c_void_p]),
    "gi_labeled_graph_get_info": (C.c_int, [C.c_void_p, C.POINTER(LabeledGraphInfo)]),
    "gi_labeled_graph_export": (C.c_int, [C.c_void_p] + [C.c_void_p] * 6),
    "gi_fsm": (C.c_int, [C.c_void_p, C.c_int, C.c_int64, C.c_int64, C.c_void_p, C.POINTER(C.c_int64),
                         C.POINTER(FsmStats)]),
    "gi_fsm_plan": (C.c_int, [C.c_int, C.c_int32, C.c_int64, C.c_int64, C.POINTER(FsmPattern), C.c_int,
                              C.POINTER(C.c_int)]),
    "gi_cost_model_load": (C.c_int, [C.c_char_p]),
    "gi_batch_create": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "gi_mlp_grad": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                              C.POINTER(C.c_float)]),
    "gi_mlp_predict": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "gi_mlp_train": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                               C.c_float, C.c_uint64, C.c_void_p, C.POINTER(C.c_float)]),
    "gi_batch_run": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Stats)]),
    "gi_batch_destroy": (C.c_int, [C.c_void_p]),
    "gi_graph_features": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "gi_graph_features_host": (C.c_int, [C.c_void_p, C.c_int32, C.c_int64, C.c_void_p, C.c_int]),
    "gi_plan_create_learned": (C.c_int, [C.c_int, C.c_char_p, C.c_int32, C.c_int64, C.c_int64, C.c_void_p, C.c_int,
                                         C.POINTER(C.c_void_p), C.POINTER(C.c_double)]),
}

_lib = None


def lib() -> C.CDLL:
    """Loads the in-tree library once; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m graphindor_b200.build`")
        handle = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(handle, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


class GIError(RuntimeError):
    def __init__(self, status: int, where: str):
        L = lib()
        msg = L.gi_last_error().decode(errors="replace")
        super().__init__(f"{where}: {L.gi_status_string(status).decode()} ({msg})")
        self.status = status


def check(status: int, where: str) -> None:
    if status != GI_OK:
        raise GIError(status, where)
