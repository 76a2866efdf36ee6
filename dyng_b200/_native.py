"""ctypes binding of the C ABI in include/dyngb200.h (dyng_b200/libdyngb200.so).

There is no fallback: if the CUDA library is missing, importing the package's compute paths
raises NativeLibraryError.  Build it with ``python -m dyng_b200.build``.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdyngb200.so")

c_i32p = ctypes.POINTER(ctypes.c_int32)
c_i64p = ctypes.POINTER(ctypes.c_int64)
c_u8p = ctypes.POINTER(ctypes.c_uint8)
c_f32p = ctypes.POINTER(ctypes.c_float)
c_f64p = ctypes.POINTER(ctypes.c_double)
c_void_p = ctypes.c_void_p


class NativeLibraryError(ImportError):
    pass


class Props(ctypes.Structure):
    _fields_ = [("directed", ctypes.c_int32), ("sorted", ctypes.c_int32),
                ("allow_multi", ctypes.c_int32), ("on_existing_insert", ctypes.c_int32),
                ("on_missing_delete", ctypes.c_int32), ("on_self_loop", ctypes.c_int32),
                ("deletions_first", ctypes.c_int32), ("allow_vertex_growth", ctypes.c_int32),
                ("headroom", ctypes.c_double)]


class Batch(ctypes.Structure):
    _fields_ = [("insert_src", c_i32p), ("insert_dst", c_i32p), ("insert_weights", c_i32p),
                ("num_insertions", ctypes.c_int64), ("delete_src", c_i32p),
                ("delete_dst", c_i32p), ("num_deletions", ctypes.c_int64),
                ("num_weights", ctypes.c_int32), ("memory", ctypes.c_int32)]


class ApplySummary(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in (
        "inserted_edges", "deleted_edges", "updated_edges", "ignored_insertions",
        "ignored_deletions", "dropped_self_loops", "inserted_vertices", "num_vertices_after")]


class Stats(ctypes.Structure):
    _fields_ = [("batch", ApplySummary), ("invalidated", ctypes.c_int64),
                ("affected", ctypes.c_int64), ("iterations", ctypes.c_int64),
                ("epochs", ctypes.c_int64), ("pushes", ctypes.c_int64),
                ("packed_parents", ctypes.c_int32), ("engine_used", ctypes.c_int32),
                ("delta", ctypes.c_int64), ("max_weight", ctypes.c_int64),
                ("grid_blocks", ctypes.c_int32), ("invalidation", ctypes.c_int32),
                ("apply_ms", ctypes.c_float), ("sssp_ms", ctypes.c_float),
                ("rounds", ctypes.c_int64), ("touched", ctypes.c_int64),
                ("work", ctypes.c_int64 * 32), ("phase_ms", ctypes.c_float * 7),
                ("trace_len", ctypes.c_int32), ("trace_light", ctypes.c_int32 * 64),
                ("trace_heavy", ctypes.c_int32 * 64), ("trace_us", ctypes.c_float * 64),
                ("features", ctypes.c_float * 12), ("schedule_classes", ctypes.c_int32 * 3),
                ("kernel_launches", ctypes.c_int64), ("pj_round_us", ctypes.c_float * 24),
                ("pj_done_us", ctypes.c_float * 24), ("apply_step_us", ctypes.c_float * 12),
                ("host_us", ctypes.c_float * 4)]


class Options(ctypes.Structure):
    _fields_ = [("delta", ctypes.c_int64), ("objective", ctypes.c_int32),
                ("cuda_engine", ctypes.c_int32), ("validate_inputs", ctypes.c_int32)]


class Schedule(ctypes.Structure):
    _fields_ = [("delta", ctypes.c_int64), ("grid_blocks", ctypes.c_int32),
                ("invalidation", ctypes.c_int32), ("small_frontier", ctypes.c_int32),
                ("heavy_degree", ctypes.c_int32), ("record_features", ctypes.c_int32)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("max_group", ctypes.c_int32),
                ("small_changes", ctypes.c_int64), ("hbm_reserve_bytes", ctypes.c_int64),
                ("lanes", ctypes.c_int32)]


class RequestTimes(ctypes.Structure):
    _fields_ = [("queued_ms", ctypes.c_double), ("service_ms", ctypes.c_double),
                ("total_ms", ctypes.c_double), ("group_size", ctypes.c_int32),
                ("begin_ms", ctypes.c_double), ("round_ms", ctypes.c_double),
                ("copy_ms", ctypes.c_double), ("lane", ctypes.c_int32)]


class GraphStorage(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in (
        "vertex_capacity", "arena_slots", "out_top", "in_top", "out_garbage", "in_garbage",
        "index_slots", "arena_growths", "compactions", "index_builds")] + [
        (n, ctypes.c_double) for n in ("grow_ms", "compact_ms", "index_ms", "maintenance_ms_max")]


class MospOptions(ctypes.Structure):
    _fields_ = [("num_objectives", ctypes.c_int32), ("num_preferences", ctypes.c_int32),
                ("preferences", ctypes.POINTER(ctypes.c_int32)), ("delta", ctypes.c_int64),
                ("compute_path_costs", ctypes.c_int32), ("validate_inputs", ctypes.c_int32)]


class MospStats(ctypes.Structure):
    _fields_ = [("batch", ApplySummary), ("affected", ctypes.c_int64),
                ("combined_edges", ctypes.c_int64), ("preference_scale", ctypes.c_int64),
                ("iterations", ctypes.c_int64), ("converged", ctypes.c_int32),
                ("combine_ms", ctypes.c_float), ("solve_ms", ctypes.c_float),
                ("costs_ms", ctypes.c_float)]


class ServerInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("submitted", "completed", "failed", "rounds",
                                              "max_group", "waiting", "admission_us_max",
                                              "lanes", "large_rounds")]


# Every symbol of include/dyngb200.h with (restype, argtypes).
class TestHooks(ctypes.Structure):
    """dyngb200_test_hooks: host-side failure injection for the tests (no GPU fault)."""

    _fields_ = [("barrier_timeout_ns", ctypes.c_int64), ("barrier_extra_arrivals", ctypes.c_int32),
                ("no_cooperative_launch", ctypes.c_int32), ("barrier_kernel", ctypes.c_int32)]


SIGNATURES = {
    "dyngb200_last_error_message": (ctypes.c_char_p, []),
    "dyngb200_status_name": (ctypes.c_char_p, [ctypes.c_int]),
    "dyngb200_abi_version": (ctypes.c_int, []),
    "dyngb200_context_create": (ctypes.c_int, [ctypes.c_int, c_void_p, ctypes.POINTER(c_void_p)]),
    "dyngb200_context_destroy": (ctypes.c_int, [c_void_p]),
    "dyngb200_context_synchronize": (ctypes.c_int, [c_void_p]),
    "dyngb200_context_set_test_hooks": (ctypes.c_int, [c_void_p, ctypes.POINTER(TestHooks)]),
    "dyngb200_debug_device_allocations": (ctypes.c_int, [c_i64p]),
    "dyngb200_debug_fail_device_allocation": (ctypes.c_int, [ctypes.c_int64]),
    "dyngb200_props_default": (None, [ctypes.POINTER(Props)]),
    "dyngb200_props_mosp_compatible": (None, [ctypes.POINTER(Props)]),
    "dyngb200_graph_from_edges": (ctypes.c_int, [c_void_p, ctypes.c_int64, c_i32p, c_i32p, c_i32p,
                                                 ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                                                 ctypes.POINTER(Props), ctypes.POINTER(c_void_p)]),
    "dyngb200_graph_from_csr": (ctypes.c_int, [c_void_p, ctypes.c_int64, c_i64p, c_i32p, c_i32p,
                                               ctypes.c_int32, ctypes.c_int32,
                                               ctypes.POINTER(Props), ctypes.POINTER(c_void_p)]),
    "dyngb200_graph_destroy": (ctypes.c_int, [c_void_p]),
    "dyngb200_graph_info": (ctypes.c_int, [c_void_p, c_i64p, c_i64p, c_i32p,
                                           ctypes.POINTER(ctypes.c_uint64)]),
    "dyngb200_graph_apply": (ctypes.c_int, [c_void_p, c_void_p, ctypes.POINTER(Batch),
                                            ctypes.POINTER(ApplySummary)]),
    "dyngb200_graph_apply_classified": (ctypes.c_int, [c_void_p, c_void_p, ctypes.POINTER(Batch),
                                                       ctypes.POINTER(ApplySummary), c_u8p]),
    "dyngb200_graph_to_csr": (ctypes.c_int, [c_void_p, c_void_p, c_i64p, c_i32p, c_i32p, c_i64p,
                                             c_i32p, c_i32p]),
    "dyngb200_graph_device_bytes": (ctypes.c_int, [c_void_p, c_i64p]),
    "dyngb200_scheduler_set_feature_range": (ctypes.c_int, [c_void_p, c_f32p, c_f32p]),
    "dyngb200_scheduler_get_feature_range": (ctypes.c_int, [c_void_p, c_f32p, c_f32p,
                                                            ctypes.POINTER(ctypes.c_int32)]),
    "dyngb200_mosp_compute": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int32,
                                             ctypes.POINTER(MospOptions), ctypes.POINTER(c_void_p)]),
    "dyngb200_mosp_from_arrays": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int32, ctypes.c_int32,
                                                 ctypes.POINTER(c_i64p), ctypes.POINTER(c_i32p),
                                                 ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                                                 ctypes.POINTER(MospOptions),
                                                 ctypes.POINTER(c_void_p)]),
    "dyngb200_mosp_update": (ctypes.c_int, [c_void_p, c_void_p, ctypes.POINTER(Batch), c_void_p,
                                            ctypes.POINTER(MospStats), ctypes.POINTER(Stats)]),
    "dyngb200_mosp_destroy": (ctypes.c_int, [c_void_p]),
    "dyngb200_mosp_info": (ctypes.c_int, [c_void_p, ctypes.POINTER(ctypes.c_int32), c_i64p, c_i64p,
                                          ctypes.POINTER(ctypes.c_int32),
                                          ctypes.POINTER(ctypes.c_uint64)]),
    "dyngb200_mosp_tree": (ctypes.c_int, [c_void_p, ctypes.c_int32, ctypes.POINTER(c_void_p)]),
    "dyngb200_mosp_combined": (ctypes.c_int, [c_void_p, c_i64p, c_i32p, ctypes.c_int32]),
    "dyngb200_mosp_path_costs": (ctypes.c_int, [c_void_p, c_i64p]),
    "dyngb200_mosp_path_costs_columns": (ctypes.c_int, [c_void_p, c_void_p, c_void_p,
                                                        ctypes.c_int32, c_i64p]),
    "dyngb200_mosp_set_options": (ctypes.c_int, [c_void_p, ctypes.POINTER(MospOptions)]),
    "dyngb200_graph_storage_get": (ctypes.c_int, [c_void_p, ctypes.POINTER(GraphStorage)]),
    "dyngb200_sssp_compute": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int32,
                                             ctypes.POINTER(Options), ctypes.POINTER(c_void_p),
                                             ctypes.POINTER(Stats)]),
    "dyngb200_sssp_compute_static_scratch": (ctypes.c_int, [c_void_p, ctypes.c_int32,
                                                            ctypes.c_int32, ctypes.c_int64, c_i64p,
                                                            c_i32p, c_void_p]),
    "dyngb200_sssp_update": (ctypes.c_int, [c_void_p, c_void_p, ctypes.POINTER(Batch), c_void_p,
                                            ctypes.POINTER(Stats)]),
    "dyngb200_sssp_update_scheduled": (ctypes.c_int, [c_void_p, c_void_p, ctypes.POINTER(Batch),
                                                      c_void_p, ctypes.POINTER(Schedule),
                                                      ctypes.POINTER(Stats)]),
    "dyngb200_tree_from_arrays": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int32, c_i64p,
                                                 c_i32p, ctypes.c_int64, ctypes.c_int32,
                                                 ctypes.c_int32, ctypes.POINTER(Options),
                                                 ctypes.POINTER(c_void_p)]),
    "dyngb200_tree_clone": (ctypes.c_int, [c_void_p, c_void_p, ctypes.POINTER(c_void_p)]),
    "dyngb200_tree_destroy": (ctypes.c_int, [c_void_p]),
    "dyngb200_tree_distances": (ctypes.c_int, [c_void_p, c_void_p, c_i64p, ctypes.c_int32]),
    "dyngb200_tree_parents": (ctypes.c_int, [c_void_p, c_void_p, c_i32p, ctypes.c_int32]),
    "dyngb200_tree_device_arrays": (ctypes.c_int, [c_void_p, ctypes.POINTER(c_i64p),
                                                   ctypes.POINTER(c_i32p)]),
    "dyngb200_tree_info": (ctypes.c_int, [c_void_p, ctypes.POINTER(ctypes.c_int32), c_i64p,
                                          ctypes.POINTER(ctypes.c_uint64),
                                          ctypes.POINTER(ctypes.c_int32),
                                          ctypes.POINTER(Options)]),
    "dyngb200_tree_set_options": (ctypes.c_int, [c_void_p, ctypes.POINTER(Options)]),
    "dyngb200_tree_copy_from": (ctypes.c_int, [c_void_p, c_void_p, c_void_p]),
    "dyngb200_graph_clone": (ctypes.c_int, [c_void_p, c_void_p, ctypes.POINTER(c_void_p)]),
    "dyngb200_graph_copy_from": (ctypes.c_int, [c_void_p, c_void_p, c_void_p]),
    "dyngb200_sssp_update_learned": (ctypes.c_int, [c_void_p, c_void_p, ctypes.POINTER(Batch),
                                                    c_void_p, c_void_p, ctypes.POINTER(Stats)]),
    "dyngb200_scheduler_num_params": (ctypes.c_int64, []),
    "dyngb200_sssp_update_each": (ctypes.c_int, [c_void_p, c_void_p, ctypes.POINTER(Batch),
                                                 ctypes.POINTER(c_void_p), ctypes.c_int32,
                                                 ctypes.POINTER(Stats)]),
    "dyngb200_server_create": (ctypes.c_int, [ctypes.POINTER(ServerConfig), c_void_p,
                                              ctypes.POINTER(c_void_p)]),
    "dyngb200_server_add_graph": (ctypes.c_int, [c_void_p, c_void_p, c_void_p,
                                                 ctypes.POINTER(ctypes.c_int32)]),
    "dyngb200_server_submit": (ctypes.c_int, [c_void_p, ctypes.c_int32, ctypes.POINTER(Batch),
                                              ctypes.POINTER(ctypes.c_uint64)]),
    "dyngb200_server_wait": (ctypes.c_int, [c_void_p, ctypes.c_uint64, ctypes.POINTER(Stats),
                                            ctypes.POINTER(RequestTimes)]),
    "dyngb200_server_drain": (ctypes.c_int, [c_void_p]),
    "dyngb200_server_info_get": (ctypes.c_int, [c_void_p, ctypes.POINTER(ServerInfo)]),
    "dyngb200_server_destroy": (ctypes.c_int, [c_void_p]),
    "dyngb200_scheduler_create": (ctypes.c_int, [c_void_p, ctypes.c_uint64,
                                                 ctypes.POINTER(c_void_p)]),
    "dyngb200_scheduler_destroy": (ctypes.c_int, [c_void_p]),
    "dyngb200_scheduler_set_params": (ctypes.c_int, [c_void_p, c_void_p, c_f32p, c_f32p, c_f32p]),
    "dyngb200_scheduler_get_params": (ctypes.c_int, [c_void_p, c_void_p, c_f32p, c_f32p, c_f32p]),
    "dyngb200_scheduler_forward": (ctypes.c_int, [c_void_p, c_void_p, c_f32p, ctypes.c_int64,
                                                  c_f32p]),
    "dyngb200_scheduler_gradients": (ctypes.c_int, [c_void_p, c_void_p, c_f32p, c_i32p,
                                                    ctypes.c_int64, c_f32p, c_f64p]),
    "dyngb200_scheduler_train": (ctypes.c_int, [c_void_p, c_void_p, c_f32p, c_i32p,
                                                ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                                                ctypes.c_float, ctypes.c_uint64, c_f64p]),
}

_lib = None


def lib():
    """The loaded library (raises NativeLibraryError when it is not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise NativeLibraryError(
                f"{LIB_PATH} is missing: build it with `python -m dyng_b200.build` "
                "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def declared_symbols(header: str) -> list:
    """Names of the functions declared in a header of include/ (for the ABI tests)."""
    import re
    text = open(header).read()
    return sorted(set(re.findall(r"\b(dyngb200_[a-z0-9_]+)\s*\(", text)))
