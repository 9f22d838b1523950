"""ctypes bindings of ``lib/libsparkalog_b200.so`` (declared in include/sparkalog_b200.h).

The library is the product: every operator and the fixpoint loop run in it on
the GPU. There is no CPU fallback; importing this module without the built
library raises.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libsparkalog_b200.so"

c_u32p = ctypes.POINTER(ctypes.c_uint32)
c_u64p = ctypes.POINTER(ctypes.c_uint64)
c_sizep = ctypes.POINTER(ctypes.c_size_t)
vp = ctypes.c_void_p

# Symbols of include/sparkalog_b200.h, in declaration order.
TIER_A = [
    "sparkalog_stream_synchronize",
    "sparkalog_join_u32_temporary_bytes",
    "sparkalog_join_u32_count",
    "sparkalog_join_u32_emit",
    "sparkalog_distinct_u32_temporary_bytes",
    "sparkalog_distinct_u32",
    "sparkalog_anti_join_u32_temporary_bytes",
    "sparkalog_anti_join_u32",
    "sparkalog_filter_u32_temporary_bytes",
    "sparkalog_filter_u32",
    "sparkalog_fill_mod_u32",
    "sparkalog_add_one_i32",
    "sparkalog_union_u32_temporary_bytes",
    "sparkalog_union_u32",
    "sparkalog_anti_join_u32_no_alloc",
    "sparkalog_anti_join_u32_no_alloc_error",
    "sparkalog_b200_device_error",
]
TIER_B = [
    "sparkalog_store_create",
    "sparkalog_store_destroy",
    "sparkalog_store_insert_static",
    "sparkalog_store_insert_recursive",
    "sparkalog_store_rows",
    "sparkalog_store_read",
    "sparkalog_store_anti_join",
    "sparkalog_store_drop",
    "sparkalog_store_compact",
    "sparkalog_store_select",
    "sparkalog_store_join",
    "sparkalog_store_load_binary_u32",
    "sparkalog_store_load_delimited_u32",
    "sparkalog_store_load_delimited_values",
    "sparkalog_catalog_export",
    "sparkalog_catalog_create",
    "sparkalog_catalog_destroy",
    "sparkalog_catalog_intern_u32",
    "sparkalog_catalog_decode_u32",
    "sparkalog_catalog_size",
    "sparkalog_executor_compile",
    "sparkalog_executor_step",
    "sparkalog_store_append",
    "sparkalog_store_extract_segment",
    "sparkalog_store_extract_segment_untagged",
    "sparkalog_store_remove_segments",
    "sparkalog_executor_destroy",
    "sparkalog_executor_run",
    "sparkalog_executor_track_segments",
    "sparkalog_executor_segment_stats",
    "sparkalog_executor_set_profiling",
    "sparkalog_executor_set_fused",
    "sparkalog_executor_set_member_set",
    "sparkalog_executor_set_device_loop",
    "sparkalog_executor_device_loop_stats",
    "sparkalog_tuning_defaults",
    "sparkalog_executor_set_tuning",
    "sparkalog_executor_get_tuning",
    "sparkalog_executor_stats",
    "sparkalog_executor_trace",
    "sparkalog_reserve_device_memory",
    "sparkalog_last_error",
]
EXPORTED = TIER_A + TIER_B


class RulePlanC(ctypes.Structure):
    """sparkalog_rule_plan."""

    _fields_ = [
        ("target", ctypes.c_uint32),
        ("delta_input", ctypes.c_uint32),
        ("right_input", ctypes.c_uint32),
        ("left_key", ctypes.c_uint32),
        ("right_key", ctypes.c_uint32),
        ("proj_side", ctypes.c_uint32 * 2),
        ("proj_col", ctypes.c_uint32 * 2),
        ("distinct_cols", ctypes.c_uint32 * 2),
        ("anti_left", ctypes.c_uint32 * 2),
        ("anti_right", ctypes.c_uint32 * 2),
        ("union_left", ctypes.c_uint32 * 2),
        ("union_right", ctypes.c_uint32 * 2),
    ]


class SccSummaryC(ctypes.Structure):
    """sparkalog_scc_summary."""

    _fields_ = [
        ("iterations", ctypes.c_uint64),
        ("total_new_rows", ctypes.c_uint64),
        ("relation_count", ctypes.c_uint64),
        ("relation_ids", c_u32p),
        ("relation_rows", c_u64p),
    ]


class TuningC(ctypes.Structure):
    """sparkalog_tuning."""

    _fields_ = [
        ("dir_rows_log2", ctypes.c_uint32),
        ("group_lanes", ctypes.c_uint32),
        ("group_candidates", ctypes.c_uint64),
        ("sparse_candidates", ctypes.c_uint64),
        ("fused_rows_cap", ctypes.c_uint32),
        ("merge_items", ctypes.c_uint32),
        ("level_ratio", ctypes.c_uint32),
        ("levels", ctypes.c_uint32),
        ("bloom_bits", ctypes.c_uint32),
        ("merge_anti_ratio", ctypes.c_uint32),
        ("sparse_items", ctypes.c_uint32),
        ("compact_index", ctypes.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


class SelectC(ctypes.Structure):
    """sparkalog_select."""

    _fields_ = [
        ("where_mask", ctypes.c_uint32),
        ("where_value", ctypes.c_uint32 * 2),
        ("out_source", ctypes.c_uint32 * 2),
        ("out_value", ctypes.c_uint32 * 2),
    ]


KERNEL_CLASSES = ["join", "sort_histogram", "sort_pass", "anti_join", "merge", "index", "join_distinct"]


class KernelStatsC(ctypes.Structure):
    """sparkalog_kernel_stats."""

    _fields_ = [
        ("launches", ctypes.c_uint64 * 8),
        ("milliseconds", ctypes.c_double * 8),
        ("bytes", ctypes.c_double * 8),
        ("total_launches", ctypes.c_uint64),
        ("rounds", ctypes.c_uint64),
    ]


class LoadErrorC(ctypes.Structure):
    """sparkalog_load_error."""

    _fields_ = [("kind", ctypes.c_int32), ("column", ctypes.c_uint32), ("line", ctypes.c_uint64),
                ("field_offset", ctypes.c_uint64), ("field_length", ctypes.c_uint64)]


class RoundTraceC(ctypes.Structure):
    """sparkalog_round_trace."""

    _fields_ = [(name, ctypes.c_uint64) for name in
                ("round", "delta_rows", "join_rows", "unique_rows", "new_rows", "full_rows")]


_lib = None


def declare_operator_abi(L: ctypes.CDLL) -> None:
    """Argument types of the operator ABI that this library shares with the
    reference's column_ops.cu (crates/sparkalog-execution/native/column_ops.cu:231-775)."""
    L.sparkalog_stream_synchronize.argtypes = [vp]
    L.sparkalog_join_u32_temporary_bytes.argtypes = [vp, vp, ctypes.c_size_t, c_sizep, vp]
    L.sparkalog_join_u32_count.argtypes = [vp, ctypes.c_size_t, vp, vp, ctypes.c_size_t, vp, vp, vp, vp,
                                           ctypes.c_size_t, vp]
    L.sparkalog_join_u32_emit.argtypes = [vp, ctypes.c_size_t, vp, vp, vp, ctypes.c_size_t, vp, ctypes.c_uint32,
                                          vp, ctypes.c_uint32, vp, vp, vp, vp]
    L.sparkalog_distinct_u32_temporary_bytes.argtypes = [vp, vp, vp, ctypes.c_size_t, c_sizep, vp]
    L.sparkalog_distinct_u32.argtypes = [vp, vp, ctypes.c_size_t, vp, vp, vp, vp, vp, vp, ctypes.c_size_t, vp]
    L.sparkalog_anti_join_u32_temporary_bytes.argtypes = [vp, vp, vp, ctypes.c_size_t, c_sizep, vp]
    L.sparkalog_anti_join_u32.argtypes = [vp, vp, ctypes.c_size_t, vp, vp, ctypes.c_size_t, vp, vp, vp, vp, vp, vp,
                                          ctypes.c_size_t, vp]
    L.sparkalog_filter_u32_temporary_bytes.argtypes = [vp, vp, vp, ctypes.c_size_t, c_sizep, vp]
    L.sparkalog_filter_u32.argtypes = [vp, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint32, vp, vp, vp, vp,
                                       ctypes.c_size_t, vp]
    L.sparkalog_fill_mod_u32.argtypes = [vp, ctypes.c_size_t, ctypes.c_uint32, vp]
    L.sparkalog_add_one_i32.argtypes = [vp, ctypes.c_size_t, vp]
    L.sparkalog_union_u32_temporary_bytes.argtypes = [vp, ctypes.c_size_t, vp, ctypes.c_size_t, vp, vp, vp, c_sizep,
                                                      vp]
    L.sparkalog_union_u32.argtypes = [vp, vp, ctypes.c_size_t, vp, vp, ctypes.c_size_t, vp, vp, vp, vp, vp, vp, vp,
                                      vp, ctypes.c_size_t, vp]


def load() -> ctypes.CDLL:
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m sparkalog_b200.build` "
            "(sparkalog_b200 has no CPU fallback)")
    L = ctypes.CDLL(str(LIB_PATH))
    i = ctypes.c_int
    declare_operator_abi(L)
    L.sparkalog_anti_join_u32_no_alloc.argtypes = [vp, vp, ctypes.c_size_t, vp, vp, ctypes.c_size_t, vp, vp, vp,
                                                   vp, vp, vp]
    L.sparkalog_anti_join_u32_no_alloc_error.argtypes = [c_u32p, i]
    L.sparkalog_b200_device_error.argtypes = [c_u32p, i]
    for name in TIER_A:
        getattr(L, name).restype = i
    L.sparkalog_store_create.argtypes = [vp, ctypes.POINTER(vp)]
    L.sparkalog_store_create.restype = i
    L.sparkalog_store_destroy.argtypes = [vp]
    L.sparkalog_store_destroy.restype = None
    L.sparkalog_store_insert_static.argtypes = [vp, ctypes.c_uint32, vp, vp, ctypes.c_size_t, i]
    L.sparkalog_store_insert_static.restype = i
    L.sparkalog_store_insert_recursive.argtypes = [vp, ctypes.c_uint32, vp, vp, ctypes.c_size_t, vp, vp,
                                                   ctypes.c_size_t, i]
    L.sparkalog_store_insert_recursive.restype = i
    L.sparkalog_store_rows.argtypes = [vp, ctypes.c_uint32, i, c_sizep]
    L.sparkalog_store_rows.restype = i
    L.sparkalog_store_read.argtypes = [vp, ctypes.c_uint32, i, vp, vp, i]
    L.sparkalog_store_read.restype = i
    L.sparkalog_store_anti_join.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]
    L.sparkalog_store_anti_join.restype = i
    L.sparkalog_store_drop.argtypes = [vp, ctypes.c_uint32]
    L.sparkalog_store_drop.restype = i
    L.sparkalog_store_compact.argtypes = [vp, ctypes.c_uint32]
    L.sparkalog_store_compact.restype = i
    L.sparkalog_store_select.argtypes = [vp, ctypes.c_uint32, ctypes.POINTER(SelectC), ctypes.c_uint32, c_sizep]
    L.sparkalog_store_select.restype = i
    L.sparkalog_store_join.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                       c_u32p, c_u32p, ctypes.c_uint32, c_sizep]
    L.sparkalog_store_join.restype = i
    L.sparkalog_store_load_binary_u32.argtypes = [vp, ctypes.c_uint32, vp, ctypes.c_size_t, i, i, c_sizep,
                                                   ctypes.POINTER(LoadErrorC)]
    L.sparkalog_store_load_binary_u32.restype = i
    L.sparkalog_store_load_delimited_u32.argtypes = [vp, ctypes.c_uint32, vp, ctypes.c_size_t, i, ctypes.c_ubyte, i,
                                                     i, c_sizep, ctypes.POINTER(LoadErrorC)]
    L.sparkalog_store_load_delimited_u32.restype = i
    L.sparkalog_store_load_delimited_values.argtypes = [vp, vp, ctypes.c_uint32, vp, ctypes.c_size_t, i,
                                                        ctypes.c_ubyte, i, i, c_sizep, ctypes.POINTER(LoadErrorC)]
    L.sparkalog_store_load_delimited_values.restype = i
    L.sparkalog_catalog_export.argtypes = [vp, c_u32p, c_u32p, c_u64p, vp, ctypes.c_size_t, c_sizep]
    L.sparkalog_catalog_export.restype = i
    L.sparkalog_catalog_create.argtypes = [vp, ctypes.POINTER(vp)]
    L.sparkalog_catalog_create.restype = i
    L.sparkalog_catalog_destroy.argtypes = [vp]
    L.sparkalog_catalog_destroy.restype = None
    L.sparkalog_catalog_intern_u32.argtypes = [vp, vp, ctypes.c_size_t, i, vp, c_sizep]
    L.sparkalog_catalog_intern_u32.restype = i
    L.sparkalog_catalog_decode_u32.argtypes = [vp, vp, ctypes.c_size_t, i, vp]
    L.sparkalog_catalog_decode_u32.restype = i
    L.sparkalog_catalog_size.argtypes = [vp, c_sizep]
    L.sparkalog_catalog_size.restype = i
    L.sparkalog_executor_step.argtypes = [vp, vp, ctypes.c_size_t, ctypes.POINTER(SccSummaryC),
                                          ctypes.POINTER(ctypes.c_int)]
    L.sparkalog_executor_step.restype = i
    L.sparkalog_store_append.argtypes = [vp, ctypes.c_uint32, vp, vp, ctypes.c_size_t, i]
    L.sparkalog_store_append.restype = i
    L.sparkalog_store_extract_segment.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, vp, vp, i,
                                                  c_sizep]
    L.sparkalog_store_extract_segment.restype = i
    L.sparkalog_store_extract_segment_untagged.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, i,
                                                           vp, vp, i, c_sizep]
    L.sparkalog_store_extract_segment_untagged.restype = i
    L.sparkalog_store_remove_segments.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, c_u32p, ctypes.c_size_t]
    L.sparkalog_store_remove_segments.restype = i
    L.sparkalog_executor_compile.argtypes = [vp, c_u32p, ctypes.c_size_t, ctypes.POINTER(RulePlanC), ctypes.c_size_t,
                                             ctypes.POINTER(vp)]
    L.sparkalog_executor_compile.restype = i
    L.sparkalog_executor_destroy.argtypes = [vp]
    L.sparkalog_executor_destroy.restype = None
    L.sparkalog_executor_run.argtypes = [vp, vp, ctypes.c_size_t, ctypes.POINTER(SccSummaryC)]
    L.sparkalog_executor_run.restype = i
    L.sparkalog_executor_track_segments.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32]
    L.sparkalog_executor_track_segments.restype = i
    L.sparkalog_executor_segment_stats.argtypes = [vp, c_u32p, c_u64p]
    L.sparkalog_executor_segment_stats.restype = i
    L.sparkalog_executor_set_profiling.argtypes = [vp, i]
    L.sparkalog_executor_set_profiling.restype = i
    L.sparkalog_executor_set_fused.argtypes = [vp, i]
    L.sparkalog_executor_set_fused.restype = i
    L.sparkalog_executor_set_member_set.argtypes = [vp, i]
    L.sparkalog_executor_set_member_set.restype = i
    L.sparkalog_executor_set_device_loop.argtypes = [vp, i]
    L.sparkalog_executor_set_device_loop.restype = i
    L.sparkalog_executor_device_loop_stats.argtypes = [vp, c_u64p, c_u64p]
    L.sparkalog_executor_device_loop_stats.restype = i
    L.sparkalog_tuning_defaults.argtypes = [ctypes.POINTER(TuningC)]
    L.sparkalog_tuning_defaults.restype = i
    L.sparkalog_executor_set_tuning.argtypes = [vp, ctypes.POINTER(TuningC)]
    L.sparkalog_executor_set_tuning.restype = i
    L.sparkalog_executor_get_tuning.argtypes = [vp, ctypes.POINTER(TuningC)]
    L.sparkalog_executor_get_tuning.restype = i
    L.sparkalog_executor_stats.argtypes = [vp, ctypes.POINTER(KernelStatsC), i]
    L.sparkalog_executor_stats.restype = i
    L.sparkalog_executor_trace.argtypes = [vp, ctypes.POINTER(RoundTraceC), ctypes.c_size_t, c_sizep, i]
    L.sparkalog_executor_trace.restype = i
    L.sparkalog_reserve_device_memory.argtypes = [ctypes.c_size_t, vp]
    L.sparkalog_reserve_device_memory.restype = i
    L.sparkalog_last_error.argtypes = []
    L.sparkalog_last_error.restype = ctypes.c_char_p
    _lib = L
    return L


def last_error() -> str:
    msg = load().sparkalog_last_error()
    return msg.decode() if msg else ""
