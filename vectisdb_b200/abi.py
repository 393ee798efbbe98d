"""ctypes declarations of include/vgpu.h and loading of the in-tree libvgpu.so.

The library is REQUIRED: importing this module raises when it is missing or does not export the ABI
version the bindings were written for. There is no CPU fallback anywhere in the package.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libvgpu.so"

ABI_VERSION = 2

# vgpu_status
OK, ERR_INVALID_ARGUMENT, ERR_UNSUPPORTED, ERR_CUDA, ERR_OUT_OF_MEMORY, ERR_COMPILE, \
    ERR_NOT_READY, ERR_TIMEOUT, ERR_REJECTED, ERR_INTERNAL = range(10)
MEM_HOST, MEM_DEVICE = 0, 1
EXEC_NO_SYNC = 1
# vgpu_shard_op
SHARD_OUT_WORD, SHARD_OUT_KEY, SHARD_OUT_I128, SHARD_OUT_AVG_F64, SHARD_OUT_AVG_I128, SHARD_OUT_F64_FROM_ORDER = range(6)


class vgpu_expr(C.Structure):
    _fields_ = [("source", C.c_char_p), ("input_columns", C.POINTER(C.c_char_p)),
                ("n_input_columns", C.c_uint32), ("output_type", C.c_uint32),
                ("window_primitive", C.c_uint32), ("estimated_ops_per_row", C.c_double)]


class vgpu_aggregate(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("output_type", C.c_uint32), ("input_column", C.c_char_p)]


class vgpu_plan_node(C.Structure):
    _fields_ = [
        ("op", C.c_uint32), ("n_children", C.c_uint32), ("children", C.POINTER(C.c_uint32)),
        ("catalog", C.c_char_p), ("schema", C.c_char_p), ("table", C.c_char_p),
        ("column_names", C.POINTER(C.c_char_p)), ("n_column_names", C.c_uint32),
        ("expressions", C.POINTER(vgpu_expr)), ("n_expressions", C.c_uint32),
        ("build_keys", C.POINTER(C.c_char_p)), ("n_build_keys", C.c_uint32),
        ("probe_keys", C.POINTER(C.c_char_p)), ("n_probe_keys", C.c_uint32),
        ("output_columns", C.POINTER(C.c_char_p)), ("n_output_columns", C.c_uint32),
        ("group_keys", C.POINTER(C.c_char_p)), ("n_group_keys", C.c_uint32),
        ("aggregates", C.POINTER(vgpu_aggregate)), ("n_aggregates", C.c_uint32),
        ("estimated_rows", C.c_uint64), ("estimated_row_width_bytes", C.c_uint32),
        ("aggregate_exprs", C.POINTER(C.c_char_p)), ("n_aggregate_exprs", C.c_uint32),
    ]


class vgpu_plan(C.Structure):
    _fields_ = [("nodes", C.POINTER(vgpu_plan_node)), ("n_nodes", C.c_uint32), ("root", C.c_uint32)]


class vgpu_column(C.Structure):
    _fields_ = [("name", C.c_char_p), ("type", C.c_uint32), ("memory", C.c_uint32),
                ("data", C.c_void_p), ("validity", C.c_void_p), ("row_count", C.c_uint64)]


class vgpu_shard_output(C.Structure):
    _fields_ = [("op", C.c_int32), ("key_type", C.c_int32), ("key_shift", C.c_int32), ("key_bits", C.c_int32),
                ("key_min", C.c_int64), ("src", vgpu_column * 4), ("count", vgpu_column), ("dst", C.c_void_p)]


class vgpu_exec_options(C.Structure):
    _fields_ = [("stage_scan_to_cache", C.c_int32), ("serve_whole_scan_from_cache", C.c_int32),
                ("cache_chunk_index", C.c_int64), ("output_memory", C.c_int32), ("flags", C.c_int32),
                ("stream", C.c_void_p)]


class vgpu_batch_options(C.Structure):
    _fields_ = [("block", C.c_int32), ("items", C.c_int32), ("tile_rows", C.c_int32), ("smem_slots", C.c_int32),
                ("use_graph", C.c_int32), ("autotune", C.c_int32)]


class vgpu_batch_stats(C.Structure):
    _fields_ = [("batched", C.c_uint64), ("fallback", C.c_uint64), ("templates", C.c_uint64),
                ("graph_replays", C.c_uint64), ("block", C.c_int32), ("items", C.c_int32),
                ("tile_rows", C.c_int32), ("smem_slots", C.c_int32)]


class vgpu_server_options(C.Structure):
    _fields_ = [("slots", C.c_int32), ("batch_max", C.c_int32), ("memory_budget_bytes", C.c_uint64)]


class vgpu_request_info(C.Structure):
    _fields_ = [("status", C.c_int32), ("batch_size", C.c_int32), ("queued_ms", C.c_double), ("run_ms", C.c_double),
                ("estimated_bytes", C.c_uint64), ("error", C.c_char * 256)]


class vgpu_server_stats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("submitted", "completed", "failed", "rejected", "batches",
                                          "batched_requests", "in_flight", "queued", "reserved_bytes",
                                          "peak_reserved_bytes", "budget_bytes", "peak_in_flight")]


class vgpu_device_info(C.Structure):
    _fields_ = [("device", C.c_int32), ("sm_count", C.c_int32), ("cc_major", C.c_int32),
                ("cc_minor", C.c_int32), ("total_memory", C.c_uint64), ("free_memory", C.c_uint64),
                ("l2_bytes", C.c_uint64), ("smem_per_block_optin", C.c_uint64), ("name", C.c_char * 128)]


class vgpu_kernel_timing(C.Structure):
    _fields_ = [("name", C.c_char * 48), ("ms", C.c_float), ("bytes", C.c_uint64), ("rows", C.c_uint64)]


class vgpu_kernel_cache_stats(C.Structure):
    _fields_ = [("entries", C.c_uint64), ("hits", C.c_uint64), ("misses", C.c_uint64),
                ("disk_hits", C.c_uint64), ("compiles", C.c_uint64), ("compile_ms_total", C.c_double)]


class vgpu_working_set(C.Structure):
    _fields_ = [("total_bytes", C.c_uint64), ("chunk_capped", C.c_int32), ("largest_bytes", C.c_uint64),
                ("largest_operator", C.c_char * 32)]


class vgpu_plan_shape(C.Structure):
    _fields_ = [("scanned_rows", C.c_uint64), ("scanned_bytes", C.c_uint64), ("max_rows", C.c_uint64),
                ("total_ops", C.c_double), ("ops_per_scanned_row", C.c_double),
                ("ops_per_scanned_byte", C.c_double), ("density", C.c_uint32), ("amplification", C.c_double)]


class vgpu_memory_stats(C.Structure):
    _fields_ = [("budget_bytes", C.c_uint64), ("in_use_bytes", C.c_uint64), ("peak_bytes", C.c_uint64),
                ("allocations", C.c_uint64), ("failed_allocations", C.c_uint64)]


class vgpu_bexpr(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("return_type", C.c_uint32), ("name", C.c_char_p),
                ("children", C.POINTER(C.c_uint32)), ("n_children", C.c_uint32), ("is_null", C.c_uint32),
                ("i64", C.c_int64), ("f64", C.c_double)]


class vgpu_vector(C.Structure):
    _fields_ = [("data", C.c_void_p), ("sel", C.POINTER(C.c_uint32)), ("validity", C.POINTER(C.c_uint64)),
                ("constant", C.c_uint32)]


class vgpu_table_ref(C.Structure):
    _fields_ = [("catalog", C.c_char_p), ("schema", C.c_char_p), ("table", C.c_char_p)]


# (name, restype, argtypes) for every function include/vgpu.h declares.
SIGNATURES = [
    ("vgpu_exec_options_init", None, [C.POINTER(vgpu_exec_options)]),
    ("vgpu_execute_plan", C.c_int, [C.POINTER(vgpu_plan), C.POINTER(vgpu_column), C.c_size_t,
                                    C.POINTER(vgpu_exec_options), C.POINTER(C.c_void_p)]),
    ("vgpu_result_column_count", C.c_size_t, [C.c_void_p]),
    ("vgpu_result_column_range", C.c_int, [C.c_void_p, C.c_size_t, C.c_uint64, C.c_uint64, C.POINTER(vgpu_column)]),
    ("vgpu_result_get_column", C.c_int, [C.c_void_p, C.c_size_t, C.POINTER(vgpu_column)]),
    ("vgpu_result_free", None, [C.c_void_p]),
    ("vgpu_batch_options_init", None, [C.POINTER(vgpu_batch_options)]),
    ("vgpu_execute_batch", C.c_int, [C.POINTER(C.POINTER(vgpu_plan)), C.POINTER(C.POINTER(vgpu_column)),
                                     C.POINTER(C.c_size_t), C.c_size_t, C.POINTER(vgpu_exec_options),
                                     C.POINTER(vgpu_batch_options), C.POINTER(C.c_void_p),
                                     C.POINTER(vgpu_batch_stats)]),
    ("vgpu_batch_prepare", C.c_int, [C.POINTER(C.POINTER(vgpu_plan)), C.c_size_t, C.POINTER(C.c_void_p)]),
    ("vgpu_batch_size", C.c_size_t, [C.c_void_p]),
    ("vgpu_batch_execute", C.c_int, [C.c_void_p, C.POINTER(C.POINTER(vgpu_column)), C.POINTER(C.c_size_t),
                                     C.POINTER(vgpu_exec_options), C.POINTER(vgpu_batch_options),
                                     C.POINTER(C.c_void_p), C.POINTER(vgpu_batch_stats)]),
    ("vgpu_batch_free", None, [C.c_void_p]),
    ("vgpu_batch_template", C.c_int, [C.c_char_p, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t),
                                      C.POINTER(C.c_size_t)]),
    ("vgpu_batch_clear", C.c_int, []),
    ("vgpu_pipeline_supports", C.c_int, [C.POINTER(vgpu_plan)]),
    ("vgpu_pipeline_create", C.c_int, [C.POINTER(vgpu_plan), C.POINTER(C.c_char_p), C.POINTER(C.c_int32), C.c_size_t,
                                       C.c_uint64, C.c_int32, C.POINTER(C.c_void_p)]),
    ("vgpu_pipeline_output_count", C.c_size_t, [C.c_void_p]),
    ("vgpu_pipeline_output_type", C.c_int32, [C.c_void_p, C.c_size_t]),
    ("vgpu_pipeline_poll", None, [C.c_void_p]),
    ("vgpu_pipeline_can_submit", C.c_int, [C.c_void_p]),
    ("vgpu_pipeline_submit", C.c_int, [C.c_void_p, C.POINTER(vgpu_column), C.c_size_t, C.c_uint64]),
    ("vgpu_pipeline_try_take", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    ("vgpu_pipeline_take_blocking", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    ("vgpu_pipeline_in_flight", C.c_size_t, [C.c_void_p]),
    ("vgpu_pipeline_result_rows", C.c_uint64, [C.c_void_p]),
    ("vgpu_pipeline_result_column_count", C.c_size_t, [C.c_void_p]),
    ("vgpu_pipeline_result_get_column", C.c_int, [C.c_void_p, C.c_size_t, C.POINTER(vgpu_column)]),
    ("vgpu_pipeline_result_release", None, [C.c_void_p]),
    ("vgpu_pipeline_destroy", None, [C.c_void_p]),
    ("vgpu_server_options_init", None, [C.POINTER(vgpu_server_options)]),
    ("vgpu_server_create", C.c_int, [C.POINTER(vgpu_server_options), C.POINTER(C.c_void_p)]),
    ("vgpu_server_submit", C.c_int, [C.c_void_p, C.POINTER(vgpu_plan), C.POINTER(vgpu_column), C.c_size_t,
                                     C.POINTER(vgpu_exec_options), C.POINTER(C.c_uint64)]),
    ("vgpu_server_wait", C.c_int, [C.c_void_p, C.c_uint64, C.c_double, C.POINTER(C.c_void_p),
                                   C.POINTER(vgpu_request_info), C.POINTER(C.c_int)]),
    ("vgpu_server_stats_get", C.c_int, [C.c_void_p, C.POINTER(vgpu_server_stats)]),
    ("vgpu_server_destroy", None, [C.c_void_p]),
    ("vgpu_copy_to_host", C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]),
    ("vgpu_last_error", C.c_char_p, []),
    ("vgpu_status_string", C.c_char_p, [C.c_int]),
    ("vgpu_abi_version", C.c_int, []),
    ("vgpu_set_device", C.c_int, [C.c_int]),
    ("vgpu_get_device_info", C.c_int, [C.POINTER(vgpu_device_info)]),
    ("vgpu_synchronize", C.c_int, [C.c_void_p]),
    ("vgpu_profile_enable", C.c_int, [C.c_int]),
    ("vgpu_profile_collect", C.c_int, [C.POINTER(vgpu_kernel_timing), C.c_size_t, C.POINTER(C.c_size_t)]),
    ("vgpu_launch_count", C.c_uint64, []),
    ("vgpu_sha256_hex", None, [C.c_void_p, C.c_size_t, C.c_char_p]),
    ("vgpu_kernel_cache_stats_get", C.c_int, [C.POINTER(vgpu_kernel_cache_stats)]),
    ("vgpu_nvrtc_compile_check", C.c_int, [C.c_char_p, C.POINTER(C.c_size_t)]),
    ("vgpu_generate_source", C.c_int, [C.POINTER(vgpu_plan), C.POINTER(vgpu_column), C.c_size_t,
                                       C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    ("vgpu_is_row_independent", C.c_int, [C.POINTER(vgpu_plan)]),
    ("vgpu_estimate_working_set", C.c_int, [C.POINTER(vgpu_plan), C.c_uint64, C.POINTER(vgpu_working_set)]),
    ("vgpu_convert_vector", C.c_int, [C.POINTER(vgpu_vector), C.c_uint32, C.c_uint64, C.POINTER(C.c_uint32),
                                       C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]),
    ("vgpu_ingest_create", C.c_int, [C.POINTER(vgpu_table_ref), C.POINTER(C.c_char_p), C.POINTER(C.c_int32),
                                      C.c_size_t, C.c_uint64, C.POINTER(C.c_void_p)]),
    ("vgpu_ingest_append", C.c_int, [C.c_void_p, C.POINTER(vgpu_vector), C.c_uint64, C.POINTER(C.c_uint32)]),
    ("vgpu_ingest_finish", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    ("vgpu_ingest_destroy", None, [C.c_void_p]),
    ("vgpu_translate_expression", C.c_int, [C.POINTER(vgpu_bexpr), C.c_uint32, C.c_uint32, C.c_uint32, C.c_char_p,
                                             C.c_size_t, C.POINTER(C.c_size_t), C.c_char_p, C.c_size_t,
                                             C.POINTER(C.c_size_t), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    ("vgpu_estimate_working_set_for", C.c_int, [C.POINTER(vgpu_plan), C.POINTER(vgpu_column), C.c_size_t,
                                                 C.POINTER(vgpu_exec_options), C.POINTER(vgpu_working_set)]),
    ("vgpu_analyze_plan_shape", C.c_int, [C.POINTER(vgpu_plan), C.POINTER(vgpu_plan_shape)]),
    ("vgpu_estimate_columns_size", C.c_int, [C.POINTER(vgpu_plan), C.POINTER(C.c_uint64)]),
    ("vgpu_determine_execution_mode", C.c_int, [C.POINTER(vgpu_plan), C.c_uint64, C.c_double,
                                                 C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]),
    ("vgpu_memory_set_budget", C.c_int, [C.c_uint64]),
    ("vgpu_memory_stats_get", C.c_int, [C.POINTER(vgpu_memory_stats)]),
    ("vgpu_memory_has_headroom", C.c_int, [C.c_uint64]),
    ("vgpu_memory_reset_peak", C.c_int, []),
    ("vgpu_cache_init", C.c_int, [C.c_double]),
    ("vgpu_cache_begin_staging", C.c_int, [C.POINTER(vgpu_table_ref)]),
    ("vgpu_cache_stage_chunk", C.c_int, [C.POINTER(vgpu_table_ref), C.POINTER(vgpu_column), C.POINTER(C.c_int)]),
    ("vgpu_cache_commit_staging", C.c_int, [C.POINTER(vgpu_table_ref), C.c_uint64]),
    ("vgpu_cache_abort_staging", C.c_int, [C.POINTER(vgpu_table_ref)]),
    ("vgpu_cache_replayable_chunk_rows", C.c_int, [C.POINTER(vgpu_table_ref), C.POINTER(C.c_char_p), C.c_size_t,
                                                   C.POINTER(C.c_uint64), C.c_size_t, C.POINTER(C.c_size_t)]),
    ("vgpu_cache_try_get_chunk", C.c_int, [C.POINTER(vgpu_table_ref), C.c_char_p, C.c_uint64,
                                           C.POINTER(vgpu_column), C.POINTER(C.c_int)]),
    ("vgpu_cache_invalidate_table", C.c_int, [C.POINTER(vgpu_table_ref)]),
    ("vgpu_cache_invalidate_all", C.c_int, []),
    ("vgpu_cache_current_bytes", C.c_uint64, []),
    ("vgpu_cache_table_generation", C.c_uint64, [C.POINTER(vgpu_table_ref)]),
    ("vgpu_group_by_count_sum_noalloc", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int32, C.c_uint32,
                                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("vgpu_shard_words", C.c_int32, [C.POINTER(C.c_int32), C.c_int32]),
    ("vgpu_shard_route", C.c_int, [C.POINTER(vgpu_column), C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int32),
                                   C.POINTER(vgpu_column), C.POINTER(C.c_int32), C.c_int32, C.c_uint64, C.c_int32,
                                   C.c_void_p, C.POINTER(C.c_uint64), C.c_void_p]),
    ("vgpu_shard_columns", C.c_int, [C.c_void_p, C.c_uint64, C.c_int32, C.c_void_p, C.c_void_p]),
    ("vgpu_shard_finish", C.c_int, [C.POINTER(vgpu_shard_output), C.c_int32, C.c_uint64, C.c_void_p]),
]

_LIB = None


def lib() -> C.CDLL:
    """The loaded engine library (loads and validates it on first use)."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m vectisdb_b200.build`")
        handle = C.CDLL(str(LIB_PATH))
        for name, restype, argtypes in SIGNATURES:
            fn = getattr(handle, name)
            fn.restype = restype
            fn.argtypes = argtypes
        if handle.vgpu_abi_version() != ABI_VERSION:
            raise RuntimeError("libvgpu.so ABI version mismatch")
        _LIB = handle
    return _LIB


class VgpuError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{status_name(status)}: {message}")
        self.status = status
        self.message = message


def status_name(status: int) -> str:
    return lib().vgpu_status_string(status).decode()


def check(status: int) -> None:
    if status != OK:
        raise VgpuError(status, lib().vgpu_last_error().decode(errors="replace"))


def last_error() -> str:
    return lib().vgpu_last_error().decode(errors="replace")


def declared_functions() -> list[str]:
    """Function names declared in include/vgpu.h (parsed from the header text)."""
    import re
    text = (PKG.parent / "include" / "vgpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(vgpu_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))
