"""ctypes binding of libmettle_cuda.so (include/mettle_cuda.h).

The shared library is built in-tree by ``mettle_b200.build``. There is no
fallback: if the library is missing or cannot be loaded, every entry point
raises ``MettleError`` instead of silently computing on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libmettle_cuda.so"

# status codes (include/mettle_cuda.h)
OK = 0
UNSUPPORTED = 1
BUDGET_EXCEEDED = 2
OOM = 3
DEVICE_ERROR = 4
TIMEOUT = 5
INVALID = 6
NOT_INITIALIZED = 7
OVERFLOW = 8
STATUS_NAMES = {
    OK: "OK", UNSUPPORTED: "UNSUPPORTED", BUDGET_EXCEEDED: "BUDGET_EXCEEDED", OOM: "OOM",
    DEVICE_ERROR: "DEVICE_ERROR", TIMEOUT: "TIMEOUT", INVALID: "INVALID",
    NOT_INITIALIZED: "NOT_INITIALIZED", OVERFLOW: "OVERFLOW",
}

# logical types
T_INTEGER, T_BIGINT, T_FLOAT, T_DOUBLE, T_DATE, T_TIMESTAMP, T_DECIMAL, T_VARCHAR = 1, 2, 3, 4, 5, 6, 7, 8
T_HUGEINT, T_BOOLEAN, T_DECIMAL128 = 9, 10, 11

PIN_COPY, PIN_BORROW, PIN_UPLOAD = 0, 1, 2
HOOK_ADD, HOOK_MUL = 0, 1


class MettleError(RuntimeError):
    """An error status from the library; ``code`` is the MTL_* status."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code
        self.status = STATUS_NAMES.get(code, str(code))


class Budgets(C.Structure):
    _fields_ = [("cache_region_bytes", C.c_uint64), ("processing_region_bytes", C.c_uint64),
                ("pinned_region_bytes", C.c_uint64)]


class ColumnDesc(C.Structure):
    _fields_ = [("name", C.c_char_p), ("type", C.c_int32), ("scale", C.c_int32), ("data", C.c_void_p),
                ("dict", C.POINTER(C.c_char_p)), ("dict_size", C.c_int32), ("pad", C.c_int32)]


class PinSummary(C.Structure):
    _fields_ = [("row_count", C.c_uint64), ("byte_count", C.c_uint64), ("skipped_columns", C.c_char * 256)]


class CacheStats(C.Structure):
    _fields_ = [(n, C.c_int64) for n in (
        "entries", "cached_bytes", "hits", "misses", "evictions", "bypasses", "input_entries",
        "input_cached_bytes", "selection_entries", "selection_cached_bytes", "join_result_entries",
        "join_result_cached_bytes", "source_selection_entries", "source_selection_bytes",
        "grouped_topk_entries", "grouped_topk_bytes", "query_result_entries", "query_result_bytes")]


class ServeStats(C.Structure):
    _fields_ = [(n, C.c_int64) for n in (
        "submitted", "completed", "rejected", "in_flight", "queued", "admitted_bytes", "batched_launches",
        "program_reuses", "cached_programs", "graph_updates", "builds_kept")]


# (name, restype, argtypes) of every exported entry point
SIGNATURES = [
    ("mtl_parse_buffer_config", C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(Budgets), C.c_char_p,
                                          C.c_size_t]),
    ("mtl_ctx_create", C.c_int, [C.POINTER(Budgets), C.c_int, C.POINTER(C.c_void_p)]),
    ("mtl_ctx_destroy", None, [C.c_void_p]),
    ("mtl_device_info", C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t, C.c_char_p, C.c_size_t,
                                  C.POINTER(C.c_uint64), C.POINTER(C.c_int32)]),
    ("mtl_last_error", C.c_char_p, [C.c_void_p]),
    ("mtl_last_execution_mode", C.c_char_p, [C.c_void_p]),
    ("mtl_table_register", C.c_int, [C.c_void_p, C.c_char_p, C.c_uint64, C.c_int32, C.POINTER(ColumnDesc),
                                     C.c_uint32, C.POINTER(PinSummary)]),
    ("mtl_table_drop", C.c_int, [C.c_void_p, C.c_char_p]),
    ("mtl_column_evict", C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p]),
    ("mtl_processing", C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_void_p)]),
    ("mtl_stmt_prepare", C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_void_p)]),
    ("mtl_stmt_launch", C.c_int, [C.c_void_p, C.c_void_p]),
    ("mtl_stmt_fetch", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    ("mtl_stmt_device_ms", C.c_double, [C.c_void_p]),
    ("mtl_stmt_kernel_count", C.c_int32, [C.c_void_p]),
    ("mtl_stmt_set_profiling", C.c_int, [C.c_void_p, C.c_int32]),
    ("mtl_stmt_step_count", C.c_int32, [C.c_void_p]),
    ("mtl_stmt_step_name", C.c_char_p, [C.c_void_p, C.c_int32]),
    ("mtl_stmt_step_ms", C.c_double, [C.c_void_p, C.c_int32]),
    ("mtl_stmt_free", None, [C.c_void_p]),
    ("mtl_query_submit", C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_void_p)]),
    ("mtl_request_wait", C.c_int, [C.c_void_p, C.c_int64, C.POINTER(C.c_void_p)]),
    ("mtl_request_latency_ms", C.c_double, [C.c_void_p]),
    ("mtl_request_free", None, [C.c_void_p]),
    ("mtl_result_rows", C.c_int64, [C.c_void_p]),
    ("mtl_result_columns", C.c_int32, [C.c_void_p]),
    ("mtl_result_column_name", C.c_char_p, [C.c_void_p, C.c_int32]),
    ("mtl_result_column_type", C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]),
    ("mtl_result_column_data", C.c_void_p, [C.c_void_p, C.c_int32]),
    ("mtl_result_column_valid", C.c_void_p, [C.c_void_p, C.c_int32]),
    ("mtl_result_dict", C.c_char_p, [C.c_void_p, C.c_int32, C.c_int32]),
    ("mtl_result_device_ms", C.c_double, [C.c_void_p]),
    ("mtl_result_free", None, [C.c_void_p]),
    ("mtl_cache_stats_get", C.c_int, [C.c_void_p, C.POINTER(CacheStats)]),
    ("mtl_cache_reset", C.c_int, [C.c_void_p]),
    ("mtl_rewrite_query", C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_size_t]),
    ("mtl_scalar_arith", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_uint64, C.c_int64,
                                   C.c_double, C.c_void_p]),
    ("mtl_scalar_compare", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_uint64, C.c_int64,
                                     C.c_double, C.c_void_p]),
    ("mtl_serve_stats_get", C.c_int, [C.c_void_p, C.POINTER(ServeStats)]),
    ("mtl_serve_set_slots", C.c_int, [C.c_void_p, C.c_int32]),
    ("mtl_debug_inject", C.c_int, [C.c_void_p, C.c_int32, C.c_uint32]),
    ("mtl_autotune", C.c_int, [C.c_void_p, C.c_char_p, C.c_int32, C.c_char_p, C.c_size_t]),
    ("mtl_topk_noalloc", C.c_int, [C.c_int32, C.c_void_p, C.c_uint64, C.c_int32, C.c_int32, C.c_void_p,
                                   C.c_void_p, C.c_void_p]),
]

_lib = None


def header_symbols() -> list[str]:
    """Every function name declared in include/mettle_cuda.h."""
    import re
    text = (HERE.parent / "include" / "mettle_cuda.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w ]+?\*?\s*\**(mtl_\w+)\s*\(", text, re.M)))


def load() -> C.CDLL:
    """Loads the library once; raises MettleError when it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise MettleError(DEVICE_ERROR, f"{LIB_PATH.name} is not built; run mettle_b200.build.build() "
                                        "(there is no CPU fallback for the offloaded subset)")
    lib = C.CDLL(str(LIB_PATH))
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int, ctx=None) -> None:
    if rc != OK:
        lib = load()
        msg = lib.mtl_last_error(ctx).decode(errors="replace") if lib else ""
        raise MettleError(rc, msg or STATUS_NAMES.get(rc, str(rc)))


def library_path() -> str:
    return os.fspath(LIB_PATH)
