"""ctypes mirror of include/vexq_cuda.h and the loader for libvexqcuda.so.

The structures here are the C ABI a Go cgo shim binds; Python uses them for
tests and the benchmark. Loading fails loudly when the shared library has not
been built: there is no CPU fallback behind this API.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvexqcuda.so")

# ---- constants (same values as the header) ----------------------------------
OK, EINVAL, ENOMEM, EADMIT, ETIMEDOUT, EDEVICE, ECANCELED, ENOTSUP, EJIT, ECORRUPT = (
    0, -22, -12, -11, -110, -5, -125, -95, -201, -74)

TYPE_INT64, TYPE_FLOAT64, TYPE_BOOL, TYPE_STRING, TYPE_DATE = 1, 2, 3, 4, 5
TYPE_NAMES = {1: "INT64", 2: "FLOAT64", 3: "BOOL", 4: "STRING", 5: "DATE"}

E_COLUMN, E_LITERAL, E_BINARY, E_AND, E_OR, E_NOT, E_NEG, E_IS_NULL, \
    E_IS_NOT_NULL, E_BETWEEN, E_IN, E_LIKE, E_CASE = range(1, 14)
OP_EQ, OP_NE, OP_LT, OP_LE, OP_GT, OP_GE, OP_ADD, OP_SUB, OP_MUL, OP_DIV = range(1, 11)
LIT_INT, LIT_FLOAT, LIT_STRING, LIT_BOOL = 1, 2, 3, 4
AGG_COUNT, AGG_SUM, AGG_AVG, AGG_MIN, AGG_MAX, AGG_COUNT_DISTINCT = 0, 1, 2, 3, 4, 5

BLOCK_ROWS = 1024
ROW_GROUP_ROWS = 65536


class ColumnDesc(C.Structure):
    _fields_ = [
        ("name", C.c_char_p),
        ("type", C.c_int32),
        ("values", C.c_void_p),
        ("validity", C.c_void_p),
        ("dict_rg_first", C.c_void_p),
        ("dict_str_off", C.c_void_p),
        ("dict_bytes", C.c_void_p),
        ("dict_entries", C.c_int64),
    ]


class VxqSummary(C.Structure):
    _fields_ = [
        ("nrows", C.c_int64),
        ("ncols", C.c_int32),
        ("n_rg", C.c_int32),
        ("rg_rows", C.c_int32),
        ("null_columns", C.c_int32),
        ("bytes_checked", C.c_int64),
    ]


class ZoneMap(C.Structure):
    _fields_ = [
        ("null_count", C.c_int64),
        ("sum", C.c_int64),
        ("min", C.c_uint64),
        ("max", C.c_uint64),
        ("has_min_max", C.c_int32),
    ]


class Expr(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("op", C.c_int32),
        ("column", C.c_int32),
        ("lit_kind", C.c_int32),
        ("lit_int", C.c_int64),
        ("lit_float", C.c_double),
        ("lit_str", C.c_char_p),
        ("child0", C.c_int32),
        ("nchildren", C.c_int32),
    ]


class AggDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("input", C.c_int32), ("out_name", C.c_char_p)]


class ResultSummary(C.Structure):
    _fields_ = [("nrows", C.c_int64), ("ncols", C.c_int32), ("launches", C.c_int32), ("kernel_ms", C.c_double),
                ("scan_ms", C.c_double), ("rows_scanned", C.c_int64), ("bytes_scanned", C.c_int64)]


class OrderDesc(C.Structure):
    _fields_ = [("sort_col", C.c_int32), ("descending", C.c_int32), ("limit", C.c_int64)]


class AggPlanDesc(C.Structure):
    _fields_ = [
        ("nodes", C.POINTER(Expr)), ("nnodes", C.c_int32),
        ("children", C.POINTER(C.c_int32)), ("nchildren", C.c_int32),
        ("predicate", C.c_int32),
        ("group_by", C.POINTER(C.c_int32)), ("ngroup_by", C.c_int32),
        ("aggs", C.POINTER(AggDesc)), ("naggs", C.c_int32),
        ("order", OrderDesc),
    ]


class JoinPlanDesc(C.Structure):
    _fields_ = [
        ("nodes", C.POINTER(Expr)), ("nnodes", C.c_int32),
        ("children", C.POINTER(C.c_int32)), ("nchildren", C.c_int32),
        ("build_key", C.c_int32), ("probe_key", C.c_int32),
        ("build_predicate", C.c_int32), ("probe_predicate", C.c_int32),
        ("residual", C.c_int32),
        ("group_by", C.POINTER(C.c_int32)), ("ngroup_by", C.c_int32),
        ("aggs", C.POINTER(AggDesc)), ("naggs", C.c_int32),
        ("order", OrderDesc),
        ("radix_bits", C.c_int32),
    ]


class VectorView(C.Structure):
    _fields_ = [
        ("name", C.c_char_p),
        ("type", C.c_int32),
        ("values", C.c_void_p),
        ("validity", C.c_void_p),
        ("dict_str_off", C.c_void_p),
        ("dict_bytes", C.c_void_p),
        ("dict_len", C.c_int32),
    ]


class BatchView(C.Structure):
    _fields_ = [("ncols", C.c_int32), ("length", C.c_int32), ("cols", C.POINTER(VectorView))]


class FilterBatch(C.Structure):
    _fields_ = [("ncols", C.c_int32), ("length", C.c_int32), ("physical", C.c_int32), ("rg", C.c_int32),
                ("row0", C.c_int64), ("sel", C.POINTER(C.c_uint16)), ("cols", C.POINTER(VectorView))]


# Every symbol include/vexq_cuda.h declares (checked by the CPU test suite).
BATCH_AUTOTUNE = 1  # VEXQ_BATCH_AUTOTUNE
BATCH_RETUNE = 2    # VEXQ_BATCH_RETUNE
PLAN_RETUNE = 1     # VEXQ_PLAN_RETUNE
SERVE_NO_BATCH = 1  # VEXQ_SERVE_NO_BATCH

EXPORTS = [
    "vexq_init", "vexq_last_error", "vexq_abi_version",
    "vexq_table_upload", "vexq_table_destroy", "vexq_table_num_row_groups",
    "vexq_table_device_bytes", "vexq_table_zone_map", "vexq_table_dict_size",
    "vexq_table_dict_entry", "vexq_table_load_vxq", "vexq_vxq_verify",
    "vexq_agg_plan_create", "vexq_join_plan_create", "vexq_plan_destroy",
    "vexq_plan_explain", "vexq_plan_set_having", "vexq_zone_prune", "vexq_plan_run", "vexq_plan_submit", "vexq_plan_run_host",
    "vexq_result_num_rows", "vexq_result_num_cols", "vexq_result_next",
    "vexq_result_free", "vexq_result_stats", "vexq_result_scan_ms", "vexq_result_info", "vexq_plan_set_stream",
    "vexq_filter_run", "vexq_selvec_from_bits",
    "vexq_filter_open", "vexq_filter_next", "vexq_filter_stats", "vexq_filter_close", "vexq_project_run",
    "vexq_batch_run",
    "vexq_server_start", "vexq_server_submit", "vexq_server_poll",
    "vexq_server_wait", "vexq_server_latency", "vexq_server_stop",
    "vexq_cancel", "vexq_debug_fail_alloc", "vexq_debug_live_device_bytes", "vexq_debug_join_spec", "vexq_plan_autotune",
    "vexq_plan_run_partial", "vexq_partial_info", "vexq_partial_serialize", "vexq_partial_deserialize",
    "vexq_partial_merge", "vexq_partial_free",
    "vexq_plan_run_global_noalloc",
    "vexq_batch_create",
    "vexq_batch_exec",
    "vexq_batch_stats",
    "vexq_batch_explain",
    "vexq_batch_destroy",
    "vexq_server_stats",
]

_lib = None


class VexqError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"vexq status {status}: {msg}")
        self.status = status


def load() -> C.CDLL:
    """Loads libvexqcuda.so (built by vexq_b200.build). Raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m vexq_b200.build` "
            "(the GPU path has no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    i32, i64, vp = C.c_int32, C.c_int64, C.c_void_p
    sig = {
        "vexq_init": (i32, [i32, C.c_uint32]),
        "vexq_last_error": (C.c_char_p, []),
        "vexq_abi_version": (i32, []),
        "vexq_table_upload": (i32, [C.POINTER(ColumnDesc), i32, i64, i32, C.POINTER(vp)]),
        "vexq_table_destroy": (i32, [vp]),
        "vexq_table_num_row_groups": (i32, [vp, C.POINTER(i32)]),
        "vexq_table_device_bytes": (i32, [vp, C.POINTER(i64)]),
        "vexq_table_zone_map": (i32, [vp, i32, i32, C.POINTER(ZoneMap)]),
        "vexq_table_load_vxq": (i32, [C.c_char_p, C.POINTER(C.c_char_p), i32, C.POINTER(vp)]),
        "vexq_vxq_verify": (i32, [C.c_char_p, C.POINTER(VxqSummary)]),
        "vexq_table_dict_size": (i32, [vp, i32, C.POINTER(i32)]),
        "vexq_table_dict_entry": (i32, [vp, i32, i32, C.POINTER(C.c_char_p), C.POINTER(i32)]),
        "vexq_agg_plan_create": (i32, [vp, C.POINTER(AggPlanDesc), C.POINTER(vp)]),
        "vexq_join_plan_create": (i32, [vp, vp, C.POINTER(JoinPlanDesc), C.POINTER(vp)]),
        "vexq_plan_destroy": (i32, [vp]),
        "vexq_plan_explain": (C.c_char_p, [vp]),
        "vexq_plan_set_having": (i32, [vp, C.POINTER(Expr), i32, C.POINTER(i32), i32, i32, i32]),
        "vexq_zone_prune": (i32, [vp, C.POINTER(C.c_uint8), i32]),
        "vexq_plan_run": (i32, [vp, i32, i32, C.POINTER(vp)]),
        "vexq_plan_submit": (i32, [vp, i32, i32, C.POINTER(vp)]),
        "vexq_plan_run_host": (i32, [vp, C.POINTER(ColumnDesc), i32, C.POINTER(vp)]),
        "vexq_result_num_rows": (i32, [vp, C.POINTER(i64)]),
        "vexq_result_num_cols": (i32, [vp, C.POINTER(i32)]),
        "vexq_result_next": (i32, [vp, C.POINTER(BatchView)]),
        "vexq_result_free": (i32, [vp]),
        "vexq_result_stats": (i32, [vp, C.POINTER(C.c_double), C.POINTER(i32), C.POINTER(i64), C.POINTER(i64)]),
        "vexq_result_scan_ms": (i32, [vp, C.POINTER(C.c_double)]),
        "vexq_result_info": (i32, [vp, C.POINTER(ResultSummary)]),
        "vexq_plan_set_stream": (i32, [vp, vp]),
        "vexq_filter_run": (i32, [vp, C.POINTER(Expr), i32, C.POINTER(i32), i32, i32, i64, i64,
                                  C.POINTER(C.c_uint8), C.POINTER(i64)]),
        "vexq_selvec_from_bits": (i32, [C.POINTER(C.c_uint8), i64, i64, C.POINTER(C.c_uint16), C.POINTER(i32)]),
        "vexq_filter_open": (i32, [vp, C.POINTER(Expr), i32, C.POINTER(i32), i32, i32, i32, i32, C.POINTER(vp)]),
        "vexq_filter_next": (i32, [vp, C.POINTER(FilterBatch)]),
        "vexq_filter_stats": (i32, [vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(C.c_double)]),
        "vexq_filter_close": (i32, [vp]),
        "vexq_project_run": (i32, [vp, C.POINTER(Expr), i32, C.POINTER(i32), i32, i32, C.POINTER(i32),
                                   C.POINTER(C.c_char_p), i32, i32, i32, C.POINTER(vp)]),
        "vexq_batch_run": (i32, [C.POINTER(vp), i32, C.POINTER(vp)]),
        "vexq_server_start": (i32, [i64, i32, i32, C.c_uint32, C.POINTER(vp)]),
        "vexq_server_stats": (i32, [vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(i32), C.POINTER(i32)]),
        "vexq_server_submit": (i32, [vp, vp, C.POINTER(i64)]),
        "vexq_server_poll": (i32, [vp, i64, C.POINTER(i32), C.POINTER(vp)]),
        "vexq_server_wait": (i32, [vp, i64, i64, C.POINTER(vp)]),
        "vexq_server_latency": (i32, [vp, i64, C.POINTER(C.c_double)]),
        "vexq_server_stop": (i32, [vp]),
        "vexq_cancel": (i32, [vp]),
        "vexq_debug_fail_alloc": (i32, [i32]),
        "vexq_plan_autotune": (i32, [vp, C.c_uint32, C.POINTER(i32), C.POINTER(C.c_double)]),
        "vexq_plan_run_partial": (i32, [vp, i32, i32, C.POINTER(vp)]),
        "vexq_partial_info": (i32, [vp, C.POINTER(i64), C.POINTER(C.c_double)]),
        "vexq_partial_serialize": (i32, [vp, C.POINTER(vp), C.POINTER(i64)]),
        "vexq_partial_deserialize": (i32, [vp, vp, i64, C.POINTER(vp)]),
        "vexq_partial_merge": (i32, [vp, C.POINTER(vp), i32, C.POINTER(vp)]),
        "vexq_partial_free": (i32, [vp]),
        "vexq_debug_live_device_bytes": (i32, [C.POINTER(i64)]),
        "vexq_debug_join_spec": (i32, [C.c_void_p, i64]),
        "vexq_plan_run_global_noalloc": (i32, [vp, i32, i32, vp, C.POINTER(i64), C.POINTER(C.c_uint8), i32]),
        "vexq_batch_create": (i32, [C.POINTER(vp), i32, C.c_uint32, C.POINTER(vp)]),
        "vexq_batch_exec": (i32, [vp, C.POINTER(vp)]),
        "vexq_batch_stats": (i32, [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(i64), C.POINTER(i64)]),
        "vexq_batch_explain": (C.c_char_p, [vp]),
        "vexq_batch_destroy": (i32, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(status: int) -> None:
    if status != OK:
        msg = load().vexq_last_error()
        raise VexqError(status, msg.decode() if msg else "")
