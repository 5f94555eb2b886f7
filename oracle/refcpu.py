"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle (refcpu.cpp).

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg;
the product package (vexq_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from vexq_b200 import abi  # noqa: E402  (descriptor structs only)
from vexq_b200.table import HostTable  # noqa: E402

from . import build as _build  # noqa: E402

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = _build.build_oracle()
        L = C.CDLL(path)
        vp, i32, i64 = C.c_void_p, C.c_int32, C.c_int64
        L.ref_table_new.argtypes = [C.POINTER(abi.ColumnDesc), i32, i64, i32, C.POINTER(vp)]
        L.ref_table_new.restype = i32
        L.ref_table_free.argtypes = [vp]
        L.ref_table_zone_map.argtypes = [vp, i32, i32, C.POINTER(abi.ZoneMap)]
        L.ref_table_zone_map.restype = i32
        L.ref_agg_run.argtypes = [vp, C.POINTER(abi.AggPlanDesc), i32, i32, i32, C.POINTER(vp)]
        L.ref_agg_run.restype = i32
        L.ref_join_run.argtypes = [vp, vp, C.POINTER(abi.JoinPlanDesc), i32, C.POINTER(vp)]
        L.ref_join_run.restype = i32
        L.ref_zone_prune.argtypes = [vp, C.POINTER(abi.AggPlanDesc), C.POINTER(C.c_uint8), i32]
        L.ref_zone_prune.restype = i32
        L.ref_filter_run.argtypes = [vp, C.POINTER(abi.Expr), i32, C.POINTER(i32), i32, i32,
                                     C.POINTER(C.c_uint8), C.POINTER(i64)]
        L.ref_filter_run.restype = i32
        L.ref_project_run.argtypes = [vp, C.POINTER(abi.Expr), i32, C.POINTER(i32), i32, i32, C.POINTER(i32), i32,
                                      i32, i32, C.POINTER(vp)]
        L.ref_project_run.restype = i32
        L.ref_result_rows.argtypes = [vp]
        L.ref_result_rows.restype = i64
        L.ref_result_cols.argtypes = [vp]
        L.ref_result_cols.restype = i32
        L.ref_result_col_type.argtypes = [vp, i32]
        L.ref_result_col_type.restype = i32
        L.ref_result_col_name.argtypes = [vp, i32]
        L.ref_result_col_name.restype = C.c_char_p
        L.ref_result_get.argtypes = [vp, i64, i32, C.POINTER(i64), C.POINTER(i32),
                                     C.POINTER(C.c_char_p), C.POINTER(i32)]
        L.ref_result_get.restype = i32
        L.ref_result_exact.argtypes = [vp, i64, i32, C.POINTER(C.c_double)]
        L.ref_result_exact.restype = i32
        L.ref_result_free.argtypes = [vp]
        L.ref_result_having.argtypes = [vp, C.POINTER(abi.Expr), i32, C.POINTER(i32), i32, i32, i32,
                                        C.POINTER(abi.OrderDesc)]
        L.ref_result_having.restype = i32
        L.ref_last_error.restype = C.c_char_p
        L.ref_radix_bits_for.argtypes = [i64]
        L.ref_radix_bits_for.restype = i32
        L.ref_radix_part.argtypes = [i64, C.c_uint64]
        L.ref_radix_part.restype = i32
        _lib = L
    return _lib


class OracleError(RuntimeError):
    pass


def _check(st):
    if st != 0:
        raise OracleError(f"oracle status {st}: {lib().ref_last_error().decode()}")


def decode_value(t: int, bits: int):
    if t == abi.TYPE_FLOAT64:
        return struct.unpack("<d", struct.pack("<q", bits))[0]
    if t == abi.TYPE_BOOL:
        return bool(bits)
    return int(bits)


class RefTable:
    def __init__(self, t: HostTable):
        self.host = t
        self.h = C.c_void_p()
        _check(lib().ref_table_new(t.descs(), len(t.columns), t.nrows, t.rg_rows, C.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.ref_table_free(self.h)
            self.h = None

    def zone_map(self, col, rg):
        z = abi.ZoneMap()
        _check(lib().ref_table_zone_map(self.h, col, rg, C.byref(z)))
        return z


class RefResult:
    """Columns as Python lists (None = NULL), plus exact sums per float cell."""

    def __init__(self, h):
        L = lib()
        self.nrows = L.ref_result_rows(h)
        self.ncols = L.ref_result_cols(h)
        self.types = [L.ref_result_col_type(h, c) for c in range(self.ncols)]
        self.names = [L.ref_result_col_name(h, c).decode() for c in range(self.ncols)]
        self.columns = [[None] * self.nrows for _ in range(self.ncols)]
        self.exact = [[math.nan] * self.nrows for _ in range(self.ncols)]
        bits, valid, s, ln, ex = C.c_int64(), C.c_int32(), C.c_char_p(), C.c_int32(), C.c_double()
        for c in range(self.ncols):
            t = self.types[c]
            col = self.columns[c]
            for r in range(self.nrows):
                _check(L.ref_result_get(h, r, c, C.byref(bits), C.byref(valid), C.byref(s), C.byref(ln)))
                if valid.value:
                    col[r] = C.string_at(s, ln.value).decode() if t == abi.TYPE_STRING else decode_value(t, bits.value)
                if t == abi.TYPE_FLOAT64:
                    _check(L.ref_result_exact(h, r, c, C.byref(ex)))
                    self.exact[c][r] = ex.value
        L.ref_result_free(h)

    def rows(self):
        return [tuple(self.columns[c][r] for c in range(self.ncols)) for r in range(self.nrows)]


def agg(table: RefTable, plan, workers: int = 0, rg_start: int = 0, rg_end: int = -1) -> RefResult:
    h = C.c_void_p()
    _check(lib().ref_agg_run(table.h, C.byref(plan.desc), rg_start, rg_end, workers, C.byref(h)))
    return RefResult(h)


def _having(h, having, visible: int, order):
    from vexq_b200.plan import predicate_arrays
    keep, nodes, nn, ch, nc, root = predicate_arrays(having)
    o = abi.OrderDesc(*order) if order is not None else abi.OrderDesc(-1, 0, -1)
    try:
        _check(lib().ref_result_having(h, nodes, nn, ch, nc, root, visible, C.byref(o)))
    except Exception:
        lib().ref_result_free(h)
        raise


def agg_having(table: RefTable, plan, having, visible: int = -1, order=None, workers: int = 0) -> RefResult:
    """The aggregate of `plan` (which must carry no ORDER BY / LIMIT), then
    HAVING, the column cut and `order` = (column, descending, limit)."""
    h = C.c_void_p()
    _check(lib().ref_agg_run(table.h, C.byref(plan.desc), 0, -1, workers, C.byref(h)))
    _having(h, having, visible, order)
    return RefResult(h)


def join_having(build: RefTable, probe: RefTable, plan, having, visible: int = -1, order=None,
                workers: int = 0) -> RefResult:
    h = C.c_void_p()
    _check(lib().ref_join_run(build.h, probe.h, C.byref(plan.desc), workers, C.byref(h)))
    _having(h, having, visible, order)
    return RefResult(h)


def agg_raw(table: RefTable, plan, workers: int = 0) -> int:
    """Runs the aggregate and frees the result; returns its row count (timing)."""
    h = C.c_void_p()
    _check(lib().ref_agg_run(table.h, C.byref(plan.desc), 0, -1, workers, C.byref(h)))
    n = lib().ref_result_rows(h)
    lib().ref_result_free(h)
    return n


def join(build: RefTable, probe: RefTable, plan, workers: int = 0) -> RefResult:
    h = C.c_void_p()
    _check(lib().ref_join_run(build.h, probe.h, C.byref(plan.desc), workers, C.byref(h)))
    return RefResult(h)


def join_raw(build: RefTable, probe: RefTable, plan, workers: int = 0) -> int:
    h = C.c_void_p()
    _check(lib().ref_join_run(build.h, probe.h, C.byref(plan.desc), workers, C.byref(h)))
    n = lib().ref_result_rows(h)
    lib().ref_result_free(h)
    return n


def zone_prune(table: RefTable, plan):
    n = table.host.n_rg
    m = (C.c_uint8 * max(n, 1))()
    _check(lib().ref_zone_prune(table.h, C.byref(plan.desc), m, n))
    return [int(m[i]) for i in range(n)]


def filter_bits(table: RefTable, pred):
    from vexq_b200.plan import predicate_arrays
    keep, nodes, nn, ch, nc, root = predicate_arrays(pred)
    nbytes = (table.host.nrows + 7) // 8
    out = (C.c_uint8 * max(nbytes, 1))()
    cnt = C.c_int64()
    _check(lib().ref_filter_run(table.h, nodes, nn, ch, nc, root, out, C.byref(cnt)))
    return bytes(out)[:nbytes], cnt.value


def project(table: RefTable, exprs, predicate=None, rg_start: int = 0, rg_end: int = -1) -> RefResult:
    """Filter → Project over the table (ref_project_run): rows in row order."""
    from vexq_b200.plan import project_arrays
    keep, nodes, nn, ch, nc, root, roots = project_arrays(predicate, exprs)
    r = (C.c_int32 * max(len(roots), 1))(*roots)
    h = C.c_void_p()
    _check(lib().ref_project_run(table.h, nodes, nn, ch, nc, root, r, len(roots), rg_start, rg_end, C.byref(h)))
    return RefResult(h)


# ---- the reference's own AVX2 filter kernel (oracle/_ref) -------------------
_ref_filter = None


def ref_filter_lib():
    """bench/simd_filter/cpp/filter_kernel.cpp compiled from the reference's
    sources; None when neither the sources nor a prebuilt copy are present or
    the host CPU lacks AVX2."""
    global _ref_filter
    if _ref_filter is None:
        path = _build.build_ref_filter()
        if path is None or not os.path.exists(path):
            return None
        try:
            with open("/proc/cpuinfo") as f:
                if " avx2" not in f.read():
                    return None
        except OSError:
            return None
        L = C.CDLL(path)
        for nm, vt in (("_Z18filter_gt_i64_avx2PKlmlPj", C.c_int64), ("_Z20filter_gt_i64_scalarPKlmlPj", C.c_int64),
                       ("_Z18filter_gt_i32_avx2PKimiPj", C.c_int32), ("_Z20filter_gt_i32_scalarPKimiPj", C.c_int32)):
            f = getattr(L, nm)
            f.argtypes = [C.c_void_p, C.c_size_t, vt, C.c_void_p]
            f.restype = C.c_size_t
        _ref_filter = L
    return _ref_filter


def radix_bits_for(est_rows: int) -> int:
    """RadixBitsFor (exec/parallel_join.go:72-81) as the oracle restates it."""
    return int(lib().ref_radix_bits_for(int(est_rows)))


def radix_part(key: int, mask: int) -> int:
    """radixPart (exec/parallel_join.go:91-109): fmix64 of the key, masked."""
    return int(lib().ref_radix_part(int(key), int(mask)))
