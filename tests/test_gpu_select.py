"""GPU tests of the Filter operator (vexq_filter_open/next/close) and the
Project export (vexq_project_run), through the C ABI.

Filter: every batch is one 1024-row block of one row group with its SelVec
installed; the union of the SelVecs equals the oracle's selection over the
whole table (BoolToSelVecInto, exec/expr.go:1545-1564); blocks with no kept
row are skipped (exec/filter.go:67-71); the batch's vectors are the table's
values for those rows. Project: the kept rows' expression values in row
order equal the oracle's Filter → Project (Project.materialize,
exec/project.go:128-196) bit for bit."""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import refcpu as R
from vexq_b200 import abi, datagen as D, plan as P, workloads as W
from vexq_b200.table import HostTable, date_column, float_column, int_column, string_column

from tests.helpers import assert_rows_match

pytestmark = pytest.mark.gpu


def nullable_table(n=30_000, seed=9, rg_rows=4096):
    rng = np.random.default_rng(seed)
    a = rng.integers(-50, 50, n)
    b = np.round(rng.normal(0, 100, n), 3)
    d = (10000 + rng.integers(0, 400, n)).astype(np.int32)
    s = rng.integers(0, 5, n)
    va, vb, vd, vs = (rng.random(n) > p for p in (0.1, 0.15, 0.05, 0.2))
    cols = [int_column("a", a, va), float_column("b", b, vb), date_column("d", d, vd),
            string_column("s", s, ["x", "y", "zz", "w", ""], n, rg_rows, vs)]
    return HostTable(cols, n, rg_rows)


def host_value(t: HostTable, c: int, r: int):
    col = t.columns[c]
    if col.validity is not None and not (col.validity[r >> 3] >> (r & 7)) & 1:
        return None
    v = col.values[r]
    if col.type == abi.TYPE_STRING:
        rg = r // t.rg_rows
        base = int(col.dict_rg_first[rg]) if col.dict_rg_first is not None else 0
        off = col.dict_str_off
        e = base + int(v)
        return bytes(col.dict_bytes[off[e]:off[e + 1]]).decode()
    if col.type == abi.TYPE_FLOAT64:
        return float(v)
    if col.type == abi.TYPE_BOOL:
        return bool(v)
    return int(v)


def drain(f):
    out = []
    while True:
        b = f.next()
        if b is None:
            return out
        out.append(b)


def check_filter(X, host, pred, rg_start=0, rg_end=-1, value_checks=200, seed=0):
    gt = X.GpuTable(host)
    f = X.GpuFilter(gt, pred, rg_start, rg_end)
    try:
        batches = drain(f)
        bits, cnt = R.filter_bits(R.RefTable(host), pred)
        keep = np.unpackbits(np.frombuffer(bits, np.uint8), bitorder="little", count=host.nrows).astype(bool)
        lo = rg_start * host.rg_rows
        hi = host.nrows if rg_end < 0 else min(host.nrows, rg_end * host.rg_rows)
        keep[:lo] = False
        keep[hi:] = False
        got = np.zeros(host.nrows, dtype=bool)
        prev = -1
        rng = np.random.default_rng(seed)
        for b in batches:
            assert b.length > 0 and b.physical <= 1024
            assert b.row0 > prev
            prev = b.row0
            rg = b.row0 // host.rg_rows
            assert b.rg == rg and (b.row0 + b.physical - 1) // host.rg_rows == rg
            assert b.sel == sorted(b.sel) and len(set(b.sel)) == len(b.sel)
            assert all(0 <= i < b.physical for i in b.sel)
            for i in b.sel:
                got[b.row0 + i] = True
            # the batch's vectors are the scan's: table values of the physical rows
            for _ in range(max(1, value_checks // max(len(batches), 1))):
                i = int(rng.integers(0, b.physical))
                c = int(rng.integers(0, len(host.columns)))
                want = host_value(host, c, b.row0 + i)
                have = b.vectors[c].values[i]
                assert have == want or (isinstance(want, float) and math.isnan(want) and math.isnan(have)), \
                    (b.row0 + i, c, have, want)
        assert np.array_equal(got, keep)
        sel, blocks, ms = f.stats()
        assert sel == int(keep.sum()) and blocks >= len(batches)
        return batches
    finally:
        f.close()
        gt.close()


def test_filter_operator_lineitem(gpu_lib):
    host = D.lineitem(300_000, seed=3, rg_rows=65536)
    bs = check_filter(gpu_lib, host, W.q6_plan().predicate)
    assert 0 < len(bs) <= (300_000 + 1023) // 1024
    check_filter(gpu_lib, host, W.q1_plan().predicate)


@pytest.mark.parametrize("k", range(6))
def test_filter_operator_nullable(gpu_lib, k):
    preds = [P.col(0) > 3, P.and_(P.col(1) >= -20.5, P.col(0) <= 10), P.or_(P.col(3) == "zz", P.col(0) < -30),
             P.not_(P.col(3) == "x"), P.is_null(P.col(1)), P.in_(P.col(3), ["x", "", "nope"])]
    check_filter(gpu_lib, nullable_table(), preds[k], seed=k)


def test_filter_operator_ragged_row_groups(gpu_lib):
    # row groups of 100 rows: blocks start off word and byte boundaries
    host = nullable_table(n=5_000, seed=4, rg_rows=100)
    check_filter(gpu_lib, host, P.col(0) > 0)
    check_filter(gpu_lib, host, P.col(1) < 50.0, rg_start=7, rg_end=31)


def test_filter_operator_zone_pruning_and_empty(gpu_lib):
    X = gpu_lib
    n = 200_000
    rng = np.random.default_rng(1)
    d = np.sort(8000 + rng.integers(0, 3000, n)).astype(np.int32)
    host = HostTable([date_column("d", d), float_column("v", rng.random(n))], n, 16384)
    pred = P.and_(P.col(0) >= "1994-01-01", P.col(0) < "1994-03-01")
    bs = check_filter(X, host, pred)
    rgs = {b.rg for b in bs}
    assert 0 < len(rgs) < host.n_rg
    assert check_filter(X, host, P.col(0) < "1900-01-01") == []


def run_project(X, host, exprs, pred=None, rg_start=0, rg_end=-1):
    gt = X.GpuTable(host)
    try:
        r = X.GpuProject(gt, exprs, None, pred, rg_start, rg_end).run()
        rows = r.rows()
        r.close()
        ref = R.project(R.RefTable(host), exprs, pred, rg_start, rg_end)
        return rows, ref.rows()
    finally:
        gt.close()


def test_project_lineitem_q6_filter(gpu_lib):
    host = D.lineitem(400_000, seed=5, rg_rows=65536)
    price, disc, tax = P.col(D.L_PRICE), P.col(D.L_DISC), P.col(D.L_TAX)
    exprs = [price * (1 - disc), price * (1 - disc) * (1 + tax), P.col(D.L_FLAG), P.col(D.L_SHIPDATE),
             P.col(D.L_QTY) * 2 + 1, disc > 0.05]
    rows, ref = run_project(gpu_lib, host, exprs, W.q6_plan().predicate)
    assert len(rows) > 1000
    assert_rows_match(rows, ref, ordered=True, rtol=0.0)


def test_project_nullable_and_no_predicate(gpu_lib):
    host = nullable_table()
    exprs = [P.col(0), P.col(1) * 2 - 1, P.col(3), P.col(2), P.case([(P.col(0) > 0, P.col(1))], 0.5),
             P.col(1) / P.col(0), P.is_null(P.col(1)), P.col(0) + 7, P.col(1)]
    rows, ref = run_project(gpu_lib, host, exprs, P.or_(P.col(3) == "zz", P.col(0) < -30))
    assert_rows_match(rows, ref, ordered=True, rtol=0.0)
    rows, ref = run_project(gpu_lib, host, exprs[:4])
    assert len(rows) == host.nrows
    assert_rows_match(rows, ref, ordered=True, rtol=0.0)


def test_project_row_group_range_and_empty(gpu_lib):
    host = nullable_table(n=20_000, seed=6, rg_rows=100)
    rows, ref = run_project(gpu_lib, host, [P.col(1), P.col(3)], P.col(0) > 10, rg_start=3, rg_end=57)
    assert_rows_match(rows, ref, ordered=True, rtol=0.0)
    rows, ref = run_project(gpu_lib, host, [P.col(0)], P.col(0) > 1000)
    assert rows == [] and ref == []
