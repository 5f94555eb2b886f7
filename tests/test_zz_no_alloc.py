"""GPU tests of vexq_plan_run_global_noalloc, the aggregate entry point that
allocates no memory, called through the C ABI.

Every case compares it with the allocating entry point (vexq_plan_run) on the
same plan, over two calls in a row. The file name sorts last, so a full run
exercises it after every other GPU test in the same process; it also passes
on its own in a fresh process, where its first call does the set-up.
"""
from __future__ import annotations

import ctypes as C
import math
import struct

import numpy as np
import pytest

from vexq_b200 import abi, datagen as D, plan as P, workloads as W
from vexq_b200.table import HostTable, date_column, float_column, int_column

pytestmark = pytest.mark.gpu

# The scan kernel is the same. The merge may differ: where vexq_plan_run merges
# float sums exactly inside the scan, this entry point merges the per-block
# partials with the fixed-order TwoSum merge, so float cells agree to
# rounding; every other cell is compared exactly.
FLOAT_RTOL = 1e-12


def noalloc(op, n_out, rg_start=0, rg_end=-1, stream=None):
    vals = (C.c_int64 * max(n_out, 1))()
    valid = (C.c_uint8 * max(n_out, 1))()
    st = abi.load().vexq_plan_run_global_noalloc(op.h, rg_start, rg_end, stream, vals, valid, n_out)
    return st, list(vals)[:n_out], list(valid)[:n_out]


def decode(types, vals, valid):
    row = []
    for t, v, ok in zip(types, vals, valid):
        if not ok:
            row.append(None)
        elif t == abi.TYPE_FLOAT64:
            row.append(struct.unpack("<d", struct.pack("<q", v))[0])
        elif t == abi.TYPE_BOOL:
            row.append(v != 0)
        else:
            row.append(v)
    return tuple(row)


def same(a, b):
    assert len(a) == len(b)
    for x, y in zip(a, b):
        if x is None or y is None:
            assert x is None and y is None, (a, b)
        elif isinstance(x, float):
            if math.isnan(x) or math.isnan(y):
                assert math.isnan(x) and math.isnan(y), (a, b)
            else:
                assert abs(x - y) <= FLOAT_RTOL * max(abs(x), abs(y), 1e-300), (a, b)
        else:
            assert x == y, (a, b)


def check_plan(X, table, plan, rg_start=0, rg_end=-1, stream=None):
    op = X.GpuHashAggregate(table, plan)
    try:
        ref = op.run(rg_start, rg_end)
        ref.collect()
        expect = ref.rows()
        assert len(expect) == 1
        n = ref.ncols
        rows = []
        for _ in range(2):  # two calls in a row
            st, vals, valid = noalloc(op, n, rg_start, rg_end, stream)
            assert st == abi.OK, abi.load().vexq_last_error()
            rows.append(decode(ref.types, vals, valid))
        same(rows[0], expect[0])
        same(rows[1], expect[0])
        assert rows[0] == rows[1] or all(
            (a is None and b is None) or a == b or (isinstance(a, float) and math.isnan(a) and math.isnan(b))
            for a, b in zip(rows[0], rows[1]))
        ref.close()
        return rows[0]
    finally:
        op.close()


@pytest.fixture(scope="module")
def lineitem(gpu_lib):
    return gpu_lib.GpuTable(D.lineitem(1_000_000, seed=5, rg_rows=65536))


def test_q6_range_sum(gpu_lib, lineitem):
    row = check_plan(gpu_lib, lineitem, W.q6_plan())
    assert row[0] is not None and row[0] > 0


def test_many_aggregates(gpu_lib, lineitem):
    L = D
    aggs = [P.count_star("n"), P.count(P.col(L.L_QTY), "nq"), P.sum_(P.col(L.L_QTY), "sq"),
            P.sum_(P.col(L.L_PRICE), "sp"), P.avg(P.col(L.L_DISC), "ad"), P.avg(P.col(L.L_QTY), "aq"),
            P.min_(P.col(L.L_PRICE), "minp"), P.max_(P.col(L.L_PRICE), "maxp"),
            P.min_(P.col(L.L_SHIPDATE), "mind"), P.max_(P.col(L.L_QTY), "maxq"),
            P.sum_(P.col(L.L_PRICE) * (1 - P.col(L.L_DISC)), "rev")]
    plan = P.AggPlan(P.col(L.L_SHIPDATE) <= P.lit("1998-09-02"), [], aggs)
    check_plan(gpu_lib, lineitem, plan)


def test_row_group_subrange_and_stream(gpu_lib, lineitem):
    import torch
    s = torch.cuda.Stream()
    check_plan(gpu_lib, lineitem, W.q6_plan(), rg_start=3, rg_end=11, stream=C.c_void_p(s.cuda_stream))


def test_everything_pruned(gpu_lib, lineitem):
    # zone maps drop every row group: COUNT is 0 and the other aggregates NULL
    plan = P.AggPlan(P.col(D.L_SHIPDATE) < P.lit("1980-01-01"),
                     [], [P.count_star("n"), P.sum_(P.col(D.L_PRICE), "s"), P.min_(P.col(D.L_QTY), "m")])
    row = check_plan(gpu_lib, lineitem, plan)
    assert row == (0, None, None)


def test_nullable_columns(gpu_lib):
    rng = np.random.default_rng(3)
    n = 50_000
    a = rng.integers(-50, 50, n)
    b = np.round(rng.normal(0, 100, n), 3)
    d = (10000 + rng.integers(0, 400, n)).astype(np.int32)
    va, vb, vd = (rng.random(n) > p for p in (0.1, 0.15, 0.05))
    t = gpu_lib.GpuTable(HostTable([int_column("a", a, va), float_column("b", b, vb), date_column("d", d, vd)], n, 4096))
    aggs = [P.count_star("n"), P.count(P.col(1), "nb"), P.sum_(P.col(0), "sa"), P.avg(P.col(1), "ab"),
            P.min_(P.col(2), "mind"), P.max_(P.col(1), "maxb"), P.sum_(P.col(1) * 2 - 1, "sb")]
    check_plan(gpu_lib, t, P.AggPlan(P.col(0) > -10, [], aggs))
    # a predicate nothing satisfies: the empty-aggregate row
    row = check_plan(gpu_lib, t, P.AggPlan(P.col(0) > 1000, [], aggs))
    assert row[0] == 0 and row[1] == 0 and all(v is None for v in row[2:])


def test_no_device_memory_taken(gpu_lib, lineitem):
    import torch
    op = gpu_lib.GpuHashAggregate(lineitem, W.q6_plan())
    try:
        st, _, _ = noalloc(op, 1)  # set-up call
        assert st == abi.OK
        torch.cuda.mem_get_info()
        free0, _ = torch.cuda.mem_get_info()
        outs = [noalloc(op, 1) for _ in range(2)]
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0
        assert outs[0] == outs[1]
    finally:
        op.close()


def test_rejections(gpu_lib, lineitem):
    L = abi.load()
    # GROUP BY plans are not served by this entry point
    op = gpu_lib.GpuHashAggregate(lineitem, W.q1_plan())
    try:
        st, _, _ = noalloc(op, 10)
        assert st == abi.ENOTSUP and b"GROUP BY" in L.vexq_last_error()
    finally:
        op.close()
    # output count must match the plan
    op = gpu_lib.GpuHashAggregate(lineitem, W.q6_plan())
    try:
        st, _, _ = noalloc(op, 3)
        assert st == abi.EINVAL and b"n_out" in L.vexq_last_error()
    finally:
        op.close()
    # more row ranges after zone-map pruning than the entry point keeps
    rg, nrg = 1024, 1200
    k = (np.arange(nrg * rg) // rg) % 2  # constant per row group: even groups 0, odd 1
    t = gpu_lib.GpuTable(HostTable([int_column("k", k.astype(np.int64))], nrg * rg, rg))
    op = gpu_lib.GpuHashAggregate(t, P.AggPlan(P.col(0) == 0, [], [P.count_star("n")]))
    try:
        st, _, _ = noalloc(op, 1)
        assert st == abi.EINVAL and b"512" in L.vexq_last_error()
        # the allocating entry point still answers: 600 row groups of 1024 rows
        r = op.run()
        assert r.rows() == [(600 * rg,)]
        r.close()
    finally:
        op.close()
