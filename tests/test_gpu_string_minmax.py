"""GPU tests of MIN/MAX over STRING columns (HashAggregate.strAccs,
exec/aggregate.go:98-110; mergePartialAgg, exec/parallel.go:283-297): the
slot keeps the string's rank in the dictionary's byte order, so results must
equal the oracle's byte-wise string comparison — empty strings, prefixes,
bytes above 0x7F, NULLs and all-NULL groups — on the register, dense and
hash paths, in a join (a build-side string), under HAVING and ORDER BY, and in
a batch."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import refcpu as R
from tests.helpers import assert_rows_match
from vexq_b200 import abi, datagen as D, plan as P
from vexq_b200.plan import JoinPlan, col, lit
from vexq_b200.table import HostTable, int_column, string_column

pytestmark = pytest.mark.gpu

WORDS = ["", "a", "ab", "abc", "abd", "b", "B", "Z", "zz", "été", "é", "a b", "abÿ", "0", "9",
         "TRUCK", "AIR", "REG AIR", "~", "aaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaaa"]


def string_table(n: int, ngroups: int, seed: int, rg: int = 8192) -> HostTable:
    rng = np.random.default_rng(seed)
    g = rng.integers(0, ngroups, n)
    widx = rng.integers(0, len(WORDS), n)
    valid = rng.random(n) > 0.15
    valid[g == ngroups - 1] = False  # one group with only NULL strings
    kidx = rng.integers(0, 3, n)
    cols = [int_column("g", g.astype(np.int64)), string_column("w", widx, WORDS, n, rg, valid),
            string_column("k", kidx, ["x", "y", "z"], n, rg)]
    return HostTable(cols, n, rg)


def run(X, table, plan):
    op = X.GpuHashAggregate(table, plan)
    try:
        return op.run().rows(), op.explain()
    finally:
        op.close()


AGGS = [P.min_(P.col(1), "mn"), P.max_(P.col(1), "mx"), P.count(P.col(1), "c"), P.count_star("n")]


@pytest.mark.parametrize("ngroups,path", [(3, "regs"), (1000, "dense"), (60000, "hash")])
def test_string_min_max_by_path(gpu_lib, ngroups, path):
    X = gpu_lib
    host = string_table(300_000, ngroups, 31)
    gt, rt = X.GpuTable(host), R.RefTable(host)
    key = [2] if path == "regs" else [0]
    if path == "hash":  # int64 keys spread over a wide range
        host.columns[0].values[:] = host.columns[0].values * 1_000_003 + 17
        gt = X.GpuTable(host)
        rt = R.RefTable(host)
    rows, ex = run(X, gt, P.AggPlan(None, key, AGGS))
    assert f"path={path}" in ex, ex
    assert_rows_match(rows, R.agg(rt, P.AggPlan(None, key, AGGS), workers=0).rows(), ordered=True)


def test_all_null_group_and_global_aggregate(gpu_lib):
    X = gpu_lib
    host = string_table(50_000, 5, 32)
    gt, rt = X.GpuTable(host), R.RefTable(host)
    rows, _ = run(X, gt, P.AggPlan(None, [0], AGGS))
    assert any(r[1] is None and r[2] is None and r[3] == 0 for r in rows)  # the all-NULL group
    assert_rows_match(rows, R.agg(rt, P.AggPlan(None, [0], AGGS), workers=0).rows(), ordered=True)
    plan = P.AggPlan(P.col(0) < 4, [], AGGS)
    rows, _ = run(X, gt, plan)
    assert rows == R.agg(rt, plan, workers=0).rows()


def test_having_and_order_by_a_string_min(gpu_lib):
    X = gpu_lib
    host = string_table(200_000, 400, 33)
    gt, rt = X.GpuTable(host), R.RefTable(host)
    having = P.or_(P.col(1) == P.lit(""), P.col(2) == P.lit("~"))
    plan = P.AggPlan(None, [0], AGGS, order_col=1, descending=True, limit=25, having=having)
    rows, _ = run(X, gt, plan)
    ref = R.agg_having(rt, P.AggPlan(None, [0], AGGS), having, -1, order=(1, 1, 25))
    assert_rows_match(rows, ref.rows(), ordered=True)


def test_build_side_string_in_a_join(gpu_lib):
    X = gpu_lib
    ob = D.orders(200_000, seed=5)
    it = D.items(800_000, 200_000, seed=6)
    plan = JoinPlan(D.O_KEY, D.I_FK, None, col(D.I_SHIPDATE) > lit(D.join_mid(0.5)), None,
                    [3 + D.I_MODE], [P.min_(P.col(D.O_PRIORITY), "pmin"), P.max_(P.col(D.O_PRIORITY), "pmax"),
                                     P.count_star("n")])
    op = X.GpuParallelHashJoinAggregate(X.GpuTable(ob), X.GpuTable(it), plan)
    try:
        rows = op.run().rows()
    finally:
        op.close()
    assert_rows_match(rows, R.join(R.RefTable(ob), R.RefTable(it), plan, workers=0).rows(), ordered=True)


def test_string_min_max_in_a_batch(gpu_lib):
    X = gpu_lib
    host = string_table(100_000, 50, 34)
    gt, rt = X.GpuTable(host), R.RefTable(host)
    plans = [P.AggPlan(None, [2], AGGS), P.AggPlan(None, [0], AGGS), P.AggPlan(P.col(0) > 10, [], AGGS)]
    ops = [X.GpuHashAggregate(gt, pl) for pl in plans]
    b = X.GpuBatch(ops)
    try:
        for res, pl in zip(b.exec(), plans):
            assert_rows_match(res.rows(), R.agg(rt, pl, workers=0).rows(), ordered=True)
            res.close()
    finally:
        b.close()
        for op in ops:
            op.close()


def test_no_allocation_run_refuses_string_min(gpu_lib):
    X = gpu_lib
    host = string_table(10_000, 3, 35)
    op = X.GpuHashAggregate(X.GpuTable(host), P.AggPlan(None, [], [P.min_(P.col(1), "mn")]))
    try:
        import ctypes as C
        vals = (C.c_int64 * 4)()
        valid = (C.c_uint8 * 4)()
        rc = abi.load().vexq_plan_run_global_noalloc(op.h, 0, -1, None, vals, valid, 1)
        assert rc == abi.ENOTSUP
    finally:
        op.close()
