"""GPU tests of COUNT(DISTINCT) (exec/aggregate.go:117-124, 474-493,
810-823), through the C ABI: the reference's own cases (the known answers
in tests/golden, run by test_gpu_parity), then larger plans against the
oracle on every path — the register path (≤16 groups), a dense group table,
a hash table — with NULLs, float images (+0 / -0 and NaN payloads count
apart, as raw bits do), strings that carry different codes per row group,
a predicate, HAVING and ORDER BY over the count, and the refusals."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import refcpu as R
from vexq_b200 import abi, datagen as D, plan as P
from vexq_b200.table import HostTable, date_column, float_column, int_column, string_column

from tests.helpers import assert_rows_match

pytestmark = pytest.mark.gpu


def table(n=400_000, seed=1, groups=7, rg_rows=65536):
    rng = np.random.default_rng(seed)
    g = rng.integers(0, groups, n)
    small = rng.integers(0, 50, n)
    wide = rng.integers(0, 1 << 40, 30_000)[rng.integers(0, 30_000, n)]
    f = np.round(rng.normal(0, 10, n), 1)
    f[rng.random(n) < 0.01] = -0.0
    d = (9000 + rng.integers(0, 900, n)).astype(np.int32)
    s = rng.integers(0, 300, n)
    vs, vf = rng.random(n) > 0.1, rng.random(n) > 0.05
    cols = [int_column("g", g), int_column("small", small, vs), int_column("wide", wide), float_column("f", f, vf),
            date_column("d", d), string_column("s", s, [f"v{i:03d}" for i in range(300)], n, rg_rows)]
    return HostTable(cols, n, rg_rows)


def check(X, host, plan):
    op = X.GpuHashAggregate(X.GpuTable(host), plan)
    try:
        rows = op.run().rows()
        ex = op.explain()
    finally:
        op.close()
    ref = R.agg(R.RefTable(host), plan, workers=0)
    assert_rows_match(rows, ref.rows(), ordered=True, rtol=0.0)
    return rows, ex


def aggs():
    return [P.count_distinct(P.col(1), "d_small"), P.count_distinct(P.col(2), "d_wide"),
            P.count_distinct(P.col(3), "d_f"), P.count_distinct(P.col(4), "d_d"), P.count_star("n"),
            P.count(P.col(1), "n_small")]


@pytest.mark.parametrize("groups,path", [(1, "regs"), (7, "regs"), (5000, "dense")])
def test_count_distinct_paths(gpu_lib, groups, path):
    host = table(groups=groups)
    gb = [] if groups == 1 else [0]
    rows, ex = check(gpu_lib, host, P.AggPlan(None, gb, aggs()))
    assert f"path={path}" in ex, ex
    rows, _ = check(gpu_lib, host, P.AggPlan(P.col(4) < "1995-06-01", gb, aggs()[:3] + [P.sum_(P.col(1), "s")]))


def test_count_distinct_hash_path_and_strings(gpu_lib):
    host = table(n=300_000, seed=2)
    # GROUP BY a wide int64 column: the hash path; distinct strings per group
    rows, ex = check(gpu_lib, host, P.AggPlan(None, [2], [P.count_distinct(P.col(5), "d_s"), P.count_star("n")]))
    assert "path=hash" in ex, ex
    # strings with per-row-group dictionaries, grouped by a string
    rows, _ = check(gpu_lib, host, P.AggPlan(None, [5], [P.count_distinct(P.col(1), "d"), P.min_(P.col(5), "lo")]))


def test_count_distinct_float_images(gpu_lib):
    vals = np.array([0.0, -0.0, 1.5, 1.5, float("nan"), float("nan"), float("inf"), 2.0], dtype=np.float64)
    n = 8
    host = HostTable([int_column("g", np.array([0, 0, 0, 1, 1, 1, 1, 1])), float_column("f", vals)], n, 65536)
    rows, _ = check(gpu_lib, host, P.AggPlan(None, [0], [P.count_distinct(P.col(1), "d")]))
    assert rows == [(0, 3), (1, 4)]


def test_count_distinct_having_and_order(gpu_lib):
    host = table(n=200_000, seed=3, groups=5000)
    plan = P.AggPlan(None, [0], [P.count_distinct(P.col(1), "d"), P.count_star("n")], order_col=1, descending=True,
                     limit=20, having=P.col(1) >= 40)
    X = gpu_lib
    op = X.GpuHashAggregate(X.GpuTable(host), plan)
    try:
        rows = op.run().rows()
    finally:
        op.close()
    ref = R.agg_having(R.RefTable(host), P.AggPlan(None, [0], plan.aggs), P.col(1) >= 40, -1, order=(1, 1, 20))
    assert_rows_match(rows, ref.rows(), ordered=True, rtol=0.0)


def test_count_distinct_twice_and_refusals(gpu_lib):
    X = gpu_lib
    host = table(n=100_000, seed=4)
    gt = X.GpuTable(host)
    op = X.GpuHashAggregate(gt, P.AggPlan(None, [0], aggs()))
    try:
        a = op.run().rows()
        b = op.run().rows()
        assert a == b  # the sets start empty on every run
        # the no-allocation entry point refuses (its sets would need memory)
        g = X.GpuHashAggregate(gt, P.AggPlan(None, [], [P.count_distinct(P.col(1), "d")]))
        import ctypes as C
        vals, valid = (C.c_int64 * 1)(), (C.c_uint8 * 1)()
        assert abi.load().vexq_plan_run_global_noalloc(g.h, 0, -1, None, vals, valid, 1) == abi.ENOTSUP
        g.close()
    finally:
        op.close()
    o, i = X.GpuTable(D.orders(1000, seed=1)), X.GpuTable(D.items(4000, 1000, seed=2))
    with pytest.raises(abi.VexqError) as e:
        X.GpuParallelHashJoinAggregate(o, i, P.JoinPlan(0, 0, None, None, None, [0], [P.count_distinct(P.col(4), "d")]))
    assert e.value.status == abi.ENOTSUP
