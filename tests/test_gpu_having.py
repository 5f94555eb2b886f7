"""GPU tests of HAVING over the merged aggregate (vexq_plan_set_having): the
reference's own cases (planner/having_test.go, through the CASES table the
oracle is pinned on), then larger plans checked against the oracle's HAVING
(exec.Filter over the output, the column cut, ExternalSort + Limit): float
AVG ranges, string keys, NULL aggregates, HAVING before ORDER BY / LIMIT on a
hash-path aggregate with many groups (no device top-k), and a join."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import refcpu as R
from tests.helpers import assert_float_vs_exact, assert_rows_match
from tests.test_having_oracle import CASES, grouped_table
from tests.test_vxq_cpu import mixed_table
from vexq_b200 import abi, datagen as D, plan as P
from vexq_b200.plan import JoinPlan, col, lit, sum_
from vexq_b200.table import HostTable, float_column, int_column

pytestmark = pytest.mark.gpu


def gpu_rows(X, table, plan):
    op = X.GpuHashAggregate(table, plan)
    try:
        return op.run().rows(), op.explain()
    finally:
        op.close()


def test_reference_cases(gpu_lib):
    X = gpu_lib
    gt = X.GpuTable(grouped_table())
    for name, (aggs, having, visible, want) in CASES.items():
        rows, _ = gpu_rows(X, gt, P.AggPlan(None, [0], aggs, having=having, visible=visible))
        assert {r[0]: r for r in rows} == want, (name, rows)


def test_reference_cases_on_device(gpu_lib, monkeypatch):
    """The reference's six HAVING cases with the groups in a device group
    table (the register path turned off for the fixture's few groups), so the
    predicate runs on the device (vq_having) before the groups come back."""
    X = gpu_lib
    monkeypatch.setenv("VEXQ_TUNE", "regs_groups=0")
    gt = X.GpuTable(grouped_table())
    for name, (aggs, having, visible, want) in CASES.items():
        rows, explain = gpu_rows(X, gt, P.AggPlan(None, [0], aggs, having=having, visible=visible))
        assert "path=dense" in explain and "having=device" in explain, (name, explain)
        assert {r[0]: r for r in rows} == want, (name, rows)


def test_having_over_float_avg_string_keys_and_nulls(gpu_lib):
    X = gpu_lib
    n = 200_000
    host = mixed_table(n, 65536, 21)
    rt = R.RefTable(host)
    gt = X.GpuTable(host)
    aggs = [P.count_star("n"), P.avg(P.col(1), "af"), P.sum_(P.col(0), "si"), P.min_(P.col(2), "md"),
            P.max_(P.col(0), "mx")]
    cases = [
        # AVG(f) in a range, over (string, bool) groups: outputs s, b, n, af, si, md, mx
        (P.between(P.col(3), -1.0, 1.0), -1),
        (P.and_(P.col(0) == P.lit("MAIL"), P.col(2) > 1000), -1),
        (P.or_(P.is_null(P.col(0)), P.is_null(P.col(1))), 4),  # NULL keys; keep s, b, n, af
        (P.not_(P.col(5) >= P.lit("1995-01-01")), -1),
        (P.col(2) * 2 > P.col(2) + 3000, 3),
    ]
    for having, visible in cases:
        plan = P.AggPlan(None, [3, 4], aggs, having=having, visible=visible)
        rows, _ = gpu_rows(X, gt, plan)
        ref = R.agg_having(rt, P.AggPlan(None, [3, 4], aggs), having, visible)
        assert_rows_match(rows, ref.rows(), ordered=True)
        assert_float_vs_exact(rows, ref)
    # SUM / MIN / MAX over a group whose values are all NULL are NULL
    grp = np.array([0] * 4 + [1] * 4, dtype=np.int64)
    val = np.array([5, 6, 7, 8, 0, 0, 0, 0], dtype=np.int64)
    valid = np.array([1, 1, 1, 1, 0, 0, 0, 0], dtype=bool)
    small = HostTable([int_column("g", grp), int_column("v", val, valid)], 8, 65536)
    plan_aggs = [P.sum_(P.col(1), "s"), P.count(P.col(1), "c")]
    for having in (P.is_null(P.col(1)), P.col(1) > 0, P.col(2) == 0):
        rows, _ = gpu_rows(X, X.GpuTable(small), P.AggPlan(None, [0], plan_aggs, having=having))
        ref = R.agg_having(R.RefTable(small), P.AggPlan(None, [0], plan_aggs), having)
        assert rows == ref.rows(), (rows, ref.rows())


def test_having_before_order_and_limit_on_many_groups(gpu_lib):
    """200,000 int64 keys (hash path): HAVING keeps groups with at least four
    rows, then ORDER BY the sum DESC LIMIT 10 over what is left."""
    X = gpu_lib
    rng = np.random.default_rng(22)
    n = 2_000_000
    keys = rng.integers(0, 1 << 40, 200_000)[rng.integers(0, 200_000, n)]
    vals = np.rint(rng.uniform(0, 1e5, n)) / 100.0
    host = HostTable([int_column("k", keys), float_column("v", vals)], n, 65536)
    aggs = [P.sum_(P.col(1), "s"), P.count_star("c")]
    having = P.col(2) >= 14
    plan = P.AggPlan(None, [0], aggs, order_col=1, descending=True, limit=10, having=having)
    rows, ex = gpu_rows(X, X.GpuTable(host), plan)
    assert "path=hash" in ex and "having=device" in ex, ex
    ref = R.agg_having(R.RefTable(host), P.AggPlan(None, [0], aggs), having, -1, order=(1, 1, 10))
    assert len(rows) == 10 and all(r[2] >= 14 for r in rows)
    assert_rows_match(rows, ref.rows(), ordered=True)


def test_having_on_a_join(gpu_lib):
    X = gpu_lib
    ob = D.orders(300_000, seed=3)
    it = D.items(1_200_000, 300_000, seed=4)
    bmid, pmid = D.join_mid(0.5), D.join_mid(0.4)
    price, disc = col(3 + D.I_PRICE), col(3 + D.I_DISC)

    def plan(order):
        kw = dict(order_col=1, descending=True, limit=10) if order else {}
        return JoinPlan(D.O_KEY, D.I_FK, col(D.O_DATE) < lit(bmid), col(D.I_SHIPDATE) > lit(pmid), None,
                        [D.O_KEY], [sum_(price * (1 - disc), "revenue"), P.count_star("n")],
                        having=(P.col(2) >= 3) if order else None, **kw)
    op = X.GpuParallelHashJoinAggregate(X.GpuTable(ob), X.GpuTable(it), plan(True))
    try:
        rows = op.run().rows()
    finally:
        op.close()
    ref = R.join_having(R.RefTable(ob), R.RefTable(it), plan(False), P.col(2) >= 3, -1, order=(1, 1, 10))
    assert len(rows) == 10 and all(r[2] >= 3 for r in rows)
    assert_rows_match(rows, ref.rows(), ordered=True)


def test_having_errors(gpu_lib):
    X = gpu_lib
    gt = X.GpuTable(grouped_table())
    with pytest.raises(abi.VexqError):  # not a boolean
        X.GpuHashAggregate(gt, P.AggPlan(None, [0], [P.count_star("c")], having=P.col(1) + 1))
    with pytest.raises(abi.VexqError):  # more columns kept than the aggregate outputs
        X.GpuHashAggregate(gt, P.AggPlan(None, [0], [P.count_star("c")], having=P.col(1) > 1, visible=3))
    with pytest.raises(abi.VexqError):  # an output column that does not exist
        X.GpuHashAggregate(gt, P.AggPlan(None, [0], [P.count_star("c")], having=P.col(2) > 1))
