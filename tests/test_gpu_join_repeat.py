"""GPU tests of repeated join runs with the one-pass hash build turned on
(VEXQ_TUNE=fastbuild=1, the direct-mapped build off): a join plan whose
last build inserted every key once builds its next table in one pass
straight into the probe's slots (group numbers claimed per warp when the
GROUP BY is the join key); a first run takes the general build. Both must
give the same rows, and the reference's join known answers (duplicate keys,
NULL keys, the sentinel and extreme int64 keys) must hold on every run."""
from __future__ import annotations

import pytest

from oracle import refcpu as R
from tests.golden.fixtures import load_cases, make_plan, make_table, normalize
from tests.helpers import assert_rows_match, assert_sorted_rows_match
from vexq_b200 import datagen as D, workloads as W

pytestmark = pytest.mark.gpu

JOIN_CASES = [c for c in load_cases() if c["kind"] == "join"]


@pytest.mark.parametrize("case", JOIN_CASES, ids=[c["name"] for c in JOIN_CASES])
def test_known_answers_every_run(gpu_lib, case, monkeypatch):
    monkeypatch.setenv("VEXQ_TUNE", "fastbuild=1,dmap=0")
    X = gpu_lib
    b, p = X.GpuTable(make_table(case["tables"]["build"])), X.GpuTable(make_table(case["tables"]["probe"]))
    op = X.GpuParallelHashJoinAggregate(b, p, make_plan(case))
    ordered = case["expect"]["ordered"]
    try:
        for _ in range(3):
            assert normalize(op.run().rows(), ordered) == normalize(case["expect"]["rows"], ordered)
    finally:
        op.close()


@pytest.mark.parametrize("q", ["q3", "q3_all", "q12"])
def test_repeated_runs_agree(gpu_lib, q, monkeypatch):
    monkeypatch.setenv("VEXQ_TUNE", "fastbuild=1,dmap=0")
    X = gpu_lib
    o, i = D.orders(300_000, seed=21), D.items(1_200_000, 300_000, seed=22)
    plan = {"q3": W.q3_plan(), "q3_all": W.q3_plan(limit=-1), "q12": W.q12_plan()}[q]
    op = X.GpuParallelHashJoinAggregate(X.GpuTable(o), X.GpuTable(i), plan)
    try:
        first = op.run()
        rows1, l1 = first.rows(), first.launches
        second = op.run()
        rows2, l2 = second.rows(), second.launches
        third = op.run().rows()
    finally:
        op.close()
    assert rows1 == rows2 == third  # group-table sums are exact, so bit for bit
    assert l2 < l1, (l1, l2)        # the one-pass build: fewer launches
    ref = R.join(R.RefTable(o), R.RefTable(i), plan, workers=0)
    if q == "q12":
        assert_rows_match(rows2, ref.rows(), ordered=True, rtol=0.0)
    else:  # ORDER BY revenue: groups with equal exact sums may come in either order
        assert_sorted_rows_match(rows2, ref.rows(), plan.order_col, plan.descending)
