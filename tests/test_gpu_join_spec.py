"""GPU tests of the speculative direct-mapped join build: when the last build
of a plan was direct-mapped over the same rows, the next build is launched
and the probe follows it without the host reading the build's outcome; the
probe's first thread raises a failed build (a repeated key), an empty build,
or more build keys than the group table sized from the last build holds, and
the host runs the query again reading the build first. The state that makes
a run speculate is set on the host (vexq_debug_join_spec); every case must
give the oracle's rows (joinHashTable semantics, exec/join_table.go:111-569;
an empty build joins no row, exec/parallel_join.go:790-795)."""
from __future__ import annotations

import ctypes as C

import pytest

from oracle import refcpu as R
from tests.helpers import assert_rows_match, assert_sorted_rows_match
from tests.test_gpu_join import bits_equal
from tests.test_gpu_join_direct import sparse_tables
from vexq_b200 import abi, datagen as D, workloads as W
from vexq_b200.plan import JoinPlan, col, count_star, sum_

pytestmark = pytest.mark.gpu


def speculate(op, keys_seen):
    abi.check(abi.load().vexq_debug_join_spec(op.h, C.c_int64(keys_seen)))


def test_more_keys_than_the_table_holds(gpu_lib):
    X = gpu_lib
    o, i = D.orders(100_000, seed=51), D.items(400_000, 100_000, seed=52)
    go, gi = X.GpuTable(o), X.GpuTable(i)
    plan = W.q3_plan(limit=-1)
    op = X.GpuParallelHashJoinAggregate(go, gi, plan)
    try:
        first = op.run().rows()
        assert "build=direct" in op.explain()
        speculate(op, 10)  # a group table of 10 slots for ~48K keys: the probe raises it
        second = op.run().rows()
        third = op.run().rows()  # speculative again, now with the true key count
        assert bits_equal(first, second) and bits_equal(first, third)
        ref = R.join(R.RefTable(o), R.RefTable(i), plan, workers=0)
        assert_sorted_rows_match(second, ref.rows(), plan.order_col, plan.descending)
    finally:
        op.close()
        go.close()
        gi.close()


def test_repeated_key_under_speculation(gpu_lib):
    X = gpu_lib
    b, p = sparse_tables(dup=True)
    gb, gp = X.GpuTable(b), X.GpuTable(p)
    plan = JoinPlan(0, 0, None, None, None, [0], [sum_(col(3), "s"), count_star("n")], order_col=0)
    op = X.GpuParallelHashJoinAggregate(gb, gp, plan)
    try:
        first = op.run().rows()
        assert "build=hash" in op.explain()
        speculate(op, 2500)  # forget the repeated key: the next build is direct-mapped, unchecked
        second = op.run().rows()
        assert "build=hash" in op.explain()
        ref = R.join(R.RefTable(b), R.RefTable(p), plan, workers=0)
        assert bits_equal(first, second)
        assert_rows_match(second, ref.rows(), ordered=True)
    finally:
        op.close()
        gb.close()
        gp.close()


@pytest.mark.parametrize("grouped", [False, True])
def test_empty_build_under_speculation(gpu_lib, grouped):
    X = gpu_lib
    b, p = sparse_tables()
    gb, gp = X.GpuTable(b), X.GpuTable(p)
    none = col(1) > 1000  # the build values are 0..99: no build row passes
    plan = JoinPlan(0, 0, none, None, None, [0] if grouped else [], [sum_(col(3), "s"), count_star("n")],
                    order_col=0 if grouped else -1)
    op = X.GpuParallelHashJoinAggregate(gb, gp, plan)
    try:
        first = op.run().rows()
        speculate(op, 5)
        second = op.run().rows()
        ref = R.join(R.RefTable(b), R.RefTable(p), plan, workers=0)
        # no group, or the one all-NULL row of a global aggregate over no rows
        assert first == second == ref.rows(), (first, second, ref.rows())
    finally:
        op.close()
        gb.close()
        gp.close()
