"""GPU tests of sharded execution: N shards of row groups (run one after
another on one GPU, as N ranks would run them on N GPUs), each a partial
through vexq_plan_run_partial, serialised, read back and merged in shard
order (vexq_partial_merge). The merged result must equal the single run and
the oracle: keys, counts, integer aggregates and MIN/MAX exact; float sums
within 1e-12 of the oracle's serial fold and 1e-13 of the exact sum (each
shard's sum is rounded once before the merge)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from oracle import refcpu as R
from vexq_b200 import abi, datagen as D, plan as P, workloads as W
from vexq_b200.sharded import merge_in_rank_order, shard_range
from vexq_b200.table import HostTable, float_column, int_column

from tests.helpers import assert_float_vs_exact, assert_rows_match

pytestmark = pytest.mark.gpu


def sharded_rows(op, n_rg, world):
    parts = [op.run_partial(*shard_range(n_rg, r, world)) for r in range(world)]
    r = merge_in_rank_order(op, parts)
    try:
        return r.rows()
    finally:
        r.close()


@pytest.fixture(scope="module")
def lineitem(gpu_lib):
    host = D.lineitem(1_000_000, seed=61, rg_rows=65536)
    return host, gpu_lib.GpuTable(host), R.RefTable(host)


@pytest.mark.parametrize("world", [1, 2, 3, 7])
@pytest.mark.parametrize("q", ["q1", "q6"])
def test_sharded_register_path(gpu_lib, lineitem, q, world):
    host, gt, rt = lineitem
    plan = W.q1_plan() if q == "q1" else W.q6_plan()
    op = gpu_lib.GpuHashAggregate(gt, plan)
    try:
        rows = sharded_rows(op, host.n_rg, world)
        ref = R.agg(rt, plan, workers=0)
        assert_float_vs_exact(rows, ref, ordered=True)
    finally:
        op.close()


@pytest.mark.parametrize("card", [97, 65536])
def test_sharded_dense_table(gpu_lib, card):
    X = gpu_lib
    host = D.zipf_groups(600_000, card, seed=card, rg_rows=32768)
    op = X.GpuHashAggregate(X.GpuTable(host), W.batch_plan())
    try:
        ref = R.agg(R.RefTable(host), W.batch_plan(), workers=0)
        for world in (2, 5):
            assert_float_vs_exact(sharded_rows(op, host.n_rg, world), ref, ordered=True)
    finally:
        op.close()


def test_sharded_hash_path_having_order_limit(gpu_lib):
    X = gpu_lib
    rng = np.random.default_rng(8)
    n = 800_000
    keys = rng.integers(0, 1 << 40, 60_000)[rng.integers(0, 60_000, n)]
    vals = np.rint(rng.uniform(0, 1e5, n)) / 100.0
    host = HostTable([int_column("k", keys), float_column("v", vals)], n, 65536)
    aggs = [P.sum_(P.col(1), "s"), P.count_star("c"), P.max_(P.col(1), "m")]
    plan = P.AggPlan(None, [0], aggs, order_col=1, descending=True, limit=25, having=P.col(2) >= 12)
    op = X.GpuHashAggregate(X.GpuTable(host), plan)
    try:
        rows = sharded_rows(op, host.n_rg, 4)
        assert "path=hash" in op.explain()
    finally:
        op.close()
    ref = R.agg_having(R.RefTable(host), P.AggPlan(None, [0], aggs), P.col(2) >= 12, -1, order=(1, 1, 25))
    assert_rows_match(rows, ref.rows(), ordered=True)


def test_sharded_join_probe_side(gpu_lib):
    X = gpu_lib
    o, i = D.orders(200_000, seed=12), D.items(800_000, 200_000, seed=13, rg_rows=65536)
    op = X.GpuParallelHashJoinAggregate(X.GpuTable(o), X.GpuTable(i), W.q3_plan(limit=-1))
    try:
        rows = sharded_rows(op, i.n_rg, 3)
        single = op.run().rows()
    finally:
        op.close()
    ref = R.join(R.RefTable(o), R.RefTable(i), W.q3_plan(limit=-1), workers=0)
    assert len(rows) == len(single) == ref.nrows
    assert_float_vs_exact(rows, ref, ordered=True)


def test_partial_errors(gpu_lib, lineitem):
    X = gpu_lib
    host, gt, _ = lineitem
    q1, q6 = X.GpuHashAggregate(gt, W.q1_plan()), X.GpuHashAggregate(gt, W.q6_plan())
    L = abi.load()
    try:
        b = q1.run_partial(0, 3)
        # another plan's shape, bad magic, truncated bytes
        for bad, plan in ((b, q6), (b"XXXX" + b[4:], q1), (b[:-8], q1)):
            h = C.c_void_p()
            buf = C.create_string_buffer(bad, len(bad))
            assert L.vexq_partial_deserialize(plan.h, buf, len(bad), C.byref(h)) == abi.EINVAL
        d = X.GpuHashAggregate(gt, P.AggPlan(None, [0], [P.count_distinct(P.col(2), "d")]))
        part = C.c_void_p()
        assert L.vexq_plan_run_partial(d.h, 0, -1, C.byref(part)) == abi.ENOTSUP
        d.close()
        # no shards: the empty global aggregate's one row (COUNT 0)
        r = q6.merge_partials([])
        assert r.rows() == [(None,)]
    finally:
        q1.close()
        q6.close()
