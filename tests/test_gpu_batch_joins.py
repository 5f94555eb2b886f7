"""GPU tests of joins inside the batched launch (vexq_batch_*): a join whose
build can be direct-mapped runs its build as work units of a build-class
persistent launch and its probe as units of the register or group-table
class launch, in the same captured graph as the batch's aggregates. Every
batched join result must equal the join run on its own bit for bit (group
tables are exact; the register-path join counts are integers) and the
oracle (exec/parallel_join.go:780-988). A join whose key range is too wide
for a direct-mapped table, and one whose build repeats a key, run on their
own after the graph and still give the oracle's rows."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import refcpu as R
from tests.helpers import assert_rows_match, assert_sorted_rows_match
from tests.test_gpu_join import bits_equal
from tests.test_gpu_join_direct import sparse_plans, sparse_tables
from vexq_b200 import datagen as D, workloads as W
from vexq_b200.plan import JoinPlan, col, count_star, sum_
from vexq_b200.table import HostTable, float_column, int_column

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def join_batch(gpu_lib):
    X = gpu_lib
    o, i = D.orders(200_000, seed=41), D.items(800_000, 200_000, seed=42)
    b, p = sparse_tables()
    bd, pd = sparse_tables(dup=True)
    rng = np.random.default_rng(8)
    wk = np.unique(rng.integers(0, 1 << 40, 6000))[:5000]
    rng.shuffle(wk)
    wp = np.concatenate([wk[rng.integers(0, 5000, 20_000)], rng.integers(0, 1 << 40, 5000)])
    wb = HostTable([int_column("k", wk)], 5000, 1024)
    wpr = HostTable([int_column("fk", wp), float_column("v", np.round(rng.random(25_000) * 100, 2))], 25_000, 4096)
    li = D.lineitem(300_000, seed=43, rg_rows=65536)
    host = {"o": o, "i": i, "b": b, "p": p, "bd": bd, "pd": pd, "wb": wb, "wp": wpr, "li": li}
    tabs = {k: X.GpuTable(v) for k, v in host.items()}
    sp = sparse_plans()
    by_key = JoinPlan(0, 0, None, None, None, [0], [sum_(col(3), "s"), count_star("n")], order_col=0)
    wide = JoinPlan(0, 0, None, None, None, [0], [sum_(col(2), "s"), count_star("n")], order_col=0)
    cases = [  # (name, kind, build, probe, plan, batched)
        ("q3", "join", "o", "i", W.q3_plan(), True),
        ("q3_all", "join", "o", "i", W.q3_plan(limit=-1), True),
        ("q12", "join", "o", "i", W.q12_plan(), True),
        ("sparse_by_key", "join", "b", "p", sp["by_key"], True),
        ("sparse_by_build_col", "join", "b", "p", sp["by_build_col"], True),
        ("sparse_global", "join", "b", "p", sp["global"], True),
        ("repeated_key", "join", "bd", "pd", by_key, False),  # its single run below sends it to the hash build
        ("wide_range", "join", "wb", "wp", wide, False),
        ("q1", "agg", "li", None, W.q1_plan(), None),
        ("q6", "agg", "li", None, W.q6_plan(), None),
    ]
    ops = [X.GpuParallelHashJoinAggregate(tabs[bt], tabs[pt], plan) if kind == "join" else X.GpuHashAggregate(tabs[bt], plan)
           for _, kind, bt, pt, plan, _ in cases]
    yield X, cases, ops, host
    for op in ops:
        op.close()
    for t in tabs.values():
        t.close()


def single_rows(ops):
    out = []
    for op in ops:
        r = op.run()
        out.append(r.rows())
        r.close()
    return out


def test_batched_joins_match_single_runs_and_oracle(join_batch):
    X, cases, ops, host = join_batch
    single = single_rows(ops)
    b = X.GpuBatch(ops)
    try:
        ex = b.explain()
        assert f"joins={sum(1 for c in cases if c[5])}" in ex, ex
        for attempt in range(2):  # the first execution captures the graph, the second replays it
            res = b.exec()
            for k, (name, kind, bt, pt, plan, _) in enumerate(cases):
                rows = res[k].rows()
                if kind == "agg":
                    assert_rows_match(rows, single[k], ordered=True, rtol=1e-13)
                    continue
                assert bits_equal(rows, single[k]), (name, attempt)
                ref = R.join(R.RefTable(host[bt]), R.RefTable(host[pt]), plan, workers=0)
                if name.startswith("q3"):
                    assert_sorted_rows_match(rows, ref.rows(), plan.order_col, plan.descending)
                else:
                    assert_rows_match(rows, ref.rows(), ordered=True)
        assert "build=hash" in ops[[c[0] for c in cases].index("repeated_key")].explain()
        ms, kms, nbytes, nrows = b.stats()
        assert ms >= kms > 0 and nbytes > 0 and nrows > 0
    finally:
        b.close()


def test_batched_repeated_key_falls_back(gpu_lib):
    """A join batched before any single run whose build repeats a key: the
    build raises it, the join runs on its own (hash build) and its rows are
    the oracle's; the next batch leaves it out."""
    X = gpu_lib
    bd, pd = sparse_tables(dup=True)
    gb, gp = X.GpuTable(bd), X.GpuTable(pd)
    plan = JoinPlan(0, 0, None, None, None, [0], [sum_(col(3), "s"), count_star("n")], order_col=0)
    op = X.GpuParallelHashJoinAggregate(gb, gp, plan)
    try:
        b = X.GpuBatch([op])
        try:
            assert "joins=1" in b.explain()
            rows = b.exec()[0].rows()
        finally:
            b.close()
        ref = R.join(R.RefTable(bd), R.RefTable(pd), plan, workers=0)
        assert_rows_match(rows, ref.rows(), ordered=True)
        assert "build=hash" in op.explain()
        b2 = X.GpuBatch([op])
        try:
            assert "joins=0" in b2.explain()
        finally:
            b2.close()
    finally:
        op.close()
        gb.close()
        gp.close()


def test_batched_joins_beat_one_by_one(join_batch):
    """Kernel time of one batched execution of the batchable joins against
    the same plans run one by one (their kernel times summed)."""
    X, cases, ops, _ = join_batch
    sel = [op for op, c in zip(ops, cases) if c[5]]
    b = X.GpuBatch(sel)
    try:
        for _ in range(3):
            for r in b.exec():
                r.close()
        times = []
        for _ in range(5):
            for r in b.exec():
                r.close()
            times.append(b.stats()[1])  # the replay's kernels, start to end
        batched = min(times)
        plain = 0.0
        for op in sel:
            for _ in range(2):
                op.run().close()
            ts = []
            for _ in range(5):
                r = op.run()
                ts.append(r.kernel_ms)
                r.close()
            plain += min(ts)
        assert batched < plain, (batched, plain)
    finally:
        b.close()
