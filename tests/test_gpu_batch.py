"""GPU tests of batched execution (vexq_batch_*): many plans in one
persistent launch per path class under a captured CUDA graph.

Every batched result is compared with the same plan run on its own
(vexq_plan_run) and, for group-table plans, with the oracle's exact sums."""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import refcpu as R
from vexq_b200 import abi, datagen as D, plan as P, workloads as W
from vexq_b200.table import HostTable, float_column, int_column

from tests.helpers import assert_rows_match
from tests.test_gpu_parity import assert_sums_exact

pytestmark = pytest.mark.gpu

BATCH_RTOL = 1e-13  # register-path FP64 sums: a different row partition than the single run


def mix_aggs(v):
    return [P.sum_(v, "sum"), P.count_star("count"), P.min_(v, "min"), P.max_(v, "max"), P.avg(v, "avg")]


@pytest.fixture(scope="module")
def mixed(gpu_lib):
    """Tables and plans covering every batch class: register path (Q1 at two
    cutoffs, Q6, Zipf GROUP BY over 2 and 9 groups), dense tables (30 to
    65,536 groups), a hash table (int64 keys), a plan that zone maps prune
    entirely, and a join (run on its own after the graph)."""
    X = gpu_lib
    li = D.lineitem(400_000, seed=21, rg_rows=65536)
    gli = X.GpuTable(li)
    tabs, ops, hosts = [gli], [], []
    for pl in (W.q1_plan(), W.q1_plan("1995-06-17"), W.q6_plan(), W.q6_plan("1996-01-01", "1996-07-01"),
               P.AggPlan(P.col(D.L_SHIPDATE) < P.lit("1980-01-01"), [], [P.count_star("n"), P.sum_(P.col(D.L_PRICE), "s")])):
        ops.append(X.GpuHashAggregate(gli, pl))
        hosts.append((li, pl))
    for k, (card, rows) in enumerate([(2, 30_000), (9, 120_000), (30, 250_000), (1000, 90_000), (65536, 600_000)]):
        t = D.zipf_groups(rows, card, seed=100 + k)
        g = X.GpuTable(t)
        tabs.append(g)
        for pl in (P.AggPlan(None, [0], mix_aggs(P.col(1))),
                   P.AggPlan(P.col(1) > 5000.0, [0], [P.sum_(P.col(1), "s"), P.count_star("n")])):
            ops.append(X.GpuHashAggregate(g, pl))
            hosts.append((t, pl))
    rng = np.random.default_rng(5)
    n = 200_000
    keys = rng.integers(0, 1 << 40, 5000)[rng.integers(0, 5000, n)]
    vals = np.rint(rng.uniform(0, 1e6, n)) / 100.0
    ht = HostTable([int_column("k", keys.astype(np.int64)), float_column("v", vals)], n, 65536)
    g = X.GpuTable(ht)
    tabs.append(g)
    pl = P.AggPlan(None, [0], [P.sum_(P.col(1), "s"), P.max_(P.col(1), "m"), P.count_star("n")])
    ops.append(X.GpuHashAggregate(g, pl))
    hosts.append((ht, pl))
    o, i = D.orders(50_000, seed=3), D.items(200_000, 50_000, seed=4)
    go, gi = X.GpuTable(o), X.GpuTable(i)
    tabs += [go, gi]
    ops.append(X.GpuParallelHashJoinAggregate(go, gi, W.q3_plan()))
    hosts.append(None)
    yield X, tabs, ops, hosts
    for op in ops:
        op.close()


def single_rows(ops):
    out = []
    for op in ops:
        r = op.run()
        out.append(r.rows())
        r.close()
    return out


def check_against_single(results, single, ops):
    for k, (res, ref) in enumerate(zip(results, single)):
        rows = res.rows()
        assert_rows_match(rows, ref, ordered=True, rtol=BATCH_RTOL)
        if "path=regs" not in ops[k].explain():
            assert rows == ref or all(  # group tables: bit for bit
                all(a == b or (isinstance(a, float) and math.isnan(a) and math.isnan(b)) for a, b in zip(x, y))
                for x, y in zip(rows, ref)), k


def test_batch_matches_single_runs(mixed):
    X, _, ops, _ = mixed
    single = single_rows(ops)
    b = X.GpuBatch(ops)
    try:
        ex = b.explain()
        assert "regs_plans=" in ex and "table_plans=" in ex
        first = b.exec()
        check_against_single(first, single, ops)
        again = b.exec()  # a replay gives identical bits
        for r1, r2 in zip(first, again):
            assert r1.rows() == r2.rows() or all(
                all(a == c or (isinstance(a, float) and math.isnan(a) and math.isnan(c)) for a, c in zip(x, y))
                for x, y in zip(r1.rows(), r2.rows()))
        ms, kms, nbytes, nrows = b.stats()
        assert ms >= kms > 0 and nbytes > 0 and nrows > 0
    finally:
        b.close()


def test_batch_group_tables_exact(mixed):
    X, _, ops, hosts = mixed
    b = X.GpuBatch(ops)
    try:
        res = b.exec()
        checked = 0
        for k, op in enumerate(ops):
            if hosts[k] is None or "path=regs" in op.explain():
                continue
            t, pl = hosts[k]
            ref = R.agg(R.RefTable(t), pl, workers=0)
            rows = res[k].rows()
            assert_rows_match(rows, ref.rows(), ordered=True)
            if ref.nrows and any(tp == abi.TYPE_FLOAT64 for tp in ref.types):
                assert_sums_exact(res[k], ref)
            checked += 1
        assert checked >= 6
    finally:
        b.close()


def test_batch_autotune(mixed):
    """Autotuning over cache size, unit size and block shapes; a second batch
    of the same shape takes the stored choice without timing, a retune times
    again; every tuning gives the single runs' results."""
    import ctypes as C
    X, _, ops, _ = mixed
    single = single_rows(ops)
    L = abi.load()
    arr = (C.c_void_p * len(ops))(*[op.h for op in ops])

    def batch(flags):
        h = C.c_void_p()
        abi.check(L.vexq_batch_create(arr, len(ops), flags, C.byref(h)))
        return h

    for flags, want in ((abi.BATCH_RETUNE, "candidates"), (abi.BATCH_AUTOTUNE, "autotuned(cached")):
        h = batch(flags)
        try:
            assert want in L.vexq_batch_explain(h).decode(), L.vexq_batch_explain(h)
            outs = (C.c_void_p * len(ops))()
            abi.check(L.vexq_batch_exec(h, outs))
            check_against_single([X.Result(C.c_void_p(outs[k])) for k in range(len(ops))], single, ops)
        finally:
            L.vexq_batch_destroy(h)


def test_batch_run_and_empty(mixed):
    import ctypes as C
    X, _, ops, _ = mixed
    L = abi.load()
    single = single_rows(ops[:3])
    plans = (C.c_void_p * 3)(*[op.h for op in ops[:3]])
    outs = (C.c_void_p * 3)()
    abi.check(L.vexq_batch_run(plans, 3, outs))
    check_against_single([X.Result(C.c_void_p(outs[k])) for k in range(3)], single, ops[:3])
    abi.check(L.vexq_batch_run(plans, 0, outs))


def test_c3_batch_as_configured(gpu_lib):
    """The batching workload as configured: 256 GROUP BYs, rows log-uniform
    over 10K-4M, 2-65,536 Zipf(1.1) groups, mixed SUM/COUNT/MIN/MAX/AVG, one
    autotuned batch. Every result against the oracle's serial fold: keys,
    counts, MIN and MAX exact; group-table float sums equal to the exact sum
    bit for bit; register-path float cells within 1e-12 of the serial fold
    and 1e-13 of the exact sum."""
    import bench
    from tests.helpers import assert_float_vs_exact
    X = gpu_lib
    hosts, plans = bench.batch_plans(256)
    assert sum(h.nrows for h in hosts) > 100_000_000
    tabs = [X.GpuTable(h) for h in hosts]
    ops = [X.GpuHashAggregate(t, p) for t, p in zip(tabs, plans)]
    try:
        b = X.GpuBatch(ops, autotune=True)
        res = b.exec()
        regs = table = 0
        for k, (h, pl, r) in enumerate(zip(hosts, plans, res)):
            rows = r.rows()
            ref = R.agg(R.RefTable(h), pl, workers=0)
            if "path=regs" in ops[k].explain():
                assert_float_vs_exact(rows, ref, ordered=True)
                regs += 1
            else:
                assert_rows_match(rows, ref.rows(), ordered=True)
                if any(k in (abi.AGG_SUM, abi.AGG_AVG) for k in (a.kind for a in pl.aggs)):
                    assert_sums_exact(r, ref)
                table += 1
            r.close()
        assert regs > 0 and table > 0
        b.close()
    finally:
        for op in ops:
            op.close()
        for t in tabs:
            t.close()
