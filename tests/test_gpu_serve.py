"""GPU tests of the serving loop: admission by HBM footprint and continuous
batching. Every served result must equal the same plan run alone
(vexq_plan_run) within the stated tolerance, in every mix."""
from __future__ import annotations

import ctypes as C
import datetime
import time

import numpy as np
import pytest

from vexq_b200 import abi, datagen as D, workloads as W

from tests.helpers import assert_rows_match

pytestmark = pytest.mark.gpu

SERVE_RTOL = 1e-13  # register-path FP64 sums: another row partition than the single run


def day(n: int) -> str:
    return (datetime.date(1970, 1, 1) + datetime.timedelta(days=int(n))).isoformat()


@pytest.fixture(scope="module")
def tables(gpu_lib):
    X = gpu_lib
    li = X.GpuTable(D.lineitem(600_000, seed=31, rg_rows=65536))
    o, i = X.GpuTable(D.orders(60_000, seed=5)), X.GpuTable(D.items(240_000, 60_000, seed=6))
    return X, li, o, i


def make_queries(X, li, o, i, n, seed):
    """The serving mix: 50% Q1-shape GROUP BY, 20% Q6-shape range SUM, 30%
    Q3-shape join, with randomised date cutoffs."""
    rng = np.random.default_rng(seed)
    ops = []
    for _ in range(n):
        u = rng.random()
        if u < 0.5:
            ops.append(X.GpuHashAggregate(li, W.q1_plan(day(8036 + rng.integers(1500, 2526)))))
        elif u < 0.7:
            lo = 8036 + int(rng.integers(0, 2000))
            ops.append(X.GpuHashAggregate(li, W.q6_plan(day(lo), day(lo + 365))))
        else:
            ops.append(X.GpuParallelHashJoinAggregate(o, i, W.q3_plan(float(rng.uniform(0.3, 0.6)),
                                                                      float(rng.uniform(0.3, 0.6)))))
    return ops


def alone(ops):
    out = []
    for op in ops:
        r = op.run()
        out.append(r.rows())
        r.close()
    return out


def serve(X, ops, budget=1 << 36, max_inflight=8, workers=2, flags=0, gap_s=0.0):
    L = abi.load()
    srv = C.c_void_p()
    abi.check(L.vexq_server_start(budget, max_inflight, workers, flags, C.byref(srv)))
    try:
        tickets = []
        for op in ops:
            tk = C.c_int64()
            abi.check(L.vexq_server_submit(srv, op.h, C.byref(tk)))
            tickets.append(tk.value)
            if gap_s:
                time.sleep(gap_s)
        rows, lat = [], []
        for tk in tickets:
            h = C.c_void_p()
            abi.check(L.vexq_server_wait(srv, tk, 120000, C.byref(h)))
            rows.append(X.Result(h).rows())
            ms = C.c_double()
            abi.check(L.vexq_server_latency(srv, tk, C.byref(ms)))
            lat.append(ms.value)
        la, q, mb, mc = C.c_int64(), C.c_int64(), C.c_int32(), C.c_int32()
        abi.check(L.vexq_server_stats(srv, C.byref(la), C.byref(q), C.byref(mb), C.byref(mc)))
        return rows, lat, (la.value, q.value, mb.value, mc.value)
    finally:
        abi.check(L.vexq_server_stop(srv))


def test_continuous_batching_matches_alone(tables):
    X, li, o, i = tables
    ops = make_queries(X, li, o, i, 24, seed=11)
    try:
        ref = alone(ops)
        rows, lat, (launches, queries, max_batch, _) = serve(X, ops)
        assert queries == len(ops)
        assert max_batch >= 2 and launches < len(ops)  # queries shared launches
        for k, (a, b) in enumerate(zip(rows, ref)):
            assert_rows_match(a, b, ordered=True, rtol=SERVE_RTOL)
        assert all(x > 0 for x in lat)
        # arrivals while earlier launches are on the GPU join later launches
        rows2, _, (launches2, _, _, max_running) = serve(X, ops, gap_s=0.002)
        for a, b in zip(rows2, ref):
            assert_rows_match(a, b, ordered=True, rtol=SERVE_RTOL)
        assert launches2 >= 2 and max_running >= 1
    finally:
        for op in ops:
            op.close()


def test_plain_serving_one_query_per_launch(tables):
    X, li, o, i = tables
    ops = make_queries(X, li, o, i, 8, seed=12)
    try:
        ref = alone(ops)
        rows, _, (launches, queries, max_batch, _) = serve(X, ops, flags=abi.SERVE_NO_BATCH)
        assert launches == queries == len(ops) and max_batch == 1
        for a, b in zip(rows, ref):
            assert_rows_match(a, b, ordered=True, rtol=SERVE_RTOL)
    finally:
        for op in ops:
            op.close()


def test_admission_by_footprint(tables):
    X, li, o, i = tables
    ops = [X.GpuParallelHashJoinAggregate(o, i, W.q3_plan()) for _ in range(3)]
    try:
        ref = alone(ops[:1])[0]
        # footprint of one join query fits, two do not: they run one at a time
        rows, _, (launches, _, max_batch, max_running) = serve(X, ops, budget=1 << 23, workers=2)
        assert max_batch == 1 and max_running == 1 and launches == 3
        for r in rows:
            assert_rows_match(r, ref, ordered=True)
        L = abi.load()
        srv = C.c_void_p()
        abi.check(L.vexq_server_start(1 << 10, 4, 1, 0, C.byref(srv)))
        try:
            tk = C.c_int64()
            assert L.vexq_server_submit(srv, ops[0].h, C.byref(tk)) == abi.EADMIT
        finally:
            abi.check(L.vexq_server_stop(srv))
    finally:
        for op in ops:
            op.close()


def test_two_workers_same_handles_repeated(tables):
    """The same few plan handles submitted many times to two batching
    workers: batches of one worker read a plan while the other worker's
    batch (or join) uses the same handle, and batch workspaces grow between
    launches. Every result must equal the plan's single run."""
    X, li, o, i = tables
    ops = make_queries(X, li, o, i, 7, seed=13)
    try:
        ref = alone(ops)
        rng = np.random.default_rng(14)
        for rep in range(3):
            order = [int(k) for k in rng.integers(0, len(ops), 60)]
            seq = [ops[k] for k in order]
            rows, _, (launches, queries, max_batch, max_running) = serve(
                X, seq, max_inflight=16, workers=2, gap_s=0.0005 * rep)
            assert queries == len(seq)
            for k, r in zip(order, rows):
                assert_rows_match(r, ref[k], ordered=True, rtol=SERVE_RTOL)
    finally:
        for op in ops:
            op.close()
