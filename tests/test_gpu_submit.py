"""GPU tests of vexq_plan_submit: a register-path run returns once its
launches are queued and its result settles at the first read, as the
reference's ParallelHashAggregate does its work in the first Next
(exec/parallel.go:109-120). Submitted results must equal vexq_plan_run's bit
for bit (the same kernels over the same rows), in every order of reads,
reruns, frees and plan destruction; other plans return finished results."""
from __future__ import annotations

import ctypes as C

import pytest
import torch

from oracle import refcpu as R
from tests.helpers import assert_rows_match, assert_float_vs_exact
from tests.test_gpu_join import bits_equal
from vexq_b200 import abi, datagen as D, workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lineitem(gpu_lib):
    X = gpu_lib
    host = D.lineitem(600_000, seed=61, rg_rows=65536)
    gt = X.GpuTable(host)
    yield X, host, gt
    gt.close()


def plans():
    return [W.q1_plan(), W.q6_plan(), W.q1_plan("1998-09-02"), W.q6_plan("1995-01-01", "1996-01-01")]


def test_submitted_runs_match_run_and_oracle(lineitem):
    X, host, gt = lineitem
    ops = [X.GpuHashAggregate(gt, pl) for pl in plans()]
    stream = torch.cuda.Stream()
    try:
        for op in ops:
            op.set_stream(stream.cuda_stream)
        ref = [op.run().rows() for op in ops]
        for _ in range(3):
            pend = [op.submit() for op in ops]  # all four queued on one stream before any read
            for k in reversed(range(len(ops))):  # read back to front: the last waits for the earlier ones
                r = pend[k]
                assert bits_equal(r.rows(), ref[k]), k
                assert r.kernel_ms > 0 and r.launches >= 1 and r.bytes_scanned > 0
                r.close()
        tbl = R.RefTable(host)
        for k, pl in enumerate(plans()):
            assert_float_vs_exact(ref[k], R.agg(tbl, pl, workers=0), ordered=True)
    finally:
        for op in ops:
            op.close()


def test_rerun_settles_the_pending_result(lineitem):
    """The plan's next run settles the pending result first: both results
    read correctly afterwards, in either order."""
    X, _, gt = lineitem
    op = X.GpuHashAggregate(gt, W.q1_plan())
    try:
        ref = op.run().rows()
        a = op.submit()
        b = op.submit()  # settles a before reusing the plan's staging buffer
        c = op.run()
        assert bits_equal(c.rows(), ref) and bits_equal(b.rows(), ref) and bits_equal(a.rows(), ref)
        for r in (a, b, c):
            r.close()
    finally:
        op.close()


def test_result_outlives_its_plan_and_free_unread(lineitem):
    X, _, gt = lineitem
    op = X.GpuHashAggregate(gt, W.q6_plan())
    ref = op.run().rows()
    r = op.submit()
    op.close()  # destroying the plan settles the run: the result stays readable
    assert bits_equal(r.rows(), ref)
    r.close()
    op = X.GpuHashAggregate(gt, W.q6_plan())
    try:
        for _ in range(3):
            op.submit().close()  # freed unread: the plan stops waiting for it
        assert bits_equal(op.run().rows(), ref)
    finally:
        op.close()


def test_cancelled_submit(lineitem):
    """A cancelled plan fails at submit (before anything is queued) with
    VEXQ_ECANCELED, and its next submitted run is correct."""
    X, _, gt = lineitem
    op = X.GpuHashAggregate(gt, W.q1_plan())
    try:
        ref = op.run().rows()
        abi.check(abi.load().vexq_cancel(op.h))
        with pytest.raises(abi.VexqError) as e:
            op.submit()
        assert e.value.status == abi.ECANCELED
        r = op.submit()
        assert bits_equal(r.rows(), ref)
        r.close()
    finally:
        op.close()


def test_join_submit_returns_finished_result(gpu_lib):
    X = gpu_lib
    o, i = D.orders(50_000, seed=62), D.items(200_000, 50_000, seed=63)
    go, gi = X.GpuTable(o), X.GpuTable(i)
    op = X.GpuParallelHashJoinAggregate(go, gi, W.q12_plan())
    try:
        ref = op.run().rows()
        r = op.submit()
        assert bits_equal(r.rows(), ref)
        assert_rows_match(r.rows(), R.join(R.RefTable(o), R.RefTable(i), W.q12_plan(), workers=0).rows(),
                          ordered=True, rtol=0.0)
        r.close()
    finally:
        op.close()
        go.close()
        gi.close()


def test_direct_launches_match_the_graph(lineitem, monkeypatch):
    """VEXQ_TUNE graph=0: the register path's launches go out directly (the
    path a refused capture falls back to) with the same rows, through run and
    submit, as the replayed graph."""
    X, _, gt = lineitem
    ref = []
    for pl in (W.q1_plan(), W.q6_plan()):
        op = X.GpuHashAggregate(gt, pl)
        try:
            ref.append(op.run().rows())
        finally:
            op.close()
    monkeypatch.setenv("VEXQ_TUNE", "graph=0")
    for k, pl in enumerate((W.q1_plan(), W.q6_plan())):
        op = X.GpuHashAggregate(gt, pl)
        try:
            for _ in range(2):
                assert bits_equal(op.run().rows(), ref[k])
                r = op.submit()
                assert bits_equal(r.rows(), ref[k]) and r.kernel_ms > 0
                r.close()
        finally:
            op.close()
