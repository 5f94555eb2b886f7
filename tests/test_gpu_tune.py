"""GPU tests of per-plan tuning (vexq_plan_autotune): the choice is one of
the candidates, results after tuning equal the untuned plan's bit for bit
(group-table sums are exact whatever the table layout), and a second plan of
the same shape takes the stored choice without timing."""
from __future__ import annotations

import pytest

from vexq_b200 import datagen as D, workloads as W

pytestmark = pytest.mark.gpu


def test_join_radix_bits_tuned(gpu_lib):
    X = gpu_lib
    o, i = X.GpuTable(D.orders(200_000, seed=31)), X.GpuTable(D.items(800_000, 200_000, seed=32))
    for make in (lambda: W.q3_plan(limit=-1), W.q12_plan):
        op = X.GpuParallelHashJoinAggregate(o, i, make())
        try:
            want = op.run().rows()
            choice, ms = op.autotune(retune=True)
            assert choice in (0, 6, 8, 10, 12) and ms > 0
            assert f"tuned=radix_bits:{choice}" in op.explain()
            assert op.run().rows() == want
        finally:
            op.close()
        op2 = X.GpuParallelHashJoinAggregate(o, i, make())
        try:
            c2, ms2 = op2.autotune()
            assert c2 == choice and ms2 == 0  # stored choice, no timing
            assert op2.run().rows() == want
        finally:
            op2.close()


def test_dense_cache_tuned(gpu_lib):
    X = gpu_lib
    t = X.GpuTable(D.zipf_groups(1_000_000, 20_000, seed=33))
    op = X.GpuHashAggregate(t, W.batch_plan())
    try:
        want = op.run().rows()
        choice, ms = op.autotune(retune=True)
        assert choice in (0, 48, 96, 160) and ms > 0
        assert op.run().rows() == want
    finally:
        op.close()
    # the register path has nothing to choose
    g = X.GpuHashAggregate(X.GpuTable(D.lineitem(100_000, seed=3)), W.q1_plan())
    try:
        assert g.autotune() == (-1, 0.0)
    finally:
        g.close()
