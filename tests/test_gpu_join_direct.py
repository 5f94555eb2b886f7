"""GPU tests of the direct-mapped join build table: a build key column whose
value range is at most a few times its rows gets one table word per key
value (indexed by key - min), filled with one CAS a build row and read with
one load a probe row. The rows must equal the hash-table build's (VEXQ_TUNE
dmap=0) bit for bit and the oracle's (joinHashTable semantics,
exec/join_table.go:111-569, probe exec/join.go:84-155): probe keys outside
the build range, NULL keys on either side and build predicates that leave
gaps in the range; a build with a repeated key switches to the hash table in
the same run and stays there."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import refcpu as R
from tests.helpers import assert_rows_match, assert_sorted_rows_match
from tests.test_gpu_join import bits_equal
from vexq_b200 import datagen as D, workloads as W
from vexq_b200.plan import JoinPlan, col, count_star, max_, min_, sum_
from vexq_b200.table import HostTable, float_column, int_column

pytestmark = pytest.mark.gpu


def run_rows(X, go, gi, plan, tune=None, monkeypatch=None):
    if tune is not None:
        monkeypatch.setenv("VEXQ_TUNE", tune)
    op = X.GpuParallelHashJoinAggregate(go, gi, plan)
    try:
        rows = [op.run().rows() for _ in range(2)]
        return rows, op.explain()
    finally:
        op.close()
        if tune is not None:
            monkeypatch.delenv("VEXQ_TUNE")


@pytest.fixture(scope="module")
def orders_items(gpu_lib):
    X = gpu_lib
    o, i = D.orders(200_000, seed=31), D.items(800_000, 200_000, seed=32)
    return X, o, i, X.GpuTable(o), X.GpuTable(i)


@pytest.mark.parametrize("shape", ["q3", "q3_all", "q12"])
def test_direct_matches_hash_build_and_oracle(orders_items, shape, monkeypatch):
    X, o, i, go, gi = orders_items
    plan = {"q3": W.q3_plan(), "q3_all": W.q3_plan(limit=-1), "q12": W.q12_plan()}[shape]
    (d1, d2), ex = run_rows(X, go, gi, plan)
    assert "build=direct" in ex, ex
    (h1, h2), exh = run_rows(X, go, gi, plan, "dmap=0", monkeypatch)
    assert "build=hash" in exh, exh
    assert bits_equal(d1, h1) and bits_equal(d1, d2) and bits_equal(h1, h2)
    ref = R.join(R.RefTable(o), R.RefTable(i), plan, workers=0)
    if shape == "q12":
        assert_rows_match(d1, ref.rows(), ordered=True, rtol=0.0)
    else:
        assert_sorted_rows_match(d1, ref.rows(), plan.order_col, plan.descending)


def sparse_tables(n_build=3000, n_probe=40_000, seed=3, dup=False):
    """Build keys 1..n_build (a permutation), about 3% NULL, with a value
    column the plans' build predicate filters on (gaps in the key range);
    probe keys from -50 to n_build + 50 (outside the build range at both
    ends), about 5% NULL. dup: one key on two (non-NULL) build rows."""
    rng = np.random.default_rng(seed)
    bk = rng.permutation(np.arange(1, n_build + 1, dtype=np.int64))
    if dup:
        bk[17] = bk[4]  # one key on two build rows
    bval = rng.integers(0, 100, n_build)
    bnull = rng.random(n_build) > 0.03
    bnull[[4, 17]] = True
    pk = rng.integers(-50, n_build + 51, n_probe)
    pnull = rng.random(n_probe) > 0.05
    pv = np.round(rng.normal(50, 20, n_probe), 2)
    b = HostTable([int_column("k", bk, bnull), int_column("bv", bval)], n_build, 1024)
    p = HostTable([int_column("fk", pk, pnull), float_column("v", pv)], n_probe, 4096)
    return b, p


def sparse_plans():
    # joined schema: build columns 0..1, probe columns 2..3
    keep = col(1) >= 34  # about a third of the build rows (and their keys) filtered out
    return {
        "by_key": JoinPlan(0, 0, keep, None, None, [0], [sum_(col(3), "s"), count_star("n"), max_(col(1), "mb")],
                           order_col=0),
        "by_build_col": JoinPlan(0, 0, keep, col(1) > -1000.0, None, [1],
                                 [sum_(col(3), "s"), count_star("n"), min_(col(2), "mk")], order_col=0),
        "global": JoinPlan(0, 0, None, None, None, [], [sum_(col(3), "s"), count_star("n")]),
    }


@pytest.mark.parametrize("name", ["by_key", "by_build_col", "global"])
def test_direct_ranges_nulls_and_gaps(gpu_lib, name, monkeypatch):
    X = gpu_lib
    b, p = sparse_tables()
    plan = sparse_plans()[name]
    gb, gp = X.GpuTable(b), X.GpuTable(p)
    try:
        (d1, _), ex = run_rows(X, gb, gp, plan)
        assert "build=direct" in ex, ex
        (h1, _), _ = run_rows(X, gb, gp, plan, "dmap=0", monkeypatch)
        assert bits_equal(d1, h1)
        ref = R.join(R.RefTable(b), R.RefTable(p), plan, workers=0)
        assert_rows_match(d1, ref.rows(), ordered=True)
    finally:
        gb.close()
        gp.close()


def test_direct_repeated_key_falls_back(gpu_lib):
    X = gpu_lib
    b, p = sparse_tables(dup=True)
    plan = JoinPlan(0, 0, None, None, None, [0], [sum_(col(3), "s"), count_star("n")], order_col=0)
    gb, gp = X.GpuTable(b), X.GpuTable(p)
    op = X.GpuParallelHashJoinAggregate(gb, gp, plan)
    try:
        first = op.run().rows()
        assert "build=hash" in op.explain()
        second = op.run().rows()
        assert "build=hash" in op.explain()
        ref = R.join(R.RefTable(b), R.RefTable(p), plan, workers=0)
        assert bits_equal(first, second)
        assert_rows_match(first, ref.rows(), ordered=True)
    finally:
        op.close()
        gb.close()
        gp.close()


def test_direct_wide_range_takes_hash(gpu_lib):
    X = gpu_lib
    rng = np.random.default_rng(8)
    bk = np.unique(rng.integers(0, 1 << 40, 6000))[:5000]
    rng.shuffle(bk)
    pk = np.concatenate([bk[rng.integers(0, 5000, 20_000)], rng.integers(0, 1 << 40, 5000)])
    b = HostTable([int_column("k", bk)], 5000, 1024)
    p = HostTable([int_column("fk", pk), float_column("v", np.round(rng.random(25_000) * 100, 2))], 25_000, 4096)
    plan = JoinPlan(0, 0, None, None, None, [0], [sum_(col(2), "s"), count_star("n")], order_col=0)
    gb, gp = X.GpuTable(b), X.GpuTable(p)
    op = X.GpuParallelHashJoinAggregate(gb, gp, plan)
    try:
        rows = op.run().rows()
        assert "build=hash" in op.explain()
        ref = R.join(R.RefTable(b), R.RefTable(p), plan, workers=0)
        assert_rows_match(rows, ref.rows(), ordered=True)
    finally:
        op.close()
        gb.close()
        gp.close()
