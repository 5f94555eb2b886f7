"""GPU tests of the register-path accumulator forms: integer-valued sums kept
as exact doubles (COUNT, integer SUM, AVG over an integer column sharing
SUM's accumulator), float sums updated by FMA against the group's 0/1 hit
when no value can be NaN/±inf, and the fallbacks when neither holds (NaN and
±inf in a float column, integer sums that could pass 2^53). Every case is
compared with the oracle; a table re-filled with values outside the ranges a
plan was compiled for is refused."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import refcpu as R
from tests.helpers import assert_float_vs_exact, assert_rows_match
from vexq_b200 import abi, plan as P
from vexq_b200.table import HostTable, date_column, float_column, int_column, string_column

pytestmark = pytest.mark.gpu


def key_table(n, seed, vals=None, ivals=None, valid=None, rg=8192):
    rng = np.random.default_rng(seed)
    keys, flag = rng.integers(0, 3, n), rng.integers(0, 2, n)
    v = vals if vals is not None else np.rint(rng.uniform(0, 1e5, n)) / 100.0
    iv = ivals if ivals is not None else rng.integers(1, 51, n)
    d = (8036 + rng.integers(0, 2500, n)).astype(np.int32)
    cols = [string_column("k", keys, ["A", "N", "R"], n, rg), string_column("f", flag, ["F", "O"], n, rg), float_column("v", v),
            int_column("q", iv.astype(np.int64), valid), date_column("d", d)]
    return HostTable(cols, n, rg)


def aggs():
    return [P.count_star("n"), P.sum_(P.col(3), "sq"), P.avg(P.col(3), "aq"), P.count(P.col(3), "cq"),
            P.sum_(P.col(2), "sv"), P.avg(P.col(2), "av"), P.sum_(P.col(2) * (1 - P.col(2) / 1e6), "se"),
            P.min_(P.col(2), "mn"), P.max_(P.col(3), "mx")]


def run(X, host, plan):
    op = X.GpuHashAggregate(X.GpuTable(host), plan)
    try:
        g = op.run()
        g.collect()
        return g, op.explain()
    finally:
        op.close()


def check(X, host, plan):
    g, ex = run(X, host, plan)
    r = R.agg(R.RefTable(host), plan, workers=0)
    assert_rows_match(g.rows(), r.rows(), ordered=True)
    assert_float_vs_exact(g.rows(), r)
    return g, r, ex


def test_exact_integer_sums_and_fma_float_sums(gpu_lib):
    host = key_table(300_000, 1)
    plan = P.AggPlan(P.col(4) <= P.lit("1998-09-02"), [0, 1], aggs())
    g, r, ex = check(gpu_lib, host, plan)
    # COUNT(*) and SUM(q) exact doubles, AVG(q) shares SUM(q); SUM(v) (which
    # AVG(v) reuses) and the expression sum are FMA sums
    assert "path=regs" in ex and "exact_int_sums=2" in ex and "shared_sums=1" in ex and "fma_sums=2" in ex, ex
    # integer SUM and AVG(int) are exact: equal to the oracle bit for bit
    for i, (a, b) in enumerate(zip(g.rows(), r.rows())):
        assert a[3] == b[3] and a[4] == b[4] and a[5] == b[5], (i, a, b)


def test_nullable_integer_column(gpu_lib):
    n = 120_000
    valid = np.random.default_rng(4).random(n) > 0.2
    host = key_table(n, 2, valid=valid)
    g, r, ex = check(gpu_lib, host, P.AggPlan(None, [0, 1], aggs()))
    assert "exact_int_sums=" in ex
    for a, b in zip(g.rows(), r.rows()):
        assert a[3:6] == b[3:6]


def test_nan_and_inf_take_the_selected_add(gpu_lib):
    n = 100_000
    rng = np.random.default_rng(3)
    v = np.rint(rng.uniform(0, 1e5, n)) / 100.0
    v[rng.choice(n, 5, replace=False)] = np.nan
    v[rng.choice(np.arange(50_000, n), 3, replace=False)] = np.inf
    host = key_table(n, 3, vals=v)
    g, ex = run(gpu_lib, host, P.AggPlan(None, [0, 1], aggs()))
    assert "fma_sums=0" in ex, ex
    r = R.agg(R.RefTable(host), P.AggPlan(None, [0, 1], aggs()), workers=0)
    assert_rows_match(g.rows(), r.rows(), ordered=True)


def test_large_integers_keep_integer_accumulators(gpu_lib):
    n = 40_000
    rng = np.random.default_rng(5)
    iv = rng.integers(-(1 << 50), 1 << 50, n)
    host = key_table(n, 5, ivals=iv)
    plan = P.AggPlan(None, [0], [P.sum_(P.col(3), "s"), P.avg(P.col(3), "a"), P.count_star("n")])
    g, ex = run(gpu_lib, host, plan)
    # |value| × rows passes 2^53: the integer SUM stays an int64 accumulator
    assert "exact_int_sums=1" in ex and "shared_sums=0" in ex, ex
    r = R.agg(R.RefTable(host), plan, workers=0)
    assert [row[:2] for row in g.rows()] == [row[:2] for row in r.rows()]
    assert_rows_match(g.rows(), r.rows(), ordered=True)


def test_refill_outside_compiled_range_is_refused(gpu_lib):
    X = gpu_lib
    host = key_table(50_000, 6)
    gt = X.GpuTable(host)
    plan = P.AggPlan(None, [0, 1], aggs())
    op = X.GpuHashAggregate(gt, plan)
    other = X.GpuHashAggregate(gt, P.AggPlan(None, [], [P.sum_(P.col(2), "s")]))
    try:
        same = op.run_host(host).rows()  # same values: the compiled ranges still hold
        assert same == op.run().rows()
        wide = key_table(50_000, 6, ivals=np.full(50_000, 10**6))
        with pytest.raises(abi.VexqError) as e:
            op.run_host(wide)
        assert e.value.status == abi.EINVAL and "compile the plan again" in str(e.value)
        with pytest.raises(abi.VexqError):
            other.run()  # every plan compiled before the re-fill refuses
        fresh = X.GpuHashAggregate(gt, plan)  # a plan compiled now sees the new values
        try:
            g = fresh.run()
            r = R.agg(R.RefTable(wide), plan, workers=0)
            assert_rows_match(g.rows(), r.rows(), ordered=True)
        finally:
            fresh.close()
    finally:
        op.close()
        other.close()


def test_hash_table_sized_from_the_last_run(gpu_lib):
    """The hash path sizes a rerun's table from the groups the last run
    found. A first run over one row group (100 keys) then a run over the
    whole table (about 100,000 keys): the small table hits its probe limit,
    the rerun takes the row-bounded size, and results match the oracle; a
    third run reuses the right size."""
    X = gpu_lib
    rg, nrg = 65536, 5
    n = rg * nrg
    rng = np.random.default_rng(11)
    keys = rng.integers(0, 1 << 40, 100_000)[rng.integers(0, 100_000, n)]
    keys[:rg] = rng.integers(0, 1 << 40, 100)[rng.integers(0, 100, rg)]
    vals = np.rint(rng.uniform(0, 1e7, n)) / 100.0
    host = HostTable([int_column("k", keys), float_column("v", vals)], n, rg)
    plan = P.AggPlan(None, [0], [P.sum_(P.col(1), "s"), P.count_star("n"), P.max_(P.col(1), "m")])
    op = X.GpuHashAggregate(X.GpuTable(host), plan)
    try:
        assert "path=hash" in op.explain()
        first = op.run(0, 1)
        first.collect()
        sub = HostTable([int_column("k", keys[:rg]), float_column("v", vals[:rg])], rg, rg)
        assert_rows_match(first.rows(), R.agg(R.RefTable(sub), plan, workers=0).rows(), ordered=True)
        ref = R.agg(R.RefTable(host), plan, workers=0)
        for _ in range(2):
            g = op.run()
            g.collect()
            assert_rows_match(g.rows(), ref.rows(), ordered=True)
            assert_float_vs_exact(g.rows(), ref)
    finally:
        op.close()


@pytest.mark.parametrize("order_col,desc,limit", [(1, False, 7), (1, True, 100), (2, True, 10), (3, False, 25), (4, True, 3)])
def test_device_top_k_matches_oracle(gpu_lib, order_col, desc, limit):
    """ORDER BY an aggregate LIMIT k over 60,000 hash-table groups (device
    threshold, selection and gather): COUNT with heavy ties at the cut, float
    SUM, a MIN that is NULL for some groups (NULLs sort first), AVG; rows and
    order equal the oracle's stable sort."""
    X = gpu_lib
    rng = np.random.default_rng(31)
    n = 400_000
    keys = rng.integers(0, 1 << 40, 60_000)[rng.integers(0, 60_000, n)]
    vals = np.rint(rng.uniform(-1e5, 1e5, n)) / 100.0
    valid = rng.random(n) > 0.3
    valid[keys % 97 == 0] = False  # every value of some groups NULL
    host = HostTable([int_column("k", keys), float_column("v", vals, valid)], n, 65536)
    plan = P.AggPlan(None, [0], [P.count_star("n"), P.sum_(P.col(1), "s"), P.min_(P.col(1), "m"), P.avg(P.col(1), "a")],
                     order_col=order_col, descending=desc, limit=limit)
    op = X.GpuHashAggregate(X.GpuTable(host), plan)
    try:
        for _ in range(2):  # the second run sizes the hash table from the first
            g = op.run()
            g.collect()
            r = R.agg(R.RefTable(host), plan, workers=0)
            assert len(g.rows()) == limit
            assert_rows_match(g.rows(), r.rows(), ordered=True)
    finally:
        op.close()


def fused_aggs():
    return [P.count_star("n"), P.sum_(P.col(3), "sq"), P.avg(P.col(3), "aq"), P.count(P.col(3), "cq"),
            P.sum_(P.col(2), "sv"), P.avg(P.col(2), "av"), P.sum_(P.col(2) * (1 - P.col(2) / 1e6), "se"),
            P.min_(P.col(3), "mn"), P.max_(P.col(3), "mx")]


def test_merge_inside_the_scan_resets_between_runs(gpu_lib, monkeypatch):
    """Sums of finite bounded floats, integer sums, integer MIN/MAX and counts:
    the scan merges its own block partials (global accumulators in 8 copies,
    block b adding into copy b % 8; the last block folds the copies, writes
    the row and restores the identities). Repeated runs, runs over
    sub-ranges of row groups and a run that prunes every row group each match
    the oracle, so nothing of one run leaks into the next."""
    X = gpu_lib
    monkeypatch.setenv("VEXQ_TUNE", "rfuse=2")
    n, rg = 400_000, 8192
    valid = np.random.default_rng(8).random(n) > 0.1
    iv = np.random.default_rng(9).integers(-500, 500, n)
    host = key_table(n, 7, ivals=iv, valid=valid, rg=rg)
    plan = P.AggPlan(P.col(4) <= P.lit("1998-09-02"), [0, 1], fused_aggs())
    op = X.GpuHashAggregate(X.GpuTable(host), plan)
    try:
        assert "merge=in_scan" in op.explain(), op.explain()
        ref = R.agg(R.RefTable(host), plan, workers=0)
        first = op.run().rows()
        assert_rows_match(first, ref.rows(), ordered=True)
        assert_float_vs_exact(first, ref)
        for _ in range(3):
            assert op.run().rows() == first  # the same value each run, bit for bit
        nrg = (n + rg - 1) // rg
        rt = R.RefTable(host)
        for a, b in ((0, 1), (3, 17), (nrg - 2, nrg), (5, 5)):
            g = op.run(a, b)
            assert_rows_match(g.rows(), R.agg(rt, plan, workers=0, rg_start=a, rg_end=b).rows(), ordered=True)
        assert op.run().rows() == first
    finally:
        op.close()
    none = P.AggPlan(P.col(4) < P.lit("1990-01-01"), [0, 1], fused_aggs())  # zone maps prune every row group
    g, ex = run(X, host, none)
    assert "merge=in_scan" in ex and g.rows() == R.agg(R.RefTable(host), none, workers=0).rows()


def test_merge_inside_the_scan_agrees_with_the_merge_kernel(gpu_lib, monkeypatch):
    """The same plan compiled with the separate merge kernel: integer entries
    equal bit for bit, float sums within the float tolerance (the in-scan
    merge adds the block partials exactly, the kernel with TwoSum)."""
    X = gpu_lib
    host = key_table(600_000, 10)
    plan = P.AggPlan(None, [0, 1], fused_aggs())
    monkeypatch.setenv("VEXQ_TUNE", "rfuse=2")
    g1, ex1 = run(X, host, plan)
    monkeypatch.setenv("VEXQ_TUNE", "rfuse=0")
    g2, ex2 = run(X, host, plan)
    assert "merge=in_scan" in ex1 and "merge=kernel" in ex2, (ex1, ex2)
    assert_rows_match(g1.rows(), g2.rows(), ordered=True)
    for a, b in zip(g1.rows(), g2.rows()):
        assert [v for v in a if not isinstance(v, float)] == [v for v in b if not isinstance(v, float)]
    r = R.agg(R.RefTable(host), plan, workers=0)
    assert_float_vs_exact(g1.rows(), r)
    assert_float_vs_exact(g2.rows(), r)


def test_float_min_max_keep_the_merge_kernel(gpu_lib):
    X = gpu_lib
    host = key_table(50_000, 11)
    g, ex = run(X, host, P.AggPlan(None, [0], [P.min_(P.col(2), "mn"), P.sum_(P.col(2), "s")]))
    assert "merge=kernel" in ex, ex
    r = R.agg(R.RefTable(host), P.AggPlan(None, [0], [P.min_(P.col(2), "mn"), P.sum_(P.col(2), "s")]), workers=0)
    assert_rows_match(g.rows(), r.rows(), ordered=True)


def test_merge_placement_by_accumulator_count(gpu_lib, monkeypatch):
    """Default placement: a one-group sum and count merges inside the scan
    into one set of accumulators; six groups of eight (84 atomics a block)
    merge inside the scan into 8 copies; a bank of more than 128 atomics a
    block keeps the merge kernel."""
    X = gpu_lib
    monkeypatch.delenv("VEXQ_TUNE", raising=False)
    host = key_table(200_000, 12)
    small = P.AggPlan(P.col(4) <= P.lit("1997-01-01"), [], [P.sum_(P.col(2) * P.col(3), "s"), P.count_star("n")])
    g, ex = run(X, host, small)
    assert "merge=in_scan" in ex, ex
    r = R.agg(R.RefTable(host), small, workers=0)
    assert_rows_match(g.rows(), r.rows(), ordered=True)
    assert_float_vs_exact(g.rows(), r)
    assert "rcopies" not in ex, ex
    six = P.AggPlan(None, [0, 1], fused_aggs())
    g, ex = run(X, host, six)
    assert "merge=in_scan" in ex and "rcopies=8" in ex, ex
    r = R.agg(R.RefTable(host), six, workers=0)
    assert_rows_match(g.rows(), r.rows(), ordered=True)
    assert_float_vs_exact(g.rows(), r)
    # eight float sums over six groups (plus the row count the plan keeps):
    # 6 x 10 accumulators fit the register path, and a block would add
    # 6 x (8 x 3 digits + the count + the first-row key) = 156 atomics
    wide = P.AggPlan(None, [0, 1], [P.sum_(P.col(2) * float(c), f"s{c}") for c in range(2, 10)])
    g, ex = run(X, host, wide)
    assert "path=regs" in ex and "merge=kernel" in ex, ex
    r = R.agg(R.RefTable(host), wide, workers=0)
    assert_rows_match(g.rows(), r.rows(), ordered=True)
    assert_float_vs_exact(g.rows(), r)
