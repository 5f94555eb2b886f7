"""GPU parity: the CUDA library (through its C ABI) against the CPU oracle on
the same seeded inputs. Keys, COUNTs, integer sums and join row sets are
bit-exact; float64 SUM/AVG within 1e-12 relative of the oracle's serial
(row-order) result, and float sums are also checked against the exact sum."""
import math

import numpy as np
import pytest

from oracle import refcpu as R
from tests.golden.fixtures import load_cases, make_plan, make_table, normalize
from tests.helpers import assert_float_vs_exact, assert_rows_match, assert_sorted_rows_match, close
from vexq_b200 import abi, datagen as D, workloads as W
from vexq_b200 import plan as P
from vexq_b200.table import HostTable, date_column, float_column, int_column, string_column

pytestmark = pytest.mark.gpu

CASES = [c for c in load_cases() if c.get("device", True)]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_gpu_matches_reference_known_answer(gpu_lib, case):
    X = gpu_lib
    plan = make_plan(case)
    if case["kind"] == "join":
        b, p = X.GpuTable(make_table(case["tables"]["build"])), X.GpuTable(make_table(case["tables"]["probe"]))
        op = X.GpuParallelHashJoinAggregate(b, p, plan)
    else:
        op = X.GpuHashAggregate(X.GpuTable(make_table(case["tables"]["t"])), plan)
    res = op.run()
    ordered = case["expect"]["ordered"]
    assert normalize(res.rows(), ordered) == normalize(case["expect"]["rows"], ordered)


def run_both(X, host, plan, oracle_workers=0):
    gt = X.GpuTable(host)
    op = X.GpuHashAggregate(gt, plan)
    g = op.run()
    g.collect()
    rt = R.RefTable(host)
    r = R.agg(rt, plan, workers=oracle_workers)
    return g, r


def assert_sums_exact(g, r):
    """Dense and hash group tables accumulate float sums as fixed-point
    integers, so every float SUM/AVG cell equals the correctly rounded exact
    sum (the oracle's Shewchuk sum) bit for bit when the inputs' bits all lie
    inside the accumulation window, as they do for these 2-decimal values."""
    checked = 0
    for c, t in enumerate(r.types):
        if t != abi.TYPE_FLOAT64:
            continue
        for i in range(r.nrows):
            ex = r.exact[c][i]
            if math.isnan(ex) or g.columns[c][i] is None:
                continue
            assert g.columns[c][i] == ex, f"row {i} col {c}: gpu={g.columns[c][i]!r} exact={ex!r}"
            checked += 1
    assert checked > 0


@pytest.fixture(scope="module")
def lineitem_1m():
    return D.lineitem(1_000_000, seed=42)


@pytest.fixture(scope="module")
def lineitem_6m():
    return D.lineitem(6_000_000, seed=43, rg_rows=122880)


def test_q1_group_by_1m(gpu_lib, lineitem_1m):
    g, r = run_both(gpu_lib, lineitem_1m, W.q1_plan())
    assert g.nrows == 6
    eg, er = assert_float_vs_exact(g.rows(), r)
    print(f"q1 1M: worst GPU error vs exact {eg:.3g}, reference {er:.3g}")


def test_q1_group_by_6m(gpu_lib, lineitem_6m):
    g, r = run_both(gpu_lib, lineitem_6m, W.q1_plan())
    eg, er = assert_float_vs_exact(g.rows(), r)
    print(f"q1 6M: worst GPU error vs exact {eg:.3g}, reference {er:.3g}")


def test_q6_range_sum_6m(gpu_lib, lineitem_6m):
    g, r = run_both(gpu_lib, lineitem_6m, W.q6_plan())
    assert g.nrows == 1
    eg, er = assert_float_vs_exact(g.rows(), r)
    print(f"q6 6M: GPU error vs exact {eg:.3g}, reference {er:.3g}")


def test_q1_parallel_oracle_agrees(gpu_lib, lineitem_1m):
    g, r = run_both(gpu_lib, lineitem_1m, W.q1_plan(), oracle_workers=4)
    assert_rows_match(g.rows(), r.rows(), ordered=False, rtol=1e-9)


@pytest.fixture(scope="module")
def join_small():
    return D.orders(150_000, seed=5), D.items(600_000, 150_000, seed=6)


@pytest.fixture(scope="module")
def join_full():
    return D.orders(1_500_000, seed=7), D.items(6_000_000, 1_500_000, seed=11)


def run_join(X, o, i, plan, workers=0):
    op = X.GpuParallelHashJoinAggregate(X.GpuTable(o), X.GpuTable(i), plan)
    g = op.run()
    r = R.join(R.RefTable(o), R.RefTable(i), plan, workers=workers)
    return g, r


def test_q3_join_top10_small(gpu_lib, join_small):
    o, i = join_small
    g, r = run_join(gpu_lib, o, i, W.q3_plan())
    assert g.nrows == 10
    assert_rows_match(g.rows(), r.rows(), ordered=True)


def test_q3_join_all_groups_small(gpu_lib, join_small):
    o, i = join_small
    plan = W.q3_plan(limit=-1)
    g, r = run_join(gpu_lib, o, i, plan)
    assert g.nrows > 10000
    assert_sorted_rows_match(g.rows(), r.rows(), plan.order_col, plan.descending)
    assert_sums_exact(g, r)


def test_q3_join_top10_full(gpu_lib, join_full):
    """The join workload at full size (1.5M build x 6M probe rows) against the
    oracle's serial fold: keys exact, revenue within 1e-12, and every revenue
    equal to the exact sum bit for bit (the group table sums in fixed point)."""
    o, i = join_full
    g, r = run_join(gpu_lib, o, i, W.q3_plan(), workers=0)
    assert g.nrows == 10
    assert_rows_match(g.rows(), r.rows(), ordered=True)
    assert_sums_exact(g, r)


def test_q12_join_full(gpu_lib, join_full):
    """The Q12-shape join at full size against the serial oracle: the CASE
    counts are integer sums, compared bit for bit."""
    o, i = join_full
    g, r = run_join(gpu_lib, o, i, W.q12_plan(), workers=0)
    assert g.nrows == 2
    assert_rows_match(g.rows(), r.rows(), ordered=True, rtol=0.0)


def test_q12_join_case_counts(gpu_lib, join_small):
    o, i = join_small
    g, r = run_join(gpu_lib, o, i, W.q12_plan())
    assert g.nrows == 2
    assert_rows_match(g.rows(), r.rows(), ordered=True)


@pytest.mark.parametrize("card", [2, 97, 4096, 65536])
def test_zipf_group_by(gpu_lib, card):
    t = D.zipf_groups(300_000, card, seed=card)
    g, r = run_both(gpu_lib, t, W.batch_plan())
    assert_rows_match(g.rows(), r.rows(), ordered=True)
    if card > 16:  # group-table paths (the register path folds in FP64)
        assert_sums_exact(g, r)


def nullable_table(n=20_000, seed=9, rg_rows=4096):
    rng = np.random.default_rng(seed)
    a = rng.integers(-50, 50, n)
    b = np.round(rng.normal(0, 100, n), 3)
    d = (10000 + rng.integers(0, 400, n)).astype(np.int32)
    s = rng.integers(0, 5, n)
    va, vb, vd, vs = (rng.random(n) > p for p in (0.1, 0.15, 0.05, 0.2))
    cols = [int_column("a", a, va), float_column("b", b, vb), date_column("d", d, vd),
            string_column("s", s, ["x", "y", "zz", "w", ""], n, rg_rows, vs)]
    return HostTable(cols, n, rg_rows)


EXPRS = [
    (P.col(0) > 3, [0]),
    (P.and_(P.col(1) >= -20.5, P.col(0) <= 10), [3]),
    (P.or_(P.col(3) == "zz", P.col(0) < -30), [3]),
    (P.not_(P.col(3) == "x"), [0]),
    (P.col(3) != "w", [2]),
    (P.in_(P.col(3), ["x", "", "nope"]), [3, 0]),
    (P.like(P.col(3), "%z"), []),
    (P.between(P.col(2), "1997-06-01", "1997-09-30"), [3]),
    (P.is_null(P.col(1)), [3]),
    (P.and_(P.is_not_null(P.col(0)), P.col(1) / P.col(0) > 1.0), []),
    (P.in_(P.col(0), [1, 2, 3, -7]), [3]),
]


@pytest.mark.parametrize("k", range(len(EXPRS)))
def test_expression_semantics_with_nulls(gpu_lib, k):
    pred, gb = EXPRS[k]
    t = nullable_table()
    aggs = [P.count_star("n"), P.count(P.col(1), "nb"), P.sum_(P.col(0), "sa"), P.sum_(P.col(1) * 2 - 1, "sb"),
            P.avg(P.col(0), "aa"), P.min_(P.col(1), "mnb"), P.max_(P.col(2), "mxd"), P.min_(P.col(0), "mna"),
            P.sum_(P.case([(P.col(0) > 0, P.col(1))], 0.5), "sc")]
    g, r = run_both(gpu_lib, t, P.AggPlan(pred, gb, aggs))
    assert_rows_match(g.rows(), r.rows(), ordered=True)


def test_zone_pruning_matches_oracle(gpu_lib):
    n = 300_000
    rng = np.random.default_rng(1)
    d = np.sort(8000 + rng.integers(0, 3000, n)).astype(np.int32)  # clustered: zone maps prune
    t = HostTable([date_column("d", d), float_column("v", rng.random(n))], n, 16384)
    plan = P.AggPlan(P.and_(P.col(0) >= "1994-01-01", P.col(0) < "1994-07-01"), [], [P.sum_(P.col(1), "s"),
                                                                                     P.count_star("n")])
    X = gpu_lib
    op = X.GpuHashAggregate(X.GpuTable(t), plan)
    mask = op.zone_prune()
    rt = R.RefTable(t)
    assert mask == R.zone_prune(rt, plan)
    assert 0 < sum(mask) < len(mask)
    assert_rows_match(op.run().rows(), R.agg(rt, plan).rows())


@pytest.mark.parametrize("n,rg", [(0, 65536), (1, 65536), (127, 5), (1029, 100), (70000, 65536)])
def test_ragged_sizes(gpu_lib, n, rg):
    rng = np.random.default_rng(n)
    t = HostTable([int_column("k", rng.integers(0, 3, n)), float_column("v", rng.random(n))], n, rg)
    for plan in (P.AggPlan(None, [], [P.count_star("n"), P.sum_(P.col(1), "s")]),
                 P.AggPlan(P.col(1) > 0.5, [0], [P.count_star("n"), P.avg(P.col(1), "a")]),
                 P.AggPlan(P.col(1) > 2.0, [], [P.count_star("n"), P.max_(P.col(1), "m")])):
        g, r = run_both(gpu_lib, t, plan)
        assert_rows_match(g.rows(), r.rows(), ordered=True)


def test_filter_selection_matches_reference_avx2_kernel(gpu_lib):
    """vexq_filter_run against bench/simd_filter's filter_gt_i64 (the
    reference's own C++ kernel, built from its sources into oracle/_ref)."""
    ref = R.ref_filter_lib()
    if ref is None:
        pytest.skip("reference filter kernel not built (sources absent) or no AVX2")
    import ctypes as C
    # xorshift64* data of bench/simd_filter/cpp/main.cpp:27-40 (first 200,000 rows)
    n = 200_000
    vals = np.empty(n, dtype=np.int64)
    s, M = 42, (1 << 64) - 1
    for i in range(n):
        s ^= s >> 12
        s ^= (s << 25) & M
        s ^= s >> 27
        vals[i] = ((s * 0x2545F4914F6CDD1D) & M) % 50 + 1
    out = np.zeros(n, dtype=np.uint32)
    cnt = ref._Z18filter_gt_i64_avx2PKlmlPj(vals.ctypes.data, n, 25, out.ctypes.data)
    X = gpu_lib
    t = HostTable([int_column("x", vals)], n)
    f = X.GpuFilter(X.GpuTable(t), P.col(0) > 25)
    bits, gcnt = f.bitmap()
    sel = np.flatnonzero(np.unpackbits(np.frombuffer(bits, np.uint8), bitorder="little", count=n))
    assert gcnt == cnt
    assert np.array_equal(sel.astype(np.uint32), out[:cnt])


def test_filter_matches_oracle_with_nulls(gpu_lib):
    t = nullable_table(50_000, seed=4)
    X = gpu_lib
    gt = X.GpuTable(t)
    rt = R.RefTable(t)
    for pred, _ in EXPRS:
        f = X.GpuFilter(gt, pred)
        bits, cnt = f.bitmap()
        rbits, rcnt = R.filter_bits(rt, pred)
        assert cnt == rcnt
        assert bits == rbits
        # the per-block SelVec a downstream operator reads
        assert X.GpuFilter.selvec(bits, t.nrows, 3) == [i - 3072 for i in range(3072, 4096)
                                                         if (rbits[i >> 3] >> (i & 7)) & 1]


def test_run_host_end_to_end_equals_resident(gpu_lib, lineitem_1m):
    X = gpu_lib
    op = X.GpuHashAggregate(X.GpuTable(lineitem_1m), W.q1_plan())
    a = op.run().rows()
    b = op.run_host(lineitem_1m).rows()
    assert a == b


def test_batch_and_server_equal_single_runs(gpu_lib, lineitem_1m):
    import ctypes as C
    X = gpu_lib
    L = abi.load()
    gt = X.GpuTable(lineitem_1m)
    ops = [X.GpuHashAggregate(gt, W.q1_plan()), X.GpuHashAggregate(gt, W.q6_plan())]
    single = [op.run().rows() for op in ops]
    plans = (C.c_void_p * 2)(ops[0].h, ops[1].h)
    outs = (C.c_void_p * 2)()
    abi.check(L.vexq_batch_run(plans, 2, outs))
    for k in range(2):  # register-path FP64 sums: another row partition, last-bit differences
        assert_rows_match(X.Result(C.c_void_p(outs[k])).rows(), single[k], ordered=True, rtol=1e-13)
    srv = C.c_void_p()
    abi.check(L.vexq_server_start(1 << 34, 3, 2, 0, C.byref(srv)))
    tickets = []
    for k in range(8):
        tk = C.c_int64()
        abi.check(L.vexq_server_submit(srv, ops[k % 2].h, C.byref(tk)))
        tickets.append(tk.value)
    for k, tk in enumerate(tickets):
        h = C.c_void_p()
        abi.check(L.vexq_server_wait(srv, tk, 60000, C.byref(h)))
        assert_rows_match(X.Result(h).rows(), single[k % 2], ordered=True, rtol=1e-13)
    abi.check(L.vexq_server_stop(srv))


@pytest.mark.parametrize("lo,hi", [(0, -1), (5, -1), (1237, 40001), (8, 16), (3, 4), (777, 777), (49_999, 50_000)])
def test_filter_row_subranges(gpu_lib, lo, hi):
    """Bitmaps of row sub-ranges at every bit offset: bit i of the output is
    row lo + i, and bits past the range stay clear."""
    t = nullable_table(50_000, seed=6)
    X = gpu_lib
    pred = EXPRS[0][0]
    rbits, _ = R.filter_bits(R.RefTable(t), pred)
    allrows = np.unpackbits(np.frombuffer(rbits, np.uint8), bitorder="little", count=t.nrows)
    end = t.nrows if hi < 0 else hi
    bits, cnt = X.GpuFilter(X.GpuTable(t), pred).bitmap(lo, hi)
    n = end - lo
    got = np.unpackbits(np.frombuffer(bits, np.uint8), bitorder="little")
    assert np.array_equal(got[:n], allrows[lo:end])
    assert not got[n:].any()
    assert cnt == int(allrows[lo:end].sum())


@pytest.mark.parametrize("shape", ["nullable", "lineitem", "allnull_rg"])
def test_zone_maps_match_oracle(gpu_lib, shape):
    """Zone maps computed on the device (row groups split into slices, the
    slices combined in order) against the oracle's: null counts, has-min-max,
    min and max bits and integer sums exact; float sums within 1e-12 relative
    (a different summation order), NaN/±inf alike."""
    import struct
    if shape == "nullable":
        t = nullable_table(70_000, seed=12, rg_rows=16384)
    elif shape == "lineitem":
        t = D.lineitem(300_000, seed=3, rg_rows=65536)
    else:  # one row group entirely NULL, one float column with NaN and inf
        n = 3 * 8192
        rng = np.random.default_rng(2)
        v = rng.normal(0, 10, n)
        v[100] = np.nan
        v[9000] = np.inf
        valid = np.ones(n, bool)
        valid[8192:16384] = False
        t = HostTable([int_column("a", rng.integers(-9, 9, n), valid), float_column("v", v, valid)], n, 8192)
    X = gpu_lib
    g, r = X.GpuTable(t), R.RefTable(t)
    nrg = (t.nrows + t.rg_rows - 1) // t.rg_rows
    for c, col in enumerate(t.columns):
        for rg in range(nrg):
            a, b = g.zone_map(c, rg), r.zone_map(c, rg)
            assert (a.null_count, a.has_min_max) == (b.null_count, b.has_min_max), (c, rg)
            if not b.has_min_max:
                continue
            assert (a.min, a.max) == (b.min, b.max), (c, rg)
            if col.type == abi.TYPE_FLOAT64:
                fa, fb = (struct.unpack("<d", struct.pack("<q", z.sum))[0] for z in (a, b))
                assert close(fa, fb, 1e-12), (c, rg, fa, fb)
            elif col.type == abi.TYPE_INT64:
                assert a.sum == b.sum, (c, rg)
