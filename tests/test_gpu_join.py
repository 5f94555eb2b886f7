"""GPU tests of the radix-partitioned join against the global-table join and
the oracle: the same plan with partitioning off (radix_bits 0), automatic,
and forced to few bits (partitions that overflow shared memory make the bits
grow), a build side whose one key repeats beyond a partition's capacity (the
join falls back to the global table), and the reference's join known-answer
cases with partitioning forced."""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import refcpu as R
from tests.golden.fixtures import load_cases, make_plan, make_table, normalize
from tests.helpers import assert_rows_match
from tests.test_gpu_parity import assert_sums_exact
from vexq_b200 import datagen as D, plan as P, workloads as W
from vexq_b200.table import HostTable, date_column, float_column, int_column

pytestmark = pytest.mark.gpu

JOIN_CASES = [c for c in load_cases() if c["kind"] == "join"]


def bits_equal(a, b):
    return len(a) == len(b) and all(
        len(x) == len(y) and all(u == v or (isinstance(u, float) and math.isnan(u) and math.isnan(v)) for u, v in zip(x, y))
        for x, y in zip(a, b))


@pytest.fixture(scope="module")
def tables(gpu_lib):
    X = gpu_lib
    o, i = D.orders(150_000, seed=5), D.items(600_000, 150_000, seed=6)
    return X, o, i, X.GpuTable(o), X.GpuTable(i)


def run(X, go, gi, plan):
    op = X.GpuParallelHashJoinAggregate(go, gi, plan)
    try:
        r = op.run()
        r.collect()
        return r
    finally:
        op.close()


@pytest.mark.parametrize("shape", ["q3_all", "q3_top10", "q12"])
def test_radix_matches_global_and_oracle(tables, shape):
    X, o, i, go, gi = tables
    mk = {"q3_all": lambda b: W.q3_plan(limit=-1, radix_bits=b), "q3_top10": lambda b: W.q3_plan(radix_bits=b),
          "q12": lambda b: W.q12_plan(radix_bits=b)}[shape]
    glob = run(X, go, gi, mk(0))
    ref = R.join(R.RefTable(o), R.RefTable(i), mk(0), workers=0)
    assert_rows_match(glob.rows(), ref.rows(), ordered=True)
    for bits in (-1, 3, 12):
        rad = run(X, go, gi, mk(bits))
        assert bits_equal(rad.rows(), glob.rows()), (shape, bits)
    if shape == "q3_all":
        assert_sums_exact(rad, ref)


def test_skewed_build_key_falls_back(gpu_lib):
    """One build key repeats 6,000 times (more than a partition holds): the
    partitioned build gives up at the largest bit count and the global-table
    join answers, with chains in build-row order."""
    X = gpu_lib
    rng = np.random.default_rng(8)
    nb = 80_000
    keys = np.arange(1, nb + 1, dtype=np.int64)
    keys[rng.choice(nb, 6000, replace=False)] = 7
    bdate = (8036 + rng.integers(0, 2400, nb)).astype(np.int32)
    bt = HostTable([int_column("k", keys), date_column("d", bdate)], nb, 65536)
    npr = 300_000
    fk = rng.integers(1, nb + 1, npr).astype(np.int64)
    fk[rng.random(npr) < 0.01] = 7
    val = np.rint(rng.uniform(0, 1e5, npr)) / 100.0
    pt = HostTable([int_column("fk", fk), float_column("v", val)], npr, 65536)
    plan = P.JoinPlan(0, 0, None, None, None, [1], [P.count_star("n"), P.sum_(P.col(3), "s"), P.min_(P.col(1), "d")])
    g = run(X, X.GpuTable(bt), X.GpuTable(pt), plan)
    ref = R.join(R.RefTable(bt), R.RefTable(pt), plan, workers=0)
    assert_rows_match(g.rows(), ref.rows(), ordered=True)
    assert_sums_exact(g, ref)


@pytest.mark.parametrize("case", JOIN_CASES, ids=[c["name"] for c in JOIN_CASES])
def test_join_known_answers_with_partitioning(gpu_lib, case):
    X = gpu_lib
    b, p = X.GpuTable(make_table(case["tables"]["build"])), X.GpuTable(make_table(case["tables"]["probe"]))
    op = X.GpuParallelHashJoinAggregate(b, p, make_plan(case, radix_bits=2))
    try:
        res = op.run()
        ordered = case["expect"]["ordered"]
        assert normalize(res.rows(), ordered) == normalize(case["expect"]["rows"], ordered)
    finally:
        op.close()


def test_build_table_sized_from_the_last_build(gpu_lib):
    """The build table is sized from the keys the plan's last build inserted.
    The plan first runs with a build filter that keeps 500 rows; the build
    table is then re-filled (through an aggregate plan's host-buffer run,
    values inside the original ranges) so that every row passes: the small
    table hits its probe limit and the build reruns at the row-bounded size."""
    X = gpu_lib
    rng = np.random.default_rng(21)
    nb = 200_000
    keys = rng.permutation(nb).astype(np.int64) + 1
    d = np.full(nb, 9000, np.int32)
    d[:500] = 8000  # only 500 build rows pass date < 8500
    bt = HostTable([int_column("k", keys), date_column("d", d)], nb, 65536)
    npr = 400_000
    fk = rng.integers(1, nb + 1, npr).astype(np.int64)
    val = np.rint(rng.uniform(0, 1e5, npr)) / 100.0
    pt = HostTable([int_column("fk", fk), float_column("v", val)], npr, 65536)
    plan = P.JoinPlan(0, 0, P.col(1) < P.lit("1993-04-10"), None, None, [], [P.count_star("n"), P.sum_(P.col(3), "s")])
    gb, gp = X.GpuTable(bt), X.GpuTable(pt)
    op = X.GpuParallelHashJoinAggregate(gb, gp, plan)
    filler = X.GpuHashAggregate(gb, P.AggPlan(None, [], [P.count_star("n")]))
    try:
        ref = R.join(R.RefTable(bt), R.RefTable(pt), plan, workers=0)
        for _ in range(2):
            assert_rows_match(op.run().rows(), ref.rows(), ordered=True)
        bt2 = HostTable([int_column("k", keys), date_column("d", np.full(nb, 8000, np.int32))], nb, 65536)
        filler.run_host(bt2).close()
        ref2 = R.join(R.RefTable(bt2), R.RefTable(pt), plan, workers=0)
        for _ in range(2):
            g = op.run()
            g.collect()
            assert_rows_match(g.rows(), ref2.rows(), ordered=True)
            assert_sums_exact(g, ref2)
    finally:
        op.close()
        filler.close()
