"""The oracle's Filter and Filter → Project against answers the reference's
own tests assert: stacked filters with literal operands and BETWEEN
(exec/stacked_filter_test.go:76-176: a stacked filter is the AND of the two
predicates over the rows the first kept), unary minus and mixed-type
arithmetic with NULL propagation in projections (exec/expr_eval_test.go:249-
573), and the scan operators of exec/exec_test.go:125-450 and 762-853
(Filter, Project, Filter → Project, zone-map pruning by row group, LIMIT
after a filter, CASE with string results with and without ELSE)."""
from __future__ import annotations

import numpy as np

from oracle import refcpu as R
from vexq_b200 import plan as P
from vexq_b200.table import HostTable, float_column, int_column


def one_col(values):
    return HostTable([int_column("a", np.asarray(values, dtype=np.int64))], len(values), 65536)


def test_stacked_literal_filters():
    t = R.RefTable(one_col([1, 5, 9, 12, 20]))
    pred = P.and_(P.col(0) > 4, P.col(0) < 31)
    assert R.project(t, [P.col(0)], pred).rows() == [(5,), (9,), (12,), (20,)]
    bits, n = R.filter_bits(t, pred)
    assert n == 4 and bits[0] == 0b11110


def test_stacked_literal_filters_wide_batch():
    t = R.RefTable(one_col(list(range(1024))))  # BlockRows values 0..1023
    pred = P.and_(P.col(0) > 0, P.col(0) < (1 << 30))
    rows = R.project(t, [P.col(0)], pred).rows()
    assert rows == [(i,) for i in range(1, 1024)]


def test_stacked_between_filter():
    t = R.RefTable(one_col([1, 5, 9, 12, 20]))
    pred = P.and_(P.col(0) > 4, P.between(P.col(0), P.lit(5), P.lit(20)))
    assert R.project(t, [P.col(0)], pred).rows() == [(5,), (9,), (12,), (20,)]


def expr_table(n):
    # exec/expr_eval_test.go:15-57: id = i, amount = i * 2.5
    return R.RefTable(HostTable([int_column("id", np.arange(n, dtype=np.int64)),
                                 float_column("amount", np.arange(n) * 2.5)], n, 65536))


def test_unary_minus_projection():
    rows = R.project(expr_table(10), [P.col(0), P.neg(P.col(1)), P.neg(P.col(0))]).rows()
    assert len(rows) == 10
    assert rows[1][1] == -2.5 and rows[5][2] == -5  # the values the reference test checks
    assert all(r[1] == -(i * 2.5) and r[2] == -i for i, r in enumerate(rows))


def test_mixed_type_arithmetic_null_propagation():
    x = int_column("x", np.array([10, 20, 30, 40], dtype=np.int64), np.array([1, 0, 1, 1], dtype=bool))
    y = float_column("y", np.array([1.5, 2.5, 3.5, 4.5]), np.array([1, 1, 0, 1], dtype=bool))
    t = R.RefTable(HostTable([x, y], 4, 65536))
    assert R.project(t, [P.col(0) * P.col(1)]).rows() == [(15.0,), (None,), (None,), (180.0,)]


def test_mixed_type_arithmetic_under_selection():
    rows = R.project(expr_table(20), [P.col(1) * P.col(0)], P.col(0) > 15).rows()
    assert rows == [(640.0,), (722.5,), (810.0,), (902.5,)]


def scan_table(n, rg=65536):
    # exec/exec_test.go:20-54 writeTestFile: id = i, val = i * 2.5, 65,536-row row groups
    return R.RefTable(HostTable([int_column("id", np.arange(n, dtype=np.int64)),
                                 float_column("val", np.arange(n) * 2.5)], n, rg))


def test_filter_project_operators():
    # exec/exec_test.go:125-265: Filter id >= 1024 over 2,048 rows; Project id * 2
    # over 512 rows; Filter id < 100 then Project id over two row groups
    bits, n = R.filter_bits(scan_table(2048), P.col(0) >= 1024)
    assert n == 1024
    assert R.project(scan_table(512), [P.col(0) * 2]).rows() == [(2 * i,) for i in range(512)]
    rows = R.project(scan_table(2 * 65536), [P.col(0)], P.col(0) < 100).rows()
    assert len(rows) == 100 and max(r[0] for r in rows) == 99


def test_zone_map_pruning():
    # exec/exec_test.go:267-302: four row groups, only those whose max(id) >=
    # 131,072 are read (row groups 2 and 3, 2 x 65,536 rows)
    t = scan_table(4 * 65536)
    plan = P.AggPlan(P.col(0) >= 131072, [], [P.count_star("n")])
    assert R.zone_prune(t, plan) == [0, 0, 1, 1]
    assert R.agg(t, plan, workers=0).rows() == [(2 * 65536,)]


def test_case_when_string_branches():
    # exec/exec_test.go:762-853: CASE over val with string results, with and without ELSE
    def vals(v):
        return R.RefTable(HostTable([float_column("val", np.asarray(v, dtype=np.float64))], len(v), 65536))
    x = P.col(0)
    three = P.case([(x > 500.0, P.lit("high")), (x > 200.0, P.lit("medium"))], P.lit("low"))
    assert R.project(vals([100, 300, 600, 50]), [three]).rows() == [("low",), ("medium",), ("high",), ("low",)]
    no_else = P.case([(x > 500.0, P.lit("high"))], None)
    assert R.project(vals([100, 300, 600, 800]), [no_else]).rows() == [(None,), (None,), ("high",), ("high",)]


def test_limit_after_filter():
    # exec/exec_test.go:353-415: LIMIT 2 over the rows id >= 5 keeps ids 5 and 6
    # (the first rows the filter passes, not the first physical rows); restated
    # as the first two groups, in first-occurrence order, of a GROUP BY id
    plan = P.AggPlan(P.col(0) >= 5, [0], [P.count_star("n")], limit=2)
    assert R.agg(scan_table(10), plan, workers=0).rows() == [(5, 1), (6, 1)]
    # exec/exec_test.go:417-450: LIMIT 3 with no filter keeps the first three
    assert R.agg(scan_table(100), P.AggPlan(None, [0], [P.count_star("n")], limit=3), workers=0).rows() == \
        [(0, 1), (1, 1), (2, 1)]
