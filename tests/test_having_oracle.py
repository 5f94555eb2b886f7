"""HAVING in the oracle, pinned on the reference's own cases
(planner/having_test.go): the 17-row grouped fixture — group 1: five rows of
val 10, group 2: two rows of val 100, group 3: ten rows of val 1 — and the
six queries the reference checks on it, with the answers it expects."""
from __future__ import annotations

import numpy as np

from oracle import refcpu as R
from vexq_b200 import plan as P
from vexq_b200.table import HostTable, int_column


def grouped_table() -> HostTable:
    grp = np.array([1] * 5 + [2] * 2 + [3] * 10, dtype=np.int64)
    val = np.array([10] * 5 + [100] * 2 + [1] * 10, dtype=np.int64)
    return HostTable([int_column("grp", grp), int_column("val", val)], 17, 65536)


# (aggregates, HAVING over the output columns, visible columns, expected rows
# as {grp: row}); output columns: 0 grp, then the aggregates in order
CASES = {
    # SELECT grp, COUNT(*) AS cnt ... HAVING COUNT(*) > 3  (TestHavingAggReuse)
    "reuse": ([P.count_star("cnt")], P.col(1) > 3, -1, {1: (1, 5), 3: (3, 10)}),
    # ... HAVING SUM(val) > 50, SUM hidden  (TestHavingAggHidden)
    "hidden": ([P.count_star("cnt"), P.sum_(P.col(1), "_having_agg_1")], P.col(2) > 50, 2, {2: (2, 2)}),
    # SELECT grp ... HAVING COUNT(*) > 4  (TestHavingCountStar)
    "count_star": ([P.count_star("_having_agg_0")], P.col(1) > 4, 1, {1: (1,), 3: (3,)}),
    # SELECT grp ... HAVING COUNT(val) > 4  (TestHavingCountCol)
    "count_col": ([P.count(P.col(1), "_having_agg_0")], P.col(1) > 4, 1, {1: (1,), 3: (3,)}),
    # ... HAVING COUNT(*) > 9999  (TestHavingFiltersAllGroups)
    "all_filtered": ([P.count_star("cnt")], P.col(1) > 9999, -1, {}),
    # ... HAVING cnt > 1 AND COUNT(*) > 4  (TestHavingMixedAliasAndAggregate)
    "mixed": ([P.count_star("cnt")], P.and_(P.col(1) > 1, P.col(1) > 4), -1, {1: (1, 5), 3: (3, 10)}),
}


def test_oracle_having_reproduces_the_reference_cases():
    rt = R.RefTable(grouped_table())
    for name, (aggs, having, visible, want) in CASES.items():
        res = R.agg_having(rt, P.AggPlan(None, [0], aggs), having, visible)
        got = {r[0]: r for r in res.rows()}
        assert got == want, (name, got)
        assert res.ncols == (len(aggs) + 1 if visible < 0 else visible), name


def test_oracle_having_then_order_and_limit():
    rt = R.RefTable(grouped_table())
    res = R.agg_having(rt, P.AggPlan(None, [0], [P.count_star("cnt"), P.sum_(P.col(1), "s")]),
                       P.col(2) >= 10, -1, order=(2, 1, 2))
    assert res.rows() == [(2, 2, 200), (1, 5, 50)]


def test_oracle_string_min_max_is_byte_order():
    """Go compares strings byte by byte (exec/aggregate.go:98-110): "é"
    (0xC3 0xA9) sorts after "z", "B" before "a", and "" first."""
    from vexq_b200.table import string_column
    words = ["z", "é", "", "a", "B", "ab"]
    idx = np.arange(len(words))
    t = HostTable([int_column("g", np.zeros(len(words), np.int64)), string_column("s", idx, words, len(words), 65536)],
                  len(words), 65536)
    res = R.agg(R.RefTable(t), P.AggPlan(None, [0], [P.min_(P.col(1), "mn"), P.max_(P.col(1), "mx")]), workers=0)
    assert res.rows() == [(0, "", "é")]
    assert sorted(w.encode() for w in words)[1] == b"B"
