"""Known-answer fixtures transcribed from the reference's own tests.

Each case restates one test of the vexq repository as a table + plan + the
expected rows the test asserts (file:line given per case). The reference is
Go and no Go toolchain exists here, so the expected values are the literal
answers those tests check, not outputs of a run. Running this module writes
known_answers.json next to it; tests/ load the JSON.

    python tests/golden/known_answers.py
"""
from __future__ import annotations

import json
import os

NULL = None

CASES = []


def case(name, ref, tables, plan, rows, ordered=False, kind="agg", device=True):
    """device: the case is also part of the GPU known-answer test (False:
    checked on the oracle only, until the device run of it is recorded)."""
    CASES.append({"name": name, "ref": ref, "kind": kind, "tables": tables, "plan": plan,
                  "expect": {"ordered": ordered, "rows": rows}, "device": device})


def strcol(name, rg_dicts, codes, valid=None):
    return {"name": name, "type": "STRING", "rg_dicts": rg_dicts, "codes": codes, "valid": valid}


def col(name, type_, values, valid=None):
    return {"name": name, "type": type_, "values": values, "valid": valid}


# exec/agg_intkey_test.go:221-312 TestIntKeyMultiRowGroupDictInstability:
# the same strings carry different codes per row group.
case("intkey_multi_rg_dict_instability", "exec/agg_intkey_test.go:221-312",
     {"t": {"rg_rows": 4, "nrows": 8, "columns": [
         strcol("flag", [["R", "A", "N"], ["A", "N", "R"]], [0, 1, 2, 0, 0, 1, 2, 0]),
         col("value", "INT64", [10, 20, 30, 40, 100, 200, 300, 400])]}},
     {"predicate": None, "group_by": [0], "aggs": [["SUM", ["col", 1], "sum_val"], ["COUNT", None, "cnt"]]},
     [["A", 520, 3], ["N", 230, 2], ["R", 350, 3]])

# exec/aggregate_rows_test.go:219-247 twoSelVecBatches + :249-327
# TestAccumulateSelVecFourPaths. The batches' selection vectors select the
# flag-'A' rows, so the selection is the predicate flag = 'A'. Columns: flag,
# region, price, qty; the second batch's dictionary order is reversed.
SELVEC_TABLE = {"rg_rows": 8, "nrows": 16, "columns": [
    strcol("flag", [["A", "B"], ["B", "A"]], [0, 1, 0, 1, 0, 1, 0, 1, 0, 0, 0, 0, 0, 0, 0, 1]),
    col("region", "INT64", [1, 1, 2, 2, 1, 1, 2, 2, 9, 9, 9, 9, 9, 9, 9, 1]),
    col("price", "FLOAT64", [1.0, 100.0, 2.0, 200.0, 4.0, 400.0, 8.0, 800.0,
                             -1.0, -1.0, -1.0, -1.0, -1.0, -1.0, -1.0, 16.0]),
    col("qty", "INT64", [1] * 16)]}
SEL_A = ["bin", "EQ", ["col", 0], ["lit", "A"]]
case("selvec_no_group_by_direct", "exec/aggregate_rows_test.go:262-272",
     {"t": SELVEC_TABLE},
     {"predicate": SEL_A, "group_by": [],
      "aggs": [["SUM", ["col", 2], "sum_price"], ["COUNT", None, "cnt"], ["MIN", ["col", 2], "min_price"],
               ["MAX", ["col", 2], "max_price"]]},
     [[31.0, 5, 1.0, 16.0]])
case("selvec_int_key_dict_string_group", "exec/aggregate_rows_test.go:273-281",
     {"t": SELVEC_TABLE},
     {"predicate": SEL_A, "group_by": [0], "aggs": [["SUM", ["col", 2], "sum_price"], ["COUNT", None, "cnt"]]},
     [["A", 31.0, 5]])
case("selvec_composite_string_key_group", "exec/aggregate_rows_test.go:282-291",
     {"t": SELVEC_TABLE},
     {"predicate": SEL_A, "group_by": [1, 0], "aggs": [["SUM", ["col", 2], "sum_price"], ["COUNT", None, "cnt"]]},
     [[1, "A", 21.0, 3], [2, "A", 10.0, 2]])

# exec/parallel_test.go:8-43 TestMergePartialAggNonNullCounts: two partials
# each holding sum s and non-null count 2 (4 and 6) merge to AVG 2.5. As
# table rows: one row group per partial.
case("merge_partial_avg_non_null_counts", "exec/parallel_test.go:8-43",
     {"t": {"rg_rows": 2, "nrows": 4, "columns": [col("value", "FLOAT64", [1.0, 3.0, 2.0, 4.0])]}},
     {"predicate": None, "group_by": [], "aggs": [["AVG", ["col", 0], "avg_value"]]},
     [[2.5]])

# exec/exec_test.go:561-598 TestAvgWithNulls: AVG over [1, NULL, 3] = 2.
case("avg_with_nulls", "exec/exec_test.go:561-598",
     {"t": {"rg_rows": 65536, "nrows": 3, "columns": [col("val", "FLOAT64", [1.0, 0.0, 3.0], [1, 0, 1])]}},
     {"predicate": None, "group_by": [], "aggs": [["AVG", ["col", 0], "avg_val"]]},
     [[2.0]])

# exec/exec_test.go:600-629 TestSumAllNull: SUM over all-NULL is NULL.
case("sum_all_null", "exec/exec_test.go:600-629",
     {"t": {"rg_rows": 65536, "nrows": 3, "columns": [col("val", "FLOAT64", [0.0, 0.0, 0.0], [0, 0, 0])]}},
     {"predicate": None, "group_by": [], "aggs": [["SUM", ["col", 0], "sum_val"]]},
     [[NULL]])

# exec/exec_test.go:631-672 TestMinMaxAllNull: MIN/MAX over all-NULL are NULL.
case("min_max_all_null", "exec/exec_test.go:631-672",
     {"t": {"rg_rows": 65536, "nrows": 2, "columns": [col("val", "INT64", [0, 0], [0, 0])]}},
     {"predicate": None, "group_by": [], "aggs": [["MIN", ["col", 0], "min"], ["MAX", ["col", 0], "max"]]},
     [[NULL, NULL]])

# exec/exec_test.go:674-721 TestEmptyTableAggregate: COUNT 0, SUM/AVG NULL, one row.
case("empty_table_aggregate", "exec/exec_test.go:674-721",
     {"t": {"rg_rows": 65536, "nrows": 0, "columns": [col("val", "FLOAT64", [])]}},
     {"predicate": None, "group_by": [],
      "aggs": [["COUNT", None, "cnt"], ["SUM", ["col", 0], "sum_val"], ["AVG", ["col", 0], "avg_val"]]},
     [[0, NULL, NULL]])

# exec/exec_test.go:723-760 TestCountColumnWithNulls: COUNT(col) 3, COUNT(*) 5.
case("count_column_with_nulls", "exec/exec_test.go:723-760",
     {"t": {"rg_rows": 65536, "nrows": 5, "columns": [col("val", "INT64", [1, 0, 3, 0, 5], [1, 0, 1, 0, 1])]}},
     {"predicate": None, "group_by": [], "aggs": [["COUNT", ["col", 0], "cnt_val"], ["COUNT", None, "cnt_star"]]},
     [[3, 5]])

# Join pair tests (exec/join_perbatch_test.go): the emitted (build payload,
# probe payload) pairs in output order are the groups of GROUP BY (bp, pp) in
# insertion order, so they are checked as an ordered aggregate.
JOIN_GB = {"build_key": 0, "probe_key": 0, "build_predicate": None, "probe_predicate": None,
           "residual": None, "group_by": [1, 3], "aggs": [["COUNT", None, "n"]]}


def two_col(kname, pname, keys, payload, valid=None):
    return {"rg_rows": 65536, "nrows": len(keys), "columns": [col(kname, "INT64", keys, valid),
                                                              col(pname, "INT64", payload)]}


case("join_probe_null_keys_dropped", "exec/join_perbatch_test.go:248-271",
     {"build": two_col("bk", "bp", [1, 2], [100, 200]),
      "probe": two_col("pk", "pp", [1, 0, 2], [10, 11, 12], [1, 0, 1])},
     JOIN_GB, [[100, 10, 1], [200, 12, 1]], ordered=True, kind="join")
case("join_build_null_keys_dropped", "exec/join_perbatch_test.go:273-286",
     {"build": two_col("bk", "bp", [1, 0, 2], [100, 999, 200], [1, 0, 1]),
      "probe": two_col("pk", "pp", [0, 1, 2], [10, 11, 12])},
     JOIN_GB, [[100, 11, 1], [200, 12, 1]], ordered=True, kind="join")
case("join_duplicate_key_build_order", "exec/join_perbatch_test.go:288-300",
     {"build": two_col("bk", "bp", [7, 7, 7], [101, 102, 103]),
      "probe": two_col("pk", "pp", [7], [10])},
     JOIN_GB, [[101, 10, 1], [102, 10, 1], [103, 10, 1]], ordered=True, kind="join")

# exec/join_table_test.go:159-187 TestJoinTableSentinelAndExtremeKeys: 0, -1,
# 1 and the int64 extremes are ordinary keys; absent keys miss.
EXTREME = [0, -1, 1, -9223372036854775808, 9223372036854775807]
case("join_sentinel_and_extreme_keys", "exec/join_table_test.go:159-187",
     {"build": two_col("bk", "bp", EXTREME, [0, 1, 2, 3, 4]),
      "probe": two_col("pk", "pp", EXTREME + [2, -2, 999, 9223372036854775806], list(range(9)))},
     JOIN_GB, [[0, 0, 1], [1, 1, 1], [2, 2, 1], [3, 3, 1], [4, 4, 1]], ordered=True, kind="join")


# COUNT(DISTINCT) (exec/aggregate.go:117-124, 474-493, 810-823).
# exec/distinct_test.go:19-41 writeDistinctTestFile + :158-171 TestCountDistinct.
DISTINCT_T = {"rg_rows": 65536, "nrows": 10, "columns": [
    col("id", "INT64", [1, 2, 2, 3, 3, 3, 4, 4, 4, 4]),
    col("val", "INT64", [10, 20, 20, 30, 30, 30, 40, 40, 40, 40])]}
case("count_distinct_id", "exec/distinct_test.go:158-165", {"t": DISTINCT_T},
     {"predicate": None, "group_by": [], "aggs": [["COUNT_DISTINCT", ["col", 0], "d"]]}, [[4]])
case("count_distinct_val", "exec/distinct_test.go:167-171", {"t": DISTINCT_T},
     {"predicate": None, "group_by": [], "aggs": [["COUNT_DISTINCT", ["col", 1], "d"]]}, [[4]])
# exec/distinct_test.go:204-236 writeMultiRowGroupFile + :279-305: the same
# strings under different local codes in two row groups.
MULTI_RG = {"rg_rows": 4, "nrows": 8, "columns": [
    strcol("category", [["alpha", "beta", "gamma"], ["gamma", "beta", "alpha"]], [0, 1, 0, 2, 0, 1, 1, 2]),
    col("amount", "INT64", [10, 20, 30, 40, 50, 60, 70, 80])]}
case("count_distinct_multi_rg_strings", "exec/distinct_test.go:279-286", {"t": MULTI_RG},
     {"predicate": None, "group_by": [], "aggs": [["COUNT_DISTINCT", ["col", 0], "d"]]}, [[3]])
case("count_distinct_multi_rg_ints", "exec/distinct_test.go:288-292", {"t": MULTI_RG},
     {"predicate": None, "group_by": [], "aggs": [["COUNT_DISTINCT", ["col", 1], "d"]]}, [[8]])
# exec/distinct_test.go:238-270 writeNullableFile + :306-335: NULLs stay out
# of the sets.
NULLABLE_T = {"rg_rows": 65536, "nrows": 8, "columns": [
    strcol("grp", [["a", "b"]], [0, 0, 0, 0, 1, 1, 1, 1]),
    col("val", "INT64", [1, 2, 0, 1, 0, 0, 0, 3], [1, 1, 0, 1, 0, 0, 0, 1])]}
case("count_distinct_nulls_excluded", "exec/distinct_test.go:306-314", {"t": NULLABLE_T},
     {"predicate": None, "group_by": [], "aggs": [["COUNT_DISTINCT", ["col", 1], "d"]]}, [[3]])
case("count_distinct_all_null_group", "exec/distinct_test.go:316-335", {"t": NULLABLE_T},
     {"predicate": None, "group_by": [0], "aggs": [["COUNT_DISTINCT", ["col", 1], "d"]]}, [["a", 2], ["b", 1]])
# exec/distinct_test.go:337-372: every value NULL → 0, not NULL.
case("count_distinct_all_null", "exec/distinct_test.go:337-372",
     {"t": {"rg_rows": 65536, "nrows": 4, "columns": [col("id", "INT64", [0, 0, 0, 0], [0, 0, 0, 0])]}},
     {"predicate": None, "group_by": [], "aggs": [["COUNT_DISTINCT", ["col", 0], "d"]]}, [[0]])
# exec/aggregate_rows_test.go:292-299 count_distinct_disables_int_key over the
# SelVec batches above: 5 distinct prices, 1 qty, 1 flag.
case("selvec_count_distinct", "exec/aggregate_rows_test.go:292-299", {"t": SELVEC_TABLE},
     {"predicate": SEL_A, "group_by": [0],
      "aggs": [["COUNT_DISTINCT", ["col", 2], "d_price"], ["COUNT_DISTINCT", ["col", 3], "d_qty"],
               ["COUNT_DISTINCT", ["col", 0], "d_flag"]]},
     [["A", 5, 1, 1]])
# exec/agg_string_fallback_test.go:252-298 TestStringMinMaxWithCountDistinct:
# string MIN/MAX, COUNT(DISTINCT) and COUNT over one string column.
case("string_min_max_with_count_distinct", "exec/agg_string_fallback_test.go:252-298",
     {"t": {"rg_rows": 65536, "nrows": 5, "columns": [
         strcol("grp", [["east", "west"]], [0, 0, 0, 0, 1]),
         strcol("mode", [["MAIL", "AIR", "SHIP"]], [0, 1, 0, 0, 2], [1, 1, 1, 0, 1])]}},
     {"predicate": None, "group_by": [0],
      "aggs": [["MIN", ["col", 1], "lo"], ["MAX", ["col", 1], "hi"], ["COUNT_DISTINCT", ["col", 1], "ndistinct"],
               ["COUNT", ["col", 1], "n"]]},
     [["east", "AIR", "MAIL", 2, 3], ["west", "SHIP", "SHIP", 1, 1]])


# exec/expr_eval_test.go:15-57 writeExprTestFile: one row group of n rows,
# id = i, amount = i * 2.5, status cycling alpha/beta/gamma, order_date =
# 17000 + i (days). The tests count the rows a WHERE keeps or read projected
# values; here the counts are COUNT(*) and the projected values SUM(expr)
# grouped by id (one row a group, so the sum is the row's value).
def expr_table(n):
    return {"rg_rows": 65536, "nrows": n, "columns": [
        col("id", "INT64", list(range(n))),
        col("amount", "FLOAT64", [i * 2.5 for i in range(n)]),
        strcol("status", [["alpha", "beta", "gamma"]], [i % 3 for i in range(n)]),
        col("order_date", "DATE", [17000 + i for i in range(n)])]}


COUNT_ONLY = [["COUNT", None, "n"]]
case("expr_not_string_eq", "exec/expr_eval_test.go:130-148", {"t": expr_table(30)},
     {"predicate": ["not", ["bin", "EQ", ["col", 2], ["lit", "alpha"]]], "group_by": [], "aggs": COUNT_ONLY},
     [[20]], device=False)
case("expr_not_int_gt", "exec/expr_eval_test.go:150-167", {"t": expr_table(30)},
     {"predicate": ["not", ["bin", "GT", ["col", 0], ["lit", 10]]], "group_by": [], "aggs": COUNT_ONLY},
     [[11]], device=False)
case("expr_date_gt_int_literal", "exec/expr_eval_test.go:187-204", {"t": expr_table(30)},
     {"predicate": ["bin", "GT", ["col", 3], ["lit", 17010]], "group_by": [], "aggs": COUNT_ONLY},
     [[19]], device=False)
case("expr_date_between_int_literals", "exec/expr_eval_test.go:206-223", {"t": expr_table(30)},
     {"predicate": ["between", ["col", 3], ["lit", 17005], ["lit", 17015]], "group_by": [], "aggs": COUNT_ONLY},
     [[11]], device=False)
case("expr_unary_minus", "exec/expr_eval_test.go:249-304", {"t": expr_table(10)},
     {"predicate": None, "group_by": [0],
      "aggs": [["SUM", ["neg", ["col", 1]], "neg_amount"], ["SUM", ["neg", ["col", 0]], "neg_id"]]},
     [[i, -(i * 2.5), -i] for i in range(10)], device=False)
A, I = ["col", 1], ["col", 0]
case("expr_mixed_type_arith", "exec/expr_eval_test.go:389-473", {"t": expr_table(5)},
     {"predicate": None, "group_by": [0],
      "aggs": [["SUM", ["bin", "ADD", A, I], "a_plus_i"], ["SUM", ["bin", "ADD", I, A], "i_plus_a"],
               ["SUM", ["bin", "SUB", A, I], "a_minus_i"], ["SUM", ["bin", "SUB", I, A], "i_minus_a"],
               ["SUM", ["bin", "MUL", A, I], "a_times_i"], ["SUM", ["bin", "MUL", I, A], "i_times_a"]]},
     [[0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0], [1, 3.5, 3.5, 1.5, -1.5, 2.5, 2.5], [2, 7.0, 7.0, 3.0, -3.0, 10.0, 10.0],
      [3, 10.5, 10.5, 4.5, -4.5, 22.5, 22.5], [4, 14.0, 14.0, 6.0, -6.0, 40.0, 40.0]], device=False)
case("expr_mixed_type_div", "exec/expr_eval_test.go:441-456", {"t": expr_table(5)},
     {"predicate": ["bin", "GT", I, ["lit", 0]], "group_by": [0],
      "aggs": [["SUM", ["bin", "DIV", A, I], "a_div_i"], ["SUM", ["bin", "DIV", I, A], "i_div_a"]]},
     [[i, 2.5, 0.4] for i in range(1, 5)], device=False)
case("expr_mixed_type_under_selection", "exec/expr_eval_test.go:475-506", {"t": expr_table(20)},
     {"predicate": ["bin", "GT", I, ["lit", 15]], "group_by": [0], "aggs": [["SUM", ["bin", "MUL", A, I], "v"]]},
     [[16, 640.0], [17, 722.5], [18, 810.0], [19, 902.5]], device=False)
case("expr_same_type_arith", "exec/expr_eval_test.go:593-650", {"t": expr_table(5)},
     {"predicate": ["bin", "GT", I, ["lit", 0]], "group_by": [0],
      "aggs": [["SUM", ["bin", "MUL", I, I], "i_sq"], ["SUM", ["bin", "MUL", A, A], "a_sq"],
               ["SUM", ["bin", "DIV", I, I], "i_div_i"]]},
     [[i, i * i, (i * 2.5) ** 2, 1] for i in range(1, 5)], device=False)


# exec/agg_string_minmax_test.go:51-100 strAggBatch: grp and mode are
# dictionary-coded strings (mode's dictionary in the order the test gives,
# which differs from the lexicographic one); ungrouped MIN/MAX/COUNT over mode.
def str_agg_table(modes, mode_dict):
    n = len(modes)
    return {"rg_rows": 65536, "nrows": n, "columns": [
        strcol("grp", [[""]], [0] * n),
        strcol("mode", [mode_dict], [mode_dict.index(m) if m is not None else 0 for m in modes],
               [m is not None for m in modes])]}


MINMAX_COUNT = [["MIN", ["col", 1], "min_mode"], ["MAX", ["col", 1], "max_mode"], ["COUNT", ["col", 1], "cnt"]]
case("string_minmax_ungrouped", "exec/agg_string_minmax_test.go:242-274",
     {"t": str_agg_table(["MAIL", "TRUCK", "AIR", "SHIP"], ["TRUCK", "SHIP", "MAIL", "AIR"])},
     {"predicate": None, "group_by": [], "aggs": MINMAX_COUNT}, [["AIR", "TRUCK", 4]], device=False)
case("string_minmax_ungrouped_with_nulls", "exec/agg_string_minmax_test.go:276-301",
     {"t": str_agg_table([None, "MAIL", None, "AIR", None], ["MAIL", "AIR"])},
     {"predicate": None, "group_by": [], "aggs": MINMAX_COUNT}, [["AIR", "MAIL", 2]], device=False)
case("string_minmax_all_null_ungrouped", "exec/agg_string_minmax_test.go:303-326",
     {"t": str_agg_table([None, None], ["AIR"])},
     {"predicate": None, "group_by": [], "aggs": MINMAX_COUNT}, [[NULL, NULL, 0]], device=False)
case("string_minmax_empty_input", "exec/agg_string_minmax_test.go:328-348",
     {"t": str_agg_table([], ["AIR"])},
     {"predicate": None, "group_by": [],
      "aggs": [["MIN", ["col", 1], "min_mode"], ["MAX", ["col", 1], "max_mode"], ["COUNT", None, "cnt_star"]]},
     [[NULL, NULL, 0]], device=False)
case("string_minmax_empty_string_is_data", "exec/agg_string_minmax_test.go:350-376",
     {"t": str_agg_table(["MAIL", "", "AIR"], ["MAIL", "", "AIR"])},
     {"predicate": None, "group_by": [], "aggs": MINMAX_COUNT[:2]}, [["", "MAIL"]], device=False)
case("string_minmax_only_empty_string", "exec/agg_string_minmax_test.go:378-399",
     {"t": str_agg_table(["", None], [""])},
     {"predicate": None, "group_by": [], "aggs": MINMAX_COUNT[:2]}, [["", ""]], device=False)

# grouped forms (:401-528): by the grp string, by an int64 region, with the
# mode dictionary differing between row groups, and under a selection (the
# selected rows restated as a predicate on an added 0/1 column)
GRP_ROWS = [("east", "MAIL"), ("west", "TRUCK"), ("east", "AIR"), ("west", "SHIP"), ("east", None), ("solo", "RAIL")]
MODE_DICT = ["TRUCK", "SHIP", "RAIL", "MAIL", "AIR"]
case("string_minmax_grouped_by_string", "exec/agg_string_minmax_test.go:401-427",
     {"t": {"rg_rows": 65536, "nrows": 6, "columns": [
         strcol("grp", [["east", "west", "solo"]], [["east", "west", "solo"].index(g) for g, _ in GRP_ROWS]),
         strcol("mode", [MODE_DICT], [MODE_DICT.index(m) if m else 0 for _, m in GRP_ROWS],
                [m is not None for _, m in GRP_ROWS])]}},
     {"predicate": None, "group_by": [0], "aggs": MINMAX_COUNT},
     [["east", "AIR", "MAIL", 2], ["west", "SHIP", "TRUCK", 2], ["solo", "RAIL", "RAIL", 1]], device=False)
REGION_MODES = ["MAIL", "TRUCK", "AIR", "SHIP", None]
case("string_minmax_grouped_by_int", "exec/agg_string_minmax_test.go:429-462",
     {"t": {"rg_rows": 65536, "nrows": 5, "columns": [
         strcol("grp", [[""]], [0] * 5),
         strcol("mode", [["TRUCK", "SHIP", "MAIL", "AIR"]],
                [["TRUCK", "SHIP", "MAIL", "AIR"].index(m) if m else 0 for m in REGION_MODES],
                [m is not None for m in REGION_MODES]),
         col("region", "INT64", [1, 2, 1, 2, 3])]}},
     {"predicate": None, "group_by": [2], "aggs": MINMAX_COUNT[:2]},
     [[1, "AIR", "MAIL"], [2, "SHIP", "TRUCK"], [3, NULL, NULL]], device=False)
case("string_minmax_cross_row_group_dicts", "exec/agg_string_minmax_test.go:464-488",
     {"t": {"rg_rows": 2, "nrows": 4, "columns": [
         strcol("grp", [["east"], ["east"]], [0, 0, 0, 0]),
         strcol("mode", [["MAIL", "SHIP"], ["TRUCK", "AIR"]], [0, 1, 0, 1])]}},
     {"predicate": None, "group_by": [0], "aggs": MINMAX_COUNT[:2]}, [["east", "AIR", "TRUCK"]], device=False)
SEL_T = {"rg_rows": 65536, "nrows": 4, "columns": [
    strcol("grp", [["east"]], [0, 0, 0, 0]),
    strcol("mode", [["ZZZZZ", "SHIP", "MAIL", "AAAAA"]], [2, 3, 1, 0]),
    col("region", "INT64", [1, 1, 1, 1]),
    col("selected", "INT64", [1, 0, 1, 0])]}
for key, name in ((0, "string_key"), (2, "int_key")):
    case(f"string_minmax_under_selection_{name}", "exec/agg_string_minmax_test.go:490-528", {"t": SEL_T},
         {"predicate": ["bin", "EQ", ["col", 3], ["lit", 1]], "group_by": [key], "aggs": MINMAX_COUNT},
         [["east" if key == 0 else 1, "MAIL", "SHIP", 2]], device=False)

case("string_minmax_with_numeric_aggregates", "exec/agg_string_minmax_test.go:530-588",
     {"t": {"rg_rows": 65536, "nrows": 3, "columns": [
         strcol("grp", [["east"]], [0, 0, 0]),
         strcol("mode", [["MAIL", "AIR", "SHIP"]], [0, 1, 2]),
         col("region", "INT64", [0, 0, 0]),
         col("price", "FLOAT64", [10.0, 30.0, 20.0]),
         col("day", "DATE", [100, 300, 200]),
         col("flagb", "BOOL", [False, True, True])]}},
     {"predicate": None, "group_by": [0],
      "aggs": [["MIN", ["col", 1], "min_mode"], ["MAX", ["col", 1], "max_mode"], ["MIN", ["col", 3], "min_price"],
               ["MAX", ["col", 3], "max_price"], ["SUM", ["col", 3], "sum_price"], ["AVG", ["col", 3], "avg_price"],
               ["MIN", ["col", 4], "min_day"], ["MAX", ["col", 4], "max_day"], ["MIN", ["col", 5], "min_flag"],
               ["MAX", ["col", 5], "max_flag"], ["COUNT", None, "cnt_star"]]},
     [["east", "AIR", "SHIP", 10.0, 30.0, 60.0, 20.0, 100, 300, 0, 1, 3]], device=False)


# exec/agg_string_merge_test.go:63-165 mergePartialAgg over string MIN/MAX
# partials: each partial is one row group here (the oracle's parallel runs
# merge one partial a row group; the serial run folds the same rows), with
# its own dictionary.
def rg_modes(groups):
    """groups: the mode values of each row group (None = NULL), equal sizes."""
    rows = [m for g in groups for m in g]
    dicts = [sorted({m for m in g if m is not None}, key=g.index) or ["MAIL"] for g in groups]
    codes = [d.index(m) if m is not None else 0 for g, d in zip(groups, dicts) for m in g]
    return {"rg_rows": len(groups[0]), "nrows": len(rows), "columns": [
        strcol("grp", [[""] for _ in groups], [0] * len(rows)),
        strcol("mode", dicts, codes, [m is not None for m in rows])]}


UNGROUPED = {"predicate": None, "group_by": [], "aggs": MINMAX_COUNT}
case("string_merge_min_max", "exec/agg_string_merge_test.go:63-81",
     {"t": rg_modes([["MAIL", "SHIP"], ["TRUCK", "AIR"]])}, UNGROUPED, [["AIR", "TRUCK", 4]], device=False)
case("string_merge_all_null_partial_last", "exec/agg_string_merge_test.go:83-115",
     {"t": rg_modes([["MAIL", "SHIP"], [None, None]])}, UNGROUPED, [["MAIL", "SHIP", 2]], device=False)
case("string_merge_all_null_partial_first", "exec/agg_string_merge_test.go:83-115",
     {"t": rg_modes([[None, None], ["MAIL", "SHIP"]])}, UNGROUPED, [["MAIL", "SHIP", 2]], device=False)
case("string_merge_empty_string_partial", "exec/agg_string_merge_test.go:117-135",
     {"t": rg_modes([["MAIL"], [""]])}, {"predicate": None, "group_by": [], "aggs": MINMAX_COUNT[:2]},
     [["", "MAIL"]], device=False)
for order, vals in (("forward", ["MAIL", "RAIL", "TRUCK", "AIR", "FOB", "SHIP"]),
                    ("reversed", ["SHIP", "FOB", "AIR", "TRUCK", "RAIL", "MAIL"])):
    case(f"string_merge_order_invariant_{order}", "exec/agg_string_merge_test.go:137-165",
         {"t": rg_modes([[v] for v in vals])}, UNGROUPED, [["AIR", "TRUCK", 6]], device=False)


# exec/agg_string_fallback_test.go:28-123 TestStringMinMaxIntKeyNullGroupByRow:
# a nullable string GROUP BY key (rows 2 and 5 NULL form the NULL group), mode
# dictionary in reverse lexicographic order
FB_MODES = ["MAIL", "TRUCK", "ZULU", "AIR", "SHIP", "ALPHA"]
FB_DICT = ["ZULU", "TRUCK", "SHIP", "MAIL", "ALPHA", "AIR"]
case("string_minmax_null_group_key", "exec/agg_string_fallback_test.go:28-123",
     {"t": {"rg_rows": 65536, "nrows": 6, "columns": [
         strcol("grp", [["east", "west"]], [0, 1, 0, 0, 1, 0], [True, True, False, True, True, False]),
         strcol("mode", [FB_DICT], [FB_DICT.index(m) for m in FB_MODES])]}},
     {"predicate": None, "group_by": [0],
      "aggs": [["MIN", ["col", 1], "lo"], ["MAX", ["col", 1], "hi"], ["COUNT", None, "cnt"]]},
     [["east", "AIR", "MAIL", 2], ["west", "SHIP", "TRUCK", 2], [NULL, "ALPHA", "ZULU", 2]], device=False)


if __name__ == "__main__":
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "known_answers.json")
    with open(out, "w") as f:
        json.dump({"generator": "tests/golden/known_answers.py", "cases": CASES}, f, indent=1)
    print(out, len(CASES))
