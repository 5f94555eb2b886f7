"""Plan descriptors of the benchmark workloads, over the datagen tables.

  q1_plan   filtered GROUP BY flag,status with 8 aggregates (TPC-H Q1 shape)
  q6_plan   five-range-predicate scan, SUM(price*disc)        (Q6 shape)
  q3_plan   orders ⋈ items, GROUP BY orderkey, SUM(price*(1-disc)), top 10 (Q3 shape)
  q12_plan  the same join filtered on a mode IN list and a date range, CASE
            priority-bucket counts grouped by mode              (Q12 shape)
  batch_plan  one GROUP BY over a zipf_groups table (SUM/COUNT/MIN/MAX/AVG)
"""
from __future__ import annotations

from . import datagen as D
from .plan import (AggPlan, JoinPlan, and_, avg, between, case, col, count_star, in_, lit, max_, min_,
                   or_, sum_)

Q1_CUTOFF = "1998-09-02"          # date '1998-12-01' - interval '90' day
Q6_LO, Q6_HI = "1994-01-01", "1995-01-01"


def q1_plan(cutoff: str = Q1_CUTOFF) -> AggPlan:
    price, disc, tax = col(D.L_PRICE), col(D.L_DISC), col(D.L_TAX)
    disc_price = price * (1 - disc)
    return AggPlan(
        predicate=col(D.L_SHIPDATE) <= lit(cutoff),
        group_by=[D.L_FLAG, D.L_STATUS],
        aggs=[sum_(col(D.L_QTY), "sum_qty"), sum_(price, "sum_base_price"),
              sum_(disc_price, "sum_disc_price"), sum_(disc_price * (1 + tax), "sum_charge"),
              avg(col(D.L_QTY), "avg_qty"), avg(price, "avg_price"), avg(disc, "avg_disc"),
              count_star("count_order")])


def q6_plan(lo: str = Q6_LO, hi: str = Q6_HI) -> AggPlan:
    return AggPlan(
        predicate=and_(col(D.L_SHIPDATE) >= lit(lo), col(D.L_SHIPDATE) < lit(hi),
                       between(col(D.L_DISC), 0.05, 0.07), col(D.L_QTY) < 24),
        group_by=[],
        aggs=[sum_(col(D.L_PRICE) * col(D.L_DISC), "revenue")])


# joined schema: orders columns (0..2) then items columns (3..7)
NB = 3


def q3_plan(build_frac: float = 0.48, probe_frac: float = 0.46, limit: int = 10, radix_bits: int = -1) -> JoinPlan:
    """orders (date < mid, ~48%) ⋈ items (shipdate > mid, ~54%) GROUP BY key,
    SUM(price*(1-disc)) ORDER BY revenue DESC LIMIT 10."""
    bmid, pmid = D.join_mid(build_frac), D.join_mid(probe_frac)
    price, disc = col(NB + D.I_PRICE), col(NB + D.I_DISC)
    return JoinPlan(
        build_key=D.O_KEY, probe_key=D.I_FK,
        build_predicate=col(D.O_DATE) < lit(bmid),
        probe_predicate=col(D.I_SHIPDATE) > lit(pmid),
        residual=None,
        group_by=[D.O_KEY],
        aggs=[sum_(price * (1 - disc), "revenue")],
        order_col=1, descending=True, limit=limit, radix_bits=radix_bits)


def q12_plan(radix_bits: int = -1) -> JoinPlan:
    prio = col(D.O_PRIORITY)
    high = or_(prio == lit("1-URGENT"), prio == lit("2-HIGH"))
    low = and_(prio != lit("1-URGENT"), prio != lit("2-HIGH"))
    lo, hi = D.join_mid(0.30), D.join_mid(0.30 + 365.0 / D.DATE_SPAN)
    return JoinPlan(
        build_key=D.O_KEY, probe_key=D.I_FK,
        build_predicate=None,
        probe_predicate=and_(in_(col(D.I_MODE), ["MAIL", "SHIP"]),
                             col(D.I_SHIPDATE) >= lit(lo), col(D.I_SHIPDATE) < lit(hi)),
        residual=None,
        group_by=[NB + D.I_MODE],
        aggs=[sum_(case([(high, 1)], 0), "high_line_count"),
              sum_(case([(low, 1)], 0), "low_line_count")],
        order_col=0, radix_bits=radix_bits)


def batch_plan() -> AggPlan:
    v = col(1)
    return AggPlan(None, [0], [sum_(v, "sum"), count_star("count"), min_(v, "min"), max_(v, "max"),
                               avg(v, "avg")])
