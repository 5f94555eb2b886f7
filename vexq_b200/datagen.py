"""Seeded synthetic tables with the shapes of the benchmark workloads.

TPC-H data is not available here; these generators stand in for it with
the distributions the workloads specify (no TPC-H rows are reproduced):

  lineitem(n)   flag{A,R,N} weights .25/.25/.5, status{F,O}, qty U{1..50},
                price = round2(qty × U(900,105000)/100), disc k/100 k∈0..10,
                tax k/100 k∈0..8, shipdate U over 2526 days from 1992-01-02.
  orders(n)     unique shuffled keys 1..n, orderdate U over 2400 days,
                priority dict{5}.
  items(n, m)   fk U over 1..m, shipdate U over 2400 days, price, disc,
                mode dict{7}.
  zipf_groups   int32 dictionary codes with Zipf(s) frequencies over a
                cardinality, f64 values U(0,1e5) rounded to 2 decimals.
"""
from __future__ import annotations

import numpy as np

from . import abi
from .table import HostTable, date_column, float_column, int_column, string_column

EPOCH_1992_01_02 = 8036   # days since 1970-01-01
EPOCH_1998_12_01 = 10561  # 8036 + 2525
EPOCH_1992_01_01 = 8035

FLAGS = ["A", "R", "N"]
FLAG_P = [0.25, 0.25, 0.5]
STATUS = ["F", "O"]
PRIORITIES = ["1-URGENT", "2-HIGH", "3-MEDIUM", "4-NOT SPECIFIED", "5-LOW"]
MODES = ["REG AIR", "AIR", "RAIL", "SHIP", "TRUCK", "MAIL", "FOB"]

# column indices of lineitem()
L_FLAG, L_STATUS, L_QTY, L_PRICE, L_DISC, L_TAX, L_SHIPDATE = range(7)


def lineitem(nrows: int, seed: int = 42, rg_rows: int = abi.ROW_GROUP_ROWS) -> HostTable:
    rng = np.random.default_rng(seed)
    flag = rng.choice(3, size=nrows, p=FLAG_P)
    status = rng.integers(0, 2, size=nrows)
    qty = rng.integers(1, 51, size=nrows, dtype=np.int64)
    cents = np.rint(qty * rng.uniform(900.0, 105000.0, size=nrows))
    price = cents / 100.0
    disc = rng.integers(0, 11, size=nrows) / 100.0
    tax = rng.integers(0, 9, size=nrows) / 100.0
    ship = (EPOCH_1992_01_02 + rng.integers(0, 2526, size=nrows)).astype(np.int32)
    cols = [
        string_column("l_returnflag", flag, FLAGS, nrows, rg_rows),
        string_column("l_linestatus", status, STATUS, nrows, rg_rows),
        int_column("l_quantity", qty),
        float_column("l_extendedprice", price),
        float_column("l_discount", disc),
        float_column("l_tax", tax),
        date_column("l_shipdate", ship),
    ]
    return HostTable(cols, nrows, rg_rows)


# column indices of orders() / items()
O_KEY, O_DATE, O_PRIORITY = range(3)
I_FK, I_SHIPDATE, I_PRICE, I_DISC, I_MODE = range(5)
DATE_SPAN = 2400


def orders(nrows: int, seed: int = 7, rg_rows: int = abi.ROW_GROUP_ROWS) -> HostTable:
    rng = np.random.default_rng(seed)
    keys = rng.permutation(np.arange(1, nrows + 1, dtype=np.int64))
    od = (EPOCH_1992_01_01 + rng.integers(0, DATE_SPAN, size=nrows)).astype(np.int32)
    prio = rng.integers(0, 5, size=nrows)
    cols = [int_column("o_orderkey", keys), date_column("o_orderdate", od),
            string_column("o_orderpriority", prio, PRIORITIES, nrows, rg_rows)]
    return HostTable(cols, nrows, rg_rows)


def items(nrows: int, build_rows: int, seed: int = 11, rg_rows: int = abi.ROW_GROUP_ROWS) -> HostTable:
    rng = np.random.default_rng(seed)
    fk = rng.integers(1, build_rows + 1, size=nrows, dtype=np.int64)
    sd = (EPOCH_1992_01_01 + rng.integers(0, DATE_SPAN, size=nrows)).astype(np.int32)
    qty = rng.integers(1, 51, size=nrows)
    price = np.rint(qty * rng.uniform(900.0, 105000.0, size=nrows)) / 100.0
    disc = rng.integers(0, 11, size=nrows) / 100.0
    mode = rng.integers(0, 7, size=nrows)
    cols = [int_column("l_orderkey", fk), date_column("l_shipdate", sd),
            float_column("l_extendedprice", price), float_column("l_discount", disc),
            string_column("l_shipmode", mode, MODES, nrows, rg_rows)]
    return HostTable(cols, nrows, rg_rows)


def join_mid(frac: float) -> int:
    """Date cutoff leaving `frac` of a uniform 2400-day range below it."""
    return EPOCH_1992_01_01 + int(round(frac * DATE_SPAN))


def zipf_codes(rng, n: int, card: int, s: float = 1.1) -> np.ndarray:
    ranks = np.arange(1, card + 1, dtype=np.float64)
    p = ranks ** (-s)
    cdf = np.cumsum(p)
    cdf /= cdf[-1]
    return np.searchsorted(cdf, rng.random(n), side="right").clip(0, card - 1)


def zipf_groups(nrows: int, card: int, seed: int, s: float = 1.1,
                rg_rows: int = abi.ROW_GROUP_ROWS, per_rg_dicts: bool = False) -> HostTable:
    """GROUP BY input: key dictionary codes with Zipf(s) frequencies and a
    float64 value U(0,1e5) rounded to 2 decimals."""
    rng = np.random.default_rng(seed)
    rank = zipf_codes(rng, nrows, card, s)
    perm = rng.permutation(card)
    universe = [f"k{int(i):05d}" for i in range(card)]
    vals = np.rint(rng.uniform(0.0, 1e7, size=nrows)) / 100.0
    cols = [string_column("g_key", perm[rank], universe, nrows, rg_rows, per_rg=per_rg_dicts),
            float_column("g_value", vals)]
    return HostTable(cols, nrows, rg_rows)
