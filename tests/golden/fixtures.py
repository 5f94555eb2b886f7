"""Loads known_answers.json into host tables and plan descriptors."""
from __future__ import annotations

import json
import os

import numpy as np

from vexq_b200 import abi
from vexq_b200 import plan as P
from vexq_b200.table import HostColumn, HostTable, _flatten_dicts, pack_validity

HERE = os.path.dirname(os.path.abspath(__file__))
TYPES = {"INT64": abi.TYPE_INT64, "FLOAT64": abi.TYPE_FLOAT64, "DATE": abi.TYPE_DATE,
         "STRING": abi.TYPE_STRING, "BOOL": abi.TYPE_BOOL}
OPS = {"EQ": abi.OP_EQ, "NE": abi.OP_NE, "LT": abi.OP_LT, "LE": abi.OP_LE, "GT": abi.OP_GT,
       "GE": abi.OP_GE, "ADD": abi.OP_ADD, "SUB": abi.OP_SUB, "MUL": abi.OP_MUL, "DIV": abi.OP_DIV}
AGGS = {"COUNT": P.count, "SUM": P.sum_, "AVG": P.avg, "MIN": P.min_, "MAX": P.max_,
        "COUNT_DISTINCT": P.count_distinct}


def load_cases():
    with open(os.path.join(HERE, "known_answers.json")) as f:
        return json.load(f)["cases"]


def make_table(spec) -> HostTable:
    cols = []
    n = spec["nrows"]
    for c in spec["columns"]:
        t = TYPES[c["type"]]
        valid = None if c.get("valid") is None else np.asarray(c["valid"], dtype=bool)
        if t == abi.TYPE_STRING:
            entries = [s.encode() for d in c["rg_dicts"] for s in d]
            first = np.cumsum([0] + [len(d) for d in c["rg_dicts"]]).astype(np.uint32)
            off, data = _flatten_dicts(entries)
            cols.append(HostColumn(c["name"], t, np.asarray(c["codes"], dtype=np.uint32), pack_validity(valid),
                                   first, off, data))
        else:
            cols.append(HostColumn(c["name"], t, np.asarray(c["values"]), pack_validity(valid)))
    return HostTable(cols, n, spec["rg_rows"])


def expr(e):
    if e is None:
        return None
    k = e[0]
    if k == "col":
        return P.col(e[1])
    if k == "lit":
        return P.lit(e[1])
    if k == "bin":
        return P.binop(OPS[e[1]], expr(e[2]), expr(e[3]))
    if k == "and":
        return P.and_(*[expr(x) for x in e[1:]])
    if k == "or":
        return P.or_(*[expr(x) for x in e[1:]])
    if k == "not":
        return P.not_(expr(e[1]))
    if k == "neg":
        return P.neg(expr(e[1]))
    if k == "between":
        return P.between(expr(e[1]), expr(e[2]), expr(e[3]))
    if k == "in":
        return P.in_(expr(e[1]), e[2])
    if k == "case":
        return P.case([(expr(c), expr(r)) for c, r in e[1]], expr(e[2]) if len(e) > 2 else None)
    raise ValueError(k)


def aggs(spec):
    out = []
    for kind, inp, name in spec:
        out.append(P.count_star(name) if (kind == "COUNT" and inp is None) else AGGS[kind](expr(inp), name))
    return out


def make_plan(c, radix_bits: int = -1):
    p = c["plan"]
    if c["kind"] == "join":
        return P.JoinPlan(p["build_key"], p["probe_key"], expr(p["build_predicate"]), expr(p["probe_predicate"]),
                          expr(p["residual"]), p["group_by"], aggs(p["aggs"]), radix_bits=radix_bits)
    return P.AggPlan(expr(p["predicate"]), p["group_by"], aggs(p["aggs"]))


def normalize(rows, ordered):
    rows = [tuple(r) for r in rows]
    return rows if ordered else sorted(rows, key=repr)
