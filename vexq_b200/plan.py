"""Plan descriptors: SQL-level expression trees flattened into the node arrays
of include/vexq_cuda.h (vexq_expr / vexq_agg_plan_desc / vexq_join_plan_desc).

The trees mirror vexq's sql.Expr shapes (sql/ast.go); the library performs
the planner's translation to executable form (planner/physical.go:376-818).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

from . import abi


@dataclass
class E:
    kind: int
    op: int = 0
    column: int = -1
    lit_kind: int = 0
    lit_int: int = 0
    lit_float: float = 0.0
    lit_str: Optional[str] = None
    children: List["E"] = field(default_factory=list)

    # operator sugar: comparisons and arithmetic build BINARY nodes
    def _bin(self, op, other):
        return E(abi.E_BINARY, op=op, children=[self, _wrap(other)])

    def __eq__(self, o):  # type: ignore[override]
        return self._bin(abi.OP_EQ, o)

    def __ne__(self, o):  # type: ignore[override]
        return self._bin(abi.OP_NE, o)

    def __lt__(self, o):
        return self._bin(abi.OP_LT, o)

    def __le__(self, o):
        return self._bin(abi.OP_LE, o)

    def __gt__(self, o):
        return self._bin(abi.OP_GT, o)

    def __ge__(self, o):
        return self._bin(abi.OP_GE, o)

    def __add__(self, o):
        return self._bin(abi.OP_ADD, o)

    def __radd__(self, o):
        return _wrap(o)._bin(abi.OP_ADD, self)

    def __sub__(self, o):
        return self._bin(abi.OP_SUB, o)

    def __rsub__(self, o):
        return _wrap(o)._bin(abi.OP_SUB, self)

    def __mul__(self, o):
        return self._bin(abi.OP_MUL, o)

    def __rmul__(self, o):
        return _wrap(o)._bin(abi.OP_MUL, self)

    def __truediv__(self, o):
        return self._bin(abi.OP_DIV, o)

    __hash__ = None  # type: ignore[assignment]


def _wrap(v) -> E:
    return v if isinstance(v, E) else lit(v)


def col(i: int) -> E:
    return E(abi.E_COLUMN, column=int(i))


def lit(v) -> E:
    if isinstance(v, bool):
        return E(abi.E_LITERAL, lit_kind=abi.LIT_BOOL, lit_int=int(v))
    if isinstance(v, int):
        return E(abi.E_LITERAL, lit_kind=abi.LIT_INT, lit_int=v)
    if isinstance(v, float):
        return E(abi.E_LITERAL, lit_kind=abi.LIT_FLOAT, lit_float=v)
    if isinstance(v, str):
        return E(abi.E_LITERAL, lit_kind=abi.LIT_STRING, lit_str=v)
    raise TypeError(f"unsupported literal {v!r}")


def binop(op: int, l, r) -> E:
    return E(abi.E_BINARY, op=op, children=[_wrap(l), _wrap(r)])


def and_(*xs) -> E:
    return E(abi.E_AND, children=[_wrap(x) for x in xs])


def or_(*xs) -> E:
    return E(abi.E_OR, children=[_wrap(x) for x in xs])


def not_(x) -> E:
    return E(abi.E_NOT, children=[_wrap(x)])


def neg(x) -> E:
    return E(abi.E_NEG, children=[_wrap(x)])


def is_null(x) -> E:
    return E(abi.E_IS_NULL, children=[_wrap(x)])


def is_not_null(x) -> E:
    return E(abi.E_IS_NOT_NULL, children=[_wrap(x)])


def between(x, lo, hi, negate=False) -> E:
    return E(abi.E_BETWEEN, op=1 if negate else 0, children=[_wrap(x), _wrap(lo), _wrap(hi)])


def in_(x, values: Sequence, negate=False) -> E:
    return E(abi.E_IN, op=1 if negate else 0, children=[_wrap(x)] + [lit(v) for v in values])


def like(x, pattern: str, negate=False) -> E:
    return E(abi.E_LIKE, op=1 if negate else 0, children=[_wrap(x), lit(pattern)])


def case(whens: Sequence, else_=None) -> E:
    ch: List[E] = []
    for c, r in whens:
        ch += [_wrap(c), _wrap(r)]
    if else_ is not None:
        ch.append(_wrap(else_))
    return E(abi.E_CASE, op=1 if else_ is not None else 0, children=ch)


@dataclass
class Agg:
    kind: int
    input: Optional[E]
    name: str = ""


def count_star(name="count") -> Agg:
    return Agg(abi.AGG_COUNT, None, name)


def count(x, name="count") -> Agg:
    return Agg(abi.AGG_COUNT, _wrap(x), name)


def count_distinct(x, name="count_distinct") -> Agg:
    """COUNT(DISTINCT x): distinct non-NULL values per group, never NULL."""
    return Agg(abi.AGG_COUNT_DISTINCT, _wrap(x), name)


def sum_(x, name="sum") -> Agg:
    return Agg(abi.AGG_SUM, _wrap(x), name)


def avg(x, name="avg") -> Agg:
    return Agg(abi.AGG_AVG, _wrap(x), name)


def min_(x, name="min") -> Agg:
    return Agg(abi.AGG_MIN, _wrap(x), name)


def max_(x, name="max") -> Agg:
    return Agg(abi.AGG_MAX, _wrap(x), name)


class _Arena:
    """Flattens trees into the node/children arrays; keeps bytes alive."""

    def __init__(self):
        self.nodes: List[E] = []
        self.idx: List[List[int]] = []
        self.keep: list = []

    def add(self, e: Optional[E]) -> int:
        if e is None:
            return -1
        kids = [self.add(c) for c in e.children]
        self.nodes.append(e)
        self.idx.append(kids)
        return len(self.nodes) - 1

    def arrays(self):
        n = len(self.nodes)
        nodes = (abi.Expr * max(n, 1))()
        flat: List[int] = []
        for i, e in enumerate(self.nodes):
            s = e.lit_str.encode() if e.lit_str is not None else None
            self.keep.append(s)
            nodes[i] = abi.Expr(e.kind, e.op, e.column, e.lit_kind, e.lit_int, e.lit_float, s,
                                len(flat), len(self.idx[i]))
            flat += self.idx[i]
        ch = (C.c_int32 * max(len(flat), 1))(*flat)
        self.keep += [nodes, ch]
        return nodes, n, ch, len(flat)


def _aggs(arena: _Arena, aggs: Sequence[Agg]):
    arr = (abi.AggDesc * max(len(aggs), 1))()
    for j, a in enumerate(aggs):
        nm = a.name.encode()
        arena.keep.append(nm)
        arr[j] = abi.AggDesc(a.kind, arena.add(a.input), nm)
    arena.keep.append(arr)
    return arr


class AggPlan:
    """Filter → (Project) → HashAggregate over one table."""

    def __init__(self, predicate: Optional[E], group_by: Sequence[int], aggs: Sequence[Agg],
                 order_col: int = -1, descending: bool = False, limit: int = -1,
                 having: Optional[E] = None, visible: int = -1):
        self.predicate, self.group_by, self.aggs = predicate, list(group_by), list(aggs)
        self.order = (order_col, descending, limit)
        self.having = having_arrays(having, visible)
        a = _Arena()
        pred = a.add(predicate)
        aggarr = _aggs(a, self.aggs)
        nodes, nn, ch, nc = a.arrays()
        gb = (C.c_int32 * max(len(self.group_by), 1))(*self.group_by)
        a.keep.append(gb)
        self._arena = a
        self.desc = abi.AggPlanDesc(nodes, nn, ch, nc, pred, gb, len(self.group_by), aggarr,
                                    len(self.aggs), abi.OrderDesc(order_col, int(descending), limit))


class JoinPlan:
    """Filter(build) ⋈ Filter(probe) → residual Filter → HashAggregate."""

    def __init__(self, build_key: int, probe_key: int, build_predicate: Optional[E],
                 probe_predicate: Optional[E], residual: Optional[E], group_by: Sequence[int],
                 aggs: Sequence[Agg], order_col: int = -1, descending: bool = False,
                 limit: int = -1, radix_bits: int = -1, having: Optional[E] = None, visible: int = -1):
        self.group_by, self.aggs = list(group_by), list(aggs)
        self.order_col, self.descending, self.limit = order_col, descending, limit
        self.having = having_arrays(having, visible)
        a = _Arena()
        bp, pp, rp = a.add(build_predicate), a.add(probe_predicate), a.add(residual)
        aggarr = _aggs(a, self.aggs)
        nodes, nn, ch, nc = a.arrays()
        gb = (C.c_int32 * max(len(self.group_by), 1))(*self.group_by)
        a.keep.append(gb)
        self._arena = a
        self.desc = abi.JoinPlanDesc(nodes, nn, ch, nc, build_key, probe_key, bp, pp, rp, gb,
                                     len(self.group_by), aggarr, len(self.aggs),
                                     abi.OrderDesc(order_col, int(descending), limit), radix_bits)


def having_arrays(having: Optional[E], visible: int = -1):
    """HAVING (vexq_plan_set_having): a predicate over the output columns
    (group-by columns, then aggregates) and how many leading output columns
    to keep; None when there is no HAVING."""
    if having is None:
        return None
    a = _Arena()
    root = a.add(having)
    nodes, nn, ch, nc = a.arrays()
    return (a, nodes, nn, ch, nc, root, visible)


def predicate_arrays(pred: E):
    """Node arrays for a standalone predicate (vexq_filter_run)."""
    a = _Arena()
    root = a.add(pred)
    nodes, nn, ch, nc = a.arrays()
    return a, nodes, nn, ch, nc, root


def project_arrays(pred: Optional[E], exprs: Sequence[E]):
    """Node arrays for Filter → Project (vexq_project_run): one arena holding
    the predicate (root -1 when there is none) and every projected expression."""
    a = _Arena()
    root = a.add(pred) if pred is not None else -1
    roots = [a.add(e) for e in exprs]
    nodes, nn, ch, nc = a.arrays()
    return a, nodes, nn, ch, nc, root, roots
