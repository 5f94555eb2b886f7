"""Comparison helpers shared by the GPU parity tests."""
from __future__ import annotations

import math

from vexq_b200 import abi

# Float64 SUM/AVG tolerance against the serial oracle (the reference's
# deterministic row-order fold): 1e-12 relative.
FLOAT_RTOL = 1e-12


def close(a, b, rtol=FLOAT_RTOL) -> bool:
    if a is None or b is None:
        return a is None and b is None
    if isinstance(a, float) or isinstance(b, float):
        a, b = float(a), float(b)
        if math.isnan(a) or math.isnan(b):
            return math.isnan(a) and math.isnan(b)
        if math.isinf(a) or math.isinf(b):
            return a == b
        return abs(a - b) <= rtol * max(abs(a), abs(b), 1e-300)
    return a == b


def assert_rows_match(gpu_rows, ref_rows, ordered=True, rtol=FLOAT_RTOL, exact_float_cols=()):
    """Row-by-row equality: integers/strings bit-exact, floats within rtol.
    Unordered comparison matches rows on their non-float cells."""
    assert len(gpu_rows) == len(ref_rows), (len(gpu_rows), len(ref_rows), gpu_rows[:5], ref_rows[:5])
    if not ordered:
        def key(r):
            return repr(tuple(v for v in r if not isinstance(v, float)))
        gpu_rows = sorted(gpu_rows, key=key)
        ref_rows = sorted(ref_rows, key=key)
    for i, (g, r) in enumerate(zip(gpu_rows, ref_rows)):
        assert len(g) == len(r)
        for j, (a, b) in enumerate(zip(g, r)):
            tol = 0.0 if j in exact_float_cols else rtol
            assert close(a, b, tol), f"row {i} col {j}: gpu={a!r} ref={b!r}\n gpu={g}\n ref={r}"


def assert_sorted_rows_match(gpu_rows, ref_rows, order_col, descending=True, rtol=FLOAT_RTOL):
    """ORDER BY a float aggregate: the sort-column values agree position by
    position (within rtol) and the rows agree as a set. Rows whose sort values
    tie within the tolerance may come in either order: the GPU sums are exact,
    so two groups with the same exact sum tie there, while the reference's
    row-order fold can leave them an ulp apart."""
    assert len(gpu_rows) == len(ref_rows), (len(gpu_rows), len(ref_rows))
    vals = [r[order_col] for r in gpu_rows]
    assert all((a >= b) if descending else (a <= b) for a, b in zip(vals, vals[1:])), "GPU rows out of order"
    for i, (g, r) in enumerate(zip(gpu_rows, ref_rows)):
        assert close(g[order_col], r[order_col], rtol), f"row {i}: gpu={g} ref={r}"
    assert_rows_match(gpu_rows, ref_rows, ordered=False, rtol=rtol)


def assert_float_vs_exact(gpu_rows, ref, ordered=True, rtol=FLOAT_RTOL, exact_tol=1e-13):
    """Float64 SUM/AVG parity with the exact-summation oracle as arbiter.

    The reference's serial row-order fold carries its own rounding error
    (≈1e-12 relative at a million rows of k/100 values). A GPU value passes
    when it is within `exact_tol` of the exact sum and its distance to the
    reference is within `rtol` or explained by the reference's own error.
    Returns (worst GPU error vs exact, worst reference error vs exact)."""
    ref_rows = ref.rows()
    assert len(gpu_rows) == len(ref_rows)
    worst_g = worst_r = 0.0
    for i, (g, r) in enumerate(zip(gpu_rows, ref_rows)):
        for j, (a, b) in enumerate(zip(g, r)):
            ex = ref.exact[j][i] if ref.types[j] == abi.TYPE_FLOAT64 else float("nan")
            if ref.types[j] != abi.TYPE_FLOAT64 or math.isnan(ex) or a is None or b is None:
                assert close(a, b, rtol), f"row {i} col {j}: gpu={a!r} ref={b!r}"
                continue
            scale = max(abs(ex), 1e-300)
            eg, er = abs(a - ex) / scale, abs(b - ex) / scale
            worst_g, worst_r = max(worst_g, eg), max(worst_r, er)
            assert eg <= exact_tol, f"row {i} col {j}: gpu={a!r} exact={ex!r} (err {eg:.3g})"
            assert close(a, b, rtol) or abs(a - b) / scale <= er + exact_tol, \
                f"row {i} col {j}: gpu={a!r} ref={b!r} exact={ex!r}"
    return worst_g, worst_r


def float_cols(types):
    return [i for i, t in enumerate(types) if t == abi.TYPE_FLOAT64]
