"""The CPU oracle reproduces the answers the reference's own tests assert
(tests/golden/known_answers.json, transcribed from the vexq test files)."""
import pytest

from oracle import refcpu as R
from tests.golden.fixtures import load_cases, make_plan, make_table, normalize

CASES = load_cases()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
@pytest.mark.parametrize("workers", [0, 1, 3])
def test_oracle_matches_reference_known_answer(case, workers):
    plan = make_plan(case)
    if case["kind"] == "join":
        b, p = R.RefTable(make_table(case["tables"]["build"])), R.RefTable(make_table(case["tables"]["probe"]))
        res = R.join(b, p, plan, workers=workers)
    else:
        t = R.RefTable(make_table(case["tables"]["t"]))
        res = R.agg(t, plan, workers=workers)
    ordered = case["expect"]["ordered"] and workers == 0
    assert normalize(res.rows(), ordered) == normalize(case["expect"]["rows"], ordered)
