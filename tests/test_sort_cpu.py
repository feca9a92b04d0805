"""The sort oracle without a GPU, pinned to the reference's own tests: the Sort / top_k /
bottom_k cases of tests/python_integration/test_walker_sort_fused.py, and the group-by cases of
tests/python_integration/test_groupby.py, whose queries end in `.sort(keys)` (their expected rows
are in key order, nulls first); plus Polars' order rules (NaN last, -0.0 equal to 0.0, nulls
placed by nulls_last whatever the direction) against a pure-Python restatement."""

import math

import numpy as np
import pytest

from helpers import case_columns, expected_to_result, formula_columns, load_golden, pack, unpack
from oracle import pyoracle
from polars_b200 import _abi as A
from polars_b200._native import _sort_spec

SORT = load_golden()["sort"]


def sort_case_columns(case: dict) -> dict:
    if "formula" in case:
        f = case["formula"]
        x = np.random.default_rng(f["seed"]).standard_normal(f["n"]).astype(np.float32)
        return {"x": (x, None)}
    return case_columns(case)


def sort_case_expected(case: dict) -> dict:
    """{name: list of values (None for null)} in order."""
    if "formula" not in case:
        return case["expected"]
    x = sort_case_columns(case)["x"][0]
    s = case["spec"]
    v = np.sort(x)
    if s["descending"][0]:
        v = v[::-1]
    if s["limit"] >= 0:
        v = v[: s["limit"]]
    return {"x": [float(a) for a in v]}


def result_lists(res: dict) -> dict:
    n = int(res["n_groups"])
    out = {}
    for name, dt, d, v in zip(res["names"], res["dtypes"], res["data"], res["validity"]):
        vals = unpack(d, n) if dt == A.BOOL else np.asarray(d)[:n]
        ok = unpack(v, n)
        out[name] = [(vals[i].item() if ok[i] else None) for i in range(n)]
    return out


def oracle_sort(case: dict) -> dict:
    s = case["spec"]
    return pyoracle.sort_table(sort_case_columns(case), s["by"], s["descending"], s["nulls_last"], s["drop_nulls"],
                               s["offset"], s["limit"])


@pytest.mark.parametrize("case", SORT, ids=lambda c: c["name"])
def test_oracle_matches_the_reference_sort_cases(case):
    got = result_lists(oracle_sort(case))
    want = sort_case_expected(case)
    assert set(want) <= set(got)
    for name, vals in want.items():
        assert got[name] == vals, name


@pytest.mark.parametrize("case", [c for c in load_golden()["integration"] if c["formula"] != "all_unique"],
                         ids=lambda c: c["name"])
def test_oracle_group_by_then_sort_gives_the_reference_rows_in_order(case):
    cols = formula_columns(case["formula"], case["n"])
    aggs = [tuple(a) for a in case["aggs"]]
    g = pyoracle.groupby(cols, case["keys"], aggs)
    table = {name: (d, v, dt, g["n_groups"]) for name, d, v, dt in zip(g["names"], g["data"], g["validity"], g["dtypes"])}
    got = result_lists(pyoracle.sort_table(table, case["keys"]))
    for name, vals in case["expected"].items():
        if g["dtypes"][g["names"].index(name)] in (A.F32, A.F64):
            assert all((a is None and b is None) or math.isclose(a, b, rel_tol=1e-6) for a, b in zip(got[name], vals))
        else:
            assert got[name] == vals, name


def _py_key(v, desc, nulls_last):
    """Polars' order of one value restated in plain Python: (null group, value rank)."""
    if v is None:
        return (1 if nulls_last else -1, 0)
    if isinstance(v, float):
        rank = (1, 0.0) if math.isnan(v) else (0, v + 0.0)
        rank = (rank[0], rank[1])
        if desc:
            rank = (-rank[0], -rank[1])
        return (0, rank)
    return (0, (0, -v if desc else v))


@pytest.mark.parametrize("desc", [False, True])
@pytest.mark.parametrize("nulls_last", [False, True])
def test_oracle_order_rules(desc, nulls_last):
    vals = [1.5, float("nan"), -0.0, None, 0.0, float("-inf"), 2.0, None, float("inf"), -1.0, float("nan"), 0.0]
    n = len(vals)
    ok = np.array([v is not None for v in vals])
    x = np.array([0.0 if v is None else v for v in vals])
    rid = np.arange(n, dtype=np.int64)
    res = pyoracle.sort_table({"x": (x, pack(ok)), "rid": (rid, None)}, ["x"], [desc], [nulls_last])
    got_ids = list(res["data"][1])
    want_ids = sorted(range(n), key=lambda i: _py_key(vals[i], desc, nulls_last))  # sorted() is stable
    assert got_ids == want_ids


def test_oracle_many_columns_and_slices():
    rng = np.random.default_rng(4)
    n = 2_000
    a = rng.integers(0, 3, n).astype(np.int8)
    b = rng.standard_normal(n)
    bn = rng.random(n) < 0.2
    c = rng.integers(0, 2**63, n, dtype=np.uint64)
    rid = np.arange(n, dtype=np.int64)
    cols = {"a": (a, None), "b": (b, pack(~bn)), "c": (c, None), "rid": (rid, None)}
    res = pyoracle.sort_table(cols, ["a", "b", "c"], [True, False, True], [False, True, False], offset=-300, limit=100)
    key = lambda i: (-int(a[i]), (1, 0) if bn[i] else (0, b[i]), -int(c[i]), i)  # noqa: E731
    full = sorted(range(n), key=key)
    assert list(res["data"][3]) == full[n - 300: n - 200]


def test_sort_spec_broadcasts_flags_and_checks_names():
    spec, _keep = _sort_spec(["k", "s", "n"], ["s", "k"], descending=True, nulls_last=[False, True], limit=5)
    assert spec.n_by == 2 and list(spec.by[:2]) == [1, 0] and list(spec.descending[:2]) == [1, 1]
    assert list(spec.nulls_last[:2]) == [0, 1] and spec.limit == 5 and spec.offset == 0
    assert _sort_spec(["k"], "k")[0].limit == -1
    with pytest.raises(KeyError):
        _sort_spec(["k"], ["z"])
    with pytest.raises(ValueError):
        _sort_spec(["k", "s"], ["k", "s"], descending=[True])


def test_sort_plan_errors_before_any_device_work():
    from polars_b200._native import execute_sort

    with pytest.raises(ValueError, match="missing field input"):
        execute_sort({"kind": "Sort", "by_columns": ["k"]}, 0, [])
    with pytest.raises(ValueError, match="slice without sort columns"):
        execute_sort({"kind": "Sort", "input": {"keys": [], "aggs": []}, "by_columns": [], "slice": [0, 5]}, 0, [])
    with pytest.raises(ValueError, match="negative slice length"):
        _sort_spec(["k"], "k", limit=-3)
