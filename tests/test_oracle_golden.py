"""Pins the CPU oracle to the reference's own known-answer tests (no GPU needed)."""

import math

import numpy as np
import pytest

from helpers import (assert_results_match, case_columns, expected_to_result, formula_columns, load_golden, pack,
                     unpack)
from oracle import pyoracle
from polars_b200 import _abi as A

GOLD = load_golden()


@pytest.mark.parametrize("case", GOLD["groupby"], ids=lambda c: c["name"])
def test_oracle_groupby_known_answers(case):
    got = pyoracle.groupby(case_columns(case), case["keys"], [tuple(a) for a in case["aggs"]])
    want = expected_to_result(case)
    assert_results_match(got, want, len(case["keys"]), case["aggs"], case["name"])


@pytest.mark.parametrize("case", GOLD["integration"], ids=lambda c: c["name"])
def test_oracle_integration_shapes(case):
    cols = formula_columns(case["formula"], case["n"])
    got = pyoracle.groupby(cols, case["keys"], [tuple(a) for a in case["aggs"]])
    if case["formula"] == "all_unique":
        assert got["n_groups"] == case["expected"]["n_groups"]
        assert np.all(got["data"][1] == 1)
        return
    want = expected_to_result(case)
    assert_results_match(got, want, len(case["keys"]), case["aggs"], case["name"])


def _cmp_pred(op, scalar=None):
    rhs = {"kind": "LiteralF64", "value": scalar} if scalar is not None else {"kind": "Column", "name": "r"}
    return {"kind": "Compare", "op": op, "dtype": "F64", "lhs": {"kind": "Column", "name": "l"}, "rhs": rhs}


@pytest.mark.parametrize("case", GOLD["compare"], ids=lambda c: c["name"])
def test_oracle_compare_semantics(case):
    n = len(case["lhs"])
    cols = {"l": (np.array(case["lhs"], np.float64), pack(case["lhs_valid"]))}
    if "rhs" in case:
        cols["r"] = (np.array(case["rhs"], np.float64), pack(case["rhs_valid"]))
        pred = _cmp_pred(case["op"])
    else:
        pred = _cmp_pred(case["op"], case["scalar"])
    d, v = pyoracle.predicate_bits(cols, pred)
    assert list(unpack(d, n).astype(int)) == case["expected_data"]
    assert list(unpack(v, n).astype(int)) == case["expected_valid"]


def _tri_bits(vals):
    data = pack([v == "T" for v in vals])
    valid = pack([v != "N" for v in vals])
    return data, valid


def test_oracle_kleene_tables():
    case = GOLD["kleene"][0]
    ld, lv = _tri_bits(case["lhs"])
    rd, rv = _tri_bits(case["rhs"])
    n = len(case["lhs"])
    for op in ("and", "or"):
        d, v = pyoracle.bool_logic(op, ld.tobytes(), lv.tobytes(), rd.tobytes(), rv.tobytes(), n)
        dd, vv = unpack(d, n), unpack(v, n)
        got = ["N" if not vv[i] else ("T" if dd[i] else "F") for i in range(n)]
        assert got == case[op], op


def test_oracle_mod_predicate_floor_semantics():
    # Polars integer `%` is a floor modulo (sign of the divisor); x % 0 is null
    v = np.array([-7, -1, 0, 6, 7, 13, 5], np.int64)
    cols = {"v": (v, None)}
    pred = {"kind": "Compare", "op": "Eq", "dtype": "I64",
            "lhs": {"kind": "Arith", "op": "Mod", "dtype": "I64", "lhs": {"kind": "Column", "name": "v"},
                    "rhs": {"kind": "LiteralI64", "value": 7}},
            "rhs": {"kind": "LiteralI64", "value": 6}}
    keep = pyoracle.filter_mask(cols, pred)
    assert list(keep) == [False, True, False, True, False, True, False]
    pred0 = dict(pred)
    pred0["lhs"] = dict(pred["lhs"], rhs={"kind": "LiteralI64", "value": 0})
    d, vmask = pyoracle.predicate_bits(cols, pred0)
    assert not unpack(vmask, 7).any()


def test_oracle_filter_compact_and_cumsum():
    rng = np.random.default_rng(0)
    n = 1000
    a = rng.integers(-5, 5, n).astype(np.int64)
    va = rng.random(n) > 0.1
    keep = rng.random(n) > 0.5
    m, cols = pyoracle.filter_compact(keep, {"a": (a, pack(va))})
    assert m == keep.sum()
    assert np.array_equal(cols[0][1][:m], a[keep])
    assert np.array_equal(unpack(cols[0][2], m), va[keep])
    u8 = rng.integers(0, 2, n).astype(np.uint8)
    assert np.array_equal(pyoracle.cumsum_u8_to_u32(u8), np.cumsum(u8).astype(np.uint32))


def test_oracle_exact_sum_beats_naive_on_cancellation():
    # compensated summation keeps an exactly representable cancelling sum exact
    v = np.array([1e16, 1.0, -1e16, 1.0] * 1000, np.float64)
    got = pyoracle.groupby({"k": (np.zeros(v.size, np.int32), None), "v": (v, None)}, ["k"], [("Sum", "v", "s")])
    assert got["data"][1][0] == 2000.0
    assert math.fsum(v) == 2000.0


@pytest.mark.parametrize("case", GOLD["compare_i64"], ids=lambda c: c["name"])
def test_oracle_compare_i64_known_answers(case):
    n = len(case["lhs"])
    cols = {"l": (np.array(case["lhs"], np.int64), pack(case["lhs_valid"]))}
    rhs = {"kind": "LiteralI64", "value": case["scalar"]} if "scalar" in case else {"kind": "Column", "name": "r"}
    if "rhs" in case:
        cols["r"] = (np.array(case["rhs"], np.int64), pack(case["rhs_valid"]))
    pred = {"kind": "Compare", "op": case["op"], "dtype": "I64", "lhs": {"kind": "Column", "name": "l"}, "rhs": rhs}
    d, v = pyoracle.predicate_bits(cols, pred)
    valid = list(unpack(v, n).astype(int))
    assert valid == case["expected_valid"]
    assert [b for b, ok in zip(unpack(d, n).astype(int), valid) if ok] == \
        [b for b, ok in zip(case["expected_data"], valid) if ok]


@pytest.mark.parametrize("case", GOLD["pipeline"], ids=lambda c: c["name"])
def test_oracle_pipeline_known_answers(case):
    got = pyoracle.groupby(case_columns(case), case["keys"], [tuple(a) for a in case["aggs"]])
    assert_results_match(got, expected_to_result(case), len(case["keys"]), case["aggs"], case["name"])


@pytest.mark.parametrize("case", GOLD["compact"], ids=lambda c: c["name"])
def test_oracle_compaction_known_answers(case):
    from helpers import compact_case_expected, compact_case_inputs, same_values

    cols, pd, pv, n = compact_case_inputs(case)
    keep = np.array(pd, bool) & np.array(pv, bool)
    n_out, out = pyoracle.filter_compact(keep, cols)
    want = compact_case_expected(case)
    assert n_out == len(next(iter(want.values())))
    for (name, vals), (dt, data, valid) in zip(want.items(), out):
        got = list(unpack(data, n_out)) if dt == A.BOOL else list(np.asarray(data)[:n_out])
        ok = list(unpack(valid, n_out))
        assert ok == [v is not None for v in vals], name
        got = [x.item() if hasattr(x, "item") else x for x, o in zip(got, ok) if o]
        assert same_values(got, [v for v in vals if v is not None]), name


@pytest.mark.parametrize("case", GOLD["sort_build"], ids=lambda c: c["name"])
def test_oracle_sort_build_known_answers(case):
    got = pyoracle.groupby(case_columns(case), case["keys"], [tuple(a) for a in case["aggs"]])
    assert_results_match(got, expected_to_result(case), 1, case["aggs"], case["name"])


@pytest.mark.parametrize("case", GOLD["predicate_mask"], ids=lambda c: c["name"])
def test_oracle_predicate_mask_known_answers(case):
    # the oracle's compaction keeps exactly the rows of keep = data & valid (row ids carried along)
    n = case["n"]
    keep = np.array(case["data"][:n], bool) & np.array(case["valid"][:n], bool)
    n_out, out = pyoracle.filter_compact(keep, {"rid": (np.arange(n, dtype=np.int64), None)})
    assert n_out == sum(case["expected"])
    assert list(np.asarray(out[0][1])[:n_out]) == [i for i, k in enumerate(case["expected"]) if k]


def _rows_sorted(rows):
    return sorted(rows, key=lambda r: tuple((0, "") if x is None else (1, x) for x in r[:1]) +
                  tuple((0, "") if x is None else (1, x) for x in r[1:]))


@pytest.mark.parametrize("case", GOLD["polars_shapes"], ids=lambda c: c["name"])
def test_oracle_polars_shapes_through_the_arrow_layer(case):
    from helpers import arrow_to_oracle_columns, result_columns, shape_table

    table = shape_table(case)
    strings = [n for n, t in case["dtypes"].items() if t == "Utf8"]
    cols, dicts = arrow_to_oracle_columns(table, strings)
    want = case["expected"]
    if "filter" in case:
        keep = pyoracle.filter_mask(cols, case["filter"]) if len(table) else np.zeros(0, bool)
        for name, vals in want.items():
            got = [v for v, k in zip(table.column(name).to_pylist(), keep) if k]
            assert got == vals, name
        return
    keys = case["keys"]
    aggs = [tuple(a) for a in case["aggs"]]
    res = pyoracle.groupby(cols, keys, aggs, case.get("predicate"))
    got = result_columns(res)
    for name, values in dicts.items():
        got[name] = [None if c is None else values[c].as_py() for c in got[name]]
    names = keys + [a[2] for a in aggs]
    got_rows = _rows_sorted(list(zip(*[got[n] for n in names])))
    want_rows = list(zip(*[want[n] for n in names]))
    assert len(got_rows) == len(want_rows)
    for g, w in zip(got_rows, want_rows):
        for x, y in zip(g, w):
            if isinstance(y, float):
                assert math.isclose(x, y, rel_tol=1e-12), (g, w)
            else:
                assert x == y, (g, w)
