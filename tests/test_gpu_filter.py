"""GPU parity of the filter-side operator surface (compare, Kleene AND/OR, compaction, cumsum)."""

import numpy as np
import pytest

from helpers import load_golden, pack, unpack
from oracle import pyoracle
from polars_b200 import _abi as A
from polars_b200 import _native as N
from polars_b200._native import ColumnData

pytestmark = pytest.mark.gpu
GOLD = load_golden()


@pytest.mark.parametrize("case", GOLD["compare"], ids=lambda c: c["name"])
def test_compare_known_answers(case):
    n = len(case["lhs"])
    lhs = np.array(case["lhs"], np.float64).tobytes()
    lv = pack(case["lhs_valid"]).tobytes()
    if "rhs" in case:
        d, v = N.cmp_f64_col_col(lhs, lv, np.array(case["rhs"], np.float64).tobytes(), pack(case["rhs_valid"]).tobytes(),
                                 case["op"], n)
    else:
        d, v = N.cmp_f64_col_scalar(lhs, lv, case["scalar"], case["op"], n)
    assert list(unpack(np.frombuffer(d, np.uint8), n).astype(int)) == case["expected_data"]
    assert list(unpack(np.frombuffer(v, np.uint8), n).astype(int)) == case["expected_valid"]
    assert len(d) == max(4, ((n + 7) // 8 + 3) & ~3)


@pytest.mark.parametrize("n", [0, 1, 13, 4096, 100_003])
@pytest.mark.parametrize("op", ["Eq", "Ne", "Lt", "Le", "Gt", "Ge"])
def test_compare_random_vs_oracle(n, op):
    rng = np.random.default_rng(n + len(op))
    a = rng.integers(-5, 5, n).astype(np.int64)
    b = rng.integers(-5, 5, n).astype(np.int64)
    va, vb = rng.random(n) > 0.2, rng.random(n) > 0.2
    pa, pb = pack(va).tobytes() if n else b"\0", pack(vb).tobytes() if n else b"\0"
    d, v = N.cmp_i64_col_col(a.tobytes(), pa, b.tobytes(), pb, op, n)
    if n:
        pred = {"kind": "Compare", "op": op, "dtype": "I64", "lhs": {"kind": "Column", "name": "a"},
                "rhs": {"kind": "Column", "name": "b"}}
        od, ov = pyoracle.predicate_bits({"a": (a, pack(va)), "b": (b, pack(vb))}, pred)
        assert np.array_equal(unpack(np.frombuffer(d, np.uint8), n), unpack(od, n))
        assert np.array_equal(unpack(np.frombuffer(v, np.uint8), n), unpack(ov, n))
        ds, vs = N.cmp_i64_col_scalar(a.tobytes(), pa, 2, op, n)
        pred["rhs"] = {"kind": "LiteralI64", "value": 2}
        od, ov = pyoracle.predicate_bits({"a": (a, pack(va))}, pred)
        assert np.array_equal(unpack(np.frombuffer(ds, np.uint8), n), unpack(od, n))


def test_kleene_truth_tables():
    case = GOLD["kleene"][0]
    n = len(case["lhs"])
    enc = lambda vals: (pack([x == "T" for x in vals]).tobytes(), pack([x != "N" for x in vals]).tobytes())  # noqa
    ld, lv = enc(case["lhs"])
    rd, rv = enc(case["rhs"])
    for op, fn in (("and", N.bool_and_dispatch), ("or", N.bool_or_dispatch)):
        d, v = fn(ld, lv, rd, rv, n)
        dd, vv = unpack(np.frombuffer(d, np.uint8), n), unpack(np.frombuffer(v, np.uint8), n)
        got = ["N" if not vv[i] else ("T" if dd[i] else "F") for i in range(n)]
        assert got == case[op], op


@pytest.mark.parametrize("n", [0, 5, 2048, 2049, 1_000_001])
def test_filter_compact_vs_oracle(n):
    rng = np.random.default_rng(n)
    keep = rng.random(n) > 0.4
    pvalid = rng.random(n) > 0.1
    cols_np = {
        "a": (rng.integers(-1000, 1000, n).astype(np.int64), pack(rng.random(n) > 0.1)),
        "b": (rng.standard_normal(n), None),
        "c": (rng.integers(0, 255, n).astype(np.uint8), pack(rng.random(n) > 0.3)),
        "d": (pack(rng.random(n) > 0.5), pack(rng.random(n) > 0.2), A.BOOL, n),
    }
    wire = []
    for name, ent in cols_np.items():
        data, valid = ent[0], ent[1]
        tag = "Bool" if len(ent) > 2 else {"int64": "I64", "float64": "F64", "uint8": "U8"}[data.dtype.name]
        vb = valid.tobytes() if valid is not None else b"\xff" * max(1, (n + 7) // 8)
        wire.append((tag, data.tobytes(), vb))
    pd = pack(keep).tobytes() if n else b"\0"
    pv = pack(pvalid).tobytes() if n else b"\0"
    out = N.execute_filter_compact(pd, pv, n, wire)
    m, want = pyoracle.filter_compact(keep & pvalid, {k: v for k, v in cols_np.items()})
    assert all(o[2] == m for o in out)
    for (db, vb, _), (dt, wd, wv) in zip(out, want):
        assert np.array_equal(unpack(np.frombuffer(vb, np.uint8), m), unpack(wv, m))
        if dt == A.BOOL:
            assert np.array_equal(unpack(np.frombuffer(db, np.uint8), m), unpack(wd, m))
        else:
            assert np.frombuffer(db, wd.dtype)[:m].tobytes() == wd[:m].tobytes()


def test_filter_compact_expr_matches_groupby_filter():
    rng = np.random.default_rng(1)
    n = 300_000
    x = rng.standard_normal(n)
    y = rng.integers(0, 100, n).astype(np.int64)
    pred = {"kind": "And", "lhs": {"kind": "Compare", "op": "Gt", "lhs": {"kind": "Column", "name": "x"},
                                    "rhs": {"kind": "LiteralF64", "value": -0.5}},
            "rhs": {"kind": "Compare", "op": "Ne", "dtype": "I64",
                    "lhs": {"kind": "Arith", "op": "Mod", "lhs": {"kind": "Column", "name": "y"},
                            "rhs": {"kind": "LiteralI64", "value": 7}}, "rhs": {"kind": "LiteralI64", "value": 0}}}
    keep = pyoracle.filter_mask({"x": (x, None), "y": (y, None)}, pred)
    import ctypes as C

    h = N.default_handle()
    cols = [ColumnData(x), ColumnData(y)]
    abi, k = N._to_abi_columns(cols)
    expr, ek = N.compile_predicate(pred, {"x": 0, "y": 1})
    res_p = C.POINTER(A.Result)()
    h.check(h._lib.pmb_filter_compact_expr(h.raw, C.byref(expr), abi, 2, 0, C.byref(res_p)))
    try:
        r = res_p.contents
        assert r.n_groups == keep.sum()
        got = np.frombuffer(C.string_at(r.columns[0].data, 8 * r.n_groups), np.float64)
        assert np.array_equal(got, x[keep])
    finally:
        h._lib.pmb_result_free(res_p)


@pytest.mark.parametrize("n", [0, 1, 4095, 4096, 4097, 10_000_019])
def test_cumsum_u8_to_u32(n):
    rng = np.random.default_rng(n)
    a = rng.integers(0, 256, n).astype(np.uint8)
    got = N.cumsum_u8_to_u32(a)
    assert np.array_equal(got, pyoracle.cumsum_u8_to_u32(a))


@pytest.mark.parametrize("n", [2_097_152, 3_000_017])
def test_filter_columns_run_time_compiled_vs_oracle(n):
    # above 2^21 rows the predicate path compiles its compaction at run time: every output dtype,
    # nullable and not, a Bool column in the predicate, rows not a multiple of the tile
    rng = np.random.default_rng(n)
    cols_np = {
        "i8": (rng.integers(-100, 100, n).astype(np.int8), pack(rng.random(n) > 0.1)),
        "u16": (rng.integers(0, 60000, n).astype(np.uint16), None),
        "i32": (rng.integers(-2**31, 2**31, n).astype(np.int32), pack(rng.random(n) > 0.05)),
        "u64": (rng.integers(0, 2**63, n).astype(np.uint64), None),
        "f32": (rng.standard_normal(n).astype(np.float32), pack(rng.random(n) > 0.2)),
        "x": (rng.standard_normal(n), pack(rng.random(n) > 0.05)),
        "y": (rng.integers(-10**9, 10**9, n).astype(np.int64), pack(rng.random(n) > 0.05)),
        "b": (pack(rng.random(n) > 0.3), pack(rng.random(n) > 0.1), A.BOOL, n),
    }
    pred = {"kind": "And",
            "lhs": {"kind": "Or", "lhs": {"kind": "Column", "name": "b"},
                    "rhs": {"kind": "Compare", "op": "Gt", "lhs": {"kind": "Column", "name": "x"},
                            "rhs": {"kind": "LiteralF64", "value": 0.5}}},
            "rhs": {"kind": "Compare", "op": "Ne", "dtype": "I64",
                    "lhs": {"kind": "Arith", "op": "Mod", "lhs": {"kind": "Column", "name": "y"},
                            "rhs": {"kind": "LiteralI64", "value": 7}}, "rhs": {"kind": "LiteralI64", "value": 0}}}
    keep = pyoracle.filter_mask(cols_np, pred)
    m, want = pyoracle.filter_compact(keep, cols_np)
    got = N.filter_columns({k: ColumnData(*v) for k, v in cols_np.items()}, pred)
    assert got.n_groups == m == keep.sum()
    for j, (dt, wd, wv) in enumerate(want):
        assert np.array_equal(unpack(np.asarray(got.validity[j], np.uint8), m), unpack(wv, m)), got.names[j]
        if dt == A.BOOL:
            assert np.array_equal(unpack(np.asarray(got.data[j], np.uint8), m), unpack(wd, m))
        else:
            assert np.asarray(got.data[j])[:m].tobytes() == wd[:m].tobytes(), got.names[j]
