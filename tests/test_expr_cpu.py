"""Expression aggregates without a GPU: the reference's aggregation-expression wire (Column,
LiteralI64, LiteralF64, Binary with Add/Sub/Mul/Div) becomes the arithmetic nodes libpmb
evaluates, bad trees are refused, and the Arrow path hands over the columns an expression reads."""

import pytest

from polars_b200._native import _arith_wire


def col(name):
    return {"kind": "Column", "name": name}


def test_binary_nodes_become_arith_nodes():
    e = {"kind": "Binary", "op": "Div", "lhs": {"kind": "Binary", "op": "Mul", "lhs": col("a"), "rhs": col("b")},
         "rhs": {"kind": "LiteralF64", "value": 2.5}}
    w = _arith_wire(e)
    assert w == {"kind": "Arith", "op": "TrueDiv",
                 "lhs": {"kind": "Arith", "op": "Mul", "lhs": col("a"), "rhs": col("b")},
                 "rhs": {"kind": "LiteralF64", "value": 2.5}}
    assert _arith_wire(w) == w  # Arith nodes pass through
    assert _arith_wire(col("x")) == col("x")


@pytest.mark.parametrize("bad", [
    {"kind": "Binary", "op": "Pow", "lhs": col("a"), "rhs": col("b")},
    {"kind": "Compare", "op": "Gt", "lhs": col("a"), "rhs": col("b")},
    {"kind": "Binary", "op": "Add", "lhs": col("a"), "rhs": 3},
    "a",
])
def test_bad_expressions_are_refused(bad):
    with pytest.raises(ValueError, match="plan parse error"):
        _arith_wire(bad)


def test_arrow_path_hands_over_expression_columns(monkeypatch):
    pa = pytest.importorskip("pyarrow")
    from polars_b200 import arrow

    seen = {}

    def fake_groupby(cols, keys, aggs, predicate, **kw):
        seen["cols"] = sorted(cols)
        raise RuntimeError("stop")

    monkeypatch.setattr(arrow, "groupby", fake_groupby)
    t = pa.table({"k": [1, 2], "a": [1.0, 2.0], "b": [3, 4], "unused": [0, 0]})
    with pytest.raises(RuntimeError, match="stop"):
        arrow.groupby_arrow(t, ["k"], [("Sum", {"kind": "Arith", "op": "Mul", "lhs": col("a"), "rhs": col("b")}, "s")])
    assert seen["cols"] == ["a", "b", "k"]


@pytest.mark.parametrize("case", __import__("helpers").load_golden()["expression"], ids=lambda c: c["name"])
def test_oracle_pinned_to_the_reference_expression_cases(case):
    # the expression evaluated row by row in numpy, then the oracle's group-by sum of it
    import math

    from helpers import expression_columns, numpy_expr
    from oracle import pyoracle

    cols = expression_columns(case["formula"], case["n"])
    agg = case["aggs"][0]
    x = numpy_expr(agg["expr"], cols)
    res = pyoracle.groupby({"k": cols["k"], "x": (x, None)}, ["k"], [("Sum", "x", agg["output_alias"])])
    order = sorted(range(res["n_groups"]), key=lambda i: res["data"][0][i])
    assert [int(res["data"][0][i]) for i in order] == case["expected"]["k"]
    got = [float(res["data"][1][i]) for i in order]
    want = case["expected"][agg["output_alias"]]
    assert all(math.isclose(g, w, rel_tol=1e-12) for g, w in zip(got, want)), (got, want)


def _c(dtype, n=4):
    import numpy as np

    return np.zeros(n, dtype)


def _bin(op, lhs, rhs):
    return {"kind": "Arith", "op": op, "lhs": lhs, "rhs": rhs}


@pytest.mark.parametrize("a,b,op,want", [
    ("int32", "int32", "Mul", "I32"), ("int32", "float64", "Mul", "F64"), ("float32", "float32", "Mul", "F32"),
    ("float32", "int16", "Add", "F32"), ("float32", "int32", "Add", "F64"), ("int8", "uint8", "Add", "I16"),
    ("int32", "uint32", "Sub", "I64"), ("int64", "uint64", "Add", "F64"), ("uint16", "uint8", "Add", "U16"),
    ("int64", "int32", "TrueDiv", "F64"), ("float32", "float32", "TrueDiv", "F32"), ("int32", "int32", "FloorDiv", "I32"),
    ("uint64", "uint32", "Mod", "U64"),
])
def test_expression_types_follow_polars(a, b, op, want):
    from polars_b200 import _abi as A
    from polars_b200._native import expr_dtype

    got = expr_dtype({"a": _c(a), "b": _c(b)}, _bin(op, col("a"), col("b")))
    assert got == A.TAG_TO_DTYPE[want]


def test_literals_take_the_other_operands_type():
    from polars_b200 import _abi as A
    from polars_b200._native import expr_dtype

    cols = {"u": _c("uint16"), "f": _c("float32"), "i": _c("int32")}
    lit_i = {"kind": "LiteralI64", "value": 7}
    lit_f = {"kind": "LiteralF64", "value": 1.5}
    assert expr_dtype(cols, _bin("Sub", col("u"), lit_i)) == A.U16
    assert expr_dtype(cols, _bin("Mul", col("f"), lit_f)) == A.F32
    assert expr_dtype(cols, _bin("Mul", col("i"), lit_f)) == A.F64
    assert expr_dtype(cols, _bin("Mul", _bin("Add", lit_i, lit_i), col("i"))) == A.I32
    assert expr_dtype(cols, _bin("TrueDiv", col("i"), lit_i)) == A.F64
    assert expr_dtype(cols, _bin("Add", lit_i, lit_i)) == A.I32
    # the reference's Q1 shape over Float32 columns stays Float32
    assert expr_dtype(cols, _bin("Mul", col("f"), _bin("Sub", lit_f, col("f")))) == A.F32


def test_bool_columns_and_deep_trees_are_refused():
    import numpy as np

    from polars_b200 import _abi as A
    from polars_b200._native import ColumnData, expr_dtype

    b = ColumnData(np.zeros(1, np.uint8), None, dtype=A.BOOL, length=4)
    with pytest.raises(ValueError):
        expr_dtype({"b": b, "i": _c("int32")}, _bin("Add", col("b"), col("i")))
    e = col("i")
    for _ in range(9):
        e = _bin("Add", e, {"kind": "LiteralI64", "value": 1})
    with pytest.raises(ValueError):
        expr_dtype({"i": _c("int32")}, e)


@pytest.mark.parametrize("dtype,value,want", [
    # an integer literal widens its operand's type to hold its value (Polars' dynamic integers)
    ("uint8", -1, "I16"), ("uint8", 255, "U8"), ("uint8", 256, "U16"), ("int8", 1000, "I16"), ("int8", 127, "I8"),
    ("int8", -129, "I16"), ("uint16", -1, "I32"), ("int16", 40_000, "I32"), ("uint32", -1, "I64"),
    ("int32", 2**31, "I64"), ("uint32", 2**32, "U64"), ("uint64", -1, "I64"), ("int64", -(2**40), "I64"),
    ("float32", 10**9, "F32"), ("int32", 7, "I32"),
])
def test_integer_literals_widen_to_hold_their_value(dtype, value, want):
    from polars_b200 import _abi as A
    from polars_b200._native import expr_dtype

    lit = {"kind": "LiteralI64", "value": value}
    got = expr_dtype({"c": _c(dtype)}, _bin("Mul", col("c"), lit))
    assert got == A.TAG_TO_DTYPE[want], (dtype, value)
    assert expr_dtype({"c": _c(dtype)}, _bin("Add", lit, col("c"))) == A.TAG_TO_DTYPE[want]


def test_literal_only_subtrees_fold_before_typing():
    from polars_b200 import _abi as A
    from polars_b200._native import expr_dtype

    big = {"kind": "LiteralI64", "value": 3_000_000_000}
    one = {"kind": "LiteralI64", "value": 1}
    cols = {"u": _c("uint8"), "i": _c("int32")}
    assert expr_dtype(cols, _bin("Add", big, one)) == A.I64  # beyond Int32: Int64, not a wrapped Int32
    assert expr_dtype(cols, _bin("Add", one, one)) == A.I32
    # (300 - 1) beside a UInt8 column needs UInt16
    assert expr_dtype(cols, _bin("Mul", col("u"), _bin("Sub", {"kind": "LiteralI64", "value": 300}, one))) == A.U16
    # (0 - 1) beside a UInt8 column is negative: Int16
    assert expr_dtype(cols, _bin("Mul", col("u"), _bin("Sub", {"kind": "LiteralI64", "value": 0}, one))) == A.I16
