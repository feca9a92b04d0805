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
