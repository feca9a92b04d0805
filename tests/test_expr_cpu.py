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
