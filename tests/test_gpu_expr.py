"""Expression aggregates (sum(a * b), max(c - 7), mean(c / a), min(c // a)) on the GPU against the
CPU oracle run over the same expressions computed in numpy, through groupby and through the
reference's wire (`execute_groupby` with an "Expression" aggregate)."""

import numpy as np
import pytest

from helpers import as_dict, assert_results_match, pack
from oracle import pyoracle
from polars_b200 import _abi as A
from polars_b200 import _native as N

pytestmark = pytest.mark.gpu


def col(name):
    return {"kind": "Column", "name": name}


def _case(n=300_000, seed=13):
    rng = np.random.default_rng(seed)
    k = rng.integers(0, 2_000, n).astype(np.int64)
    a = rng.integers(-5, 6, n).astype(np.int32)
    av = rng.random(n) > 0.05
    b = rng.standard_normal(n)
    bv = rng.random(n) > 0.1
    c = rng.integers(-10**6, 10**6, n).astype(np.int64)
    return k, a, av, b, bv, c


def _expected_columns(k, a, av, b, bv, c):
    with np.errstate(divide="ignore", invalid="ignore"):
        ab = a.astype(np.float64) * b                    # int * float -> Float64
        cm7 = c - 7                                      # Int64
        cda = c.astype(np.float64) / a                   # true division -> Float64 (x / 0 = +-inf or nan)
        safe = np.where(a == 0, 1, a).astype(np.int64)
        cfa = np.floor_divide(c, safe)                   # floor division; // 0 is null
    return {"k": (k, None), "ab": (ab, pack(av & bv)), "cm7": (cm7, None), "cda": (cda, pack(av)),
            "cfa": (cfa, pack(av & (a != 0)))}


EXPRS = {
    "ab": {"kind": "Arith", "op": "Mul", "lhs": col("a"), "rhs": col("b")},
    "cm7": {"kind": "Arith", "op": "Sub", "lhs": col("c"), "rhs": {"kind": "LiteralI64", "value": 7}},
    "cda": {"kind": "Arith", "op": "TrueDiv", "lhs": col("c"), "rhs": col("a")},
    "cfa": {"kind": "Arith", "op": "FloorDiv", "lhs": col("c"), "rhs": col("a")},
}
OPS = [("Sum", "ab", "s_ab"), ("Max", "cm7", "mx_c"), ("Mean", "cda", "m_cda"), ("Min", "cfa", "mn_cfa"),
       ("Len", None, "n")]


def test_expression_aggregates_match_the_oracle():
    k, a, av, b, bv, c = _case()
    cols = {"k": N.ColumnData(k), "a": N.ColumnData(a, pack(av)), "b": N.ColumnData(b, pack(bv)),
            "c": N.ColumnData(c)}
    aggs = [(op, EXPRS[e] if e else None, alias) for op, e, alias in OPS]
    got = N.groupby(cols, ["k"], aggs)
    want = pyoracle.groupby(_expected_columns(k, a, av, b, bv, c), ["k"], OPS)
    assert_results_match(as_dict(got), want, 1, OPS, "expression aggregates")


def test_eval_expr_column_twice_in_a_row():
    import torch

    k, a, av, b, bv, c = _case(n=70_001, seed=5)
    cols = {"a": N.ColumnData(torch.from_numpy(a).cuda(), torch.from_numpy(pack(av)).cuda()),
            "b": N.ColumnData(torch.from_numpy(b).cuda(), torch.from_numpy(pack(bv)).cuda())}
    want = _expected_columns(k, a, av, b, bv, c)["ab"]
    for _ in range(2):
        out = N.eval_expr(cols, {"kind": "Binary", "op": "Mul", "lhs": col("a"), "rhs": col("b")})
        assert out.dtype == A.F64 and out.data.is_cuda
        v = np.unpackbits(out.validity.cpu().numpy(), bitorder="little")[: len(a)].astype(bool)
        assert np.array_equal(v, av & bv)
        assert np.array_equal(out.data.cpu().numpy()[: len(a)][v], want[0][v])


def test_expression_aggregates_on_the_reference_wire():
    k, a, av, b, bv, c = _case(n=50_000, seed=8)
    ones = lambda n: b"\xff" * ((n + 7) // 8)  # noqa: E731
    columns = [("k", "I64", k.tobytes(), ones(len(k))), ("a", "I32", a.tobytes(), pack(av).tobytes()),
               ("b", "F64", b.tobytes(), pack(bv).tobytes()), ("c", "I64", c.tobytes(), ones(len(c)))]
    plan = {"keys": [["k", "I64"]],
            "aggs": [{"kind": "Expression", "op": "Sum", "output_alias": "s_ab",
                      "expr": {"kind": "Binary", "op": "Mul", "lhs": col("a"), "rhs": col("b")}},
                     {"kind": "Expression", "op": "Max", "output_alias": "mx_c",
                      "expr": {"kind": "Binary", "op": "Sub", "lhs": col("c"),
                               "rhs": {"kind": "LiteralI64", "value": 7}}},
                     {"kind": "Length", "output_alias": "n"}]}
    out = N.execute_groupby(plan, len(k), columns)
    assert [o[0] for o in out] == ["k", "s_ab", "mx_c", "n"]
    ops = [("Sum", "ab", "s_ab"), ("Max", "cm7", "mx_c"), ("Len", None, "n")]
    want = pyoracle.groupby({kk: v for kk, v in _expected_columns(k, a, av, b, bv, c).items()
                             if kk in ("k", "ab", "cm7")}, ["k"], ops)
    n = len(np.frombuffer(out[0][2], np.int64))
    dts = [A.TAG_TO_DTYPE[o[1]] for o in out]
    assert dts[:3] == [A.I64, A.F64, A.I64]
    got = {"n_groups": n, "names": [o[0] for o in out], "dtypes": dts,
           "data": [np.frombuffer(o[2], A.NUMPY_NAME[dt]) for o, dt in zip(out, dts)],
           "validity": [np.frombuffer(o[3], np.uint8) for o in out]}
    assert_results_match(got, want, 1, ops, "wire expression aggregates")


@pytest.mark.parametrize("case", __import__("helpers").load_golden()["expression"], ids=lambda c: c["name"])
def test_reference_expression_cases_through_the_wire(case):
    import math

    from helpers import expression_columns

    cols = expression_columns(case["formula"], case["n"])
    n = case["n"]
    ones = b"\xff" * ((n + 7) // 8)
    tags = {np.dtype(np.int64): "I64", np.dtype(np.float64): "F64"}
    columns = [(name, tags[d.dtype], d.tobytes(), ones) for name, (d, _v) in cols.items()]
    plan = {"keys": [["k", "I64"]], "aggs": case["aggs"]}
    out = N.execute_groupby(plan, n, columns)
    k = np.frombuffer(out[0][2], np.int64)
    s = np.frombuffer(out[1][2], np.float64)
    order = np.argsort(k)
    assert k[order].tolist() == case["expected"]["k"]
    want = case["expected"][case["aggs"][0]["output_alias"]]
    assert all(math.isclose(g, w, rel_tol=1e-12) for g, w in zip(s[order].tolist(), want)), (s[order], want)


def _bin(op, lhs, rhs):
    return {"kind": "Arith", "op": op, "lhs": lhs, "rhs": rhs}


def test_polars_types_wrap_and_round_on_the_gpu():
    # 32-bit integer products wrap, Float32 arithmetic rounds at every node, a UInt16 minus a
    # literal wraps: as numpy (and Polars) compute them in those types
    rng = np.random.default_rng(31)
    n = 100_003
    a = rng.integers(-2**31, 2**31, n).astype(np.int32)
    b = rng.integers(-2**31, 2**31, n).astype(np.int32)
    fa = rng.standard_normal(n).astype(np.float32)
    fb = rng.standard_normal(n).astype(np.float32)
    u = rng.integers(0, 20, n).astype(np.uint16)
    s = rng.integers(-300, 300, n).astype(np.int16)
    cols = {"a": a, "b": b, "fa": fa, "fb": fb, "u": u, "s": s}
    lit = {"kind": "LiteralF64", "value": 1.5}
    seven = {"kind": "LiteralI64", "value": 7}
    cases = [
        (_bin("Mul", col("a"), col("b")), A.I32, a * b),
        (_bin("Mul", col("fa"), col("fb")), A.F32, fa * fb),
        (_bin("Mul", col("fa"), _bin("Sub", lit, col("fb"))), A.F32, fa * (np.float32(1.5) - fb)),
        (_bin("Sub", col("u"), seven), A.U16, u - np.uint16(7)),
        (_bin("Mul", col("s"), col("fa")), A.F32, s.astype(np.float32) * fa),
    ]
    for e, dt, want in cases:
        out = N.eval_expr(cols, e)
        assert out.dtype == dt
        got = np.asarray(out.data)[:n]
        assert got.dtype == want.dtype and np.array_equal(got, want), e
        assert np.unpackbits(np.asarray(out.validity), bitorder="little")[:n].all()


def test_integer_literals_beyond_the_column_type_widen_on_the_gpu():
    # UInt8 * -1 is Int16 (not a wrapped UInt8), Int8 + 1000 is Int16, UInt32 * -1 is Int64,
    # UInt32 - 5_000_000_000 is UInt64 (a non-negative literal beside an unsigned column stays
    # unsigned, and the difference wraps), the folded literal 3e9 + 1 is UInt32 beside UInt8 and
    # Int64 beside Int8: Polars' dynamic-integer rule
    rng = np.random.default_rng(37)
    n = 50_001
    u8 = rng.integers(0, 256, n).astype(np.uint8)
    i8 = rng.integers(-128, 128, n).astype(np.int8)
    u32 = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    cols = {"u8": u8, "i8": i8, "u32": u32}
    lit = lambda v: {"kind": "LiteralI64", "value": v}  # noqa: E731
    cases = [
        (_bin("Mul", col("u8"), lit(-1)), A.I16, u8.astype(np.int16) * np.int16(-1)),
        (_bin("Add", col("i8"), lit(1000)), A.I16, i8.astype(np.int16) + np.int16(1000)),
        (_bin("Mul", col("u32"), lit(-1)), A.I64, u32.astype(np.int64) * np.int64(-1)),
        (_bin("Sub", col("u32"), lit(5_000_000_000)), A.U64, u32.astype(np.uint64) - np.uint64(5_000_000_000)),
        (_bin("Mul", col("u8"), _bin("Add", lit(3_000_000_000), lit(1))), A.U32,
         u8.astype(np.uint32) * np.uint32(3_000_000_001)),
        (_bin("Mul", col("i8"), _bin("Add", lit(3_000_000_000), lit(1))), A.I64,
         i8.astype(np.int64) * np.int64(3_000_000_001)),
    ]
    for e, dt, want in cases:
        out = N.eval_expr(cols, e)
        assert out.dtype == dt, e
        got = np.asarray(out.data)[:n]
        assert got.dtype == want.dtype and np.array_equal(got, want), e


def test_reference_fused_float32_sum_of_products():
    # crates/polars-metal-kernels/tests/test_dispatch_groupby_fused.rs:185-260: sum(a * b) per
    # i % 4 over Float32 columns a = i * 0.1, b = i * 0.05 + 1, 6000 rows
    n = 6000
    i = np.arange(n)
    k = (i % 4).astype(np.int32)
    fa = (i.astype(np.float32) * np.float32(0.1)).astype(np.float32)
    fb = (i.astype(np.float32) * np.float32(0.05) + np.float32(1.0)).astype(np.float32)
    got = N.groupby({"k": k, "a": fa, "b": fb}, ["k"], [("Sum", _bin("Mul", col("a"), col("b")), "sum_ab")])
    want = pyoracle.groupby({"k": (k, None), "ab": (fa * fb, None)}, ["k"], [("Sum", "ab", "sum_ab")])
    assert got.dtypes[1] == A.F32
    assert_results_match(as_dict(got), want, 1, [("Sum", "ab", "sum_ab")], "f32 sum of products")
