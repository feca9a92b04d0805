"""The run-time compiled kernels: generated per query signature and compiled by NVRTC for
sm_100a. NVRTC needs no GPU, so every signature the GPU tests use is compiled here."""

import ctypes as C

import numpy as np
import pytest

from helpers import case_columns, load_golden
from polars_b200 import _abi as A
from polars_b200 import datagen
from polars_b200._native import ColumnData, _to_abi_columns, compile_predicate


def _lib():
    from polars_b200 import build

    L = C.CDLL(str(build.build()))
    L.pmb_debug_jit_compile.argtypes = [C.POINTER(A.Query), C.POINTER(A.Column), C.c_int32, C.c_char_p, C.c_int64]
    return L


def jit_compile(cols: dict, keys, aggs, predicate=None, batch: bool = False, part: bool = False,
                compact: bool = False) -> tuple[int, str]:
    L = _lib()
    names = list(cols)
    cds = [c if isinstance(c, ColumnData) else ColumnData(*c) for c in cols.values()]
    abi, keep = _to_abi_columns(cds)
    idx = {n: i for i, n in enumerate(names)}
    expr, ek = compile_predicate(predicate, idx)
    q = A.Query()
    ka = (C.c_int32 * len(keys))(*[idx[k] for k in keys])
    q.key_columns = ka
    q.n_keys = len(keys)
    ag = (A.Agg * max(1, len(aggs)))()
    for i, (op, col, _) in enumerate(aggs):
        ag[i].op = A.AGG_OPS[op]
        ag[i].column = -1 if op == "Len" else idx[col]
    q.aggs = ag
    q.n_aggs = len(aggs)
    q.predicate = C.pointer(expr) if expr is not None else None
    buf = C.create_string_buffer(1 << 16)
    fn = (L.pmb_debug_jit_compile_compact if compact else L.pmb_debug_jit_compile_part if part
          else L.pmb_debug_jit_compile_batch if batch else L.pmb_debug_jit_compile)
    fn.argtypes = [C.POINTER(A.Query), C.POINTER(A.Column), C.c_int32, C.c_char_p, C.c_int64]
    rc = fn(C.byref(q), abi, len(names), buf, 1 << 16)
    return rc, buf.value.decode(errors="replace")


def nvrtc_available() -> bool:
    try:
        C.CDLL("libnvrtc.so.12")
        return True
    except OSError:
        try:
            C.CDLL("/usr/local/cuda/lib64/libnvrtc.so.12")
            return True
        except OSError:
            return False


pytestmark = pytest.mark.skipif(not nvrtc_available(), reason="NVRTC not installed")


@pytest.mark.parametrize("maker", ["make_small", "make_hash"])
def test_workload_kernels_compile(maker):
    t = getattr(datagen, maker)(4096, seed=1)
    rc, log = jit_compile(datagen.to_column_data(t), t.keys, t.aggs, t.predicate)
    assert rc == 0, log


@pytest.mark.parametrize("case", load_golden()["groupby"], ids=lambda c: c["name"])
def test_golden_signatures_compile(case):
    cols = {n: ColumnData(d, v, dtype=dt, length=n_) for n, (d, v, dt, n_) in case_columns(case).items()}
    rc, log = jit_compile(cols, case["keys"], [tuple(a) for a in case["aggs"]])
    width = sum((1 if c.dtype == A.BOOL else 8 * A.DTYPE_BYTES[c.dtype]) + (c.validity is not None)
                for k, c in cols.items() if k in case["keys"])
    if width > 64:
        assert rc == A.PMB_E_UNSUPPORTED
    else:
        assert rc == 0, log


@pytest.mark.parametrize("vdt", ["int8", "int16", "int32", "int64", "uint8", "uint16", "uint32", "uint64", "float32",
                                 "float64"])
def test_value_dtypes_compile(vdt):
    n = 64
    cols = {"k": ColumnData(np.zeros(n, np.int32)), "v": ColumnData(np.zeros(n, vdt), np.zeros(8, np.uint8))}
    aggs = [("Sum", "v", "s"), ("Mean", "v", "m"), ("Min", "v", "mn"), ("Max", "v", "mx"), ("Count", "v", "c"),
            ("Len", None, "n")]
    rc, log = jit_compile(cols, ["k"], aggs)
    assert rc == 0, log


def test_predicate_forms_compile():
    n = 64
    cols = {"k": ColumnData(np.zeros(n, np.int16)), "x": ColumnData(np.zeros(n), np.zeros(8, np.uint8)),
            "y": ColumnData(np.zeros(n, np.int64), np.zeros(8, np.uint8)),
            "f": ColumnData(np.zeros(8, np.uint8), np.zeros(8, np.uint8), dtype=A.BOOL, length=n)}
    col = lambda c: {"kind": "Column", "name": c}  # noqa: E731
    preds = [
        {"kind": "Or", "lhs": {"kind": "Compare", "op": "Ge", "lhs": col("x"), "rhs": {"kind": "LiteralF64", "value": 1.0}},
         "rhs": col("f")},
        {"kind": "Not", "arg": {"kind": "And", "lhs": col("f"), "rhs": {"kind": "IsNull", "arg": col("y")}}},
        {"kind": "Compare", "op": "Gt", "lhs": {"kind": "Arith", "op": "TrueDiv", "lhs": col("y"), "rhs": col("x")},
         "rhs": {"kind": "LiteralF64", "value": float("nan")}},
        {"kind": "Compare", "op": "Eq", "dtype": "I64",
         "lhs": {"kind": "Arith", "op": "FloorDiv", "lhs": col("y"), "rhs": {"kind": "LiteralI64", "value": -(2 ** 63)}},
         "rhs": {"kind": "LiteralI64", "value": 3}},
        {"kind": "Compare", "op": "Ne", "dtype": "I64",
         "lhs": {"kind": "Arith", "op": "Mod", "lhs": col("y"), "rhs": {"kind": "LiteralI64", "value": -(2 ** 63)}},
         "rhs": {"kind": "LiteralI64", "value": 0}},
        {"kind": "LiteralBool", "value": True},
    ]
    for p in preds:
        rc, log = jit_compile(cols, ["k", "f"], [("Sum", "x", "s"), ("Len", None, "n")], p)
        assert rc == 0, log


def test_batch_kernel_compiles():
    n = 256
    cols = {"key": ColumnData(np.zeros(n, np.int32)), "v": ColumnData(np.zeros(n), np.zeros(32, np.uint8))}
    rc, log = jit_compile(cols, ["key"], datagen.AGGS_BATCH, datagen.PRED_BATCH, batch=True)
    assert rc == 0, log
    t = datagen.make_hash(4096, seed=1)
    rc, log = jit_compile(datagen.to_column_data(t), t.keys, t.aggs, t.predicate, batch=True)
    assert rc == 0, log


@pytest.mark.parametrize("maker", ["make_sort", "make_hash", "make_small"])
def test_partitioned_kernel_compiles(maker):
    # packed sort keys of one and two words; 96-bit table keys (the sort workload) included
    t = getattr(datagen, maker)(4096, seed=1)
    rc, log = jit_compile(datagen.to_column_data(t), t.keys, t.aggs, t.predicate, part=True)
    assert rc == 0, log


def test_partitioned_kernel_value_dtypes_compile():
    n = 64
    cols = {"k": ColumnData(np.zeros(n, np.int64), np.zeros(8, np.uint8)),
            "f": ColumnData(np.zeros(n, np.float32), np.zeros(8, np.uint8)),
            "u": ColumnData(np.zeros(n, np.uint16)),
            "b": ColumnData(np.zeros(8, np.uint8), np.zeros(8, np.uint8), dtype=A.BOOL, length=n)}
    aggs = [("Sum", "f", "s"), ("Mean", "u", "m"), ("Min", "f", "mn"), ("Max", "u", "mx"), ("Count", "b", "c"),
            ("Sum", "b", "sb"), ("Len", None, "n")]
    rc, log = jit_compile(cols, ["k"], aggs, part=True)
    assert rc == 0, log


@pytest.mark.parametrize("maker", ["make_hash", "make_small"])
def test_compaction_kernel_compiles(maker):
    t = getattr(datagen, maker)(1024, seed=1)
    cols = {k: ColumnData(d.numpy(), None if v is None else v.numpy()) for k, (d, v) in t.columns.items()}
    rc, log = jit_compile(cols, t.keys, t.aggs, t.predicate, compact=True)
    assert rc == 0, log


def test_compaction_kernel_all_dtypes_compile():
    # every output dtype (Bool bit-packed, 8- to 64-bit integers, floats), nullable or not, and a
    # predicate over a Bool column and an integer modulo
    rng = np.random.default_rng(3)
    n = 64
    cols = {"k": ColumnData(rng.integers(0, 5, n).astype(np.int32))}
    for i, dt in enumerate([np.int8, np.uint8, np.int16, np.uint16, np.int32, np.uint32, np.int64, np.uint64,
                            np.float32, np.float64]):
        cols[f"c{i}"] = ColumnData(rng.integers(0, 100, n).astype(dt), np.packbits(rng.random(n) > 0.2, bitorder="little"))
    cols["b"] = ColumnData(np.packbits(rng.random(n) > 0.5, bitorder="little"), None, dtype=A.BOOL, length=n)
    pred = {"kind": "And", "lhs": {"kind": "Column", "name": "b"},
            "rhs": {"kind": "Compare", "op": "Ne", "dtype": "I64",
                    "lhs": {"kind": "Arith", "op": "Mod", "lhs": {"kind": "Column", "name": "c6"},
                            "rhs": {"kind": "LiteralI64", "value": 3}},
                    "rhs": {"kind": "LiteralI64", "value": 0}}}
    rc, log = jit_compile(cols, ["k"], [("Len", None, "n")], pred, compact=True)
    assert rc == 0, log
