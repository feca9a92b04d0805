"""Shared test helpers: golden-case inputs, result canonicalisation and comparison rules.

Comparison rules (the parity bar):
  - keys, counts, integer sums and integer / float min / max: bit-exact (NaN == NaN; -0.0 and
    +0.0 are treated as equal, since the reference leaves the sign of a zero min / max to row order);
  - float64 sums and means: |gpu - oracle| <= 1e-12 * |oracle| + 1e-15 (FP64 compensated-sum oracle);
  - float32 sums and means: within 1 float32 ulp of the oracle (its float64 result rounded to float32).
Rows are sorted by the key columns (nulls first) before comparison.
"""

from __future__ import annotations

import json
import math
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "polars-metal_b200"))
sys.path.insert(0, str(ROOT))

from polars_b200 import _abi as A  # noqa: E402

GOLDEN = ROOT / "tests" / "golden" / "reference_cases.json"

F64_RTOL = 1e-12
F32_ULPS = 1  # float32 sums and means: ulps from the oracle's float64 result rounded to float32
F64_ATOL = 1e-15


def load_golden() -> dict:
    return json.loads(GOLDEN.read_text())


def pack(mask) -> np.ndarray:
    m = np.asarray(mask, dtype=bool)
    return np.packbits(m, bitorder="little") if m.size else np.zeros(1, np.uint8)


def unpack(bitmap, n) -> np.ndarray:
    if n == 0:
        return np.zeros(0, bool)
    return np.unpackbits(np.asarray(bitmap, np.uint8), bitorder="little")[:n].astype(bool)


def case_columns(case: dict) -> dict:
    """Golden case columns -> {name: (data, validity bitmap | None, dtype, length)}."""
    out = {}
    for name, c in case["columns"].items():
        dt = A.TAG_TO_DTYPE[c["dtype"]]
        vals = c["values"]
        n = len(vals)
        if dt == A.BOOL:
            data = pack([bool(v) for v in vals])
        else:
            data = np.array([float("nan") if v is None else v for v in vals], dtype=A.NUMPY_NAME[dt])
        valid = pack([bool(v) for v in c["valid"]]) if "valid" in c else None
        out[name] = (data, valid, dt, n)
    return out


def formula_columns(formula: str, n: int) -> dict:
    """Closed-form inputs of tests/python_integration/test_groupby.py (see make_reference_cases.py)."""
    i = np.arange(n, dtype=np.int64)
    ones = None
    if formula == "single_i64_key_sum":
        return {"k": (i % 7, ones), "v": (i.copy(), ones)}
    if formula == "all_aggs":
        return {"k": (i % 5, ones), "v": ((i % 100).astype(np.float64), ones)}
    if formula == "two_bool_keys":
        return {"returnflag": (pack(i % 2 == 1), ones, A.BOOL, n), "linestatus": (pack((i // 2) % 2 == 1), ones, A.BOOL, n),
                "qty": (i.copy(), ones)}
    if formula == "bool_plus_i64":
        return {"category": (pack(i % 2 == 1), ones, A.BOOL, n), "subkey": (i % 13, ones), "v": (i.astype(np.float64), ones)}
    if formula == "null_key":
        k = np.where(i % 3 != 0, 1, 0).astype(np.int64)
        return {"k": (k, pack(i % 3 != 0)), "v": (i.copy(), ones)}
    if formula == "null_values":
        return {"k": (i % 4, ones), "v": (i.astype(np.float64), pack(i % 5 != 0))}
    if formula == "all_unique":
        return {"k": (i.copy(), ones), "v": (np.ones(n, np.int64), ones)}
    if formula == "all_same":
        return {"k": (np.full(n, 7, np.int64), ones), "v": (i.copy(), ones)}
    if formula == "i32_i32":
        return {"k": ((i % 7).astype(np.int32), ones), "v": ((i % 100).astype(np.int32), ones)}
    if formula == "f32_values":
        return {"k": ((i % 5).astype(np.int32), ones), "v": ((i % 100).astype(np.float32), ones)}
    raise KeyError(formula)


def expression_columns(formula: str, n: int) -> dict:
    """Closed-form inputs of tests/python_integration/test_walker_expression_unfolding.py (see
    make_reference_cases.py): the test's short lists repeated to n rows."""
    def rep(vals, dtype):
        v = np.array(vals, dtype=dtype)
        return np.tile(v, n // len(v))
    if formula == "sum_a_times_b":
        return {"k": (rep([0, 0, 1, 1, 2, 2], np.int64), None), "a": (rep([1.0, 2.0, 3.0, 4.0, 5.0, 6.0], np.float64), None),
                "b": (rep([0.1, 0.2, 0.3, 0.4, 0.5, 0.6], np.float64), None)}
    if formula == "sum_a_times_one_minus_b":
        return {"k": (rep([0, 0, 1, 1], np.int64), None), "a": (rep([10.0, 20.0, 30.0, 40.0], np.float64), None),
                "b": (rep([0.05, 0.1, 0.15, 0.2], np.float64), None)}
    if formula == "depth_5_chain":
        return {"k": (np.zeros(n, np.int64), None), "v": (np.ones(n, np.float64), None)}
    raise KeyError(formula)


def numpy_expr(e: dict, cols: dict) -> np.ndarray:
    """An aggregation expression (reference wire shape) evaluated row by row in numpy, f64."""
    kind = e["kind"]
    if kind == "Column":
        return cols[e["name"]][0].astype(np.float64)
    if kind in ("LiteralF64", "LiteralI64"):
        return np.float64(e["value"])
    lhs, rhs = numpy_expr(e["lhs"], cols), numpy_expr(e["rhs"], cols)
    return {"Add": np.add, "Sub": np.subtract, "Mul": np.multiply, "Div": np.divide}[e["op"]](lhs, rhs)


def _values(dt: int, data: np.ndarray, n: int) -> np.ndarray:
    if dt == A.BOOL:
        return unpack(data, n)
    return np.asarray(data)[:n]


def canonical(res: dict, n_keys: int) -> dict:
    """Result dict (n_groups, names, dtypes, data, validity) -> sorted {name: (values, valid)}."""
    n = int(res["n_groups"])
    cols = []
    for dt, d, v in zip(res["dtypes"], res["data"], res["validity"]):
        cols.append((_values(dt, d, n), unpack(v, n)))
    sort_keys = []
    for j in reversed(range(n_keys)):
        vals, valid = cols[j]
        vv = np.where(valid, vals, np.zeros_like(vals)) if vals.dtype != bool else (vals & valid)
        if vv.dtype.kind == "f":  # float keys group by bit pattern (-0.0 and +0.0 are distinct groups)
            vv = vv.view(np.int32 if vv.dtype == np.float32 else np.int64)
        sort_keys.append(vv)
        sort_keys.append(valid)
    order = np.lexsort(sort_keys) if n_keys and n else np.arange(n)
    return {name: (vals[order], valid[order]) for name, (vals, valid) in zip(res["names"], cols)}


def as_dict(r) -> dict:
    """GroupByResult (product) -> plain result dict."""
    return {"n_groups": r.n_groups, "names": r.names, "dtypes": r.dtypes, "data": r.data, "validity": r.validity}


def f32_ulps(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    ia = a.astype(np.float32).view(np.int32).astype(np.int64)
    ib = b.astype(np.float32).view(np.int32).astype(np.int64)
    ia = np.where(ia < 0, -(ia & 0x7FFFFFFF), ia)
    ib = np.where(ib < 0, -(ib & 0x7FFFFFFF), ib)
    return np.abs(ia - ib)


def assert_results_match(got: dict, want: dict, n_keys: int, aggs: list, label: str = "") -> None:
    """Compares two result dicts under the parity rules above."""
    assert int(got["n_groups"]) == int(want["n_groups"]), f"{label}: n_groups {got['n_groups']} != {want['n_groups']}"
    assert list(got["dtypes"]) == list(want["dtypes"]), f"{label}: dtypes {got['dtypes']} != {want['dtypes']}"
    g = canonical(got, n_keys)
    w = canonical(want, n_keys)
    ops = [None] * n_keys + [a[0] for a in aggs]
    for idx, name in enumerate(want["names"]):
        gv, gval = g[name]
        wv, wval = w[name]
        assert np.array_equal(gval, wval), f"{label}: validity of {name} differs at {np.nonzero(gval != wval)[0][:5]}"
        gv = gv[wval]
        wv = wv[wval]
        op = ops[idx]
        if gv.dtype.kind == "f" and op in ("Sum", "Mean"):
            if gv.dtype == np.float32:
                u = f32_ulps(gv, wv)
                bad = np.nonzero((u > F32_ULPS) & ~(np.isnan(gv) & np.isnan(wv)))[0]
                assert bad.size == 0, f"{label}: {name} f32 off by {u[bad[:5]]} ulps at {bad[:5]}: {gv[bad[:5]]} vs {wv[bad[:5]]}"
            else:
                same = (gv == wv) | (np.isnan(gv) & np.isnan(wv))
                with np.errstate(invalid="ignore"):
                    diff = np.abs(gv - wv)
                    close = diff <= F64_RTOL * np.abs(wv) + F64_ATOL
                bad = np.nonzero(~same & ~close)[0]
                assert bad.size == 0, (f"{label}: {name} differs beyond 1e-12 rel at {bad[:5]}: "
                                       f"{gv[bad[:5]]} vs {wv[bad[:5]]}")
        elif gv.dtype.kind == "f":
            same = (gv == wv) | (np.isnan(gv) & np.isnan(wv))
            bad = np.nonzero(~same)[0]
            assert bad.size == 0, f"{label}: {name} differs at {bad[:5]}: {gv[bad[:5]]} vs {wv[bad[:5]]}"
        else:
            bad = np.nonzero(gv != wv)[0]
            assert bad.size == 0, f"{label}: {name} differs at {bad[:5]}: {gv[bad[:5]]} vs {wv[bad[:5]]}"


def expected_to_result(case: dict) -> dict:
    """Golden expected table -> result dict (rows given in key order)."""
    names = list(case["keys"]) + [a[2] for a in case["aggs"]]
    n = len(case["expected"][names[0]])
    data, valid, dtypes = [], [], []
    for name in names:
        dt = A.TAG_TO_DTYPE[case["dtypes"][name]]
        vals = case["expected"][name]
        mask = [v is not None for v in vals]
        if dt == A.BOOL:
            d = pack([bool(v) if v is not None else False for v in vals])
        else:
            d = np.array([v if v is not None else 0 for v in vals], dtype=A.NUMPY_NAME[dt])
        data.append(d)
        valid.append(pack(mask))
        dtypes.append(dt)
    return {"n_groups": n, "names": names, "dtypes": dtypes, "data": data, "validity": valid}


def compact_case_inputs(case: dict):
    """A compaction golden case -> (columns {name: (data, validity | None, dtype, n)}, keep data
    bits, keep validity bits, n); `keep_mod3` is the closed form of the 10k-row case."""
    if case.get("formula") == "keep_mod3":
        n = case["n"]
        r = np.arange(n)
        return {"a": (r.astype(np.int64), None, A.I64, n)}, list((r % 3 == 0).astype(int)), [1] * n, n
    cols = case_columns(case)
    n = len(case["pred_data"])
    return cols, case["pred_data"], case["pred_valid"], n


def compact_case_expected(case: dict) -> dict:
    if case.get("formula") == "keep_mod3":
        return {"a": list(range(0, case["n"], 3))}
    return case["expected"]


def same_values(got: list, want: list) -> bool:
    """Element-wise equality with NaN equal to NaN."""
    if len(got) != len(want):
        return False
    for g, w in zip(got, want):
        if isinstance(w, float) and math.isnan(w):
            if not (isinstance(g, float) and math.isnan(g)):
                return False
        elif g != w:
            return False
    return True


_PA_TYPES = {"Int8": "int8", "Int16": "int16", "Int32": "int32", "Int64": "int64", "UInt8": "uint8", "UInt16": "uint16",
             "UInt32": "uint32", "UInt64": "uint64", "Float32": "float32", "Float64": "float64", "Bool": "bool_",
             "Utf8": "string"}


def _gen_column(spec):
    if isinstance(spec, list):
        return spec
    g = spec["gen"]
    if g == "mod":
        return [i % spec["m"] for i in range(spec["n"])]
    if g == "scale":
        return [i * spec["c"] for i in range(spec["n"])]
    if g == "tile":
        return spec["values"] * spec["times"]
    raise KeyError(g)


def shape_table(case: dict):
    """The pyarrow table of a polars_shapes golden case, with its chunks."""
    import pyarrow as pa

    names = list(case["dtypes"])
    types = {n: getattr(pa, _PA_TYPES[case["dtypes"][n]])() for n in names}
    chunks = {n: [] for n in names}
    for ch in case["chunks"]:
        cols = {n: _gen_column(ch[n]) for n in names}
        rows = case.get("chunk_rows") or max(1, len(cols[names[0]]))
        total = len(cols[names[0]])
        for start in range(0, max(total, 1), rows):
            for n in names:
                chunks[n].append(pa.array(cols[n][start:start + rows], type=types[n]))
    return pa.table({n: pa.chunked_array(chunks[n], type=types[n]) for n in names})


def arrow_to_oracle_columns(table, dict_columns=()):
    """Oracle inputs of an Arrow table: numeric columns as (values, validity bitmap | None), Bool
    columns bit-packed, and the named string columns as dictionary codes from pyarrow's own
    `dictionary_encode` (first-appearance order), independent of the product's encoder: the oracle
    groups by the codes and the caller decodes them through the dictionary. Returns (columns,
    dictionaries)."""
    import pyarrow as pa

    cols, dicts = {}, {}
    for name in table.column_names:
        col = table.column(name)
        if name in dict_columns:
            flat = col.combine_chunks() if col.num_chunks else pa.array([], type=col.type)
            enc = flat.dictionary_encode()
            dicts[name] = enc.dictionary
            arr = enc.indices
        else:
            arr = col.combine_chunks() if col.num_chunks else pa.array([], type=col.type)
        n = len(arr)
        ok = ~np.asarray(arr.is_null().to_numpy(zero_copy_only=False), bool) if n else np.zeros(0, bool)
        valid = pack(ok) if arr.null_count else None
        if pa.types.is_boolean(arr.type):
            vals = np.asarray(arr.fill_null(False).to_numpy(zero_copy_only=False), bool)
            cols[name] = (pack(vals), valid, A.BOOL, n)
        else:
            np_type = np.dtype(arr.type.to_pandas_dtype())
            vals = np.asarray(arr.fill_null(0).to_numpy(zero_copy_only=False)).astype(np_type) if n else np.zeros(0, np_type)
            cols[name] = (vals, valid, {v: k for k, v in A.NUMPY_NAME.items()}[np_type.name], n)
    return cols, dicts


def result_columns(res: dict) -> dict:
    """Result dict -> {name: list of Python values, None for null}."""
    n = int(res["n_groups"])
    out = {}
    for name, dt, d, v in zip(res["names"], res["dtypes"], res["data"], res["validity"]):
        vals = unpack(d, n) if dt == A.BOOL else np.asarray(d)[:n]
        ok = unpack(v, n)
        out[name] = [vals[i].item() if ok[i] else None for i in range(n)]
    return out
