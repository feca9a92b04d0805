"""ctypes front end of the CPU oracle (oracle/oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline / reference arm, never by the product package. It reuses the product's ABI structs
and predicate lowering (host-side data structures only) so both sides read the same query.
"""

from __future__ import annotations

import ctypes as C
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
sys.path.insert(0, str(ROOT / "polars-metal_b200"))

from polars_b200 import _abi as A  # noqa: E402
from polars_b200._native import compile_predicate  # noqa: E402

LIB = HERE / "liboracle.so"
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            import importlib.util

            spec = importlib.util.spec_from_file_location("_oracle_build", HERE / "build.py")
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            mod.build()
        L = C.CDLL(str(LIB))
        L.orc_last_error.restype = C.c_char_p
        L.orc_groupby.argtypes = [C.POINTER(A.Query), C.POINTER(A.Column), C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]
        L.orc_groupby.restype = C.c_int
        for fn, res in (("orc_result_rows", C.c_int64), ("orc_result_ncols", C.c_int32)):
            getattr(L, fn).argtypes = [C.c_void_p]
            getattr(L, fn).restype = res
        L.orc_result_dtype.argtypes = [C.c_void_p, C.c_int32]
        L.orc_result_dtype.restype = C.c_int32
        for fn in ("orc_result_data", "orc_result_validity"):
            getattr(L, fn).argtypes = [C.c_void_p, C.c_int32]
            getattr(L, fn).restype = C.c_void_p
        for fn in ("orc_result_data_bytes", "orc_result_validity_bytes"):
            getattr(L, fn).argtypes = [C.c_void_p, C.c_int32]
            getattr(L, fn).restype = C.c_int64
        L.orc_result_free.argtypes = [C.c_void_p]
        L.orc_filter_mask.argtypes = [C.POINTER(A.Expr), C.POINTER(A.Column), C.c_int32, C.c_int32, C.c_void_p]
        L.orc_predicate_bits.argtypes = [C.POINTER(A.Expr), C.POINTER(A.Column), C.c_int32, C.c_void_p, C.c_void_p]
        L.orc_bool_logic.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                     C.c_void_p]
        L.orc_filter_compact.argtypes = [C.c_void_p, C.POINTER(A.Column), C.c_int32, C.POINTER(C.c_void_p)]
        L.orc_cumsum_u8_to_u32.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
        L.orc_cumsum_u8_to_u32.restype = None
        _lib = L
    return _lib


def _columns(columns: dict):
    """columns: name -> (data ndarray, validity bitmap ndarray | None[, dtype, length])."""
    names = list(columns)
    arr = (A.Column * max(1, len(names)))()
    keep = []
    for i, n in enumerate(names):
        ent = columns[n]
        data, valid = ent[0], ent[1]
        dt = ent[2] if len(ent) > 2 else {v: k for k, v in A.NUMPY_NAME.items()}[np.asarray(data).dtype.name]
        length = ent[3] if len(ent) > 3 else np.asarray(data).size
        d = np.ascontiguousarray(data)
        keep.append(d)
        arr[i].data = d.ctypes.data if d.size else None
        if valid is not None:
            v = np.ascontiguousarray(valid, dtype=np.uint8)
            keep.append(v)
            arr[i].validity = v.ctypes.data
        else:
            arr[i].validity = None
        arr[i].length = length
        arr[i].offset = 0
        arr[i].dtype = dt
        arr[i].on_device = 0
    return names, arr, keep


def _take_result(r) -> tuple[int, list]:
    L = lib()
    n = L.orc_result_rows(r)
    cols = []
    for c in range(L.orc_result_ncols(r)):
        dt = L.orc_result_dtype(r, c)
        db = L.orc_result_data_bytes(r, c)
        vb = L.orc_result_validity_bytes(r, c)
        raw = C.string_at(L.orc_result_data(r, c), db) if db else b""
        if dt == A.BOOL:
            data = np.frombuffer(raw, np.uint8).copy()
        else:
            data = np.frombuffer(raw, A.NUMPY_NAME[dt]).copy()
        valid = np.frombuffer(C.string_at(L.orc_result_validity(r, c), vb), np.uint8).copy()
        cols.append((dt, data, valid))
    L.orc_result_free(r)
    return n, cols


def groupby(columns: dict, keys, aggs, predicate=None, n_threads: int = 0) -> dict:
    """Oracle group-by. Returns {"n_groups", "names", "dtypes", "data", "validity"}, rows sorted by packed key."""
    L = lib()
    names, arr, keep = _columns(columns)
    index = {n: i for i, n in enumerate(names)}
    key_arr = (C.c_int32 * max(1, len(keys)))(*[index[k] for k in keys])
    agg_arr = (A.Agg * max(1, len(aggs)))()
    for i, (op, col, _a) in enumerate(aggs):
        agg_arr[i].op = A.AGG_OPS[op]
        agg_arr[i].column = -1 if op == "Len" else index[col]
    expr, ekeep = compile_predicate(predicate, index)
    q = A.Query()
    q.key_columns = key_arr
    q.n_keys = len(keys)
    q.aggs = agg_arr
    q.n_aggs = len(aggs)
    q.predicate = C.pointer(expr) if expr is not None else None
    out = C.c_void_p()
    rc = L.orc_groupby(C.byref(q), arr, len(names), n_threads, C.byref(out))
    if rc != 0:
        raise RuntimeError(f"oracle: {L.orc_last_error().decode()} (status {rc})")
    n, cols = _take_result(out)
    del keep, ekeep
    return {
        "n_groups": n,
        "names": list(keys) + [a[2] for a in aggs],
        "dtypes": [c[0] for c in cols],
        "data": [c[1] for c in cols],
        "validity": [c[2] for c in cols],
    }


def filter_mask(columns: dict, predicate, n_threads: int = 0) -> np.ndarray:
    L = lib()
    names, arr, keep = _columns(columns)
    expr, ekeep = compile_predicate(predicate, {n: i for i, n in enumerate(names)})
    n = arr[0].length
    out = np.zeros(max(n, 1), np.uint8)
    rc = L.orc_filter_mask(C.byref(expr), arr, len(names), n_threads, out.ctypes.data)
    if rc != 0:
        raise RuntimeError(L.orc_last_error().decode())
    return out[:n].astype(bool)


def predicate_bits(columns: dict, predicate) -> tuple[np.ndarray, np.ndarray]:
    L = lib()
    names, arr, keep = _columns(columns)
    expr, ekeep = compile_predicate(predicate, {n: i for i, n in enumerate(names)})
    n = arr[0].length
    nb = max(4, (((n + 7) // 8) + 3) & ~3)
    od = np.zeros(nb, np.uint8)
    ov = np.zeros(nb, np.uint8)
    rc = L.orc_predicate_bits(C.byref(expr), arr, len(names), od.ctypes.data, ov.ctypes.data)
    if rc != 0:
        raise RuntimeError(L.orc_last_error().decode())
    return od, ov


def bool_logic(op: str, ld, lv, rd, rv, n: int) -> tuple[np.ndarray, np.ndarray]:
    L = lib()
    nb = max(4, (((n + 7) // 8) + 3) & ~3)
    bufs = [np.ascontiguousarray(np.frombuffer(bytes(x), np.uint8)) if len(x) else np.zeros(1, np.uint8)
            for x in (ld, lv, rd, rv)]
    od = np.zeros(nb, np.uint8)
    ov = np.zeros(nb, np.uint8)
    L.orc_bool_logic(0 if op == "and" else 1, *[b.ctypes.data for b in bufs], n, od.ctypes.data, ov.ctypes.data)
    return od, ov


def filter_compact(keep: np.ndarray, columns: dict) -> tuple[int, list]:
    L = lib()
    names, arr, k = _columns(columns)
    kk = np.ascontiguousarray(keep.astype(np.uint8))
    out = C.c_void_p()
    rc = L.orc_filter_compact(kk.ctypes.data, arr, len(names), C.byref(out))
    if rc != 0:
        raise RuntimeError(L.orc_last_error().decode())
    return _take_result(out)


def cumsum_u8_to_u32(a: np.ndarray) -> np.ndarray:
    L = lib()
    a = np.ascontiguousarray(a, np.uint8)
    out = np.zeros(max(1, a.size), np.uint32)
    L.orc_cumsum_u8_to_u32(a.ctypes.data, out.ctypes.data, a.size)
    return out[: a.size]


def cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1


# ------------------------------------------------------------------------------------ sort
def _order_key(vals: np.ndarray, dt: int) -> np.ndarray:
    """Polars' order of a column's values as uint64 (polars==1.40.1, the version the reference
    pins; its Sort plans call `df.sort(by, descending, nulls_last)`, python/polars_metal/_udf.py:
    684-721): integers by value, False before True, floats with every NaN above +inf and -0.0 equal
    to 0.0."""
    if dt == A.BOOL:
        return vals.astype(np.uint64)
    if vals.dtype.kind == "i":
        return vals.astype(np.int64).view(np.uint64) ^ np.uint64(1 << 63)
    if vals.dtype.kind == "u":
        return vals.astype(np.uint64)
    x = vals.astype(np.float64)  # exact for Float32, and the order is kept
    x = np.where(np.isnan(x), np.float64("nan"), x)
    x = np.where(x == 0, 0.0, x)
    b = x.view(np.uint64)
    neg = (b >> np.uint64(63)).astype(bool)
    return np.where(neg, ~b, b | np.uint64(1 << 63))


def sort_table(columns: dict, by, descending=None, nulls_last=None, drop_nulls: bool = False, offset: int = 0,
               limit: int = -1) -> dict:
    """Oracle sort: the rows of `columns` (name -> (data, validity | None[, dtype, length]), Bool
    data bit-packed) ordered by the `by` columns, most significant first, stably; nulls first
    unless nulls_last, whatever the direction; with drop_nulls the rows whose first `by` column is
    null are left out (top_k / bottom_k); then Polars' slice(offset, limit). Returns the groupby
    result shape, rows in order."""
    names = list(columns)
    cols = []
    for name in names:
        ent = columns[name]
        data, valid = ent[0], ent[1]
        dt = ent[2] if len(ent) > 2 else {v: k for k, v in A.NUMPY_NAME.items()}[np.asarray(data).dtype.name]
        n = ent[3] if len(ent) > 3 else np.asarray(data).size
        vals = (np.unpackbits(np.asarray(data, np.uint8), bitorder="little")[:n].astype(bool) if dt == A.BOOL
                else np.asarray(data)[:n])
        ok = (np.unpackbits(np.asarray(valid, np.uint8), bitorder="little")[:n].astype(bool) if valid is not None
              else np.ones(n, bool))
        cols.append((dt, vals, ok))
    n = len(cols[0][1]) if cols else 0
    desc = list(descending) if descending is not None else [False] * len(by)
    nlast = list(nulls_last) if nulls_last is not None else [False] * len(by)
    rows = np.arange(n)
    if drop_nulls:
        rows = rows[cols[names.index(by[0])][2]]
    keys = []
    for j in reversed(range(len(by))):  # np.lexsort: the last key is the primary one
        dt, vals, ok = cols[names.index(by[j])]
        o = _order_key(vals[rows], dt)
        if desc[j]:
            o = ~o
        keys.append(np.where(ok[rows], o, np.uint64(0)))
        keys.append(~ok[rows] if nlast[j] else ok[rows])
    order = rows[np.lexsort(keys)] if len(rows) else rows
    total = len(order)
    start = min(offset, total) if offset >= 0 else max(0, total + offset)
    stop = total if limit < 0 else min(total, start + limit)
    order = order[start:stop]
    m = len(order)
    out_data, out_valid, dts = [], [], []
    for dt, vals, ok in cols:
        v = vals[order]
        out_data.append(np.packbits(v, bitorder="little") if dt == A.BOOL else v)
        out_valid.append(np.packbits(ok[order], bitorder="little") if m else np.zeros(1, np.uint8))
        dts.append(dt)
    return {"n_groups": m, "names": names, "dtypes": dts, "data": out_data, "validity": out_valid}
