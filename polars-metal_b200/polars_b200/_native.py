"""Python surface of libpmb, mirroring the reference's PyO3 `_native` module for this path.

Reference functions mirrored (same names, argument meaning and error classes):
  - execute_groupby(plan_dict, n_rows, columns)      crates/polars-metal-core/src/udf/groupby/mod.rs:747-1144
  - cmp_{i64,f64}_col_{col,scalar}(...)               crates/polars-metal-core/src/udf/compare.rs:23-145
  - bool_and_dispatch / bool_or_dispatch(...)          crates/polars-metal-core/src/udf/logical.rs:26-55
  - execute_filter_compact(pred_data, pred_valid, n_rows, columns)
                                                       crates/polars-metal-core/src/udf/compact.rs:46-147
Errors: ValueError (parse / length), KeyError (missing column), NotImplementedError (outside
this build), MemoryError, RuntimeError (device failures; the reference's ComputeError).

Also on the reference's wire: execute_sort(plan, n_rows, columns) for a Sort plan over a
GroupBy (python/polars_metal/_udf.py:684-721), and Expression aggregates inside execute_groupby
(crates/polars-metal-core/src/udf/groupby/mod.rs:266-352).

Beyond the wire-format functions, `groupby()` takes numpy arrays or CUDA tensors directly
(zero-copy for device-resident columns; `sort=` orders the result on the device), and so do
`sort_columns` / `top_k` / `bottom_k`, `filter_columns`, `eval_expr` and `groupby_batched`.
Host results of 1 MB or more are numpy arrays over the library's own buffers (no copy). `Handle`
exposes streams and per-kernel timings.
"""

from __future__ import annotations

import ctypes as C
import threading
import weakref
from dataclasses import dataclass, field
from collections.abc import Sequence
from typing import Any

import numpy as np

from . import _abi as A

_ERRORS = {
    A.PMB_E_INVALID: ValueError,
    A.PMB_E_OOM: MemoryError,
    A.PMB_E_TIMEOUT: RuntimeError,
    A.PMB_E_CUDA: RuntimeError,
    A.PMB_E_UNSUPPORTED: NotImplementedError,
    A.PMB_E_NOT_FOUND: KeyError,
}


class Handle:
    """One device context: a CUDA stream plus a growable device workspace (libpmb handle).

    selector: "default" installs the strategy-selector parameters shipped with the package (when
    present), None leaves the AUTO strategy to the plain cardinality heuristic, or a float array
    of SELECTOR_PARAMS parameters."""

    def __init__(self, device: int = 0, workspace_bytes: int = 0, selector: Any = "default"):
        self._lib = A.lib()
        self._h = C.c_void_p()
        rc = self._lib.pmb_open(C.byref(self._h), device, workspace_bytes)
        if rc != A.PMB_OK:
            raise _ERRORS.get(rc, RuntimeError)(f"polars_b200: pmb_open failed with status {rc}")
        self.device = device
        if isinstance(selector, str) and selector == "default":
            from .selector import default_params

            selector = default_params()
        if selector is not None:
            self.set_selector(selector)

    def set_selector(self, params: Any) -> None:
        """Installs MLP parameters for the AUTO strategy (None: the cardinality heuristic)."""
        if params is None:
            self.check(self._lib.pmb_selector_set(self._h, None, 0))
            return
        p = np.ascontiguousarray(np.asarray(params, dtype=np.float32).ravel())
        self.check(self._lib.pmb_selector_set(self._h, p.ctypes.data, p.size))

    @property
    def raw(self) -> C.c_void_p:
        return self._h

    def close(self) -> None:
        if self._h:
            self._lib.pmb_close(self._h)
            self._h = C.c_void_p()

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc: int) -> None:
        if rc != A.PMB_OK:
            msg = self._lib.pmb_last_error(self._h).decode(errors="replace")
            raise _ERRORS.get(rc, RuntimeError)(f"polars_b200: {msg}")

    def set_stream(self, cuda_stream: int | None) -> None:
        self.check(self._lib.pmb_set_stream(self._h, C.c_void_p(cuda_stream or 0)))

    def set_profiling(self, on: bool) -> None:
        self.check(self._lib.pmb_set_profiling(self._h, 1 if on else 0))

    def set_batching(self, on: bool) -> None:
        """False: groupby_batched runs each query alone through pmb_groupby, looped inside the
        library (host outputs only); True (default): it batches where it can."""
        self.check(self._lib.pmb_set_batching(self._h, 1 if on else 0))

    def last_stats(self) -> dict:
        s = A.Stats()
        self.check(self._lib.pmb_last_stats(self._h, C.byref(s)))
        kernels = {}
        for i in range(s.n_kernels):
            kernels[s.names[i].value.decode()] = {"launches": s.launches[i], "ms": s.ms[i]}
        return {
            "kernels": kernels,
            "total_ms": s.total_ms,
            "h2d_bytes": s.h2d_bytes,
            "d2h_bytes": s.d2h_bytes,
            "kernel_launches": s.kernel_launches,
        }


_local = threading.local()


def default_handle() -> Handle:
    h = getattr(_local, "handle", None)
    if h is None:
        h = Handle(0)
        _local.handle = h
    return h


# ------------------------------------------------------------------------------- column inputs
@dataclass
class ColumnData:
    """An Arrow-layout column: values plus an optional LSB-first validity bitmap.

    `data` / `validity` are numpy arrays (host) or CUDA torch tensors (device, zero-copy).
    Bool columns are bit-packed uint8 (LSB first). `length` defaults to len(data)."""

    data: Any
    validity: Any = None
    dtype: int | None = None
    length: int | None = None
    offset: int = 0

    def __post_init__(self):
        if self.dtype is None:
            self.dtype = _infer_dtype(self.data)
        if self.length is None:
            if self.dtype == A.BOOL:
                raise ValueError("Bool columns need an explicit length")
            self.length = int(_nelem(self.data)) - self.offset


_TORCH_TYPES: dict[type, bool] = {}


def _is_torch(x) -> bool:
    t = type(x)
    r = _TORCH_TYPES.get(t)
    if r is None:
        r = _TORCH_TYPES[t] = t.__module__.startswith("torch")
    return r


def _nelem(x) -> int:
    return int(x.numel()) if _is_torch(x) else int(np.asarray(x).size)


def _infer_dtype(x) -> int:
    if _is_torch(x):
        name = str(x.dtype).replace("torch.", "")
    else:
        name = np.asarray(x).dtype.name
    table = {v: k for k, v in A.NUMPY_NAME.items()}
    if name == "bool":
        raise ValueError("pass Bool columns bit-packed with dtype=BOOL")
    if name not in table:
        raise NotImplementedError(f"polars_b200: unsupported dtype {name}")
    return table[name]


def _ptr(x) -> tuple[int, int, Any]:
    """(address, on_device, keepalive) of a numpy array or torch tensor."""
    if x is None:
        return 0, 0, None
    if _is_torch(x):
        if not x.is_contiguous():
            x = x.contiguous()
        return int(x.data_ptr()), 1 if x.is_cuda else 0, x
    arr = np.ascontiguousarray(x)
    return int(arr.ctypes.data), 0, arr


def _to_abi_columns(cols: Sequence[ColumnData]):
    arr = (A.Column * max(1, len(cols)))()
    keep = []
    for i, c in enumerate(cols):
        dp, dd, k1 = _ptr(c.data)
        vp, vd, k2 = _ptr(c.validity)
        if c.validity is not None and vd != dd:
            raise ValueError("data and validity of a column must live in the same memory space")
        arr[i].data = dp
        arr[i].validity = vp if c.validity is not None else None
        arr[i].length = c.length
        arr[i].offset = c.offset
        arr[i].dtype = c.dtype
        arr[i].on_device = dd
        keep += [k1, k2]
    return arr, keep


# ------------------------------------------------------------------------------- predicates
def compile_predicate(pred: dict | None, col_index: dict[str, int]):
    """Lowers a predicate dict (the walker's PredicateAst wire shape, python/polars_metal/_walker.py:1508-1644,
    plus "Arith", "Not", "IsNull", "IsNotNull") into expression nodes."""
    if pred is None:
        return None, None
    nodes: list[A.ExprNode] = []

    def add(**kw) -> int:
        n = A.ExprNode()
        n.lhs = n.rhs = -1
        for k, v in kw.items():
            setattr(n, k, v)
        nodes.append(n)
        return len(nodes) - 1

    def dtype_of(tag):
        if tag is None:
            return 0
        if tag not in ("I64", "F64"):
            raise ValueError(f"polars_b200: operand dtype must be I64 or F64, got {tag!r}")
        return A.TAG_TO_DTYPE[tag]

    def walk(p: dict) -> int:
        kind = p.get("kind")
        if kind == "Column":
            name = p["name"]
            if name not in col_index:
                raise KeyError(f"polars_b200: predicate column {name!r} not found in upstream columns")
            return add(kind=A.EXPR_COLUMN, column=col_index[name])
        if kind == "LiteralI64":
            return add(kind=A.EXPR_LIT_I64, lit_i64=int(p["value"]), dtype=A.I64)
        if kind == "LiteralF64":
            return add(kind=A.EXPR_LIT_F64, lit_f64=float(p["value"]), dtype=A.F64)
        if kind == "LiteralBool":
            return add(kind=A.EXPR_LIT_BOOL, lit_i64=1 if p["value"] else 0)
        if kind == "Compare":
            if p["op"] not in A.CMP_OPS:
                raise ValueError(f"polars_b200: unknown compare op {p['op']!r}")
            l, r = walk(p["lhs"]), walk(p["rhs"])
            return add(kind=A.EXPR_COMPARE, op=A.CMP_OPS[p["op"]], lhs=l, rhs=r, dtype=dtype_of(p.get("dtype")))
        if kind in ("And", "Or"):
            l, r = walk(p["lhs"]), walk(p["rhs"])
            return add(kind=A.EXPR_AND if kind == "And" else A.EXPR_OR, lhs=l, rhs=r)
        if kind == "Not":
            return add(kind=A.EXPR_NOT, lhs=walk(p["arg"]))
        if kind in ("IsNull", "IsNotNull"):
            return add(kind=A.EXPR_IS_NULL if kind == "IsNull" else A.EXPR_IS_NOT_NULL, lhs=walk(p["arg"]))
        if kind == "Arith":
            if p["op"] not in A.ARITH_OPS:
                raise ValueError(f"polars_b200: unknown arithmetic op {p['op']!r}")
            l, r = walk(p["lhs"]), walk(p["rhs"])
            return add(kind=A.EXPR_ARITH, op=A.ARITH_OPS[p["op"]], lhs=l, rhs=r, dtype=dtype_of(p.get("dtype")))
        raise ValueError(f"polars_b200: unknown predicate node kind {kind!r}")

    root = walk(pred)
    arr = (A.ExprNode * len(nodes))(*nodes)
    expr = A.Expr(C.cast(arr, C.POINTER(A.ExprNode)), len(nodes), root)
    return expr, arr


# ------------------------------------------------------------------------------- group-by
@dataclass
class GroupByResult:
    n_groups: int
    names: list[str]
    dtypes: list[int]
    data: list[Any]  # numpy arrays (host) or device addresses (int) when output_on_device
    validity: list[Any]
    strategy: str
    rehash_count: int
    capacity: int
    stats: dict = field(default_factory=dict)

    def column(self, name: str) -> tuple[np.ndarray, np.ndarray]:
        i = self.names.index(name)
        return self.data[i], self.validity[i]


def _bitmap_bytes(n: int) -> int:
    b = (n + 7) // 8
    b = (b + 3) & ~3
    return max(b, 4)


def _host_copy(addr: int, nbytes: int, dtype) -> np.ndarray:
    """A numpy copy of `nbytes` of host memory at `addr` (one copy)."""
    return np.frombuffer((C.c_char * nbytes).from_address(addr), dtype=dtype).copy()


_TAKE_MIN = 1 << 20  # host result buffers of at least this size are taken over instead of copied


def _host_take(addr: int, nbytes: int, dtype) -> np.ndarray:
    """A numpy array over a host buffer of a result, without a copy: the array owns the buffer,
    which goes back to libpmb (pmb_host_buffer_free: its pinned pool, or free) when the last view
    of it is collected."""
    buf = (C.c_char * nbytes).from_address(addr)
    weakref.finalize(buf, A.lib().pmb_host_buffer_free, addr)
    return np.frombuffer(buf, dtype=dtype)


def _host_out(oc: A.OutColumn, field: str, nbytes: int, dtype, empty: int) -> np.ndarray:
    """One host buffer of a result column: large buffers change owner (the column's pointer is
    cleared, so pmb_result_free leaves it), small ones are copied."""
    addr = getattr(oc, field)
    if not addr or nbytes == 0:
        return np.zeros(empty, dtype)
    if nbytes >= _TAKE_MIN:
        arr = _host_take(addr, nbytes, dtype)
        setattr(oc, field, None)
        return arr
    return _host_copy(addr, nbytes, dtype)


def _read_result(res: A.Result, names, to_host: bool) -> tuple[list, list, list]:
    n = res.n_groups
    data, valid, dts = [], [], []
    for i in range(res.n_columns):
        oc = res.columns[i]
        dts.append(oc.dtype)
        if not to_host:
            data.append(int(oc.data or 0))
            valid.append(int(oc.validity or 0))
            continue
        vb = _bitmap_bytes(n)
        v = _host_out(oc, "validity", vb, np.uint8, vb)
        if oc.dtype == A.BOOL:
            d = _host_out(oc, "data", vb, np.uint8, vb)
        else:
            d = _host_out(oc, "data", n * A.DTYPE_BYTES[oc.dtype], A.NUMPY_NAME[oc.dtype], 0)
        data.append(d)
        valid.append(v)
    return data, valid, dts


_AGG_BINARY_OPS = {"Add": "Add", "Sub": "Sub", "Mul": "Mul", "Div": "TrueDiv"}


def _arith_wire(e: dict) -> dict:
    """An aggregation expression in the reference's wire shape (Column / LiteralF64 / LiteralI64 /
    Binary with Add, Sub, Mul, Div; crates/polars-metal-core/src/udf/groupby/mod.rs:266-352) as
    the arithmetic nodes of the predicate wire; "Arith" nodes pass through."""
    if not isinstance(e, dict):
        raise ValueError("polars_b200: plan parse error: wrong type for expr")
    kind = e.get("kind")
    if kind in ("Column", "LiteralI64", "LiteralF64"):
        return e
    if kind in ("Binary", "Arith"):
        op = _AGG_BINARY_OPS.get(e.get("op")) if kind == "Binary" else e.get("op")
        if op is None or op not in A.ARITH_OPS:
            raise ValueError(f"polars_b200: plan parse error: unknown op binary op {e.get('op')}")
        return {"kind": "Arith", "op": op, "lhs": _arith_wire(e.get("lhs")), "rhs": _arith_wire(e.get("rhs"))}
    raise ValueError(f"polars_b200: plan parse error: unknown op expr kind={kind}")


def expr_dtype(columns: dict[str, ColumnData | Any], expr: dict) -> int:
    """The dtype eval_expr gives `expr` over these columns (pmb_expr_dtype; no GPU work)."""
    names = list(columns)
    cols = [c if isinstance(c, ColumnData) else ColumnData(c) for c in columns.values()]
    abi, keep = _to_abi_columns(cols)
    e, ek = compile_predicate(_arith_wire(expr), {nm: i for i, nm in enumerate(names)})
    dt = C.c_int32()
    if A.lib().pmb_expr_dtype(C.byref(e), abi, len(cols), C.byref(dt)) != A.PMB_OK:
        raise ValueError("polars_b200: not an arithmetic expression of these columns")
    del keep, ek
    return dt.value


def eval_expr(columns: dict[str, ColumnData | Any], expr: dict, handle: Handle | None = None) -> ColumnData:
    """An arithmetic expression of the columns, evaluated on the GPU for every row (pmb_eval_expr),
    typed as Polars types it (operands cast to their supertype, literals take the other side's
    type, integer true division gives Float64; 32-bit results wrap or round as Polars' do); null
    where an operand is null or an integer // or % divides by zero. The new column is a CUDA tensor
    when an input column is one, else a numpy array."""
    h = handle or default_handle()
    names = list(columns)
    if not names:
        raise ValueError("polars_b200: eval_expr needs columns")
    cols = [c if isinstance(c, ColumnData) else ColumnData(c) for c in columns.values()]
    abi, keep = _to_abi_columns(cols)
    e, ek = compile_predicate(_arith_wire(expr), {nm: i for i, nm in enumerate(names)})
    n = cols[0].length
    dev = next((c.data.device for c in cols if _is_torch(c.data) and c.data.is_cuda), None)
    if dev is not None:
        import torch

        data = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
        valid = torch.zeros(_bitmap_bytes(n), dtype=torch.uint8, device=dev)
        dp, vp = data.data_ptr(), valid.data_ptr()
    else:
        data = np.empty(max(n, 1), np.int64)
        valid = np.zeros(_bitmap_bytes(n), np.uint8)
        dp, vp = data.ctypes.data, valid.ctypes.data
    dt = C.c_int32()
    h.check(h._lib.pmb_eval_expr(h.raw, C.byref(e), abi, len(cols), dp, vp, 1 if dev is not None else 0, C.byref(dt)))
    del keep, ek
    if dev is not None:
        data = data.view(getattr(torch, A.NUMPY_NAME[dt.value]))
    else:
        data = data.view(A.NUMPY_NAME[dt.value])
    return ColumnData(data, valid, dtype=dt.value, length=n)


def groupby(
    columns: dict[str, ColumnData | Any],
    keys: Sequence[str],
    aggs: Sequence[tuple[str, str | None, str]],
    predicate: dict | None = None,
    strategy: str = "auto",
    output: str = "host",
    capacity_hint: int = 0,
    handle: Handle | None = None,
    sort: dict | None = None,
) -> GroupByResult:
    """filter -> group_by -> aggregate through libpmb.

    columns: name -> ColumnData (or a bare array with no nulls); aggs: (op, input column, alias)
    with op in Sum/Mean/Count/Min/Max/Len (input None for Len), the input may also be an
    arithmetic expression dict (an expression aggregate, evaluated by eval_expr); predicate: a
    predicate dict; sort: the result sorted on the device in the same call (pmb_groupby_sorted),
    {"by": output column name(s), "descending", "nulls_last" (a flag or one per column),
    "drop_nulls", "offset", "limit"} as sort_columns takes them.
    """
    if any(isinstance(a[1], dict) for a in aggs):
        # expression aggregates: every expression is evaluated into a column of its own first
        columns = dict(columns)
        plain = []
        for i, (op, col, alias) in enumerate(aggs):
            if isinstance(col, dict):
                name = f"__expr{i}"
                while name in columns:
                    name += "_"
                columns[name] = eval_expr(columns, col, handle=handle)
                col = name
            plain.append((op, col, alias))
        aggs = plain
    names = list(columns)
    index = {n: i for i, n in enumerate(names)}
    cols = [c if isinstance(c, ColumnData) else ColumnData(c) for c in columns.values()]
    for k in keys:
        if k not in index:
            raise KeyError(f"polars_b200: key column {k!r} not found in upstream columns")
    key_arr = (C.c_int32 * max(1, len(keys)))(*[index[k] for k in keys])
    agg_arr = (A.Agg * max(1, len(aggs)))()
    for i, (op, col, _alias) in enumerate(aggs):
        if op not in A.AGG_OPS:
            raise ValueError(f"polars_b200: unknown aggregation op {op!r}")
        agg_arr[i].op = A.AGG_OPS[op]
        if op == "Len":
            agg_arr[i].column = -1
        else:
            if col not in index:
                raise KeyError(f"polars_b200: agg input column {col!r} not found in upstream columns")
            agg_arr[i].column = index[col]
    expr, expr_keep = compile_predicate(predicate, index)
    q = A.Query()
    q.key_columns = key_arr
    q.n_keys = len(keys)
    q.aggs = agg_arr
    q.n_aggs = len(aggs)
    q.predicate = C.pointer(expr) if expr is not None else None
    if strategy not in A.STRATEGIES:
        raise ValueError(f"polars_b200: unknown strategy {strategy!r}")
    q.strategy = A.STRATEGIES[strategy]
    q.output_on_device = 1 if output == "device" else 0
    q.capacity_hint = capacity_hint
    h = handle or default_handle()
    abi_cols, keep = _to_abi_columns(cols)
    res_p = C.POINTER(A.Result)()
    out_names = list(keys) + [a[2] for a in aggs]
    if sort is not None:
        spec, spec_keep = _sort_spec(out_names, **sort)
        h.check(h._lib.pmb_groupby_sorted(h.raw, C.byref(q), abi_cols, len(cols), C.byref(spec), C.byref(res_p)))
        del spec_keep
    else:
        h.check(h._lib.pmb_groupby(h.raw, C.byref(q), abi_cols, len(cols), C.byref(res_p)))
    try:
        res = res_p.contents
        data, valid, dts = _read_result(res, out_names, output != "device")
        return GroupByResult(
            n_groups=res.n_groups,
            names=out_names,
            dtypes=dts,
            data=data,
            validity=valid,
            strategy=A.STRATEGY_NAMES.get(res.strategy_used, str(res.strategy_used)),
            rehash_count=res.rehash_count,
            capacity=res.capacity,
        )
    finally:
        h._lib.pmb_result_free(res_p)
        del keep, expr_keep


def _query(columns, keys, aggs, predicate):
    names = list(columns)
    index = {n: i for i, n in enumerate(names)}
    cols = [c if isinstance(c, ColumnData) else ColumnData(c) for c in columns.values()]
    for k in keys:
        if k not in index:
            raise KeyError(f"polars_b200: key column {k!r} not found in upstream columns")
    key_arr = (C.c_int32 * max(1, len(keys)))(*[index[k] for k in keys])
    agg_arr = (A.Agg * max(1, len(aggs)))()
    for i, (op, col, _alias) in enumerate(aggs):
        if op not in A.AGG_OPS:
            raise ValueError(f"polars_b200: unknown aggregation op {op!r}")
        agg_arr[i].op = A.AGG_OPS[op]
        if op == "Len":
            agg_arr[i].column = -1
        else:
            if col not in index:
                raise KeyError(f"polars_b200: agg input column {col!r} not found in upstream columns")
            agg_arr[i].column = index[col]
    expr, expr_keep = compile_predicate(predicate, index)
    q = A.Query()
    q.key_columns = key_arr
    q.n_keys = len(keys)
    q.aggs = agg_arr
    q.n_aggs = len(aggs)
    q.predicate = C.pointer(expr) if expr is not None else None
    abi_cols, keep = _to_abi_columns(cols)
    return q, abi_cols, len(cols), (keep, expr_keep, key_arr, agg_arr, expr)


def _np_struct(S) -> np.dtype:
    """numpy dtype with the layout of a ctypes structure (pointers as 64-bit addresses)."""
    names, formats, offsets = [], [], []
    for name, t in S._fields_:
        names.append(name)
        offsets.append(getattr(S, name).offset)
        is_ptr = t is C.c_void_p or (isinstance(t, type) and issubclass(t, C._Pointer))
        formats.append("<u8" if is_ptr else np.dtype(t).str)
    return np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": C.sizeof(S)})


_COLUMN_NP = _np_struct(A.Column)
_QUERY_NP = _np_struct(A.Query)
# groupby_batched reads results as 64-bit words: n_groups | n_columns | columns | strategy_used,
# rehash_count | capacity, and every output column as data | validity | length | dtype, on_device
assert [A.Result.n_groups.offset, A.Result.n_columns.offset, A.Result.columns.offset, A.Result.strategy_used.offset,
        A.Result.rehash_count.offset, A.Result.capacity.offset, C.sizeof(A.Result)] == [0, 8, 16, 24, 28, 32, 40]
assert [A.OutColumn.data.offset, A.OutColumn.validity.offset, A.OutColumn.dtype.offset, C.sizeof(A.OutColumn)] == \
    [0, 8, 24, 32]


def _batch_args(queries, output: str):
    """The C arguments of pmb_groupby_batched: query structs, one pointer per query to its column
    structs, the column counts, plus what must stay alive during the call and the output names.
    Queries usually share keys, aggregates and filter: those parts are built once per shape, and
    the per-query structs are filled as numpy records."""
    n = len(queries)
    shapes = {}
    qrec = np.zeros(max(1, n), dtype=_QUERY_NP)
    ncols = np.zeros(max(1, n), dtype=np.int32)
    counts = [len(q[0]) for q in queries]
    crec = np.zeros(max(1, sum(counts)), dtype=_COLUMN_NP)
    first = np.zeros(max(1, n), dtype=np.uint64)
    keep, names, fields, qrows = [], [], [], []
    on_dev = 1 if output == "device" else 0
    ci = 0
    for i, (columns, keys, aggs, predicate) in enumerate(queries):
        key = (tuple(columns), tuple(keys), tuple(aggs), id(predicate))
        sh = shapes.get(key)
        if sh is None:
            parts = _query_shape(list(columns), keys, aggs, predicate)
            key_arr, nk, agg_arr, na, expr, _ek = parts
            sh = ((C.addressof(key_arr), nk, C.addressof(agg_arr), na, C.addressof(expr) if expr is not None else 0,
                   A.STRATEGIES["auto"], on_dev, 0), list(keys) + [a[2] for a in aggs], parts, predicate)
            shapes[key] = sh
            keep.append(sh)
        qrows.append(sh[0])
        names.append(sh[1])
        first[i] = ci
        for c in columns.values():
            cd = c if isinstance(c, ColumnData) else ColumnData(c)
            dp, dd, k1 = _ptr(cd.data)
            vp, vd, k2 = _ptr(cd.validity)
            if cd.validity is not None and vd != dd:
                raise ValueError("data and validity of a column must live in the same memory space")
            fields.append((dp, vp, cd.length, cd.offset, cd.dtype, dd))
            keep.append((k1, k2))
            ci += 1
    if qrows:
        qrec[:n] = qrows
        ncols[:n] = counts
    if fields:
        crec[: len(fields)] = fields
    ptrs = (first * np.uint64(_COLUMN_NP.itemsize) + np.uint64(crec.ctypes.data)).astype(np.uint64)
    keep += [qrec, crec, ptrs, ncols]
    return qrec, ptrs, ncols, keep, names


class PreparedBatch:
    """The C arguments of a batch of queries, built once (prepare_batched) and passed to
    groupby_batched any number of times: the query and column structs point at the columns'
    buffers, so they stay valid while those buffers stay where they are (their contents may change
    between calls). It keeps the buffers alive."""

    def __init__(self, queries, output: str):
        self.n = len(queries)
        self.output = output
        self.qrec, self.ptrs, self.ncols, self.keep, self.names = _batch_args(queries, output)


def prepare_batched(queries, output: str = "host") -> PreparedBatch:
    """Marshals a batch for repeated groupby_batched calls (see PreparedBatch)."""
    return PreparedBatch(queries, output)


def groupby_batched(queries, output: str = "host", handle: Handle | None = None) -> Sequence:
    """Many independent group-by queries in one call (pmb_groupby_batched).

    queries: a list of (columns, keys, aggs, predicate) with the meanings of `groupby`, or a
    PreparedBatch (its own output kind then applies). Queries of one signature run in one
    persistent launch; the results come back in query order: a list of GroupByResult for host
    outputs, a BatchResults sequence of them for device outputs."""
    h = handle or default_handle()
    if isinstance(queries, PreparedBatch):
        n, output = queries.n, queries.output
        qrec, ptrs, ncols, keep, names = queries.qrec, queries.ptrs, queries.ncols, queries.keep, queries.names
    else:
        n = len(queries)
        qrec, ptrs, ncols, keep, names = _batch_args(queries, output)
    outs = (C.POINTER(A.Result) * max(1, n))()
    h.check(h._lib.pmb_groupby_batched(h.raw, qrec.ctypes.data_as(C.POINTER(A.Query)),
                                       ptrs.ctypes.data_as(C.POINTER(C.POINTER(A.Column))),
                                       ncols.ctypes.data_as(C.POINTER(C.c_int32)), n, outs))
    outs_p = C.cast(outs, C.c_void_p)
    try:
        if output == "device":
            # device outputs: every header in one array (one C call); the per-query result
            # objects are built when they are read, so a batch of thousands of queries costs no
            # Python object per query (nor the garbage collections that many objects set off)
            n_out = [len(x) for x in names]
            cap = 4 * n + 4 * sum(n_out)
            words = np.empty(max(1, cap), dtype=np.uint64)
            got = h._lib.pmb_results_pack(outs_p, n, words.ctypes.data, cap)
            if got != cap:
                raise RuntimeError("polars_b200: pmb_results_pack failed")
            offs = np.zeros(n + 1, dtype=np.int64)
            np.cumsum(4 + 4 * np.asarray(n_out, dtype=np.int64), out=offs[1:])
            return BatchResults(words, offs, names)
        addrs = list(C.cast(outs, C.POINTER(C.c_uint64 * max(1, n))).contents)[:n]
        results = []
        head_at = (C.c_uint64 * 5).from_address  # a pmb_result read as 64-bit words (layout checked at import)
        for i in range(n):
            hw = head_at(addrs[i])[:]
            su = hw[3] & 0xFFFFFFFF
            data, valid, dts = _read_result(A.Result.from_address(addrs[i]), names[i], True)
            results.append(GroupByResult(n_groups=hw[0], names=names[i], dtypes=dts, data=data, validity=valid,
                                         strategy=A.STRATEGY_NAMES.get(su, str(su)), rehash_count=hw[3] >> 32,
                                         capacity=hw[4]))
        return results
    finally:
        h._lib.pmb_results_free(outs_p, n)
        del keep


class BatchResults(Sequence):
    """The results of a batched call with device outputs, in query order: a sequence of
    GroupByResult built on access from the packed headers (pmb_results_pack). Device addresses
    stay valid until the next call on the same handle, as for any device output."""

    def __init__(self, words: np.ndarray, offs: np.ndarray, names: list):
        self._w = words
        self._o = offs
        self._names = names

    def __len__(self) -> int:
        return len(self._names)

    def _one(self, i: int) -> GroupByResult:
        o = int(self._o[i])
        w = self._w
        nc = int(w[o + 1]) & 0xFFFFFFFF
        su = int(w[o + 1]) >> 32
        cw = w[o + 4:o + 4 + 4 * nc].tolist()
        return GroupByResult(n_groups=int(w[o]), names=self._names[i], dtypes=[x & 0xFFFFFFFF for x in cw[3::4]],
                             data=cw[0::4], validity=cw[1::4], strategy=A.STRATEGY_NAMES.get(su, str(su)),
                             rehash_count=int(w[o + 2]), capacity=int(w[o + 3]))

    def __getitem__(self, i):
        if isinstance(i, slice):
            return [self._one(j) for j in range(*i.indices(len(self)))]
        if i < 0:
            i += len(self)
        if not 0 <= i < len(self):
            raise IndexError("batch result index out of range")
        return self._one(i)


def _query_shape(names, keys, aggs, predicate):
    """The parts of a query that do not depend on the column buffers."""
    index = {n: i for i, n in enumerate(names)}
    for k in keys:
        if k not in index:
            raise KeyError(f"polars_b200: key column {k!r} not found in upstream columns")
    key_arr = (C.c_int32 * max(1, len(keys)))(*[index[k] for k in keys])
    agg_arr = (A.Agg * max(1, len(aggs)))()
    for i, (op, col, _alias) in enumerate(aggs):
        if op not in A.AGG_OPS:
            raise ValueError(f"polars_b200: unknown aggregation op {op!r}")
        agg_arr[i].op = A.AGG_OPS[op]
        if op == "Len":
            agg_arr[i].column = -1
        else:
            if col not in index:
                raise KeyError(f"polars_b200: agg input column {col!r} not found in upstream columns")
            agg_arr[i].column = index[col]
    expr, expr_keep = compile_predicate(predicate, index)
    return key_arr, len(keys), agg_arr, len(aggs), expr, expr_keep


def selector_features(columns, keys, aggs, predicate=None, handle: Handle | None = None) -> np.ndarray:
    """The learned selector's features of a query (PMB_SELECTOR_FEATURES floats), computed on the
    device from a 4096-row sample of its keys."""
    h = handle or default_handle()
    q, cols, n, keep = _query(columns, keys, aggs, predicate)
    out = np.zeros(A.SELECTOR_FEATURES, dtype=np.float32)
    h.check(h._lib.pmb_selector_features(h.raw, C.byref(q), cols, n, out.ctypes.data))
    del keep
    return out


def selector_choose(columns, keys, aggs, predicate=None, handle: Handle | None = None) -> tuple[str, int]:
    """The strategy and group count the AUTO strategy of `handle` would use for this query."""
    h = handle or default_handle()
    q, cols, n, keep = _query(columns, keys, aggs, predicate)
    s, g = C.c_int32(), C.c_int64()
    h.check(h._lib.pmb_selector_choose(h.raw, C.byref(q), cols, n, C.byref(s), C.byref(g)))
    del keep
    return A.STRATEGY_NAMES.get(s.value, str(s.value)), int(g.value)


def _dev_ptr(t) -> int:
    assert t.is_cuda and t.is_contiguous(), "expected a contiguous CUDA tensor"
    return t.data_ptr()


def mlp_forward(params, x, handle: Handle | None = None):
    """Selector MLP outputs [batch, 4] for features x [batch, 24] (CUDA float32 tensors)."""
    import torch

    h = handle or default_handle()
    out = torch.empty((x.shape[0], A.SELECTOR_OUTPUTS), dtype=torch.float32, device=x.device)
    h.check(h._lib.pmb_mlp_forward(h.raw, _dev_ptr(params), _dev_ptr(x), x.shape[0], _dev_ptr(out)))
    return out


def mlp_gradient(params, x, cls, y, sw=None, wreg: float = 0.25, handle: Handle | None = None):
    """(gradient, loss) of the selector loss on a batch (CUDA tensors; cls int32, others float32)."""
    import torch

    h = handle or default_handle()
    grad = torch.empty_like(params)
    loss = torch.empty(1, dtype=torch.float32, device=params.device)
    h.check(h._lib.pmb_mlp_gradient(h.raw, _dev_ptr(params), _dev_ptr(x), _dev_ptr(cls), _dev_ptr(y),
                                    _dev_ptr(sw) if sw is not None else None, x.shape[0], wreg, _dev_ptr(grad),
                                    _dev_ptr(loss)))
    return grad, float(loss.item())


def mlp_adam_step(params, grad, m, v, step: int, lr: float, handle: Handle | None = None) -> None:
    h = handle or default_handle()
    h.check(h._lib.pmb_mlp_adam_step(h.raw, _dev_ptr(params), _dev_ptr(grad), _dev_ptr(m), _dev_ptr(v), step, lr))


# ------------------------------------------------------------------------------- wire format
def _all_valid(valid: bytes, n: int) -> bool:
    if n == 0:
        return True
    v = np.frombuffer(valid, dtype=np.uint8, count=(n + 7) // 8)
    full = n // 8
    if full and not np.all(v[:full] == 0xFF):
        return False
    rem = n % 8
    if rem:
        m = (1 << rem) - 1
        return (int(v[full]) & m) == m
    return True


def _wire_column(tag: str, data: bytes, valid: bytes, n_rows: int, name: str) -> ColumnData:
    if tag in ("Utf8", "String"):
        raise NotImplementedError(f"polars_b200: Utf8 columns are not supported on this path ({name!r})")
    if tag not in A.TAG_TO_DTYPE:
        raise ValueError(f"polars_b200: unknown dtype tag {tag!r} for column {name!r}")
    dt = A.TAG_TO_DTYPE[tag]
    if dt == A.BOOL:
        need = (n_rows + 7) // 8
        arr = np.frombuffer(data, dtype=np.uint8, count=need) if need else np.zeros(1, np.uint8)
    else:
        need = n_rows * A.DTYPE_BYTES[dt]
        if len(data) < need:
            raise ValueError(f"polars_b200: data buffer is {len(data)} B, need at least {need} B for {n_rows} rows")
        arr = np.frombuffer(data, dtype=A.NUMPY_NAME[dt], count=n_rows)
    if len(valid) < (n_rows + 7) // 8:
        raise ValueError(
            f"polars_b200: validity buffer is {len(valid)} B, need at least {(n_rows + 7) // 8} B for {n_rows} rows"
        )
    v = None if _all_valid(valid, n_rows) else np.frombuffer(valid, dtype=np.uint8, count=(n_rows + 7) // 8)
    return ColumnData(arr, v, dtype=dt, length=n_rows)


def execute_sort(plan: dict, n_rows: int, columns: list, slice_len: int | None = None) -> list[tuple[str, str, bytes, bytes]]:
    """A Sort plan over a GroupBy (`_build_sort`, python/polars_metal/_udf.py:684-721), run on the
    device in one call: the group-by of plan["input"] (execute_groupby's plan_dict), then its
    result sorted by plan["by_columns"] with plan["descending"] / plan["nulls_last"] (one flag or
    one per column), an optional plan["slice"] = [offset, length], then the first `slice_len` rows
    (the UDF's n_rows). Same wire shapes as execute_groupby."""
    if not isinstance(plan, dict) or "input" not in plan:
        raise ValueError("polars_b200: plan parse error: missing field input")
    by = list(plan.get("by_columns", []))
    offset, length = 0, None
    if plan.get("slice") is not None:
        offset, length = int(plan["slice"][0]), plan["slice"][1]
        length = None if length is None else int(length)
    if slice_len is not None:
        length = slice_len if length is None else min(length, slice_len)
    sort = None
    if by:
        sort = {"by": by, "descending": plan.get("descending", False), "nulls_last": plan.get("nulls_last", False),
                "offset": offset, "limit": length}
    elif offset or length is not None:
        raise ValueError("polars_b200: a slice without sort columns is not a Sort over a GroupBy")
    return execute_groupby(plan["input"], n_rows, columns, _sort=sort)


def execute_groupby(plan_dict: dict, n_rows: int, columns: list, _sort: dict | None = None) -> list[tuple[str, str, bytes, bytes]]:
    """Wire-compatible `_native.execute_groupby` (crates/polars-metal-core/src/udf/groupby/mod.rs:720-746).

    plan_dict: {"keys": [[name, tag], ...], "aggs": [{"input_col", "op", "output_alias", "kind"?}],
                "predicate": <predicate dict>?}
    columns:   [(name, tag, data: bytes, valid: bytes), ...]
    returns:   [(name, tag, data, valid), ...] keys then aggs; Count/Len as U32 with all-valid bitmaps.
    """
    if "keys" not in plan_dict:
        raise ValueError("polars_b200: plan parse error: missing field keys")
    if "aggs" not in plan_dict:
        raise ValueError("polars_b200: plan parse error: missing field aggs")
    by_name: dict[str, ColumnData] = {}
    for idx, entry in enumerate(columns):
        if not isinstance(entry, tuple) or len(entry) != 4:
            raise ValueError(
                f"polars_b200: execute_groupby columns[{idx}] must have 4 elements (name, dtype, data, valid)"
            )
        name, tag, data, valid = entry
        if not isinstance(data, (bytes, bytearray, memoryview)) or not isinstance(valid, (bytes, bytearray, memoryview)):
            raise ValueError(f"polars_b200: execute_groupby columns[{idx}] data and valid must be bytes")
        by_name[name] = (tag, bytes(data), bytes(valid))
    keys = []
    for k in plan_dict["keys"]:
        if not isinstance(k, (list, tuple)) or len(k) < 2:
            raise ValueError("polars_b200: plan parse error: wrong type for key entry")
        keys.append(str(k[0]))
    aggs = []
    for a in plan_dict["aggs"]:
        if "output_alias" not in a:
            raise ValueError("polars_b200: plan parse error: wrong type for output_alias")
        kind = a.get("kind") or ("Length" if a.get("op") == "Len" else "Simple")
        if kind == "Length":
            aggs.append(("Len", None, a["output_alias"]))
        elif kind == "Simple":
            if a.get("op") not in A.AGG_OPS:
                raise ValueError(f"polars_b200: plan parse error: unknown op {a.get('op')!r}")
            aggs.append((a["op"], a.get("input_col", ""), a["output_alias"]))
        elif kind == "Expression":
            if a.get("op") not in A.AGG_OPS or a.get("op") == "Len":
                raise ValueError(f"polars_b200: plan parse error: unknown op {a.get('op')!r}")
            aggs.append((a["op"], _arith_wire(a.get("expr")), a["output_alias"]))
        else:
            raise ValueError(f"polars_b200: plan parse error: unknown op kind={kind}")
    for k in keys:
        if k not in by_name:
            raise KeyError(f"polars_b200: key column {k!r} not found in upstream columns")
    agg_cols = []
    for op, col, _ in aggs:
        refs = _predicate_columns(col) if isinstance(col, dict) else ([col] if op != "Len" else [])
        for c in refs:
            if c not in by_name:
                raise KeyError(f"polars_b200: agg input column {c!r} not found in upstream columns")
        agg_cols += refs
    needed = list(dict.fromkeys(keys + agg_cols + _predicate_columns(plan_dict.get("predicate"))))
    cols = {}
    for name in needed:
        if name not in by_name:
            raise KeyError(f"polars_b200: column {name!r} not found in upstream columns")
        tag, data, valid = by_name[name]
        cols[name] = _wire_column(tag, data, valid, n_rows, name)
    res = groupby(cols, keys, aggs, plan_dict.get("predicate"), strategy=plan_dict.get("strategy", "auto"), sort=_sort)
    out = []
    n = res.n_groups
    for i, name in enumerate(res.names):
        dt = res.dtypes[i]
        tag = A.DTYPE_TO_TAG[dt]
        d = res.data[i]
        if dt == A.BOOL:
            db = bytes(d[: _bitmap_bytes(n)])
        else:
            db = d.tobytes()
        is_count = i >= len(keys) and aggs[i - len(keys)][0] in ("Count", "Len")
        vb = b"\xff" * _bitmap_bytes(n) if is_count else bytes(res.validity[i][: _bitmap_bytes(n)])
        out.append((name, tag, db, vb))
    return out


def _predicate_columns(p: dict | None) -> list[str]:
    if p is None:
        return []
    out = []
    if p.get("kind") == "Column":
        out.append(p["name"])
    for k in ("lhs", "rhs", "arg"):
        if isinstance(p.get(k), dict):
            out += _predicate_columns(p[k])
    return out


# ------------------------------------------------------------------------------- filter side
def _cmp_common(lhs_data, lhs_valid, rhs_data, rhs_valid, scalar, op, n_rows, dtype) -> tuple[bytes, bytes]:
    h = default_handle()
    width = 8
    if len(lhs_data) < n_rows * width:
        raise ValueError(f"polars_b200: data buffer is {len(lhs_data)} B, need at least {n_rows * width} B")
    if len(lhs_valid) < (n_rows + 7) // 8:
        raise ValueError(f"polars_b200: validity buffer is {len(lhs_valid)} B, need at least {(n_rows + 7) // 8} B")
    if op not in A.CMP_OPS:
        raise ValueError(f"polars_b200: unknown compare op {op!r}")
    npdt = "int64" if dtype == A.I64 else "float64"
    lc = ColumnData(np.frombuffer(lhs_data, dtype=npdt, count=n_rows), np.frombuffer(lhs_valid, np.uint8), dtype=dtype,
                    length=n_rows)
    cols = [lc]
    if rhs_data is not None:
        if len(rhs_data) < n_rows * width or len(rhs_valid) < (n_rows + 7) // 8:
            raise ValueError("polars_b200: rhs buffers too short")
        cols.append(ColumnData(np.frombuffer(rhs_data, dtype=npdt, count=n_rows), np.frombuffer(rhs_valid, np.uint8),
                               dtype=dtype, length=n_rows))
    abi, keep = _to_abi_columns(cols)
    nb = _bitmap_bytes(n_rows)
    od = (C.c_uint8 * nb)()
    ov = (C.c_uint8 * nb)()
    rhs_ptr = C.pointer(abi[1]) if rhs_data is not None else None
    si = int(scalar) if (scalar is not None and dtype == A.I64) else 0
    sf = float(scalar) if (scalar is not None and dtype == A.F64) else 0.0
    h.check(h._lib.pmb_compare(h.raw, C.pointer(abi[0]), rhs_ptr, si, sf, A.CMP_OPS[op], od, ov, 0))
    del keep
    return bytes(od), bytes(ov)


def cmp_i64_col_scalar(data: bytes, valid: bytes, rhs: int, op: str, n_rows: int) -> tuple[bytes, bytes]:
    return _cmp_common(data, valid, None, None, rhs, op, n_rows, A.I64)


def cmp_f64_col_scalar(data: bytes, valid: bytes, rhs: float, op: str, n_rows: int) -> tuple[bytes, bytes]:
    return _cmp_common(data, valid, None, None, rhs, op, n_rows, A.F64)


def cmp_i64_col_col(lhs: bytes, lhs_valid: bytes, rhs: bytes, rhs_valid: bytes, op: str, n_rows: int):
    return _cmp_common(lhs, lhs_valid, rhs, rhs_valid, None, op, n_rows, A.I64)


def cmp_f64_col_col(lhs: bytes, lhs_valid: bytes, rhs: bytes, rhs_valid: bytes, op: str, n_rows: int):
    return _cmp_common(lhs, lhs_valid, rhs, rhs_valid, None, op, n_rows, A.F64)


def _bool_common(fn_name, ld, lv, rd, rv, n_rows):
    h = default_handle()
    need = (n_rows + 7) // 8
    for label, b in (("lhs data", ld), ("lhs valid", lv), ("rhs data", rd), ("rhs valid", rv)):
        if len(b) < need:
            raise ValueError(f"polars_b200: {label} buffer is {len(b)} B, need at least {need} B for {n_rows} rows")
    nb = _bitmap_bytes(n_rows)
    od = (C.c_uint8 * nb)()
    ov = (C.c_uint8 * nb)()
    bufs = [np.frombuffer(x, np.uint8) if len(x) else np.zeros(1, np.uint8) for x in (ld, lv, rd, rv)]
    ptrs = [b.ctypes.data for b in bufs]
    h.check(getattr(h._lib, fn_name)(h.raw, *ptrs, n_rows, od, ov, 0))
    return bytes(od), bytes(ov)


def bool_and_dispatch(lhs_data: bytes, lhs_valid: bytes, rhs_data: bytes, rhs_valid: bytes, n_rows: int):
    return _bool_common("pmb_bool_and", lhs_data, lhs_valid, rhs_data, rhs_valid, n_rows)


def bool_or_dispatch(lhs_data: bytes, lhs_valid: bytes, rhs_data: bytes, rhs_valid: bytes, n_rows: int):
    return _bool_common("pmb_bool_or", lhs_data, lhs_valid, rhs_data, rhs_valid, n_rows)


def filter_columns(columns: dict, predicate: dict, output: str = "host", handle: Handle | None = None) -> GroupByResult:
    """Top-level filter: the rows of `columns` whose predicate is valid and true, every column
    compacted in one pass (pmb_filter_compact_expr; the reference's Filter node goes through
    `_filter_via_polars`, python/polars_metal/_udf.py:550-597). The result has the input's column
    names and dtypes; its `n_groups` is the number of rows kept."""
    h = handle or default_handle()
    names = list(columns)
    cols = [c if isinstance(c, ColumnData) else ColumnData(c) for c in columns.values()]
    abi, keep = _to_abi_columns(cols)
    expr, ek = compile_predicate(predicate, {n: i for i, n in enumerate(names)})
    if expr is None:
        raise ValueError("polars_b200: filter_columns needs a predicate")
    res_p = C.POINTER(A.Result)()
    h.check(h._lib.pmb_filter_compact_expr(h.raw, C.byref(expr), abi, len(cols), 1 if output == "device" else 0,
                                           C.byref(res_p)))
    try:
        res = res_p.contents
        data, valid, dts = _read_result(res, names, output != "device")
        return GroupByResult(n_groups=res.n_groups, names=names, dtypes=dts, data=data, validity=valid,
                             strategy="filter", rehash_count=0, capacity=0)
    finally:
        h._lib.pmb_result_free(res_p)
        del keep, ek


def _sort_spec(names: Sequence[str], by, descending=False, nulls_last=False, drop_nulls: bool = False,
               offset: int = 0, limit: int | None = None):
    """A pmb_sort_spec over the named columns; a single descending / nulls_last flag applies to
    every sort column, as in Polars' `sort`."""
    by = [by] if isinstance(by, str) else list(by)
    if not by:
        raise ValueError("polars_b200: sort needs at least one column")
    index = {n: i for i, n in enumerate(names)}
    for b in by:
        if b not in index:
            raise KeyError(f"polars_b200: sort column {b!r} not found")

    def flags(v, what):
        v = [bool(v)] * len(by) if isinstance(v, (bool, int, np.bool_)) else [bool(x) for x in v]
        if len(v) != len(by):
            raise ValueError(f"polars_b200: {what} has {len(v)} flags for {len(by)} sort columns")
        return (C.c_int32 * len(by))(*v)

    spec = A.SortSpec()
    b = (C.c_int32 * len(by))(*[index[x] for x in by])
    d = flags(descending, "descending")
    nl = flags(nulls_last, "nulls_last")
    spec.by, spec.descending, spec.nulls_last = b, d, nl
    spec.n_by = len(by)
    spec.drop_nulls = 1 if drop_nulls else 0
    spec.offset = int(offset)
    spec.limit = -1 if limit is None else int(limit)
    if limit is not None and limit < 0:
        raise ValueError("polars_b200: a negative slice length")
    return spec, (b, d, nl)


def sort_columns(columns: dict, by, descending=False, nulls_last=False, drop_nulls: bool = False, offset: int = 0,
                 limit: int | None = None, output: str = "host", handle: Handle | None = None) -> GroupByResult:
    """The rows of `columns` sorted by the `by` column(s) on the GPU (pmb_sort_columns), then the
    slice(offset, limit). Polars' order: nulls first unless nulls_last, whatever the direction;
    NaN above every number; -0.0 equal to 0.0; rows with equal keys keep their order. The reference
    sorts with Polars on the CPU (python/polars_metal/_udf.py:684-721) and routes only one
    null-free Float32 column to MLX (_udf.py:724-790)."""
    h = handle or default_handle()
    names = list(columns)
    cols = [c if isinstance(c, ColumnData) else ColumnData(c) for c in columns.values()]
    spec, sk = _sort_spec(names, by, descending, nulls_last, drop_nulls, offset, limit)
    abi, keep = _to_abi_columns(cols)
    res_p = C.POINTER(A.Result)()
    h.check(h._lib.pmb_sort_columns(h.raw, abi, len(cols), C.byref(spec), 1 if output == "device" else 0,
                                    C.byref(res_p)))
    try:
        res = res_p.contents
        data, valid, dts = _read_result(res, names, output != "device")
        return GroupByResult(n_groups=res.n_groups, names=names, dtypes=dts, data=data, validity=valid,
                             strategy="sort", rehash_count=0, capacity=0)
    finally:
        h._lib.pmb_result_free(res_p)
        del keep, sk


def top_k(columns: dict, k: int, by, output: str = "host", handle: Handle | None = None) -> GroupByResult:
    """The k rows with the largest `by` values, largest first; rows whose first `by` column is
    null are left out (Polars lowers top_k to a sort, descending, after dropping nulls)."""
    return sort_columns(columns, by, descending=True, nulls_last=True, drop_nulls=True, limit=k, output=output,
                        handle=handle)


def bottom_k(columns: dict, k: int, by, output: str = "host", handle: Handle | None = None) -> GroupByResult:
    """The k rows with the smallest `by` values, smallest first; nulls left out as in top_k."""
    return sort_columns(columns, by, descending=False, nulls_last=True, drop_nulls=True, limit=k, output=output,
                        handle=handle)


def execute_filter_compact(pred_data: bytes, pred_valid: bytes, n_rows: int, columns: list) -> list:
    """Wire-compatible `_native.execute_filter_compact` (crates/polars-metal-core/src/udf/compact.rs:46-147):
    columns [(tag, data, valid)] -> [(data, valid, n_out)] compacted by keep = pred_data & pred_valid."""
    h = default_handle()
    need = (n_rows + 7) // 8
    if len(pred_data) < need or len(pred_valid) < need:
        raise ValueError("polars_b200: predicate buffers too short")
    cols = []
    for idx, entry in enumerate(columns):
        tag, data, valid = entry
        cols.append(_wire_column(tag, bytes(data), bytes(valid), n_rows, f"columns[{idx}]"))
    abi, keep = _to_abi_columns(cols)
    pd = np.frombuffer(pred_data, np.uint8) if need else np.zeros(1, np.uint8)
    pv = np.frombuffer(pred_valid, np.uint8) if need else np.zeros(1, np.uint8)
    res_p = C.POINTER(A.Result)()
    h.check(h._lib.pmb_filter_compact(h.raw, pd.ctypes.data, pv.ctypes.data, n_rows, 0, abi, len(cols), 0,
                                      C.byref(res_p)))
    try:
        res = res_p.contents
        data, valid, dts = _read_result(res, None, True)
        n = res.n_groups
        out = []
        for i in range(res.n_columns):
            d = data[i]
            db = bytes(d[: _bitmap_bytes(n)]) if dts[i] == A.BOOL else d.tobytes()
            out.append((db, bytes(valid[i][: _bitmap_bytes(n)]), n))
        return out
    finally:
        h._lib.pmb_result_free(res_p)
        del keep


def cumsum_u8_to_u32(data: np.ndarray) -> np.ndarray:
    """Inclusive prefix sum u8 -> u32 (the MLX call the reference makes, mlx-sys/src/lib.rs:47)."""
    h = default_handle()
    a = np.ascontiguousarray(data, dtype=np.uint8)
    out = np.empty(a.size, dtype=np.uint32)
    h.check(h._lib.pmb_cumsum_u8_to_u32(h.raw, a.ctypes.data if a.size else None,
                                        out.ctypes.data if a.size else None, a.size, 0))
    return out
