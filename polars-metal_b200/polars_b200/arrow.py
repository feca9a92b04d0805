"""Arrow in, Arrow out: pyarrow arrays as the group-by's input columns without copying them, and
the result as a pyarrow table.

The reference moves Arrow buffers to the GPU through its buffer crate
(crates/polars-metal-buffer/src/bridge.rs:1-60), and its Python side copies every column into
`bytes` first, combining chunks (python/polars_metal/_udf.py:1441-1456, 1484-1571). Here a
single-chunk column is handed to libpmb as the Arrow buffers themselves: the value buffer from
its start, the validity bitmap, and the array's offset, which libpmb applies to both (a bit offset
in the bitmap included). Only a column of several chunks is combined into one (a copy).
"""

from __future__ import annotations

from typing import Sequence

import numpy as np
import pyarrow as pa
import pyarrow.compute as pc

from . import _abi as A
from ._native import ColumnData, GroupByResult, Handle, filter_columns, groupby, sort_columns

_TO_PMB = {
    pa.bool_(): A.BOOL,
    pa.int8(): A.I8,
    pa.int16(): A.I16,
    pa.int32(): A.I32,
    pa.int64(): A.I64,
    pa.uint8(): A.U8,
    pa.uint16(): A.U16,
    pa.uint32(): A.U32,
    pa.uint64(): A.U64,
    pa.float32(): A.F32,
    pa.float64(): A.F64,
}
_FROM_PMB = {v: k for k, v in _TO_PMB.items()}


def _cuda() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except ImportError:
        return False


def _chunks_to_device(col: pa.ChunkedArray, dt: int) -> ColumnData:
    """A numeric column of several chunks copied chunk by chunk into one device buffer: the values
    are not concatenated on the host first. The validity bitmap (an eighth of a byte a row) is
    combined on the host by pyarrow and copied after them."""
    import torch

    n = len(col)
    elem = A.DTYPE_BYTES[dt]
    dev = torch.empty(max(n * elem, 1), dtype=torch.uint8, device="cuda")
    off = 0
    for ch in col.chunks:
        m = len(ch)
        if m:
            vals = np.frombuffer(ch.buffers()[1], dtype=A.NUMPY_NAME[dt])[ch.offset: ch.offset + m]
            dev[off * elem: (off + m) * elem].copy_(torch.from_numpy(vals.view(np.uint8)))
        off += m
    validity = None
    if col.null_count:
        bits = pc.is_valid(col).combine_chunks()
        vb = np.frombuffer(bits.buffers()[1], np.uint8)
        validity = torch.from_numpy(np.ascontiguousarray(vb[: (n + 7) // 8])).to("cuda")
    return ColumnData(dev, validity, dtype=dt, length=n)


def column_from_arrow(arr: pa.Array | pa.ChunkedArray, device: bool = False) -> ColumnData:
    """A libpmb column over an Arrow array's own buffers (no copy for a single chunk). A numeric
    column of several chunks is combined into one host array, or with `device` copied chunk by
    chunk into one CUDA buffer."""
    if isinstance(arr, pa.ChunkedArray):
        if device and arr.num_chunks > 1 and _TO_PMB.get(arr.type, A.BOOL) != A.BOOL:
            return _chunks_to_device(arr, _TO_PMB[arr.type])
        if arr.num_chunks == 1:
            arr = arr.chunk(0)
        elif arr.num_chunks == 0:
            arr = pa.array([], type=arr.type)
        else:
            arr = arr.combine_chunks()
    dt = _TO_PMB.get(arr.type)
    if dt is None:
        raise NotImplementedError(f"polars_b200: unsupported Arrow type {arr.type}")
    n = len(arr)
    validity_buf, data_buf = arr.buffers()[:2]
    if data_buf is None or data_buf.size == 0:
        data = np.zeros(max(1, (n + 7) // 8) if dt == A.BOOL else 1, np.uint8 if dt == A.BOOL else A.NUMPY_NAME[dt])
        return ColumnData(data, None, dtype=dt, length=0, offset=0)
    data = np.frombuffer(data_buf, dtype=np.uint8 if dt == A.BOOL else A.NUMPY_NAME[dt])
    validity = np.frombuffer(validity_buf, dtype=np.uint8) if validity_buf is not None and arr.null_count else None
    return ColumnData(data, validity, dtype=dt, length=n, offset=arr.offset)


def columns_from_arrow(table: pa.Table | pa.RecordBatch, names: Sequence[str] | None = None,
                       device: bool = False) -> dict:
    """{name: ColumnData} for the named columns of a table (all of them by default)."""
    names = list(table.column_names if names is None else names)
    return {name: column_from_arrow(table.column(name), device) for name in names}


def table_from_result(res: GroupByResult) -> pa.Table:
    """The group-by result (host output) as a pyarrow table: keys first, then the aggregates."""
    arrays = []
    for data, valid, dt in zip(res.data, res.validity, res.dtypes):
        if isinstance(data, int):
            raise ValueError("polars_b200: the result is on the device; ask for output='host'")
        arrays.append(pa.Array.from_buffers(_FROM_PMB[dt], res.n_groups,
                                            [pa.py_buffer(np.ascontiguousarray(valid)),
                                             pa.py_buffer(np.ascontiguousarray(data))]))
    return pa.Table.from_arrays(arrays, names=list(res.names))


def _dictionary_key(col) -> tuple[pa.Array, pa.Array] | None:
    """(int32 codes with the column's nulls, the distinct values) of a string, binary or
    dictionary column; None for other types. Strings are encoded on the host (the reference
    encodes them on the host too, crates/polars-metal-buffer/src/dict.rs:18-74); the group-by then
    runs on the codes, and the output codes are decoded through the values. The values are in
    sorted (byte-wise) order, so that the codes sort as the strings do."""
    if isinstance(col, pa.ChunkedArray):
        if pa.types.is_dictionary(col.type):
            col = col.unify_dictionaries()
        col = col.combine_chunks() if col.num_chunks else pa.array([], type=col.type)
    t = col.type
    if pa.types.is_dictionary(t):
        codes, values = col.indices, col.dictionary
    elif pa.types.is_string(t) or pa.types.is_large_string(t) or pa.types.is_binary(t) or pa.types.is_large_binary(t):
        enc = pc.dictionary_encode(col)
        codes, values = enc.indices, enc.dictionary
    else:
        return None
    order = pc.sort_indices(values)
    rank = np.empty(len(values), np.int32)
    rank[order.to_numpy()] = np.arange(len(values), dtype=np.int32)
    return pc.take(pa.array(rank, pa.int32()), codes), values.take(order)


def _predicate_columns(p, out: set) -> set:
    if isinstance(p, dict):
        if p.get("kind") == "Column":
            out.add(p["name"])
        for v in p.values():
            _predicate_columns(v, out)
    return out


def groupby_arrow(table: pa.Table | pa.RecordBatch, keys: Sequence[str], aggs: Sequence[tuple[str, str | None, str]],
                  predicate: dict | None = None, strategy: str = "auto", handle: Handle | None = None,
                  sort: dict | None = None) -> pa.Table:
    """filter -> group_by -> aggregate of an Arrow table through libpmb; the result as an Arrow
    table (keys, then the aggregates, in no particular group order unless `sort` orders it on the
    device, as groupby takes it). Key columns may be strings, binary or dictionaries (grouped by
    their dictionary codes, which sort as the strings do); only the columns the query reads are
    handed to libpmb."""
    used = set(keys) | _predicate_columns(predicate, set())
    for _op, c, _a in aggs:
        if isinstance(c, dict):  # an expression aggregate reads the columns of its expression
            _predicate_columns(c, used)
        elif c is not None:
            used.add(c)
    names = [n for n in table.column_names if n in used]
    missing = [n for n in used if n not in table.column_names]
    if missing:
        raise KeyError(f"polars_b200: column {missing[0]!r} not found in upstream columns")
    cols, dicts = {}, {}
    dev = _cuda()
    for name in names:
        enc = _dictionary_key(table.column(name)) if name in keys else None
        if enc is not None:
            cols[name] = column_from_arrow(enc[0])
            dicts[name] = enc[1]
        else:
            cols[name] = column_from_arrow(table.column(name), dev)
    res = groupby(cols, keys, aggs, predicate, strategy=strategy, output="host", handle=handle, sort=sort)
    return _decoded(table_from_result(res), dicts)


def _decoded(out: pa.Table, dicts: dict) -> pa.Table:
    for name, values in dicts.items():
        i = out.column_names.index(name)
        out = out.set_column(i, name, values.take(out.column(i)))
    return out


def sort_arrow(table: pa.Table | pa.RecordBatch, by, descending=False, nulls_last=False, offset: int = 0,
               limit: int | None = None, handle: Handle | None = None) -> pa.Table:
    """The rows of an Arrow table sorted by `by` on the GPU (sort_columns), then slice(offset,
    limit); string, binary and dictionary columns travel as their sorted-dictionary codes."""
    cols, dicts = {}, {}
    dev = _cuda()
    for name in table.column_names:
        enc = _dictionary_key(table.column(name))
        if enc is not None:
            cols[name] = column_from_arrow(enc[0])
            dicts[name] = enc[1]
        else:
            cols[name] = column_from_arrow(table.column(name), dev)
    res = sort_columns(cols, by, descending=descending, nulls_last=nulls_last, offset=offset, limit=limit,
                       output="host", handle=handle)
    return _decoded(table_from_result(res), dicts)


def filter_arrow(table: pa.Table | pa.RecordBatch, predicate: dict, handle: Handle | None = None) -> pa.Table:
    """The rows of an Arrow table whose predicate is valid and true, as an Arrow table (all its
    columns, in row order)."""
    res = filter_columns(columns_from_arrow(table, device=_cuda()), predicate, output="host", handle=handle)
    return table_from_result(res)
