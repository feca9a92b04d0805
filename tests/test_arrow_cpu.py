"""Arrow ingest and output (polars_b200.arrow) without a GPU: the columns handed to libpmb are the
Arrow buffers themselves (offsets and validity bits included), and results convert back."""

import numpy as np
import pyarrow as pa
import pytest

from polars_b200 import _abi as A
from polars_b200._native import GroupByResult
from polars_b200.arrow import column_from_arrow, columns_from_arrow, table_from_result


def _bits(buf: np.ndarray, i: int) -> bool:
    return bool((buf[i >> 3] >> (i & 7)) & 1)


def _values(cd) -> list:
    """Python values of a ColumnData as libpmb reads it (offset applied, nulls as None)."""
    out = []
    for i in range(cd.length):
        j = cd.offset + i
        if cd.validity is not None and not _bits(cd.validity, j):
            out.append(None)
        elif cd.dtype == A.BOOL:
            out.append(_bits(cd.data, j))
        else:
            out.append(cd.data[j].item())
    return out


@pytest.mark.parametrize("typ", [pa.int8(), pa.int32(), pa.int64(), pa.uint16(), pa.float32(), pa.float64()])
def test_numeric_columns_are_the_arrow_buffers(typ):
    rng = np.random.default_rng(3)
    vals = rng.integers(-100, 100, 1000).astype(typ.to_pandas_dtype())
    mask = rng.random(1000) < 0.1
    arr = pa.array(vals, type=typ, mask=mask)
    cd = column_from_arrow(arr)
    assert cd.dtype == {pa.int8(): A.I8, pa.int32(): A.I32, pa.int64(): A.I64, pa.uint16(): A.U16,
                        pa.float32(): A.F32, pa.float64(): A.F64}[typ]
    assert np.shares_memory(cd.data, np.frombuffer(arr.buffers()[1], dtype=cd.data.dtype))  # no copy
    assert _values(cd) == arr.to_pylist()


def test_slices_keep_their_offset_and_bitmap():
    arr = pa.array([1.5, None, 3.0, 4.0, None, 6.0, 7.0, 8.0, None, 10.0, 11.0], type=pa.float64())
    for start in (0, 3, 5, 9):
        part = arr.slice(start, 11 - start)
        cd = column_from_arrow(part)
        assert cd.offset == start and cd.length == 11 - start
        assert _values(cd) == part.to_pylist()


def test_bool_columns_and_columns_without_nulls():
    b = pa.array([True, False, None, True, True, False, None, False, True], type=pa.bool_()).slice(2)
    cd = column_from_arrow(b)
    assert cd.dtype == A.BOOL and _values(cd) == b.to_pylist()
    plain = column_from_arrow(pa.array(np.arange(10, dtype=np.int64)))
    assert plain.validity is None and _values(plain) == list(range(10))


def test_chunked_columns_and_tables():
    ch = pa.chunked_array([pa.array([1, 2, None], type=pa.int32()), pa.array([4, None], type=pa.int32())])
    cd = column_from_arrow(ch)  # several chunks: combined into one array (a copy)
    assert _values(cd) == [1, 2, None, 4, None]
    t = pa.table({"k": pa.array([1, 2, 3], type=pa.int64()), "v": pa.array([0.5, None, 2.0])})
    cols = columns_from_arrow(t)
    assert list(cols) == ["k", "v"] and _values(cols["v"]) == [0.5, None, 2.0]
    assert column_from_arrow(pa.chunked_array([], type=pa.int64())).length == 0


def test_unsupported_types_are_refused():
    with pytest.raises(NotImplementedError):
        column_from_arrow(pa.array(["a", "b"]))


def test_results_become_arrow_tables():
    n = 5
    keys = np.array([3, 1, 4, 1, 5], dtype=np.int64)
    sums = np.array([0.5, 1.5, 2.5, 3.5, 4.5])
    cnt = np.array([1, 2, 3, 4, 5], dtype=np.uint32)
    full = np.packbits(np.ones(8, bool), bitorder="little")
    some = np.packbits(np.array([1, 0, 1, 1, 0, 0, 0, 0], bool), bitorder="little")
    pad = lambda b: np.concatenate([b, np.zeros(3, np.uint8)])  # noqa: E731  (bitmaps padded to 4 bytes)
    res = GroupByResult(n_groups=n, names=["k", "s", "n"], dtypes=[A.I64, A.F64, A.U32], data=[keys, sums, cnt],
                        validity=[pad(full), pad(some), pad(full)], strategy="global_hash", rehash_count=0, capacity=8)
    t = table_from_result(res)
    assert t.column_names == ["k", "s", "n"]
    assert t.column("k").to_pylist() == keys.tolist()
    assert t.column("s").to_pylist() == [0.5, None, 2.5, 3.5, None]
    assert t.column("n").type == pa.uint32() and t.column("n").to_pylist() == cnt.tolist()


def test_string_and_dictionary_keys_become_codes():
    from polars_b200.arrow import _dictionary_key

    s = pa.chunked_array([pa.array(["x", None, "y"]), pa.array(["x", "zz"])])
    codes, values = _dictionary_key(s)
    assert codes.type == pa.int32()
    assert values.take(codes).to_pylist() == ["x", None, "y", "x", "zz"]
    d = pa.chunked_array([pa.array(["a", "b", "a"]).dictionary_encode(), pa.array(["c", "a"]).dictionary_encode()])
    codes, values = _dictionary_key(d)  # chunks with different dictionaries are unified
    assert values.take(codes).to_pylist() == ["a", "b", "a", "c", "a"]
    assert _dictionary_key(pa.array([1, 2, 3])) is None
