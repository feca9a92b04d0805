"""GPU parity of the Arrow path (polars_b200.arrow) against the CPU oracle: groupby_arrow on sliced
arrays (Arrow offsets, bit offsets in the validity bitmaps), nulls, a Bool key and several chunks;
filter_arrow over every dtype."""

import numpy as np
import pyarrow as pa
import pytest

from helpers import assert_results_match, pack
from oracle import pyoracle
from polars_b200 import _abi as A
from polars_b200.arrow import column_from_arrow, filter_arrow, groupby_arrow

pytestmark = pytest.mark.gpu


def _arrow_as_dict(t: pa.Table) -> dict:
    data, valid, dts = [], [], []
    for name in t.column_names:
        a = t.column(name).combine_chunks()
        cd = column_from_arrow(a)
        vb = a.buffers()[0]
        data.append(cd.data if cd.dtype == A.BOOL else cd.data[cd.offset: cd.offset + len(a)])
        valid.append(np.frombuffer(vb, np.uint8) if vb is not None else np.full(max(1, (len(a) + 7) // 8), 255, np.uint8))
        dts.append(cd.dtype)
    return {"n_groups": t.num_rows, "names": t.column_names, "dtypes": dts, "data": data, "validity": valid}


@pytest.mark.parametrize("start", [0, 3, 13])
def test_arrow_table_parity(start):
    rng = np.random.default_rng(41 + start)
    n = 200_003
    k = rng.integers(0, 5_000, n).astype(np.int64)
    kn = rng.random(n) < 0.02
    f = rng.random(n) < 0.5
    v = rng.standard_normal(n)
    vn = rng.random(n) < 0.1
    w = rng.integers(-1000, 1000, n).astype(np.int32)
    table = pa.table({"k": pa.array(k, mask=kn), "f": pa.array(f), "v": pa.array(v, mask=vn), "w": pa.array(w)})
    table = table.slice(start, n - start)
    m = n - start
    # the oracle's columns: the same rows, materialised at offset 0
    cols = {"k": (k[start:], pack(~kn[start:])), "f": (pack(f[start:]), None, A.BOOL, m),
            "v": (v[start:], pack(~vn[start:])), "w": (w[start:], None)}
    aggs = [("Sum", "v", "s"), ("Mean", "v", "m"), ("Min", "w", "lo"), ("Max", "v", "hi"), ("Count", "v", "c"),
            ("Len", None, "n")]
    pred = {"kind": "Compare", "op": "Gt", "lhs": {"kind": "Column", "name": "w"},
            "rhs": {"kind": "LiteralI64", "value": -800}}
    got = groupby_arrow(table, ["k", "f"], aggs, pred)
    want = pyoracle.groupby(cols, ["k", "f"], aggs, pred)
    assert_results_match(_arrow_as_dict(got), want, 2, aggs, f"arrow start={start}")


def test_arrow_chunked_input():
    rng = np.random.default_rng(5)
    parts = [rng.integers(0, 300, 50_000).astype(np.int32) for _ in range(3)]
    vals = [rng.standard_normal(50_000) for _ in range(3)]
    table = pa.table({"k": pa.chunked_array([pa.array(p) for p in parts]),
                      "v": pa.chunked_array([pa.array(x) for x in vals])})
    aggs = [("Sum", "v", "s"), ("Len", None, "n")]
    got = groupby_arrow(table, ["k"], aggs)
    want = pyoracle.groupby({"k": (np.concatenate(parts), None), "v": (np.concatenate(vals), None)}, ["k"], aggs)
    assert_results_match(_arrow_as_dict(got), want, 1, aggs, "arrow chunked")


def test_filter_arrow_every_dtype():
    # a top-level Filter: every column of every dtype compacted in one pass, in row order
    rng = np.random.default_rng(77)
    n = 100_003
    start = 5
    dtypes = [np.int8, np.int16, np.int32, np.int64, np.uint8, np.uint16, np.uint32, np.uint64, np.float32, np.float64]
    data = {f"c{i}": rng.integers(0, 100, n).astype(dt) for i, dt in enumerate(dtypes)}
    nulls = {name: rng.random(n) < 0.1 for name in data}
    data["b"] = rng.random(n) < 0.5
    nulls["b"] = rng.random(n) < 0.05
    table = pa.table({name: pa.array(v, mask=nulls[name]) for name, v in data.items()}).slice(start)
    pred = {"kind": "Compare", "op": "Lt", "dtype": "I64", "lhs": {"kind": "Column", "name": "c3"},
            "rhs": {"kind": "LiteralI64", "value": 60}}
    got = filter_arrow(table, pred)
    c3, c3n = data["c3"][start:], nulls["c3"][start:]
    keep = pyoracle.filter_mask({"c3": (c3, pack(~c3n))}, pred)
    assert got.num_rows == int(keep.sum()) and got.column_names == list(data)
    for name, v in data.items():
        col = got.column(name).to_numpy(zero_copy_only=False)
        want_valid = ~nulls[name][start:][keep]
        got_valid = ~np.asarray(got.column(name).is_null().to_numpy(zero_copy_only=False))
        assert np.array_equal(got_valid, want_valid), name
        assert np.array_equal(np.asarray(col)[want_valid].astype(v.dtype), v[start:][keep][want_valid]), name


def test_string_keys_through_their_dictionary():
    # a Utf8 key (with nulls) grouped by its dictionary codes; the output keys come back as strings
    import pyarrow.compute as pc

    rng = np.random.default_rng(91)
    n = 150_000
    words = np.array([f"w{i:05d}" for i in range(2_000)], dtype=object)
    s = words[rng.integers(0, 2_000, n)]
    sn = rng.random(n) < 0.03
    g = rng.integers(0, 4, n).astype(np.int16)
    v = rng.standard_normal(n)
    table = pa.table({"s": pa.array(s, mask=sn, type=pa.string()), "g": pa.array(g), "v": pa.array(v),
                      "unused": pa.array(["not read"] * n)})
    aggs = [("Sum", "v", "sv"), ("Max", "v", "mx"), ("Len", None, "n")]
    got = groupby_arrow(table, ["s", "g"], aggs)
    assert got.column("s").type == pa.string()
    enc = pc.dictionary_encode(table.column("s")).combine_chunks()
    codes = enc.indices.to_numpy(zero_copy_only=False)
    codes = np.where(np.isnan(codes), 0, codes).astype(np.int32) if codes.dtype.kind == "f" else codes.astype(np.int32)
    want = pyoracle.groupby({"s": (codes, pack(~sn)), "g": (g, None), "v": (v, None)}, ["s", "g"], aggs)
    # the product's string keys, back to the same codes
    got_codes = pc.index_in(got.column("s"), value_set=enc.dictionary)
    got_t = got.set_column(0, "s", got_codes.cast(pa.int32()))
    assert_results_match(_arrow_as_dict(got_t), want, 2, aggs, "string keys")


def test_chunked_columns_go_to_the_device_chunk_by_chunk():
    # several chunks, sliced (chunk offsets), with nulls: values copied per chunk into one device
    # buffer, validity combined on the host
    from polars_b200.arrow import column_from_arrow, sort_arrow

    rng = np.random.default_rng(17)
    sizes = [40_000, 1, 0, 77_777, 12_345]
    ks, vs, vns = [], [], []
    kch, vch = [], []
    for m in sizes:
        k = rng.integers(0, 999, m + 5).astype(np.int64)
        v = rng.standard_normal(m + 5)
        vn = rng.random(m + 5) < 0.1
        kch.append(pa.array(k).slice(5))
        vch.append(pa.array(v, mask=vn).slice(5))
        ks.append(k[5:])
        vs.append(v[5:])
        vns.append(vn[5:])
    table = pa.table({"k": pa.chunked_array(kch), "v": pa.chunked_array(vch, type=pa.float64())})
    cd = column_from_arrow(table.column("v"), device=True)
    assert cd.data.is_cuda and cd.validity.is_cuda and cd.length == sum(sizes)
    k, v, vn = np.concatenate(ks), np.concatenate(vs), np.concatenate(vns)
    aggs = [("Sum", "v", "s"), ("Count", "v", "c"), ("Max", "v", "mx"), ("Len", None, "n")]
    got = groupby_arrow(table, ["k"], aggs)
    want = pyoracle.groupby({"k": (k, None), "v": (v, pack(~vn))}, ["k"], aggs)
    assert_results_match(_arrow_as_dict(got), want, 1, aggs, "chunked on device")
    pred = {"kind": "Compare", "op": "Lt", "dtype": "I64", "lhs": {"kind": "Column", "name": "k"},
            "rhs": {"kind": "LiteralI64", "value": 100}}
    kept = filter_arrow(table, pred)
    assert kept.column("k").to_pylist() == k[k < 100].tolist()
    assert kept.column("v").is_null().to_pylist() == vn[k < 100].tolist()
    top = sort_arrow(table, ["v"], descending=True, nulls_last=True, limit=5)
    assert top.column("v").to_pylist() == sorted(v[~vn].tolist(), reverse=True)[:5]
