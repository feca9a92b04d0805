"""GPU parity of the device sort (pmb_sort_columns, pmb_groupby_sorted): the reference's own Sort /
top_k / bottom_k cases and its group-by cases (queries ending in `.sort(keys)`, expected rows in
key order), then seeded inputs of every dtype against the oracle's stable sort. Both sides are
stable sorts under the same order, so the rows must come out identical, in the same order."""

import numpy as np
import pytest

from helpers import as_dict, formula_columns, load_golden, pack
from oracle import pyoracle
from polars_b200 import _abi as A
from polars_b200 import _native as N
from test_sort_cpu import SORT, result_lists, sort_case_columns, sort_case_expected

pytestmark = pytest.mark.gpu


def cdata(ent):
    data, valid = ent[0], ent[1]
    if len(ent) > 2:
        return N.ColumnData(data, valid, dtype=ent[2], length=ent[3])
    return N.ColumnData(data, valid)


def assert_same_rows(got: dict, want: dict, label=""):
    assert int(got["n_groups"]) == int(want["n_groups"]), label
    assert list(got["dtypes"]) == list(want["dtypes"]), label
    n = int(want["n_groups"])
    for name, dt, gd, gv, wd, wv in zip(want["names"], want["dtypes"], got["data"], got["validity"], want["data"],
                                        want["validity"]):
        g_ok = np.unpackbits(np.asarray(gv, np.uint8), bitorder="little")[:n]
        w_ok = np.unpackbits(np.asarray(wv, np.uint8), bitorder="little")[:n]
        assert np.array_equal(g_ok, w_ok), f"{label}: validity of {name}"
        if dt == A.BOOL:
            g = np.unpackbits(np.asarray(gd, np.uint8), bitorder="little")[:n]
            w = np.unpackbits(np.asarray(wd, np.uint8), bitorder="little")[:n]
        else:
            g = np.asarray(gd)[:n].view(np.uint8).reshape(n, -1) if n else np.zeros((0, 1), np.uint8)
            w = np.asarray(wd)[:n].view(np.uint8).reshape(n, -1) if n else np.zeros((0, 1), np.uint8)
        m = w_ok.astype(bool)
        bad = np.nonzero(~np.all(g[m] == w[m], axis=-1) if g.ndim > 1 else g[m] != w[m])[0]
        assert bad.size == 0, f"{label}: {name} differs at rows {np.nonzero(m)[0][bad[:5]]}"


@pytest.mark.parametrize("case", SORT, ids=lambda c: c["name"])
def test_reference_sort_cases(case):
    s = case["spec"]
    cols = {k: cdata(v) for k, v in sort_case_columns(case).items()}
    got = N.sort_columns(cols, s["by"], s["descending"], s["nulls_last"], s["drop_nulls"], s["offset"],
                         None if s["limit"] < 0 else s["limit"])
    out = result_lists(as_dict(got))
    for name, vals in sort_case_expected(case).items():
        assert out[name] == vals, name


@pytest.mark.parametrize("case", load_golden()["integration"], ids=lambda c: c["name"])
def test_group_by_then_sort_in_one_call(case):
    cols = {k: cdata(v) for k, v in formula_columns(case["formula"], case["n"]).items()}
    aggs = [tuple(a) for a in case["aggs"]]
    got = N.groupby(cols, case["keys"], aggs, sort={"by": case["keys"]})
    out = result_lists(as_dict(got))
    if case["formula"] == "all_unique":  # 200,000 groups, kept as a property: keys 0..n-1 in order, sums 1
        assert got.n_groups == case["expected"]["n_groups"]
        assert out["k"] == list(range(case["n"])) and all(v == 1 for v in out["s"])
        return
    for name, vals in case["expected"].items():
        g = out[name]
        if got.dtypes[got.names.index(name)] in (A.F32, A.F64):
            assert all((a is None and b is None) or abs(a - b) <= 1e-6 * max(1.0, abs(b)) for a, b in zip(g, vals)), name
        else:
            assert g == vals, name


def _table(n, seed):
    rng = np.random.default_rng(seed)
    t = {
        "i8": (rng.integers(-3, 3, n).astype(np.int8), pack(rng.random(n) > 0.1)),
        "u16": (rng.integers(0, 50, n).astype(np.uint16), None),
        "i32": (rng.integers(-10**6, 10**6, n).astype(np.int32), pack(rng.random(n) > 0.05)),
        "i64": (rng.integers(-2**62, 2**62, n), None),
        "u64": (rng.integers(0, 2**64 - 1, n, dtype=np.uint64), None),
        "f32": (rng.choice(np.array([-0.0, 0.0, 1.5, -2.5, np.inf, -np.inf, np.nan], np.float32), n),
                pack(rng.random(n) > 0.1)),
        "f64": (rng.standard_normal(n), pack(rng.random(n) > 0.2)),
        "b": (pack(rng.random(n) > 0.5), pack(rng.random(n) > 0.1), A.BOOL, n),
        "rid": (np.arange(n, dtype=np.int64), None),
    }
    t["f64"][0][rng.random(n) < 0.05] = np.nan
    return t


SPECS = [
    (["i64"], [False], [False], False, 0, -1),
    (["f32", "i8"], [True, False], [True, False], False, 0, -1),
    (["b", "f32", "u16"], [False, True, False], [False, False, True], False, 0, -1),
    (["f64", "u64", "i64"], [True, False, True], [True, True, False], False, 0, -1),   # 192 key bits: 2 rounds
    (["i32"], [True], [True], True, 0, 1000),                                           # top_k
    (["f64"], [False], [True], True, 0, 25),                                            # bottom_k
    (["i8", "u16"], [False, False], [False, False], False, -777, 500),                  # slice from the end
    (["u16", "b"], [True, True], [False, True], False, 90_000, None),                   # offset past the rows
]


@pytest.mark.parametrize("spec", SPECS, ids=lambda s: "-".join(s[0]))
@pytest.mark.parametrize("n", [1, 4_097, 70_001])
def test_sort_matches_the_oracle(spec, n):
    by, desc, nl, drop, off, lim = spec
    t = _table(n, seed=n + len(by))
    want = pyoracle.sort_table(t, by, desc, nl, drop, off, -1 if lim is None else lim)
    got = N.sort_columns({k: cdata(v) for k, v in t.items()}, by, desc, nl, drop, off, None if lim in (None, -1) else lim)
    assert_same_rows(as_dict(got), want, f"{by} n={n}")


def test_sort_device_columns_in_and_out():
    import torch

    t = _table(100_003, seed=9)
    n = len(t["rid"][0])
    by = ["f32", "i64"]
    want = pyoracle.sort_table(t, by, [False, True], [True, False])
    rev = {v: k for k, v in A.NUMPY_NAME.items()}
    cols = {}
    for k, v in t.items():
        valid = torch.from_numpy(np.asarray(v[1])).cuda() if v[1] is not None else None
        dt = v[2] if len(v) > 2 else rev[v[0].dtype.name]
        cols[k] = N.ColumnData(torch.from_numpy(np.asarray(v[0]).view(np.uint8)).cuda(), valid, dtype=dt, length=n)
    host = N.sort_columns(cols, by, [False, True], [True, False])
    assert_same_rows(as_dict(host), want, "device in, host out")
    dev = N.sort_columns(cols, by, [False, True], [True, False], output="device")
    assert isinstance(dev.data[0], int) and dev.n_groups == want["n_groups"]


def test_empty_and_constant_inputs():
    e = N.sort_columns({"x": np.zeros(0, np.int64), "y": np.zeros(0, np.float64)}, "x")
    assert e.n_groups == 0
    c = N.sort_columns({"x": np.full(5000, 7, np.int64), "rid": np.arange(5000, dtype=np.int64)}, "x", limit=10)
    assert c.n_groups == 10 and list(c.data[1]) == list(range(10))  # equal keys keep their order


def test_large_sort_is_a_sorted_permutation():
    # 20M rows: sorted under the order, and a permutation of the input (checked by a row-id sum)
    n = 20_000_000
    rng = np.random.default_rng(21)
    k = rng.integers(-2**40, 2**40, n)
    rid = np.arange(n, dtype=np.int64)
    got = N.sort_columns({"k": k, "rid": rid}, "k", descending=True)
    gk, gr = got.data[0][:n], got.data[1][:n]
    assert np.all(gk[:-1] >= gk[1:])
    assert np.array_equal(np.sort(gr), rid)
    assert np.array_equal(k[gr], gk)


def test_group_by_sorted_by_an_aggregate_top_k():
    rng = np.random.default_rng(3)
    n = 1_000_000
    cols = {"k": rng.integers(0, 50_000, n), "v": rng.standard_normal(n)}
    aggs = [("Sum", "v", "s"), ("Len", None, "n")]
    got = N.groupby(cols, ["k"], aggs, sort={"by": ["s", "k"], "descending": True, "limit": 100})
    full = pyoracle.groupby({k: (v, None) for k, v in cols.items()}, ["k"], aggs)
    table = {nm: (d, v, dt, full["n_groups"]) for nm, d, v, dt in zip(full["names"], full["data"], full["validity"],
                                                                      full["dtypes"])}
    want = pyoracle.sort_table(table, ["s", "k"], [True, True], limit=100)
    assert got.n_groups == 100
    assert np.array_equal(got.data[0][:100], want["data"][0])
    assert np.allclose(got.data[1][:100], want["data"][1], rtol=1e-12, atol=1e-9)


def test_sort_plan_wire():
    n = 30_000
    rng = np.random.default_rng(6)
    k = rng.integers(0, 300, n)
    v = rng.integers(-100, 100, n)
    ones = b"\xff" * ((n + 7) // 8)
    columns = [("k", "I64", k.tobytes(), ones), ("v", "I64", v.tobytes(), ones)]
    inner = {"keys": [["k", "I64"]], "aggs": [{"input_col": "v", "op": "Sum", "output_alias": "s"}]}
    out = N.execute_sort({"kind": "Sort", "input": inner, "by_columns": ["s", "k"], "descending": [True, False],
                          "nulls_last": [False, False]}, n, columns, slice_len=10)
    ks = np.frombuffer(out[0][2], np.int64)
    ss = np.frombuffer(out[1][2], np.int64)
    sums = {int(a): int(v[k == a].sum()) for a in np.unique(k)}
    want = sorted(sums.items(), key=lambda kv: (-kv[1], kv[0]))[:10]
    assert list(zip(ks.tolist(), ss.tolist())) == want


def test_sort_arrow_with_strings():
    pa = pytest.importorskip("pyarrow")
    from polars_b200.arrow import groupby_arrow, sort_arrow

    words = ["pear", "apple", None, "fig", "apple", "kiwi", None, "banana"]
    t = pa.table({"w": pa.array(words), "x": pa.array([5, 3, 1, 2, 9, 4, 8, 7], pa.int64())})
    s = sort_arrow(t, ["w", "x"], nulls_last=True)
    assert s.column("w").to_pylist() == ["apple", "apple", "banana", "fig", "kiwi", "pear", None, None]
    assert s.column("x").to_pylist() == [3, 9, 7, 2, 4, 5, 1, 8]
    g = groupby_arrow(t, ["w"], [("Sum", "x", "sx")], sort={"by": "w", "descending": True})
    assert g.column("w").to_pylist() == [None, "pear", "kiwi", "fig", "banana", "apple"]
    assert g.column("sx").to_pylist() == [9, 5, 4, 2, 7, 12]
