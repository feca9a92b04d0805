"""GPU parity of the filter -> group_by -> aggregate path against the CPU oracle.

Every call goes through libpmb's C ABI (pmb_groupby) via the ctypes mirror."""

import numpy as np
import pytest

from helpers import (as_dict, assert_results_match, case_columns, expected_to_result, formula_columns, load_golden,
                     pack, unpack)
from oracle import pyoracle
from polars_b200 import _abi as A
from polars_b200 import datagen
from polars_b200._native import ColumnData, groupby

pytestmark = pytest.mark.gpu
GOLD = load_golden()
STRATEGIES = ["auto", "smem_hash", "global_hash", "sort", "partitioned"]


def _product_cols(cols: dict) -> dict:
    out = {}
    for name, ent in cols.items():
        data, valid = ent[0], ent[1]
        dt = ent[2] if len(ent) > 2 else None
        n = ent[3] if len(ent) > 3 else None
        out[name] = ColumnData(data, valid, dtype=dt, length=n)
    return out


def run_both(cols, keys, aggs, predicate=None, strategy="auto", label=""):
    got = groupby(_product_cols(cols), keys, aggs, predicate, strategy=strategy)
    want = pyoracle.groupby(cols, keys, aggs, predicate)
    assert_results_match(as_dict(got), want, len(keys), aggs, label)
    return got


@pytest.mark.parametrize("strategy", STRATEGIES)
@pytest.mark.parametrize("case", GOLD["groupby"], ids=lambda c: c["name"])
def test_known_answers(case, strategy):
    got = groupby(_product_cols(case_columns(case)), case["keys"], [tuple(a) for a in case["aggs"]], strategy=strategy)
    assert_results_match(as_dict(got), expected_to_result(case), len(case["keys"]), case["aggs"], case["name"])


@pytest.mark.parametrize("case", GOLD["integration"], ids=lambda c: c["name"])
def test_integration_shapes(case):
    cols = formula_columns(case["formula"], case["n"])
    aggs = [tuple(a) for a in case["aggs"]]
    got = groupby(_product_cols(cols), case["keys"], aggs)
    if case["formula"] == "all_unique":
        assert got.n_groups == case["expected"]["n_groups"]
        assert np.all(got.data[1] == 1)
        return
    assert_results_match(as_dict(got), expected_to_result(case), len(case["keys"]), case["aggs"], case["name"])


@pytest.mark.parametrize("strategy", STRATEGIES)
def test_small_workload_parity(strategy):
    t = datagen.make_small(1_000_000, seed=11)
    cols = datagen.to_numpy_columns(t)
    got = run_both(cols, t.keys, t.aggs, t.predicate, strategy, "small")
    assert got.n_groups == 1000


@pytest.mark.parametrize("n", [4_000_003, 1_000_000])
def test_hash_workload_parity(n):
    t = datagen.make_hash(n, seed=5)
    cols = datagen.to_numpy_columns(t)
    got = run_both(cols, t.keys, t.aggs, t.predicate, "auto", f"hash n={n}")
    assert got.strategy in ("global_hash", "smem_hash", "sort", "partitioned")


def test_hash_workload_device_resident_inputs():
    import torch

    t = datagen.make_hash(3_000_000, seed=6, device="cuda")
    torch.cuda.synchronize()
    got = groupby(datagen.to_column_data(t), t.keys, t.aggs, t.predicate)
    want = pyoracle.groupby(datagen.to_numpy_columns(t), t.keys, t.aggs, t.predicate)
    assert_results_match(as_dict(got), want, 1, t.aggs, "device inputs")


@pytest.mark.parametrize("strategy", ["auto", "sort", "partitioned"])
def test_sort_workload_shape_parity(strategy):
    # two-column key (int64 + int32): 96 data bits -> the 128-bit key table, or 20 + 6 packed bits
    # for the sort
    t = datagen.make_sort(2_000_000, seed=7, pool=20_000)
    cols = datagen.to_numpy_columns(t)
    got = run_both(cols, t.keys, t.aggs, None, strategy, f"two-key {strategy}")
    if strategy == "sort":
        assert got.strategy == "sort"


def test_sort_two_word_keys_big_groups_and_filter():
    rng = np.random.default_rng(31)
    n = 400_000
    # full-range int64 + int32 keys: more than 64 packed bits (two-word sort keys)
    k1 = rng.integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, 3000, dtype=np.int64)[rng.integers(0, 3000, n)]
    k2 = rng.integers(-2**31, 2**31 - 1, 50, dtype=np.int64).astype(np.int32)[rng.integers(0, 50, n)]
    cols = {"a": (k1, pack(rng.random(n) > 0.02)), "b": (k2, None),
            "v": (rng.standard_normal(n), pack(rng.random(n) > 0.1)),
            "w": (rng.integers(-10**6, 10**6, n).astype(np.int64), None)}
    aggs = [("Sum", "v", "s"), ("Mean", "v", "m"), ("Min", "w", "mn"), ("Max", "v", "mx"), ("Count", "v", "c"),
            ("Len", None, "n")]
    run_both(cols, ["a", "b"], aggs, None, "sort", "two-word keys")
    # a few very large groups (one CTA per group beyond 256 rows) mixed with singletons
    g = np.where(rng.random(n) < 0.5, rng.integers(0, 4, n), rng.integers(1000, 10**9, n)).astype(np.int64)
    cols2 = {"g": (g, None), "v": (rng.standard_normal(n), pack(rng.random(n) > 0.1)),
             "w": (rng.integers(-100, 100, n).astype(np.int32), None)}
    pred = {"kind": "Compare", "op": "Gt", "lhs": {"kind": "Column", "name": "v"},
            "rhs": {"kind": "LiteralF64", "value": -0.3}}
    got = run_both(cols2, ["g"], aggs[:1] + [("Min", "w", "mn"), ("Len", None, "n")], pred, "sort", "big groups")
    assert got.strategy == "sort"


@pytest.mark.parametrize("hint", [0, 50_000_000, 1])
def test_partitioned_partitions_and_fallbacks(hint):
    # hint 0: partitions sized from the sample; 50M: 2^16 partitions of a few rows each (two hash
    # passes, work items spanning many partitions); 1: too few output rows and partitions far
    # larger than their tables (the output is re-sized, then the sort strategy takes over)
    t = datagen.make_sort(1_500_000, seed=17, pool=60_000)
    cols = datagen.to_numpy_columns(t)
    got = groupby(_product_cols(cols), t.keys, t.aggs, None, strategy="partitioned", capacity_hint=hint)
    want = pyoracle.groupby(cols, t.keys, t.aggs, None)
    assert_results_match(as_dict(got), want, len(t.keys), t.aggs, f"partitioned hint={hint}")
    assert got.strategy == ("sort" if hint == 1 else "partitioned")


def test_partitioned_aggregation_without_nvrtc(monkeypatch):
    # with run-time compilation switched off the partitioned strategy aggregates with its prebuilt
    # kernel (values gathered through a per-thread stage); results must not change
    monkeypatch.setenv("PMB_JIT", "0")
    t = datagen.make_sort(400_000, seed=19, pool=3_000)
    cols = datagen.to_numpy_columns(t)
    got = run_both(cols, t.keys, t.aggs, None, "partitioned", "partitioned, prebuilt aggregation")
    assert got.strategy == "partitioned"


def test_sort_segment_reduce_without_nvrtc(monkeypatch):
    # without run-time compilation the sort strategy reduces its segments thread by thread
    monkeypatch.setenv("PMB_JIT", "0")
    t = datagen.make_sort(400_000, seed=23, pool=3_000)
    cols = datagen.to_numpy_columns(t)
    got = run_both(cols, t.keys, t.aggs, None, "sort", "sort, segment reduce")
    assert got.strategy == "sort"


def test_partitioned_heavy_keys_two_words_and_filter():
    rng = np.random.default_rng(37)
    n = 600_000
    # a handful of keys holding half the rows (partitions much longer than a work item) among
    # full-range two-column keys (two-word packed keys)
    hot = rng.random(n) < 0.5
    k1 = np.where(hot, rng.integers(0, 3, n), rng.integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, n,
                                                             dtype=np.int64)).astype(np.int64)
    k2 = np.where(hot, 7, rng.integers(-2**31, 2**31 - 1, n)).astype(np.int32)
    cols = {"a": (k1, pack(rng.random(n) > 0.02)), "b": (k2, None),
            "v": (rng.standard_normal(n), pack(rng.random(n) > 0.1)),
            "w": (rng.integers(-10**6, 10**6, n).astype(np.int64), None), "f": (rng.random(n).astype(np.float32), None)}
    aggs = [("Sum", "v", "s"), ("Mean", "v", "m"), ("Min", "w", "mn"), ("Max", "v", "mx"), ("Count", "v", "c"),
            ("Len", None, "n"), ("Sum", "f", "sf"), ("Max", "f", "mf")]
    pred = {"kind": "Compare", "op": "Gt", "lhs": {"kind": "Column", "name": "v"},
            "rhs": {"kind": "LiteralF64", "value": -0.8}}
    got = run_both(cols, ["a", "b"], aggs, pred, "partitioned", "partitioned heavy keys")
    assert got.strategy == "partitioned"


def test_empty_input():
    cols = {"k": (np.zeros(0, np.int64), None), "v": (np.zeros(0, np.float64), None)}
    got = groupby(_product_cols(cols), ["k"], [("Sum", "v", "s"), ("Len", None, "n")])
    assert got.n_groups == 0
    assert got.data[0].size == 0 and got.dtypes == [A.I64, A.F64, A.U32]


def test_everything_filtered_out():
    n = 10_000
    cols = {"k": (np.arange(n, dtype=np.int64) % 10, None), "v": (np.ones(n), None)}
    pred = {"kind": "Compare", "op": "Lt", "dtype": "F64", "lhs": {"kind": "Column", "name": "v"},
            "rhs": {"kind": "LiteralF64", "value": 0.0}}
    got = run_both(cols, ["k"], [("Sum", "v", "s")], pred, label="all filtered")
    assert got.n_groups == 0


@pytest.mark.parametrize("n", [1, 7, 127, 1023, 1024, 1025, 70_001])
def test_ragged_sizes(n):
    rng = np.random.default_rng(n)
    cols = {"k": (rng.integers(0, 50, n).astype(np.int32), pack(rng.random(n) > 0.1)),
            "v": (rng.standard_normal(n), pack(rng.random(n) > 0.2)),
            "w": (rng.integers(-100, 100, n).astype(np.int16), None)}
    aggs = [("Sum", "v", "s"), ("Mean", "v", "m"), ("Min", "w", "mn"), ("Max", "w", "mx"), ("Count", "v", "c"),
            ("Len", None, "n"), ("Sum", "w", "sw")]
    for strategy in STRATEGIES:
        run_both(cols, ["k"], aggs, None, strategy, f"ragged n={n} {strategy}")


KEY_DTYPES = ["int8", "int16", "int32", "int64", "uint8", "uint16", "uint32", "uint64", "float32", "float64"]


@pytest.mark.parametrize("strategy", ["auto", "sort", "partitioned"])
@pytest.mark.parametrize("kdt", KEY_DTYPES)
def test_key_dtypes(kdt, strategy):
    rng = np.random.default_rng(3)
    n = 50_000
    k = rng.integers(0, 100, n).astype(kdt)
    if kdt.startswith("float"):
        k[::97] = np.nan
        k[::89] = -0.0
    cols = {"k": (k, pack(rng.random(n) > 0.05)), "v": (rng.standard_normal(n).astype(np.float32), None)}
    run_both(cols, ["k"], [("Sum", "v", "s"), ("Min", "v", "mn"), ("Max", "v", "mx"), ("Len", None, "n")],
             strategy=strategy, label=f"key {kdt} {strategy}")


VALUE_DTYPES = ["int8", "int16", "int32", "int64", "uint8", "uint16", "uint32", "uint64", "float32", "float64"]


@pytest.mark.parametrize("strategy", ["auto", "sort", "partitioned"])
@pytest.mark.parametrize("vdt", VALUE_DTYPES)
def test_value_dtypes(vdt, strategy):
    rng = np.random.default_rng(4)
    n = 60_000
    if vdt.startswith("float"):
        v = (rng.standard_normal(n) * 1e3).astype(vdt)
        v[::1001] = np.nan
        v[::1003] = np.inf
    else:
        info = np.iinfo(vdt)
        v = rng.integers(info.min, info.max, n, dtype=vdt, endpoint=True)
    cols = {"k": (rng.integers(0, 300, n).astype(np.int64), None), "v": (v, pack(rng.random(n) > 0.1))}
    aggs = [("Sum", "v", "s"), ("Mean", "v", "m"), ("Min", "v", "mn"), ("Max", "v", "mx"), ("Count", "v", "c")]
    run_both(cols, ["k"], aggs, strategy=strategy, label=f"values {vdt} {strategy}")


@pytest.mark.parametrize("strategy", ["auto", "sort", "partitioned"])
def test_multi_key_with_nulls_and_bool(strategy):
    rng = np.random.default_rng(8)
    n = 100_000
    cols = {"a": (rng.integers(0, 5, n).astype(np.int64), pack(rng.random(n) > 0.1)),
            "b": (pack(rng.random(n) > 0.5), pack(rng.random(n) > 0.2), A.BOOL, n),
            "c": (rng.integers(-3, 3, n).astype(np.int16), None),
            "v": (rng.standard_normal(n), None)}
    run_both(cols, ["a", "b", "c"], [("Sum", "v", "s"), ("Len", None, "n")], strategy=strategy,
             label=f"multi-key {strategy}")


def test_high_cardinality_rehash():
    # a capacity hint far below the true group count forces overflow -> rehash, same result
    n = 500_000
    rng = np.random.default_rng(9)
    cols = {"k": (rng.permutation(n).astype(np.int64), None), "v": (rng.standard_normal(n), None)}
    got = groupby(_product_cols(cols), ["k"], [("Sum", "v", "s")], strategy="global_hash", capacity_hint=1000)
    assert got.rehash_count >= 1
    want = pyoracle.groupby(cols, ["k"], [("Sum", "v", "s")])
    assert_results_match(as_dict(got), want, 1, [("Sum", "v", "s")], "rehash")


def test_sentinel_key_values():
    # -1 in a non-null int64 key packs to all ones, the table's EMPTY pattern
    k = np.array([-1, -1, 0, 5, -1, np.iinfo(np.int64).max, np.iinfo(np.int64).min], np.int64)
    cols = {"k": (k, None), "v": (np.arange(k.size, dtype=np.float64), None)}
    for s in STRATEGIES:
        run_both(cols, ["k"], [("Sum", "v", "s"), ("Len", None, "n")], strategy=s, label=f"sentinel {s}")


def test_predicates_kleene_not_isnull_arith():
    rng = np.random.default_rng(10)
    n = 200_000
    cols = {"k": (rng.integers(0, 1000, n).astype(np.int32), None),
            "x": (rng.standard_normal(n), pack(rng.random(n) > 0.1)),
            "y": (rng.integers(-50, 50, n).astype(np.int64), pack(rng.random(n) > 0.1)),
            "f": (pack(rng.random(n) > 0.5), pack(rng.random(n) > 0.1), A.BOOL, n)}
    col = lambda c: {"kind": "Column", "name": c}  # noqa: E731
    preds = [
        {"kind": "Or", "lhs": {"kind": "Compare", "op": "Ge", "lhs": col("x"), "rhs": {"kind": "LiteralF64", "value": 1.0}},
         "rhs": col("f")},
        {"kind": "Not", "arg": {"kind": "And", "lhs": col("f"),
                                "rhs": {"kind": "Compare", "op": "Lt", "lhs": col("y"),
                                        "rhs": {"kind": "LiteralI64", "value": 0}}}},
        {"kind": "IsNull", "arg": col("x")},
        {"kind": "Compare", "op": "Eq", "dtype": "I64",
         "lhs": {"kind": "Arith", "op": "Mod", "lhs": col("y"), "rhs": {"kind": "LiteralI64", "value": -7}},
         "rhs": {"kind": "LiteralI64", "value": -3}},
        {"kind": "Compare", "op": "Gt",
         "lhs": {"kind": "Arith", "op": "TrueDiv", "lhs": col("y"), "rhs": col("x")},
         "rhs": {"kind": "LiteralF64", "value": 2.5}},
        {"kind": "Compare", "op": "Le", "dtype": "F64", "lhs": col("y"), "rhs": col("x")},
    ]
    aggs = [("Sum", "x", "s"), ("Count", "y", "c"), ("Len", None, "n")]
    for i, p in enumerate(preds):
        run_both(cols, ["k"], aggs, p, label=f"pred {i}")


@pytest.mark.parametrize("jit", ["0", "1"])
def test_remainder_zero_tests_on_both_kernels(jit, monkeypatch):
    """`x % c == 0` / `!= 0` on negative x and divisors of both signs, on the prebuilt and the
    run-time compiled kernel (the latter emits a divisibility test for these shapes)."""
    monkeypatch.setenv("PMB_JIT", jit)
    rng = np.random.default_rng(21)
    n = 300_000
    cols = {"k": (rng.integers(0, 500, n).astype(np.int32), None),
            "y": (rng.integers(-10**12, 10**12, n).astype(np.int64), pack(rng.random(n) > 0.1)),
            "x": (rng.standard_normal(n), pack(rng.random(n) > 0.05))}
    cols["y"][0][:4] = [np.iinfo(np.int64).min, np.iinfo(np.int64).max, -7, 0]
    col = lambda c: {"kind": "Column", "name": c}  # noqa: E731
    aggs = [("Sum", "x", "s"), ("Count", "y", "c"), ("Min", "y", "lo"), ("Len", None, "n")]
    for c in (7, -7, 3, 2, -1, 1000003, 12, -(2**63), 3 * 2**40):
        for op in ("Eq", "Ne"):
            p = {"kind": "Compare", "op": op, "dtype": "I64",
                 "lhs": {"kind": "Arith", "op": "Mod", "lhs": col("y"), "rhs": {"kind": "LiteralI64", "value": c}},
                 "rhs": {"kind": "LiteralI64", "value": 0}}
            run_both(cols, ["k"], aggs, p, label=f"jit={jit} y % {c} {op} 0")


def test_column_offsets_host_and_device():
    import torch

    rng = np.random.default_rng(12)
    n = 100_000
    off = 13
    k = rng.integers(0, 100, n + off).astype(np.int64)
    v = rng.standard_normal(n + off)
    vm = rng.random(n + off) > 0.2
    vb = pack(vm)
    want = pyoracle.groupby({"k": (k[off:], None), "v": (v[off:], pack(vm[off:]))}, ["k"], [("Sum", "v", "s")])
    for dev in (False, True):
        kk = torch.from_numpy(k).cuda() if dev else k
        vv = torch.from_numpy(v).cuda() if dev else v
        bb = torch.from_numpy(vb).cuda() if dev else vb
        cols = {"k": ColumnData(kk, None, A.I64, n, off), "v": ColumnData(vv, bb, A.F64, n, off)}
        got = groupby(cols, ["k"], [("Sum", "v", "s")])
        assert_results_match(as_dict(got), want, 1, [("Sum", "v", "s")], f"offset dev={dev}")


def test_device_outputs_report_groups():
    t = datagen.make_small(200_000, seed=13)
    got = groupby(datagen.to_column_data(t), t.keys, t.aggs, t.predicate, output="device")
    assert got.n_groups == 1000
    assert all(isinstance(p, int) and p != 0 for p in got.data)


@pytest.mark.parametrize("strategy", STRATEGIES)
@pytest.mark.parametrize("n", [50_000, 3_000_000])
def test_float_sum_outlier_beyond_the_fixed_point(strategy, n):
    # one value far above the rest, on a row the sample skips: the exact fixed point would truncate
    # every other group's sums, so the column moves to double-double sums and the call runs again
    rng = np.random.default_rng(41)
    v = rng.standard_normal(n)
    v[1] = 3.0e30
    cols = {"k": (rng.integers(0, 1000, n).astype(np.int32), None), "v": (v, pack(rng.random(n) > 0.05))}
    aggs = [("Sum", "v", "s"), ("Mean", "v", "m"), ("Len", None, "n")]
    run_both(cols, ["k"], aggs, None, strategy, f"outlier {strategy} n={n}")


def test_pinned_result_buffers_are_not_shared_between_live_results():
    # host results of 1 MB and more come from a recycled pool of pinned blocks: results kept alive
    # across later calls, and results dropped between calls (their blocks reused), must all still
    # hold their own values
    import gc

    tables = [datagen.make_hash(1_000_000, seed=300 + i, device="cpu", n_values=2_000_000, s=0.2) for i in range(3)]
    wants = [pyoracle.groupby(datagen.to_numpy_columns(t), t.keys, t.aggs, t.predicate) for t in tables]
    kept = []
    for rep in range(3):
        for t, want in zip(tables, wants):
            got = groupby(datagen.to_column_data(t), t.keys, t.aggs, t.predicate, output="host")
            assert max(np.asarray(d).nbytes for d in got.data) >= 1 << 20  # a pooled buffer is involved
            if rep == 0:
                kept.append((got, want, t))
            else:
                assert_results_match(as_dict(got), want, 1, t.aggs, f"pooled rep {rep}")
            del got
            gc.collect()
    for got, want, t in kept:
        assert_results_match(as_dict(got), want, 1, t.aggs, "pooled, kept alive")
