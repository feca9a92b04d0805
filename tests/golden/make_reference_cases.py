"""Writes tests/golden/reference_cases.json: known-answer cases of the reference's own tests.

The reference (dbfclark/polars-metal) is Rust + Metal and cannot run here, so its known-answer
tests are transcribed by hand: each case below names the test it comes from (file:line in the
reference tree) and carries the inputs and the expected outputs that test asserts. Where the
reference test compares against Polars CPU on a closed-form input (the Python integration tests),
the expected values are computed here in plain numpy from the closed form, independently of the
oracle under test.

Run: python tests/golden/make_reference_cases.py
"""

from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent / "reference_cases.json"


def nan():
    return float("nan")


def groupby_cases() -> list[dict]:
    cases = []
    # crates/polars-metal-kernels/tests/test_groupby_aggregate.rs:312-326 gpu_sum_i32_four_groups
    cases.append({
        "name": "sum_i32_four_groups",
        "source": "crates/polars-metal-kernels/tests/test_groupby_aggregate.rs:312-326",
        "columns": {"g": {"dtype": "I32", "values": [0, 1, 2, 3, 0, 1, 2, 3]},
                    "v": {"dtype": "I32", "values": [10, 20, 30, 40, -1, 5, 7, 8],
                          "valid": [1, 1, 1, 1, 0, 1, 1, 1]}},
        "keys": ["g"], "aggs": [["Sum", "v", "s"]],
        "expected": {"g": [0, 1, 2, 3], "s": [10, 25, 37, 48]},
        "dtypes": {"g": "I32", "s": "I32"},
    })
    # test_groupby_aggregate.rs:329-339 gpu_sum_i32_all_nulls_gives_zero
    cases.append({
        "name": "sum_i32_all_nulls_gives_zero",
        "source": "crates/polars-metal-kernels/tests/test_groupby_aggregate.rs:329-339",
        "columns": {"g": {"dtype": "I32", "values": [0, 0, 0]},
                    "v": {"dtype": "I32", "values": [100, 200, 300], "valid": [0, 0, 0]}},
        "keys": ["g"], "aggs": [["Sum", "v", "s"]],
        "expected": {"g": [0], "s": [0]},
        "dtypes": {"g": "I32", "s": "I32"},
    })
    # test_groupby_aggregate.rs:342-355 gpu_count_and_len_differ_for_nulls (also :500-510)
    cases.append({
        "name": "count_and_len_differ_for_nulls",
        "source": "crates/polars-metal-kernels/tests/test_groupby_aggregate.rs:342-355",
        "columns": {"g": {"dtype": "I32", "values": [0, 0, 0, 1, 1]},
                    "v": {"dtype": "I32", "values": [1, 2, 3, 4, 5], "valid": [1, 0, 1, 1, 0]}},
        "keys": ["g"], "aggs": [["Count", "v", "c"], ["Len", None, "n"]],
        "expected": {"g": [0, 1], "c": [2, 1], "n": [3, 2]},
        "dtypes": {"g": "I32", "c": "U32", "n": "U32"},
    })
    # test_groupby_aggregate.rs:358-403 gpu_min_max_f32_q1_shape (expected via the test's ref_min/max)
    vals = [np.float32(i * 1.5 - 37.0) for i in range(100)]
    valid = [1 if i % 7 != 0 else 0 for i in range(100)]
    g = [i % 4 for i in range(100)]
    mins, maxs = [], []
    for grp in range(4):
        vs = [float(vals[i]) for i in range(100) if g[i] == grp and valid[i]]
        mins.append(min(vs))
        maxs.append(max(vs))
    cases.append({
        "name": "min_max_f32_q1_shape",
        "source": "crates/polars-metal-kernels/tests/test_groupby_aggregate.rs:358-403",
        "columns": {"g": {"dtype": "I32", "values": g},
                    "v": {"dtype": "F32", "values": [float(x) for x in vals], "valid": valid}},
        "keys": ["g"], "aggs": [["Min", "v", "mn"], ["Max", "v", "mx"]],
        "expected": {"g": [0, 1, 2, 3], "mn": mins, "mx": maxs},
        "dtypes": {"g": "I32", "mn": "F32", "mx": "F32"},
    })
    # test_groupby_aggregate.rs:419-428 cpu_sum_i64_basic
    cases.append({
        "name": "sum_i64_basic",
        "source": "crates/polars-metal-kernels/tests/test_groupby_aggregate.rs:419-428",
        "columns": {"g": {"dtype": "I32", "values": [0, 0, 0, 1, 1, 1]},
                    "v": {"dtype": "I64", "values": [1, 2, 3, 4, 5, 6], "valid": [1, 1, 0, 1, 1, 0]}},
        "keys": ["g"], "aggs": [["Sum", "v", "s"]],
        "expected": {"g": [0, 1], "s": [3, 9]},
        "dtypes": {"g": "I32", "s": "I64"},
    })
    # test_groupby_aggregate.rs:431-441 cpu_min_i64_all_null_group_has_no_valid
    cases.append({
        "name": "min_i64_all_null_group_is_null",
        "source": "crates/polars-metal-kernels/tests/test_groupby_aggregate.rs:431-441",
        "columns": {"g": {"dtype": "I32", "values": [0, 0]},
                    "v": {"dtype": "I64", "values": [100, 200], "valid": [0, 0]}},
        "keys": ["g"], "aggs": [["Min", "v", "mn"], ["Max", "v", "mx"]],
        "expected": {"g": [0], "mn": [None], "mx": [None]},
        "dtypes": {"g": "I32", "mn": "I64", "mx": "I64"},
    })
    # test_groupby_aggregate.rs:444-452 cpu_max_i64_single_group
    cases.append({
        "name": "max_i64_single_group",
        "source": "crates/polars-metal-kernels/tests/test_groupby_aggregate.rs:444-452",
        "columns": {"g": {"dtype": "I32", "values": [0, 0, 0, 0, 0]},
                    "v": {"dtype": "I64", "values": [-5, 100, -1000, 42, 0], "valid": [1, 1, 0, 1, 1]}},
        "keys": ["g"], "aggs": [["Max", "v", "mx"], ["Min", "v", "mn"]],
        "expected": {"g": [0], "mx": [100], "mn": [-5]},
        "dtypes": {"g": "I32", "mx": "I64", "mn": "I64"},
    })
    # test_groupby_aggregate.rs:455-466 cpu_sum_f64_basic
    cases.append({
        "name": "sum_f64_basic",
        "source": "crates/polars-metal-kernels/tests/test_groupby_aggregate.rs:455-466",
        "columns": {"g": {"dtype": "I32", "values": [0, 0, 1, 1]},
                    "v": {"dtype": "F64", "values": [1.0, 2.0, 3.0, 4.0], "valid": [1, 0, 1, 1]}},
        "keys": ["g"], "aggs": [["Sum", "v", "s"]],
        "expected": {"g": [0, 1], "s": [1.0, 7.0]},
        "dtypes": {"g": "I32", "s": "F64"},
    })
    # test_groupby_aggregate.rs:469-482 / :485-497 NaN poisoning of f64 min / max
    cases.append({
        "name": "min_f64_nan_poisoning",
        "source": "crates/polars-metal-kernels/tests/test_groupby_aggregate.rs:469-482",
        "columns": {"g": {"dtype": "I32", "values": [0, 0, 0]},
                    "v": {"dtype": "F64", "values": [1.0, nan(), 3.0]}},
        "keys": ["g"], "aggs": [["Min", "v", "mn"]],
        "expected": {"g": [0], "mn": [nan()]},
        "dtypes": {"g": "I32", "mn": "F64"},
    })
    cases.append({
        "name": "max_f64_nan_poisoning",
        "source": "crates/polars-metal-kernels/tests/test_groupby_aggregate.rs:485-497",
        "columns": {"g": {"dtype": "I32", "values": [0, 0, 0]},
                    "v": {"dtype": "F64", "values": [10.0, nan(), 5.0]}},
        "keys": ["g"], "aggs": [["Max", "v", "mx"]],
        "expected": {"g": [0], "mx": [nan()]},
        "dtypes": {"g": "I32", "mx": "F64"},
    })
    # test_groupby_aggregate.rs:517-520 compute_mean_f64_handles_empty_group: sums [10, 0], counts [2, 0]
    cases.append({
        "name": "mean_f64_empty_group_is_null",
        "source": "crates/polars-metal-kernels/tests/test_groupby_aggregate.rs:517-520",
        "columns": {"g": {"dtype": "I32", "values": [0, 0, 1, 1]},
                    "v": {"dtype": "F64", "values": [4.0, 6.0, 1.0, 2.0], "valid": [1, 1, 0, 0]}},
        "keys": ["g"], "aggs": [["Mean", "v", "m"]],
        "expected": {"g": [0, 1], "m": [5.0, None]},
        "dtypes": {"g": "I32", "m": "F64"},
    })
    # test_groupby_aggregate.rs:523-526 compute_mean_i64_returns_f64_with_division: sums [10, 7], counts [4, 2]
    cases.append({
        "name": "mean_i64_returns_f64",
        "source": "crates/polars-metal-kernels/tests/test_groupby_aggregate.rs:523-526",
        "columns": {"g": {"dtype": "I32", "values": [0, 0, 0, 0, 1, 1]},
                    "v": {"dtype": "I64", "values": [1, 2, 3, 4, 3, 4]}},
        "keys": ["g"], "aggs": [["Mean", "v", "m"]],
        "expected": {"g": [0, 1], "m": [2.5, 3.5]},
        "dtypes": {"g": "I32", "m": "F64"},
    })
    # test_groupby_aggregate.rs:535-538 compute_mean_single_row_per_group
    cases.append({
        "name": "mean_single_row_per_group",
        "source": "crates/polars-metal-kernels/tests/test_groupby_aggregate.rs:535-538",
        "columns": {"g": {"dtype": "I32", "values": [0, 1, 2]},
                    "v": {"dtype": "I64", "values": [3, -6, 0]}},
        "keys": ["g"], "aggs": [["Mean", "v", "m"]],
        "expected": {"g": [0, 1, 2], "m": [3.0, -6.0, 0.0]},
        "dtypes": {"g": "I32", "m": "F64"},
    })
    # crates/polars-metal-kernels/tests/test_key_encoding.rs:24-47 single i64 key round trip
    cases.append({
        "name": "key_single_i64_round_trip",
        "source": "crates/polars-metal-kernels/tests/test_key_encoding.rs:24-47",
        "columns": {"k": {"dtype": "I64", "values": [1, 2, 3, -1]}},
        "keys": ["k"], "aggs": [["Len", None, "n"]],
        "expected": {"k": [-1, 1, 2, 3], "n": [1, 1, 1, 1]},
        "dtypes": {"k": "I64", "n": "U32"},
    })
    # test_key_encoding.rs:49-88 two Bool keys (rows: (T,T), (T,F))
    cases.append({
        "name": "key_two_bools",
        "source": "crates/polars-metal-kernels/tests/test_key_encoding.rs:49-88",
        "columns": {"a": {"dtype": "Bool", "values": [1, 1]}, "b": {"dtype": "Bool", "values": [1, 0]}},
        "keys": ["a", "b"], "aggs": [["Len", None, "n"]],
        "expected": {"a": [True, True], "b": [False, True], "n": [1, 1]},
        "dtypes": {"a": "Bool", "b": "Bool", "n": "U32"},
    })
    # test_key_encoding.rs:90-117 one i64 + one Bool key (67 bits with null bits)
    cases.append({
        "name": "key_i64_plus_bool",
        "source": "crates/polars-metal-kernels/tests/test_key_encoding.rs:90-117",
        "columns": {"i": {"dtype": "I64", "values": [42, -7], "valid": [1, 1]},
                    "b": {"dtype": "Bool", "values": [0, 1], "valid": [1, 1]}},
        "keys": ["i", "b"], "aggs": [["Len", None, "n"]],
        "expected": {"i": [-7, 42], "b": [True, False], "n": [1, 1]},
        "dtypes": {"i": "I64", "b": "Bool", "n": "U32"},
    })
    # test_key_encoding.rs:119-140 a null key decodes as null, the valid one keeps its value
    cases.append({
        "name": "key_null_value",
        "source": "crates/polars-metal-kernels/tests/test_key_encoding.rs:119-140",
        "columns": {"k": {"dtype": "I64", "values": [99, 0], "valid": [1, 0]}},
        "keys": ["k"], "aggs": [["Len", None, "n"]],
        "expected": {"k": [None, 99], "n": [1, 1]},
        "dtypes": {"k": "I64", "n": "U32"},
    })
    return cases


def integration_cases() -> list[dict]:
    """tests/python_integration/test_groupby.py shapes (n = 200,000, engine vs Polars CPU).

    Inputs are closed-form (`formula`), expected values computed here with numpy."""
    n = 200_000
    i = np.arange(n, dtype=np.int64)
    cases = []

    def grp(keys: np.ndarray, vals: np.ndarray, mask=None):
        out = {}
        for k in np.unique(keys):
            sel = keys == k
            if mask is not None:
                sel_v = sel & mask
            else:
                sel_v = sel
            out[int(k)] = (vals[sel_v], int(sel.sum()))
        return out

    # :28-39 single i64 key sum
    g = grp(i % 7, i)
    cases.append({"name": "it_single_i64_key_sum", "source": "tests/python_integration/test_groupby.py:28-39",
                  "formula": "single_i64_key_sum", "n": n, "keys": ["k"], "aggs": [["Sum", "v", "s"]],
                  "expected": {"k": sorted(g), "s": [int(g[k][0].sum()) for k in sorted(g)]},
                  "dtypes": {"k": "I64", "s": "I64"}})
    # :42-66 all aggs over f64 values
    v = (i % 100).astype(np.float64)
    g = grp(i % 5, v)
    ks = sorted(g)
    cases.append({"name": "it_all_aggs", "source": "tests/python_integration/test_groupby.py:42-66",
                  "formula": "all_aggs", "n": n, "keys": ["k"],
                  "aggs": [["Sum", "v", "s"], ["Mean", "v", "m"], ["Min", "v", "mn"], ["Max", "v", "mx"],
                           ["Count", "v", "c"], ["Len", None, "n"]],
                  "expected": {"k": ks, "s": [float(math.fsum(g[k][0])) for k in ks],
                               "m": [float(math.fsum(g[k][0]) / len(g[k][0])) for k in ks],
                               "mn": [float(g[k][0].min()) for k in ks], "mx": [float(g[k][0].max()) for k in ks],
                               "c": [len(g[k][0]) for k in ks], "n": [g[k][1] for k in ks]},
                  "dtypes": {"k": "I64", "s": "F64", "m": "F64", "mn": "F64", "mx": "F64", "c": "U32", "n": "U32"}})
    # :69-89 two Bool keys
    rf = i % 2
    ls = (i // 2) % 2
    rows = sorted({(int(a), int(b)) for a, b in zip(rf[:4], ls[:4])})
    cases.append({"name": "it_two_bool_keys", "source": "tests/python_integration/test_groupby.py:69-89",
                  "formula": "two_bool_keys", "n": n, "keys": ["returnflag", "linestatus"],
                  "aggs": [["Sum", "qty", "sum_qty"]],
                  "expected": {"returnflag": [bool(a) for a, _ in rows], "linestatus": [bool(b) for _, b in rows],
                               "sum_qty": [int(i[(rf == a) & (ls == b)].sum()) for a, b in rows]},
                  "dtypes": {"returnflag": "Bool", "linestatus": "Bool", "sum_qty": "I64"}})
    # :92-112 Bool + i64 key
    cat = i % 2
    sub = i % 13
    rows = sorted({(int(a), int(b)) for a, b in zip(cat, sub)})
    vf = i.astype(np.float64)
    cases.append({"name": "it_bool_plus_i64_key", "source": "tests/python_integration/test_groupby.py:92-112",
                  "formula": "bool_plus_i64", "n": n, "keys": ["category", "subkey"], "aggs": [["Sum", "v", "sum_v"]],
                  "expected": {"category": [bool(a) for a, _ in rows], "subkey": [b for _, b in rows],
                               "sum_v": [float(math.fsum(vf[(cat == a) & (sub == b)])) for a, b in rows]},
                  "dtypes": {"category": "Bool", "subkey": "I64", "sum_v": "F64"}})
    # :115-125 null key is its own group
    isnull = (i % 3) == 0
    cases.append({"name": "it_null_key_own_group", "source": "tests/python_integration/test_groupby.py:115-125",
                  "formula": "null_key", "n": n, "keys": ["k"], "aggs": [["Sum", "v", "s"]],
                  "expected": {"k": [None, 1], "s": [int(i[isnull].sum()), int(i[~isnull].sum())]},
                  "dtypes": {"k": "I64", "s": "I64"}})
    # :128-149 nulls in values skipped by sum/mean/count, counted by len
    vmask = (i % 5) != 0
    vals = i.astype(np.float64)
    ks = [0, 1, 2, 3]
    cases.append({"name": "it_null_values_skipped", "source": "tests/python_integration/test_groupby.py:128-149",
                  "formula": "null_values", "n": n, "keys": ["k"],
                  "aggs": [["Sum", "v", "s"], ["Mean", "v", "m"], ["Count", "v", "c"], ["Len", None, "n"]],
                  "expected": {"k": ks,
                               "s": [float(math.fsum(vals[(i % 4 == k) & vmask])) for k in ks],
                               "m": [float(math.fsum(vals[(i % 4 == k) & vmask]) / ((i % 4 == k) & vmask).sum())
                                     for k in ks],
                               "c": [int(((i % 4 == k) & vmask).sum()) for k in ks],
                               "n": [int((i % 4 == k).sum()) for k in ks]},
                  "dtypes": {"k": "I64", "s": "F64", "m": "F64", "c": "U32", "n": "U32"}})
    # :152-162 all-unique keys (checked by properties: every group sums to 1)
    cases.append({"name": "it_all_unique_keys", "source": "tests/python_integration/test_groupby.py:152-162",
                  "formula": "all_unique", "n": n, "keys": ["k"], "aggs": [["Sum", "v", "s"]],
                  "expected": {"k": list(range(n)), "s": [1] * n}, "dtypes": {"k": "I64", "s": "I64"}})
    # :165-181 all-same key
    cases.append({"name": "it_all_same_key", "source": "tests/python_integration/test_groupby.py:165-181",
                  "formula": "all_same", "n": n, "keys": ["k"], "aggs": [["Sum", "v", "s"], ["Count", "v", "c"]],
                  "expected": {"k": [7], "s": [int(i.sum())], "c": [n]}, "dtypes": {"k": "I64", "s": "I64", "c": "U32"}})
    # :188-216 i32 key + i32 values: Polars CPU gives an f64 mean
    vi = (i % 100).astype(np.int64)
    g = grp(i % 7, vi)
    ks = sorted(g)
    cases.append({"name": "it_i32_keys_i32_values", "source": "tests/python_integration/test_groupby.py:188-216",
                  "formula": "i32_i32", "n": n, "keys": ["k"],
                  "aggs": [["Sum", "v", "s"], ["Mean", "v", "m"], ["Min", "v", "mn"], ["Max", "v", "mx"],
                           ["Count", "v", "c"], ["Len", None, "n"]],
                  "expected": {"k": ks, "s": [int(g[k][0].sum()) for k in ks],
                               "m": [float(g[k][0].sum()) / len(g[k][0]) for k in ks],
                               "mn": [int(g[k][0].min()) for k in ks], "mx": [int(g[k][0].max()) for k in ks],
                               "c": [len(g[k][0]) for k in ks], "n": [g[k][1] for k in ks]},
                  "dtypes": {"k": "I32", "s": "I32", "m": "F64", "mn": "I32", "mx": "I32", "c": "U32", "n": "U32"}})
    # :219-241 i32 key + f32 values
    v32 = (i % 100).astype(np.float32)
    g = grp(i % 5, v32)
    ks = sorted(g)
    cases.append({"name": "it_f32_values", "source": "tests/python_integration/test_groupby.py:219-241",
                  "formula": "f32_values", "n": n, "keys": ["k"], "aggs": [["Sum", "v", "s"], ["Mean", "v", "m"]],
                  "expected": {"k": ks, "s": [float(np.float32(math.fsum(g[k][0].astype(np.float64)))) for k in ks],
                               "m": [float(np.float32(math.fsum(g[k][0].astype(np.float64)) / len(g[k][0])))
                                     for k in ks]},
                  "dtypes": {"k": "I32", "s": "F32", "m": "F32"}})
    return cases


def compare_cases() -> list[dict]:
    """crates/polars-metal-kernels/tests/test_cmp_f64.rs NaN / signed-zero / special values (IEEE)."""
    ops = ["Eq", "Ne", "Lt", "Le", "Gt", "Ge"]
    fn = {"Eq": lambda a, b: a == b, "Ne": lambda a, b: a != b, "Lt": lambda a, b: a < b,
          "Le": lambda a, b: a <= b, "Gt": lambda a, b: a > b, "Ge": lambda a, b: a >= b}
    mp = 2.2250738585072014e-308
    sets = [
        ("nan_vs_value", "crates/polars-metal-kernels/tests/test_cmp_f64.rs:164-216",
         [nan(), 1.0, 2.0, nan()], [1.0, nan(), 2.0, nan()], [1, 1, 1, 1], [1, 1, 1, 1]),
        ("special_values", "crates/polars-metal-kernels/tests/test_cmp_f64.rs:318-370",
         [math.inf, -math.inf, 0.0, -0.0, mp, -mp, 1.0, -1.0], [0.0, 0.0, -0.0, 0.0, 0.0, 0.0, -1.0, 1.0],
         [1] * 8, [1] * 8),
        ("signed_zero", "crates/polars-metal-kernels/tests/test_cmp_f64.rs:372-433",
         [0.0, -0.0, 0.0, -0.0], [-0.0, 0.0, 0.0, -0.0], [1] * 4, [1] * 4),
        ("eq_with_nulls", "crates/polars-metal-kernels/tests/test_cmp_f64.rs:258-286",
         [1.0, 2.0, 3.0, 4.0], [1.0, 2.0, 3.0, 4.0], [0, 0, 1, 1], [1, 1, 1, 1]),
    ]
    out = []
    for name, src, lhs, rhs, lv, rv in sets:
        for op in ops:
            valid = [int(a and b) for a, b in zip(lv, rv)]
            data = [int(v and fn[op](a, b)) for a, b, v in zip(lhs, rhs, valid)]
            out.append({"name": f"{name}_{op}", "source": src, "op": op, "lhs": lhs, "rhs": rhs, "lhs_valid": lv,
                        "rhs_valid": rv, "expected_data": data, "expected_valid": valid})
    # test_cmp_f64.rs:218-256: NaN scalar, only != is true
    lhs = [1.0, nan(), -1.0, math.inf]
    for op in ops:
        out.append({"name": f"nan_scalar_{op}", "source": "crates/polars-metal-kernels/tests/test_cmp_f64.rs:218-256",
                    "op": op, "lhs": lhs, "scalar": nan(), "lhs_valid": [1, 1, 1, 1],
                    "expected_data": [1 if op == "Ne" else 0] * 4, "expected_valid": [1, 1, 1, 1]})
    return out


def kleene_cases() -> list[dict]:
    """shaders/logical_bool.metal:3-26 truth tables (T, F, null)."""
    vals = [("T", 1, 1), ("F", 0, 1), ("N", 0, 0)]
    and_t = {("T", "T"): "T", ("T", "F"): "F", ("T", "N"): "N", ("F", "T"): "F", ("F", "F"): "F", ("F", "N"): "F",
             ("N", "T"): "N", ("N", "F"): "F", ("N", "N"): "N"}
    or_t = {("T", "T"): "T", ("T", "F"): "T", ("T", "N"): "T", ("F", "T"): "T", ("F", "F"): "F", ("F", "N"): "N",
            ("N", "T"): "T", ("N", "F"): "N", ("N", "N"): "N"}
    rows_l, rows_r, exp_and, exp_or = [], [], [], []
    for a, _, _ in vals:
        for b, _, _ in vals:
            rows_l.append(a)
            rows_r.append(b)
            exp_and.append(and_t[(a, b)])
            exp_or.append(or_t[(a, b)])
    return [{"name": "kleene_truth_tables", "source": "shaders/logical_bool.metal:3-26", "lhs": rows_l, "rhs": rows_r,
             "and": exp_and, "or": exp_or}]


def sort_cases() -> list[dict]:
    """tests/python_integration/test_walker_sort_fused.py: Sort / top_k / bottom_k, engine vs Polars
    CPU. `spec` is the sort (by, descending, nulls_last, drop_nulls, offset, limit as Polars lowers
    top_k: descending + drop nulls + slice(0, k)). Closed-form inputs carry their values; the
    seeded float inputs (`_floats(n, seed)`: standard normal, Float32) carry a `formula`, and
    their expected values are computed from it with np.sort when the test runs."""
    def spec(by, desc=None, nl=None, drop=False, limit=-1):
        return {"by": by, "descending": desc or [False] * len(by), "nulls_last": nl or [False] * len(by),
                "drop_nulls": drop, "offset": 0, "limit": limit}

    x = [3.0, None, 1.0, 5.0, None, 2.0, 4.0]
    xv = [1, 0, 1, 1, 0, 1, 1]
    return [
        {"name": "sort_f32_ascending", "source": "tests/python_integration/test_walker_sort_fused.py:46-50",
         "columns": {"x": {"dtype": "F32", "values": [3.0, 1.0, 2.0, 2.0, 5.0, -1.0]}}, "spec": spec(["x"]),
         "expected": {"x": [-1.0, 1.0, 2.0, 2.0, 3.0, 5.0]}},
        {"name": "top_k_with_nulls", "source": "tests/python_integration/test_walker_sort_fused.py:77-83",
         "columns": {"x": {"dtype": "F32", "values": [v if v is not None else 0.0 for v in x], "valid": xv}},
         "spec": spec(["x"], [True], [True], drop=True, limit=3), "expected": {"x": [5.0, 4.0, 3.0]}},
        {"name": "bottom_k_with_nulls", "source": "tests/python_integration/test_walker_sort_fused.py:86-90",
         "columns": {"x": {"dtype": "F32", "values": [v if v is not None else 0.0 for v in x], "valid": xv}},
         "spec": spec(["x"], [False], [True], drop=True, limit=3), "expected": {"x": [1.0, 2.0, 3.0]}},
        {"name": "sort_nulls_first", "source": "tests/python_integration/test_walker_sort_fused.py:93-99",
         "columns": {"x": {"dtype": "F32", "values": [3.0, 0.0, 1.0, 0.0, 2.0], "valid": [1, 0, 1, 0, 1]}},
         "spec": spec(["x"]), "expected": {"x": [None, None, 1.0, 2.0, 3.0]}},
        {"name": "sort_carries_other_columns", "source": "tests/python_integration/test_walker_sort_fused.py:102-113",
         "columns": {"x": {"dtype": "F32", "values": [3.0, 1.0, 2.0]}, "y": {"dtype": "I64", "values": [10, 20, 30]}},
         "spec": spec(["x"]), "expected": {"x": [1.0, 2.0, 3.0], "y": [20, 30, 10]}},
        {"name": "sort_i64", "source": "tests/python_integration/test_walker_sort_fused.py:116-122",
         "columns": {"x": {"dtype": "I64", "values": [3, 1, 2, 5, 4]}}, "spec": spec(["x"]),
         "expected": {"x": [1, 2, 3, 4, 5]}},
        {"name": "sort_floats_ascending", "source": "tests/python_integration/test_walker_sort_fused.py:38-43",
         "formula": {"n": 10_000, "seed": 0x501}, "spec": spec(["x"])},
        {"name": "sort_floats_descending", "source": "tests/python_integration/test_walker_sort_fused.py:53-57",
         "formula": {"n": 5_000, "seed": 0x501}, "spec": spec(["x"], [True])},
        {"name": "top_k_100", "source": "tests/python_integration/test_walker_sort_fused.py:60-67",
         "formula": {"n": 10_000, "seed": 0x501}, "spec": spec(["x"], [True], [True], drop=True, limit=100)},
        {"name": "bottom_k_100", "source": "tests/python_integration/test_walker_sort_fused.py:70-74",
         "formula": {"n": 10_000, "seed": 0x501}, "spec": spec(["x"], [False], [True], drop=True, limit=100)},
    ]


def expression_cases() -> list[dict]:
    """tests/python_integration/test_walker_expression_unfolding.py: group-by aggregates of
    arithmetic expressions, engine vs Polars CPU. Inputs are closed forms (`formula`, built by
    tests/helpers.py expression_columns); an expression is in the reference's aggregation wire
    shape (Column / LiteralF64 / Binary). Expected sums: every row's product rounded to f64 as
    Polars computes it, then summed exactly (math.fsum)."""
    def col(c):
        return {"kind": "Column", "name": c}

    def lit(x):
        return {"kind": "LiteralF64", "value": x}

    def binop(op, a, b):
        return {"kind": "Binary", "op": op, "lhs": a, "rhs": b}

    cases = []
    k, a, b = [0, 0, 1, 1, 2, 2], [1.0, 2.0, 3.0, 4.0, 5.0, 6.0], [0.1, 0.2, 0.3, 0.4, 0.5, 0.6]
    rows = [(kk, aa * bb) for kk, aa, bb in zip(k, a, b)]
    cases.append({"name": "sum_a_times_b", "source": "tests/python_integration/test_walker_expression_unfolding.py:17-35",
                  "formula": "sum_a_times_b", "n": 6000, "keys": ["k"],
                  "aggs": [{"kind": "Expression", "op": "Sum", "output_alias": "sum_ab",
                            "expr": binop("Mul", col("a"), col("b"))}],
                  "expected": {"k": [0, 1, 2], "sum_ab": [math.fsum([p for kk, p in rows if kk == g] * 1000)
                                                          for g in (0, 1, 2)]}})
    k, a, b = [0, 0, 1, 1], [10.0, 20.0, 30.0, 40.0], [0.05, 0.1, 0.15, 0.2]
    rows = [(kk, aa * (1.0 - bb)) for kk, aa, bb in zip(k, a, b)]
    cases.append({"name": "sum_a_times_one_minus_b",
                  "source": "tests/python_integration/test_walker_expression_unfolding.py:38-56",
                  "formula": "sum_a_times_one_minus_b", "n": 20000, "keys": ["k"],
                  "aggs": [{"kind": "Expression", "op": "Sum", "output_alias": "disc",
                            "expr": binop("Mul", col("a"), binop("Sub", lit(1.0), col("b")))}],
                  "expected": {"k": [0, 1], "disc": [math.fsum([p for kk, p in rows if kk == g] * 5000)
                                                     for g in (0, 1)]}})
    e = col("v")
    for _ in range(5):
        e = binop("Add", e, lit(1.0))
    cases.append({"name": "depth_5_chain", "source": "tests/python_integration/test_walker_expression_unfolding.py:68-78",
                  "formula": "depth_5_chain", "n": 100, "keys": ["k"],
                  "aggs": [{"kind": "Expression", "op": "Sum", "output_alias": "s", "expr": e}],
                  "expected": {"k": [0], "s": [600.0]}})
    return cases


def compare_i64_cases() -> list[dict]:
    """crates/polars-metal-kernels/tests/test_cmp_i64.rs known answers: column-column and
    column-scalar compares with nulls, an unaligned row count, extreme values. `scalar` marks a
    column-scalar case; expected bits written out from each test's assertions."""
    src = "crates/polars-metal-kernels/tests/test_cmp_i64.rs"
    lo, hi = -(1 << 63), (1 << 63) - 1
    cases = [
        {"name": "lt_basic", "source": f"{src}:127-153", "op": "Lt", "lhs": [1, 2, 3, 4, 5, 6, 7, 8], "rhs": [5] * 8,
         "lhs_valid": [1] * 8, "rhs_valid": [1] * 8, "expected_data": [1, 1, 1, 1, 0, 0, 0, 0],
         "expected_valid": [1] * 8},
        {"name": "eq_with_nulls", "source": f"{src}:156-183", "op": "Eq", "lhs": [10] * 4, "rhs": [10] * 4,
         "lhs_valid": [0, 0, 1, 1], "rhs_valid": [1] * 4, "expected_data": [0, 0, 1, 1], "expected_valid": [0, 0, 1, 1]},
        {"name": "lt_scalar_basic", "source": f"{src}:186-208", "op": "Lt", "lhs": list(range(8)), "scalar": 4,
         "lhs_valid": [1] * 8, "expected_data": [1, 1, 1, 1, 0, 0, 0, 0], "expected_valid": [1] * 8},
        {"name": "scalar_with_nulls", "source": f"{src}:211-237", "op": "Lt", "lhs": list(range(8)), "scalar": 5,
         "lhs_valid": [1, 0, 1, 0, 1, 0, 1, 0], "expected_data": [1, 0, 1, 0, 1, 0, 0, 0],
         "expected_valid": [1, 0, 1, 0, 1, 0, 1, 0]},
        {"name": "unaligned_row_count", "source": f"{src}:344-387", "op": "Lt", "lhs": list(range(13)), "rhs": [6] * 13,
         "lhs_valid": [1] * 13, "rhs_valid": [1] * 13, "expected_data": [1] * 6 + [0] * 7, "expected_valid": [1] * 13},
        {"name": "extreme_values", "source": f"{src}:501-528", "op": "Lt", "lhs": [lo, -1, 0, 1, hi], "rhs": [0] * 5,
         "lhs_valid": [1] * 5, "rhs_valid": [1] * 5, "expected_data": [1, 1, 0, 0, 0], "expected_valid": [1] * 5},
    ]
    return cases


def pipeline_cases() -> list[dict]:
    """crates/polars-metal-kernels/tests/test_groupby_pipeline.rs known answers (sum and len of an
    i64 column per i64 key; the empty input; a single row). Expected rows in key order."""
    src = "crates/polars-metal-kernels/tests/test_groupby_pipeline.rs"
    n = 1024
    return [
        {"name": "four_groups_single_i64_key", "source": f"{src}:244-316",
         "columns": {"a": {"dtype": "I64", "values": [i % 4 for i in range(n)]},
                     "v": {"dtype": "I64", "values": list(range(n))}},
         "keys": ["a"], "aggs": [["Sum", "v", "s"], ["Len", None, "n"]],
         "expected": {"a": [0, 1, 2, 3], "s": [sum(i for i in range(n) if i % 4 == k) for k in range(4)],
                      "n": [256] * 4},
         "dtypes": {"a": "I64", "s": "I64", "n": "U32"}},
        {"name": "empty_input", "source": f"{src}:319-359",
         "columns": {"k": {"dtype": "I64", "values": []}, "v": {"dtype": "I64", "values": []}},
         "keys": ["k"], "aggs": [["Sum", "v", "s"]], "expected": {"k": [], "s": []},
         "dtypes": {"k": "I64", "s": "I64"}},
        {"name": "single_row", "source": f"{src}:362-407",
         "columns": {"k": {"dtype": "I64", "values": [42]}, "v": {"dtype": "I64", "values": [100]}},
         "keys": ["k"], "aggs": [["Sum", "v", "s"]], "expected": {"k": [42], "s": [100]},
         "dtypes": {"k": "I64", "s": "I64"}},
    ]


def compact_cases() -> list[dict]:
    """crates/polars-metal-kernels/tests/test_compaction_pipeline.rs known answers: columns
    compacted by a predicate bitmap (keep = data & valid). `columns` holds the inputs; the expected
    kept values follow each test's assertions (a `formula` stands for a long closed form)."""
    src = "crates/polars-metal-kernels/tests/test_compaction_pipeline.rs"
    even = [1, 0] * 8
    nan_ = nan()
    return [
        {"name": "i64_basic", "source": f"{src}:139-161", "columns": {"a": {"dtype": "I64", "values": list(range(16))}},
         "pred_data": even, "pred_valid": [1] * 16, "expected": {"a": list(range(0, 16, 2))}},
        {"name": "i64_empty_result", "source": f"{src}:164-183", "columns": {"a": {"dtype": "I64", "values": list(range(8))}},
         "pred_data": [0] * 8, "pred_valid": [1] * 8, "expected": {"a": []}},
        {"name": "i64_all_kept", "source": f"{src}:208-227", "columns": {"a": {"dtype": "I64", "values": list(range(16))}},
         "pred_data": [1] * 16, "pred_valid": [1] * 16, "expected": {"a": list(range(16))}},
        {"name": "i64_threadgroup_boundary_10k", "source": f"{src}:230-259", "formula": "keep_mod3", "n": 10_000},
        {"name": "reusable_across_columns", "source": f"{src}:262-295",
         "columns": {"a": {"dtype": "I64", "values": list(range(16))},
                     "b": {"dtype": "I64", "values": list(range(100, 116))}},
         "pred_data": even, "pred_valid": [1] * 16,
         "expected": {"a": list(range(0, 16, 2)), "b": list(range(100, 116, 2))}},
        {"name": "f64_preserves_nan", "source": f"{src}:298-326",
         "columns": {"a": {"dtype": "F64", "values": [1.0, nan_, 3.0, nan_]}},
         "pred_data": [1] * 4, "pred_valid": [1] * 4, "expected": {"a": [1.0, nan_, 3.0, nan_]}},
        {"name": "bool_round_trips", "source": f"{src}:329-349",
         "columns": {"a": {"dtype": "Bool", "values": [0, 0, 1, 0, 1, 1, 0, 1]}},
         "pred_data": [1] * 8, "pred_valid": [1] * 8, "expected": {"a": [False, False, True, False, True, True, False, True]}},
        {"name": "i64_single_row", "source": f"{src}:352-374", "columns": {"a": {"dtype": "I64", "values": [42]}},
         "pred_data": [1], "pred_valid": [1], "expected": {"a": [42]}},
        {"name": "null_predicate_drops_row", "source": f"{src}:377-401",
         "columns": {"a": {"dtype": "I64", "values": [10, 20, 30, 40]}},
         "pred_data": [1, 1, 1, 1], "pred_valid": [0, 1, 0, 1], "expected": {"a": [20, 40]}},
        # test_filter_scatter_f64.rs / test_filter_scatter_bool.rs: source nulls keep their place
        {"name": "f64_null_inputs_stay_null", "source": "crates/polars-metal-kernels/tests/test_filter_scatter_f64.rs:220-245",
         "columns": {"a": {"dtype": "F64", "values": [i * 1.5 for i in range(8)], "valid": [1, 1, 0, 1, 1, 0, 1, 1]}},
         "pred_data": [1] * 8, "pred_valid": [1] * 8,
         "expected": {"a": [0.0, 1.5, None, 4.5, 6.0, None, 9.0, 10.5]}},
        {"name": "bool_null_propagates", "source": "crates/polars-metal-kernels/tests/test_filter_scatter_bool.rs:151-189",
         "columns": {"a": {"dtype": "Bool", "values": [1] * 8, "valid": [1, 1, 0, 1, 1, 0, 1, 1]}},
         "pred_data": [1] * 8, "pred_valid": [1] * 8,
         "expected": {"a": [True, True, None, True, True, None, True, True]}},
        {"name": "bool_unaligned_row_count", "source": "crates/polars-metal-kernels/tests/test_filter_scatter_bool.rs:404-440",
         "columns": {"a": {"dtype": "Bool", "values": [0, 1, 0, 1, 0, 1, 0, 1, 1, 1, 1, 0, 0]}},
         "pred_data": [1] * 13, "pred_valid": [1] * 13,
         "expected": {"a": [False, True, False, True, False, True, False, True, True, True, True, False, False]}},
    ]


def sort_build_cases() -> list[dict]:
    """The sort build's known answers (crates/polars-metal-kernels/tests/test_groupby_segment.rs,
    test_groupby_build_sort_reference.rs): group counts of key lanes, here as an Int64 key column
    with the rows per group (Len), expected in key order."""
    seg = "crates/polars-metal-kernels/tests/test_groupby_segment.rs"
    ref = "crates/polars-metal-kernels/tests/test_groupby_build_sort_reference.rs"

    def case(name, source, keys):
        ks = sorted(set(keys))
        return {"name": name, "source": source, "columns": {"k": {"dtype": "I64", "values": keys}},
                "keys": ["k"], "aggs": [["Len", None, "n"]],
                "expected": {"k": ks, "n": [keys.count(k) for k in ks]}, "dtypes": {"k": "I64", "n": "U32"}}

    return [
        case("empty_input", f"{seg}:9-14", []),
        case("all_same_100", f"{seg}:17-23", [42] * 100),
        case("all_distinct_200", f"{seg}:26-31", list(range(200))),
        case("all_unique_1000", f"{ref}:10-14", list(range(1000))),
        case("duplicates_collapsed", f"{ref}:25-33", [10, 20, 10, 30, 20, 10]),
    ]


def predicate_mask_cases() -> list[dict]:
    """crates/polars-metal-kernels/tests/test_filter_predicate.rs: a predicate's (data, valid) bits
    to the keep mask, keep = data & valid, bits past the last row ignored."""
    src = "crates/polars-metal-kernels/tests/test_filter_predicate.rs"
    return [
        {"name": "all_true_no_nulls", "source": f"{src}:31-43", "data": [1] * 16, "valid": [1] * 16,
         "n": 16, "expected": [1] * 16},
        {"name": "null_rows_mask_to_zero", "source": f"{src}:46-54", "data": [1] * 8, "valid": [1, 1, 1, 1, 0, 0, 0, 0],
         "n": 8, "expected": [1, 1, 1, 1, 0, 0, 0, 0]},
        {"name": "false_rows_mask_to_zero", "source": f"{src}:57-65", "data": [1, 1, 1, 1, 0, 0, 0, 0], "valid": [1] * 8,
         "n": 8, "expected": [1, 1, 1, 1, 0, 0, 0, 0]},
        {"name": "empty_input", "source": f"{src}:68-78", "data": [], "valid": [], "n": 0, "expected": []},
        {"name": "padding_bits_ignored", "source": f"{src}:81-96", "data": [1, 0, 1, 1, 1, 1, 0, 1], "valid": [1] * 8,
         "n": 7, "expected": [1, 0, 1, 1, 1, 1, 0]},
    ]


def polars_shape_cases() -> list[dict]:
    """Engine-vs-Polars cases of the reference's Python integration tests with closed-form inputs
    (small integer keys, string keys, several chunks, filter edges). A case gives its table as
    `chunks` (a list of column dicts, each list one chunk; None is a null), the query (`keys`,
    `aggs`, optional `predicate` in the wire shape, or `filter` alone), and the expected rows in the
    order the test sorts them (`expected`, by column). Float sums are exact sums (math.fsum). A long
    column is a generator: {"gen": "mod", "m", "n"} is i % m, {"gen": "scale", "c", "n"} is i * c,
    {"gen": "tile", "values", "times"} repeats the values, and `chunk_rows` cuts a generated table
    into chunks of that many rows (tests/helpers.py shape_table builds them)."""
    it = "tests/python_integration"
    cases = []

    def grouped(rows, keyf, vals, n_keys=1):
        out = {}
        for r in rows:
            out.setdefault(keyf(r), []).append(vals(r))
        return out

    def sort_key(k):
        return tuple((0, "") if x is None else (1, x) for x in (k if isinstance(k, tuple) else (k,)))

    n = 10_000
    for tag, src in (("Int8", "22-23"), ("Int16", "26-27"), ("Int32", "30-32"), ("UInt8", "35-36")):
        g = grouped(range(n), lambda i: i % 4, lambda i: i * 1.5)
        ks = sorted(g)
        cases.append({"name": f"small_int_key_{tag}", "source": f"{it}/test_groupby_small_int_keys.py:{src}",
                      "chunks": [{"k": {"gen": "mod", "m": 4, "n": n}, "v": {"gen": "scale", "c": 1.5, "n": n}}],
                      "dtypes": {"k": tag, "v": "Float64"}, "keys": ["k"], "aggs": [["Sum", "v", "v"], ["Len", None, "len"]],
                      "expected": {"k": ks, "v": [math.fsum(g[k]) for k in ks], "len": [len(g[k]) for k in ks]}})
    g = grouped(range(n), lambda i: (i % 4, i % 8), lambda i: i * 1.5)
    ks = sorted(g)
    cases.append({"name": "u16_u32_mixed_keys", "source": f"{it}/test_groupby_small_int_keys.py:39-49",
                  "chunks": [{"k1": {"gen": "mod", "m": 4, "n": n}, "k2": {"gen": "mod", "m": 8, "n": n},
                              "v": {"gen": "scale", "c": 1.5, "n": n}}],
                  "dtypes": {"k1": "UInt16", "k2": "UInt32", "v": "Float64"}, "keys": ["k1", "k2"], "aggs": [["Sum", "v", "v"]],
                  "expected": {"k1": [a for a, _ in ks], "k2": [b for _, b in ks], "v": [math.fsum(g[k]) for k in ks]}})

    def string_case(name, src, pattern, times, keys, dtypes):
        cols = {c: vals * times for c, vals in pattern.items()}
        m = len(cols["v"])
        g = grouped(range(m), lambda i: tuple(cols[k][i] for k in keys), lambda i: cols["v"][i])
        ks = sorted(g, key=sort_key)
        exp = {k: [key[j] for key in ks] for j, k in enumerate(keys)}
        exp["s"] = [math.fsum(g[key]) for key in ks]
        chunk = {c: {"gen": "tile", "values": vals, "times": times} for c, vals in pattern.items()}
        return {"name": name, "source": src, "chunks": [chunk], "dtypes": dtypes, "keys": keys,
                "aggs": [["Sum", "v", "s"]], "expected": exp}

    cases.append(string_case("string_low_cardinality", f"{it}/test_string_groupby.py:17-27",
                             {"k": ["A", "B", "A", "C", "B", "A"], "v": [1.0, 2.0, 3.0, 4.0, 5.0, 6.0]}, 1000,
                             ["k"], {"k": "Utf8", "v": "Float64"}))
    cases.append(string_case("string_null_keys", f"{it}/test_string_groupby.py:30-40",
                             {"k": ["A", None, "A", "B", None, "B"], "v": [1.0, 2.0, 3.0, 4.0, 5.0, 6.0]}, 100,
                             ["k"], {"k": "Utf8", "v": "Float64"}))
    cases.append(string_case("string_and_int_keys", f"{it}/test_string_groupby.py:43-54",
                             {"k_s": ["X", "Y", "X", "Z"], "k_i": [1, 2, 1, 3], "v": [1.0, 2.0, 3.0, 4.0]}, 1000,
                             ["k_s", "k_i"], {"k_s": "Utf8", "k_i": "Int64", "v": "Float64"}))

    def chunked_case(name, src, chunks, dtypes, predicate=None, keep=lambda v: True):
        ks_all = [k for c in chunks for k in c["k"]]
        vs_all = [v for c in chunks for v in c["v"]]
        g = grouped([i for i in range(len(vs_all)) if keep(vs_all[i])], lambda i: ks_all[i], lambda i: vs_all[i])
        ks = sorted(g, key=sort_key)
        case = {"name": name, "source": src, "chunks": chunks, "dtypes": dtypes, "keys": ["k"],
                "aggs": [["Sum", "v", "s"]], "expected": {"k": ks, "s": [math.fsum(g[k]) for k in ks]}}
        if predicate:
            case["predicate"] = predicate
        return case

    cases.append(chunked_case("two_chunks", f"{it}/test_multichunk.py:19-29",
                              [{"k": [0, 0, 1, 1], "v": [1.0, 2.0, 3.0, 4.0]}, {"k": [0, 1, 0, 1], "v": [5.0, 6.0, 7.0, 8.0]}],
                              {"k": "Int64", "v": "Float64"}))
    c = chunked_case("thousand_chunks", f"{it}/test_multichunk.py:32-41",
                     [{"k": [i % 4], "v": [float(i)]} for i in range(1000)], {"k": "Int64", "v": "Float64"})
    # stored as one generated table cut into 1000 one-row chunks
    c["chunks"] = [{"k": {"gen": "mod", "m": 4, "n": 1000}, "v": {"gen": "scale", "c": 1.0, "n": 1000}}]
    c["chunk_rows"] = 1
    cases.append(c)
    cases.append(chunked_case("string_keys_two_chunks", f"{it}/test_multichunk.py:44-54",
                              [{"k": ["A", "A", "B"], "v": [1.0, 2.0, 3.0]}, {"k": ["B", "C", "A"], "v": [4.0, 5.0, 6.0]}],
                              {"k": "Utf8", "v": "Float64"}))
    cases.append(chunked_case("filter_two_chunks", f"{it}/test_multichunk.py:57-67",
                              [{"k": [0, 1, 2, 0], "v": [10.0, 20.0, 30.0, 40.0]}, {"k": [1, 2, 0, 1], "v": [50.0, 60.0, 70.0, 80.0]}],
                              {"k": "Int64", "v": "Float64"},
                              predicate={"kind": "Compare", "op": "Gt", "dtype": "F64", "lhs": {"kind": "Column", "name": "v"},
                                         "rhs": {"kind": "LiteralF64", "value": 25.0}},
                              keep=lambda v: v > 25.0))

    # test_filter_edges.py: top-level filters; `expected` = the kept rows of every column
    fe = f"{it}/test_filter_edges.py"

    def col_(c):
        return {"kind": "Column", "name": c}

    def cmp_(op, l, r, dt):
        return {"kind": "Compare", "op": op, "dtype": dt, "lhs": l, "rhs": r}

    def filt(name, src, cols, dtypes, pred, kept_rows):
        return {"name": name, "source": f"{fe}:{src}", "chunks": [cols], "dtypes": dtypes, "filter": pred,
                "expected": {c: [cols[c][i] for i in kept_rows] for c in cols}}

    lit0 = {"kind": "LiteralI64", "value": 0}
    cases += [
        filt("empty_frame", "23-29", {"a": []}, {"a": "Int64"}, cmp_("Gt", col_("a"), lit0, "I64"), []),
        filt("single_row_true", "32-36", {"a": [5], "mask": [True]}, {"a": "Int64", "mask": "Bool"}, col_("mask"), [0]),
        filt("single_row_false", "39-43", {"a": [5], "mask": [False]}, {"a": "Int64", "mask": "Bool"}, col_("mask"), []),
        filt("single_row_null", "46-51", {"a": [5], "mask": [None]}, {"a": "Int64", "mask": "Bool"}, col_("mask"), []),
        filt("all_null_column", "54-60", {"a": [None] * 4}, {"a": "Int64"}, cmp_("Gt", col_("a"), lit0, "I64"), []),
        filt("predicate_all_true", "63-70", {"a": [1, 2, 3, 4], "b": [10, 20, 30, 40]}, {"a": "Int64", "b": "Int64"},
             cmp_("Eq", col_("a"), col_("a"), "I64"), [0, 1, 2, 3]),
        filt("predicate_all_false", "73-79", {"a": [1, 2, 3, 4], "b": [10, 20, 30, 40]}, {"a": "Int64", "b": "Int64"},
             cmp_("Ne", col_("a"), col_("a"), "I64"), []),
        filt("predicate_all_null", "82-93", {"a": [1, 2, 3, 4], "mask": [None] * 4}, {"a": "Int64", "mask": "Bool"},
             col_("mask"), []),
        filt("predicate_empty_subset", "95-101", {"a": [1, 2, 3, 4], "b": [10, 20, 30, 40]}, {"a": "Int64", "b": "Int64"},
             cmp_("Gt", col_("a"), {"kind": "LiteralI64", "value": 1000}, "I64"), []),
        filt("finite_f64_predicate", "104-110", {"x": [-1.5, 0.0, 1.5, 2.5]}, {"x": "Float64"},
             cmp_("Gt", col_("x"), {"kind": "LiteralF64", "value": 0.0}, "F64"), [2, 3]),
    ]
    return cases


def main():
    doc = {"groupby": groupby_cases(), "integration": integration_cases(), "compare": compare_cases(),
           "kleene": kleene_cases(), "sort": sort_cases(),
           "expression": expression_cases(), "compare_i64": compare_i64_cases(), "pipeline": pipeline_cases(),
           "compact": compact_cases(), "sort_build": sort_build_cases(),
           "predicate_mask": predicate_mask_cases(), "polars_shapes": polars_shape_cases()}
    # the all-unique case is large; keep only its shape and check it by property
    for c in doc["integration"]:
        if c["formula"] == "all_unique":
            c["expected"] = {"n_groups": 200_000, "s_all": 1}
    OUT.write_text(json.dumps(doc, indent=0, allow_nan=True))
    print(OUT, OUT.stat().st_size)


if __name__ == "__main__":
    main()
