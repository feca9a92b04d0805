"""The product against more of the reference's known-answer tests: i64 compares
(test_cmp_i64.rs), the group-by pipeline (test_groupby_pipeline.rs) and compaction
(test_compaction_pipeline.rs), through the reference's wire functions."""

import numpy as np
import pytest

from helpers import (as_dict, assert_results_match, case_columns, compact_case_expected, compact_case_inputs,
                     expected_to_result, load_golden, pack, same_values, unpack)
from polars_b200 import _abi as A
from polars_b200 import _native as N

pytestmark = pytest.mark.gpu
GOLD = load_golden()


@pytest.mark.parametrize("case", GOLD["compare_i64"], ids=lambda c: c["name"])
def test_compare_i64_known_answers(case):
    n = len(case["lhs"])
    lhs = np.array(case["lhs"], np.int64).tobytes()
    lv = pack(case["lhs_valid"]).tobytes()
    if "scalar" in case:
        d, v = N.cmp_i64_col_scalar(lhs, lv, case["scalar"], case["op"], n)
    else:
        d, v = N.cmp_i64_col_col(lhs, lv, np.array(case["rhs"], np.int64).tobytes(), pack(case["rhs_valid"]).tobytes(),
                                 case["op"], n)
    valid = list(unpack(np.frombuffer(v, np.uint8), n).astype(int))
    assert valid == case["expected_valid"]
    data = unpack(np.frombuffer(d, np.uint8), n).astype(int)
    assert [b for b, ok in zip(data, valid) if ok] == [b for b, ok in zip(case["expected_data"], valid) if ok]
    # bits past the last row stay zero
    assert not np.unpackbits(np.frombuffer(d, np.uint8), bitorder="little")[n:].any()


@pytest.mark.parametrize("case", GOLD["pipeline"], ids=lambda c: c["name"])
def test_pipeline_known_answers(case):
    cols = {k: N.ColumnData(v[0], v[1], dtype=v[2], length=v[3]) for k, v in case_columns(case).items()}
    got = N.groupby(cols, case["keys"], [tuple(a) for a in case["aggs"]])
    assert_results_match(as_dict(got), expected_to_result(case), len(case["keys"]), case["aggs"], case["name"])


@pytest.mark.parametrize("case", GOLD["compact"], ids=lambda c: c["name"])
def test_compaction_known_answers(case):
    cols, pd, pv, n = compact_case_inputs(case)
    columns = []
    for name, (data, valid, dt, m) in cols.items():
        vb = (np.asarray(valid, np.uint8) if valid is not None else np.full(max(1, (m + 7) // 8), 255, np.uint8)).tobytes()
        columns.append((A.DTYPE_TO_TAG[dt], np.asarray(data).tobytes(), vb))
    out = N.execute_filter_compact(pack(pd).tobytes(), pack(pv).tobytes(), n, columns)
    want = compact_case_expected(case)
    for (name, vals), (_d, _v, dt, _m), (db, vbytes, n_out) in zip(want.items(), cols.values(), out):
        assert n_out == len(vals)
        if dt == A.BOOL:
            got = [bool(x) for x in unpack(np.frombuffer(db, np.uint8), n_out)] if n_out else []
        else:
            got = np.frombuffer(db, A.NUMPY_NAME[dt])[:n_out].tolist()
        ok = list(unpack(np.frombuffer(vbytes, np.uint8), n_out)) if n_out else []
        assert ok == [v is not None for v in vals], name
        assert same_values([g for g, o in zip(got, ok) if o], [v for v in vals if v is not None]), name


@pytest.mark.parametrize("strategy", ["sort", "partitioned", "global_hash", "smem_hash"])
@pytest.mark.parametrize("case", GOLD["sort_build"], ids=lambda c: c["name"])
def test_sort_build_known_answers(case, strategy):
    cols = {k: N.ColumnData(v[0], v[1], dtype=v[2], length=v[3]) for k, v in case_columns(case).items()}
    got = N.groupby(cols, case["keys"], [tuple(a) for a in case["aggs"]], strategy=strategy)
    assert_results_match(as_dict(got), expected_to_result(case), 1, case["aggs"], f"{case['name']} {strategy}")
