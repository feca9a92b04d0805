"""The C ABI without a GPU: the library loads, exports every symbol include/pmb.h declares, and
the ctypes mirror has the C layout; host-side argument checks run before any device call."""

import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from polars_b200 import _abi as A
from polars_b200 import _native as N
from polars_b200 import datagen

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "pmb.h"


def header_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pmb_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib_path():
    from polars_b200 import build

    return build.build()


def test_library_exports_every_declared_symbol(lib_path):
    lib = C.CDLL(str(lib_path))
    names = header_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_mirror_covers_the_header(lib_path):
    assert set(header_functions()) == set(A.SIGNATURES)
    A.lib()  # binds every signature


def test_struct_layouts_match_c(tmp_path):
    src = tmp_path / "sz.c"
    structs = ["pmb_column", "pmb_expr_node", "pmb_expr", "pmb_agg", "pmb_query", "pmb_out_column", "pmb_result",
               "pmb_stats", "pmb_sort_spec", "struct ArrowSchema", "struct ArrowArray", "struct ArrowDeviceArray"]
    src.write_text('#include <stdio.h>\n#include "pmb.h"\nint main(void){\n' +
                   "".join(f'printf("%zu\\n", sizeof({s}));\n' for s in structs) + "return 0;}\n")
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    sizes = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    mirror = [A.Column, A.ExprNode, A.Expr, A.Agg, A.Query, A.OutColumn, A.Result, A.Stats, A.SortSpec,
              A.ArrowSchema, A.ArrowArray, A.ArrowDeviceArray]
    assert sizes == [C.sizeof(m) for m in mirror]


def test_oracle_library_loads():
    from oracle import pyoracle

    L = pyoracle.lib()
    for sym in ("orc_groupby", "orc_filter_mask", "orc_predicate_bits", "orc_bool_logic", "orc_filter_compact",
                "orc_cumsum_u8_to_u32"):
        assert hasattr(L, sym)


def test_predicate_lowering_of_the_hash_workload():
    expr, keep = N.compile_predicate(datagen.PRED_HASH, {"key": 0, "v1": 1, "v2": 2, "v3": 3})
    kinds = [expr.nodes[i].kind for i in range(expr.n_nodes)]
    assert kinds == [A.EXPR_COLUMN, A.EXPR_LIT_F64, A.EXPR_COMPARE, A.EXPR_COLUMN, A.EXPR_LIT_I64, A.EXPR_ARITH,
                     A.EXPR_LIT_I64, A.EXPR_COMPARE, A.EXPR_AND]
    root = expr.nodes[expr.root]
    assert root.kind == A.EXPR_AND
    assert expr.nodes[5].op == A.ARITH_OPS["Mod"]


def test_wire_errors_are_raised_before_any_device_call():
    cols = [("k", "I64", np.arange(4, dtype=np.int64).tobytes(), b"\xff")]
    with pytest.raises(ValueError):
        N.execute_groupby({"aggs": []}, 4, cols)
    with pytest.raises(KeyError):
        N.execute_groupby({"keys": [["missing", "I64"]], "aggs": []}, 4, cols)
    with pytest.raises(KeyError):
        N.execute_groupby({"keys": [["k", "I64"]], "aggs": [{"input_col": "nope", "op": "Sum", "output_alias": "s"}]},
                          4, cols)
    with pytest.raises(NotImplementedError):
        N.execute_groupby({"keys": [["s", "Utf8"]], "aggs": []}, 4, cols + [("s", "Utf8", b"\0" * 8, b"\xff")])
    with pytest.raises(ValueError):
        N.execute_groupby({"keys": [["k", "I64"]], "aggs": []}, 8, cols)  # data too short
    with pytest.raises(ValueError):
        N.execute_groupby({"keys": [["k", "I64"]], "aggs": [{"input_col": "k", "op": "Median", "output_alias": "m"}]},
                          4, cols)
    with pytest.raises(ValueError):
        N.compile_predicate({"kind": "Compare", "op": "Like", "lhs": {}, "rhs": {}}, {})


def test_all_valid_bitmap_detection():
    assert N._all_valid(b"\xff\x07", 11)
    assert not N._all_valid(b"\xff\x03", 11)
    assert N._all_valid(b"", 0)


def test_pack_bits_matches_numpy():
    import torch

    m = torch.rand(1003) > 0.3
    got = datagen.pack_bits(m).numpy()
    want = np.packbits(m.numpy(), bitorder="little")
    assert np.array_equal(got, want)


def test_batched_arguments_are_the_c_structs():
    # the numpy records handed to pmb_groupby_batched read back as the C structs they stand for
    tables = datagen.make_batch(5, seed=3, max_total=20_000)
    qs = [(datagen.to_column_data(t), t.keys, t.aggs, t.predicate) for t in tables]
    qrec, ptrs, ncols, keep, names = N._batch_args(qs, "device")
    assert qrec.itemsize == C.sizeof(A.Query)
    for i, (cols, keys, aggs, _pred) in enumerate(qs):
        q = A.Query.from_address(qrec.ctypes.data + i * qrec.itemsize)
        order = list(cols)
        assert q.n_keys == len(keys) and [q.key_columns[k] for k in range(q.n_keys)] == [order.index(k) for k in keys]
        assert q.n_aggs == len(aggs)
        assert [(q.aggs[a].op, q.aggs[a].column) for a in range(q.n_aggs)] == \
            [(A.AGG_OPS[op], -1 if op == "Len" else order.index(c)) for op, c, _ in aggs]
        assert bool(q.predicate) and q.strategy == A.STRATEGIES["auto"] and q.output_on_device == 1
        assert ncols[i] == len(cols)
        col = (A.Column * len(cols)).from_address(int(ptrs[i]))
        for j, cd in enumerate(cols.values()):
            assert col[j].data == cd.data.data_ptr() and col[j].length == cd.length and col[j].dtype == cd.dtype
            assert (col[j].validity or 0) == (cd.validity.data_ptr() if cd.validity is not None else 0)
            assert col[j].on_device == 0
        assert names[i] == list(keys) + [a[2] for a in aggs]


def test_large_host_results_change_owner_small_ones_are_copied():
    import gc

    import numpy as np

    from polars_b200 import _native as N

    libc = C.CDLL(None)
    libc.malloc.restype = C.c_void_p
    libc.malloc.argtypes = [C.c_size_t]
    libc.free.argtypes = [C.c_void_p]
    big, small = 1 << 21, 4096
    oc = A.OutColumn()
    oc.data = libc.malloc(big)
    oc.validity = libc.malloc(small)
    C.memset(oc.data, 7, big)
    C.memset(oc.validity, 255, small)
    d = N._host_out(oc, "data", big, np.uint8, 0)
    v = N._host_out(oc, "validity", small, np.uint8, 0)
    assert oc.data is None          # taken over: pmb_result_free would leave it
    assert oc.validity is not None  # copied: still the result's to free
    assert d.size == big and np.all(d == 7) and np.all(v == 255)
    view = d[10:20]
    del d
    gc.collect()
    assert np.all(view == 7)        # the buffer lives while any view of it does
    libc.free(oc.validity)
    assert N._host_out(A.OutColumn(), "data", 0, np.int64, 0).size == 0


def test_results_pack_reads_headers_and_columns_in_one_array():
    import numpy as np

    from polars_b200._native import BatchResults

    lib = A.lib()
    cols = (A.OutColumn * 2)()
    cols[0].data, cols[0].validity, cols[0].length, cols[0].dtype, cols[0].on_device = 0x1000, 0x2000, 5, 7, 1
    cols[1].data, cols[1].validity, cols[1].length, cols[1].dtype, cols[1].on_device = 0x3000, 0x4000, 5, 11, 1
    r = A.Result()
    r.n_groups, r.n_columns, r.columns = 5, 2, C.cast(cols, C.POINTER(A.OutColumn))
    r.strategy_used, r.rehash_count, r.capacity = 2, 1, 1024
    rs = (C.POINTER(A.Result) * 2)(C.pointer(r), None)  # a NULL result packs as no columns
    words = np.zeros(16, dtype=np.uint64)
    assert lib.pmb_results_pack(C.cast(rs, C.c_void_p), 2, words.ctypes.data, 16) == 16
    assert lib.pmb_results_pack(C.cast(rs, C.c_void_p), 2, words.ctypes.data, 15) == -1
    assert words[:4].tolist() == [5, 2 | (2 << 32), 1, 1024]
    assert words[4:12].tolist() == [0x1000, 0x2000, 5, 7 | (1 << 32), 0x3000, 0x4000, 5, 11 | (1 << 32)]
    assert words[12:].tolist() == [0, 0, 0, 0]
    res = BatchResults(words, np.array([0, 12, 16]), [["k", "s"], []])
    assert len(res) == 2
    g = res[0]
    assert (g.n_groups, g.dtypes, g.data, g.validity, g.rehash_count, g.capacity) == (
        5, [7, 11], [0x1000, 0x3000], [0x2000, 0x4000], 1, 1024)
    assert res[-1].n_groups == 0 and res[1].data == []
    assert [x.n_groups for x in res] == [5, 0]
