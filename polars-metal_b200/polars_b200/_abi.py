"""ctypes mirror of include/pmb.h and the loader of libpmb.so.

The library is the product: every compute call goes through it. There is no CPU path in this
package; when the shared library cannot be loaded, `lib()` raises.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libpmb.so"

# ---- status codes
PMB_OK = 0
PMB_E_INVALID = 1
PMB_E_OOM = 2
PMB_E_TIMEOUT = 3
PMB_E_CUDA = 4
PMB_E_UNSUPPORTED = 5
PMB_E_NOT_FOUND = 6

# ---- dtypes (wire tags of the reference, crates/polars-metal-core/src/plan/mod.rs MetalDtype)
BOOL, I8, I16, I32, I64, U8, U16, U32, U64, F32, F64 = range(11)
TAG_TO_DTYPE = {
    "Bool": BOOL,
    "I8": I8,
    "I16": I16,
    "I32": I32,
    "I64": I64,
    "U8": U8,
    "U16": U16,
    "U32": U32,
    "U64": U64,
    "F32": F32,
    "F64": F64,
    "Date": I32,
}
DTYPE_TO_TAG = {v: k for k, v in TAG_TO_DTYPE.items() if k != "Date"}
DTYPE_BYTES = {BOOL: 0, I8: 1, I16: 2, I32: 4, I64: 8, U8: 1, U16: 2, U32: 4, U64: 8, F32: 4, F64: 8}
NUMPY_NAME = {
    I8: "int8",
    I16: "int16",
    I32: "int32",
    I64: "int64",
    U8: "uint8",
    U16: "uint16",
    U32: "uint32",
    U64: "uint64",
    F32: "float32",
    F64: "float64",
}

# ---- expression nodes
EXPR_COLUMN, EXPR_LIT_I64, EXPR_LIT_F64, EXPR_LIT_BOOL, EXPR_COMPARE, EXPR_AND, EXPR_OR, EXPR_NOT = range(8)
EXPR_ARITH, EXPR_IS_NULL, EXPR_IS_NOT_NULL = 8, 9, 10
CMP_OPS = {"Eq": 0, "Ne": 1, "Lt": 2, "Le": 3, "Gt": 4, "Ge": 5}
ARITH_OPS = {"Add": 0, "Sub": 1, "Mul": 2, "TrueDiv": 3, "FloorDiv": 4, "Mod": 5}

# ---- aggregations
AGG_OPS = {"Sum": 0, "Mean": 1, "Count": 2, "Min": 3, "Max": 4, "Len": 5}
AGG_LEN = 5

# ---- strategies
STRATEGIES = {"auto": 0, "smem_hash": 1, "global_hash": 2, "sort": 3, "partitioned": 4}
STRATEGY_NAMES = {v: k for k, v in STRATEGIES.items()}


class Column(C.Structure):
    _fields_ = [
        ("data", C.c_void_p),
        ("validity", C.c_void_p),
        ("length", C.c_int64),
        ("offset", C.c_int64),
        ("dtype", C.c_int32),
        ("on_device", C.c_int32),
    ]


class ExprNode(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("op", C.c_int32),
        ("lhs", C.c_int32),
        ("rhs", C.c_int32),
        ("column", C.c_int32),
        ("dtype", C.c_int32),
        ("lit_i64", C.c_int64),
        ("lit_f64", C.c_double),
    ]


class Expr(C.Structure):
    _fields_ = [("nodes", C.POINTER(ExprNode)), ("n_nodes", C.c_int32), ("root", C.c_int32)]


class Agg(C.Structure):
    _fields_ = [("op", C.c_int32), ("column", C.c_int32)]


class Query(C.Structure):
    _fields_ = [
        ("key_columns", C.POINTER(C.c_int32)),
        ("n_keys", C.c_int32),
        ("aggs", C.POINTER(Agg)),
        ("n_aggs", C.c_int32),
        ("predicate", C.POINTER(Expr)),
        ("strategy", C.c_int32),
        ("output_on_device", C.c_int32),
        ("capacity_hint", C.c_int64),
    ]


class OutColumn(C.Structure):
    _fields_ = [
        ("data", C.c_void_p),
        ("validity", C.c_void_p),
        ("length", C.c_int64),
        ("dtype", C.c_int32),
        ("on_device", C.c_int32),
    ]


class Result(C.Structure):
    _fields_ = [
        ("n_groups", C.c_int64),
        ("n_columns", C.c_int32),
        ("columns", C.POINTER(OutColumn)),
        ("strategy_used", C.c_int32),
        ("rehash_count", C.c_int32),
        ("capacity", C.c_int64),
    ]


class SortSpec(C.Structure):
    _fields_ = [
        ("by", C.POINTER(C.c_int32)),
        ("descending", C.POINTER(C.c_int32)),
        ("nulls_last", C.POINTER(C.c_int32)),
        ("n_by", C.c_int32),
        ("drop_nulls", C.c_int32),
        ("offset", C.c_int64),
        ("limit", C.c_int64),
    ]


class ArrowSchema(C.Structure):
    pass


ArrowSchema._fields_ = [
    ("format", C.c_char_p),
    ("name", C.c_char_p),
    ("metadata", C.c_char_p),
    ("flags", C.c_int64),
    ("n_children", C.c_int64),
    ("children", C.POINTER(C.POINTER(ArrowSchema))),
    ("dictionary", C.POINTER(ArrowSchema)),
    ("release", C.c_void_p),
    ("private_data", C.c_void_p),
]


class ArrowArray(C.Structure):
    pass


ArrowArray._fields_ = [
    ("length", C.c_int64),
    ("null_count", C.c_int64),
    ("offset", C.c_int64),
    ("n_buffers", C.c_int64),
    ("n_children", C.c_int64),
    ("buffers", C.POINTER(C.c_void_p)),
    ("children", C.POINTER(C.POINTER(ArrowArray))),
    ("dictionary", C.POINTER(ArrowArray)),
    ("release", C.c_void_p),
    ("private_data", C.c_void_p),
]


class ArrowDeviceArray(C.Structure):
    _fields_ = [
        ("array", ArrowArray),
        ("device_id", C.c_int64),
        ("device_type", C.c_int32),
        ("sync_event", C.c_void_p),
        ("reserved", C.c_int64 * 3),
    ]


ARROW_DEVICE_CPU, ARROW_DEVICE_CUDA, ARROW_DEVICE_CUDA_HOST = 1, 2, 3

MAX_STAT_KERNELS = 16


class Stats(C.Structure):
    _fields_ = [
        ("n_kernels", C.c_int32),
        ("launches", C.c_int32 * MAX_STAT_KERNELS),
        ("ms", C.c_float * MAX_STAT_KERNELS),
        ("names", (C.c_char * 32) * MAX_STAT_KERNELS),
        ("total_ms", C.c_float),
        ("h2d_bytes", C.c_int64),
        ("d2h_bytes", C.c_int64),
        ("kernel_launches", C.c_int32),
    ]


# every entry point declared in include/pmb.h: name -> (restype, argtypes)
_H = C.c_void_p
_P = C.c_void_p
SIGNATURES = {
    "pmb_open": (C.c_int, [C.POINTER(_H), C.c_int32, C.c_uint64]),
    "pmb_close": (None, [_H]),
    "pmb_last_error": (C.c_char_p, [_H]),
    "pmb_set_stream": (C.c_int, [_H, _P]),
    "pmb_set_profiling": (C.c_int, [_H, C.c_int32]),
    "pmb_set_batching": (C.c_int, [_H, C.c_int32]),
    "pmb_last_stats": (C.c_int, [_H, C.POINTER(Stats)]),
    "pmb_version": (C.c_char_p, []),
    "pmb_groupby": (C.c_int, [_H, C.POINTER(Query), C.POINTER(Column), C.c_int32, C.POINTER(C.POINTER(Result))]),
    "pmb_groupby_batched": (
        C.c_int,
        [_H, C.POINTER(Query), C.POINTER(C.POINTER(Column)), C.POINTER(C.c_int32), C.c_int32,
         C.POINTER(C.POINTER(Result))],
    ),
    "pmb_result_free": (None, [C.POINTER(Result)]),
    "pmb_results_pack": (C.c_int64, [_P, C.c_int32, _P, C.c_int64]),
    "pmb_results_free": (None, [_P, C.c_int32]),
    "pmb_host_buffer_free": (None, [_P]),
    "pmb_column_from_arrow": (C.c_int, [C.POINTER(ArrowArray), C.POINTER(ArrowSchema), C.POINTER(Column)]),
    "pmb_column_from_arrow_device": (C.c_int, [C.POINTER(ArrowDeviceArray), C.POINTER(ArrowSchema),
                                               C.POINTER(Column)]),
    "pmb_column_is_dictionary": (C.c_int, [C.POINTER(ArrowSchema)]),
    "pmb_sort_columns": (C.c_int, [_H, C.POINTER(Column), C.c_int32, C.POINTER(SortSpec), C.c_int32,
                                   C.POINTER(C.POINTER(Result))]),
    "pmb_groupby_sorted": (C.c_int, [_H, C.POINTER(Query), C.POINTER(Column), C.c_int32, C.POINTER(SortSpec),
                                     C.POINTER(C.POINTER(Result))]),
    "pmb_eval_expr": (C.c_int, [_H, C.POINTER(Expr), C.POINTER(Column), C.c_int32, _P, _P, C.c_int32,
                                C.POINTER(C.c_int32)]),
    "pmb_expr_dtype": (C.c_int, [C.POINTER(Expr), C.POINTER(Column), C.c_int32, C.POINTER(C.c_int32)]),
    "pmb_compare": (C.c_int, [_H, C.POINTER(Column), C.POINTER(Column), C.c_int64, C.c_double, C.c_int32, _P, _P,
                              C.c_int32]),
    "pmb_bool_and": (C.c_int, [_H, _P, _P, _P, _P, C.c_int64, _P, _P, C.c_int32]),
    "pmb_bool_or": (C.c_int, [_H, _P, _P, _P, _P, C.c_int64, _P, _P, C.c_int32]),
    "pmb_filter_compact": (C.c_int, [_H, _P, _P, C.c_int64, C.c_int32, C.POINTER(Column), C.c_int32, C.c_int32,
                                     C.POINTER(C.POINTER(Result))]),
    "pmb_filter_compact_expr": (C.c_int, [_H, C.POINTER(Expr), C.POINTER(Column), C.c_int32, C.c_int32,
                                          C.POINTER(C.POINTER(Result))]),
    "pmb_cumsum_u8_to_u32": (C.c_int, [_H, _P, _P, C.c_int64, C.c_int32]),
    "pmb_cumsum_u8_to_u32_noalloc": (C.c_int, [_P, _P, C.c_int64, _P]),
    "pmb_selector_features": (C.c_int, [_H, C.POINTER(Query), C.POINTER(Column), C.c_int32, _P]),
    "pmb_selector_set": (C.c_int, [_H, _P, C.c_int32]),
    "pmb_selector_choose": (C.c_int, [_H, C.POINTER(Query), C.POINTER(Column), C.c_int32, C.POINTER(C.c_int32),
                                      C.POINTER(C.c_int64)]),
    "pmb_mlp_forward": (C.c_int, [_H, _P, _P, C.c_int32, _P]),
    "pmb_mlp_gradient": (C.c_int, [_H, _P, _P, _P, _P, _P, C.c_int32, C.c_float, _P, _P]),
    "pmb_mlp_adam_step": (C.c_int, [_H, _P, _P, _P, _P, C.c_int32, C.c_float]),
}

# learned strategy selector (include/pmb.h)
SELECTOR_FEATURES = 24
SELECTOR_HIDDEN = 64
SELECTOR_STRATEGIES_N = 4
SELECTOR_OUTPUTS = SELECTOR_STRATEGIES_N + 1
SELECTOR_PARAMS = (SELECTOR_HIDDEN * SELECTOR_FEATURES + SELECTOR_HIDDEN + SELECTOR_HIDDEN * SELECTOR_HIDDEN
                   + SELECTOR_HIDDEN + SELECTOR_OUTPUTS * SELECTOR_HIDDEN + SELECTOR_OUTPUTS)
# strategy index of the selector's scores
SELECTOR_STRATEGIES = ["smem_hash", "global_hash", "sort", "partitioned"]

# largest n of pmb_cumsum_u8_to_u32_noalloc (its fixed scratch array)
NOALLOC_MAX_ROWS = 1 << 27

_LIB: C.CDLL | None = None


def lib() -> C.CDLL:
    """Loads libpmb.so (raises when it is missing: there is no fallback)."""
    global _LIB
    if _LIB is None:
        path = os.environ.get("PMB_LIBRARY", str(LIB_PATH))
        if not Path(path).exists():
            raise RuntimeError(
                f"libpmb.so not found at {path}; build it with `python -m polars_b200.build` "
                "(the B200 library is required, there is no CPU fallback)"
            )
        L = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB
