"""polars_b200 — B200 (sm_100a) implementation of polars-metal's filter -> group_by -> aggregate path.

The compute lives in libpmb.so (CUDA kernels + C ABI, declared in include/pmb.h); this package
is the host-side mirror of the reference's `_native` operator surface.
"""

from ._native import (  # noqa: F401
    ColumnData,
    GroupByResult,
    Handle,
    bool_and_dispatch,
    bool_or_dispatch,
    cmp_f64_col_col,
    cmp_f64_col_scalar,
    cmp_i64_col_col,
    cmp_i64_col_scalar,
    cumsum_u8_to_u32,
    default_handle,
    execute_filter_compact,
    execute_groupby,
    execute_sort,
    bottom_k,
    eval_expr,
    filter_columns,
    groupby,
    groupby_batched,
    sort_columns,
    top_k,
)

__version__ = "0.1.0"
