/*
 * pmb.h — C ABI of libpmb, the B200 (sm_100a) implementation of polars-metal's
 * filter -> group_by -> fused-aggregate path.
 *
 * Every entry point is plain C: pointers, sizes and status codes, no C++ or torch
 * types. Each declaration names the reference interface it replaces
 * (file:line inside the dbfclark/polars-metal tree).
 *
 * Conventions shared by all entry points
 *   - Return value: PMB_OK (0) or a PMB_E_* code; pmb_last_error() gives text.
 *   - Columns follow the Arrow layout the reference's buffer crate uses
 *     (crates/polars-metal-buffer/src/null_bitmap.rs:29-92): dense little-endian
 *     values (Bool bit-packed LSB-first) and an optional validity bitmap,
 *     LSB-first, 1 = valid, NULL = all rows valid.
 *   - `on_device` = 1 means the pointer is CUDA device memory on the handle's
 *     device; 0 means host memory (pinned or pageable), copied in by the call.
 *   - A handle owns one CUDA stream and one device workspace; it is not
 *     thread-safe. Use one handle per host thread.
 *   - Results are owned by the library until pmb_result_free(). Device-resident
 *     result buffers live in the handle's workspace and stay valid until the next
 *     call on the same handle.
 */
#ifndef PMB_H
#define PMB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (EngineError mapping: crates/polars-metal-core/src/error.rs:19-34) ---- */
enum {
  PMB_OK = 0,
  PMB_E_INVALID = 1,     /* bad argument / buffer too short  (PyValueError)          */
  PMB_E_OOM = 2,         /* device or host allocation failed                          */
  PMB_E_TIMEOUT = 3,     /* a bounded device wait gave up; the context stays usable   */
  PMB_E_CUDA = 4,        /* a CUDA runtime call failed                                */
  PMB_E_UNSUPPORTED = 5, /* valid request outside this build (PyNotImplementedError)  */
  PMB_E_NOT_FOUND = 6    /* a referenced column index does not exist (PyKeyError)     */
};

/* ---- dtypes: the reference's wire tags (crates/polars-metal-core/src/plan/mod.rs MetalDtype) ---- */
enum {
  PMB_BOOL = 0,
  PMB_I8 = 1,
  PMB_I16 = 2,
  PMB_I32 = 3,
  PMB_I64 = 4,
  PMB_U8 = 5,
  PMB_U16 = 6,
  PMB_U32 = 7,
  PMB_U64 = 8,
  PMB_F32 = 9,
  PMB_F64 = 10
};

/* One Arrow-layout column (replaces the `(name, tag, data: bytes, valid: bytes)` tuples of
 * `_native.execute_groupby`, crates/polars-metal-core/src/udf/groupby/mod.rs:747-820). */
typedef struct pmb_column {
  const void* data;        /* values at row 0 of the array (before `offset`)          */
  const uint8_t* validity; /* Arrow validity bitmap or NULL (= all valid)              */
  int64_t length;          /* rows in this column                                      */
  int64_t offset;          /* Arrow row offset applied to data and validity            */
  int32_t dtype;           /* PMB_* dtype                                              */
  int32_t on_device;       /* 1 = device pointers, 0 = host pointers                   */
} pmb_column;

/* ---- Arrow C Data Interface and C Device Data Interface (the Apache Arrow specification's
 *      stable ABI, declared here under its own guards as the specification asks) ---- */
#ifndef ARROW_C_DATA_INTERFACE
#define ARROW_C_DATA_INTERFACE
#define ARROW_FLAG_DICTIONARY_ORDERED 1
#define ARROW_FLAG_NULLABLE 2
#define ARROW_FLAG_MAP_KEYS_SORTED 4
struct ArrowSchema {
  const char* format;
  const char* name;
  const char* metadata;
  int64_t flags;
  int64_t n_children;
  struct ArrowSchema** children;
  struct ArrowSchema* dictionary;
  void (*release)(struct ArrowSchema*);
  void* private_data;
};
struct ArrowArray {
  int64_t length;
  int64_t null_count;
  int64_t offset;
  int64_t n_buffers;
  int64_t n_children;
  const void** buffers;
  struct ArrowArray** children;
  struct ArrowArray* dictionary;
  void (*release)(struct ArrowArray*);
  void* private_data;
};
#endif
#ifndef ARROW_C_DEVICE_DATA_INTERFACE
#define ARROW_C_DEVICE_DATA_INTERFACE
typedef int32_t ArrowDeviceType;
#define ARROW_DEVICE_CPU 1
#define ARROW_DEVICE_CUDA 2
#define ARROW_DEVICE_CUDA_HOST 3
struct ArrowDeviceArray {
  struct ArrowArray array;
  int64_t device_id;
  ArrowDeviceType device_type;
  void* sync_event;
  int64_t reserved[3];
};
#endif

/* A column over an exported Arrow array's own buffers, without a copy: the values buffer, the
 * validity bitmap (NULL when the array has no nulls) and the array's offset. Primitive formats
 * b c C s S i I l L f g (Bool, Int8..UInt64, Float32, Float64); a dictionary-encoded array gives
 * its integer codes: such a column is only meaningful as a group key (group by the codes, then
 * decode through the dictionary); summing, comparing or filtering it works on the codes, not on
 * the dictionary's values. `pmb_column_is_dictionary` tells such arrays apart. Returns
 * PMB_E_UNSUPPORTED for other formats and PMB_E_INVALID for a malformed or released array. The
 * array stays owned by its producer and must outlive every call that reads the column.
 * Replaces the reference's Arrow -> Metal buffer bridge (crates/polars-metal-buffer/src/bridge.rs:1-60)
 * and the Python copies it is fed from (python/polars_metal/_udf.py:1441-1456). No GPU is
 * touched; no handle is needed. */
int pmb_column_from_arrow(const struct ArrowArray* array, const struct ArrowSchema* schema, pmb_column* out);

/* The same for an array of the C Device Data Interface: ARROW_DEVICE_CUDA buffers give a device
 * column (used in place by the kernels), ARROW_DEVICE_CPU and ARROW_DEVICE_CUDA_HOST a host one.
 * A CUDA array must live on the calling thread's current CUDA device (`device_id` equal to it, and
 * the handle that reads the column opened on that device): another device's array returns
 * PMB_E_INVALID, and a process without a usable CUDA device PMB_E_UNSUPPORTED. The handle checks
 * the pointers of every device column again when a call stages them.
 * A non-NULL `sync_event` (a cudaEvent_t* for CUDA) is left to the caller to wait on before the
 * column is used. Other device types return PMB_E_UNSUPPORTED. */
int pmb_column_from_arrow_device(const struct ArrowDeviceArray* array, const struct ArrowSchema* schema,
                                 pmb_column* out);

/* 1 when `schema` describes a dictionary-encoded array (its column holds codes: use it only as a
 * group key), 0 when it does not, PMB_E_INVALID for a NULL or released schema. The reference keeps
 * the dictionary beside the codes in its Utf8 key path (crates/polars-metal-buffer/src/dict.rs:18-74). */
int pmb_column_is_dictionary(const struct ArrowSchema* schema);

/* ---- predicate expression (PredicateAst, crates/polars-metal-core/src/plan/mod.rs:42-60,
 *      plus the Arith / Not / IsNull nodes this build adds) ---- */
enum {
  PMB_EXPR_COLUMN = 0,
  PMB_EXPR_LIT_I64 = 1,
  PMB_EXPR_LIT_F64 = 2,
  PMB_EXPR_LIT_BOOL = 3,
  PMB_EXPR_COMPARE = 4,
  PMB_EXPR_AND = 5,
  PMB_EXPR_OR = 6,
  PMB_EXPR_NOT = 7,
  PMB_EXPR_ARITH = 8,
  PMB_EXPR_IS_NULL = 9,
  PMB_EXPR_IS_NOT_NULL = 10
};
enum { PMB_CMP_EQ = 0, PMB_CMP_NE = 1, PMB_CMP_LT = 2, PMB_CMP_LE = 3, PMB_CMP_GT = 4, PMB_CMP_GE = 5 };
enum {
  PMB_ARITH_ADD = 0,
  PMB_ARITH_SUB = 1,
  PMB_ARITH_MUL = 2,
  PMB_ARITH_TRUEDIV = 3,  /* always F64 */
  PMB_ARITH_FLOORDIV = 4,
  PMB_ARITH_MOD = 5       /* floor modulo: result takes the divisor's sign; x % 0 is null for ints */
};

typedef struct pmb_expr_node {
  int32_t kind;    /* PMB_EXPR_*                                                  */
  int32_t op;      /* PMB_CMP_* for COMPARE, PMB_ARITH_* for ARITH                */
  int32_t lhs;     /* child node index (-1 when unused)                           */
  int32_t rhs;     /* child node index (-1 when unused)                           */
  int32_t column;  /* column index for PMB_EXPR_COLUMN                            */
  int32_t dtype;   /* operand dtype for COMPARE / ARITH: PMB_I64 or PMB_F64       */
  int64_t lit_i64; /* LIT_I64 value; LIT_BOOL uses 0/1                            */
  double lit_f64;  /* LIT_F64 value                                               */
} pmb_expr_node;

typedef struct pmb_expr {
  const pmb_expr_node* nodes;
  int32_t n_nodes;
  int32_t root;
} pmb_expr;

/* ---- aggregations (AggOp, crates/polars-metal-core/src/plan/mod.rs:62-70) ---- */
enum { PMB_AGG_SUM = 0, PMB_AGG_MEAN = 1, PMB_AGG_COUNT = 2, PMB_AGG_MIN = 3, PMB_AGG_MAX = 4, PMB_AGG_LEN = 5 };
typedef struct pmb_agg {
  int32_t op;     /* PMB_AGG_*                                  */
  int32_t column; /* input column index; ignored for PMB_AGG_LEN */
} pmb_agg;

/* ---- group-by strategies (build archetypes A1/A2/A3 of crates/polars-metal-kernels/src/groupby.rs:450-538) ---- */
enum {
  PMB_STRATEGY_AUTO = 0,        /* sketch + learned selector, heuristic fallback   */
  PMB_STRATEGY_SMEM_HASH = 1,   /* per-CTA shared-memory tables + small global merge */
  PMB_STRATEGY_GLOBAL_HASH = 2, /* global open addressing with a shared-memory hot cache */
  PMB_STRATEGY_SORT = 3,        /* packed-key LSD radix sort + segmented reduce   */
  PMB_STRATEGY_PARTITIONED = 4  /* rows scattered by key-hash partition, then one
                                   shared-memory table per partition            */
};

typedef struct pmb_query {
  const int32_t* key_columns; /* indices into the column array                     */
  int32_t n_keys;
  const pmb_agg* aggs;
  int32_t n_aggs;
  const pmb_expr* predicate;  /* NULL = no filter                                  */
  int32_t strategy;           /* PMB_STRATEGY_*                                    */
  int32_t output_on_device;   /* 1 = result columns in device memory               */
  int64_t capacity_hint;      /* expected distinct groups; 0 = let the library pick */
} pmb_query;

typedef struct pmb_out_column {
  void* data;        /* values; Bool outputs bit-packed                             */
  uint8_t* validity; /* bitmap, LSB-first, padded to a 4-byte multiple (never NULL) */
  int64_t length;
  int32_t dtype;
  int32_t on_device;
} pmb_out_column;

typedef struct pmb_result {
  int64_t n_groups;         /* rows in every output column                        */
  int32_t n_columns;        /* group-by: keys then aggs; filter: one per input   */
  pmb_out_column* columns;
  int32_t strategy_used;    /* PMB_STRATEGY_* actually executed                   */
  int32_t rehash_count;     /* capacity overflows retried with a larger table     */
  int64_t capacity;         /* hash slots of the final attempt (0 for sort)       */
} pmb_result;

typedef struct pmb_handle pmb_handle;

/* Per-call timing record, filled when profiling is enabled (pmb_set_profiling). */
#define PMB_MAX_STAT_KERNELS 16
typedef struct pmb_stats {
  int32_t n_kernels;
  int32_t launches[PMB_MAX_STAT_KERNELS];
  float ms[PMB_MAX_STAT_KERNELS];        /* device time per kernel name, summed over launches */
  char names[PMB_MAX_STAT_KERNELS][32];
  float total_ms;                        /* device time of the whole call                     */
  int64_t h2d_bytes;
  int64_t d2h_bytes;
  int32_t kernel_launches;               /* every kernel this call launched                   */
} pmb_stats;

/* ---- lifetime ---- */

/* Creates a handle on `device` with an initial device workspace (grown on demand).
 * Replaces MetalDevice::system_default + CommandQueue::new
 * (crates/polars-metal-core/src/udf/groupby/mod.rs:996-1000, crates/polars-metal-kernels/src/command.rs:95). */
int pmb_open(pmb_handle** out, int32_t device, uint64_t workspace_bytes);
void pmb_close(pmb_handle* h);
/* Last error text of this handle (EngineError's Display, crates/polars-metal-core/src/error.rs:19-34). */
const char* pmb_last_error(const pmb_handle* h);
/* Makes the handle launch on an existing cudaStream_t (NULL = the handle's own stream). */
int pmb_set_stream(pmb_handle* h, void* cuda_stream);
/* 1 = record per-kernel CUDA-event timings of every call (readable with pmb_last_stats). */
int pmb_set_profiling(pmb_handle* h, int32_t enabled);
int pmb_last_stats(const pmb_handle* h, pmb_stats* out);
/* Library version string. */
const char* pmb_version(void);

/* ---- the hot path ---- */

/* filter -> group_by -> fused aggregate in one call.
 * Replaces `_native.execute_groupby(plan_dict, n_rows, columns)`
 * (crates/polars-metal-core/src/udf/groupby/mod.rs:747-1144) together with the CPU
 * filter it is fed from (`_filter_via_polars`, python/polars_metal/_udf.py:550-597).
 * Output columns: keys (in key order) then one column per aggregation. */
int pmb_groupby(pmb_handle* h, const pmb_query* q, const pmb_column* cols, int32_t n_cols,
                pmb_result** out);

/* Many independent queries in one persistent launch over a device work queue.
 * No reference counterpart (new batching layer); each query follows pmb_groupby's semantics and
 * results. cols[i] holds n_cols[i] columns of query i; outs[i] receives query i's result.
 * Two or more queries of one signature (same column dtypes and nullability, keys, aggregates and
 * filter; keys of at most 64 packed bits; strategy AUTO, no capacity hint) run batched: one
 * sampling launch, one run-time compiled persistent kernel over all their rows, one finalize,
 * replayed from a CUDA graph while the launch shape repeats. Otherwise the queries run one by one
 * through pmb_groupby with host outputs (a device output request then returns PMB_E_UNSUPPORTED).
 * Device outputs stay valid until the next call on the handle. */
int pmb_groupby_batched(pmb_handle* h, const pmb_query* qs, const pmb_column* const* cols,
                        const int32_t* n_cols, int32_t n_queries, pmb_result** outs);

/* 0 = pmb_groupby_batched runs every query alone through pmb_groupby, in a loop inside the
 * library (host outputs only): the plain single-query form of a batch, without the batching; 1 =
 * batch where it can (the default). No reference counterpart (the reference runs one query per
 * call). */
int pmb_set_batching(pmb_handle* h, int32_t enabled);

/* Order of rows for pmb_sort_columns and pmb_groupby_sorted: `by` lists column indices, most
 * significant first; `descending` and `nulls_last` hold one flag per `by` column (NULL = all 0:
 * ascending, nulls first). Polars' order: NaN above every number, -0.0 equal to 0.0, nulls placed
 * by `nulls_last` whatever the direction. Rows with equal sort keys keep their input order.
 * `drop_nulls` = 1 leaves out the rows whose first `by` column is null (top_k / bottom_k). Then the
 * slice of the sorted rows is kept as Polars' `slice(offset, length)` takes it: `offset` < 0
 * counts from the end, `limit` < 0 keeps every row from `offset` on. */
typedef struct pmb_sort_spec {
  const int32_t* by;
  const int32_t* descending;
  const int32_t* nulls_last;
  int32_t n_by;
  int32_t drop_nulls;
  int64_t offset;
  int64_t limit;
} pmb_sort_spec;

/* The rows of `cols` (all of them, at most 2^32 - 1) reordered by the spec; one output column per
 * input column. Replaces the CPU sort of the reference's Sort plans (`df.sort(by, descending,
 * nulls_last)` then the slice, python/polars_metal/_udf.py:684-721) and its single-column F32
 * sort routed to MLX (_build_sort_fused, python/polars_metal/_udf.py:724-790). */
int pmb_sort_columns(pmb_handle* h, const pmb_column* cols, int32_t n_cols, const pmb_sort_spec* spec,
                     int32_t output_on_device, pmb_result** out);

/* pmb_groupby, then the sort of its result on the device in the same call (the result does not
 * leave the device in between): `spec->by` indexes the result's columns (keys first, then the
 * aggregations). A Sort over a GroupBy (`_build_sort` with a GroupBy input,
 * python/polars_metal/_udf.py:684-721). */
int pmb_groupby_sorted(pmb_handle* h, const pmb_query* q, const pmb_column* cols, int32_t n_cols,
                       const pmb_sort_spec* spec, pmb_result** out);

/* Frees a result. Host output buffers come from the C library's allocator (malloc, or
 * posix_memalign for large ones) and each non-NULL one is released with free(): a caller may take
 * a buffer over by setting its pointer in the result to NULL and calling free() on it later.
 * Device outputs live in the handle's workspace and are not freed here. */
void pmb_result_free(pmb_result* r);

/* ---- many results at once (bindings that read a batch's results) ----
 * No counterpart in the reference, whose batch of one query per call returns one PyO3 tuple per
 * call. pmb_results_pack copies the headers of n results into one array of 64-bit words: per
 * result 4 words (n_groups; n_columns | strategy_used << 32; rehash_count; capacity), then 4 per
 * column (data; validity; length; dtype | on_device << 32). A NULL result packs as 0 columns.
 * It returns the words written, or -1 when they do not fit in cap_words. The addresses stay the
 * results' own: pack before pmb_results_free, and read device addresses only while they are valid.
 * pmb_results_free is pmb_result_free of each of the n results. */
int64_t pmb_results_pack(pmb_result* const* rs, int32_t n, uint64_t* words, int64_t cap_words);
void pmb_results_free(pmb_result* const* rs, int32_t n);

/* Releases one host buffer of a result column that the caller took over: it copied the column's
 * data or validity pointer and set it to NULL in the result, so pmb_result_free leaves it. Host
 * buffers of 1 MB and more are page-locked blocks of a pool that the library recycles (the copy
 * back from the device then needs no staging and no page faults); they must come back through
 * here, not through free(). No counterpart in the reference, whose results are PyO3 objects. */
void pmb_host_buffer_free(void* p);

/* ---- learned strategy selection ----
 * No counterpart in the reference, whose routing is a row-count threshold and an estimated-
 * cardinality gate (crates/polars-metal-core/src/router/cost.rs:35-52,
 * crates/polars-metal-kernels/src/groupby.rs:475-486). A query's features are computed on the
 * device from a 4096-row sample of its keys (HyperLogLog registers, hash-bucket occupancy, null
 * and filter fractions, sample frequency profile, key width); an MLP (PMB_SELECTOR_FEATURES ->
 * 64 -> 64 -> 5, fp32) maps them to four strategy scores (shared-memory hash, global hash, sort,
 * partitioned) and log2 of the group count, which sizes the hash table. Without installed
 * parameters, or for a non-finite output, the plain cardinality heuristic decides (with its
 * switch to the partitioned strategy for many groups and no heavy key). The strategy never
 * changes a result: every strategy is exact, and an undersized table is rebuilt larger. */
#define PMB_SELECTOR_FEATURES 24
#define PMB_SELECTOR_HIDDEN 64
#define PMB_SELECTOR_STRATEGIES 4
#define PMB_SELECTOR_OUTPUTS (PMB_SELECTOR_STRATEGIES + 1)
/* parameter count: W1[64][24] b1[64] W2[64][64] b2[64] W3[5][64] b3[5], in that order */
#define PMB_SELECTOR_PARAMS                                                                   \
  (PMB_SELECTOR_HIDDEN * PMB_SELECTOR_FEATURES + PMB_SELECTOR_HIDDEN +                       \
   PMB_SELECTOR_HIDDEN * PMB_SELECTOR_HIDDEN + PMB_SELECTOR_HIDDEN +                         \
   PMB_SELECTOR_OUTPUTS * PMB_SELECTOR_HIDDEN + PMB_SELECTOR_OUTPUTS)

/* Features of a group-by query (filter applied) into `out` (host, PMB_SELECTOR_FEATURES floats). */
int pmb_selector_features(pmb_handle* h, const pmb_query* q, const pmb_column* cols, int32_t n_cols, float* out);
/* Installs selector parameters (host, PMB_SELECTOR_PARAMS floats) on the handle; NULL removes them. */
int pmb_selector_set(pmb_handle* h, const float* params, int32_t n_params);
/* The strategy and group count the handle's AUTO strategy would use for this query. */
int pmb_selector_choose(pmb_handle* h, const pmb_query* q, const pmb_column* cols, int32_t n_cols,
                        int32_t* strategy, int64_t* groups);
/* MLP kernels on device buffers (params, features x[batch][24], outputs out[batch][4]). */
int pmb_mlp_forward(pmb_handle* h, const float* params, const float* x, int32_t batch, float* out);
/* Gradient of the mean loss over the batch, sum_b sw[b] * (CE(softmax(out[b][0:3]), cls[b]) +
 * wreg * (out[b][3] - y[b])^2) / batch (sw may be NULL for all ones), into grad (overwritten),
 * and that loss into *loss (device float). */
int pmb_mlp_gradient(pmb_handle* h, const float* params, const float* x, const int32_t* cls, const float* y,
                     const float* sw, int32_t batch, float wreg, float* grad, float* loss);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8; `step` counts from 1) on device buffers. */
int pmb_mlp_adam_step(pmb_handle* h, float* params, const float* grad, float* m, float* v, int32_t step, float lr);

/* ---- the operator surface on the filter side ---- */

/* Null-aware comparison -> bit-packed (data, validity); rhs == NULL compares with the scalar
 * (rhs_i64 for PMB_I64 columns, rhs_f64 for PMB_F64). Output buffers must hold
 * max(4, round_up_4(ceil(n/8))) bytes each and live where `out_on_device` says.
 * Replaces `_native.cmp_{i64,f64}_col_{col,scalar}` (crates/polars-metal-core/src/udf/compare.rs:23-145)
 * and dispatch_cmp_* (crates/polars-metal-kernels/src/cmp.rs:180-641). */
int pmb_compare(pmb_handle* h, const pmb_column* lhs, const pmb_column* rhs, int64_t rhs_i64,
                double rhs_f64, int32_t op, uint8_t* out_data, uint8_t* out_valid,
                int32_t out_on_device);

/* Kleene AND / OR of two bit-packed nullable Boolean columns of n rows.
 * Replaces `_native.bool_{and,or}_dispatch` (crates/polars-metal-core/src/udf/logical.rs:26-55). */
int pmb_bool_and(pmb_handle* h, const uint8_t* lhs_data, const uint8_t* lhs_valid,
                 const uint8_t* rhs_data, const uint8_t* rhs_valid, int64_t n, uint8_t* out_data,
                 uint8_t* out_valid, int32_t on_device);
int pmb_bool_or(pmb_handle* h, const uint8_t* lhs_data, const uint8_t* lhs_valid,
                const uint8_t* rhs_data, const uint8_t* rhs_valid, int64_t n, uint8_t* out_data,
                uint8_t* out_valid, int32_t on_device);

/* One arithmetic expression of columns and literals (PMB_EXPR_COLUMN, _LIT_I64, _LIT_F64 and
 * _ARITH nodes, at most 8 levels and 32 nodes) evaluated for every row into `out_data` and
 * `out_valid` (a bit-packed bitmap): the input column of an expression aggregate. Types follow
 * Polars: each node computes in the supertype of its operands (literals take the other operand's
 * type; an integer true division is Float64), wrapping or rounding to it, and `*out_dtype`
 * receives the root's type; `out_data` holds one value of that type a row (allocate 8 bytes a row
 * to take any). A null operand, or an integer // or % by zero, gives null.
 * Replaces the expression side of the reference's Expression aggregations
 * (crates/polars-metal-core/src/udf/groupby/mod.rs:266-352, python/polars_metal/_walker.py:1205-1278). */
int pmb_eval_expr(pmb_handle* h, const pmb_expr* expr, const pmb_column* cols, int32_t n_cols, void* out_data,
                  uint8_t* out_valid, int32_t out_on_device, int32_t* out_dtype);

/* The type pmb_eval_expr gives an expression over these columns (only their dtypes are read); no
 * GPU is touched and no handle is needed. PMB_E_INVALID for an expression pmb_eval_expr refuses. */
int pmb_expr_dtype(const pmb_expr* expr, const pmb_column* cols, int32_t n_cols, int32_t* out_dtype);

/* Stream compaction of `cols` by a bit-packed predicate (keep = data & valid).
 * Replaces `_native.execute_filter_compact(pred_data, pred_valid, n_rows, columns)`
 * (crates/polars-metal-core/src/udf/compact.rs:46-147) and compute_keep_and_prefix +
 * compact_* (crates/polars-metal-kernels/src/pipeline.rs:103-270). */
int pmb_filter_compact(pmb_handle* h, const uint8_t* pred_data, const uint8_t* pred_valid,
                       int64_t n_rows, int32_t pred_on_device, const pmb_column* cols,
                       int32_t n_cols, int32_t output_on_device, pmb_result** out);

/* Same compaction with the predicate evaluated on the device from an expression. */
int pmb_filter_compact_expr(pmb_handle* h, const pmb_expr* predicate, const pmb_column* cols,
                            int32_t n_cols, int32_t output_on_device, pmb_result** out);

/* Inclusive prefix sum of n bytes into n uint32 values.
 * Replaces polars-metal-mlx-sys `cumsum_u8_to_u32(&[u8], &mut [u32])`
 * (crates/polars-metal-mlx-sys/src/lib.rs:47, cxx/mlx_bridge.cc:59-89). */
int pmb_cumsum_u8_to_u32(pmb_handle* h, const uint8_t* in, uint32_t* out, int64_t n,
                         int32_t on_device);

/* The same prefix sum for callers that must not allocate device memory (a host framework that
 * already reserved the device's memory for its own pool, or a latency-critical loop in which
 * cudaMalloc/cudaFree would synchronise the device). No counterpart in the reference.
 * `in` and `out` are device pointers of n elements on the current device; `cuda_stream` may be
 * NULL. The call allocates nothing: its scratch is a fixed array of about 256 KB that every GPU
 * loading this library holds until the process exits, so n may be at most PMB_NOALLOC_MAX_ROWS
 * (larger n returns PMB_E_INVALID without touching the GPU). The first call on a device looks up
 * that array's device address, so make it before capturing work on that device. All calls share
 * the array: calls that overlap on the GPU (other streams or host threads) race. The call waits
 * for its stream before returning. Returns PMB_OK, PMB_E_INVALID, PMB_E_TIMEOUT or PMB_E_CUDA. */
#define PMB_NOALLOC_MAX_ROWS (1LL << 27)
int pmb_cumsum_u8_to_u32_noalloc(const uint8_t* in, uint32_t* out, int64_t n, void* cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* PMB_H */
