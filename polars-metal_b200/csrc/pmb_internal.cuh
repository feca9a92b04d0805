// pmb_internal.cuh — shared internals of libpmb: handle, workspace arena, device helpers,
// the compiled query descriptor and the PTX wrappers for bulk copies and mbarriers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/pmb.h"
#include "pmb_device.cuh"

// ----------------------------------------------------------------------------- limits
#define PMB_MAX_COLS 16    // distinct columns one query may touch
#define PMB_MAX_KEYS 8     // key columns
#define PMB_MAX_FIELDS 24  // aggregation state fields
#define PMB_MAX_AGGS 24
#define PMB_MAX_TERMS 12   // predicate leaf terms
#define PMB_MAX_OPS 32     // predicate circuit ops

// ----------------------------------------------------------------------------- dtype helpers
__host__ __device__ inline int pmb_dtype_bytes(int dt) {
  switch (dt) {
    case PMB_BOOL: return 0;
    case PMB_I8: case PMB_U8: return 1;
    case PMB_I16: case PMB_U16: return 2;
    case PMB_I32: case PMB_U32: case PMB_F32: return 4;
    default: return 8;
  }
}
__host__ __device__ inline int pmb_dtype_bits(int dt) { return dt == PMB_BOOL ? 1 : 8 * pmb_dtype_bytes(dt); }
__host__ __device__ inline bool pmb_is_float(int dt) { return dt == PMB_F32 || dt == PMB_F64; }
__host__ __device__ inline bool pmb_is_signed(int dt) {
  return dt == PMB_I8 || dt == PMB_I16 || dt == PMB_I32 || dt == PMB_I64;
}

// Polars output dtype of an aggregation (sum of narrow ints widens to Int64, count/len are
// UInt32, mean of non-f32 input is Float64).
__host__ __device__ inline int pmb_agg_out_dtype(int op, int in_dt) {
  switch (op) {
    case PMB_AGG_COUNT: case PMB_AGG_LEN: return PMB_U32;
    case PMB_AGG_MEAN: return in_dt == PMB_F32 ? PMB_F32 : PMB_F64;
    case PMB_AGG_SUM:
      switch (in_dt) {
        case PMB_I8: case PMB_I16: case PMB_U8: case PMB_U16: return PMB_I64;
        case PMB_BOOL: return PMB_U32;
        default: return in_dt;
      }
    default: return in_dt;
  }
}

// ----------------------------------------------------------------------------- device descriptor
// A column as the kernels see it: data at row 0 (the Arrow offset already applied; 16-byte
// aligned), validity at row 0 (bit 0 = row 0; 16-byte aligned) or null.
struct DCol {
  const uint8_t* data;
  const uint8_t* valid;
  int32_t dtype;
  int32_t elem;  // bytes per value, 0 for bit-packed Bool
};

// predicate leaf: a column or a literal, read as the operand dtype (I64 or F64)
struct DLeaf {
  int32_t col;  // -1 = literal
  int32_t pad;
  int64_t i;
  double f;
};
// operand: a leaf, or `a <arith> b` computed in `adtype`
struct DOperand {
  int8_t arith;   // -1 = none, else PMB_ARITH_*
  int8_t adtype;  // PMB_I64 / PMB_F64
  int8_t pad[6];
  DLeaf a, b;
};
enum { T_CMP = 0, T_BOOLCOL = 1, T_ISNULL = 2, T_ISNOTNULL = 3, T_LITBOOL = 4 };
struct DTerm {
  int8_t kind;
  int8_t op;     // PMB_CMP_*
  int8_t dtype;  // compare dtype: PMB_I64 / PMB_F64
  int8_t pad[5];
  DOperand lhs, rhs;
};
// circuit ops: >= 0 push term k; OP_AND / OP_OR / OP_NOT combine the Kleene stack
#define OP_AND (-1)
#define OP_OR (-2)
#define OP_NOT (-3)
struct DProgram {
  int32_t n_terms;
  int32_t n_ops;  // 0 = no predicate (keep all rows)
  DTerm term[PMB_MAX_TERMS];
  int8_t ops[PMB_MAX_OPS];
};

// key field inside the packed key (bits [data_off, data_off + bits) plus an optional null bit)
struct DKey {
  int16_t col;
  int8_t nullable;
  int8_t bits;
  int16_t null_off;
  int16_t data_off;
};

// aggregation state field kinds
enum {
  F_LEN = 0,     // u32 rows
  F_CNT = 1,     // u32 non-null rows of col
  F_SUM_DD = 2,  // double-double sum (hi f64, lo f64) of a float column
  F_SUM_I = 3,   // wrapping u64 sum of an integer / bool column
  F_MIN_I = 4,   // i64 min of a signed / bool column
  F_MAX_I = 5,
  F_MIN_U = 6,   // u64 min of an unsigned column
  F_MAX_U = 7,
  F_MIN_F = 8,   // ordered-i64 key min of a float column (NaN poisons)
  F_MAX_F = 9,
  F_SUM_FX = 10  // exact fixed-point sum of a float column: 3 x u64 limb sums + u32 non-finite flags
};
struct DField {
  int8_t kind;
  int8_t fx_slot;  // F_SUM_FX: index of this column's range report in the status words
  int16_t col;
  int16_t off;     // byte offset inside the group record
  int16_t fx;      // F_SUM_FX: fraction bits F (values are summed as integers x * 2^F)
};

// output column recipe for an aggregation
struct DAggOut {
  int8_t op;
  int8_t out_dtype;
  int8_t in_dtype;
  int8_t pad;
  int16_t f_main;  // field index: sum / min / max (or -1)
  int16_t f_cnt;   // field index of the count used for mean / validity (or -1)
  int16_t f_len;   // LEN field (always present)
  int16_t pad2;
};

struct DQuery {
  int32_t n_cols;
  int32_t n_keys;
  int32_t n_fields;
  int32_t n_aggs;
  int32_t key_bits;  // total packed key width
  int32_t rec_bytes; // bytes per group record
  int64_t n_rows;
  int16_t fx_e[8];   // exact float sums: every value of slot i satisfies |x| < 2^fx_e[i]
  uint32_t valid_if_kept;  // bit c: column c is non-null in every row the filter keeps
  uint32_t pad_vk;
  DCol col[PMB_MAX_COLS];
  DKey key[PMB_MAX_KEYS];
  DField field[PMB_MAX_FIELDS];
  DAggOut agg[PMB_MAX_AGGS];
  DProgram prog;
};

// ----------------------------------------------------------------------------- handle + arena
struct KernelTiming {
  std::string name;
  cudaEvent_t start, stop;
};

struct pmb_handle {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  // device workspace: a list of blocks, bump-allocated per call; consolidated into one
  // block at the start of the next call when a call had to grow it
  struct Block {
    uint8_t* ptr;
    size_t cap;
    size_t top;
  };
  std::vector<Block> ws;
  size_t ws_cur = 0;  // block that pmb_ws_alloc bumps from (earlier blocks are full or in use)
  // pinned host staging (64 KiB) for status words, counts and the sketch histogram
  uint8_t* pinned = nullptr;
  std::string err;
  int sm_count = 148;
  int max_smem_optin = 227 * 1024;
  // pinned host staging (pmb_host_stage)
  uint8_t* hstage = nullptr;
  size_t hstage_cap = 0, hstage_used = 0, hstage_want = 0;
  // profiling
  bool profiling = false;
  bool batching = true;  // pmb_groupby_batched may batch (else: one pmb_groupby per query)
  std::vector<std::pair<uintptr_t, uintptr_t>> ptr_ok;  // device ranges of the handle's GPU seen this call
  // host phases of a call (PMB_CALL_TIMING=1 prints them to stderr at the end of the call)
  bool phase_timing = false;
  std::vector<std::pair<const char*, double>> phases;
  double phase_t0 = 0.0;
  std::vector<KernelTiming> timings;
  std::vector<cudaEvent_t> event_pool;
  size_t event_next = 0;
  cudaEvent_t call_start = nullptr, call_stop = nullptr;
  pmb_stats last_stats{};
  // strategy selector: MLP parameters on the device (nullptr: the cardinality heuristic decides)
  float* selector = nullptr;
  int32_t launches = 0;
  int64_t h2d = 0, d2h = 0;
};

// status helpers (pmb_runtime.cu)
int pmb_fail(pmb_handle* h, int code, const std::string& msg);
int pmb_cuda_check(pmb_handle* h, cudaError_t e, const char* what);
#define PMB_CUDA(h, call)                                     \
  do {                                                         \
    cudaError_t _e = (call);                                   \
    if (_e != cudaSuccess) return pmb_cuda_check((h), _e, #call); \
  } while (0)

// workspace: pmb_ws_begin starts a call (frees the previous call's device results and merges
// blocks); pmb_ws_alloc bumps 256-byte aligned chunks and adds a block when one is full, so
// earlier allocations of the same call never move. Returns nullptr when the device is full.
int pmb_ws_begin(pmb_handle* h);
// a position in the workspace, and giving back everything allocated after it (only when no device
// work still uses that memory)
struct WsMark {
  size_t blocks;
  size_t top;
};
WsMark pmb_ws_mark(const pmb_handle* h);
void pmb_ws_release(pmb_handle* h, WsMark m);
void* pmb_ws_alloc(pmb_handle* h, size_t bytes);
// pinned host staging for bulk uploads of a call: bump-allocated, reset by pmb_ws_begin, and sized
// to what the previous call asked for; nullptr when the current area is full (the caller then
// uploads from its own memory)
void* pmb_host_stage(pmb_handle* h, size_t bytes);
inline size_t pmb_align(size_t x, size_t a) { return (x + a - 1) / a * a; }

// profiling around launches (pmb_runtime.cu)
void pmb_call_begin(pmb_handle* h);
void pmb_call_end(pmb_handle* h);  // after the final stream synchronisation
void pmb_phase(pmb_handle* h, const char* name);  // host time since the previous phase mark
void pmb_kernel_begin(pmb_handle* h, const char* name);
void pmb_kernel_end(pmb_handle* h);

// result allocation (pmb_runtime.cu)
pmb_result* pmb_result_new(int32_t n_columns);

// column staging (pmb_runtime.cu): makes a device view of a column, copying host data in
// and realigning device data whose offset breaks 16-byte alignment.
int pmb_stage_column(pmb_handle* h, const pmb_column& c, int64_t n_rows, DCol* out);

// output: copies n rows of device output columns to host memory when requested
int pmb_finish_outputs(pmb_handle* h, pmb_result* r, bool to_host);

// ----------------------------------------------------------------------------- device helpers
// read the raw bits (zero-extended) of element r of a column chunk
__device__ __forceinline__ uint64_t pmb_load_bits(const uint8_t* d, int elem, int64_t r) {
  switch (elem) {
    case 0: return (d[r >> 3] >> (r & 7)) & 1u;
    case 1: return d[r];
    case 2: return reinterpret_cast<const uint16_t*>(d)[r];
    case 4: return reinterpret_cast<const uint32_t*>(d)[r];
    default: return reinterpret_cast<const uint64_t*>(d)[r];
  }
}
__device__ __forceinline__ bool pmb_valid_bit(const uint8_t* v, int64_t r) {
  return v == nullptr || ((v[r >> 3] >> (r & 7)) & 1u);
}
__device__ __forceinline__ int64_t pmb_bits_to_i64(uint64_t b, int dt) {
  switch (dt) {
    case PMB_I8: return (int8_t)b;
    case PMB_I16: return (int16_t)b;
    case PMB_I32: return (int32_t)b;
    case PMB_F32: return (int64_t)__uint_as_float((uint32_t)b);
    case PMB_F64: return (int64_t)__longlong_as_double((long long)b);
    default: return (int64_t)b;
  }
}
__device__ __forceinline__ double pmb_bits_to_f64(uint64_t b, int dt) {
  switch (dt) {
    case PMB_I8: return (double)(int8_t)b;
    case PMB_I16: return (double)(int16_t)b;
    case PMB_I32: return (double)(int32_t)b;
    case PMB_I64: return (double)(int64_t)b;
    case PMB_F32: return (double)__uint_as_float((uint32_t)b);
    case PMB_F64: return __longlong_as_double((long long)b);
    default: return (double)b;
  }
}

// decoupled look-back (Merrill & Garland 2016): tile `tile` publishes its count and learns
// the exclusive prefix of all earlier tiles. `status` entries pack a 2-bit flag (1 = local
// aggregate, 2 = inclusive prefix) above a 62-bit value and must start zeroed. Tiles must be
// numbered in launch-acquisition order (a dynamic ticket) so earlier tiles always progress.
// Called by one thread. On a bounded-spin timeout it sets PMB_ST_TIMEOUT and returns 0.
__device__ __forceinline__ unsigned long long pmb_lookback(unsigned long long* status, long long tile,
                                                           unsigned long long count, unsigned int* st) {
  const unsigned long long VAL = (1ULL << 62) - 1;
  if (tile == 0) {
    atomicExch(&status[0], (2ULL << 62) | count);
    return 0;
  }
  atomicExch(&status[tile], (1ULL << 62) | count);
  unsigned long long excl = 0;
  long long t = tile - 1;
  uint32_t spins = 0;
  while (t >= 0) {
    unsigned long long s = *((volatile unsigned long long*)&status[t]);
    unsigned long long flag = s >> 62;
    if (flag == 0) {
      if (++spins > PMB_SPIN_LIMIT) {
        atomicOr(st, PMB_ST_TIMEOUT);
        return 0;
      }
      continue;
    }
    excl += s & VAL;
    if (flag == 2) break;
    t--;
  }
  atomicExch(&status[tile], (2ULL << 62) | (excl + count));
  return excl;
}

// pmb_lookback for a whole warp (every lane calls it; all get the tile's exclusive prefix): the
// lanes read 32 predecessor states at once, so a look-back costs one L2 round trip per 32 tiles
// instead of one per tile. The window is summed up to its nearest inclusive prefix; a window that
// still holds an unpublished state before that point is read again (bounded: PMB_ST_TIMEOUT).
__device__ __forceinline__ unsigned long long pmb_lookback_warp(unsigned long long* status, long long tile,
                                                                unsigned long long count, unsigned int* st) {
  const unsigned long long VAL = (1ULL << 62) - 1;
  const int lane = threadIdx.x & 31;
  if (tile == 0) {
    if (lane == 0) atomicExch(&status[0], (2ULL << 62) | count);
    return 0;
  }
  if (lane == 0) atomicExch(&status[tile], (1ULL << 62) | count);
  unsigned long long excl = 0;
  long long top = tile - 1;
  uint32_t spins = 0;
  for (;;) {
    const long long t = top - lane;
    const unsigned long long s = t >= 0 ? *((volatile unsigned long long*)&status[t]) : (2ULL << 62);
    const unsigned flag = (unsigned)(s >> 62);
    const unsigned incl = __ballot_sync(0xffffffffu, flag == 2u), none = __ballot_sync(0xffffffffu, flag == 0u);
    const int first = incl ? __ffs(incl) - 1 : 32;
    const unsigned need = first == 32 ? 0xffffffffu : (0xffffffffu >> (31 - first));  // lanes 0..first
    if (none & need) {
      if (++spins > PMB_SPIN_LIMIT) {
        if (lane == 0) atomicOr(st, PMB_ST_TIMEOUT);
        return 0;
      }
      continue;
    }
    unsigned long long v = lane <= first ? (s & VAL) : 0ULL;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    excl += v;
    if (first < 32) break;
    top -= 32;
  }
  if (lane == 0) atomicExch(&status[tile], (2ULL << 62) | (excl + count));
  return excl;
}

// the same over states spaced `stride` apart (state of tile t at status[t * stride])
__device__ __forceinline__ unsigned long long pmb_lookback_strided(unsigned long long* status, long long tile,
                                                                   long long stride, unsigned long long count,
                                                                   unsigned int* st) {
  const unsigned long long VAL = (1ULL << 62) - 1;
  if (tile == 0) {
    atomicExch(&status[0], (2ULL << 62) | count);
    return 0;
  }
  atomicExch(&status[tile * stride], (1ULL << 62) | count);
  unsigned long long excl = 0;
  long long t = tile - 1;
  uint32_t spins = 0;
  while (t >= 0) {
    unsigned long long s = *((volatile unsigned long long*)&status[t * stride]);
    unsigned long long flag = s >> 62;
    if (flag == 0) {
      if (++spins > PMB_SPIN_LIMIT) {
        atomicOr(st, PMB_ST_TIMEOUT);
        return 0;
      }
      continue;
    }
    excl += s & VAL;
    if (flag == 2) break;
    t--;
  }
  atomicExch(&status[tile * stride], (2ULL << 62) | (excl + count));
  return excl;
}
