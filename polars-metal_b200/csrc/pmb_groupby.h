// pmb_groupby.h — kernel parameter blocks and finalisation helpers of the hash group-by.
#pragma once

#include "pmb_plan.h"

struct RecInit {
  uint64_t w[48];  // identity record words (records up to 384 bytes)
};

// parameters of k_hash_agg (passed as a __grid_constant__ kernel parameter)
struct HashParams {
  DQuery q;
  RecInit rec_init;
  int32_t tile_rows;
  int32_t stages;
  int32_t n_staged;
  int32_t staged_col[PMB_MAX_COLS];
  int32_t stage_data_off[PMB_MAX_COLS];  // per compact column, offset inside a stage
  int32_t stage_valid_off[PMB_MAX_COLS];
  int32_t stage_bytes;       // bytes per stage (padded)
  int32_t stage_bytes_used;  // bytes the bulk copies of one tile deliver
  int32_t stage_region_off;
  int32_t smem_slots;        // shared table slots (0 = no shared table)
  int32_t smem_probe;
  int32_t smem_keys_off;
  int32_t smem_recs_off;
  int32_t tail_rows;
  int64_t n_full_tiles;
  unsigned long long* gkeys;  // global table keys, gcap + 1 slots (the last is the EMPTY-key slot)
  uint8_t* grecs;             // global records, (gcap + 1) * rec_bytes
  uint64_t gcap;
  int32_t gprobe;
  unsigned int* status;       // [0] status bits, [1] EMPTY-key slot used
  unsigned long long* kstats; // optional phase counters (PMB_KSTATS=1), else nullptr
  // hot keys (heaviest keys of the sketch sample): per-warp private records, no atomics
  const unsigned long long* hot_keys;
  const unsigned int* hot_n;  // device count (<= hot_cap)
  int32_t hot_cap;
  int32_t hot_lut_slots;      // power of two >= 2 * hot_cap
  int32_t hot_lut_off;        // shared: u64 keys[hot_lut_slots] then int idx[hot_lut_slots]
  int32_t hot_recs_off;       // shared: warps * hot_cap records
  // warm keys (next heaviest): preloaded into the CTA-shared table
  const unsigned long long* warm_keys;
  const unsigned int* warm_n;
};

#define PMB_MAX_OUT (PMB_MAX_KEYS + PMB_MAX_AGGS)

struct FinParams {
  DQuery q;
  const unsigned long long* gkeys;
  const uint8_t* grecs;
  uint64_t gcap;
  unsigned int* status;
  unsigned long long* lb_status;  // look-back tile states
  unsigned long long* ticket;     // tile ticket counter
  unsigned long long* n_groups;
  uint8_t* out_data[PMB_MAX_OUT];
  uint8_t* out_valid[PMB_MAX_OUT];
};

#define SK_HIST 1024

struct SketchOut {
  int64_t samples;
  int64_t distinct;
  int64_t singletons;
  int64_t doubletons;
  unsigned int hist[SK_HIST];  // keys of the sample by occurrence count (last bin: >= SK_HIST - 1)
  unsigned int fx_expo[PMB_MAX_FX];  // largest biased exponent of each float-sum column in the sample
  // device-resident sample set (valid until the next workspace reset)
  const unsigned long long* set_keys;
  const unsigned int* set_cnt;
};

int pmb_groupby_sketch(pmb_handle* h, const CompiledQuery& cq, SketchOut* out);
int64_t pmb_estimate_groups(const SketchOut& s, int64_t n_rows);
int pmb_choose_strategy(pmb_handle* h, const CompiledQuery& cq, const SketchOut& sk, int64_t est);
// AUTO's switch from a chosen global-table or sort strategy to the partitioned strategy
bool pmb_prefer_partitioned(const CompiledQuery& cq, const SketchOut& sk, int strategy, int64_t est);
// the most frequent sampled key stands for more than 256K rows: the sort's and the partitioned
// strategy's work for it would be one CTA's serial segment
bool pmb_heavy_key(const CompiledQuery& cq, const SketchOut& sk);
// a learned pick that AUTO overrules with the heuristic (see pmb_groupby.cu)
bool pmb_selector_vetoed(const CompiledQuery& cq, const SketchOut& sk, int strategy);
int pmb_plan_hash(pmb_handle* h, int max_smem_optin, CompiledQuery& cq, int strategy, int64_t est, bool have_sketch,
                  HashParams& P, int& nt, int& smem);
// est_learned: est is the larger of the sample estimate and the strategy selector's predicted
// group count (two estimates, so the table is sized tighter: 2 slots per group instead of 4)
int pmb_groupby_hash(pmb_handle* h, CompiledQuery& cq, const pmb_query* uq, int strategy, int64_t est,
                     const SketchOut* sk, pmb_result* r, bool est_learned = false);
// compiles the query again with cq.dd_user_cols, keeping the staged column pointers
int recompile_dd(pmb_handle* h, const pmb_query* q, const pmb_column* cols, int32_t n_cols, CompiledQuery& cq);
// keys = EMPTY, records = identity (k_table_init) on stream s
void k_table_init_pub(unsigned long long* keys, int64_t key_words, uint64_t* recs, int64_t n_recs, int rec_words,
                      const RecInit& ri, int blocks, cudaStream_t s);
// sort strategy (pmb_sort.cu): packed-key LSD radix sort + segmented reduce
// the sort strategy (part_groups == 0), or the partitioned strategy sized for part_groups groups
int pmb_groupby_sort(pmb_handle* h, CompiledQuery& cq, pmb_result* r, int64_t part_groups);
// stable LSD sort of (W-word key, u32 row index) pairs over 8-bit digits 0 .. n_passes-1, the
// group-by sort's pass kernel (pmb_sort.cu); *k / *i end up pointing at the sorted buffers
int pmb_sort_pairs(pmb_handle* h, int W, unsigned long long** k, unsigned long long** k_alt, unsigned int** i,
                   unsigned int** i_alt, uint64_t cap, int64_t n, int n_passes, const unsigned int* hist_dev,
                   const unsigned int* hist_host);
// output sort (pmb_order.cu): the n rows of the device columns in the order of the spec, the first
// `limit` of them, as device columns of r (r->n_groups set); the workspace is not reset
int pmb_order_columns(pmb_handle* h, const DCol* cols, int n_cols, int64_t n, const pmb_sort_spec& s, pmb_result* r);
// learned selector (pmb_learned.cu): strategy and group count for AUTO; false when no selector is
// installed or its output is unusable
bool pmb_selector_pick(pmb_handle* h, const CompiledQuery& cq, int* strategy, int64_t* groups);
// the same in two halves: the launch queues the selector's kernels and the copy of its outputs into
// the pinned staging at PMB_SEL_PINNED_OFF (false: no selector); the read decodes them after the
// caller's next stream synchronisation
#define PMB_SEL_PINNED_OFF 61440
bool pmb_selector_launch(pmb_handle* h, const CompiledQuery& cq);
bool pmb_selector_read(pmb_handle* h, const CompiledQuery& cq, int* strategy, int64_t* groups);
// group counts the selector predicts for a batch of queries (device DQuery array); false without
// an installed selector
bool pmb_selector_predict_batch(pmb_handle* h, const DQuery* d_qs, int nq, int64_t* out_groups, const int64_t* n_rows);
const float* pmb_selector_batch_launch(pmb_handle* h, const DQuery* d_qs, int nq);
void pmb_selector_batch_groups(const float* ho, int nq, int64_t* out_groups, const int64_t* n_rows);

// Sets bit p of a bitmap for every lane whose `bit` is true. The warp's positions are
// consecutive from p_first, so they touch at most two 32-bit words: one atomicOr each.
__device__ __forceinline__ void warp_set_bits(unsigned int* words, int64_t p, int64_t p_first, bool bit) {
  const int64_t w0 = p_first >> 5;
  unsigned m0 = __reduce_or_sync(0xffffffffu, (bit && (p >> 5) == w0) ? (1u << (p & 31)) : 0u);
  unsigned m1 = __reduce_or_sync(0xffffffffu, (bit && (p >> 5) == w0 + 1) ? (1u << (p & 31)) : 0u);
  if ((threadIdx.x & 31) == 0) {
    if (m0) atomicOr(&words[w0], m0);
    if (m1) atomicOr(&words[w0 + 1], m1);
  }
}

// Correctly rounded double of the exact fixed-point sum (its two words l, fraction bits F, flags).
__device__ __forceinline__ double fx_value(const unsigned long long* l, int F, unsigned flags) {
  if ((flags & PMB_FX_NAN) || ((flags & PMB_FX_PINF) && (flags & PMB_FX_NINF)))
    return __longlong_as_double(0x7FF8000000000000LL);
  if (flags & PMB_FX_PINF) return __longlong_as_double(0x7FF0000000000000LL);
  if (flags & PMB_FX_NINF) return __longlong_as_double((long long)0xFFF0000000000000ULL);
  __int128 S = ((__int128)(long long)l[1] << 32) + (__int128)l[0];
  bool neg = S < 0;
  unsigned __int128 M = neg ? (unsigned __int128)(-S) : (unsigned __int128)S;
  unsigned long long hi = (unsigned long long)(M >> 64), lo = (unsigned long long)M;
  double v;
  int sc = 0;
  if (hi == 0) {
    v = __ull2double_rn(lo);
  } else {
    int lz = __clzll(hi);
    int sh = 64 - lz;  // bits to drop so that the value fits 64 bits
    unsigned long long top = lz ? ((hi << lz) | (lo >> sh)) : hi;
    unsigned long long dropped = sh == 64 ? lo : (lo & ((1ULL << sh) - 1ULL));
    top |= dropped ? 1ULL : 0ULL;  // sticky bit below the rounding position
    v = __ull2double_rn(top);
    sc = sh;
  }
  v = ldexp(v, sc - F);
  return neg ? -v : v;
}

// Final value of aggregation A from a group record (Polars rules: all-null sum = 0, mean /
// min / max of no valid value = null, NaN poisons float min / max, ints wrap).
__device__ __forceinline__ void finalize_agg(const DQuery& q, const DAggOut& A, const uint8_t* rec, bool& valid,
                                             uint64_t& bits) {
  valid = true;
  bits = 0;
  auto u32 = [&](int f) { return *reinterpret_cast<const unsigned int*>(rec + q.field[f].off); };
  auto u64 = [&](int f) { return *reinterpret_cast<const unsigned long long*>(rec + q.field[f].off); };
  auto ddv = [&](int f) {
    const DField& F = q.field[f];
    if (F.kind == F_SUM_FX) {
      const unsigned long long* l = reinterpret_cast<const unsigned long long*>(rec + F.off);
      return fx_value(l, F.fx, *reinterpret_cast<const unsigned int*>(rec + F.off + 16));
    }
    const double* p = reinterpret_cast<const double*>(rec + F.off);
    return p[0] + p[1];
  };
  const bool fl = pmb_is_float(A.in_dtype);
  switch (A.op) {
    case PMB_AGG_LEN: bits = u32(A.f_len); return;
    case PMB_AGG_COUNT: bits = u32(A.f_cnt); return;
    case PMB_AGG_SUM:
      if (fl) {
        double v = ddv(A.f_main);
        if (A.out_dtype == PMB_F32) bits = __float_as_uint((float)v);
        else bits = (uint64_t)__double_as_longlong(v);
      } else {
        bits = u64(A.f_main);
      }
      return;
    case PMB_AGG_MEAN: {
      unsigned int c = u32(A.f_cnt);
      if (c == 0) {
        valid = false;
        return;
      }
      double v;
      if (fl) v = ddv(A.f_main) / (double)c;
      else if (pmb_is_signed(A.in_dtype) || A.in_dtype == PMB_BOOL) v = (double)(long long)u64(A.f_main) / (double)c;
      else v = (double)u64(A.f_main) / (double)c;
      if (A.out_dtype == PMB_F32) bits = __float_as_uint((float)v);
      else bits = (uint64_t)__double_as_longlong(v);
      return;
    }
    default: {  // min / max
      long long k = (long long)u64(A.f_main);
      if (fl) {
        bool mn = A.op == PMB_AGG_MIN;
        long long ident = mn ? 0x7FFFFFFFFFFFFFFFLL : (long long)0x8000000000000000LL;
        long long nanm = mn ? (long long)0x8000000000000000LL : 0x7FFFFFFFFFFFFFFFLL;
        if (k == ident) {
          valid = false;
          return;
        }
        double v = (k == nanm) ? __longlong_as_double(0x7FF8000000000000LL) : pmb_f64_from_key(k);
        if (A.in_dtype == PMB_F32) bits = __float_as_uint((float)v);
        else bits = (uint64_t)__double_as_longlong(v);
        return;
      }
      if (A.f_cnt >= 0 && u32(A.f_cnt) == 0) {
        valid = false;
        return;
      }
      bits = (uint64_t)k;
      return;
    }
  }
}
