// pmb_expr.cuh — device-side row access, predicate evaluation, key packing and the
// aggregation-state update/merge primitives shared by the group-by and filter kernels.
//
// Predicate semantics follow the reference: IEEE compares (NaN compares false except !=,
// -0.0 == +0.0; crates/polars-metal-kernels/src/cmp.rs:14-28), a compare is null when an
// operand is null (cmp.rs:9-13), Kleene AND/OR (shaders/logical_bool.metal:3-26), and a row
// survives the filter iff the predicate is valid and true. Each leaf term yields a pair of
// bits (T = "valid and true", F = "valid and false"); AND/OR/NOT on those pairs is exactly
// Kleene logic, so the circuit runs on two small bit stacks held in registers.
#pragma once

#include "pmb_internal.cuh"

// Where the current tile's column chunks live: a shared-memory stage (sbase != nullptr, with
// per-column offsets doff/voff) or global memory starting at row `row0`.
struct TileCtx {
  const uint8_t* sbase;
  const int32_t* doff;
  const int32_t* voff;
  int64_t row0;
};

__device__ __forceinline__ const uint8_t* tc_data(const DQuery& q, const TileCtx& t, int c) {
  if (t.sbase) return t.sbase + t.doff[c];
  int e = q.col[c].elem;
  return q.col[c].data + (e ? t.row0 * e : t.row0 / 8);
}
__device__ __forceinline__ const uint8_t* tc_valid(const DQuery& q, const TileCtx& t, int c) {
  const uint8_t* v = q.col[c].valid;
  if (!v) return nullptr;
  return t.sbase ? t.sbase + t.voff[c] : v + t.row0 / 8;
}
__device__ __forceinline__ uint64_t tc_bits(const DQuery& q, const TileCtx& t, int c, int64_t lr) {
  return pmb_load_bits(tc_data(q, t, c), q.col[c].elem, lr);
}
__device__ __forceinline__ bool tc_isvalid(const DQuery& q, const TileCtx& t, int c, int64_t lr) {
  return pmb_valid_bit(tc_valid(q, t, c), lr);
}

// ------------------------------------------------------------------ predicate
struct OpVal {
  bool valid;
  int64_t i;
  double f;
};

__device__ __forceinline__ OpVal eval_leaf(const DQuery& q, const TileCtx& t, const DLeaf& L, int dt, int64_t lr) {
  OpVal v;
  if (L.col < 0) {
    v.valid = true;
    v.i = L.i;
    v.f = L.f;
    return v;
  }
  v.valid = tc_isvalid(q, t, L.col, lr);
  uint64_t b = tc_bits(q, t, L.col, lr);
  int cdt = q.col[L.col].dtype;
  if (dt == PMB_F64) v.f = pmb_bits_to_f64(b, cdt), v.i = 0;
  else v.i = pmb_bits_to_i64(b, cdt), v.f = 0.0;
  return v;
}

__device__ __forceinline__ double pmb_py_fmod(double a, double b) {
  double r = fmod(a, b);
  if (r != 0.0 && ((r < 0.0) != (b < 0.0))) r += b;
  return r;
}

// a op b in Float64 (Polars floor division and modulo)
__device__ __forceinline__ double pmb_arith_f64(int op, double a, double b) {
  switch (op) {
    case PMB_ARITH_ADD: return a + b;
    case PMB_ARITH_SUB: return a - b;
    case PMB_ARITH_MUL: return a * b;
    case PMB_ARITH_TRUEDIV: return a / b;
    case PMB_ARITH_FLOORDIV: return floor(a / b);
    default: return pmb_py_fmod(a, b);
  }
}

// a op b in Int64: wrapping +, -, *; floor division and modulo with the divisor's sign; `valid`
// turns false on a division by zero
__device__ __forceinline__ int64_t pmb_arith_i64(int op, int64_t a, int64_t b, bool& valid) {
  const uint64_t x = (uint64_t)a, y = (uint64_t)b;
  switch (op) {
    case PMB_ARITH_ADD: return (int64_t)(x + y);
    case PMB_ARITH_SUB: return (int64_t)(x - y);
    case PMB_ARITH_MUL: return (int64_t)(x * y);
    case PMB_ARITH_FLOORDIV: {
      if (b == 0) {
        valid = false;
        return 0;
      }
      if (a == INT64_MIN && b == -1) return INT64_MIN;
      int64_t qq = a / b;
      if ((a % b != 0) && ((a < 0) != (b < 0))) qq -= 1;
      return qq;
    }
    default: {
      if (b == 0) {
        valid = false;
        return 0;
      }
      if (b == -1) return 0;
      int64_t m = a % b;
      if (m != 0 && ((m < 0) != (b < 0))) m += b;
      return m;
    }
  }
}

__device__ __forceinline__ OpVal eval_operand(const DQuery& q, const TileCtx& t, const DOperand& o, int dt, int64_t lr) {
  OpVal a = eval_leaf(q, t, o.a, dt, lr);
  if (o.arith < 0) return a;
  OpVal b = eval_leaf(q, t, o.b, dt, lr);
  OpVal r;
  r.valid = a.valid && b.valid;
  r.i = 0;
  r.f = 0.0;
  if (dt == PMB_F64) r.f = pmb_arith_f64(o.arith, a.f, b.f);
  else r.i = pmb_arith_i64(o.arith, a.i, b.i, r.valid);
  return r;
}

__device__ __forceinline__ void eval_term(const DQuery& q, const TileCtx& t, const DTerm& T, int64_t lr,uint32_t& tt,
                                          uint32_t& ff) {
  switch (T.kind) {
    case T_CMP: {
      OpVal a = eval_operand(q, t, T.lhs, T.dtype, lr);
      OpVal b = eval_operand(q, t, T.rhs, T.dtype, lr);
      if (!(a.valid && b.valid)) {
        tt = ff = 0;
        return;
      }
      bool c;
      if (T.dtype == PMB_F64) {
        switch (T.op) {
          case PMB_CMP_EQ: c = a.f == b.f; break;
          case PMB_CMP_NE: c = a.f != b.f; break;
          case PMB_CMP_LT: c = a.f < b.f; break;
          case PMB_CMP_LE: c = a.f <= b.f; break;
          case PMB_CMP_GT: c = a.f > b.f; break;
          default: c = a.f >= b.f; break;
        }
      } else {
        switch (T.op) {
          case PMB_CMP_EQ: c = a.i == b.i; break;
          case PMB_CMP_NE: c = a.i != b.i; break;
          case PMB_CMP_LT: c = a.i < b.i; break;
          case PMB_CMP_LE: c = a.i <= b.i; break;
          case PMB_CMP_GT: c = a.i > b.i; break;
          default: c = a.i >= b.i; break;
        }
      }
      tt = c;
      ff = !c;
      return;
    }
    case T_BOOLCOL: {
      int c = T.lhs.a.col;
      bool v = tc_isvalid(q, t, c, lr);
      bool b = tc_bits(q, t, c, lr) != 0;
      tt = v && b;
      ff = v && !b;
      return;
    }
    case T_ISNULL:
    case T_ISNOTNULL: {
      bool v = eval_operand(q, t, T.lhs, T.dtype, lr).valid;
      bool isnull = !v;
      tt = (T.kind == T_ISNULL) ? isnull : !isnull;
      ff = !tt;
      return;
    }
    default:  // T_LITBOOL
      tt = T.lhs.a.i != 0;
      ff = !tt;
      return;
  }
}

// true iff the row survives the filter (predicate valid and true)
__device__ __forceinline__ bool eval_keep(const DQuery& q, const TileCtx& t, int64_t lr) {
  const DProgram& P = q.prog;
  if (P.n_ops == 0) return true;
  uint32_t ts = 0, fs = 0;
  for (int i = 0; i < P.n_ops; i++) {
    int op = P.ops[i];
    if (op >= 0) {
      uint32_t a, b;
      eval_term(q, t, P.term[op], lr, a, b);
      ts = (ts << 1) | a;
      fs = (fs << 1) | b;
    } else if (op == OP_NOT) {
      uint32_t a = ts & 1u, b = fs & 1u;
      ts = (ts & ~1u) | b;
      fs = (fs & ~1u) | a;
    } else {
      uint32_t tb = ts & 1u, fb = fs & 1u;
      ts >>= 1;
      fs >>= 1;
      uint32_t ta = ts & 1u, fa = fs & 1u, r_t, r_f;
      if (op == OP_AND) {
        r_t = ta & tb;
        r_f = fa | fb;
      } else {
        r_t = ta | tb;
        r_f = fa & fb;
      }
      ts = (ts & ~1u) | r_t;
      fs = (fs & ~1u) | r_f;
    }
  }
  return (ts & 1u) != 0;
}

// Kleene (T, F) of the whole predicate, for bit-packed (data, validity) outputs
__device__ __forceinline__ void eval_pred_tf(const DQuery& q, const TileCtx& t, int64_t lr,bool& valid, bool& truth) {
  const DProgram& P = q.prog;
  uint32_t ts = 0, fs = 0;
  for (int i = 0; i < P.n_ops; i++) {
    int op = P.ops[i];
    if (op >= 0) {
      uint32_t a, b;
      eval_term(q, t, P.term[op], lr, a, b);
      ts = (ts << 1) | a;
      fs = (fs << 1) | b;
    } else if (op == OP_NOT) {
      uint32_t a = ts & 1u, b = fs & 1u;
      ts = (ts & ~1u) | b;
      fs = (fs & ~1u) | a;
    } else {
      uint32_t tb = ts & 1u, fb = fs & 1u;
      ts >>= 1;
      fs >>= 1;
      uint32_t ta = ts & 1u, fa = fs & 1u, r_t, r_f;
      if (op == OP_AND) {
        r_t = ta & tb;
        r_f = fa | fb;
      } else {
        r_t = ta | tb;
        r_f = fa & fb;
      }
      ts = (ts & ~1u) | r_t;
      fs = (fs & ~1u) | r_f;
    }
  }
  truth = (ts & 1u) != 0;
  valid = truth || (fs & 1u);
}

// ------------------------------------------------------------------ keys

__device__ __forceinline__ uint64_t pack_key64(const DQuery& q, const TileCtx& t, int64_t lr) {
  uint64_t k = 0;
  for (int i = 0; i < q.n_keys; i++) {
    const DKey& K = q.key[i];
    if (K.nullable && !tc_isvalid(q, t, K.col, lr)) {
      k |= 1ULL << K.null_off;
      continue;
    }
    uint64_t v = tc_bits(q, t, K.col, lr);
    if (K.bits < 64) v &= (1ULL << K.bits) - 1ULL;
    k |= v << K.data_off;
  }
  return k;
}

struct Key128 {
  uint64_t lo, hi;
};
__device__ __forceinline__ Key128 pack_key128(const DQuery& q, const TileCtx& t, int64_t lr) {
  Key128 k{0, 0};
  for (int i = 0; i < q.n_keys; i++) {
    const DKey& K = q.key[i];
    if (K.nullable && !tc_isvalid(q, t, K.col, lr)) {
      if (K.null_off < 64) k.lo |= 1ULL << K.null_off;
      else k.hi |= 1ULL << (K.null_off - 64);
      continue;
    }
    uint64_t v = tc_bits(q, t, K.col, lr);
    if (K.bits < 64) v &= (1ULL << K.bits) - 1ULL;
    int o = K.data_off;
    if (o < 64) {
      k.lo |= v << o;
      if (o > 0 && o + K.bits > 64) k.hi |= v >> (64 - o);
    } else {
      k.hi |= v << (o - 64);
    }
  }
  return k;
}

// decode the raw data bits of key field K from a packed key; returns false when null
__device__ __forceinline__ bool unpack_field(const DKey& K, uint64_t lo, uint64_t hi, uint64_t& v) {
  if (K.nullable) {
    uint64_t nb = K.null_off < 64 ? (lo >> K.null_off) & 1ULL : (hi >> (K.null_off - 64)) & 1ULL;
    if (nb) {
      v = 0;
      return false;
    }
  }
  int o = K.data_off;
  if (o < 64) {
    v = lo >> o;
    if (o > 0 && o + K.bits > 64) v |= hi << (64 - o);
  } else {
    v = hi >> (o - 64);
  }
  if (K.bits < 64) v &= (1ULL << K.bits) - 1ULL;
  return true;
}

// ------------------------------------------------------------------ aggregation state
// identity value word(s) of a field, written at record init
__host__ __device__ inline void field_identity(int kind, uint64_t* w0, uint64_t* w1, int* nwords, int* bytes) {
  *w1 = 0;
  *nwords = 1;
  switch (kind) {
    case F_LEN: case F_CNT: *w0 = 0; *bytes = 4; break;
    case F_SUM_DD: *w0 = 0; *nwords = 2; *bytes = 16; break;
    case F_SUM_FX: *w0 = 0; *nwords = 3; *bytes = 24; break;
    case F_SUM_I: *w0 = 0; *bytes = 8; break;
    case F_MIN_I: case F_MIN_F: *w0 = 0x7FFFFFFFFFFFFFFFULL; *bytes = 8; break;
    case F_MAX_I: case F_MAX_F: *w0 = 0x8000000000000000ULL; *bytes = 8; break;
    case F_MIN_U: *w0 = 0xFFFFFFFFFFFFFFFFULL; *bytes = 8; break;
    default: *w0 = 0; *bytes = 8; break;  // F_MAX_U
  }
}

// One row's contribution to a group record. Three variants, by who may touch the record:
//   apply_row_private — records owned by one warp, updated by a single lane (no atomics);
//   apply_row_shared  — the CTA-shared table (shared-memory atomics; on sm_100 only 32-bit
//                       adds and 64-bit min/max are native there, so min/max skip when the
//                       stored value already dominates and the rest stays low-contention);
//   apply_row_global  — the global table (fire-and-forget L2 updates, pmb_red_*:
//                       adjacent 32-bit counters share one 64-bit add, min/max are issued only
//                       when the row improves on a possibly stale read).
__device__ __forceinline__ long long minmax_key(const DField& F, uint64_t b, int dt, bool is_min) {
  double x = pmb_bits_to_f64(b, dt);
  if (isnan(x)) return is_min ? (long long)0x8000000000000000LL : 0x7FFFFFFFFFFFFFFFLL;
  return pmb_f64_key(x);
}

__device__ __forceinline__ void apply_row_private(const DQuery& q, const TileCtx& t, uint8_t* rec, int64_t lr) {
  for (int i = 0; i < q.n_fields; i++) {
    const DField F = q.field[i];
    uint8_t* p = rec + F.off;
    if (F.kind == F_LEN) {
      *(unsigned int*)p += 1u;
      continue;
    }
    if (!tc_isvalid(q, t, F.col, lr)) continue;
    if (F.kind == F_CNT) {
      *(unsigned int*)p += 1u;
      continue;
    }
    uint64_t b = tc_bits(q, t, F.col, lr);
    int dt = q.col[F.col].dtype;
    switch (F.kind) {
      case F_SUM_DD: dd_plain_add((double*)p, (double*)(p + 8), pmb_bits_to_f64(b, dt)); break;
      case F_SUM_FX: {
        double x = pmb_bits_to_f64(b, dt);
        unsigned fl = pmb_fx_flag(x);
        if (fl) {
          *(unsigned int*)(p + 16) |= fl;
        } else if (pmb_fx_in_range(x, q.fx_e[F.fx_slot])) {
          unsigned long long w0, w1;
          pmb_fx_words(x, F.fx, w0, w1);
          ((unsigned long long*)p)[0] += w0;
          ((unsigned long long*)p)[1] += w1;
        }
        break;
      }
      case F_SUM_I: *(unsigned long long*)p += (unsigned long long)pmb_bits_to_i64(b, dt); break;
      case F_MIN_I: {
        long long v = (long long)pmb_bits_to_i64(b, dt);
        if (v < *(long long*)p) *(long long*)p = v;
        break;
      }
      case F_MAX_I: {
        long long v = (long long)pmb_bits_to_i64(b, dt);
        if (v > *(long long*)p) *(long long*)p = v;
        break;
      }
      case F_MIN_U:
        if (b < *(unsigned long long*)p) *(unsigned long long*)p = b;
        break;
      case F_MAX_U:
        if (b > *(unsigned long long*)p) *(unsigned long long*)p = b;
        break;
      case F_MIN_F: {
        long long k = minmax_key(F, b, dt, true);
        if (k < *(long long*)p) *(long long*)p = k;
        break;
      }
      default: {
        long long k = minmax_key(F, b, dt, false);
        if (k > *(long long*)p) *(long long*)p = k;
        break;
      }
    }
  }
}

__device__ __forceinline__ void apply_row_shared(const DQuery& q, const TileCtx& t, uint8_t* rec, int64_t lr) {
  for (int i = 0; i < q.n_fields; i++) {
    const DField F = q.field[i];
    uint8_t* p = rec + F.off;
    if (F.kind == F_LEN) {
      atomicAdd((unsigned int*)p, 1u);
      continue;
    }
    if (!tc_isvalid(q, t, F.col, lr)) continue;
    if (F.kind == F_CNT) {
      atomicAdd((unsigned int*)p, 1u);
      continue;
    }
    uint64_t b = tc_bits(q, t, F.col, lr);
    int dt = q.col[F.col].dtype;
    switch (F.kind) {
      case F_SUM_DD: dd_atomic_add((double*)p, (double*)(p + 8), pmb_bits_to_f64(b, dt)); break;
      case F_SUM_FX: {
        double x = pmb_bits_to_f64(b, dt);
        unsigned fl = pmb_fx_flag(x);
        if (fl) {
          atomicOr((unsigned int*)(p + 16), fl);
        } else if (pmb_fx_in_range(x, q.fx_e[F.fx_slot])) {
          unsigned long long w0, w1;
          pmb_fx_words(x, F.fx, w0, w1);
          if (w0) atomicAdd((unsigned long long*)p, w0);
          if (w1) atomicAdd((unsigned long long*)p + 1, w1);
        }
        break;
      }
      case F_SUM_I: atomicAdd((unsigned long long*)p, (unsigned long long)pmb_bits_to_i64(b, dt)); break;
      case F_MIN_I: {
        long long v = (long long)pmb_bits_to_i64(b, dt);
        if (v < *(volatile long long*)p) atomicMin((long long*)p, v);
        break;
      }
      case F_MAX_I: {
        long long v = (long long)pmb_bits_to_i64(b, dt);
        if (v > *(volatile long long*)p) atomicMax((long long*)p, v);
        break;
      }
      case F_MIN_U:
        if (b < *(volatile unsigned long long*)p) atomicMin((unsigned long long*)p, (unsigned long long)b);
        break;
      case F_MAX_U:
        if (b > *(volatile unsigned long long*)p) atomicMax((unsigned long long*)p, (unsigned long long)b);
        break;
      case F_MIN_F: {
        long long k = minmax_key(F, b, dt, true);
        if (k < *(volatile long long*)p) atomicMin((long long*)p, k);
        break;
      }
      default: {
        long long k = minmax_key(F, b, dt, false);
        if (k > *(volatile long long*)p) atomicMax((long long*)p, k);
        break;
      }
    }
  }
}

__device__ __forceinline__ void apply_row_global(const DQuery& q, const TileCtx& t, uint8_t* rec, int64_t lr) {
  unsigned long long pend = 0;  // packed 32-bit counter increments of one 8-byte word
  int pend_off = -1;
  for (int i = 0; i < q.n_fields; i++) {
    const DField F = q.field[i];
    uint8_t* p = rec + F.off;
    if (F.kind == F_LEN || F.kind == F_CNT) {
      unsigned long long inc = (F.kind == F_LEN || tc_isvalid(q, t, F.col, lr)) ? 1ULL : 0ULL;
      int w = F.off & ~7;
      if (w != pend_off) {
        if (pend) pmb_red_add((unsigned long long*)(rec + pend_off), pend);
        pend = 0;
        pend_off = w;
      }
      pend += inc << ((F.off & 4) ? 32 : 0);
      continue;
    }
    if (!tc_isvalid(q, t, F.col, lr)) continue;
    uint64_t b = tc_bits(q, t, F.col, lr);
    int dt = q.col[F.col].dtype;
    switch (F.kind) {
      case F_SUM_DD: dd_atomic_add((double*)p, (double*)(p + 8), pmb_bits_to_f64(b, dt)); break;
      case F_SUM_FX: {
        double x = pmb_bits_to_f64(b, dt);
        unsigned fl = pmb_fx_flag(x);
        if (fl) {
          pmb_rec_or32(rec, F.off + 16, fl);
        } else if (pmb_fx_in_range(x, q.fx_e[F.fx_slot])) {
          unsigned long long w0, w1;
          pmb_fx_words(x, F.fx, w0, w1);
          if (w0) pmb_red_add((unsigned long long*)p, w0);
          if (w1) pmb_red_add((unsigned long long*)p + 1, w1);
        }
        break;
      }
      case F_SUM_I: pmb_red_add((unsigned long long*)p, (unsigned long long)pmb_bits_to_i64(b, dt)); break;
      // a stale read can only be weaker than the stored extreme, so skipping is safe
      case F_MIN_I: {
        long long v = (long long)pmb_bits_to_i64(b, dt);
        if (v < *(const long long*)p) pmb_red_min((long long*)p, v);
        break;
      }
      case F_MAX_I: {
        long long v = (long long)pmb_bits_to_i64(b, dt);
        if (v > *(const long long*)p) pmb_red_max((long long*)p, v);
        break;
      }
      case F_MIN_U:
        if (b < *(const unsigned long long*)p) pmb_red_min((unsigned long long*)p, (unsigned long long)b);
        break;
      case F_MAX_U:
        if (b > *(const unsigned long long*)p) pmb_red_max((unsigned long long*)p, (unsigned long long)b);
        break;
      case F_MIN_F: {
        long long k = minmax_key(F, b, dt, true);
        if (k < *(const long long*)p) pmb_red_min((long long*)p, k);
        break;
      }
      default: {
        long long k = minmax_key(F, b, dt, false);
        if (k > *(const long long*)p) pmb_red_max((long long*)p, k);
        break;
      }
    }
  }
  if (pend) pmb_red_add((unsigned long long*)(rec + pend_off), pend);
}

// Merges a finished record `src` into `dst` (global memory, atomics).
__device__ __forceinline__ void merge_record(const DQuery& q, uint8_t* dst, const uint8_t* src) {
  for (int i = 0; i < q.n_fields; i++) {
    const DField F = q.field[i];
    uint8_t* d = dst + F.off;
    const uint8_t* s = src + F.off;
    switch (F.kind) {
      case F_LEN:
      case F_CNT: {
        unsigned int v = *(const unsigned int*)s;
        if (v) pmb_rec_add32(dst, F.off, v);
        break;
      }
      case F_SUM_DD: {
        double hi = *(const double*)s, lo = *(const double*)(s + 8);
        if (hi != 0.0) dd_atomic_add((double*)d, (double*)(d + 8), hi);
        if (lo != 0.0) atomicAdd((double*)(d + 8), lo);
        break;
      }
      case F_SUM_FX: {
        const unsigned long long* l = (const unsigned long long*)s;
        for (int w = 0; w < 2; w++)
          if (l[w]) pmb_red_add((unsigned long long*)d + w, l[w]);
        unsigned fl = *(const unsigned int*)(s + 16);
        if (fl) pmb_rec_or32(dst, F.off + 16, fl);
        break;
      }
      case F_SUM_I: {
        unsigned long long v = *(const unsigned long long*)s;
        if (v) pmb_red_add((unsigned long long*)d, v);
        break;
      }
      case F_MIN_I:
      case F_MIN_F: {
        long long v = *(const long long*)s;
        if (v != 0x7FFFFFFFFFFFFFFFLL) pmb_red_min((long long*)d, v);
        break;
      }
      case F_MAX_I:
      case F_MAX_F: {
        long long v = *(const long long*)s;
        if (v != (long long)0x8000000000000000LL) pmb_red_max((long long*)d, v);
        break;
      }
      case F_MIN_U: {
        unsigned long long v = *(const unsigned long long*)s;
        if (v != 0xFFFFFFFFFFFFFFFFULL) pmb_red_min((unsigned long long*)d, v);
        break;
      }
      default: {
        unsigned long long v = *(const unsigned long long*)s;
        if (v) pmb_red_max((unsigned long long*)d, v);
        break;
      }
    }
  }
}

// Merges record `src` into `dst` when one thread owns both (no atomics).
__device__ __forceinline__ void merge_private(const DQuery& q, uint8_t* dst, const uint8_t* src) {
  for (int i = 0; i < q.n_fields; i++) {
    const DField F = q.field[i];
    uint8_t* d = dst + F.off;
    const uint8_t* s = src + F.off;
    switch (F.kind) {
      case F_LEN:
      case F_CNT: *(unsigned int*)d += *(const unsigned int*)s; break;
      case F_SUM_DD: {
        double hi = *(const double*)s, lo = *(const double*)(s + 8);
        dd_plain_add((double*)d, (double*)(d + 8), hi);
        *(double*)(d + 8) += lo;
        break;
      }
      case F_SUM_FX: {
        const unsigned long long* l = (const unsigned long long*)s;
        for (int w = 0; w < 2; w++) ((unsigned long long*)d)[w] += l[w];
        *(unsigned int*)(d + 16) |= *(const unsigned int*)(s + 16);
        break;
      }
      case F_SUM_I: *(unsigned long long*)d += *(const unsigned long long*)s; break;
      case F_MIN_I:
      case F_MIN_F: {
        long long v = *(const long long*)s;
        if (v < *(long long*)d) *(long long*)d = v;
        break;
      }
      case F_MAX_I:
      case F_MAX_F: {
        long long v = *(const long long*)s;
        if (v > *(long long*)d) *(long long*)d = v;
        break;
      }
      case F_MIN_U: {
        unsigned long long v = *(const unsigned long long*)s;
        if (v < *(unsigned long long*)d) *(unsigned long long*)d = v;
        break;
      }
      default: {
        unsigned long long v = *(const unsigned long long*)s;
        if (v > *(unsigned long long*)d) *(unsigned long long*)d = v;
        break;
      }
    }
  }
}

// Reports float-sum values outside their column's fixed-point range (the call is then re-run
// with a wider range); called once per surviving row.
__device__ __forceinline__ void fx_range_check(const DQuery& q, const TileCtx& t, int64_t lr, unsigned int* status) {
  for (int i = 0; i < q.n_fields; i++) {
    const DField F = q.field[i];
    if (F.kind != F_SUM_FX || !tc_isvalid(q, t, F.col, lr)) continue;
    double x = pmb_bits_to_f64(tc_bits(q, t, F.col, lr), q.col[F.col].dtype);
    if (!pmb_fx_flag(x) && !pmb_fx_in_range(x, q.fx_e[F.fx_slot])) {
      atomicOr(status, PMB_ST_FXRANGE);
      atomicMax(&status[4 + F.fx_slot], (unsigned)pmb_fx_expo(x));
    }
  }
}
