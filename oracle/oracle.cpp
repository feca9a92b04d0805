// oracle.cpp — CPU restatement of polars-metal's filter -> group_by -> aggregate semantics.
//
// TEST INFRASTRUCTURE ONLY. This file is the correctness oracle and the timed CPU baseline;
// it is never linked into, loaded by, or called from the product library (libpmb). Only
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm use it.
//
// What it restates (reference files, dbfclark/polars-metal):
//   - key packing into a u128 lane, one null bit then the data bits per key column, LSB first:
//       crates/polars-metal-kernels/src/groupby.rs:155-302 (encode_keys), :1833-1985 (decode_keys)
//   - grouping (hash map from packed key to dense group id):
//       crates/polars-metal-kernels/src/groupby.rs:497-520 (cpu_hashmap_build)
//   - aggregation null rules: sum skips nulls and an all-null group sums to 0; count skips
//     nulls; len counts every row; min/max of an all-null group is null; f64 min/max are
//     poisoned by NaN; i64 sum wraps; mean = sum / count and is null when count == 0:
//       crates/polars-metal-kernels/src/groupby.rs:1268-1700
//   - predicate semantics: IEEE compares (NaN compares false except !=, -0.0 == +0.0),
//     output validity = AND of operand validities, Kleene AND/OR:
//       crates/polars-metal-kernels/src/cmp.rs:14-28, shaders/cmp_f64.metal:36-115,
//       shaders/logical_bool.metal:3-26
//   - filter keeps a row iff the predicate is valid and true (Polars DataFrame.filter,
//       python/polars_metal/_udf.py:550-597; crates/polars-metal-kernels/src/pipeline.rs:103-126)
//   - output dtypes: count/len -> UInt32 (crates/polars-metal-core/src/udf/groupby/mod.rs:680-706);
//     integer mean -> Float64 (Polars CPU; tests/python_integration/test_groupby.py:188-193).
//
// Float sums use Neumaier's compensated summation (Neumaier 1974), merged across threads by
// the same error-free transformation, so sums and means are accurate to ~1 ulp of the exact
// sum: the "FP64 compensated-sum oracle".
//
// Build: oracle/build.py (g++ -O3 -fopenmp -shared). Exposed through a C ABI for ctypes.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <string>
#include <unordered_map>
#include <vector>

#include <omp.h>

#include "../include/pmb.h"

namespace {

thread_local std::string g_err;

struct U128 {
  uint64_t lo = 0, hi = 0;
  bool operator==(const U128& o) const { return lo == o.lo && hi == o.hi; }
  bool operator<(const U128& o) const { return hi != o.hi ? hi < o.hi : lo < o.lo; }
};
struct U128Hash {
  size_t operator()(const U128& k) const {
    uint64_t h = k.lo * 0x9E3779B97F4A7C15ull ^ (k.hi + 0x632BE59BD9B4E019ull);
    h ^= h >> 29;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 32;
    return (size_t)h;
  }
};

int dtype_bytes(int dt) {
  switch (dt) {
    case PMB_BOOL: return 0;
    case PMB_I8: case PMB_U8: return 1;
    case PMB_I16: case PMB_U16: return 2;
    case PMB_I32: case PMB_U32: case PMB_F32: return 4;
    default: return 8;
  }
}
int dtype_bits(int dt) { return dt == PMB_BOOL ? 1 : 8 * dtype_bytes(dt); }
bool is_float(int dt) { return dt == PMB_F32 || dt == PMB_F64; }
bool is_signed(int dt) { return dt == PMB_I8 || dt == PMB_I16 || dt == PMB_I32 || dt == PMB_I64; }

struct Col {
  const uint8_t* data;
  const uint8_t* valid;
  int64_t off;
  int dtype;
  bool is_valid(int64_t r) const {
    if (!valid) return true;
    int64_t b = r + off;
    return (valid[b >> 3] >> (b & 7)) & 1;
  }
  // raw bits, zero-extended
  uint64_t bits(int64_t r) const {
    int64_t i = r + off;
    switch (dtype) {
      case PMB_BOOL: return (data[i >> 3] >> (i & 7)) & 1;
      case PMB_I8: case PMB_U8: return data[i];
      case PMB_I16: case PMB_U16: { uint16_t v; memcpy(&v, data + 2 * i, 2); return v; }
      case PMB_I32: case PMB_U32: case PMB_F32: { uint32_t v; memcpy(&v, data + 4 * i, 4); return v; }
      default: { uint64_t v; memcpy(&v, data + 8 * i, 8); return v; }
    }
  }
  int64_t as_i64(int64_t r) const {
    uint64_t b = bits(r);
    switch (dtype) {
      case PMB_I8: return (int8_t)b;
      case PMB_I16: return (int16_t)b;
      case PMB_I32: return (int32_t)b;
      case PMB_F32: { float f; uint32_t u = (uint32_t)b; memcpy(&f, &u, 4); return (int64_t)f; }
      case PMB_F64: { double d; memcpy(&d, &b, 8); return (int64_t)d; }
      default: return (int64_t)b;
    }
  }
  double as_f64(int64_t r) const {
    uint64_t b = bits(r);
    switch (dtype) {
      case PMB_I8: return (double)(int8_t)b;
      case PMB_I16: return (double)(int16_t)b;
      case PMB_I32: return (double)(int32_t)b;
      case PMB_I64: return (double)(int64_t)b;
      case PMB_F32: { float f; uint32_t u = (uint32_t)b; memcpy(&f, &u, 4); return (double)f; }
      case PMB_F64: { double d; memcpy(&d, &b, 8); return d; }
      default: return (double)b;
    }
  }
};

// ---------------------------------------------------------------- predicate evaluation
struct Val {
  bool valid;
  bool is_f;
  int64_t i;
  double f;
};

struct Tri {  // Kleene value: valid + truth
  bool valid, truth;
};

double py_fmod(double a, double b) {
  double r = std::fmod(a, b);
  if (r != 0.0 && ((r < 0) != (b < 0))) r += b;
  return r;
}
int64_t floor_div(int64_t a, int64_t b) {
  int64_t q = a / b;
  if ((a % b != 0) && ((a < 0) != (b < 0))) q -= 1;
  return q;
}
int64_t floor_mod(int64_t a, int64_t b) {
  int64_t r = a % b;
  if (r != 0 && ((r < 0) != (b < 0))) r += b;
  return r;
}

struct Evaluator {
  const pmb_expr_node* nodes;
  const std::vector<Col>* cols;

  bool wants_float(int n) const {
    const pmb_expr_node& e = nodes[n];
    switch (e.kind) {
      case PMB_EXPR_LIT_F64: return true;
      case PMB_EXPR_COLUMN: return is_float((*cols)[e.column].dtype);
      case PMB_EXPR_ARITH:
        return e.op == PMB_ARITH_TRUEDIV || e.dtype == PMB_F64 || wants_float(e.lhs) || wants_float(e.rhs);
      default: return false;
    }
  }
  // operand dtype of a compare: the node's tag when given, else F64 if any operand is float;
  // true division always computes in F64
  int compare_dtype(int n) const {
    const pmb_expr_node& e = nodes[n];
    int dt = (e.dtype == PMB_I64 || e.dtype == PMB_F64) ? e.dtype
                                                         : ((wants_float(e.lhs) || wants_float(e.rhs)) ? PMB_F64 : PMB_I64);
    for (int side : {e.lhs, e.rhs}) {
      const pmb_expr_node& s = nodes[side];
      if (s.kind == PMB_EXPR_ARITH && s.op == PMB_ARITH_TRUEDIV) dt = PMB_F64;
    }
    return dt;
  }

  // value of a numeric node read as the operand dtype `dt` of the enclosing compare
  // (PMB_I64 or PMB_F64), the way the reference widens compare operands (_walker.py:1544-1553)
  Val value(int n, int64_t r, int dt) const {
    const pmb_expr_node& e = nodes[n];
    Val v{true, false, 0, 0.0};
    switch (e.kind) {
      case PMB_EXPR_COLUMN: {
        const Col& c = (*cols)[e.column];
        v.valid = c.is_valid(r);
        if (dt == PMB_F64) { v.is_f = true; v.f = c.as_f64(r); }
        else { v.i = c.as_i64(r); }
        return v;
      }
      case PMB_EXPR_LIT_I64:
        if (dt == PMB_F64) { v.is_f = true; v.f = (double)e.lit_i64; } else v.i = e.lit_i64;
        return v;
      case PMB_EXPR_LIT_F64:
        if (dt == PMB_I64) { v.i = (int64_t)e.lit_f64; } else { v.is_f = true; v.f = e.lit_f64; }
        return v;
      case PMB_EXPR_ARITH: {
        Val a = value(e.lhs, r, dt), b = value(e.rhs, r, dt);
        v.valid = a.valid && b.valid;
        if (dt == PMB_F64) {
          double x = a.is_f ? a.f : (double)a.i, y = b.is_f ? b.f : (double)b.i;
          v.is_f = true;
          switch (e.op) {
            case PMB_ARITH_ADD: v.f = x + y; break;
            case PMB_ARITH_SUB: v.f = x - y; break;
            case PMB_ARITH_MUL: v.f = x * y; break;
            case PMB_ARITH_TRUEDIV: v.f = x / y; break;
            case PMB_ARITH_FLOORDIV: v.f = std::floor(x / y); break;
            default: v.f = py_fmod(x, y); break;
          }
        } else {
          uint64_t x = (uint64_t)a.i, y = (uint64_t)b.i;
          switch (e.op) {
            case PMB_ARITH_ADD: v.i = (int64_t)(x + y); break;
            case PMB_ARITH_SUB: v.i = (int64_t)(x - y); break;
            case PMB_ARITH_MUL: v.i = (int64_t)(x * y); break;
            case PMB_ARITH_FLOORDIV:
              if (b.i == 0) { v.valid = false; v.i = 0; }
              else if (a.i == INT64_MIN && b.i == -1) v.i = INT64_MIN;
              else v.i = floor_div(a.i, b.i);
              break;
            default:
              if (b.i == 0) { v.valid = false; v.i = 0; }
              else if (b.i == -1) v.i = 0;
              else v.i = floor_mod(a.i, b.i);
              break;
          }
        }
        return v;
      }
      default:
        v.valid = false;
        return v;
    }
  }

  Tri truth(int n, int64_t r) const {
    const pmb_expr_node& e = nodes[n];
    switch (e.kind) {
      case PMB_EXPR_COLUMN: {
        const Col& c = (*cols)[e.column];
        return {c.is_valid(r), c.bits(r) != 0};
      }
      case PMB_EXPR_LIT_BOOL: return {true, e.lit_i64 != 0};
      case PMB_EXPR_IS_NULL: {
        Val a = value(e.lhs, r, PMB_I64);
        return {true, !a.valid};
      }
      case PMB_EXPR_IS_NOT_NULL: {
        Val a = value(e.lhs, r, PMB_I64);
        return {true, a.valid};
      }
      case PMB_EXPR_NOT: {
        Tri a = truth(e.lhs, r);
        return {a.valid, !a.truth};
      }
      case PMB_EXPR_AND: {
        Tri a = truth(e.lhs, r), b = truth(e.rhs, r);
        // false dominates null (shaders/logical_bool.metal:6-16)
        if ((a.valid && !a.truth) || (b.valid && !b.truth)) return {true, false};
        if (a.valid && b.valid) return {true, true};
        return {false, false};
      }
      case PMB_EXPR_OR: {
        Tri a = truth(e.lhs, r), b = truth(e.rhs, r);
        // true dominates null (shaders/logical_bool.metal:18-26)
        if ((a.valid && a.truth) || (b.valid && b.truth)) return {true, true};
        if (a.valid && b.valid) return {true, false};
        return {false, false};
      }
      case PMB_EXPR_COMPARE: {
        int dt = compare_dtype(n);
        Val a = value(e.lhs, r, dt), b = value(e.rhs, r, dt);
        Tri t{a.valid && b.valid, false};
        if (!t.valid) return t;
        if (dt == PMB_F64) {
          double x = a.is_f ? a.f : (double)a.i, y = b.is_f ? b.f : (double)b.i;
          switch (e.op) {
            case PMB_CMP_EQ: t.truth = x == y; break;
            case PMB_CMP_NE: t.truth = x != y; break;
            case PMB_CMP_LT: t.truth = x < y; break;
            case PMB_CMP_LE: t.truth = x <= y; break;
            case PMB_CMP_GT: t.truth = x > y; break;
            default: t.truth = x >= y; break;
          }
        } else {
          int64_t x = a.i, y = b.i;
          switch (e.op) {
            case PMB_CMP_EQ: t.truth = x == y; break;
            case PMB_CMP_NE: t.truth = x != y; break;
            case PMB_CMP_LT: t.truth = x < y; break;
            case PMB_CMP_LE: t.truth = x <= y; break;
            case PMB_CMP_GT: t.truth = x > y; break;
            default: t.truth = x >= y; break;
          }
        }
        return t;
      }
      default:
        return {false, false};
    }
  }
};

// ---------------------------------------------------------------- aggregation state
struct Neumaier {
  double s = 0.0, c = 0.0;
  void add(double x) {
    double t = s + x;
    if (std::isfinite(t)) {  // once the sum is inf / NaN it stays so; no compensation term
      if (std::fabs(s) >= std::fabs(x)) c += (s - t) + x;
      else c += (x - t) + s;
    }
    s = t;
  }
  void merge(const Neumaier& o) {
    add(o.s);
    c += o.c;
  }
  double value() const { return s + c; }
};

struct AggState {
  Neumaier fsum;
  uint64_t isum = 0;  // wrapping
  uint64_t count = 0, len = 0;
  bool has = false, nan = false;
  double fmin = 0, fmax = 0;
  int64_t imin = 0, imax = 0;
  uint64_t umin = 0, umax = 0;
};

int out_dtype(int op, int in_dt) {
  switch (op) {
    case PMB_AGG_COUNT: case PMB_AGG_LEN: return PMB_U32;
    case PMB_AGG_MEAN: return in_dt == PMB_F32 ? PMB_F32 : PMB_F64;
    case PMB_AGG_SUM:
      switch (in_dt) {
        case PMB_I8: case PMB_I16: case PMB_U8: case PMB_U16: return PMB_I64;
        case PMB_BOOL: return PMB_U32;
        default: return in_dt;
      }
    default: return in_dt;  // min / max
  }
}

struct OutCol {
  int dtype;
  std::vector<uint8_t> data;
  std::vector<uint8_t> valid;
};

}  // namespace

struct orc_result {
  int64_t n_rows = 0;
  std::vector<OutCol> cols;
};

namespace {

void set_bit(std::vector<uint8_t>& v, int64_t i, bool b) {
  if (b) v[i >> 3] |= (uint8_t)(1u << (i & 7));
}
size_t bitmap_bytes(int64_t n) {
  size_t b = (size_t)((n + 7) / 8);
  b = (b + 3) & ~(size_t)3;
  return b < 4 ? 4 : b;
}

template <class T>
void put(std::vector<uint8_t>& d, int64_t i, T v) {
  memcpy(d.data() + sizeof(T) * i, &v, sizeof(T));
}

void put_value(OutCol& oc, int64_t i, int dt, uint64_t bits) {
  switch (dt) {
    case PMB_BOOL: set_bit(oc.data, i, bits & 1); break;
    case PMB_I8: case PMB_U8: oc.data[i] = (uint8_t)bits; break;
    case PMB_I16: case PMB_U16: put<uint16_t>(oc.data, i, (uint16_t)bits); break;
    case PMB_I32: case PMB_U32: case PMB_F32: put<uint32_t>(oc.data, i, (uint32_t)bits); break;
    default: put<uint64_t>(oc.data, i, bits); break;
  }
}

bool check_columns(const pmb_column* cols, int32_t n_cols, int64_t* n_rows) {
  if (n_cols <= 0) { g_err = "no columns"; return false; }
  *n_rows = cols[0].length;
  for (int i = 0; i < n_cols; i++) {
    if (cols[i].length != *n_rows) { g_err = "row count mismatch"; return false; }
    if (cols[i].on_device) { g_err = "oracle takes host columns only"; return false; }
    if (cols[i].dtype < PMB_BOOL || cols[i].dtype > PMB_F64) { g_err = "bad dtype"; return false; }
  }
  return true;
}

std::vector<Col> make_cols(const pmb_column* cols, int32_t n_cols) {
  std::vector<Col> v(n_cols);
  for (int i = 0; i < n_cols; i++)
    v[i] = Col{(const uint8_t*)cols[i].data, cols[i].validity, cols[i].offset, cols[i].dtype};
  return v;
}

void eval_keep(const pmb_expr* pred, const std::vector<Col>& cols, int64_t n, int n_threads,
               std::vector<uint8_t>& keep) {
  keep.assign((size_t)n, 1);
  if (!pred) return;
  Evaluator ev{pred->nodes, &cols};
#pragma omp parallel for num_threads(n_threads) schedule(static)
  for (int64_t r = 0; r < n; r++) {
    Tri t = ev.truth(pred->root, r);
    keep[r] = (t.valid && t.truth) ? 1 : 0;
  }
}

}  // namespace

extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }

// Group-by oracle. Output: key columns then aggs, rows sorted by the packed u128 key.
int orc_groupby(const pmb_query* q, const pmb_column* cols_in, int32_t n_cols, int32_t n_threads,
                orc_result** out) {
  *out = nullptr;
  int64_t n;
  if (!check_columns(cols_in, n_cols, &n)) return PMB_E_INVALID;
  if (q->n_keys <= 0) { g_err = "no key columns"; return PMB_E_INVALID; }
  if (n_threads <= 0) n_threads = omp_get_max_threads();
  std::vector<Col> cols = make_cols(cols_in, n_cols);

  // key layout (groupby.rs:195-224): per field null bit, then data bits
  struct KF { int col, dt, null_off, data_off, bits; };
  std::vector<KF> kf;
  int off = 0;
  for (int k = 0; k < q->n_keys; k++) {
    int c = q->key_columns[k];
    if (c < 0 || c >= n_cols) { g_err = "key column out of range"; return PMB_E_NOT_FOUND; }
    int dt = cols[c].dtype, b = dtype_bits(dt);
    kf.push_back({c, dt, off, off + 1, b});
    off += 1 + b;
  }
  if (off > 128) { g_err = "composite key wider than 128 bits"; return PMB_E_UNSUPPORTED; }
  for (int a = 0; a < q->n_aggs; a++) {
    if (q->aggs[a].op != PMB_AGG_LEN && (q->aggs[a].column < 0 || q->aggs[a].column >= n_cols)) {
      g_err = "agg column out of range";
      return PMB_E_NOT_FOUND;
    }
  }

  std::vector<uint8_t> keep;
  eval_keep(q->predicate, cols, n, n_threads, keep);

  auto pack = [&](int64_t r) {
    U128 k;
    for (const KF& f : kf) {
      const Col& c = cols[f.col];
      if (!c.is_valid(r)) {
        if (f.null_off < 64) k.lo |= 1ull << f.null_off; else k.hi |= 1ull << (f.null_off - 64);
        continue;
      }
      uint64_t v = c.bits(r);
      if (f.bits < 64) v &= (1ull << f.bits) - 1;
      int o = f.data_off;
      if (o < 64) {
        k.lo |= v << o;
        if (o > 0 && o + f.bits > 64) k.hi |= v >> (64 - o);
      } else {
        k.hi |= v << (o - 64);
      }
    }
    return k;
  };

  const int na = q->n_aggs;
  auto update = [&](AggState* st, int64_t r) {
    for (int a = 0; a < na; a++) {
      AggState& s = st[a];
      s.len++;
      if (q->aggs[a].op == PMB_AGG_LEN) continue;
      const Col& c = cols[q->aggs[a].column];
      if (!c.is_valid(r)) continue;
      s.count++;
      int dt = c.dtype;
      if (is_float(dt)) {
        double x = c.as_f64(r);
        s.fsum.add(x);
        if (std::isnan(x)) s.nan = true;
        else if (!s.has) { s.fmin = s.fmax = x; }
        else { if (x < s.fmin) s.fmin = x; if (x > s.fmax) s.fmax = x; }
      } else if (is_signed(dt) || dt == PMB_BOOL) {
        int64_t x = c.as_i64(r);
        s.isum += (uint64_t)x;
        if (!s.has) { s.imin = s.imax = x; }
        else { s.imin = std::min(s.imin, x); s.imax = std::max(s.imax, x); }
      } else {
        uint64_t x = c.bits(r);
        s.isum += x;
        if (!s.has) { s.umin = s.umax = x; }
        else { s.umin = std::min(s.umin, x); s.umax = std::max(s.umax, x); }
      }
      s.has = true;
    }
  };
  auto merge = [&](AggState* d, const AggState* s) {
    for (int a = 0; a < na; a++) {
      AggState& x = d[a];
      const AggState& y = s[a];
      x.len += y.len;
      x.count += y.count;
      x.isum += y.isum;
      x.fsum.merge(y.fsum);
      x.nan = x.nan || y.nan;
      if (y.has) {
        if (!x.has) { x.fmin = y.fmin; x.fmax = y.fmax; x.imin = y.imin; x.imax = y.imax; x.umin = y.umin; x.umax = y.umax; }
        else {
          x.fmin = std::min(x.fmin, y.fmin); x.fmax = std::max(x.fmax, y.fmax);
          x.imin = std::min(x.imin, y.imin); x.imax = std::max(x.imax, y.imax);
          x.umin = std::min(x.umin, y.umin); x.umax = std::max(x.umax, y.umax);
        }
        x.has = true;
      }
    }
  };
  // NaN-only groups: has stays false for min/max values unless a non-NaN arrived; track via
  // count (has = any valid row) for validity, and nan for poisoning.

  // thread-local maps over contiguous row chunks, merged in chunk order
  std::vector<std::unordered_map<U128, int64_t, U128Hash>> maps(n_threads);
  std::vector<std::vector<U128>> tkeys(n_threads);
  std::vector<std::vector<AggState>> tstate(n_threads);
#pragma omp parallel num_threads(n_threads)
  {
    int t = omp_get_thread_num();
    int nt = omp_get_num_threads();
    int64_t lo = n * t / nt, hi = n * (t + 1) / nt;
    auto& m = maps[t];
    auto& ks = tkeys[t];
    auto& st = tstate[t];
    for (int64_t r = lo; r < hi; r++) {
      if (!keep[r]) continue;
      U128 k = pack(r);
      auto it = m.find(k);
      int64_t g;
      if (it == m.end()) {
        g = (int64_t)ks.size();
        m.emplace(k, g);
        ks.push_back(k);
        st.resize(st.size() + na);
      } else {
        g = it->second;
      }
      update(&st[g * na], r);
    }
  }
  std::unordered_map<U128, int64_t, U128Hash> gm;
  std::vector<U128> keys;
  std::vector<AggState> state;
  for (int t = 0; t < n_threads; t++) {
    for (size_t i = 0; i < tkeys[t].size(); i++) {
      const U128& k = tkeys[t][i];
      auto it = gm.find(k);
      int64_t g;
      if (it == gm.end()) {
        g = (int64_t)keys.size();
        gm.emplace(k, g);
        keys.push_back(k);
        state.resize(state.size() + na);
      } else {
        g = it->second;
      }
      merge(&state[g * na], &tstate[t][i * na]);
    }
    tkeys[t].clear(); tkeys[t].shrink_to_fit();
    tstate[t].clear(); tstate[t].shrink_to_fit();
    maps[t].clear();
  }
  std::vector<int64_t> order(keys.size());
  for (size_t i = 0; i < order.size(); i++) order[i] = (int64_t)i;
  std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return keys[a] < keys[b]; });

  const int64_t G = (int64_t)keys.size();
  orc_result* res = new orc_result();
  res->n_rows = G;
  // keys
  for (const KF& f : kf) {
    OutCol oc;
    oc.dtype = f.dt;
    oc.data.assign(f.dt == PMB_BOOL ? bitmap_bytes(G) : (size_t)(G * dtype_bytes(f.dt)), 0);
    oc.valid.assign(bitmap_bytes(G), 0);
    for (int64_t i = 0; i < G; i++) {
      const U128& k = keys[order[i]];
      auto bit = [&](int p) -> uint64_t { return p < 64 ? (k.lo >> p) & 1 : (k.hi >> (p - 64)) & 1; };
      bool isnull = bit(f.null_off);
      set_bit(oc.valid, i, !isnull);
      uint64_t v = 0;
      if (!isnull) {
        int o = f.data_off;
        if (o < 64) {
          v = k.lo >> o;
          if (o > 0 && o + f.bits > 64) v |= k.hi << (64 - o);
        } else {
          v = k.hi >> (o - 64);
        }
        if (f.bits < 64) v &= (1ull << f.bits) - 1;
      }
      put_value(oc, i, f.dt, v);
    }
    res->cols.push_back(std::move(oc));
  }
  // aggs
  for (int a = 0; a < na; a++) {
    int op = q->aggs[a].op;
    int in_dt = op == PMB_AGG_LEN ? PMB_U32 : cols[q->aggs[a].column].dtype;
    int odt = out_dtype(op, in_dt);
    OutCol oc;
    oc.dtype = odt;
    oc.data.assign(odt == PMB_BOOL ? bitmap_bytes(G) : (size_t)(G * dtype_bytes(odt)), 0);
    oc.valid.assign(bitmap_bytes(G), 0);
    for (int64_t i = 0; i < G; i++) {
      const AggState& s = state[order[i] * na + a];
      bool valid = true;
      uint64_t bits = 0;
      switch (op) {
        case PMB_AGG_LEN: bits = (uint32_t)s.len; break;
        case PMB_AGG_COUNT: bits = (uint32_t)s.count; break;
        case PMB_AGG_SUM:
          if (is_float(in_dt)) {
            double v = s.fsum.value();
            if (odt == PMB_F32) { float f = (float)v; uint32_t u; memcpy(&u, &f, 4); bits = u; }
            else memcpy(&bits, &v, 8);
          } else {
            bits = s.isum;
          }
          break;
        case PMB_AGG_MEAN: {
          if (s.count == 0) { valid = false; break; }
          double v;
          if (is_float(in_dt)) v = s.fsum.value() / (double)s.count;
          else if (is_signed(in_dt) || in_dt == PMB_BOOL) v = (double)(int64_t)s.isum / (double)s.count;
          else v = (double)s.isum / (double)s.count;
          if (odt == PMB_F32) { float f = (float)v; uint32_t u; memcpy(&u, &f, 4); bits = u; }
          else memcpy(&bits, &v, 8);
          break;
        }
        case PMB_AGG_MIN: case PMB_AGG_MAX: {
          if (s.count == 0) { valid = false; break; }
          bool mn = op == PMB_AGG_MIN;
          if (is_float(in_dt)) {
            double v = s.nan ? std::numeric_limits<double>::quiet_NaN() : (mn ? s.fmin : s.fmax);
            if (in_dt == PMB_F32) { float f = (float)v; uint32_t u; memcpy(&u, &f, 4); bits = u; }
            else memcpy(&bits, &v, 8);
          } else if (is_signed(in_dt) || in_dt == PMB_BOOL) {
            bits = (uint64_t)(mn ? s.imin : s.imax);
          } else {
            bits = mn ? s.umin : s.umax;
          }
          break;
        }
      }
      set_bit(oc.valid, i, valid);
      if (valid) put_value(oc, i, odt, bits);
    }
    res->cols.push_back(std::move(oc));
  }
  *out = res;
  return PMB_OK;
}

int64_t orc_result_rows(const orc_result* r) { return r->n_rows; }
int32_t orc_result_ncols(const orc_result* r) { return (int32_t)r->cols.size(); }
int32_t orc_result_dtype(const orc_result* r, int32_t c) { return r->cols[c].dtype; }
const void* orc_result_data(const orc_result* r, int32_t c) { return r->cols[c].data.data(); }
int64_t orc_result_data_bytes(const orc_result* r, int32_t c) { return (int64_t)r->cols[c].data.size(); }
const uint8_t* orc_result_validity(const orc_result* r, int32_t c) { return r->cols[c].valid.data(); }
int64_t orc_result_validity_bytes(const orc_result* r, int32_t c) { return (int64_t)r->cols[c].valid.size(); }
void orc_result_free(orc_result* r) { delete r; }

// Predicate -> keep mask (one byte per row, 1 = keep).
int orc_filter_mask(const pmb_expr* pred, const pmb_column* cols_in, int32_t n_cols, int32_t n_threads,
                    uint8_t* keep_out) {
  int64_t n;
  if (!check_columns(cols_in, n_cols, &n)) return PMB_E_INVALID;
  if (n_threads <= 0) n_threads = omp_get_max_threads();
  std::vector<Col> cols = make_cols(cols_in, n_cols);
  std::vector<uint8_t> keep;
  eval_keep(pred, cols, n, n_threads, keep);
  memcpy(keep_out, keep.data(), (size_t)n);
  return PMB_OK;
}

// Predicate -> bit-packed (data, valid) like the reference's cmp/bool kernels
// (crates/polars-metal-kernels/src/cmp.rs:9-13: data bit set only where valid and true).
int orc_predicate_bits(const pmb_expr* pred, const pmb_column* cols_in, int32_t n_cols,
                       uint8_t* out_data, uint8_t* out_valid) {
  int64_t n;
  if (!check_columns(cols_in, n_cols, &n)) return PMB_E_INVALID;
  std::vector<Col> cols = make_cols(cols_in, n_cols);
  Evaluator ev{pred->nodes, &cols};
  size_t nb = bitmap_bytes(n);
  memset(out_data, 0, nb);
  memset(out_valid, 0, nb);
  for (int64_t r = 0; r < n; r++) {
    Tri t = ev.truth(pred->root, r);
    if (t.valid) out_valid[r >> 3] |= (uint8_t)(1u << (r & 7));
    if (t.valid && t.truth) out_data[r >> 3] |= (uint8_t)(1u << (r & 7));
  }
  return PMB_OK;
}

// Kleene AND (op = 0) / OR (op = 1) of bit-packed nullable booleans
// (shaders/logical_bool.metal:3-26).
int orc_bool_logic(int32_t op, const uint8_t* ld, const uint8_t* lv, const uint8_t* rd, const uint8_t* rv,
                   int64_t n, uint8_t* od, uint8_t* ov) {
  size_t nb = bitmap_bytes(n);
  memset(od, 0, nb);
  memset(ov, 0, nb);
  for (int64_t r = 0; r < n; r++) {
    bool a_v = (lv[r >> 3] >> (r & 7)) & 1, a_t = (ld[r >> 3] >> (r & 7)) & 1;
    bool b_v = (rv[r >> 3] >> (r & 7)) & 1, b_t = (rd[r >> 3] >> (r & 7)) & 1;
    bool v, t;
    if (op == 0) {
      if ((a_v && !a_t) || (b_v && !b_t)) { v = true; t = false; }
      else if (a_v && b_v) { v = true; t = true; }
      else { v = false; t = false; }
    } else {
      if ((a_v && a_t) || (b_v && b_t)) { v = true; t = true; }
      else if (a_v && b_v) { v = true; t = false; }
      else { v = false; t = false; }
    }
    if (v) ov[r >> 3] |= (uint8_t)(1u << (r & 7));
    if (v && t) od[r >> 3] |= (uint8_t)(1u << (r & 7));
  }
  return PMB_OK;
}

// Stream compaction by a keep mask (one byte per row). Output columns keep their dtype;
// validity of dropped-in rows is carried over (filter_scatter.metal:52-185).
int orc_filter_compact(const uint8_t* keep, const pmb_column* cols_in, int32_t n_cols, orc_result** out) {
  int64_t n;
  *out = nullptr;
  if (!check_columns(cols_in, n_cols, &n)) return PMB_E_INVALID;
  std::vector<Col> cols = make_cols(cols_in, n_cols);
  int64_t m = 0;
  for (int64_t r = 0; r < n; r++) m += keep[r] ? 1 : 0;
  orc_result* res = new orc_result();
  res->n_rows = m;
  for (int c = 0; c < n_cols; c++) {
    OutCol oc;
    oc.dtype = cols[c].dtype;
    oc.data.assign(oc.dtype == PMB_BOOL ? bitmap_bytes(m) : (size_t)(m * dtype_bytes(oc.dtype)), 0);
    oc.valid.assign(bitmap_bytes(m), 0);
    int64_t o = 0;
    for (int64_t r = 0; r < n; r++) {
      if (!keep[r]) continue;
      set_bit(oc.valid, o, cols[c].is_valid(r));
      put_value(oc, o, oc.dtype, cols[c].bits(r));
      o++;
    }
    res->cols.push_back(std::move(oc));
  }
  *out = res;
  return PMB_OK;
}

// Inclusive u8 -> u32 prefix sum (the MLX cumsum the reference calls, mlx_bridge.cc:59-89).
void orc_cumsum_u8_to_u32(const uint8_t* in, uint32_t* out, int64_t n) {
  uint32_t acc = 0;
  for (int64_t i = 0; i < n; i++) { acc += in[i]; out[i] = acc; }
}

}  // extern "C"
