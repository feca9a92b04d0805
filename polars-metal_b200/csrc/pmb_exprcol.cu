// pmb_exprcol.cu — an arithmetic expression of columns and literals evaluated for every row into
// a new column: the input of an expression aggregate such as sum(a * b) or mean(x - 1.5).
//
// The reference lowers such aggregates to trees of Column / LiteralF64 / LiteralI64 / Binary
// (Add, Sub, Mul, Div) nodes, at most 4 deep (python/polars_metal/_walker.py:1205-1278), parsed in
// crates/polars-metal-core/src/udf/groupby/mod.rs:266-352 and emitted into its fused kernel. Here
// the tree (pmb_expr nodes: PMB_EXPR_COLUMN, _LIT_I64, _LIT_F64, _ARITH) is flattened on the host
// into a postfix program that one kernel runs per row on a small value stack; the column it
// writes then goes into pmb_groupby like any other. Types follow Polars: both operands of a node
// are cast to their supertype (the wider integer; a signed and an unsigned integer to the signed
// type that holds both, Float64 past 64 bits; Float32 with an 8- or 16-bit integer, Float64 with a
// wider one), a float literal takes the other operand's float type (Float64 beside an integer), an
// integer literal takes the supertype of the other operand and the smallest integer type that holds
// its value (UInt8 - 1 is Int16, Int8 + 1000 is Int16, UInt64 with a negative literal is Int64), a
// subtree of literals alone is folded to its value first (Int32 when that fits, else Int64), and a
// true division of integers is Float64. Every node's value is wrapped (integers) or rounded (Float32) to its type, so 32-bit
// arithmetic wraps and rounds as Polars' does; the column has the root's type. Floor division and
// modulo follow Polars (floor, the sign of the divisor); a null operand, or an integer // or % by
// zero, makes the row null.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "pmb_groupby.h"

namespace {

constexpr int EC_MAX = 32;  // program steps (a tree 4 levels deep has at most 31 nodes)
enum { EC_COL = 0, EC_LIT_I = 1, EC_LIT_F = 2, EC_OP = 3 };

struct ECProg {
  int n;
  int out_dtype;    // the root's type
  int kind[EC_MAX];
  int arg[EC_MAX];  // column slot, or arithmetic op
  int dt[EC_MAX];   // the step's value type (an op: the type it computes in)
  int ldt[EC_MAX];  // an op's operand types
  int rdt[EC_MAX];
  long long li[EC_MAX];
  double lf[EC_MAX];
  int n_cols;
  const uint8_t* data[PMB_MAX_COLS];
  const uint8_t* valid[PMB_MAX_COLS];
  int elem[PMB_MAX_COLS];
  int dtype[PMB_MAX_COLS];
};

__host__ __device__ __forceinline__ bool ec_float(int dt) { return dt == PMB_F32 || dt == PMB_F64; }

// an integer result wrapped to its type: sign-extended for signed, zero-extended for unsigned
__device__ __forceinline__ long long ec_wrap(long long v, int dt) {
  switch (dt) {
    case PMB_I8: return (int8_t)v;
    case PMB_I16: return (int16_t)v;
    case PMB_I32: return (int32_t)v;
    case PMB_U8: return v & 0xFFLL;
    case PMB_U16: return v & 0xFFFFLL;
    case PMB_U32: return v & 0xFFFFFFFFLL;
    default: return v;
  }
}

// every warp takes 32 consecutive rows at a time, so its ballot is one whole validity word
__global__ void __launch_bounds__(256) k_eval_expr(const __grid_constant__ ECProg P, int64_t n,
                                                   uint8_t* __restrict__ out, unsigned int* __restrict__ out_valid) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x / 32);
  const int elem = pmb_dtype_bytes(P.out_dtype);
  for (int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32; w * 32 < n; w += warps) {
    const int64_t r = w * 32 + lane;
    bool ok = false;
    if (r < n) {
      double sf[EC_MAX];
      long long si[EC_MAX];
      bool sv[EC_MAX];
      int sp = 0;
      for (int k = 0; k < P.n; k++) {
        const int kind = P.kind[k];
        const int dt = P.dt[k];
        if (kind == EC_COL) {
          const int c = P.arg[k];
          const uint64_t b = pmb_load_bits(P.data[c], P.elem[c], r);
          sv[sp] = pmb_valid_bit(P.valid[c], r);
          if (ec_float(dt)) sf[sp] = pmb_bits_to_f64(b, dt);
          else si[sp] = ec_wrap((long long)b, dt);
          sp++;
        } else if (kind == EC_LIT_I) {
          if (ec_float(dt)) sf[sp] = dt == PMB_F32 ? (double)(float)P.li[k] : (double)P.li[k];
          else si[sp] = ec_wrap(P.li[k], dt);
          sv[sp++] = true;
        } else if (kind == EC_LIT_F) {
          sf[sp] = dt == PMB_F32 ? (double)(float)P.lf[k] : P.lf[k];
          si[sp] = 0;
          sv[sp++] = true;
        } else {
          sp--;
          bool v = sv[sp - 1] && sv[sp];
          const int op = P.arg[k];
          if (ec_float(dt)) {
            // operands cast to the node's float type: an integer operand converts once
            double a = ec_float(P.ldt[k]) ? sf[sp - 1] : pmb_bits_to_f64((uint64_t)si[sp - 1], P.ldt[k]);
            double b = ec_float(P.rdt[k]) ? sf[sp] : pmb_bits_to_f64((uint64_t)si[sp], P.rdt[k]);
            if (dt == PMB_F32) {
              a = (double)(float)a;
              b = (double)(float)b;
            }
            const double x = pmb_arith_f64(op, a, b);
            sf[sp - 1] = dt == PMB_F32 ? (double)(float)x : x;
          } else if (dt == PMB_U64 && (op == PMB_ARITH_FLOORDIV || op == PMB_ARITH_MOD)) {
            const unsigned long long a = (unsigned long long)si[sp - 1], b = (unsigned long long)si[sp];
            if (b == 0) {
              v = false;
              si[sp - 1] = 0;
            } else {
              si[sp - 1] = (long long)(op == PMB_ARITH_FLOORDIV ? a / b : a % b);
            }
          } else {
            si[sp - 1] = ec_wrap(pmb_arith_i64(op, si[sp - 1], si[sp], v), dt);
          }
          sv[sp - 1] = v;
        }
      }
      ok = sv[0];
      uint64_t bits = 0;
      if (ok) {
        if (P.out_dtype == PMB_F32) bits = __float_as_uint((float)sf[0]);
        else if (P.out_dtype == PMB_F64) bits = (uint64_t)__double_as_longlong(sf[0]);
        else bits = (uint64_t)si[0];
      }
      switch (elem) {
        case 1: out[r] = (uint8_t)bits; break;
        case 2: reinterpret_cast<uint16_t*>(out)[r] = (uint16_t)bits; break;
        case 4: reinterpret_cast<uint32_t*>(out)[r] = (uint32_t)bits; break;
        default: reinterpret_cast<uint64_t*>(out)[r] = bits; break;
      }
    }
    const unsigned b = __ballot_sync(0xffffffffu, ok);
    if (lane == 0) out_valid[w] = b;
  }
}

constexpr int DYN_INT = -1;    // an integer literal (or literals only): takes the other operand's type
constexpr int DYN_FLOAT = -2;  // a float literal: the other operand's float type, else Float64

bool ec_signed(int dt) { return dt == PMB_I8 || dt == PMB_I16 || dt == PMB_I32 || dt == PMB_I64; }
int ec_bits(int dt) { return 8 * pmb_dtype_bytes(dt); }
int ec_signed_of_bits(int bits) {
  return bits <= 8 ? PMB_I8 : bits <= 16 ? PMB_I16 : bits <= 32 ? PMB_I32 : PMB_I64;
}

// Polars' supertype of two numeric types
int ec_supertype(int a, int b) {
  if (a == b) return a;
  if (ec_float(a) || ec_float(b)) {
    if (a == PMB_F64 || b == PMB_F64) return PMB_F64;
    const int other = a == PMB_F32 ? b : a;
    return (other == PMB_I8 || other == PMB_I16 || other == PMB_U8 || other == PMB_U16) ? PMB_F32 : PMB_F64;
  }
  if (ec_signed(a) == ec_signed(b)) return ec_bits(a) >= ec_bits(b) ? a : b;
  const int sg = ec_signed(a) ? a : b, un = ec_signed(a) ? b : a;
  if (ec_bits(un) < ec_bits(sg)) return sg;
  return 2 * ec_bits(un) <= 64 ? ec_signed_of_bits(2 * ec_bits(un)) : PMB_F64;
}

bool ec_unsigned(int dt) { return dt == PMB_U8 || dt == PMB_U16 || dt == PMB_U32 || dt == PMB_U64; }

// the smallest integer type that holds v: unsigned when `want_unsigned` and v >= 0, else signed
int ec_fit(long long v, bool want_unsigned) {
  if (want_unsigned && v >= 0) {
    const unsigned long long u = (unsigned long long)v;
    return u <= 0xFFull ? PMB_U8 : u <= 0xFFFFull ? PMB_U16 : u <= 0xFFFFFFFFull ? PMB_U32 : PMB_U64;
  }
  if (v >= -128 && v <= 127) return PMB_I8;
  if (v >= -32768 && v <= 32767) return PMB_I16;
  if (v >= -2147483648LL && v <= 2147483647LL) return PMB_I32;
  return PMB_I64;
}

// the type of an integer literal of value v (when `known`) beside an operand of type t: Polars'
// supertype of t and the smallest type holding v (its rule for a dynamic integer literal); a
// literal beside a float operand takes the float type
int ec_adopt_int(long long v, bool known, int t) {
  if (ec_float(t)) return t;
  if (!known) return t;
  const int fit = ec_fit(v, ec_unsigned(t));
  if (t == PMB_U64 && ec_signed(fit)) return PMB_I64;  // not Float64: a literal never forces floats
  return ec_supertype(t, fit);
}

int ec_adopt_float(int t) { return ec_float(t) ? t : PMB_F64; }

// a subtree of integer literals alone, folded to one value (Polars folds literal arithmetic before
// typing); false when the fold divides by zero
bool ec_fold(int op, long long a, long long b, long long* out) {
  const unsigned long long ua = (unsigned long long)a, ub = (unsigned long long)b;
  switch (op) {
    case PMB_ARITH_ADD: *out = (long long)(ua + ub); return true;
    case PMB_ARITH_SUB: *out = (long long)(ua - ub); return true;
    case PMB_ARITH_MUL: *out = (long long)(ua * ub); return true;
    case PMB_ARITH_FLOORDIV:
    case PMB_ARITH_MOD: {
      if (b == 0) return false;
      if (b == -1) {
        *out = op == PMB_ARITH_MOD ? 0 : (long long)(0ull - ua);
        return true;
      }
      long long q = a / b, m = a % b;
      if (m != 0 && ((m < 0) != (b < 0))) {
        q -= 1;
        m += b;
      }
      *out = op == PMB_ARITH_MOD ? m : q;
      return true;
    }
    default: return false;
  }
}

int ec_concrete(int t, int ctx, long long v, bool known) {
  if (t >= 0) return t;
  if (t == DYN_INT) {
    if (ctx >= 0) return ctx;
    return (known && ec_fit(v, false) == PMB_I64) ? PMB_I64 : PMB_I32;  // Int32 unless the value needs 64 bits
  }
  return (ctx >= 0 && ec_float(ctx)) ? ctx : PMB_F64;
}

struct Flatten {
  const pmb_expr* e;
  int n_user;
  const pmb_column* cols;
  ECProg* P;
  std::vector<int> slot_of;  // user column -> slot
  std::vector<int> user_of;  // slot -> user column
  std::vector<int> node_t;   // per node: its type, or DYN_INT / DYN_FLOAT
  std::vector<long long> node_v;  // per DYN_INT node: its folded value
  std::vector<char> node_known;   // ... when the fold succeeded
  std::string err;
  int count = 0;

  // pass 1: checks and types, bottom-up
  bool type(int i, int depth, int* t) {
    if (i < 0 || i >= e->n_nodes) return fail("node index out of range");
    if (depth > 8) return fail("expression deeper than 8 levels");
    if (++count > EC_MAX) return fail("expression has more than 32 nodes");
    const pmb_expr_node& nd = e->nodes[i];
    switch (nd.kind) {
      case PMB_EXPR_COLUMN: {
        if (nd.column < 0 || nd.column >= n_user) return fail("column index out of range");
        const int dt = cols[nd.column].dtype;
        if (dt == PMB_BOOL) return fail("Bool columns have no arithmetic");
        if (dt < PMB_BOOL || dt > PMB_F64) return fail("unknown column dtype");
        *t = dt;
        break;
      }
      case PMB_EXPR_LIT_I64:
        *t = DYN_INT;
        node_v[i] = nd.lit_i64;
        node_known[i] = 1;
        break;
      case PMB_EXPR_LIT_F64: *t = DYN_FLOAT; break;
      case PMB_EXPR_ARITH: {
        if (nd.op < PMB_ARITH_ADD || nd.op > PMB_ARITH_MOD) return fail("unknown arithmetic op");
        int a, b;
        if (!type(nd.lhs, depth + 1, &a) || !type(nd.rhs, depth + 1, &b)) return false;
        int r;
        if (a < 0 && b < 0) {
          r = (a == DYN_FLOAT || b == DYN_FLOAT || nd.op == PMB_ARITH_TRUEDIV) ? DYN_FLOAT : DYN_INT;
          if (r == DYN_INT && node_known[nd.lhs] && node_known[nd.rhs]) {
            long long v;
            if (ec_fold(nd.op, node_v[nd.lhs], node_v[nd.rhs], &v)) {
              node_v[i] = v;
              node_known[i] = 1;
            }
          }
        } else if (a < 0) {
          r = a == DYN_INT ? ec_adopt_int(node_v[nd.lhs], node_known[nd.lhs], b) : ec_adopt_float(b);
        } else if (b < 0) {
          r = b == DYN_INT ? ec_adopt_int(node_v[nd.rhs], node_known[nd.rhs], a) : ec_adopt_float(a);
        } else {
          r = ec_supertype(a, b);
        }
        if (r >= 0 && nd.op == PMB_ARITH_TRUEDIV && !ec_float(r)) r = PMB_F64;
        *t = r;
        break;
      }
      default:
        return fail("an arithmetic expression has columns, literals and arithmetic only");
    }
    node_t[i] = *t;
    return true;
  }

  // pass 2: literals and literal-only nodes take their context's type; postfix program
  bool emit(int i, int ctx, int* out_t) {
    const pmb_expr_node& nd = e->nodes[i];
    const int t = ec_concrete(node_t[i], ctx, node_v[i], node_known[i] != 0);
    if (P->n >= EC_MAX) return fail("expression has more than 32 nodes");
    switch (nd.kind) {
      case PMB_EXPR_COLUMN:
        if (slot_of[nd.column] < 0) {
          if ((int)user_of.size() >= PMB_MAX_COLS) return fail("expression reads too many columns");
          slot_of[nd.column] = (int)user_of.size();
          user_of.push_back(nd.column);
        }
        P->kind[P->n] = EC_COL;
        P->arg[P->n] = slot_of[nd.column];
        break;
      case PMB_EXPR_LIT_I64:
        P->kind[P->n] = EC_LIT_I;
        P->li[P->n] = nd.lit_i64;
        break;
      case PMB_EXPR_LIT_F64:
        P->kind[P->n] = EC_LIT_F;
        P->lf[P->n] = nd.lit_f64;
        break;
      default: {
        int lt, rt;
        if (!emit(nd.lhs, t, &lt) || !emit(nd.rhs, t, &rt)) return false;
        if (P->n >= EC_MAX) return fail("expression has more than 32 nodes");
        P->kind[P->n] = EC_OP;
        P->arg[P->n] = nd.op;
        P->ldt[P->n] = lt;
        P->rdt[P->n] = rt;
        break;
      }
    }
    P->dt[P->n++] = t;
    *out_t = t;
    return true;
  }

  bool run(int root) {
    node_t.assign(e->n_nodes, 0);
    node_v.assign(e->n_nodes, 0);
    node_known.assign(e->n_nodes, 0);
    int t;
    if (!type(root, 0, &t)) return false;
    int out;
    if (!emit(root, -1, &out)) return false;
    P->out_dtype = out;
    return true;
  }

  bool fail(const char* m) {
    err = m;
    return false;
  }
};

}  // namespace

extern "C" int pmb_eval_expr(pmb_handle* h, const pmb_expr* expr, const pmb_column* cols, int32_t n_cols,
                             void* out_data, uint8_t* out_valid, int32_t out_on_device, int32_t* out_dtype) {
  if (!h) return PMB_E_INVALID;
  if (!expr || !expr->nodes || !cols || n_cols <= 0 || !out_data || !out_valid || !out_dtype)
    return pmb_fail(h, PMB_E_INVALID, "expression, columns and outputs are required");
  const int64_t n = cols[0].length;
  for (int c = 1; c < n_cols; c++)
    if (cols[c].length != n) return pmb_fail(h, PMB_E_INVALID, "expression columns differ in length");
  ECProg P;
  memset(&P, 0, sizeof(P));
  Flatten F{expr, n_cols, cols, &P, std::vector<int>(n_cols, -1), {}, {}, {}, {}, {}};
  if (!F.run(expr->root)) return pmb_fail(h, PMB_E_INVALID, "expression: " + F.err);
  *out_dtype = P.out_dtype;
  PMB_CUDA(h, cudaSetDevice(h->device));
  int rc = pmb_ws_begin(h);
  if (rc) return rc;
  pmb_call_begin(h);
  P.n_cols = (int)F.user_of.size();
  for (int s = 0; s < P.n_cols; s++) {
    DCol d;
    memset(&d, 0, sizeof(d));
    rc = pmb_stage_column(h, cols[F.user_of[s]], n, &d);
    if (rc) return rc;
    P.data[s] = d.data;
    P.valid[s] = d.valid;
    P.elem[s] = d.elem;
    P.dtype[s] = d.dtype;
  }
  const int64_t words = (n + 31) / 32;
  const size_t vbytes = (size_t)((n + 7) / 8);
  const size_t ob = (size_t)n * pmb_dtype_bytes(P.out_dtype);
  uint8_t* dd = (uint8_t*)pmb_ws_alloc(h, ob + 16);
  unsigned int* dv = (unsigned int*)pmb_ws_alloc(h, (size_t)words * 4 + 16);
  if (!dd || !dv) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (expression column)");
  if (n > 0) {
    const int blocks = (int)std::min<int64_t>((words + 7) / 8, (int64_t)h->sm_count * 8);
    pmb_kernel_begin(h, "eval_expr");
    k_eval_expr<<<blocks, 256, 0, h->stream>>>(P, n, dd, dv);
    pmb_kernel_end(h);
    PMB_CUDA(h, cudaGetLastError());
    const cudaMemcpyKind kind = out_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    PMB_CUDA(h, cudaMemcpyAsync(out_data, dd, ob, kind, h->stream));
    PMB_CUDA(h, cudaMemcpyAsync(out_valid, dv, vbytes, kind, h->stream));
    if (!out_on_device) h->d2h += (int64_t)(ob + vbytes);
  }
  PMB_CUDA(h, cudaStreamSynchronize(h->stream));
  pmb_call_end(h);
  return PMB_OK;
}

extern "C" int pmb_expr_dtype(const pmb_expr* expr, const pmb_column* cols, int32_t n_cols, int32_t* out_dtype) {
  if (!expr || !expr->nodes || !cols || n_cols <= 0 || !out_dtype) return PMB_E_INVALID;
  ECProg P;
  memset(&P, 0, sizeof(P));
  Flatten F{expr, n_cols, cols, &P, std::vector<int>(n_cols, -1), {}, {}, {}, {}, {}};
  if (!F.run(expr->root)) return PMB_E_INVALID;
  *out_dtype = P.out_dtype;
  return PMB_OK;
}
