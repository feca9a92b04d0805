// pmb_exprcol.cu — an arithmetic expression of columns and literals evaluated for every row into
// a new column: the input of an expression aggregate such as sum(a * b) or mean(x - 1.5).
//
// The reference lowers such aggregates to trees of Column / LiteralF64 / LiteralI64 / Binary
// (Add, Sub, Mul, Div) nodes, at most 4 deep (python/polars_metal/_walker.py:1205-1278), parsed in
// crates/polars-metal-core/src/udf/groupby/mod.rs:266-352 and emitted into its fused kernel. Here
// the tree (pmb_expr nodes: PMB_EXPR_COLUMN, _LIT_I64, _LIT_F64, _ARITH) is flattened on the host
// into a postfix program that one kernel runs per row on a small value stack; the column it
// writes then goes into pmb_groupby like any other. Arithmetic: Float64 when a float column, a
// float literal or a true division takes part, else Int64 with wrapping; floor division and
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
  int as_f64;
  int kind[EC_MAX];
  int arg[EC_MAX];  // column slot, or arithmetic op
  long long li[EC_MAX];
  double lf[EC_MAX];
  int n_cols;
  const uint8_t* data[PMB_MAX_COLS];
  const uint8_t* valid[PMB_MAX_COLS];
  int elem[PMB_MAX_COLS];
  int dtype[PMB_MAX_COLS];
};

// every warp takes 32 consecutive rows at a time, so its ballot is one whole validity word
__global__ void __launch_bounds__(256) k_eval_expr(const __grid_constant__ ECProg P, int64_t n,
                                                   unsigned long long* __restrict__ out,
                                                   unsigned int* __restrict__ out_valid) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x / 32);
  for (int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32; w * 32 < n; w += warps) {
    const int64_t r = w * 32 + lane;
    bool ok = false;
    unsigned long long bits = 0;
    if (r < n) {
      double sf[EC_MAX];
      long long si[EC_MAX];
      bool sv[EC_MAX];
      int sp = 0;
      for (int k = 0; k < P.n; k++) {
        const int kind = P.kind[k];
        if (kind == EC_COL) {
          const int c = P.arg[k];
          const uint64_t b = pmb_load_bits(P.data[c], P.elem[c], r);
          sv[sp] = pmb_valid_bit(P.valid[c], r);
          if (P.as_f64) sf[sp] = pmb_bits_to_f64(b, P.dtype[c]);
          else si[sp] = (long long)pmb_bits_to_i64(b, P.dtype[c]);
          sp++;
        } else if (kind == EC_LIT_I) {
          sf[sp] = (double)P.li[k];
          si[sp] = P.li[k];
          sv[sp++] = true;
        } else if (kind == EC_LIT_F) {
          sf[sp] = P.lf[k];
          si[sp] = 0;
          sv[sp++] = true;
        } else {
          sp--;
          bool v = sv[sp - 1] && sv[sp];
          if (P.as_f64) sf[sp - 1] = pmb_arith_f64(P.arg[k], sf[sp - 1], sf[sp]);
          else si[sp - 1] = pmb_arith_i64(P.arg[k], si[sp - 1], si[sp], v);
          sv[sp - 1] = v;
        }
      }
      ok = sv[0];
      bits = P.as_f64 ? (unsigned long long)__double_as_longlong(sf[0]) : (unsigned long long)si[0];
      out[r] = ok ? bits : 0ULL;
    }
    const unsigned b = __ballot_sync(0xffffffffu, ok);
    if (lane == 0) out_valid[w] = b;
  }
}

struct Flatten {
  const pmb_expr* e;
  int n_user;
  const pmb_column* cols;
  ECProg* P;
  std::vector<int> slot_of;  // user column -> slot
  std::vector<int> user_of;  // slot -> user column
  std::string err;
  bool floaty = false;

  bool walk(int i, int depth) {
    if (i < 0 || i >= e->n_nodes) return fail("node index out of range");
    if (depth > 8) return fail("expression deeper than 8 levels");
    const pmb_expr_node& nd = e->nodes[i];
    if (P->n >= EC_MAX) return fail("expression has more than 32 nodes");
    switch (nd.kind) {
      case PMB_EXPR_COLUMN: {
        if (nd.column < 0 || nd.column >= n_user) return fail("column index out of range");
        const int dt = cols[nd.column].dtype;
        if (dt == PMB_BOOL) return fail("Bool columns have no arithmetic");
        if (dt == PMB_F32 || dt == PMB_F64) floaty = true;
        if (slot_of[nd.column] < 0) {
          if ((int)user_of.size() >= PMB_MAX_COLS) return fail("expression reads too many columns");
          slot_of[nd.column] = (int)user_of.size();
          user_of.push_back(nd.column);
        }
        P->kind[P->n] = EC_COL;
        P->arg[P->n++] = slot_of[nd.column];
        return true;
      }
      case PMB_EXPR_LIT_I64:
        P->kind[P->n] = EC_LIT_I;
        P->li[P->n++] = nd.lit_i64;
        return true;
      case PMB_EXPR_LIT_F64:
        floaty = true;
        P->kind[P->n] = EC_LIT_F;
        P->lf[P->n++] = nd.lit_f64;
        return true;
      case PMB_EXPR_ARITH:
        if (nd.op < PMB_ARITH_ADD || nd.op > PMB_ARITH_MOD) return fail("unknown arithmetic op");
        if (nd.op == PMB_ARITH_TRUEDIV) floaty = true;
        if (!walk(nd.lhs, depth + 1) || !walk(nd.rhs, depth + 1)) return false;
        if (P->n >= EC_MAX) return fail("expression has more than 32 nodes");
        P->kind[P->n] = EC_OP;
        P->arg[P->n++] = nd.op;
        return true;
      default:
        return fail("an arithmetic expression has columns, literals and arithmetic only");
    }
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
  Flatten F{expr, n_cols, cols, &P, std::vector<int>(n_cols, -1), {}, {}, false};
  if (!F.walk(expr->root, 0)) return pmb_fail(h, PMB_E_INVALID, "expression: " + F.err);
  P.as_f64 = F.floaty ? 1 : 0;
  *out_dtype = F.floaty ? PMB_F64 : PMB_I64;
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
  unsigned long long* dd = (unsigned long long*)pmb_ws_alloc(h, (size_t)n * 8 + 16);
  unsigned int* dv = (unsigned int*)pmb_ws_alloc(h, (size_t)words * 4 + 16);
  if (!dd || !dv) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (expression column)");
  if (n > 0) {
    const int blocks = (int)std::min<int64_t>((words + 7) / 8, (int64_t)h->sm_count * 8);
    pmb_kernel_begin(h, "eval_expr");
    k_eval_expr<<<blocks, 256, 0, h->stream>>>(P, n, dd, dv);
    pmb_kernel_end(h);
    PMB_CUDA(h, cudaGetLastError());
    const cudaMemcpyKind kind = out_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    PMB_CUDA(h, cudaMemcpyAsync(out_data, dd, (size_t)n * 8, kind, h->stream));
    PMB_CUDA(h, cudaMemcpyAsync(out_valid, dv, vbytes, kind, h->stream));
    if (!out_on_device) h->d2h += (int64_t)((size_t)n * 8 + vbytes);
  }
  PMB_CUDA(h, cudaStreamSynchronize(h->stream));
  pmb_call_end(h);
  return PMB_OK;
}
