// pmb_plan.cu — host-side compilation of a query into the device descriptor DQuery.
//
// Mirrors the reference's plan parsing and routing inputs: key/agg parsing
// (crates/polars-metal-core/src/udf/groupby/mod.rs:362-501), the predicate AST
// (crates/polars-metal-core/src/plan/mod.rs:42-60, python/polars_metal/_walker.py:1508-1644)
// and the key layout (crates/polars-metal-kernels/src/groupby.rs:195-224: per key column a
// null bit then the data bits, LSB first). Difference by design: a key column without a
// validity bitmap gets no null bit, so a non-null Int64 key packs into 64 bits.
#include <algorithm>
#include <string>
#include <vector>

#include "pmb_plan.h"

int ColMap::use(pmb_handle* h, int user_col, int32_t n_user_cols) {
  if (user_col < 0 || user_col >= n_user_cols)
    return -1 - pmb_fail(h, PMB_E_NOT_FOUND, "column index " + std::to_string(user_col) + " out of range");
  for (size_t i = 0; i < user.size(); i++)
    if (user[i] == user_col) return (int)i;
  if (user.size() >= PMB_MAX_COLS)
    return -1 - pmb_fail(h, PMB_E_UNSUPPORTED, "a query may touch at most 16 distinct columns");
  user.push_back(user_col);
  return (int)user.size() - 1;
}

namespace {

struct PredCompiler {
  pmb_handle* h;
  const pmb_expr* e;
  ColMap* map;
  int32_t n_user_cols;
  const pmb_column* cols;
  DProgram* P;
  int depth = 0, max_depth = 0;

  int fail(int code, const std::string& m) { return pmb_fail(h, code, m); }

  const pmb_expr_node* node(int i) const {
    if (i < 0 || i >= e->n_nodes) return nullptr;
    return &e->nodes[i];
  }

  bool is_value_kind(const pmb_expr_node* n) const {
    if (!n) return false;
    if (n->kind == PMB_EXPR_LIT_I64 || n->kind == PMB_EXPR_LIT_F64 || n->kind == PMB_EXPR_ARITH) return true;
    if (n->kind == PMB_EXPR_COLUMN)
      return n->column >= 0 && n->column < n_user_cols && cols[n->column].dtype != PMB_BOOL;
    return false;
  }

  // does the value subtree need float arithmetic?
  bool wants_float(const pmb_expr_node* n) const {
    if (!n) return false;
    switch (n->kind) {
      case PMB_EXPR_LIT_F64: return true;
      case PMB_EXPR_COLUMN: return n->column >= 0 && n->column < n_user_cols && pmb_is_float(cols[n->column].dtype);
      case PMB_EXPR_ARITH:
        return n->op == PMB_ARITH_TRUEDIV || n->dtype == PMB_F64 || wants_float(node(n->lhs)) ||
               wants_float(node(n->rhs));
      default: return false;
    }
  }

  int leaf(const pmb_expr_node* n, DLeaf* L) {
    L->pad = 0;
    L->i = 0;
    L->f = 0.0;
    if (n->kind == PMB_EXPR_COLUMN) {
      int c = map->use(h, n->column, n_user_cols);
      if (c < 0) return -1 - c;
      L->col = c;
      return PMB_OK;
    }
    L->col = -1;
    if (n->kind == PMB_EXPR_LIT_I64) {
      L->i = n->lit_i64;
      L->f = (double)n->lit_i64;
      return PMB_OK;
    }
    if (n->kind == PMB_EXPR_LIT_F64) {
      L->f = n->lit_f64;
      L->i = (int64_t)n->lit_f64;
      return PMB_OK;
    }
    return fail(PMB_E_UNSUPPORTED, "predicate operand must be a column or literal");
  }

  int operand(const pmb_expr_node* n, DOperand* o) {
    o->arith = -1;
    o->adtype = PMB_I64;
    for (int i = 0; i < 6; i++) o->pad[i] = 0;
    o->b = DLeaf{-1, 0, 0, 0.0};
    if (!is_value_kind(n)) return fail(PMB_E_INVALID, "compare operand is not a numeric value");
    if (n->kind == PMB_EXPR_ARITH) {
      const pmb_expr_node* a = node(n->lhs);
      const pmb_expr_node* b = node(n->rhs);
      if (!a || !b || a->kind == PMB_EXPR_ARITH || b->kind == PMB_EXPR_ARITH)
        return fail(PMB_E_UNSUPPORTED, "arithmetic in a predicate supports one level: (column|literal) op (column|literal)");
      if (n->op < PMB_ARITH_ADD || n->op > PMB_ARITH_MOD) return fail(PMB_E_INVALID, "unknown arithmetic op");
      o->arith = (int8_t)n->op;
      int rc = leaf(a, &o->a);
      if (rc) return rc;
      return leaf(b, &o->b);
    }
    return leaf(n, &o->a);
  }

  int push_term(const DTerm& t) {
    if (P->n_terms >= PMB_MAX_TERMS) return fail(PMB_E_UNSUPPORTED, "predicate has too many leaf terms (max 12)");
    P->term[P->n_terms] = t;
    return emit((int8_t)P->n_terms++);
  }
  int emit(int8_t op) {
    if (P->n_ops >= PMB_MAX_OPS) return fail(PMB_E_UNSUPPORTED, "predicate too large (max 32 ops)");
    P->ops[P->n_ops++] = op;
    if (op >= 0) {
      depth++;
      max_depth = std::max(max_depth, depth);
    } else if (op != OP_NOT) {
      depth--;
    }
    if (max_depth > 30) return fail(PMB_E_UNSUPPORTED, "predicate nesting too deep");
    return PMB_OK;
  }

  int boolean(int idx, int guard) {
    if (guard > 64) return fail(PMB_E_INVALID, "predicate graph has a cycle or is too deep");
    const pmb_expr_node* n = node(idx);
    if (!n) return fail(PMB_E_INVALID, "predicate node index out of range");
    DTerm t;
    memset(&t, 0, sizeof(t));
    t.lhs.arith = t.rhs.arith = -1;
    t.lhs.a.col = t.lhs.b.col = t.rhs.a.col = t.rhs.b.col = -1;
    switch (n->kind) {
      case PMB_EXPR_AND:
      case PMB_EXPR_OR: {
        int rc = boolean(n->lhs, guard + 1);
        if (rc) return rc;
        rc = boolean(n->rhs, guard + 1);
        if (rc) return rc;
        return emit(n->kind == PMB_EXPR_AND ? OP_AND : OP_OR);
      }
      case PMB_EXPR_NOT: {
        int rc = boolean(n->lhs, guard + 1);
        if (rc) return rc;
        return emit(OP_NOT);
      }
      case PMB_EXPR_LIT_BOOL:
        t.kind = T_LITBOOL;
        t.lhs.a.i = n->lit_i64 != 0;
        return push_term(t);
      case PMB_EXPR_COLUMN: {
        if (n->column < 0 || n->column >= n_user_cols)
          return fail(PMB_E_NOT_FOUND, "predicate column index out of range");
        if (cols[n->column].dtype != PMB_BOOL)
          return fail(PMB_E_INVALID, "a bare column in predicate position must be Boolean");
        int c = map->use(h, n->column, n_user_cols);
        if (c < 0) return -1 - c;
        t.kind = T_BOOLCOL;
        t.lhs.a.col = c;
        return push_term(t);
      }
      case PMB_EXPR_IS_NULL:
      case PMB_EXPR_IS_NOT_NULL: {
        const pmb_expr_node* a = node(n->lhs);
        if (!a || a->kind != PMB_EXPR_COLUMN) return fail(PMB_E_UNSUPPORTED, "is_null takes a column");
        int c = map->use(h, a->column, n_user_cols);
        if (c < 0) return -1 - c;
        t.kind = n->kind == PMB_EXPR_IS_NULL ? T_ISNULL : T_ISNOTNULL;
        t.dtype = PMB_I64;
        t.lhs.a.col = c;
        return push_term(t);
      }
      case PMB_EXPR_COMPARE: {
        const pmb_expr_node* a = node(n->lhs);
        const pmb_expr_node* b = node(n->rhs);
        if (!a || !b) return fail(PMB_E_INVALID, "compare node is missing an operand");
        if (n->op < PMB_CMP_EQ || n->op > PMB_CMP_GE) return fail(PMB_E_INVALID, "unknown compare op");
        int dt;
        if (n->dtype == PMB_I64 || n->dtype == PMB_F64) dt = n->dtype;
        else dt = (wants_float(a) || wants_float(b)) ? PMB_F64 : PMB_I64;
        // true division always computes in f64
        if ((a->kind == PMB_EXPR_ARITH && a->op == PMB_ARITH_TRUEDIV) ||
            (b->kind == PMB_EXPR_ARITH && b->op == PMB_ARITH_TRUEDIV))
          dt = PMB_F64;
        t.kind = T_CMP;
        t.op = (int8_t)n->op;
        t.dtype = (int8_t)dt;
        int rc = operand(a, &t.lhs);
        if (rc) return rc;
        rc = operand(b, &t.rhs);
        if (rc) return rc;
        t.lhs.adtype = t.rhs.adtype = (int8_t)dt;
        return push_term(t);
      }
      default:
        return fail(PMB_E_INVALID, "node is not a Boolean predicate");
    }
  }
};

}  // namespace

int pmb_compile_predicate(pmb_handle* h, const pmb_expr* e, ColMap* map, const pmb_column* cols,
                          int32_t n_user_cols, DProgram* out) {
  memset(out, 0, sizeof(DProgram));
  if (!e) return PMB_OK;
  if (!e->nodes || e->n_nodes <= 0) return pmb_fail(h, PMB_E_INVALID, "empty predicate");
  PredCompiler pc{h, e, map, n_user_cols, cols, out};
  return pc.boolean(e->root, 0);
}

// User columns that are non-null in every row where node `i` of the predicate is `pol` (true or
// false; a null verdict is neither) under Kleene logic: a compare or a Bool column is true or false
// only where its columns are valid, is_null is false and is_not_null true only on valid rows, AND
// is true where both sides are (false where either is), OR the other way round, NOT flips.
static void implied_valid(const pmb_expr* e, int i, bool pol, int n_user, std::vector<char>& out, int depth = 0) {
  out.assign(n_user, 0);
  if (!e || i < 0 || i >= e->n_nodes || depth > 64) return;
  const pmb_expr_node& n = e->nodes[i];
  auto columns_under = [&](auto&& self, int j, int d) -> void {
    if (j < 0 || j >= e->n_nodes || d > 64) return;
    const pmb_expr_node& m = e->nodes[j];
    if (m.kind == PMB_EXPR_COLUMN) {
      if (m.column >= 0 && m.column < n_user) out[m.column] = 1;
    } else if (m.kind == PMB_EXPR_ARITH) {
      self(self, m.lhs, d + 1);
      self(self, m.rhs, d + 1);
    }
  };
  switch (n.kind) {
    case PMB_EXPR_COMPARE:
      columns_under(columns_under, n.lhs, depth + 1);
      columns_under(columns_under, n.rhs, depth + 1);
      break;
    case PMB_EXPR_COLUMN: columns_under(columns_under, i, depth); break;
    case PMB_EXPR_IS_NULL:
      if (!pol) columns_under(columns_under, n.lhs, depth + 1);
      break;
    case PMB_EXPR_IS_NOT_NULL:
      if (pol) columns_under(columns_under, n.lhs, depth + 1);
      break;
    case PMB_EXPR_NOT: implied_valid(e, n.lhs, !pol, n_user, out, depth + 1); break;
    case PMB_EXPR_AND:
    case PMB_EXPR_OR: {
      std::vector<char> a, b;
      implied_valid(e, n.lhs, pol, n_user, a, depth + 1);
      implied_valid(e, n.rhs, pol, n_user, b, depth + 1);
      const bool uni = (n.kind == PMB_EXPR_AND) == pol;  // both sides hold: union; either: intersection
      for (int c = 0; c < n_user; c++) out[c] = uni ? (a[c] | b[c]) : (a[c] & b[c]);
      break;
    }
    default: break;
  }
}

int pmb_compile_groupby(pmb_handle* h, const pmb_query* q, const pmb_column* cols, int32_t n_cols, CompiledQuery* cq) {
  memset(&cq->dq, 0, sizeof(DQuery));
  cq->map.user.clear();
  if (!q || !cols || n_cols <= 0) return pmb_fail(h, PMB_E_INVALID, "query and columns are required");
  if (q->n_keys <= 0 || !q->key_columns) return pmb_fail(h, PMB_E_INVALID, "no key columns provided");
  if (q->n_keys > PMB_MAX_KEYS) return pmb_fail(h, PMB_E_UNSUPPORTED, "at most 8 key columns");
  if (q->n_aggs < 0 || q->n_aggs > PMB_MAX_AGGS || (q->n_aggs > 0 && !q->aggs))
    return pmb_fail(h, PMB_E_INVALID, "bad aggregation list");
  for (int i = 0; i < n_cols; i++) {
    if (cols[i].dtype < PMB_BOOL || cols[i].dtype > PMB_F64)
      return pmb_fail(h, PMB_E_INVALID, "column " + std::to_string(i) + " has an unknown dtype");
  }
  DQuery& d = cq->dq;
  // keys
  int off = 0;
  for (int k = 0; k < q->n_keys; k++) {
    int c = cq->map.use(h, q->key_columns[k], n_cols);
    if (c < 0) return -1 - c;
    const pmb_column& uc = cols[q->key_columns[k]];
    DKey& K = d.key[k];
    K.col = (int16_t)c;
    K.nullable = uc.validity != nullptr;
    K.bits = (int8_t)pmb_dtype_bits(uc.dtype);
    K.null_off = (int16_t)off;
    off += K.nullable ? 1 : 0;
    K.data_off = (int16_t)off;
    off += K.bits;
  }
  if (off > 128)
    return pmb_fail(h, PMB_E_UNSUPPORTED, "composite key width " + std::to_string(off) + " bits exceeds 128-bit budget");
  d.n_keys = q->n_keys;
  d.key_bits = off;

  // columns the filter only keeps where they are valid: their non-null count is the row count
  std::vector<char> kept_valid;
  if (q->predicate && q->predicate->nodes && q->predicate->n_nodes > 0)
    implied_valid(q->predicate, q->predicate->root, true, n_cols, kept_valid);
  else
    kept_valid.assign(n_cols, 0);

  // fields (deduplicated by kind + column)
  std::vector<DField> fields;
  auto field = [&](int kind, int col) -> int {
    for (size_t i = 0; i < fields.size(); i++)
      if (fields[i].kind == kind && (kind == F_LEN || fields[i].col == col)) return (int)i;
    DField f{};
    f.kind = (int8_t)kind;
    f.col = (int16_t)(kind == F_LEN ? 0 : col);
    fields.push_back(f);
    return (int)fields.size() - 1;
  };
  // every record carries a row count: it tells a touched group from an untouched slot
  field(F_LEN, 0);
  for (int a = 0; a < q->n_aggs; a++) {
    const pmb_agg& A = q->aggs[a];
    DAggOut& o = d.agg[a];
    o.op = (int8_t)A.op;
    o.f_main = o.f_cnt = o.f_len = -1;
    if (A.op < PMB_AGG_SUM || A.op > PMB_AGG_LEN) return pmb_fail(h, PMB_E_INVALID, "unknown aggregation op");
    if (A.op == PMB_AGG_LEN) {
      o.in_dtype = PMB_U32;
      o.out_dtype = PMB_U32;
      o.f_len = (int16_t)field(F_LEN, 0);
      continue;
    }
    int c = cq->map.use(h, A.column, n_cols);
    if (c < 0) return -1 - c;
    const pmb_column& uc = cols[A.column];
    int dt = uc.dtype;
    bool nullable = uc.validity != nullptr;
    o.in_dtype = (int8_t)dt;
    o.out_dtype = (int8_t)pmb_agg_out_dtype(A.op, dt);
    // the column's non-null count, created only for the aggregates that read it (count, mean, and
    // integer min/max, whose identity value is also a valid value); sums and float min/max need none
    auto cnt = [&]() { return (int16_t)(nullable && !kept_valid[A.column] ? field(F_CNT, c) : field(F_LEN, 0)); };
    const int fsum = std::find(cq->dd_user_cols.begin(), cq->dd_user_cols.end(), A.column) != cq->dd_user_cols.end()
                         ? F_SUM_DD
                         : F_SUM_FX;
    switch (A.op) {
      case PMB_AGG_COUNT: o.f_cnt = cnt(); break;
      case PMB_AGG_SUM:
        o.f_main = (int16_t)field(pmb_is_float(dt) ? fsum : F_SUM_I, c);
        break;
      case PMB_AGG_MEAN:
        o.f_main = (int16_t)field(pmb_is_float(dt) ? fsum : F_SUM_I, c);
        o.f_cnt = cnt();
        break;
      default: {  // min / max
        bool mn = A.op == PMB_AGG_MIN;
        if (pmb_is_float(dt)) {
          o.f_main = (int16_t)field(mn ? F_MIN_F : F_MAX_F, c);
        } else if (pmb_is_signed(dt) || dt == PMB_BOOL) {
          o.f_main = (int16_t)field(mn ? F_MIN_I : F_MAX_I, c);
          o.f_cnt = cnt();
        } else {
          o.f_main = (int16_t)field(mn ? F_MIN_U : F_MAX_U, c);
          o.f_cnt = cnt();
        }
        break;
      }
    }
  }
  if (fields.size() > PMB_MAX_FIELDS) return pmb_fail(h, PMB_E_UNSUPPORTED, "too many aggregation state fields");
  // record layout: 24-byte fields (exact float sums), then 16-, 8- and 4-byte ones, so every
  // field stays aligned to its size (at most 8)
  // (a 4-byte field first takes the spare last word of an exact float sum's 24 bytes, so the
  // hash workload's record is 48 bytes: two 32-byte sectors wherever it sits)
  int rec = 0;
  static const int kSizes[4] = {24, 16, 8, 4};
  size_t placed = 0;
  std::vector<int> spare;  // free 4-byte words inside placed fields
  for (int pass = 0; pass < 4; pass++) {
    int want = kSizes[pass];
    for (DField& f : fields) {
      uint64_t w0, w1;
      int nw, bytes;
      field_identity(f.kind, &w0, &w1, &nw, &bytes);
      if (bytes != want) continue;
      if (bytes == 4 && !spare.empty()) {
        f.off = (int16_t)spare.back();
        spare.pop_back();
      } else {
        f.off = (int16_t)rec;
        rec += bytes;
      }
      if (f.kind == F_SUM_FX) spare.push_back(f.off + 20);
      placed++;
    }
  }
  if (placed != fields.size()) return pmb_fail(h, PMB_E_CUDA, "internal: a record field has no layout slot");
  rec = (int)pmb_align((size_t)std::max(rec, 8), 8);
  // exact float sums: one range slot per column (fraction bits are set from the data sample)
  cq->fx_cols.clear();
  for (DField& f : fields) {
    if (f.kind != F_SUM_FX) continue;
    if (cq->fx_cols.size() >= PMB_MAX_FX) return pmb_fail(h, PMB_E_UNSUPPORTED, "at most 8 float-sum columns");
    f.fx_slot = (int8_t)cq->fx_cols.size();
    f.fx = 60;
    cq->fx_cols.push_back(f.col);
  }
  d.n_fields = (int)fields.size();
  for (size_t i = 0; i < fields.size(); i++) d.field[i] = fields[i];
  d.rec_bytes = rec;
  d.n_aggs = q->n_aggs;

  // predicate
  int rc = pmb_compile_predicate(h, q->predicate, &cq->map, cols, n_cols, &d.prog);
  if (rc) return rc;

  // columns and row count (pointers are filled in when the columns are staged)
  d.n_cols = (int)cq->map.user.size();
  d.valid_if_kept = 0;
  for (int c = 0; c < d.n_cols; c++) {
    d.col[c].dtype = cols[cq->map.user[c]].dtype;
    d.col[c].elem = pmb_dtype_bytes(d.col[c].dtype);
    if (kept_valid[cq->map.user[c]]) d.valid_if_kept |= 1u << c;
  }
  int64_t n = cols[cq->map.user[0]].length;
  for (int u : cq->map.user) {
    if (cols[u].length != n)
      return pmb_fail(h, PMB_E_INVALID, "row count mismatch across columns: " + std::to_string(n) + " vs " +
                                            std::to_string(cols[u].length));
  }
  if (n < 0) return pmb_fail(h, PMB_E_INVALID, "negative row count");
  if (n >= (1LL << 32) - 1) return pmb_fail(h, PMB_E_UNSUPPORTED, "a call processes fewer than 2^32 - 1 rows");
  d.n_rows = n;
  // record identity words
  cq->rec_words = rec / 8;
  std::vector<uint64_t> w(cq->rec_words, 0);
  for (const DField& f : fields) {
    uint64_t w0, w1;
    int nw, bytes;
    field_identity(f.kind, &w0, &w1, &nw, &bytes);
    if (bytes == 4) {
      // two 4-byte fields may share a word; identities of 4-byte fields are 0
      continue;
    }
    w[f.off / 8] = w0;
    if (nw == 2) w[f.off / 8 + 1] = w1;
  }
  cq->rec_init = w;
  return PMB_OK;
}
