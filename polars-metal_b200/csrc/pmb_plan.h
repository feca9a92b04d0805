// pmb_plan.h — host-side query compilation (see pmb_plan.cu).
#pragma once

#include <cstring>
#include <vector>

#include "pmb_expr.cuh"

// Maps the caller's column indices to the compact per-query column list the kernels use.
struct ColMap {
  std::vector<int> user;  // compact index -> caller's index
  // returns the compact index, or a negative value -1 - code after recording the error
  int use(pmb_handle* h, int user_col, int32_t n_user_cols);
};

#define PMB_MAX_FX 8  // float-sum columns per query

struct CompiledQuery {
  DQuery dq;
  ColMap map;
  int rec_words = 0;
  std::vector<uint64_t> rec_init;  // identity record, one u64 per 8 bytes
  std::vector<int> fx_cols;        // compact column of each exact float-sum slot
};

// fraction bits of the fixed-point float sums: |x| < 2^(94 - F); `max_expo` is the largest
// biased exponent seen, `headroom` extra powers of two on top
inline int pmb_fx_bits(unsigned max_expo, int headroom) {
  int e = (int)max_expo - 1022 + headroom;  // |x| < 2^e
  return 94 - e;
}
// set every float-sum field's fraction bits from per-slot exponents
inline void pmb_set_fx(DQuery& q, const unsigned* max_expo, int headroom) {
  for (int i = 0; i < q.n_fields; i++)
    if (q.field[i].kind == F_SUM_FX) q.field[i].fx = (int16_t)pmb_fx_bits(max_expo[q.field[i].fx_slot], headroom);
}

int pmb_compile_predicate(pmb_handle* h, const pmb_expr* e, ColMap* map, const pmb_column* cols,
                          int32_t n_user_cols, DProgram* out);
int pmb_compile_groupby(pmb_handle* h, const pmb_query* q, const pmb_column* cols, int32_t n_cols,
                        CompiledQuery* cq);
