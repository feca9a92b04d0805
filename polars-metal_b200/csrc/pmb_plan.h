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

struct CompiledQuery {
  DQuery dq;
  ColMap map;
  int rec_words = 0;
  std::vector<uint64_t> rec_init;  // identity record, one u64 per 8 bytes
};

int pmb_compile_predicate(pmb_handle* h, const pmb_expr* e, ColMap* map, const pmb_column* cols,
                          int32_t n_user_cols, DProgram* out);
int pmb_compile_groupby(pmb_handle* h, const pmb_query* q, const pmb_column* cols, int32_t n_cols,
                        CompiledQuery* cq);
