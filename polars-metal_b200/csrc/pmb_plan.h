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
  // caller's columns whose float sums use double-double accumulation instead of the exact
  // fixed point (kept by pmb_compile_groupby; see PMB_FX_MIN_F)
  std::vector<int> dd_user_cols;
};

// Fewest fraction bits an exact float sum may have. A column whose range needs more integer bits
// than that leaves (an outlier far above the other values) would truncate every other group's
// small values: it is summed in double-double instead (accurate relative to each group's own
// magnitude), and the call runs again.
#define PMB_FX_MIN_F 48
// internal status: a float-sum column moved to double-double, compile the query again and re-run
#define PMB_RETRY_DD 100

// true (and the caller's columns added to cq.dd_user_cols) when a float-sum field has fewer than
// PMB_FX_MIN_F fraction bits
inline bool pmb_fx_to_dd(CompiledQuery& cq) {
  bool any = false;
  for (int i = 0; i < cq.dq.n_fields; i++) {
    const DField& f = cq.dq.field[i];
    if (f.kind != F_SUM_FX || f.fx >= PMB_FX_MIN_F) continue;
    cq.dd_user_cols.push_back(cq.map.user[f.col]);
    any = true;
  }
  return any;
}

// Fixed-point range of the exact float sums. Every value of a slot satisfies |x| < 2^E, E taken
// from the largest biased exponent seen plus `headroom` powers of two. The fraction bits F keep
// two sums in range: a partial sum of up to 2^partial_bits values (a CTA's 96-bit shared-memory
// accumulator: E + F + partial_bits <= 94) and the global table's signed high word, the sum of
// all 2^total_bits values shifted right by 32 (E + F - 32 + total_bits <= 62).
inline void pmb_set_fx(DQuery& q, const unsigned* max_expo, int headroom, int partial_bits, int total_bits) {
  for (int i = 0; i < q.n_fields; i++) {
    DField& f = q.field[i];
    if (f.kind != F_SUM_FX) continue;
    int e = (int)max_expo[f.fx_slot] - 1022 + headroom;
    q.fx_e[f.fx_slot] = (int16_t)e;
    int F = 94 - e - partial_bits;
    if (94 - e - total_bits < F) F = 94 - e - total_bits;
    f.fx = (int16_t)F;
  }
}

int pmb_compile_predicate(pmb_handle* h, const pmb_expr* e, ColMap* map, const pmb_column* cols,
                          int32_t n_user_cols, DProgram* out);
int pmb_compile_groupby(pmb_handle* h, const pmb_query* q, const pmb_column* cols, int32_t n_cols,
                        CompiledQuery* cq);
