// pmb_batched.cu — many independent group-by queries in one persistent launch.
#include "pmb_groupby.h"

extern "C" int pmb_groupby_batched(pmb_handle* h, const pmb_query* qs, const pmb_column* const* cols,
                                   const int32_t* n_cols, int32_t n_queries, pmb_result** outs) {
  if (!h) return PMB_E_INVALID;
  for (int i = 0; i < n_queries; i++) {
    int rc = pmb_groupby(h, &qs[i], cols[i], n_cols[i], &outs[i]);
    if (rc) return rc;
  }
  return PMB_OK;
}
