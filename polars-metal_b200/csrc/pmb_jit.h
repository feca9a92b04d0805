// pmb_jit.h — run-time compiled (NVRTC) group-by kernels, see pmb_jit.cu.
#pragma once

#include "pmb_groupby.h"

// host mirror of JParams in pmb_jit_skeleton.cuh (same member order and types)
struct JitParams {
  const uint8_t* col_data[16];
  const uint8_t* col_valid[16];
  long long n_rows;
  long long n_units;
  int gprobe;
  unsigned int occ_limit;
  unsigned long long* gkeys;
  uint8_t* grecs;
  unsigned long long gcap;
  unsigned int* status;
  const unsigned long long* hot_keys;
  const unsigned int* hot_n;
  const unsigned long long* warm_keys;
  const unsigned int* warm_n;
  unsigned long long* kstats;
  const uint8_t* ttab;
  int tnb;
  int flags;  // batched kernel: bit 0 = fill the CTA's warm table
  int fx[8];
  int fx_e[8];
};

// shared-memory layout of the run-time kernel: per-warp 128-row unit buffers and queues, the
// table of sampled keys, hot records (one per warp and key) and warm records (one per key)
struct JitPlan {
  int nt, nbuf;       // threads per CTA; unit buffers per warp (2: the next unit is in flight)
  int wait_ns;        // > 0: unit waits sleep up to this many ns per test instead of spinning
  int buf_bytes;      // one unit buffer
  int tx_bytes;       // bytes the bulk copies of one unit deliver
  int doff[16];       // column data offset inside a unit buffer
  int voff[16];       // column validity offset (-1: no bitmap)
  int hot_cap;        // hot keys
  int warm_cap;       // warm keys
  int tkey;           // bytes of a key in the sampled-key table (4 for keys of at most 32 bits, else 8)
  int tnb;            // buckets of the sampled-key table (4 slots each; even), 0 without sampled keys
  int srec;           // bytes of a shared-memory record
  int off_bars, off_buf, off_q, off_tkeys, off_tval, off_srecs, smem;
};

// field offsets, size and identity words of the shared-memory record
#include <vector>
struct JitSLayout {
  std::vector<int> off;
  int bytes = 0;
  std::vector<unsigned> ident;
};
void pmb_jit_slayout(const DQuery& q, JitSLayout* S);

int pmb_plan_jit(pmb_handle* h, const CompiledQuery& cq, bool have_sketch, int max_smem_optin, JitPlan* J);

// JIT policy: PMB_JIT=0 never, PMB_JIT=1 always, otherwise inputs of at least 2M rows
bool pmb_jit_enabled(int64_t n_rows);
// compiled kernel for this signature and layout (cached); PMB_E_UNSUPPORTED when unavailable
int pmb_jit_hash_kernel(pmb_handle* h, const CompiledQuery& cq, const JitPlan& J, cudaKernel_t* out);
// host mirrors of JBatchItem / JBatch in pmb_jit_batch.cuh
struct JBatchItemH {
  int q;
  int pad;
  long long u0, u1;
};
struct JBatchH {
  const JitParams* qp;
  const JBatchItemH* items;
  long long n_items;
  unsigned long long* ticket;
};

// host mirror of JPart in pmb_jit_part.cuh (same member order and types)
struct JPartH {
  JitParams qp;
  const unsigned long long* keys;
  unsigned long long kcap;
  const unsigned int* idx;
  const unsigned long long* pstart;
  const unsigned int* items;
  long long n_items;
  int slots;
  int pad;
  unsigned long long* ticket;
  unsigned long long* gkeys;
  unsigned char* grecs;
  unsigned long long gcap;
  unsigned long long* n_groups;
};
// the partitioned strategy's aggregation kernel (pmb_jit_part.cuh) for packed keys of
// `key_words` words (cas64: one-word keys that never equal all ones, claimed by a CAS on the key);
// J receives the plan (threads, shared-memory record bytes)
int pmb_jit_part_kernel(pmb_handle* h, const CompiledQuery& cq, int key_words, bool cas64, JitPlan* J,
                        cudaKernel_t* out);

// the batched kernel (pmb_jit_batch.cuh): layout for `nt` threads with `nbuf` unit buffers per
// warp, and its compiled kernel
// warm_max > 0 caps the CTA's warm table (slots; the largest power of two that fits otherwise)
int pmb_plan_jit_batch(pmb_handle* h, const CompiledQuery& cq, int nt, int nbuf, int max_smem_optin, JitPlan* J,
                       int warm_max = 0);
int pmb_jit_batch_kernel(pmb_handle* h, const CompiledQuery& cq, const JitPlan& J, cudaKernel_t* out);
// launch parameters of pmb_jit_compact (the layout of JCParams in pmb_jit_compact.cuh)
struct JitCompactParams {
  const unsigned char* col_data[16];
  const unsigned char* col_valid[16];
  long long n_rows;
  unsigned long long* lb;
  unsigned long long* ticket;
  unsigned long long* n_out;
  unsigned int* status;
  unsigned char* out_data[16];
  unsigned int* out_valid[16];
};
constexpr int JC_TILE_ROWS = 256 * 4;  // rows per tile of pmb_jit_compact (JC_TILE)

// the top-level filter's compaction of the first n_out columns by the query's predicate
// (pmb_jit_compact.cuh); the source alone for the compile checks
std::string pmb_jit_compact_source(const CompiledQuery& cq, const JitPlan& J, int n_out);
int pmb_jit_compact_kernel(pmb_handle* h, const CompiledQuery& cq, int n_out, cudaKernel_t* out);
// launches over the global table and key lists set up in P (gkeys, grecs, gcap, status, lists)
int pmb_jit_launch(pmb_handle* h, cudaKernel_t k, const CompiledQuery& cq, const JitPlan& J, const HashParams& P,
                   int grid, const uint8_t* ttab, int tnb);
