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
  int pad;
  unsigned long long* gkeys;
  uint8_t* grecs;
  unsigned long long gcap;
  unsigned int* status;
  const unsigned long long* hot_keys;
  const unsigned int* hot_n;
  const unsigned long long* warm_keys;
  const unsigned int* warm_n;
  unsigned long long* kstats;
  int fx[8];
  int fx_e[8];
};

// shared-memory layout of the run-time kernel (per-warp 128-row unit buffers, hot and warm tiers)
struct JitPlan {
  int nt;
  int buf_bytes;      // one warp's unit buffer
  int tx_bytes;       // bytes the bulk copies of one unit deliver
  int doff[16];       // column data offset inside a unit buffer
  int voff[16];       // column validity offset (-1: no bitmap)
  int hot_cap, hot_lut, S;
  int off_buf, off_hot_lut, off_hot_recs, off_skeys, off_srecs, smem;
};

int pmb_plan_jit(pmb_handle* h, const CompiledQuery& cq, bool have_sketch, int max_smem_optin, JitPlan* J);

// JIT policy: PMB_JIT=0 never, PMB_JIT=1 always, otherwise inputs of at least 2M rows
bool pmb_jit_enabled(int64_t n_rows);
// compiled kernel for this signature and layout (cached); PMB_E_UNSUPPORTED when unavailable
int pmb_jit_hash_kernel(pmb_handle* h, const CompiledQuery& cq, const JitPlan& J, cudaKernel_t* out);
// launches over the global table and key lists set up in P (gkeys, grecs, gcap, status, lists)
int pmb_jit_launch(pmb_handle* h, cudaKernel_t k, const CompiledQuery& cq, const JitPlan& J, const HashParams& P,
                   int grid);
