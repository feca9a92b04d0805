// pmb_groupby.cu — filter -> group_by -> fused aggregate on sm_100a.
//
// Replaces, for this path: `_native.execute_groupby` (crates/polars-metal-core/src/udf/groupby/mod.rs:747-1144),
// the CPU compaction it is fed from (python/polars_metal/_udf.py:550-597), key encoding
// (crates/polars-metal-kernels/src/groupby.rs:155-302), the build strategies A1/A3
// (groupby.rs:450-538, src/groupby_build_partitioned/gpu.rs:115-258, src/groupby_global_hash/gpu.rs:34-123),
// the per-aggregation CPU folds (groupby.rs:1268-1700) and the fused-aggregate kernel
// (groupby.rs:2599-2833, src/aggregate_fused/emitter.rs:189-393).
//
// Design (one pass over the input, no row_to_group materialisation):
//   k_sketch     — 65,536 sampled rows -> distinct / singleton counts -> group estimate
//   k_table_init — global open-addressing table: keys = EMPTY, records = identity
//   k_hash_agg   — persistent CTAs; each column tile arrives in shared memory by 1-D TMA bulk
//                  copies (cp.async.bulk + mbarrier, multi-stage ring); per row: predicate in
//                  registers -> packed key -> per-CTA shared-memory table (hot keys) or the
//                  global table -> fused state update with atomics; at exit the shared table is
//                  merged into the global one.
//   k_finalize   — occupied slots -> dense output columns in slot order (single pass,
//                  decoupled look-back), keys decoded, aggregates finalised (Arrow layout).
// A capacity overflow (probe limit) sets a status bit; the host re-runs with 4x capacity, so
// the estimate can only cost time, never change results.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pmb_groupby.h"
#include "pmb_jit.h"

// ============================================================================ sketch
#define SK_SAMPLES 65536
#define SK_SLOTS (1 << 18)

struct FxCols {
  int n;
  int col[PMB_MAX_FX];
};

template <bool K128>
__global__ void k_sketch(const __grid_constant__ DQuery q, int64_t m, unsigned long long* __restrict__ set_keys,
                         unsigned int* __restrict__ set_cnt, const __grid_constant__ FxCols fxc,
                         unsigned int* __restrict__ fx_expo) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  int64_t row = (m == q.n_rows) ? i : (int64_t)((double)i * (double)q.n_rows / (double)m);
  if (row >= q.n_rows) row = q.n_rows - 1;
  TileCtx t{nullptr, nullptr, nullptr, 0};
  // largest exponent of the finite values of each float-sum column (fixed-point range)
  for (int f = 0; f < fxc.n; f++) {
    int c = fxc.col[f];
    if (!tc_isvalid(q, t, c, row)) continue;
    double x = pmb_bits_to_f64(tc_bits(q, t, c, row), q.col[c].dtype);
    if (!pmb_fx_flag(x)) atomicMax(&fx_expo[f], (unsigned)pmb_fx_expo(x));
  }
  uint64_t k;
  if (K128) {
    Key128 kk = pack_key128(q, t, row);
    k = pmb_fmix64(kk.lo ^ pmb_fmix64(kk.hi + 0x9E3779B97F4A7C15ULL));
  } else {
    k = pack_key64(q, t, row);
  }
  if (k == PMB_EMPTY64) k = PMB_EMPTY64 - 1;
  uint32_t s = (uint32_t)(pmb_fmix64(k) & (SK_SLOTS - 1));
  for (int p = 0; p < SK_SLOTS; p++) {
    unsigned long long cur = set_keys[s];
    if (cur == k) break;
    if (cur == PMB_EMPTY64) {
      unsigned long long old = atomicCAS(&set_keys[s], PMB_EMPTY64, k);
      if (old == PMB_EMPTY64 || old == k) break;
    }
    s = (s + 1) & (SK_SLOTS - 1);
  }
  atomicAdd(&set_cnt[s], 1u);
}

// distinct count, singletons, doubletons and the histogram of per-key sample counts
__global__ void k_sketch_reduce(const unsigned long long* __restrict__ set_keys,
                                const unsigned int* __restrict__ set_cnt, unsigned long long* __restrict__ out,
                                unsigned int* __restrict__ hist) {
  __shared__ unsigned long long acc[3];
  __shared__ unsigned int sh[SK_HIST];
  if (threadIdx.x < 3) acc[threadIdx.x] = 0;
  for (int i = threadIdx.x; i < SK_HIST; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  unsigned long long d = 0, f1 = 0, f2 = 0;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < SK_SLOTS; s += gridDim.x * blockDim.x) {
    if (set_keys[s] != PMB_EMPTY64) {
      d++;
      unsigned int c = set_cnt[s];
      f1 += c == 1;
      f2 += c == 2;
      atomicAdd(&sh[c < SK_HIST ? c : SK_HIST - 1], 1u);
    }
  }
  atomicAdd(&acc[0], d);
  atomicAdd(&acc[1], f1);
  atomicAdd(&acc[2], f2);
  __syncthreads();
  if (threadIdx.x < 3) atomicAdd(&out[threadIdx.x], acc[threadIdx.x]);
  for (int i = threadIdx.x; i < SK_HIST; i += blockDim.x)
    if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// keys of the sample with count >= t1 -> hot list, t2 <= count < t1 -> warm list
__global__ void k_sketch_select(const unsigned long long* __restrict__ set_keys, const unsigned int* __restrict__ set_cnt,
                                unsigned int t1, unsigned int t2, unsigned long long* __restrict__ hot,
                                unsigned int* __restrict__ hot_n, unsigned int hot_cap,
                                unsigned long long* __restrict__ warm, unsigned int* __restrict__ warm_n,
                                unsigned int warm_cap) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < SK_SLOTS; s += gridDim.x * blockDim.x) {
    unsigned long long k = set_keys[s];
    if (k == PMB_EMPTY64) continue;
    unsigned int c = set_cnt[s];
    if (c >= t1) {
      unsigned int i = atomicAdd(hot_n, 1u);
      if (i < hot_cap) hot[i] = k;
    } else if (c >= t2) {
      unsigned int i = atomicAdd(warm_n, 1u);
      if (i < warm_cap) warm[i] = k;
    }
  }
}

// The run-time kernel's table of sampled keys, built on the device from the hot and warm lists so
// the host never reads them back: `tnb` buckets of 4 slots, keys (4-byte keys when `narrow`, else
// 8-byte) then 16-bit values (0x8000 | hot index, or the warm index). A key takes a slot of its
// first bucket (the kernel's j_hash) and, only when that bucket is full, of its second: so a first
// bucket with an empty slot holds every key whose first choice it is, and the lookup stops there.
// Hot keys go in first; a key that finds both buckets full is left out and its rows take the
// global table, which gives the same results. Empty slots hold the value 0xFFFF. A bucket that
// turned a key away (more than 4 keys tried it) gets bit 14 set in its first slot's value (a full
// bucket's first slot is never empty, and indices stay below 2^14), so a lookup of an absent key
// reads the second bucket only behind such a bucket, not behind every full one. One CTA.
__device__ __forceinline__ void sample_table_insert(unsigned long long k, unsigned short v, unsigned tnb, bool narrow,
                                                    unsigned char* tab, unsigned int* fill) {
  if (k == PMB_EMPTY64 || (narrow && k > 0xFFFFFFFFull)) return;  // never looked up in the table
  unsigned long long hk;
  if (narrow) {
    const uint32_t x = pmb_fmix32((uint32_t)k);
    hk = ((unsigned long long)x << 32) | x;
  } else {
    hk = pmb_fmix64(k);
  }
  const unsigned a = (unsigned)(hk >> 32);
  unsigned bk = __umulhi(a, tnb), sl = atomicAdd(&fill[bk], 1u);
  if (sl >= 4u) {
    bk = __umulhi(pmb_mix32b(a), tnb);
    sl = atomicAdd(&fill[bk], 1u);
    if (sl >= 4u) return;
  }
  const unsigned at = 4u * bk + sl;
  if (narrow) reinterpret_cast<unsigned int*>(tab)[at] = (unsigned int)k;
  else reinterpret_cast<unsigned long long*>(tab)[at] = k;
  reinterpret_cast<unsigned short*>(tab + (size_t)tnb * 4u * (narrow ? 4u : 8u))[at] = v;
}

__global__ void __launch_bounds__(1024) k_sample_table(const unsigned long long* __restrict__ hot,
                                                       const unsigned int* __restrict__ hot_n, unsigned hot_cap,
                                                       const unsigned long long* __restrict__ warm,
                                                       const unsigned int* __restrict__ warm_n, unsigned warm_cap,
                                                       unsigned tnb, int narrow, unsigned char* __restrict__ tab,
                                                       unsigned int* __restrict__ fill) {
  const unsigned slots = 4u * tnb;
  const unsigned kb = slots * (narrow ? 4u : 8u);
  for (unsigned i = threadIdx.x; i < slots; i += blockDim.x) {
    if (narrow) reinterpret_cast<unsigned int*>(tab)[i] = 0xFFFFFFFFu;
    else reinterpret_cast<unsigned long long*>(tab)[i] = PMB_EMPTY64;
    reinterpret_cast<unsigned short*>(tab + kb)[i] = 0xFFFFu;
  }
  for (unsigned i = threadIdx.x; i < tnb; i += blockDim.x) fill[i] = 0u;
  __syncthreads();
  const unsigned nh = hot ? min(*hot_n, hot_cap) : 0u;
  for (unsigned i = threadIdx.x; i < nh; i += blockDim.x)
    sample_table_insert(hot[i], (unsigned short)(0x8000u | i), tnb, narrow != 0, tab, fill);
  __syncthreads();
  const unsigned nw = warm ? min(*warm_n, warm_cap) : 0u;
  for (unsigned i = threadIdx.x; i < nw; i += blockDim.x)
    sample_table_insert(warm[i], (unsigned short)i, tnb, narrow != 0, tab, fill);
  __syncthreads();
  unsigned short* vals = reinterpret_cast<unsigned short*>(tab + kb);
  for (unsigned i = threadIdx.x; i < tnb; i += blockDim.x)
    if (fill[i] > 4u) vals[4u * i] |= 0x4000u;
}

// ============================================================================ table init
// Regions of 32-bit words to clear in the same launch as the table (a call's status words,
// look-back states and output bitmaps), instead of one cudaMemsetAsync each.
struct ZeroList {
  int n;
  unsigned int* p[24];
  int64_t words[24];
};
// adds `bytes` (a multiple of 4) at p; false when the list is full (the caller clears it itself)
static bool zl_add(ZeroList& z, void* p, size_t bytes) {
  if (z.n == 24 || (bytes & 3u) || ((uintptr_t)p & 3u)) return false;
  z.p[z.n] = (unsigned int*)p;
  z.words[z.n++] = (int64_t)(bytes / 4);
  return true;
}

__global__ void k_table_init(unsigned long long* __restrict__ keys, int64_t key_words, uint64_t* __restrict__ recs,
                             int64_t n_recs, int rec_words, const __grid_constant__ RecInit ri,
                             const __grid_constant__ ZeroList z) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t k = i; k < key_words; k += stride) keys[k] = PMB_EMPTY64;
  int64_t total = n_recs * rec_words;
  for (int64_t w = i; w < total; w += stride) recs[w] = ri.w[w % rec_words];
  for (int j = 0; j < z.n; j++)
    for (int64_t w = i; w < z.words[j]; w += stride) z.p[j][w] = 0u;
}

// launcher of k_table_init for other translation units (batched tables)
void k_table_init_pub(unsigned long long* keys, int64_t key_words, uint64_t* recs, int64_t n_recs, int rec_words,
                      const RecInit& ri, int blocks, cudaStream_t s) {
  ZeroList z;
  z.n = 0;
  k_table_init<<<blocks, 256, 0, s>>>(keys, key_words, recs, n_recs, rec_words, ri, z);
}

// ============================================================================ global table
__device__ __forceinline__ int64_t gfind64(const HashParams& P, uint64_t key, uint64_t h) {
  if (key == PMB_EMPTY64) {
    if (*(volatile unsigned int*)&P.status[1] == 0) atomicOr(&P.status[1], 1u);
    return (int64_t)P.gcap;
  }
  uint64_t i = pmb_slot(h, P.gcap);
  unsigned long long* keys = P.gkeys;
  for (int p = 0; p < P.gprobe; p++) {
    unsigned long long k = keys[i];
    if (k == key) return (int64_t)i;
    if (k == PMB_EMPTY64) {
      unsigned long long old = atomicCAS(&keys[i], PMB_EMPTY64, key);
      if (old == PMB_EMPTY64 || old == key) return (int64_t)i;
    }
    i = (i + 1 == P.gcap) ? 0 : i + 1;
  }
  atomicOr(P.status, PMB_ST_OVERFLOW);
  return -1;
}

struct __align__(16) K128Slot {
  unsigned long long lo, hi;
};

__device__ __forceinline__ int64_t gfind128(const HashParams& P, Key128 key, uint64_t h) {
  if (key.lo == PMB_EMPTY64 && key.hi == PMB_EMPTY64) {
    if (*(volatile unsigned int*)&P.status[1] == 0) atomicOr(&P.status[1], 1u);
    return (int64_t)P.gcap;
  }
  uint64_t i = pmb_slot(h, P.gcap);
  K128Slot* keys = reinterpret_cast<K128Slot*>(P.gkeys);
  for (int p = 0; p < P.gprobe; p++) {
    K128Slot cur = keys[i];
    if (cur.lo == key.lo && cur.hi == key.hi) return (int64_t)i;
    // a 16-byte load may observe a slot mid-publication: any EMPTY half means "ask the CAS"
    if (cur.lo == PMB_EMPTY64 || cur.hi == PMB_EMPTY64) {
      K128Slot want{key.lo, key.hi}, empty{PMB_EMPTY64, PMB_EMPTY64};
      K128Slot old = atomicCAS(&keys[i], empty, want);
      if ((old.lo == PMB_EMPTY64 && old.hi == PMB_EMPTY64) || (old.lo == key.lo && old.hi == key.hi))
        return (int64_t)i;
    }
    i = (i + 1 == P.gcap) ? 0 : i + 1;
  }
  atomicOr(P.status, PMB_ST_OVERFLOW);
  return -1;
}

// ============================================================================ fused hash aggregation
__device__ __forceinline__ int sfind64(unsigned long long* skeys, int S, int probes, uint64_t key, uint64_t h) {
  if (key == PMB_EMPTY64) return -1;
  int i = (int)((h >> 40) & (uint64_t)(S - 1));
  for (int p = 0; p < probes; p++) {
    unsigned long long k = skeys[i];
    if (k == key) return i;
    if (k == PMB_EMPTY64) {
      unsigned long long old = atomicCAS(&skeys[i], PMB_EMPTY64, (unsigned long long)key);
      if (old == PMB_EMPTY64 || old == key) return i;
    }
    i = (i + 1) & (S - 1);
  }
  return -1;
}

// read-only lookup in the hot-key table (built once per CTA); -1 when the key is not hot
__device__ __forceinline__ int hot_find(const unsigned long long* lk, const int* li, int slots, uint64_t key, uint64_t h) {
  int i = (int)((h >> 24) & (uint64_t)(slots - 1));
  for (int p = 0; p < slots; p++) {
    unsigned long long k = lk[i];
    if (k == key) return li[i];
    if (k == PMB_EMPTY64) return -1;
    i = (i + 1) & (slots - 1);
  }
  return -1;
}

// per-thread cycle accumulators of the optional phase counters
struct PathCycles {
  long long pred = 0, hot = 0, smem = 0, sfind = 0, gfind = 0, apply = 0;
};

// Processes rows [base, base + NT) of a tile, one row per thread, the whole warp together:
//   hot keys    -> warp-private records: lanes with the same hot key are grouped with
//                  __match_any_sync and the group's first lane applies all their rows (no atomics);
//   other keys  -> the CTA-shared table when the key is (or can be) there, else the global table.
// Returns bit 0 = row went to the shared table, bit 1 = row went global (for phase counters).
template <int NT, bool K128>
__device__ __forceinline__ int process_rows(const HashParams& P, const DQuery& q, const TileCtx& t, int lr, bool in_range,
                                            unsigned long long* skeys, uint8_t* srecs, const unsigned long long* hlk,
                                            const int* hli, uint8_t* hrecs, int n_hot, PathCycles& pc) {
  const int lane = threadIdx.x & 31;
  const int rb = q.rec_bytes;
  const bool ks = P.kstats != nullptr;
  long long ck0 = ks ? clock64() : 0;
  bool keep = in_range && eval_keep(q, t, lr);
  if (keep) fx_range_check(q, t, lr, P.status);
  if (K128) {
    if (!keep) return 0;
    Key128 key = pack_key128(q, t, lr);
    uint64_t h = pmb_fmix64(key.lo ^ pmb_fmix64(key.hi + 0x9E3779B97F4A7C15ULL));
    int64_t gi = gfind128(P, key, h);
    if (gi >= 0) apply_row_global(q, t, P.grecs + (size_t)gi * rb, lr);
    return 2;
  }
  uint64_t key = keep ? pack_key64(q, t, lr) : 0;
  uint64_t h = pmb_fmix64(key);
  int hot = -1;
  if (n_hot && keep && key != PMB_EMPTY64) hot = hot_find(hlk, hli, P.hot_lut_slots, key, h);
  long long ck1 = ks ? clock64() : 0;
  unsigned hot_mask = __ballot_sync(0xffffffffu, hot >= 0);
  if (hot_mask) {
    unsigned peers = __match_any_sync(0xffffffffu, hot) & hot_mask;
    if (hot >= 0 && lane == __ffs(peers) - 1) {
      uint8_t* rec = hrecs + ((size_t)(threadIdx.x >> 5) * P.hot_cap + hot) * rb;
      for (unsigned m = peers; m; m &= m - 1) apply_row_private(q, t, rec, lr - lane + (__ffs(m) - 1));
    }
  }
  __syncwarp();
  long long ck2 = ks ? clock64() : 0;
  if (ks) {
    pc.pred += ck1 - ck0;
    pc.hot += ck2 - ck1;
  }
  if (!keep || hot >= 0) return 0;
  if (P.smem_slots) {
    int si = sfind64(skeys, P.smem_slots, P.smem_probe, key, h);
    if (si >= 0) {
      apply_row_shared(q, t, srecs + (size_t)si * rb, lr);
      if (ks) pc.smem += clock64() - ck2;
      return 1;
    }
  }
  long long ck3 = ks ? clock64() : 0;
  int64_t gi = gfind64(P, key, h);
  long long ck4 = ks ? clock64() : 0;
  if (gi >= 0) apply_row_global(q, t, P.grecs + (size_t)gi * rb, lr);
  if (ks) {
    pc.sfind += ck3 - ck2;
    pc.gfind += ck4 - ck3;
    pc.apply += clock64() - ck4;
  }
  return 2;
}

template <int NT, bool K128>
__global__ void __launch_bounds__(NT, 1) k_hash_agg(const __grid_constant__ HashParams P) {
  extern __shared__ __align__(128) uint8_t sm[];
  __shared__ int32_t s_doff[PMB_MAX_COLS];
  __shared__ int32_t s_voff[PMB_MAX_COLS];
  __shared__ int s_abort;
  // the query descriptor is read with data-dependent indices on every row: keep a copy in
  // shared memory (parameter space would serialise those reads through the constant cache)
  __shared__ __align__(16) DQuery sq;
  const int tid = threadIdx.x;
  for (int i = tid; i < (int)(sizeof(DQuery) / 4); i += NT)
    reinterpret_cast<uint32_t*>(&sq)[i] = reinterpret_cast<const uint32_t*>(&P.q)[i];
  __syncthreads();
  const DQuery& q = sq;
  constexpr int W = NT / 32;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm);
  unsigned long long* skeys = reinterpret_cast<unsigned long long*>(sm + P.smem_keys_off);
  uint8_t* srecs = sm + P.smem_recs_off;
  unsigned long long* hlk = reinterpret_cast<unsigned long long*>(sm + P.hot_lut_off);
  int* hli = reinterpret_cast<int*>(sm + P.hot_lut_off + 8 * P.hot_lut_slots);
  uint8_t* hrecs = sm + P.hot_recs_off;
  const int S = P.smem_slots;
  const int TILE = P.tile_rows;
  const int STAGES = P.stages;
  const int rw = q.rec_bytes / 8;
  const int rb = q.rec_bytes;
  const int n_hot = (K128 || !P.hot_keys) ? 0 : (int)min(*P.hot_n, (unsigned)P.hot_cap);
  const int n_warm = (K128 || !P.warm_keys || !S) ? 0 : (int)min(*P.warm_n, (unsigned)(S / 2));

  // shared table and hot records start at identity, so claiming a slot needs no publication
  for (int i = tid; i < S; i += NT) skeys[i] = PMB_EMPTY64;
  for (int w = tid; w < S * rw; w += NT) reinterpret_cast<uint64_t*>(srecs)[w] = P.rec_init.w[w % rw];
  if (n_hot) {
    for (int i = tid; i < P.hot_lut_slots; i += NT) hlk[i] = PMB_EMPTY64;
    for (int w = tid; w < W * P.hot_cap * rw; w += NT)
      reinterpret_cast<uint64_t*>(hrecs)[w] = P.rec_init.w[w % rw];
  }
  if (tid < PMB_MAX_COLS) {
    s_doff[tid] = P.stage_data_off[tid];
    s_voff[tid] = P.stage_valid_off[tid];
  }
  if (tid == 0) {
    for (int s = 0; s < STAGES; s++) mbar_init(&bars[s], 1);
    mbar_fence_init();
    s_abort = 0;
  }
  __syncthreads();
  // hot-key lookup table (distinct keys: each insert claims its own slot)
  for (int i = tid; i < n_hot; i += NT) {
    unsigned long long k = P.hot_keys[i];
    int j = (int)((pmb_fmix64(k) >> 24) & (uint64_t)(P.hot_lut_slots - 1));
    for (int p = 0; p < P.hot_lut_slots; p++) {
      if (atomicCAS(&hlk[j], PMB_EMPTY64, k) == PMB_EMPTY64) {
        hli[j] = i;
        break;
      }
      j = (j + 1) & (P.hot_lut_slots - 1);
    }
  }
  // warm keys preloaded into the shared table
  for (int i = tid; i < n_warm; i += NT) {
    unsigned long long k = P.warm_keys[i];
    sfind64(skeys, S, S, k, pmb_fmix64(k));
  }
  __syncthreads();

  const int64_t G = gridDim.x;
  const int64_t n_full = P.n_full_tiles;
  const int64_t my_tiles = n_full > (int64_t)blockIdx.x ? (n_full - 1 - blockIdx.x) / G + 1 : 0;

  auto issue = [&](int64_t k) {
    int s = (int)(k % STAGES);
    int64_t tile = blockIdx.x + k * G;
    uint8_t* base = sm + P.stage_region_off + (size_t)s * P.stage_bytes;
    mbar_arrive_expect_tx(&bars[s], (uint32_t)P.stage_bytes_used);
    for (int j = 0; j < P.n_staged; j++) {
      int c = P.staged_col[j];
      const DCol& C = q.col[c];
      uint32_t db = C.elem ? (uint32_t)(TILE * C.elem) : (uint32_t)(TILE / 8);
      const uint8_t* src = C.data + (C.elem ? tile * TILE * C.elem : tile * TILE / 8);
      bulk_g2s(base + P.stage_data_off[c], src, db, &bars[s]);
      if (C.valid) bulk_g2s(base + P.stage_valid_off[c], C.valid + tile * TILE / 8, (uint32_t)(TILE / 8), &bars[s]);
    }
  };

  if (tid == 0) {
    for (int64_t k = 0; k < STAGES && k < my_tiles; k++) issue(k);
  }

  const bool ks = P.kstats != nullptr;
  long long c_wait = 0, c_proc = 0, c0 = 0;
  unsigned int n_smem = 0, n_glob = 0;
  PathCycles pc;
  int64_t k = 0;
  for (; k < my_tiles; k++) {
    int s = (int)(k % STAGES);
    uint32_t parity = (uint32_t)((k / STAGES) & 1);
    if (ks && tid == 0) c0 = clock64();
    bool ok = mbar_wait_bounded(&bars[s], parity);
    if (ks && tid == 0) {
      long long c1 = clock64();
      c_wait += c1 - c0;
      c0 = c1;
    }
    if (!ok) s_abort = 1;
    __syncwarp();
    // every lane of a warp takes the same path (the warp-level grouping needs all 32)
    bool wok = __all_sync(0xffffffffu, ok);
    if (wok) {
      TileCtx t{sm + P.stage_region_off + (size_t)s * P.stage_bytes, s_doff, s_voff, 0};
      for (int base = 0; base < TILE; base += NT) {
        int path = process_rows<NT, K128>(P, q, t, base + tid, base + tid < TILE, skeys, srecs, hlk, hli, hrecs, n_hot, pc);
        n_smem += path == 1;
        n_glob += path == 2;
      }
    }
    __syncthreads();
    if (ks && tid == 0) c_proc += clock64() - c0;
    if (s_abort) break;
    if (tid == 0 && k + STAGES < my_tiles) {
      fence_proxy_async();
      issue(k + STAGES);
    }
  }
  if (ks) {
    long long v[6] = {pc.pred, pc.hot, pc.smem, pc.sfind, pc.gfind, pc.apply};
    for (int i = 0; i < 6; i++) {
      long long x = v[i];
      for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if ((tid & 31) == 0) atomicAdd(&P.kstats[6 + i], (unsigned long long)x);
    }
    atomicAdd(&P.kstats[4], (unsigned long long)n_smem);
    atomicAdd(&P.kstats[5], (unsigned long long)n_glob);
    if (tid == 0) {
      atomicAdd(&P.kstats[0], (unsigned long long)c_wait);
      atomicAdd(&P.kstats[1], (unsigned long long)c_proc);
      atomicAdd(&P.kstats[3], (unsigned long long)my_tiles);
      c0 = clock64();
    }
  }
  if (s_abort) {
    // report, then wait (bounded) for this CTA's copies still in flight before exiting
    if (tid == 0) {
      atomicOr(P.status, PMB_ST_TIMEOUT);
      for (int64_t j = k; j < my_tiles && j < k + STAGES; j++)
        mbar_wait_bounded(&bars[j % STAGES], (uint32_t)((j / STAGES) & 1));
    }
    __syncthreads();
    return;
  }

  // ragged tail tile straight from global memory
  if (P.tail_rows > 0 && (int64_t)blockIdx.x == n_full % G) {
    TileCtx t{nullptr, s_doff, s_voff, n_full * TILE};
    for (int base = 0; base < P.tail_rows; base += NT)
      process_rows<NT, K128>(P, q, t, base + tid, base + tid < P.tail_rows, skeys, srecs, hlk, hli, hrecs, n_hot, pc);
  }
  __syncthreads();

  if (!K128) {
    // hot keys: fold the warps' private records, then one merge per touched key
    const int len_off = q.field[0].off;  // field 0 is always the row count
    for (int i = tid; i < n_hot; i += NT) {
      uint8_t* r0 = hrecs + (size_t)i * rb;
      for (int w = 1; w < W; w++) merge_private(q, r0, hrecs + ((size_t)w * P.hot_cap + i) * rb);
      if (*reinterpret_cast<const unsigned int*>(r0 + len_off) == 0) continue;
      unsigned long long key = P.hot_keys[i];
      int64_t gi = gfind64(P, key, pmb_fmix64(key));
      if (gi >= 0) merge_record(q, P.grecs + (size_t)gi * rb, r0);
    }
    // the shared table (preloaded warm keys may have seen no rows)
    for (int i = tid; i < S; i += NT) {
      unsigned long long key = skeys[i];
      if (key == PMB_EMPTY64) continue;
      const uint8_t* r = srecs + (size_t)i * rb;
      if (*reinterpret_cast<const unsigned int*>(r + len_off) == 0) continue;
      int64_t gi = gfind64(P, key, pmb_fmix64(key));
      if (gi >= 0) merge_record(q, P.grecs + (size_t)gi * rb, r);
    }
  }
  if (ks) {
    __syncthreads();
    if (tid == 0) atomicAdd(&P.kstats[2], (unsigned long long)(clock64() - c0));
  }
}

// ============================================================================ finalize
template <int NT, int PER, bool K128>
__global__ void __launch_bounds__(NT) k_finalize(const __grid_constant__ FinParams F) {
  __shared__ int s_cnt[PER][NT / 32];
  __shared__ int s_off[PER][NT / 32];
  __shared__ long long s_tile;
  __shared__ unsigned long long s_base;
  const DQuery& q = F.q;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_tile = (long long)atomicAdd(F.ticket, 1ULL);
  __syncthreads();
  const long long tile = s_tile;
  const int64_t nslots = (int64_t)F.gcap + 1;  // + sentinel slot
  bool occ[PER];
  int64_t slot[PER];
  const bool sentinel_used = F.status[1] != 0;
  for (int j = 0; j < PER; j++) {
    slot[j] = tile * (NT * PER) + (int64_t)j * NT + tid;
    bool o = false;
    if (slot[j] < (int64_t)F.gcap) {
      if (K128) {
        const unsigned long long* kk = F.gkeys + 2 * slot[j];
        o = !(kk[0] == PMB_EMPTY64 && kk[1] == PMB_EMPTY64);
      } else {
        o = F.gkeys[slot[j]] != PMB_EMPTY64;
      }
    } else if (slot[j] == (int64_t)F.gcap) {
      o = sentinel_used;
    }
    occ[j] = o && slot[j] < nslots;
    unsigned b = __ballot_sync(0xffffffffu, occ[j]);
    if (lane == 0) s_cnt[j][warp] = __popc(b);
  }
  __syncthreads();
  if (warp == 0) {
    int acc = 0;
    if (lane == 0) {
      for (int j = 0; j < PER; j++)
        for (int w = 0; w < NT / 32; w++) {
          s_off[j][w] = acc;
          acc += s_cnt[j][w];
        }
    }
    acc = __shfl_sync(0xffffffffu, acc, 0);
    const unsigned long long base = pmb_lookback_warp(F.lb_status, tile, (unsigned long long)acc, F.status);
    if (lane == 0) {
      s_base = base;
      if (tile == (long long)gridDim.x - 1) *F.n_groups = base + acc;
    }
  }
  __syncthreads();
  const unsigned long long base = s_base;
  for (int j = 0; j < PER; j++) {
    unsigned b = __ballot_sync(0xffffffffu, occ[j]);
    if (b == 0) continue;
    int rank = __popc(b & ((1u << lane) - 1u));
    int64_t p = (int64_t)(base + s_off[j][warp] + rank);
    int64_t p_first = (int64_t)(base + s_off[j][warp]);
    uint64_t klo = PMB_EMPTY64, khi = PMB_EMPTY64;
    const uint8_t* rec = nullptr;
    if (occ[j]) {
      if (slot[j] < (int64_t)F.gcap) {
        if (K128) {
          klo = F.gkeys[2 * slot[j]];
          khi = F.gkeys[2 * slot[j] + 1];
        } else {
          klo = F.gkeys[slot[j]];
          khi = 0;
        }
      } else if (!K128) {
        khi = 0;
      }
      rec = F.grecs + (size_t)slot[j] * q.rec_bytes;
    }
    int oc = 0;
    // keys
    for (int k = 0; k < q.n_keys; k++, oc++) {
      const DKey& K = q.key[k];
      uint64_t v = 0;
      bool valid = false;
      if (occ[j]) valid = unpack_field(K, klo, khi, v);
      int dt = q.col[K.col].dtype;
      uint8_t* d = F.out_data[oc];
      if (occ[j]) {
        switch (pmb_dtype_bytes(dt)) {
          case 0: break;
          case 1: d[p] = (uint8_t)v; break;
          case 2: reinterpret_cast<uint16_t*>(d)[p] = (uint16_t)v; break;
          case 4: reinterpret_cast<uint32_t*>(d)[p] = (uint32_t)v; break;
          default: reinterpret_cast<uint64_t*>(d)[p] = v; break;
        }
      }
      if (dt == PMB_BOOL) warp_set_bits(reinterpret_cast<unsigned int*>(d), p, p_first, occ[j] && valid && v);
      warp_set_bits(reinterpret_cast<unsigned int*>(F.out_valid[oc]), p, p_first, occ[j] && valid);
    }
    // aggregates
    for (int a = 0; a < q.n_aggs; a++, oc++) {
      const DAggOut& A = q.agg[a];
      bool valid = true;
      uint64_t bits = 0;
      if (occ[j]) finalize_agg(q, A, rec, valid, bits);
      uint8_t* d = F.out_data[oc];
      if (occ[j]) {
        switch (pmb_dtype_bytes(A.out_dtype)) {
          case 0: break;
          case 1: d[p] = (uint8_t)bits; break;
          case 2: reinterpret_cast<uint16_t*>(d)[p] = (uint16_t)bits; break;
          case 4: reinterpret_cast<uint32_t*>(d)[p] = (uint32_t)bits; break;
          default: reinterpret_cast<uint64_t*>(d)[p] = bits; break;
        }
      }
      warp_set_bits(reinterpret_cast<unsigned int*>(F.out_valid[oc]), p, p_first, occ[j] && valid);
    }
  }
}

// ============================================================================ host side
static int smem_table_bytes(int S, int rec) { return S * (8 + rec); }

struct Plan {
  int tile = 1024;
  int stages = 3;
  int nt = 512;
  int smem_slots = 0;
  int smem_probe = 8;
  uint64_t gcap = 1024;
  int strategy = PMB_STRATEGY_GLOBAL_HASH;
};

static uint64_t next_pow2(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

// stage layout in shared memory for the columns the query touches
static int layout_stage(const CompiledQuery& cq, int tile, HashParams& P) {
  const DQuery& q = cq.dq;
  int off = 0;
  int used = 0;
  P.n_staged = 0;
  for (int c = 0; c < PMB_MAX_COLS; c++) {
    P.stage_data_off[c] = 0;
    P.stage_valid_off[c] = 0;
  }
  for (int c = 0; c < q.n_cols; c++) {
    int db = q.col[c].elem ? tile * q.col[c].elem : tile / 8;
    P.stage_data_off[c] = off;
    off += (int)pmb_align((size_t)db, 16);
    used += db;
    if (q.col[c].valid) {
      P.stage_valid_off[c] = off;
      off += (int)pmb_align((size_t)(tile / 8), 16);
      used += tile / 8;
    }
    P.staged_col[P.n_staged++] = c;
  }
  P.stage_bytes = (int)pmb_align((size_t)off, 128);
  P.stage_bytes_used = used;
  return P.stage_bytes;
}

template <int NT, bool K128>
static int launch_hash(pmb_handle* h, const HashParams& P, int smem, int grid) {
  auto kern = k_hash_agg<NT, K128>;
  PMB_CUDA(h, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  pmb_kernel_begin(h, "hash_agg");
  kern<<<grid, NT, smem, h->stream>>>(P);
  pmb_kernel_end(h);
  PMB_CUDA(h, cudaGetLastError());
  return PMB_OK;
}

template <bool K128>
static int launch_finalize(pmb_handle* h, const FinParams& F, int64_t nslots) {
  constexpr int NT = 256, PER = 4;
  int64_t tiles = (nslots + NT * PER - 1) / (NT * PER);
  pmb_kernel_begin(h, "finalize");
  k_finalize<NT, PER, K128><<<(unsigned)tiles, NT, 0, h->stream>>>(F);
  pmb_kernel_end(h);
  PMB_CUDA(h, cudaGetLastError());
  return PMB_OK;
}

int pmb_groupby_sketch(pmb_handle* h, const CompiledQuery& cq, SketchOut* out) {
  const DQuery& q = cq.dq;
  int64_t m = std::min<int64_t>(q.n_rows, SK_SAMPLES);
  out->samples = m;
  out->distinct = out->singletons = out->doubletons = 0;
  memset(out->hist, 0, sizeof(out->hist));
  memset(out->fx_expo, 0, sizeof(out->fx_expo));
  out->set_keys = nullptr;
  out->set_cnt = nullptr;
  if (m == 0) return PMB_OK;
  unsigned long long* keys = (unsigned long long*)pmb_ws_alloc(h, sizeof(unsigned long long) * SK_SLOTS);
  unsigned int* cnt = (unsigned int*)pmb_ws_alloc(h, sizeof(unsigned int) * SK_SLOTS);
  unsigned long long* res = (unsigned long long*)pmb_ws_alloc(h, 64 + 4 * SK_HIST);
  if (!keys || !cnt || !res) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (sketch)");
  unsigned int* hist = (unsigned int*)(res + 8);
  unsigned int* fx_expo = (unsigned int*)(res + 4);  // res[4..7]: 8 x u32
  FxCols fxc;
  memset(&fxc, 0, sizeof(fxc));
  fxc.n = (int)cq.fx_cols.size();
  for (int f = 0; f < fxc.n; f++) fxc.col[f] = cq.fx_cols[f];
  PMB_CUDA(h, cudaMemsetAsync(keys, 0xFF, sizeof(unsigned long long) * SK_SLOTS, h->stream));
  PMB_CUDA(h, cudaMemsetAsync(cnt, 0, sizeof(unsigned int) * SK_SLOTS, h->stream));
  PMB_CUDA(h, cudaMemsetAsync(res, 0, 64 + 4 * SK_HIST, h->stream));
  pmb_kernel_begin(h, "sketch");
  if (q.key_bits > 64)
    k_sketch<true><<<(unsigned)((m + 255) / 256), 256, 0, h->stream>>>(q, m, keys, cnt, fxc, fx_expo);
  else
    k_sketch<false><<<(unsigned)((m + 255) / 256), 256, 0, h->stream>>>(q, m, keys, cnt, fxc, fx_expo);
  pmb_kernel_end(h);
  PMB_CUDA(h, cudaGetLastError());
  pmb_kernel_begin(h, "sketch_reduce");
  k_sketch_reduce<<<64, 256, 0, h->stream>>>(keys, cnt, res, hist);
  pmb_kernel_end(h);
  PMB_CUDA(h, cudaGetLastError());
  PMB_CUDA(h, cudaMemcpyAsync(h->pinned, res, 64 + 4 * SK_HIST, cudaMemcpyDeviceToHost, h->stream));
  PMB_CUDA(h, cudaStreamSynchronize(h->stream));
  const unsigned long long* r = (const unsigned long long*)h->pinned;
  out->distinct = (int64_t)r[0];
  out->singletons = (int64_t)r[1];
  out->doubletons = (int64_t)r[2];
  memcpy(out->fx_expo, h->pinned + 32, 4 * PMB_MAX_FX);
  memcpy(out->hist, h->pinned + 64, 4 * SK_HIST);
  out->set_keys = keys;
  out->set_cnt = cnt;
  return PMB_OK;
}

// Distinct-group estimate from the sample: exact when the sample is the whole input, else the
// GEE estimator (Charikar, Chaudhuri, Motwani, Narasayya 2000): sqrt(n/m) * f1 + (d - f1).
int64_t pmb_estimate_groups(const SketchOut& s, int64_t n_rows) {
  if (s.samples <= 0) return 0;
  if (s.samples >= n_rows) return s.distinct;
  double scale = std::sqrt((double)n_rows / (double)s.samples);
  double est = scale * (double)s.singletons + (double)(s.distinct - s.singletons);
  if ((double)s.singletons > 0.9 * (double)s.samples) est = (double)n_rows;  // near-unique keys
  est = std::max(est, (double)s.distinct);
  est = std::min(est, (double)n_rows);
  return (int64_t)est;
}

static void build_output_columns(const CompiledQuery& cq, pmb_result* r, const pmb_column* cols) {
  const DQuery& q = cq.dq;
  int oc = 0;
  for (int k = 0; k < q.n_keys; k++, oc++) r->columns[oc].dtype = q.col[q.key[k].col].dtype;
  for (int a = 0; a < q.n_aggs; a++, oc++) r->columns[oc].dtype = q.agg[a].out_dtype;
  (void)cols;
}

// Shared-memory layout and launch shape of the hash kernel for one query (host-only, no device
// calls): stage ring, hot-key tier, CTA-shared table. Used by the launch and by the JIT check.
int pmb_plan_hash(pmb_handle* h, int max_smem_optin, CompiledQuery& cq, int strategy, int64_t est, bool have_sketch,
                  HashParams& P, int& nt, int& smem) {
  DQuery& q = cq.dq;
  const bool K128 = q.key_bits > 64;
  const int rec = q.rec_bytes;
  int tile = 1024;
  if (const char* e = getenv("PMB_TILE")) {
    int v = atoi(e);
    if (v >= 256 && v <= 8192 && v % 128 == 0) tile = v;
  }
  memset(&P, 0, sizeof(P));
  P.q = q;
  P.tile_rows = tile;
  layout_stage(cq, tile, P);
  const int budget = max_smem_optin - 4096;  // static shared memory (descriptor copy) comes on top
  int stages = 2;
  if (const char* e = getenv("PMB_STAGES")) stages = std::max(1, std::min(atoi(e), 4));
  while (stages > 1 && 128 + stages * P.stage_bytes > budget / 2) stages--;
  int smem_fixed = 128 + stages * P.stage_bytes;
  if (smem_fixed > budget / 2) {
    // very wide queries: smaller tiles
    tile = 512;
    P.tile_rows = tile;
    layout_stage(cq, tile, P);
    stages = 1;
    smem_fixed = 128 + stages * P.stage_bytes;
    if (smem_fixed > budget) return pmb_fail(h, PMB_E_UNSUPPORTED, "query touches too many columns for one tile");
  }
  // hot tier: per-warp private records for the heaviest sample keys (at most 64 KB)
  nt = 1024;
  if (const char* e = getenv("PMB_NT")) nt = atoi(e);
  if (nt != 256 && nt != 512 && nt != 1024) nt = 1024;
  if (K128) nt = 512;
  int hot_cap = (K128 || !have_sketch) ? 0 : 32;
  if (const char* e = getenv("PMB_HOT")) hot_cap = std::max(0, std::min(atoi(e), 128));
  while (hot_cap > 0 && ((nt / 32) * hot_cap * rec > (64 << 10) || smem_fixed + (nt / 32) * hot_cap * rec > budget))
    hot_cap /= 2;
  int hot_lut = hot_cap ? (int)next_pow2((uint64_t)(2 * hot_cap)) : 0;
  P.hot_cap = hot_cap;
  P.hot_lut_slots = hot_lut;
  P.hot_lut_off = (int)pmb_align((size_t)smem_fixed, 16);
  P.hot_recs_off = (int)pmb_align((size_t)(P.hot_lut_off + hot_lut * 12), 16);
  smem_fixed = P.hot_recs_off + (nt / 32) * hot_cap * rec;
  int S = 0;
  if (!K128) {
    int room = budget - smem_fixed;
    S = 1;
    while (smem_table_bytes(S * 2, rec) <= room && S * 2 <= 4096) S *= 2;
    if (S < 64) S = 0;
    if (strategy == PMB_STRATEGY_SMEM_HASH && est > 0) {
      int want = (int)next_pow2((uint64_t)std::max<int64_t>(2 * est, 64));
      if (want < S) S = want;
    }
    // tuning override: PMB_SMEM_SLOTS=<pow2> (0 disables the shared-memory table)
    if (const char* e = getenv("PMB_SMEM_SLOTS")) {
      int v = atoi(e);
      if (v == 0) S = 0;
      else if (v > 0 && v < S) S = (int)next_pow2((uint64_t)v);
    }
  }
  P.stages = stages;
  P.smem_slots = S;
  P.smem_probe = S ? std::min(S, (strategy == PMB_STRATEGY_SMEM_HASH) ? 64 : 16) : 0;
  P.stage_region_off = 128;
  P.smem_keys_off = (int)pmb_align((size_t)smem_fixed, 16);
  P.smem_recs_off = P.smem_keys_off + S * 8;
  smem = P.smem_recs_off + S * rec;
  const int64_t n = q.n_rows;
  P.n_full_tiles = n / tile;
  P.tail_rows = (int32_t)(n % tile);
  if (cq.rec_words > (int)(sizeof(P.rec_init.w) / 8)) return pmb_fail(h, PMB_E_UNSUPPORTED, "record too large");
  for (int w = 0; w < cq.rec_words; w++) P.rec_init.w[w] = cq.rec_init[w];
  return PMB_OK;
}

int pmb_groupby_hash(pmb_handle* h, CompiledQuery& cq, const pmb_query* uq, int strategy, int64_t est,
                     const SketchOut* sk, pmb_result* r, bool est_learned) {
  DQuery& q = cq.dq;
  const bool K128 = q.key_bits > 64;
  HashParams P;
  int nt = 1024, smem = 0;
  int prc = pmb_plan_hash(h, h->max_smem_optin, cq, strategy, est, sk && sk->set_keys, P, nt, smem);
  if (prc) return prc;
  // run-time compiled kernel (warp-independent units) when enabled; its own tier sizes
  JitPlan J;
  cudaKernel_t jk = nullptr;
  if (!K128 && pmb_jit_enabled(q.n_rows) && pmb_plan_jit(h, cq, sk && sk->set_keys, h->max_smem_optin, &J) == PMB_OK) {
    std::string keep_err = h->err;
    if (pmb_jit_hash_kernel(h, cq, J, &jk) != PMB_OK) jk = nullptr;  // prebuilt generic kernel: same results
    h->err = keep_err;
  }
  pmb_phase(h, "jit");
  const int hot_cap = jk ? J.hot_cap : P.hot_cap;
  const int S = jk ? 2 * J.warm_cap : P.smem_slots;
  const int rec = q.rec_bytes;
  Plan pl;
  pl.strategy = (K128 && strategy == PMB_STRATEGY_SMEM_HASH) ? PMB_STRATEGY_GLOBAL_HASH : strategy;
  pl.tile = P.tile_rows;
  // hot / warm key lists from the sample histogram
  if (hot_cap || S) {
    if (sk && sk->set_keys) {
      unsigned int suffix[SK_HIST + 1];
      suffix[SK_HIST] = 0;
      for (int c = SK_HIST - 1; c >= 0; c--) suffix[c] = suffix[c + 1] + sk->hist[c];
      unsigned int t1 = SK_HIST;
      for (int c = 4; c < SK_HIST; c++)
        if (suffix[c] <= (unsigned)hot_cap) {
          t1 = c;
          break;
        }
      if (!hot_cap) t1 = SK_HIST;
      unsigned int warm_cap = (unsigned)(S / 2);
      unsigned int t2 = t1;
      for (int c = 2; c < (int)t1; c++)
        if (suffix[c] - suffix[t1] <= warm_cap) {
          t2 = c;
          break;
        }
      unsigned long long* lists = (unsigned long long*)pmb_ws_alloc(h, 8 * ((size_t)hot_cap + warm_cap) + 64);
      if (!lists) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (hot keys)");
      unsigned int* counts = (unsigned int*)(lists + hot_cap + warm_cap);
      PMB_CUDA(h, cudaMemsetAsync(counts, 0, 16, h->stream));
      pmb_kernel_begin(h, "sketch_select");
      k_sketch_select<<<64, 256, 0, h->stream>>>(sk->set_keys, sk->set_cnt, t1, t2, lists, counts, (unsigned)hot_cap,
                                                 lists + hot_cap, counts + 1, warm_cap);
      pmb_kernel_end(h);
      PMB_CUDA(h, cudaGetLastError());
      P.hot_keys = hot_cap ? lists : nullptr;
      P.hot_n = counts;
      P.warm_keys = warm_cap ? lists + hot_cap : nullptr;
      P.warm_n = counts + 1;
    }
  }
  if (!P.hot_keys) {
    P.hot_cap = 0;
    P.hot_lut_slots = 0;
  }
  // run-time kernel: its sampled-key table is built on the device from the selected key lists,
  // so the launches of this call follow each other without a host round trip
  uint8_t* ttab = nullptr;
  int tnb = 0;
  if (jk && P.hot_n && (P.hot_keys || P.warm_keys) && J.tnb > 0) {
    tnb = J.tnb;
    const size_t tbytes = (size_t)tnb * 4 * (J.tkey + 2);
    ttab = (uint8_t*)pmb_ws_alloc(h, tbytes + 16);
    unsigned int* fill = (unsigned int*)pmb_ws_alloc(h, 4 * (size_t)tnb + 16);
    if (!ttab || !fill) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (sampled-key table)");
    pmb_kernel_begin(h, "sample_table");
    k_sample_table<<<1, 1024, 0, h->stream>>>(P.hot_keys, P.hot_n, (unsigned)hot_cap, P.warm_keys, P.warm_n,
                                              (unsigned)(S / 2), (unsigned)tnb, J.tkey == 4 ? 1 : 0, ttab, fill);
    pmb_kernel_end(h);
    PMB_CUDA(h, cudaGetLastError());
  }
  const int64_t n = q.n_rows;
  pmb_phase(h, "keys");

  // Capacity: 4 slots per estimated group (any size: slots come from a multiply-shift, not a
  // mask; sample estimates of skewed keys run low), 2 per group of a caller's hint or when the
  // estimate is the larger of the sample estimate and the selector's prediction (hash workload,
  // 100M rows, 945K groups: table init, aggregation and finalize 1.68 ms with 4, 1.59 ms with 2).
  // A table that fills up is rebuilt 3x larger; the estimate only sets how often that happens,
  // never the result.
  uint64_t cap = (uint64_t)std::max<int64_t>((est_learned ? 2 : 4) * est, 1024);
  if (uq->capacity_hint > 0) cap = (uint64_t)std::max<int64_t>(2 * uq->capacity_hint, 1024);
  const uint64_t cap_max = (uint64_t)std::max<int64_t>(2 * n, 1024);
  // tuning override: PMB_GCAP_MULT=<k> multiplies the global table capacity
  if (const char* e = getenv("PMB_GCAP_MULT")) {
    double k = atof(e);
    if (k > 0) cap = (uint64_t)std::max(1024.0, (double)cap * k);
  }
  cap = (std::min(cap, cap_max) + 3) & ~3ULL;  // whole 4-slot buckets

  const int n_out = q.n_keys + q.n_aggs;
  int fx_reruns = 0;
  for (int attempt = 0;; attempt++) {
    const int key_words = K128 ? 2 : 1;
    size_t keys_bytes = (size_t)(cap + 1) * 8 * key_words;
    size_t recs_bytes = (size_t)(cap + 1) * rec;
    unsigned long long* gkeys = (unsigned long long*)pmb_ws_alloc(h, keys_bytes);
    uint8_t* grecs = (uint8_t*)pmb_ws_alloc(h, recs_bytes);
    unsigned int* status = (unsigned int*)pmb_ws_alloc(h, 64);
    int64_t nslots = (int64_t)cap + 1;
    int64_t fin_tiles = (nslots + 1024 - 1) / 1024;
    unsigned long long* lb = (unsigned long long*)pmb_ws_alloc(h, (size_t)fin_tiles * 8 + 64);
    if (!gkeys || !grecs || !status || !lb) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (hash table)");
    FinParams F;
    memset(&F, 0, sizeof(F));
    F.q = q;
    ZeroList zl;  // cleared by the table init's launch
    zl.n = 0;
    for (int c = 0; c < n_out; c++) {
      int dt = r->columns[c].dtype;
      size_t db = dt == PMB_BOOL ? (size_t)((nslots + 31) / 32 * 4) : (size_t)nslots * pmb_dtype_bytes(dt);
      F.out_data[c] = (uint8_t*)pmb_ws_alloc(h, db + 16);
      F.out_valid[c] = (uint8_t*)pmb_ws_alloc(h, (size_t)((nslots + 31) / 32 * 4) + 16);
      if (!F.out_data[c] || !F.out_valid[c]) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (outputs)");
      if (!zl_add(zl, F.out_valid[c], (size_t)((nslots + 31) / 32 * 4)))
        PMB_CUDA(h, cudaMemsetAsync(F.out_valid[c], 0, (size_t)((nslots + 31) / 32 * 4), h->stream));
      if (dt == PMB_BOOL && !zl_add(zl, F.out_data[c], db)) PMB_CUDA(h, cudaMemsetAsync(F.out_data[c], 0, db, h->stream));
    }
    if (!zl_add(zl, status, 64)) PMB_CUDA(h, cudaMemsetAsync(status, 0, 64, h->stream));
    if (!zl_add(zl, lb, (size_t)fin_tiles * 8 + 64)) PMB_CUDA(h, cudaMemsetAsync(lb, 0, (size_t)fin_tiles * 8 + 64, h->stream));
    // table init
    {
      int64_t work = std::max<int64_t>((int64_t)(cap + 1) * key_words, (int64_t)(cap + 1) * cq.rec_words);
      int blocks = (int)std::min<int64_t>((work + 255) / 256, (int64_t)h->sm_count * 16);
      pmb_kernel_begin(h, "table_init");
      k_table_init<<<blocks, 256, 0, h->stream>>>(gkeys, (int64_t)(cap + 1) * key_words, (uint64_t*)grecs,
                                                  (int64_t)(cap + 1), cq.rec_words, P.rec_init, zl);
      pmb_kernel_end(h);
      PMB_CUDA(h, cudaGetLastError());
    }
    P.gkeys = gkeys;
    P.grecs = grecs;
    P.gcap = cap;
    P.gprobe = (int)std::min<uint64_t>(cap, 1024);
    P.status = status;
    int grid = (int)std::max<int64_t>(1, std::min<int64_t>(P.n_full_tiles, (int64_t)h->sm_count));
    unsigned long long* kst = nullptr;
    if (getenv("PMB_KSTATS")) {
      kst = (unsigned long long*)pmb_ws_alloc(h, 128);
      if (!kst) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (kstats)");
      PMB_CUDA(h, cudaMemsetAsync(kst, 0, 128, h->stream));
    }
    P.kstats = kst;
    int rc;
    if (jk) rc = pmb_jit_launch(h, jk, cq, J, P, h->sm_count, ttab, tnb);
    else if (K128) rc = launch_hash<512, true>(h, P, smem, grid);
    else if (nt == 1024) rc = launch_hash<1024, false>(h, P, smem, grid);
    else if (nt == 256) rc = launch_hash<256, false>(h, P, smem, grid);
    else rc = launch_hash<512, false>(h, P, smem, grid);
    if (rc) return rc;
    if (kst && jk) {
      unsigned long long hk[16];
      PMB_CUDA(h, cudaMemcpyAsync(hk, kst, 128, cudaMemcpyDeviceToHost, h->stream));
      PMB_CUDA(h, cudaStreamSynchronize(h->stream));
      double warps = (double)(hk[7] ? hk[7] : 1);
      fprintf(stderr, "jit kstats: nt=%d nbuf=%d hot=%d warm=%d tnb=%d srec=%d smem=%d cap=%llu | per warp (Mcycles): wait %.2f "
              "classify %.2f shared %.2f cold %.2f | rows shared %llu cold %llu\n", J.nt, J.nbuf, J.hot_cap, J.warm_cap, tnb,
              J.srec, J.smem, (unsigned long long)cap, hk[0] / warps / 1e6, hk[1] / warps / 1e6, hk[2] / warps / 1e6,
              hk[3] / warps / 1e6, hk[4], hk[5]);
    } else if (kst) {
      unsigned long long hk[16];
      PMB_CUDA(h, cudaMemcpyAsync(hk, kst, 128, cudaMemcpyDeviceToHost, h->stream));
      PMB_CUDA(h, cudaStreamSynchronize(h->stream));
      fprintf(stderr, "kstats: grid=%d nt=%d hot=%d S=%d tile=%d stages=%d tiles=%llu wait_cyc/tile=%.0f proc_cyc/tile=%.0f "
              "flush_cyc/cta=%.0f smem_rows=%llu global_rows=%llu\n", grid, nt, P.hot_cap, P.smem_slots, P.tile_rows, P.stages,
              hk[3], (double)hk[0] / (double)(hk[3] ? hk[3] : 1), (double)hk[1] / (double)(hk[3] ? hk[3] : 1),
              (double)hk[2] / grid, hk[4], hk[5]);
      double rows = (double)q.n_rows;
      fprintf(stderr, "  per-row cycles (thread-summed): pred+key %.0f, hot-warp %.0f | per smem row %.0f | per global row: "
              "sfind %.0f gfind %.0f apply %.0f\n", hk[6] / rows, hk[7] / rows, hk[8] / (double)(hk[4] ? hk[4] : 1),
              hk[9] / (double)(hk[5] ? hk[5] : 1), hk[10] / (double)(hk[5] ? hk[5] : 1),
              hk[11] / (double)(hk[5] ? hk[5] : 1));
    }
    F.gkeys = gkeys;
    F.grecs = grecs;
    F.gcap = cap;
    F.status = status;
    F.lb_status = lb;
    F.ticket = lb + fin_tiles;
    F.n_groups = lb + fin_tiles + 1;
    rc = K128 ? launch_finalize<true>(h, F, nslots) : launch_finalize<false>(h, F, nslots);
    if (rc) return rc;
    pmb_phase(h, "launch");
    PMB_CUDA(h, cudaMemcpyAsync(h->pinned, status, 8, cudaMemcpyDeviceToHost, h->stream));
    PMB_CUDA(h, cudaMemcpyAsync(h->pinned + 8, F.n_groups, 8, cudaMemcpyDeviceToHost, h->stream));
    PMB_CUDA(h, cudaStreamSynchronize(h->stream));
    pmb_phase(h, "device");
    unsigned int st = *(unsigned int*)h->pinned;
    if (st & PMB_ST_TIMEOUT) return pmb_fail(h, PMB_E_TIMEOUT, "a bounded device wait timed out");
    if (st & PMB_ST_FXRANGE) {
      // a float sum left its fixed-point range: widen to the largest exponent seen, run again
      unsigned expo[PMB_MAX_FX];
      PMB_CUDA(h, cudaMemcpy(expo, status + 4, sizeof(expo), cudaMemcpyDeviceToHost));
      for (int i = 0; i < q.n_fields; i++) {
        DField& f = q.field[i];
        if (f.kind != F_SUM_FX || expo[f.fx_slot] == 0) continue;
        int e = (int)expo[f.fx_slot] - 1022 + 1;  // the value seen fits with one spare power of two
        if (e > q.fx_e[f.fx_slot]) {
          f.fx = (int16_t)(f.fx - (e - q.fx_e[f.fx_slot]));
          q.fx_e[f.fx_slot] = (int16_t)e;
        }
        P.q.field[i].fx = f.fx;
        P.q.fx_e[f.fx_slot] = q.fx_e[f.fx_slot];
      }
      if (pmb_fx_to_dd(cq)) return PMB_RETRY_DD;
      if (++fx_reruns > 4) return pmb_fail(h, PMB_E_CUDA, "float-sum range did not converge");
      continue;
    }
    if (st & PMB_ST_OVERFLOW) {
      if (cap >= cap_max) return pmb_fail(h, PMB_E_OOM, "hash table overflow at maximum capacity");
      cap = (std::min(cap * 3, cap_max) + 3) & ~3ULL;
      r->rehash_count++;
      continue;
    }
    r->n_groups = (int64_t) * (unsigned long long*)(h->pinned + 8);
    r->capacity = (int64_t)cap;
    r->strategy_used = pl.strategy;
    for (int c = 0; c < n_out; c++) {
      r->columns[c].data = F.out_data[c];
      r->columns[c].validity = F.out_valid[c];
    }
    return PMB_OK;
  }
}

// compiles the query again (its float-sum columns listed in cq.dd_user_cols in double-double),
// keeping the staged column pointers: the same columns come in the same order
int recompile_dd(pmb_handle* h, const pmb_query* q, const pmb_column* cols, int32_t n_cols, CompiledQuery& cq) {
  CompiledQuery nc;
  nc.dd_user_cols = cq.dd_user_cols;
  int rc = pmb_compile_groupby(h, q, cols, n_cols, &nc);
  if (rc) return rc;
  for (int c = 0; c < nc.dq.n_cols; c++) {
    nc.dq.col[c].data = cq.dq.col[c].data;
    nc.dq.col[c].valid = cq.dq.col[c].valid;
  }
  cq = nc;
  return PMB_OK;
}

extern "C" int pmb_groupby(pmb_handle* h, const pmb_query* q, const pmb_column* cols, int32_t n_cols,
                           pmb_result** out) {
  if (!h) return PMB_E_INVALID;
  if (!out) return pmb_fail(h, PMB_E_INVALID, "out is NULL");
  *out = nullptr;
  if (q && (q->strategy < PMB_STRATEGY_AUTO || q->strategy > PMB_STRATEGY_PARTITIONED))
    return pmb_fail(h, PMB_E_INVALID, "unknown strategy");
  PMB_CUDA(h, cudaSetDevice(h->device));
  CompiledQuery cq;
  int rc = pmb_compile_groupby(h, q, cols, n_cols, &cq);
  if (rc) return rc;
  rc = pmb_ws_begin(h);
  if (rc) return rc;
  pmb_call_begin(h);
  pmb_phase(h, "compile");
  pmb_result* r = pmb_result_new(cq.dq.n_keys + cq.dq.n_aggs);
  if (!r) return pmb_fail(h, PMB_E_OOM, "host allocation failed");
  build_output_columns(cq, r, cols);
  auto bail = [&](int code) {
    pmb_result_free(r);
    return code;
  };
  // stage the touched columns
  for (int c = 0; c < cq.dq.n_cols; c++) {
    rc = pmb_stage_column(h, cols[cq.map.user[c]], cq.dq.n_rows, &cq.dq.col[c]);
    if (rc) return bail(rc);
  }
  pmb_phase(h, "stage");
  if (cq.dq.n_rows == 0) {
    r->n_groups = 0;
    r->strategy_used = q->strategy ? q->strategy : PMB_STRATEGY_GLOBAL_HASH;
    for (int c = 0; c < r->n_columns; c++) {
      r->columns[c].data = pmb_ws_alloc(h, 16);
      r->columns[c].validity = (uint8_t*)pmb_ws_alloc(h, 16);
    }
  } else for (int pass = 0;; pass++) {
    int strategy = q->strategy;
    int64_t est = q->capacity_hint;
    bool est_learned = false;
    static thread_local SketchOut sk;  // large (histogram); one per host thread
    bool have_sk = true;
    // the selector's kernels go in before the sketch's readback, whose synchronisation serves both
    const bool sel = strategy == PMB_STRATEGY_AUTO && pmb_selector_launch(h, cq);
    rc = pmb_groupby_sketch(h, cq, &sk);
    if (rc) return bail(rc);
    pmb_phase(h, "sketch");
    // fixed-point range of the float sums: sample maximum with 8x headroom; partial sums of a
    // CTA (at most n / SMs values, with margin) must fit as well
    int pbits = 2, tbits = 2;
    while ((1LL << pbits) < cq.dq.n_rows / h->sm_count + 1) pbits++;
    while ((1LL << tbits) < cq.dq.n_rows + 1) tbits++;
    pmb_set_fx(cq.dq, sk.fx_expo, 3, pbits + 1, tbits + 1);
    if (pass < 3 && pmb_fx_to_dd(cq)) {
      // a float-sum column's range leaves too few fraction bits: sum it in double-double
      rc = recompile_dd(h, q, cols, n_cols, cq);
      if (rc) return bail(rc);
      continue;
    }
    int64_t e = pmb_estimate_groups(sk, cq.dq.n_rows);
    if (strategy == PMB_STRATEGY_AUTO) {
      // the learned selector when installed, else the plain cardinality heuristic. The predicted
      // group count can only enlarge the table: an undersized table costs a rebuild, an oversized
      // one only its initialisation
      int s = 0;
      int64_t g = 0;
      if (sel && pmb_selector_read(h, cq, &s, &g) &&
          !(pmb_selector_vetoed(cq, sk, s))) {
        // the network scores all four strategies; pmb_selector_vetoed picks are overruled by the
        // heuristic below
        strategy = s;
        if (est <= 0) {
          est = std::max<int64_t>(e, std::min<int64_t>(g, cq.dq.n_rows));
          est_learned = true;
        }
      } else {
        if (est <= 0) est = e;
        strategy = pmb_choose_strategy(h, cq, sk, est);
        if (pmb_prefer_partitioned(cq, sk, strategy, est)) strategy = PMB_STRATEGY_PARTITIONED;
      }
    }
    if (est <= 0) est = e;
    pmb_phase(h, "choose");
    if (strategy == PMB_STRATEGY_SORT) rc = pmb_groupby_sort(h, cq, r, 0);
    else if (strategy == PMB_STRATEGY_PARTITIONED) rc = pmb_groupby_sort(h, cq, r, std::max<int64_t>(est, 1));
    else rc = pmb_groupby_hash(h, cq, q, strategy, est, have_sk ? &sk : nullptr, r, est_learned);
    if (rc == PMB_RETRY_DD && pass < 3) {
      // a float sum outgrew the fixed point: its column now sums in double-double
      rc = recompile_dd(h, q, cols, n_cols, cq);
      if (rc) return bail(rc);
      continue;
    }
    if (rc) return bail(rc == PMB_RETRY_DD ? pmb_fail(h, PMB_E_CUDA, "float-sum range did not converge") : rc);
    break;
  }
  pmb_phase(h, "strategy");
  rc = pmb_finish_outputs(h, r, q->output_on_device == 0);
  if (rc) return bail(rc);
  PMB_CUDA(h, cudaStreamSynchronize(h->stream));
  pmb_phase(h, "outputs");
  pmb_call_end(h);
  *out = r;
  return PMB_OK;
}

// Many groups and no heavy key: partition the rows by key hash and aggregate every partition in a
// shared-memory table instead of a global table (or a full sort) that lives in HBM. Measured on
// 100M uniform rows: 64-bit keys tie with the global table near 250K groups and win 2.3x from 1M
// groups on; 96-bit keys (the prebuilt 128-bit hash kernel) win 2x from 2M groups and tie at
// 200K. A heavy key would make its partition one CTA's serial work, so the most frequent sampled
// key must stand for at most 256K rows.
bool pmb_heavy_key(const CompiledQuery& cq, const SketchOut& sk) {
  if (sk.samples <= 0) return false;
  int top = 0;
  for (int c = SK_HIST - 1; c > 0; c--)
    if (sk.hist[c]) {
      top = c;
      break;
    }
  const double top_rows = (double)top * (double)cq.dq.n_rows / (double)sk.samples;
  return top >= SK_HIST - 1 || top_rows > 262144.0;
}

// A sort or partitioned pick of the network for a key of at most 64 packed bits with a heavy key
// in the sample: over the 13,000 timed tables of the selector's training data, such queries never
// ran faster than the run-time compiled hash kernel (vetoing them would have cost 22 ms of 1,520 ms
// there), while a heavy key can make its segment one CTA's serial work (the hash workload: 27.8 ms
// sorted against 2.0 ms hashed). Wider keys keep the network's pick: their hash path is the slower
// prebuilt 128-bit kernel, and there the sort and partitioned strategies often win.
bool pmb_selector_vetoed(const CompiledQuery& cq, const SketchOut& sk, int strategy) {
  return (strategy == PMB_STRATEGY_SORT || strategy == PMB_STRATEGY_PARTITIONED) && cq.dq.key_bits <= 64 &&
         pmb_heavy_key(cq, sk);
}

bool pmb_prefer_partitioned(const CompiledQuery& cq, const SketchOut& sk, int strategy, int64_t est) {
  if (strategy != PMB_STRATEGY_GLOBAL_HASH && strategy != PMB_STRATEGY_SORT) return false;
  if (est < (cq.dq.key_bits > 64 ? 200000 : 500000) || sk.samples <= 0) return false;
  return !pmb_heavy_key(cq, sk);
}

// Plain cardinality heuristic (the fallback of the learned selector): shared-memory tables
// when every group fits a CTA's table, else the global table with a hot-key cache.
int pmb_choose_strategy(pmb_handle* h, const CompiledQuery& cq, const SketchOut& sk, int64_t est) {
  (void)h;
  (void)sk;
  if (cq.dq.key_bits > 64) return PMB_STRATEGY_GLOBAL_HASH;
  return est <= 1024 ? PMB_STRATEGY_SMEM_HASH : PMB_STRATEGY_GLOBAL_HASH;
}
