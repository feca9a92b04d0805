// pmb_jit_skeleton.cuh — the fused filter -> group_by -> aggregate kernel compiled at run time
// for one query signature (NVRTC). This text follows pmb_device.cuh and a generated section that
// defines, for that signature, the J_* constants and the row functions:
//   j_issue_unit   one warp's bulk copies (TMA, cp.async.bulk) of a 128-row unit into its buffer
//   j_copy_unit    plain copy of a partial last unit
//   JRow, j_load   the values of one row of the buffer and the filter verdict (with the range
//                  report of exact float sums when `check`)
//   j_load_vals    the aggregated values only
//   j_key          the packed 64-bit group key
//   j_private / j_shared / j_global      one row into a warp-private / CTA-shared / global record
//                  (float sums: double-double in the private and shared tiers, fixed-point limbs in
//                  the global table)
//   j_merge_private / j_merge_global     a finished private / shared record into another / the table
//   J_IDENT        the identity record (u64 words)
//
// Execution: persistent CTAs, every warp independent (no CTA barrier in the main loop). A warp
// takes 128-row units round-robin over all warps of the grid; lane 0 bulk-copies the unit's
// column chunks into the warp's shared buffer (one mbarrier per warp, bounded wait), then each
// lane handles rows lane, lane + 32, lane + 64, lane + 96 of the unit:
//   1. filter, key, hot lookup for the 4 rows; hot rows: lanes with the same hot key are grouped
//      (__match_any_sync) and the group's first lane applies the group to the warp's private
//      record (no atomics);
//   2. warm rows (keys preloaded into the CTA-shared table): shared-memory atomics;
//   3. cold rows: the 4 probe loads of the global table are issued back to back, then resolved
//      and the rows applied with fire-and-forget atomics.
// At exit the warps' private records and the shared table are merged into the global table.

struct JParams {
  const unsigned char* col_data[16];
  const unsigned char* col_valid[16];
  long long n_rows;
  long long n_units;  // ceil(n_rows / 128)
  int gprobe;
  int pad;
  unsigned long long* gkeys;
  unsigned char* grecs;
  unsigned long long gcap;
  unsigned int* status;
  const unsigned long long* hot_keys;
  const unsigned int* hot_n;
  const unsigned long long* warm_keys;
  const unsigned int* warm_n;
  unsigned long long* kstats;
  int fx[8];    // fraction bits F of each exact float-sum slot (global limbs hold x * 2^F)
  int fx_e[8];  // every value of the slot satisfies |x| < 2^fx_e
};

#define J_UNIT 128

// first probe slot of `key` (shared by the batched probe and the resolve step)
__device__ __forceinline__ long long j_gresolve(const JParams& P, unsigned long long key, unsigned long long h,
                                                unsigned long long first) {
  if (key == PMB_EMPTY64) {
    if (*(volatile unsigned int*)&P.status[1] == 0) atomicOr(&P.status[1], 1u);
    return (long long)P.gcap;
  }
  unsigned long long mask = P.gcap - 1, i = h & mask;
  unsigned long long k = first;
  for (int p = 0; p < P.gprobe; p++) {
    if (k == key) return (long long)i;
    if (k == PMB_EMPTY64) {
      unsigned long long old = atomicCAS(&P.gkeys[i], PMB_EMPTY64, key);
      if (old == PMB_EMPTY64 || old == key) return (long long)i;
    }
    i = (i + 1) & mask;
    k = P.gkeys[i];
  }
  atomicOr(P.status, PMB_ST_OVERFLOW);
  return -1;
}

__device__ __forceinline__ long long j_gfind(const JParams& P, unsigned long long key, unsigned long long h) {
  if (key == PMB_EMPTY64) return j_gresolve(P, key, h, 0ULL);
  return j_gresolve(P, key, h, P.gkeys[h & (P.gcap - 1)]);
}

// read-only lookup in the warm table (keys preloaded per CTA); -1 when absent
__device__ __forceinline__ int j_sfind_ro(const unsigned long long* skeys, unsigned long long key, unsigned long long h) {
  if (J_S == 0 || key == PMB_EMPTY64) return -1;
  int i = (int)((h >> 40) & (unsigned long long)(J_S - 1));
  for (int p = 0; p < J_S; p++) {
    unsigned long long k = skeys[i];
    if (k == key) return i;
    if (k == PMB_EMPTY64) return -1;
    i = (i + 1) & (J_S - 1);
  }
  return -1;
}

__device__ __forceinline__ void j_sinsert(unsigned long long* skeys, unsigned long long key) {
  int i = (int)((pmb_fmix64(key) >> 40) & (unsigned long long)(J_S - 1));
  for (int p = 0; p < J_S; p++) {
    unsigned long long old = atomicCAS(&skeys[i], PMB_EMPTY64, key);
    if (old == PMB_EMPTY64 || old == key) return;
    i = (i + 1) & (J_S - 1);
  }
}

__device__ __forceinline__ int j_hot_find(const unsigned long long* lk, const int* li, unsigned long long key,
                                          unsigned long long h) {
  int i = (int)((h >> 24) & (unsigned long long)(J_HOT_LUT - 1));
  for (int p = 0; p < J_HOT_LUT; p++) {
    unsigned long long k = lk[i];
    if (k == key) return li[i];
    if (k == PMB_EMPTY64) return -1;
    i = (i + 1) & (J_HOT_LUT - 1);
  }
  return -1;
}

extern "C" __global__ void __launch_bounds__(J_NT, 1) pmb_jit_hash_agg(const __grid_constant__ JParams P) {
  extern __shared__ __align__(128) unsigned char sm[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int W = J_NT / 32;
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(sm);  // one per warp
  unsigned char* buf = sm + J_OFF_BUF + warp * J_BUF_BYTES;
  unsigned long long* skeys = reinterpret_cast<unsigned long long*>(sm + J_OFF_SKEYS);
  unsigned char* srecs = sm + J_OFF_SRECS;
  unsigned long long* hlk = reinterpret_cast<unsigned long long*>(sm + J_OFF_HOT_LUT);
  int* hli = reinterpret_cast<int*>(sm + J_OFF_HOT_LUT + 8 * J_HOT_LUT);
  unsigned char* hrecs = sm + J_OFF_HOT_RECS;
  unsigned char* my_hot = hrecs + warp * J_HOT_CAP * J_REC;
  const int n_hot = (J_HOT_CAP > 0 && P.hot_keys) ? (int)min(*P.hot_n, (unsigned)J_HOT_CAP) : 0;
  const int n_warm = (J_S > 0 && P.warm_keys) ? (int)min(*P.warm_n, (unsigned)(J_S / 2)) : 0;

  for (int i = tid; i < J_S; i += J_NT) skeys[i] = PMB_EMPTY64;
  for (int w = tid; w < J_S * J_REC_WORDS; w += J_NT)
    reinterpret_cast<unsigned long long*>(srecs)[w] = J_IDENT[w % J_REC_WORDS];
  if (J_HOT_CAP > 0) {
    for (int i = tid; i < J_HOT_LUT; i += J_NT) hlk[i] = PMB_EMPTY64;
    for (int w = tid; w < W * J_HOT_CAP * J_REC_WORDS; w += J_NT)
      reinterpret_cast<unsigned long long*>(hrecs)[w] = J_IDENT[w % J_REC_WORDS];
  }
  if (tid == 0) {
    for (int w = 0; w < W; w++) mbar_init(&bars[w], 1);
    mbar_fence_init();
  }
  __syncthreads();
  for (int i = tid; i < n_hot; i += J_NT) {
    unsigned long long k = P.hot_keys[i];
    int j = (int)((pmb_fmix64(k) >> 24) & (unsigned long long)(J_HOT_LUT - 1));
    for (int p = 0; p < J_HOT_LUT; p++) {
      if (atomicCAS(&hlk[j], PMB_EMPTY64, k) == PMB_EMPTY64) {
        hli[j] = i;
        break;
      }
      j = (j + 1) & (J_HOT_LUT - 1);
    }
  }
  for (int i = tid; i < n_warm; i += J_NT) j_sinsert(skeys, P.warm_keys[i]);
  __syncthreads();

  const long long gw = (long long)blockIdx.x * W + warp, n_warps = (long long)gridDim.x * W;
  unsigned phase = 0;
  bool aborted = false;
  // optional phase counters (P.kstats): cycles in copy wait / filter+hot / warm / cold, rows per tier
  const bool ks = P.kstats != nullptr;
  long long c_wait = 0, c_p1 = 0, c_p2 = 0, c_p3 = 0, c0 = 0;
  unsigned n_hot_rows = 0, n_warm_rows = 0, n_cold_rows = 0;
  for (long long u = gw; u < P.n_units; u += n_warps) {
    const long long row0 = u * J_UNIT;
    const int rows = (int)min((long long)J_UNIT, P.n_rows - row0);
    if (ks) c0 = clock64();
    if (rows == J_UNIT) {
      if (lane == 0) {
        fence_proxy_async();  // the warp's reads of the previous unit come before the copy's writes
        j_issue_unit(P, buf, u, &bars[warp]);
      }
      bool ok = true;
      if (lane == 0) ok = mbar_wait_bounded(&bars[warp], phase);
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) {
        // give the copy in flight one more bounded wait before leaving its buffer
        if (lane == 0) mbar_wait_bounded(&bars[warp], phase);
        aborted = true;
        break;
      }
      phase ^= 1u;
    } else {
      j_copy_unit(P, buf, row0, rows);
    }
    __syncwarp();
    if (ks) {
      long long c1 = clock64();
      c_wait += c1 - c0;
      c0 = c1;
    }

    // 1. filter, key, hot tier; remember cold rows for the batched probe
    unsigned long long ck[4], ch[4];
    unsigned cold = 0, warm = 0;
    int wslot[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int lr = lane + 32 * j;
      JRow r;
      bool keep = lr < rows && j_load(P, buf, lr, r, true);
      unsigned long long key = keep ? j_key(r) : 0ULL;
      unsigned long long h = pmb_fmix64(key);
      int hot = -1;
      if (J_HOT_CAP > 0 && n_hot && keep && key != PMB_EMPTY64) hot = j_hot_find(hlk, hli, key, h);
      if (J_HOT_CAP > 0) {
        unsigned hm = __ballot_sync(0xffffffffu, hot >= 0);
        if (hm) {
          unsigned peers = __match_any_sync(0xffffffffu, hot) & hm;
          if (hot >= 0 && lane == __ffs(peers) - 1) {
            unsigned char* rec = my_hot + hot * J_REC;
            j_private(P, rec, r);
            for (unsigned m = peers & (peers - 1); m; m &= m - 1) {
              JRow rp;
              j_load_vals(P, buf, (__ffs(m) - 1) + 32 * j, rp);
              j_private(P, rec, rp);
            }
          }
        }
      }
      if (ks && hot >= 0) n_hot_rows++;
      ck[j] = key;
      ch[j] = h;
      wslot[j] = -1;
      if (keep && hot < 0) {
        int si = j_sfind_ro(skeys, key, h);
        if (si >= 0) {
          wslot[j] = si;
          warm |= 1u << j;
        } else {
          cold |= 1u << j;
        }
      }
    }
    if (ks) {
      long long c1 = clock64();
      c_p1 += c1 - c0;
      c0 = c1;
      n_warm_rows += __popc(warm);
      n_cold_rows += __popc(cold);
    }
    // 2. warm rows
#pragma unroll
    for (int j = 0; j < 4; j++) {
      if (warm & (1u << j)) {
        JRow r;
        j_load_vals(P, buf, lane + 32 * j, r);
        j_shared(P, srecs + wslot[j] * J_REC, r);
      }
    }
    if (ks) {
      long long c1 = clock64();
      c_p2 += c1 - c0;
      c0 = c1;
    }
    // 3. cold rows: probe loads first, then resolve and apply
    unsigned long long first[4];
#pragma unroll
    for (int j = 0; j < 4; j++)
      first[j] = ((cold >> j) & 1u) && ck[j] != PMB_EMPTY64 ? P.gkeys[ch[j] & (P.gcap - 1)] : 0ULL;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      if (cold & (1u << j)) {
        long long gi = j_gresolve(P, ck[j], ch[j], first[j]);
        if (gi >= 0) {
          JRow r;
          j_load_vals(P, buf, lane + 32 * j, r);
          j_global(P, P.grecs + (unsigned long long)gi * J_REC, r);
        }
      }
    }
    __syncwarp();
    if (ks) c_p3 += clock64() - c0;
  }
  if (ks) {
    if (lane == 0) {
      atomicAdd(&P.kstats[0], (unsigned long long)c_wait);
      atomicAdd(&P.kstats[1], (unsigned long long)c_p1);
      atomicAdd(&P.kstats[2], (unsigned long long)c_p2);
      atomicAdd(&P.kstats[3], (unsigned long long)c_p3);
    }
    unsigned a = n_hot_rows, b = n_warm_rows, c = n_cold_rows;
    for (int o = 16; o; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      b += __shfl_xor_sync(0xffffffffu, b, o);
      c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if (lane == 0) {
      atomicAdd(&P.kstats[4], (unsigned long long)a);
      atomicAdd(&P.kstats[5], (unsigned long long)b);
      atomicAdd(&P.kstats[6], (unsigned long long)c);
      atomicAdd(&P.kstats[7], 1ULL);
    }
  }
  if (aborted && lane == 0) atomicOr(P.status, PMB_ST_TIMEOUT);
  __syncthreads();
  // hot keys: fold the warps' private records, then one merge per touched key
  for (int i = tid; i < n_hot; i += J_NT) {
    unsigned char* r0 = hrecs + i * J_REC;
    for (int w = 1; w < W; w++) j_merge_private(r0, hrecs + (w * J_HOT_CAP + i) * J_REC);
    if (*reinterpret_cast<const unsigned int*>(r0 + J_LEN_OFF) == 0) continue;
    unsigned long long key = P.hot_keys[i];
    long long gi = j_gfind(P, key, pmb_fmix64(key));
    if (gi >= 0) j_merge_global(P, P.grecs + (unsigned long long)gi * J_REC, r0);
  }
  // the warm table (preloaded keys may have seen no rows)
  for (int i = tid; i < J_S; i += J_NT) {
    unsigned long long key = skeys[i];
    if (key == PMB_EMPTY64) continue;
    const unsigned char* r = srecs + i * J_REC;
    if (*reinterpret_cast<const unsigned int*>(r + J_LEN_OFF) == 0) continue;
    long long gi = j_gfind(P, key, pmb_fmix64(key));
    if (gi >= 0) j_merge_global(P, P.grecs + (unsigned long long)gi * J_REC, r);
  }
}
