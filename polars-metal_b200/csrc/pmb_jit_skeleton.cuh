// pmb_jit_skeleton.cuh — the fused filter -> group_by -> aggregate kernel compiled at run time
// for one query signature (NVRTC). This text follows pmb_device.cuh and a generated section that
// defines, for that signature, the J_* layout constants and the row functions:
//   j_issue_unit   one warp's bulk copies (TMA, cp.async.bulk) of a 128-row unit into a buffer
//   j_copy_unit    plain copy of a partial last unit
//   JRow           the values of one row of a unit buffer
//   j_load_pk      the predicate and key columns of a row, and the filter verdict
//   j_load_vals    the aggregated columns of a row
//   j_key          the packed 64-bit group key
//   j_fxcheck      range report of the exact float sums (the call is re-run wider on a report)
//   j_shared       one row into a shared-memory record (native 32-bit atomics only: counters,
//                  carry-chained 32-bit words for the exact sums, 64-bit min/max)
//   j_global       one row into a global-table record (fire-and-forget 64-bit atomics)
//   j_sfold        a shared-memory record into another (one owner)
//   j_merge_sg     a shared-memory record into a global-table record
//   J_SIDENT       the identity shared-memory record (u32 words)
//
// Execution: persistent CTAs whose warps run independently (no CTA barrier in the main loop). A
// warp takes 128-row units round-robin over all warps of the grid; lane 0 bulk-copies a unit's
// column chunks into one of the warp's J_NBUF buffers (one mbarrier each, bounded waits), so with
// two buffers the next unit is in flight while this one is processed. Per unit:
//   1. classify: each lane evaluates the filter and the key of rows lane, lane+32, lane+64,
//      lane+96 and looks the key up in the CTA's read-only table of sampled keys (every lane,
//      kept row or not, so the lookup never diverges). Rows of sampled
//      keys ("hot": the heaviest, with one record per warp; "warm": one record per CTA) and the
//      other kept rows ("cold") are compacted with ballots into the warp's queue;
//   2. the queued shared-tier rows are applied 32 at a time, every lane busy;
//   3. the queued cold rows are applied to the global table 32 at a time.
// A table overflow (probe limit) or a failed wait makes every warp stop at its next unit; the
// host then re-runs with a larger table. At exit the hot records of all warps are folded and, with
// the warm records, merged into the global table.

struct JParams {
  const unsigned char* col_data[16];
  const unsigned char* col_valid[16];
  long long n_rows;
  long long n_units;  // ceil(n_rows / 128)
  int gprobe;              // probe limit, in 4-slot buckets
  unsigned int occ_limit;  // claimed slots at which the table counts as full (overflow)
  unsigned long long* gkeys;
  unsigned char* grecs;
  unsigned long long gcap;
  unsigned int* status;
  const unsigned long long* hot_keys;
  const unsigned int* hot_n;
  const unsigned long long* warm_keys;
  const unsigned int* warm_n;
  unsigned long long* kstats;
  const unsigned char* ttab;  // sampled-key table (k_sample_table): keys of all buckets, then values
  int tnb;                    // its buckets (4 slots each), at most J_TNB
  int flags;                  // batched kernel: bit 0 = fill the CTA's warm table
  int fx[8];    // fraction bits F of each exact float-sum slot (sums hold x * 2^F)
  int fx_e[8];  // every value of the slot satisfies |x| < 2^fx_e
};

#define J_UNIT 128
#define J_MISS 0xFFFFFFFFu
#define J_HOTBIT 0x40000000u

// Global table: linear probing over 4-slot buckets (one 32-byte sector of keys, read with two
// 16-byte loads), so a probe sequence costs about one round trip to L2 per 4 slots. Returns the
// slot of `key` (claiming an empty one with a CAS; `claimed` tells), or -1 and PMB_ST_OVERFLOW at
// the probe limit. The key whose bits equal the EMPTY marker has the extra slot gcap.
__device__ __forceinline__ long long j_gresolve(const JParams& P, unsigned long long key, unsigned long long h,
                                                bool& claimed) {
  claimed = false;
  if (key == PMB_EMPTY64) {
    if (*(volatile unsigned int*)&P.status[1] == 0) atomicOr(&P.status[1], 1u);
    return (long long)P.gcap;
  }
  const unsigned long long nb = P.gcap >> 2;
  unsigned long long bk = pmb_slot(h, nb);
  for (int p = 0; p < P.gprobe; p++) {
    const ulonglong2* src = reinterpret_cast<const ulonglong2*>(P.gkeys + 4 * bk);
    const ulonglong2 a = src[0], c = src[1];
    const unsigned long long ks[4] = {a.x, a.y, c.x, c.y};
#pragma unroll
    for (int s = 0; s < 4; s++) {
      if (ks[s] == key) return (long long)(4 * bk + s);
      if (ks[s] == PMB_EMPTY64) {
        unsigned long long old = atomicCAS(&P.gkeys[4 * bk + s], PMB_EMPTY64, key);
        if (old == PMB_EMPTY64) {
          claimed = true;
          return (long long)(4 * bk + s);
        }
        if (old == key) return (long long)(4 * bk + s);
      }
    }
    bk = (bk + 1 == nb) ? 0ULL : bk + 1;
  }
  atomicOr(P.status, PMB_ST_OVERFLOW);
  return -1;
}

__device__ __forceinline__ long long j_gfind(const JParams& P, unsigned long long key, unsigned long long h) {
  bool claimed;
  return j_gresolve(P, key, h, claimed);
}

// The CTA's table of sampled keys (hot and warm), built on the device by k_sample_table: a key
// sits in its first bucket (4 slots) unless that bucket was already full, then in its second.
// Empty slots hold the value 0xFFFF (a miss whatever their key word), so a first bucket with an
// empty slot ends a lookup: its keys never spilled over. A lookup reads a bucket's keys and values
// side by side; the value is J_HOTBIT | hot index, a warm index, or J_MISS. Bit 14 of a bucket's
// first value marks a bucket that turned a key away to its second bucket.
__device__ __forceinline__ unsigned j_tvalue(unsigned short v) {
  return v == 0xFFFFu ? J_MISS : ((v & 0x8000u) ? (J_HOTBIT | (v & 0x3FFFu)) : (unsigned)(v & 0x3FFFu));
}
// the 16-bit value of slot s of a bucket whose values are (lo, hi)
__device__ __forceinline__ unsigned short j_tslot(uint2 v, int s) {
  const unsigned w = (s & 2) ? v.y : v.x;
  return (unsigned short)((s & 1) ? (w >> 16) : (w & 0xFFFFu));
}
// bucket bk of the table: the key's value, or J_MISS; `full` tells whether the bucket turned a
// key away (then a missing key may sit in its second bucket). Straight-line code, no branch.
__device__ __forceinline__ unsigned j_tprobe(const unsigned char* tk, const unsigned short* tv, unsigned bk,
                                             unsigned long long key, bool& full) {
  const uint2 vx = reinterpret_cast<const uint2*>(tv)[bk];
#if J_TKEY == 4
  const unsigned k = (unsigned)key;
  const uint4 x = reinterpret_cast<const uint4*>(tk)[bk];
  const int s = x.x == k ? 0 : x.y == k ? 1 : x.z == k ? 2 : x.w == k ? 3 : -1;
#else
  const ulonglong2* t = reinterpret_cast<const ulonglong2*>(tk);
  const ulonglong2 x0 = t[2 * bk], x1 = t[2 * bk + 1];
  const int s = x0.x == key ? 0 : x0.y == key ? 1 : x1.x == key ? 2 : x1.y == key ? 3 : -1;
#endif
  const unsigned v0 = vx.x & 0xFFFFu;
  full = s < 0 && v0 != 0xFFFFu && (v0 & 0x4000u) != 0u;
  return s >= 0 ? j_tvalue(j_tslot(vx, s)) : J_MISS;
}

__device__ __forceinline__ bool j_stop(const JParams& P) {
  return (*(volatile unsigned int*)P.status & (PMB_ST_OVERFLOW | PMB_ST_TIMEOUT)) != 0u;
}

extern "C" __global__ void __launch_bounds__(J_NT, 1) pmb_jit_hash_agg(const __grid_constant__ JParams P) {
  extern __shared__ __align__(128) unsigned char sm[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int W = J_NT / 32;
  unsigned long long* all_bars = reinterpret_cast<unsigned long long*>(sm + J_OFF_BARS);
  unsigned long long* bars = all_bars + warp * J_NBUF;
  unsigned char* bufs = sm + J_OFF_BUF + warp * J_NBUF * J_BUF_BYTES;
  unsigned* q = reinterpret_cast<unsigned*>(sm + J_OFF_Q) + warp * J_UNIT;
  unsigned char* tkeys = sm + J_OFF_TKEYS;
  unsigned short* tval = reinterpret_cast<unsigned short*>(sm + J_OFF_TVAL);
  const unsigned tnb = (unsigned)min(P.tnb, J_TNB);
  unsigned char* srecs = sm + J_OFF_SRECS;
  __shared__ unsigned s_claims;  // slots this CTA claimed in the global table (published per 64)
  const int n_hot = (J_H > 0 && P.hot_keys) ? (int)min(*P.hot_n, (unsigned)J_H) : 0;
  const int n_warm = (J_SW > 0 && P.warm_keys) ? (int)min(*P.warm_n, (unsigned)J_SW) : 0;

  // the sampled-key table: keys (tnb * 4 * J_TKEY bytes), then values (tnb * 8 bytes; tnb is even)
  if (P.ttab) {
    const uint4* src = reinterpret_cast<const uint4*>(P.ttab);
    const int kw = (int)(tnb * 4u * J_TKEY / 16u), vw = (int)(tnb * 8u / 16u);
    for (int i = tid; i < kw; i += J_NT) reinterpret_cast<uint4*>(tkeys)[i] = src[i];
    for (int i = tid; i < vw; i += J_NT) reinterpret_cast<uint4*>(tval)[i] = src[kw + i];
  }
  for (int w = tid; w < (W * J_H + J_SW) * J_SREC_WORDS; w += J_NT)
    reinterpret_cast<unsigned*>(srecs)[w] = J_SIDENT[w % J_SREC_WORDS];
  if (tid == 0) {
    s_claims = 0u;
    for (int b = 0; b < W * J_NBUF; b++) mbar_init(&all_bars[b], 1);
    mbar_fence_init();
  }
  __syncthreads();

  const long long n_full = P.n_rows / J_UNIT;
  const long long gw = (long long)blockIdx.x * W + warp, n_warps = (long long)gridDim.x * W;
  const unsigned long long pol = pmb_policy_evict_first();
  unsigned parity = 0, pending = 0;  // per buffer: phase to wait for, copy in flight
  if (lane == 0) {
    for (int b = 0; b < J_NBUF; b++) {
      long long uu = gw + b * n_warps;
      if (uu < n_full) {
        j_issue_unit(P, bufs + b * J_BUF_BYTES, uu, &bars[b], pol);
        pending |= 1u << b;
      }
    }
  }
  bool aborted = false;
  const bool ks = P.kstats != nullptr;
  long long c_wait = 0, c_cls = 0, c_sh = 0, c_cold = 0, c0 = 0;
  unsigned n_sh_rows = 0, n_cold_rows = 0;
  int b = 0;
  for (long long u = gw, k = 0; u < P.n_units; u += n_warps, k++) {
    if ((k & 3) == 3) {
      bool stop = false;
      if (lane == 0) stop = j_stop(P);
      if (__shfl_sync(0xffffffffu, stop, 0)) break;
    }
    const long long row0 = u * J_UNIT;
    const int rows = (int)min((long long)J_UNIT, P.n_rows - row0);
    unsigned char* st = bufs + b * J_BUF_BYTES;
    if (ks) c0 = clock64();
    if (rows == J_UNIT) {
      bool ok = true;
      if (lane == 0) {
#if J_WAIT_NS > 0
        ok = mbar_wait_bounded_sleep(&bars[b], (parity >> b) & 1u, J_WAIT_NS);
#else
        ok = mbar_wait_bounded(&bars[b], (parity >> b) & 1u);
#endif
        if (ok) {
          parity ^= 1u << b;
          pending &= ~(1u << b);
        }
      }
      if (!__shfl_sync(0xffffffffu, ok, 0)) {
        aborted = true;
        break;
      }
    } else {
      j_copy_unit(P, st, row0, rows);
    }
    __syncwarp();
    if (ks) {
      long long c1 = clock64();
      c_wait += c1 - c0;
      c0 = c1;
    }

    // 1. classify and compact: shared-tier entries (record << 7 | row) from the front of the
    //    queue, cold rows from the back
    int ns = 0, nc = 0;
    const unsigned lt = (1u << lane) - 1u;
    unsigned ent[4];  // 0: dropped, J_MISS: cold, else shared-tier entry (record << 7 | row) + 1
    // Every lane looks up the key of each of its rows in the first bucket, kept or not (a dropped
    // row's answer is ignored), so the lookup runs with all lanes and no divergent exits; the
    // second bucket, needed only behind a bucket that turned a key away, is taken by the whole
    // warp together.
    const unsigned tnb_eff = P.ttab ? tnb : 0u;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int lr = lane + 32 * j;  // rows past a partial unit read stale buffer bytes, then drop
      JRow r;
      const bool keep = j_load_pk(P, st, lr, r) && lr < rows;
      const unsigned long long key = j_key(r);
      const unsigned a = (unsigned)(j_hash(key) >> 32);
      unsigned v = J_MISS;
      bool full = false;
      if (tnb_eff) v = j_tprobe(tkeys, tval, __umulhi(a, tnb_eff), key, full);
      if (__any_sync(0xffffffffu, keep && full)) {
        bool full2;
        if (keep && full) v = j_tprobe(tkeys, tval, __umulhi(pmb_mix32b(a), tnb_eff), key, full2);
      }
      const unsigned rec = (v & J_HOTBIT) ? (unsigned)(warp * J_H) + (v & ~J_HOTBIT) : (unsigned)(W * J_H) + v;
      ent[j] = !keep ? 0u : (v != J_MISS ? ((rec << 7) | (unsigned)lr) + 1u : J_MISS);
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const bool sh = ent[j] != 0u && ent[j] != J_MISS, cold = ent[j] == J_MISS;
      const unsigned bs = __ballot_sync(0xffffffffu, sh), bc = __ballot_sync(0xffffffffu, cold);
      if (sh) q[ns + __popc(bs & lt)] = ent[j] - 1u;
      if (cold) q[J_UNIT - 1 - (nc + __popc(bc & lt))] = (unsigned)(lane + 32 * j);
      ns += __popc(bs);
      nc += __popc(bc);
    }
    __syncwarp();
    if (ks) {
      long long c1 = clock64();
      c_cls += c1 - c0;
      c0 = c1;
      n_sh_rows += ns;
      n_cold_rows += nc;
    }
    // 2. shared tier
    for (int base = 0; base < ns; base += 32) {
      if (base + lane < ns) {
        const unsigned e = q[base + lane];
        JRow r;
        j_load_vals(P, st, (int)(e & 127u), r);
        j_fxcheck(P, r);
        j_shared(P, srecs + (e >> 7) * J_SREC, r);
      }
    }
    if (ks) {
      long long c1 = clock64();
      c_sh += c1 - c0;
      c0 = c1;
    }
    // 3. cold tier. Most cold keys already sit in their first bucket: that probe is straight-line
    //    code, and the probing loop (claims, later buckets) only runs for the other lanes. The
    //    lanes meet again before the record updates, so those run once for the whole round.
    for (int base = 0; base < nc; base += 32) {
      const bool act = base + lane < nc;
      const unsigned am = __ballot_sync(0xffffffffu, act);
      if (act) {
        const int lr = (int)q[J_UNIT - 1 - (base + lane)];
        JRow r;
        j_load_key(P, st, lr, r);
        j_load_vals(P, st, lr, r);
        const unsigned long long key = j_key(r);
        j_fxcheck(P, r);
        const unsigned long long hk = j_hash(key);
        bool claimed = false;
        long long gi = -1;
        if (key != PMB_EMPTY64) {
          const unsigned long long bk = pmb_slot(hk, P.gcap >> 2);
          const ulonglong2* src = reinterpret_cast<const ulonglong2*>(P.gkeys + 4 * bk);
          const ulonglong2 x0 = src[0], x1 = src[1];
          const int s = x0.x == key ? 0 : x0.y == key ? 1 : x1.x == key ? 2 : x1.y == key ? 3 : -1;
          if (s >= 0) gi = (long long)(4 * bk + s);
        }
        if (gi < 0) gi = j_gresolve(P, key, hk, claimed);
        __syncwarp(am);
        if (gi >= 0) j_global(P, P.grecs + (unsigned long long)gi * J_REC, r);
        if (claimed && ((atomicAdd(&s_claims, 1u) + 1u) & 63u) == 0u) {
          // every 64 claims of this CTA: publish them; past the limit the table counts as full
          if (atomicAdd(&P.status[2], 64u) + 64u > P.occ_limit) atomicOr(P.status, PMB_ST_OVERFLOW);
        }
      }
    }
    __syncwarp();
    if (ks) c_cold += clock64() - c0;
    // this buffer is free again: bring in the warp's unit J_NBUF steps ahead
    if (lane == 0) {
      const long long uu = u + (long long)J_NBUF * n_warps;
      if (uu < n_full) {
        fence_proxy_async();  // the warp's reads of this unit come before the copy's writes
        j_issue_unit(P, st, uu, &bars[b], pol);
        pending |= 1u << b;
      }
    }
    b = (b + 1 == J_NBUF) ? 0 : b + 1;
  }
  // copies still in flight land before the buffers are given up
  if (lane == 0) {
    for (int bb = 0; bb < J_NBUF; bb++)
      if ((pending >> bb) & 1u) {
        if (!mbar_wait_bounded(&bars[bb], (parity >> bb) & 1u)) aborted = true;
      }
  }
  if (ks) {
    if (lane == 0) {
      atomicAdd(&P.kstats[0], (unsigned long long)c_wait);
      atomicAdd(&P.kstats[1], (unsigned long long)c_cls);
      atomicAdd(&P.kstats[2], (unsigned long long)c_sh);
      atomicAdd(&P.kstats[3], (unsigned long long)c_cold);
      atomicAdd(&P.kstats[4], (unsigned long long)n_sh_rows);
      atomicAdd(&P.kstats[5], (unsigned long long)n_cold_rows);
      atomicAdd(&P.kstats[7], 1ULL);
    }
  }
  if (aborted && lane == 0) atomicOr(P.status, PMB_ST_TIMEOUT);
  __syncthreads();
  if (j_stop(P)) return;  // the host re-runs this call; the partial records are discarded
  // hot keys: fold the warps' records into warp 0's, then one merge per touched key
  for (int i = tid; i < n_hot; i += J_NT) {
    unsigned char* r0 = srecs + i * J_SREC;
    for (int w = 1; w < W; w++) j_sfold(r0, srecs + (w * J_H + i) * J_SREC);
    if (*reinterpret_cast<const unsigned*>(r0 + J_LEN_SOFF) == 0u) continue;
    const unsigned long long key = P.hot_keys[i];
    const long long gi = j_gfind(P, key, j_hash(key));
    if (gi >= 0) j_merge_sg(P, P.grecs + (unsigned long long)gi * J_REC, r0);
  }
  for (int i = tid; i < n_warm; i += J_NT) {
    const unsigned char* r = srecs + (W * J_H + i) * J_SREC;
    if (*reinterpret_cast<const unsigned*>(r + J_LEN_SOFF) == 0u) continue;
    const unsigned long long key = P.warm_keys[i];
    const long long gi = j_gfind(P, key, j_hash(key));
    if (gi >= 0) j_merge_sg(P, P.grecs + (unsigned long long)gi * J_REC, r);
  }
}
