// pmb_jit_batch.cuh — many group-by queries of one signature in one persistent launch (compiled at
// run time with the row functions of that signature; follows pmb_jit_skeleton.cuh in the same
// NVRTC source, whose JParams, j_gresolve and j_gfind it uses).
//
// The work queue holds items (query, unit range); each query has its own JParams (columns, global
// table, status, float-sum ranges, hot keys). A CTA takes items through a ticket. Per item:
//   1. the CTA's tables are reset: the query's hot keys (one record per warp each) and a warm
//      table filled on the fly (find-or-insert with a short probe; a full table sends the row to
//      the global table instead);
//   2. warps stream the item's 128-row units through their J_NBUF buffers (1-D TMA copies, the
//      warp's next units in flight while it works on one; bounded waits), classify rows (filter,
//      key, hot / warm / cold) into the warp queue and apply them: shared-memory records with
//      native 32-bit atomics, cold rows to the query's global table. The warm table is used only
//      for queries whose flags bit 0 the host set (few groups, or many rows per group in an item);
//      otherwise a key's rows would rarely meet in one item and the table would only add work;
//   3. after a CTA barrier the hot records of all warps are folded and, with the warm records,
//      merged into the query's global table.
// A failed wait stops the warp for the rest of the launch and reports PMB_ST_TIMEOUT in the
// item's query status; the host then fails the call.

struct JBatchItem {
  int q;
  int pad;
  long long u0, u1;  // units [u0, u1) of query q
};

struct JBatch {
  const JParams* qp;
  const JBatchItem* items;
  long long n_items;
  unsigned long long* ticket;
};

// find-or-insert in the CTA's warm table (J_SW slots, a power of two); J_MISS after 16 probes
__device__ __forceinline__ unsigned j_wfind(unsigned long long* wk, unsigned long long key, unsigned long long h) {
  if (J_SW == 0 || key == PMB_EMPTY64) return J_MISS;
  unsigned i = (unsigned)(h >> 40) & (unsigned)(J_SW - 1);
  for (int p = 0; p < 16; p++) {
    const unsigned long long k = wk[i];
    if (k == key) return i;
    if (k == PMB_EMPTY64) {
      const unsigned long long old = atomicCAS(&wk[i], PMB_EMPTY64, key);
      if (old == PMB_EMPTY64 || old == key) return i;
    }
    i = (i + 1) & (unsigned)(J_SW - 1);
  }
  return J_MISS;
}

extern "C" __global__ void __launch_bounds__(J_NT, 1) pmb_jit_batch_agg(const __grid_constant__ JBatch B) {
  extern __shared__ __align__(128) unsigned char sm[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int W = J_NT / 32;
  unsigned long long* all_bars = reinterpret_cast<unsigned long long*>(sm + J_OFF_BARS);
  unsigned long long* bars = all_bars + warp * J_NBUF;
  unsigned char* bufs = sm + J_OFF_BUF + warp * J_NBUF * J_BUF_BYTES;
  unsigned* q = reinterpret_cast<unsigned*>(sm + J_OFF_Q) + warp * J_UNIT;
  unsigned long long* wk = reinterpret_cast<unsigned long long*>(sm + J_OFF_TKEYS);  // J_SW warm keys
  unsigned long long* hk = reinterpret_cast<unsigned long long*>(sm + J_OFF_TVAL);   // J_H hot keys
  unsigned char* srecs = sm + J_OFF_SRECS;  // W * J_H hot records, then J_SW warm records
  __shared__ long long s_item;
  __shared__ int s_nhot;
  // the item's query parameters live in shared memory: the unit loop reads them for every row,
  // and the small L1 left beside the tables would keep evicting them
  __shared__ __align__(16) unsigned char s_par[sizeof(JParams)];
  const JParams& P = *reinterpret_cast<const JParams*>(s_par);
  if (tid == 0) {
    for (int b = 0; b < W * J_NBUF; b++) mbar_init(&all_bars[b], 1);
    mbar_fence_init();
  }
  unsigned parity = 0, pending = 0;  // per buffer: phase to wait for, copy in flight
  bool dead = false;  // a wait of this warp gave up: it does no more work in this launch
  const unsigned long long pol = pmb_policy_evict_first();
  const unsigned lt = (1u << lane) - 1u;
  for (;;) {
    __syncthreads();
    if (tid == 0) s_item = (long long)atomicAdd(B.ticket, 1ULL);
    __syncthreads();
    const long long it = s_item;
    if (it >= B.n_items) break;
    const JBatchItem I = B.items[it];
    for (int i = tid; i < (int)(sizeof(JParams) / 4); i += J_NT)
      reinterpret_cast<unsigned*>(s_par)[i] = reinterpret_cast<const unsigned*>(B.qp + I.q)[i];
    __syncthreads();
    const bool warm = J_SW > 0 && (P.flags & 1);
    const long long n_full = P.n_rows / J_UNIT;
    // the warp's first units of the item go in flight while the tables are reset
    if (lane == 0 && !dead) {
      for (int b = 0; b < J_NBUF; b++) {
        const long long uu = I.u0 + warp + (long long)b * W;
        if (uu < I.u1 && uu < n_full) {
          fence_proxy_async();  // the warp's reads of the buffer's previous unit come before the copy's writes
          j_issue_unit(P, bufs + b * J_BUF_BYTES, uu, &bars[b], pol);
          pending |= 1u << b;
        }
      }
    }
    if (warm)
      for (int i = tid; i < J_SW; i += J_NT) wk[i] = PMB_EMPTY64;
    for (int w = tid; w < (W * J_H + (warm ? J_SW : 0)) * J_SREC_WORDS; w += J_NT)
      reinterpret_cast<unsigned*>(srecs)[w] = J_SIDENT[w % J_SREC_WORDS];
    if (tid == 0) {
      const int nh = (J_H > 0 && P.hot_keys) ? (int)min(*P.hot_n, (unsigned)J_H) : 0;
      for (int i = 0; i < nh; i++) hk[i] = P.hot_keys[i];
      s_nhot = nh;
    }
    __syncthreads();
    const int nhot = s_nhot;
    int b = 0;
    for (long long u = I.u0 + warp; u < I.u1 && !dead; u += W) {
      const long long row0 = u * J_UNIT;
      const int rows = (int)min((long long)J_UNIT, P.n_rows - row0);
      unsigned char* st = bufs + b * J_BUF_BYTES;
      if (rows == J_UNIT) {
        bool ok = true;
        if (lane == 0) {
          ok = mbar_wait_bounded(&bars[b], (parity >> b) & 1u);
          if (ok) {
            parity ^= 1u << b;
            pending &= ~(1u << b);
          }
        }
        if (!__shfl_sync(0xffffffffu, ok, 0)) {
          dead = true;
          break;
        }
      } else {
        j_copy_unit(P, st, row0, rows);  // the query's last, partial unit: no copy was issued into this buffer
      }
      __syncwarp();
      int ns = 0, nc = 0;
      unsigned ent[4];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int lr = lane + 32 * j;
        JRow r;
        const bool keep = lr < rows && j_load_pk(P, st, lr, r);
        ent[j] = 0u;
        if (keep) {
          const unsigned long long key = j_key(r);
          unsigned rec = J_MISS;
          for (int i = 0; i < nhot; i++)
            if (hk[i] == key) rec = (unsigned)(warp * J_H + i);
          if (rec == J_MISS && warm) {
            const unsigned s = j_wfind(wk, key, j_hash(key));
            if (s != J_MISS) rec = (unsigned)(W * J_H) + s;
          }
          ent[j] = rec == J_MISS ? J_MISS : ((rec << 7) | (unsigned)lr) + 1u;
        }
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
      for (int base = 0; base < ns; base += 32) {
        if (base + lane < ns) {
          const unsigned e = q[base + lane];
          JRow r;
          j_load_vals(P, st, (int)(e & 127u), r);
          j_fxcheck(P, r);
          j_shared(P, srecs + (e >> 7) * J_SREC, r);
        }
      }
      for (int base = 0; base < nc; base += 32) {
        if (base + lane < nc) {
          const int lr = (int)q[J_UNIT - 1 - (base + lane)];
          JRow r;
          j_load_key(P, st, lr, r);
          j_load_vals(P, st, lr, r);
          const unsigned long long key = j_key(r);
          j_fxcheck(P, r);
          bool claimed;
          const long long gi = j_gresolve(P, key, j_hash(key), claimed);
          if (gi >= 0) j_global(P, P.grecs + (unsigned long long)gi * J_REC, r);
        }
      }
      __syncwarp();
      // this buffer is free again: bring in the warp's unit J_NBUF steps ahead (inside the item)
      if (lane == 0) {
        const long long uu = u + (long long)J_NBUF * W;
        if (uu < I.u1 && uu < n_full) {
          fence_proxy_async();
          j_issue_unit(P, st, uu, &bars[b], pol);
          pending |= 1u << b;
        }
      }
      b = (b + 1 == J_NBUF) ? 0 : b + 1;
    }
    if (dead && lane == 0 && pending) {
      // copies still in flight land (bounded) before the warp gives up its buffers
      for (int bb = 0; bb < J_NBUF; bb++)
        if ((pending >> bb) & 1u) mbar_wait_bounded(&bars[bb], (parity >> bb) & 1u);
      pending = 0;
      atomicOr(P.status, PMB_ST_TIMEOUT);
    }
    __syncthreads();
    // merge the item's CTA records into the query's global table
    for (int i = tid; i < nhot; i += J_NT) {
      unsigned char* r0 = srecs + i * J_SREC;
      for (int w = 1; w < W; w++) j_sfold(r0, srecs + (w * J_H + i) * J_SREC);
      if (*reinterpret_cast<const unsigned*>(r0 + J_LEN_SOFF) == 0u) continue;
      const unsigned long long key = hk[i];
      const long long gi = j_gfind(P, key, j_hash(key));
      if (gi >= 0) j_merge_sg(P, P.grecs + (unsigned long long)gi * J_REC, r0);
    }
    if (warm)
      for (int i = tid; i < J_SW; i += J_NT) {
        const unsigned long long key = wk[i];
        if (key == PMB_EMPTY64) continue;
        const unsigned char* r = srecs + (W * J_H + i) * J_SREC;
        if (*reinterpret_cast<const unsigned*>(r + J_LEN_SOFF) == 0u) continue;
        const long long gi = j_gfind(P, key, j_hash(key));
        if (gi >= 0) j_merge_sg(P, P.grecs + (unsigned long long)gi * J_REC, r);
      }
  }
}
