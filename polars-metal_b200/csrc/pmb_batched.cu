// pmb_batched.cu — many independent group-by queries in one persistent launch.
//
// No counterpart in the reference (it runs one query per call). Queries of one signature (same
// column dtypes and nullability, keys, aggregates and filter) that fit the 64-bit key path run
// together:
//   1. k_batch_sketch — one CTA per query samples 4096 rows: kept rows, distinct keys and
//      singletons (the group estimate), the heaviest keys (the hot keys of the query) and the
//      float-sum ranges; with an installed strategy selector its predicted group count can only
//      enlarge the estimate;
//   2. the host sizes every query's global table (2.5 slots per estimated group, or the tuned
//      count) inside one arena,
//      cuts the queries into work items (query, range of 128-row units) and uploads them;
//   3. one init kernel, the persistent run-time compiled kernel pmb_jit_batch_agg over the work
//      queue, and k_batch_finalize (every query's occupied slots into its output columns, in slot
//      order per query) — captured once into a CUDA graph and replayed while the launch shape
//      stays the same;
//   4. queries whose table overflowed or whose float sums left their range run again, alone in a
//      second batch round with a larger table / wider range.
// The block size, item size, unit buffers, warm rule, shared-table (warm) capacity and global-table
// capacity come from a small autotuner: the first batch of a signature times each candidate on its
// real data and keeps the fastest for the process.
// Other queries (other signatures, 128-bit keys, no NVRTC) run one by one through pmb_groupby.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "pmb_groupby.h"
#include "pmb_jit.h"

namespace {

constexpr int BS_NT = 1024;
constexpr int BS_SAMPLE = 4096;
constexpr int BS_SLOTS = 8192;
constexpr int BS_HOT = 8;

struct BatchSketch {
  long long kept, samples, distinct, f1;
  unsigned int hot_n, pad;
  unsigned int fx_expo[PMB_MAX_FX];
  unsigned long long hot[BS_HOT];
};

struct FxColsB {
  int n;
  int col[PMB_MAX_FX];
};

__global__ void __launch_bounds__(BS_NT) k_batch_sketch(const DQuery* __restrict__ qs, BatchSketch* __restrict__ out,
                                                        const __grid_constant__ FxColsB fxc) {
  extern __shared__ unsigned char smem[];
  unsigned long long* s_key = reinterpret_cast<unsigned long long*>(smem);          // BS_SLOTS
  unsigned int* s_cnt = reinterpret_cast<unsigned int*>(s_key + BS_SLOTS);           // BS_SLOTS
  unsigned int* s_cand = s_cnt + BS_SLOTS;                                            // 1024 candidates
  __shared__ unsigned int s_acc[4];  // kept, distinct, singletons, candidates
  __shared__ unsigned int s_fx[PMB_MAX_FX];
  const DQuery& q = qs[blockIdx.x];
  const int tid = threadIdx.x;
  for (int i = tid; i < BS_SLOTS; i += BS_NT) {
    s_key[i] = PMB_EMPTY64;
    s_cnt[i] = 0u;
  }
  if (tid < 4) s_acc[tid] = 0u;
  if (tid < PMB_MAX_FX) s_fx[tid] = 0u;
  __syncthreads();
  const int64_t n = q.n_rows;
  const int m = (int)(n < BS_SAMPLE ? n : BS_SAMPLE);
  const TileCtx t{nullptr, nullptr, nullptr, 0};
  const bool pred = q.prog.n_ops > 0;
  for (int i = tid; i < m; i += BS_NT) {
    const int64_t r = (int64_t)((__int128)i * n / m);
    if (pred && !eval_keep(q, t, r)) continue;
    atomicAdd(&s_acc[0], 1u);
    for (int f = 0; f < fxc.n; f++) {
      const int c = fxc.col[f];
      if (!tc_isvalid(q, t, c, r)) continue;
      const double x = pmb_bits_to_f64(tc_bits(q, t, c, r), q.col[c].dtype);
      if (!pmb_fx_flag(x)) atomicMax(&s_fx[f], (unsigned)pmb_fx_expo(x));
    }
    const unsigned long long k = pack_key64(q, t, r);
    if (k == PMB_EMPTY64) continue;  // that key always takes its table's extra slot
    unsigned s = (unsigned)(pmb_fmix64(k) & (BS_SLOTS - 1));
    for (int p = 0; p < BS_SLOTS; p++) {
      const unsigned long long cur = s_key[s];
      if (cur == k) break;
      if (cur == PMB_EMPTY64) {
        const unsigned long long old = atomicCAS(&s_key[s], PMB_EMPTY64, k);
        if (old == PMB_EMPTY64 || old == k) break;
      }
      s = (s + 1) & (BS_SLOTS - 1);
    }
    atomicAdd(&s_cnt[s], 1u);
  }
  __syncthreads();
  const unsigned kept = s_acc[0];
  const unsigned hot_min = max(4u, kept / 256u);  // hot: at least 1/256 of the sampled rows
  for (int i = tid; i < BS_SLOTS; i += BS_NT) {
    const unsigned c = s_cnt[i];
    if (!c) continue;
    atomicAdd(&s_acc[1], 1u);
    if (c == 1) atomicAdd(&s_acc[2], 1u);
    if (c >= hot_min) {
      const unsigned j = atomicAdd(&s_acc[3], 1u);
      if (j < 1024) s_cand[j] = (unsigned)i;
    }
  }
  __syncthreads();
  if (tid == 0) {
    BatchSketch& o = out[blockIdx.x];
    o.kept = kept;
    o.samples = m;
    o.distinct = s_acc[1];
    o.f1 = s_acc[2];
    for (int f = 0; f < PMB_MAX_FX; f++) o.fx_expo[f] = s_fx[f];
    // the (up to) BS_HOT heaviest candidates
    const unsigned nc = min(s_acc[3], 1024u);
    unsigned top[BS_HOT];
    int nt = 0;
    for (unsigned j = 0; j < nc; j++) {
      const unsigned slot = s_cand[j], c = s_cnt[slot];
      int pos = nt < BS_HOT ? nt : -1;
      if (pos < 0 && c > s_cnt[top[BS_HOT - 1]]) pos = BS_HOT - 1;
      if (pos < 0) continue;
      while (pos > 0 && s_cnt[top[pos - 1]] < c) {
        if (pos < BS_HOT) top[pos] = top[pos - 1];
        pos--;
      }
      top[pos] = slot;
      if (nt < BS_HOT) nt++;
    }
    o.hot_n = (unsigned)nt;
    for (int j = 0; j < nt; j++) o.hot[j] = s_key[top[j]];
  }
}

struct BatchFin {
  const DQuery* qs;
  const unsigned long long* slot_off;  // nq + 1 (global slot index of each query's first slot)
  const uint64_t* gcap;                // per query
  const unsigned long long* keys;
  const uint8_t* recs;
  int rec_bytes;
  int nq;
  int n_out;
  unsigned int* const* status;         // per query: 16 words
  unsigned long long* count;           // per query: groups written
  uint8_t* out_base;
  const unsigned long long* out_off;   // per query x output column x {data, validity}
  unsigned long long total_slots;
  const unsigned long long* chunk_off;  // nq + 1: first finalize chunk of each query
};

constexpr int FIN_NT = 256, FIN_PER = 8, FIN_CH = FIN_NT * FIN_PER;  // a finalize CTA's slots
constexpr int FIN_W = FIN_CH / 32 + 2;  // bitmap words a CTA's output rows can touch

__device__ __forceinline__ int find_query(const unsigned long long* off, int nq, unsigned long long g) {
  int lo = 0, hi = nq - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ void store_out(uint8_t* d, int bytes, unsigned long long p, uint64_t v) {
  switch (bytes) {
    case 0: break;
    case 1: d[p] = (uint8_t)v; break;
    case 2: reinterpret_cast<uint16_t*>(d)[p] = (uint16_t)v; break;
    case 4: reinterpret_cast<uint32_t*>(d)[p] = (uint32_t)v; break;
    default: reinterpret_cast<uint64_t*>(d)[p] = v; break;
  }
}

// One CTA per chunk of FIN_CH consecutive slots of one query (the extra slot of the EMPTY-bit key
// included). The occupied slots are compacted into a shared list in slot order (coalesced key
// reads, one ballot per 32 slots); after one atomic per CTA on the query's row count, every
// thread finalises list entries i, i + FIN_NT, ... into output rows base + i, so all lanes work
// and the output writes are coalesced. The validity bits (and Bool key data) are built in shared
// memory and merged into the output bitmaps with one atomic OR per word.
__global__ void __launch_bounds__(FIN_NT) k_batch_finalize(const __grid_constant__ BatchFin F) {
  __shared__ unsigned s_vb[PMB_MAX_OUT][FIN_W];
  __shared__ unsigned s_db[PMB_MAX_KEYS][FIN_W];
  __shared__ unsigned s_off[FIN_PER][FIN_NT / 32];
  __shared__ unsigned short s_list[FIN_CH];
  __shared__ unsigned long long s_base;
  __shared__ unsigned s_total;
  __shared__ __align__(16) unsigned char s_q[sizeof(DQuery)];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const unsigned long long c = blockIdx.x;
  const int qi = find_query(F.chunk_off, F.nq, c);
  // the query descriptor in shared memory: the per-row decoding reads it many times
  static_assert(sizeof(DQuery) % 4 == 0, "DQuery is copied in 4-byte words");
  for (int i = tid; i < (int)(sizeof(DQuery) / 4); i += FIN_NT)
    reinterpret_cast<unsigned*>(s_q)[i] = reinterpret_cast<const unsigned*>(F.qs + qi)[i];
  const DQuery& q = *reinterpret_cast<const DQuery*>(s_q);
  const uint64_t cap = F.gcap[qi];
  const unsigned long long g0 = F.slot_off[qi];
  const unsigned long long s0 = (c - F.chunk_off[qi]) * FIN_CH;
  const bool extra = F.status[qi][1] != 0u;  // a row had the key whose bits equal EMPTY
  const unsigned lt = (1u << lane) - 1u;
  unsigned bal[FIN_PER];
#pragma unroll
  for (int j = 0; j < FIN_PER; j++) {
    const unsigned long long s = s0 + (unsigned long long)j * FIN_NT + tid;
    bool o = false;
    if (s < cap) o = F.keys[g0 + s] != PMB_EMPTY64;
    else if (s == cap) o = extra;
    bal[j] = __ballot_sync(0xffffffffu, o);
    if (lane == 0) s_off[j][warp] = __popc(bal[j]);
  }
  for (int i = tid; i < PMB_MAX_OUT * FIN_W; i += FIN_NT) (&s_vb[0][0])[i] = 0u;
  for (int i = tid; i < PMB_MAX_KEYS * FIN_W; i += FIN_NT) (&s_db[0][0])[i] = 0u;
  __syncthreads();
  if (tid == 0) {
    unsigned acc = 0;
    for (int j = 0; j < FIN_PER; j++)
      for (int w = 0; w < FIN_NT / 32; w++) {
        const unsigned v = s_off[j][w];
        s_off[j][w] = acc;
        acc += v;
      }
    s_total = acc;
    s_base = acc ? atomicAdd(&F.count[qi], (unsigned long long)acc) : 0ULL;
  }
  __syncthreads();
  const unsigned total = s_total;
  if (total == 0) return;  // the whole CTA leaves together
#pragma unroll
  for (int j = 0; j < FIN_PER; j++)
    if ((bal[j] >> lane) & 1u) s_list[s_off[j][warp] + __popc(bal[j] & lt)] = (unsigned short)(j * FIN_NT + tid);
  __syncthreads();
  const unsigned long long base = s_base, a = base & ~31ULL;
  const unsigned long long* oo = F.out_off + (size_t)qi * F.n_out * 2;
  for (unsigned i = tid; i < total; i += FIN_NT) {
    const unsigned long long p = base + i;
    const unsigned long long g = g0 + s0 + s_list[i];
    const unsigned r = (unsigned)(p - a);  // bit of this row in the CTA's bitmaps
    const unsigned long long klo = F.keys[g];
    const uint8_t* rec = F.recs + g * (unsigned long long)F.rec_bytes;
    int oc = 0;
    for (int k = 0; k < q.n_keys; k++, oc++) {
      uint64_t v = 0;
      const bool valid = unpack_field(q.key[k], klo, 0ULL, v);
      const int dt = q.col[q.key[k].col].dtype;
      if (dt == PMB_BOOL) {
        if (valid && v) atomicOr(&s_db[k][r >> 5], 1u << (r & 31));
      } else {
        store_out(F.out_base + oo[2 * oc], pmb_dtype_bytes(dt), p, v);
      }
      if (valid) atomicOr(&s_vb[oc][r >> 5], 1u << (r & 31));
    }
    for (int ag = 0; ag < q.n_aggs; ag++, oc++) {
      const DAggOut& A = q.agg[ag];
      bool valid = true;
      uint64_t bits = 0;
      finalize_agg(q, A, rec, valid, bits);
      store_out(F.out_base + oo[2 * oc], pmb_dtype_bytes(A.out_dtype), p, bits);
      if (valid) atomicOr(&s_vb[oc][r >> 5], 1u << (r & 31));
    }
  }
  __syncthreads();
  const int nw = (int)((base - a + total + 31) / 32);
  for (int i = tid; i < F.n_out * nw; i += FIN_NT) {
    const int oc = i / nw, w = i % nw;
    const unsigned v = s_vb[oc][w];
    if (v) atomicOr(reinterpret_cast<unsigned*>(F.out_base + oo[2 * oc + 1]) + (a >> 5) + w, v);
    if (oc < q.n_keys && q.col[q.key[oc].col].dtype == PMB_BOOL) {
      const unsigned d = s_db[oc][w];
      if (d) atomicOr(reinterpret_cast<unsigned*>(F.out_base + oo[2 * oc]) + (a >> 5) + w, d);
    }
  }
}

// signature of a compiled query: everything the run-time kernel's source depends on
std::string signature(const DQuery& q) {
  std::string s;
  auto put = [&](const void* p, size_t n) { s.append(reinterpret_cast<const char*>(p), n); };
  put(&q.n_cols, 4);
  put(&q.n_keys, 4);
  put(&q.n_fields, 4);
  put(&q.n_aggs, 4);
  put(&q.key_bits, 4);
  put(&q.rec_bytes, 4);
  for (int c = 0; c < q.n_cols; c++) {
    put(&q.col[c].dtype, sizeof(q.col[c].dtype));
    put(&q.col[c].elem, sizeof(q.col[c].elem));
    s.push_back(q.col[c].valid ? 1 : 0);
  }
  put(q.key, sizeof(DKey) * q.n_keys);
  for (int f = 0; f < q.n_fields; f++) {
    DField F = q.field[f];
    F.fx = 0;  // the fraction bits are per query (kernel parameter)
    put(&F, sizeof(F));
  }
  put(q.agg, sizeof(DAggOut) * q.n_aggs);
  put(&q.prog, sizeof(q.prog));
  return s;
}

struct TuneChoice {
  int nt = 1024;
  int item_units = 256;
  int nbuf = 2;       // unit buffers per warp
  int warm_rule = 1;  // 0: every query fills a warm table; 1: only queries whose groups fit it, or
                      // whose items hold at least as many rows as the query has groups
  int warm_max = 0;   // shared-table capacity: CTA warm-table slots at most (0: the largest that fits);
                      // a smaller table is cheaper to reset at every work item
  int gslots_x2 = 5;  // global-table capacity: 2 x slots per estimated group (5 = 2.5 slots)
};
std::mutex g_tune_mu;
std::map<std::string, TuneChoice> g_tuned;  // signature + size class -> choice

struct GraphCache {
  std::string key;
  cudaGraphExec_t exec = nullptr;
};
std::mutex g_graph_mu;
std::map<const pmb_handle*, GraphCache> g_graphs;

}  // namespace

// One round of the batched path over `qidx`; fills results and returns the queries that must run
// again (overflow / float-sum range) in `again`.
static int batch_round(pmb_handle* h, std::vector<CompiledQuery>& cqs, const std::vector<int>& qidx,
                       const std::vector<int64_t>& est, const std::vector<BatchSketch>& sk, const TuneChoice& tc,
                       bool tuning, pmb_result** outs, std::vector<int>* again, float* agg_ms) {
  const int nq = (int)qidx.size();
  const CompiledQuery& c0 = cqs[qidx[0]];
  const int rec = c0.dq.rec_bytes;
  JitPlan J;
  int rc = pmb_plan_jit_batch(h, c0, tc.nt, tc.nbuf, h->max_smem_optin, &J, tc.warm_max);
  if (rc) return rc;
  cudaKernel_t k = nullptr;
  rc = pmb_jit_batch_kernel(h, c0, J, &k);
  if (rc) return rc;
  // table arena: per query cap + 1 slots rounded up to 4 (4-slot buckets stay 32-byte aligned)
  std::vector<unsigned long long> slot_off(nq + 1, 0);
  std::vector<uint64_t> cap(nq);
  for (int i = 0; i < nq; i++) {
    const CompiledQuery& cq = cqs[qidx[i]];
    uint64_t c = (uint64_t)std::max<int64_t>(est[qidx[i]] * tc.gslots_x2 / 2, 1024);  // tuned slots per group
    if (const char* e = getenv("PMB_GCAP_MULT")) {  // tuning override, as for single queries
      const double k = atof(e);
      if (k > 0) c = (uint64_t)std::max(1024.0, (double)c * k);
    }
    c = std::min<uint64_t>(c, (uint64_t)std::max<int64_t>(2 * cq.dq.n_rows, 1024));
    c = (c + 3) & ~3ULL;
    cap[i] = c;
    slot_off[i + 1] = slot_off[i] + ((c + 1 + 3) & ~3ULL);
  }
  const unsigned long long total = slot_off[nq];
  unsigned long long* keys = (unsigned long long*)pmb_ws_alloc(h, (size_t)total * 8);
  uint8_t* recs = (uint8_t*)pmb_ws_alloc(h, (size_t)total * rec);
  unsigned int* status = (unsigned int*)pmb_ws_alloc(h, (size_t)nq * 64);
  unsigned long long* hot = (unsigned long long*)pmb_ws_alloc(h, (size_t)nq * (BS_HOT * 8 + 8));
  if (!keys || !recs || !status || !hot) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (batch tables)");
  // per query parameters of the run-time kernel
  std::vector<JitParams> jp(nq);
  std::vector<unsigned long long> hot_h((size_t)nq * (BS_HOT + 1), 0);
  std::vector<JBatchItemH> items;
  for (int i = 0; i < nq; i++) {
    const CompiledQuery& cq = cqs[qidx[i]];
    const BatchSketch& s = sk[qidx[i]];
    JitParams& A = jp[i];
    memset(&A, 0, sizeof(A));
    for (int c = 0; c < cq.dq.n_cols; c++) {
      A.col_data[c] = cq.dq.col[c].data;
      A.col_valid[c] = cq.dq.col[c].valid;
    }
    A.n_rows = cq.dq.n_rows;
    A.n_units = (cq.dq.n_rows + 127) / 128;
    A.gprobe = (int)std::min<unsigned long long>(cap[i] / 4, 256);
    A.occ_limit = 0xFFFFFFFFu;
    A.gkeys = keys + slot_off[i];
    A.grecs = recs + slot_off[i] * (unsigned long long)rec;
    A.gcap = cap[i];
    A.status = status + 16 * i;
    unsigned long long* hb = hot_h.data() + (size_t)i * (BS_HOT + 1);
    const unsigned nh = std::min<unsigned>(s.hot_n, (unsigned)J.hot_cap);
    for (unsigned j = 0; j < nh; j++) hb[j] = s.hot[j];
    reinterpret_cast<unsigned int*>(hb + BS_HOT)[0] = nh;
    A.hot_keys = nh ? hot + (size_t)i * (BS_HOT + 1) : nullptr;
    A.hot_n = reinterpret_cast<const unsigned int*>(hot + (size_t)i * (BS_HOT + 1) + BS_HOT);
    for (int f = 0; f < cq.dq.n_fields; f++)
      if (cq.dq.field[f].kind == F_SUM_FX) {
        A.fx[cq.dq.field[f].fx_slot] = cq.dq.field[f].fx;
        A.fx_e[cq.dq.field[f].fx_slot] = cq.dq.fx_e[cq.dq.field[f].fx_slot];
      }
    const int64_t g = std::max<int64_t>(est[qidx[i]], 1);
    A.flags = (tc.warm_rule == 0 || g <= 2LL * J.warm_cap || (int64_t)tc.item_units * 128 >= g) ? 1 : 0;
    for (long long u0 = 0; u0 < A.n_units; u0 += tc.item_units)
      items.push_back({i, 0, u0, std::min<long long>(A.n_units, u0 + tc.item_units)});
  }
  JitParams* d_jp = (JitParams*)pmb_ws_alloc(h, sizeof(JitParams) * nq);
  JBatchItemH* d_items = (JBatchItemH*)pmb_ws_alloc(h, sizeof(JBatchItemH) * std::max<size_t>(items.size(), 1));
  unsigned long long* ctr = (unsigned long long*)pmb_ws_alloc(h, 8 * ((size_t)nq + 1));  // ticket, counts
  DQuery* d_qs = (DQuery*)pmb_ws_alloc(h, sizeof(DQuery) * nq);
  unsigned long long* d_soff = (unsigned long long*)pmb_ws_alloc(h, 8 * ((size_t)nq + 1));
  uint64_t* d_cap = (uint64_t*)pmb_ws_alloc(h, 8 * (size_t)nq);
  unsigned int** d_st = (unsigned int**)pmb_ws_alloc(h, sizeof(void*) * nq);
  unsigned long long* d_coff = (unsigned long long*)pmb_ws_alloc(h, 8 * ((size_t)nq + 1));
  if (!d_jp || !d_items || !ctr || !d_qs || !d_soff || !d_cap || !d_st || !d_coff)
    return pmb_fail(h, PMB_E_OOM, "workspace exhausted (batch plan)");
  // outputs: per query and output column a data block and a validity bitmap (sized by capacity)
  const int n_out = c0.dq.n_keys + c0.dq.n_aggs;
  std::vector<int> out_dt(n_out);
  for (int k2 = 0; k2 < c0.dq.n_keys; k2++) out_dt[k2] = c0.dq.col[c0.dq.key[k2].col].dtype;
  for (int a = 0; a < c0.dq.n_aggs; a++) out_dt[c0.dq.n_keys + a] = c0.dq.agg[a].out_dtype;
  // data blocks first, then every bitmap (validity and Bool data) in one region that is zeroed
  std::vector<unsigned long long> out_off((size_t)nq * n_out * 2);
  unsigned long long ob = 0;
  for (int i = 0; i < nq; i++)
    for (int c = 0; c < n_out; c++) {
      if (out_dt[c] == PMB_BOOL) continue;
      out_off[((size_t)i * n_out + c) * 2] = ob;
      ob += ((cap[i] + 1) * (unsigned long long)pmb_dtype_bytes(out_dt[c]) + 15) & ~15ULL;
    }
  const unsigned long long bits_start = ob;
  for (int i = 0; i < nq; i++)
    for (int c = 0; c < n_out; c++) {
      const unsigned long long vb = (((cap[i] + 1 + 31) / 32) * 4 + 15) & ~15ULL;
      if (out_dt[c] == PMB_BOOL) {
        out_off[((size_t)i * n_out + c) * 2] = ob;
        ob += vb;
      }
      out_off[((size_t)i * n_out + c) * 2 + 1] = ob;
      ob += vb;
    }
  uint8_t* out_base = (uint8_t*)pmb_ws_alloc(h, (size_t)ob + 16);
  unsigned long long* d_ooff = (unsigned long long*)pmb_ws_alloc(h, 8 * out_off.size());
  if (!out_base || !d_ooff) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (batch outputs)");
  // the round's descriptors go up from the pinned staging area when it has room
  std::vector<DQuery> hq_own;
  DQuery* hq = (DQuery*)pmb_host_stage(h, sizeof(DQuery) * nq);
  if (!hq) {
    hq_own.resize(nq);
    hq = hq_own.data();
  }
  std::vector<unsigned int*> hst(nq);
  for (int i = 0; i < nq; i++) {
    hq[i] = cqs[qidx[i]].dq;
    hst[i] = status + 16 * i;
  }
  auto upload = [&](void* dst, const void* src, size_t bytes) -> cudaError_t {
    if (void* st = pmb_host_stage(h, bytes)) {
      memcpy(st, src, bytes);
      src = st;
    }
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->stream);
  };
  PMB_CUDA(h, upload(d_jp, jp.data(), sizeof(JitParams) * nq));
  PMB_CUDA(h, upload(d_items, items.data(), sizeof(JBatchItemH) * items.size()));
  PMB_CUDA(h, upload(hot, hot_h.data(), 8 * hot_h.size()));
  PMB_CUDA(h, cudaMemcpyAsync(d_qs, hq, sizeof(DQuery) * nq, cudaMemcpyHostToDevice, h->stream));
  PMB_CUDA(h, cudaMemcpyAsync(d_soff, slot_off.data(), 8 * slot_off.size(), cudaMemcpyHostToDevice, h->stream));
  PMB_CUDA(h, cudaMemcpyAsync(d_cap, cap.data(), 8 * cap.size(), cudaMemcpyHostToDevice, h->stream));
  PMB_CUDA(h, cudaMemcpyAsync(d_st, hst.data(), sizeof(void*) * nq, cudaMemcpyHostToDevice, h->stream));
  PMB_CUDA(h, cudaMemcpyAsync(d_ooff, out_off.data(), 8 * out_off.size(), cudaMemcpyHostToDevice, h->stream));
  std::vector<unsigned long long> chunk_off(nq + 1, 0);
  for (int i = 0; i < nq; i++) chunk_off[i + 1] = chunk_off[i] + (cap[i] + 1 + FIN_CH - 1) / FIN_CH;
  PMB_CUDA(h, cudaMemcpyAsync(d_coff, chunk_off.data(), 8 * chunk_off.size(), cudaMemcpyHostToDevice, h->stream));
  // record identity (every query of the round has the same record layout)
  RecInit ri;
  memset(&ri, 0, sizeof(ri));
  for (size_t w = 0; w < c0.rec_init.size() && w < 48; w++) ri.w[w] = c0.rec_init[w];
  JBatchH B{d_jp, d_items, (long long)items.size(), ctr};
  BatchFin F;
  F.qs = d_qs;
  F.slot_off = d_soff;
  F.gcap = d_cap;
  F.keys = keys;
  F.recs = recs;
  F.rec_bytes = rec;
  F.nq = nq;
  F.n_out = n_out;
  F.status = d_st;
  F.count = ctr + 1;
  F.out_base = out_base;
  F.out_off = d_ooff;
  F.total_slots = total;
  F.chunk_off = d_coff;
  PMB_CUDA(h, cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize, J.smem));
  const int init_blocks = (int)std::max<int64_t>(1, std::min<int64_t>(((int64_t)total * std::max(1, rec / 8) + 255) / 256,
                                                                      (int64_t)h->sm_count * 16));
  const int fin_blocks = (int)chunk_off[nq];
  // the device work of the round: one graph, replayed while the launch shape is the same; with
  // profiling on it runs eagerly with an event pair around each kernel
  auto enqueue = [&](cudaStream_t s, bool prof, cudaEvent_t a0, cudaEvent_t a1) -> cudaError_t {
    cudaError_t e;
    if ((e = cudaMemsetAsync(status, 0, (size_t)nq * 64, s))) return e;
    if ((e = cudaMemsetAsync(ctr, 0, 8 * ((size_t)nq + 1), s))) return e;
    if ((e = cudaMemsetAsync(out_base + bits_start, 0, (size_t)(ob - bits_start), s))) return e;
    if (prof) pmb_kernel_begin(h, "batch_table_init");
    k_table_init_pub(keys, (int64_t)total, (uint64_t*)recs, (int64_t)total, rec / 8, ri, init_blocks, s);
    if (prof) pmb_kernel_end(h);
    if (a0 && (e = cudaEventRecord(a0, s))) return e;
    if (prof) pmb_kernel_begin(h, "batch_agg");
    void* args[] = {&B};
    if ((e = cudaLaunchKernel((const void*)k, dim3(h->sm_count), dim3(J.nt), args, (size_t)J.smem, s))) return e;
    if (prof) pmb_kernel_end(h);
    if (a1 && (e = cudaEventRecord(a1, s))) return e;
    if (prof) pmb_kernel_begin(h, "batch_finalize");
    k_batch_finalize<<<fin_blocks, FIN_NT, 0, s>>>(F);
    if (prof) pmb_kernel_end(h);
    return cudaGetLastError();
  };
  if (tuning) {
    cudaEvent_t a0, a1;
    PMB_CUDA(h, cudaEventCreate(&a0));
    PMB_CUDA(h, cudaEventCreate(&a1));
    cudaError_t e = enqueue(h->stream, false, a0, a1);
    if (e == cudaSuccess) e = cudaEventSynchronize(a1);
    float ms = 0;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, a0, a1);
    cudaEventDestroy(a0);
    cudaEventDestroy(a1);
    PMB_CUDA(h, e);
    if (agg_ms) *agg_ms = ms;
  } else if (h->profiling) {
    PMB_CUDA(h, enqueue(h->stream, true, nullptr, nullptr));
  } else {
    // graph key: everything the captured launches read
    std::string key;
    auto put = [&](const void* p, size_t n) { key.append(reinterpret_cast<const char*>(p), n); };
    put(&k, sizeof(k));
    put(&B, sizeof(B));
    put(&F, sizeof(F));
    put(&J.smem, 4);
    put(&J.nt, 4);
    put(&ob, 8);
    put(&init_blocks, 4);
    put(&fin_blocks, 4);
    std::lock_guard<std::mutex> lock(g_graph_mu);
    GraphCache& gc = g_graphs[h];
    if (gc.key != key || !gc.exec) {
      if (gc.exec) cudaGraphExecDestroy(gc.exec);
      gc.exec = nullptr;
      gc.key.clear();
      cudaGraph_t g;
      PMB_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
      cudaError_t e = enqueue(h->stream, false, nullptr, nullptr);
      cudaError_t e2 = cudaStreamEndCapture(h->stream, &g);
      PMB_CUDA(h, e);
      PMB_CUDA(h, e2);
      e = cudaGraphInstantiate(&gc.exec, g, 0);
      cudaGraphDestroy(g);
      PMB_CUDA(h, e);
      gc.key = key;
    }
    h->launches += 3;  // table init, aggregation, finalize
    PMB_CUDA(h, cudaGraphLaunch(gc.exec, h->stream));
  }
  // group counts and status words of every query
  std::vector<unsigned long long> cnt(nq + 1);
  std::vector<unsigned int> sth((size_t)nq * 16);
  PMB_CUDA(h, cudaMemcpyAsync(cnt.data(), ctr, 8 * ((size_t)nq + 1), cudaMemcpyDeviceToHost, h->stream));
  PMB_CUDA(h, cudaMemcpyAsync(sth.data(), status, 64 * (size_t)nq, cudaMemcpyDeviceToHost, h->stream));
  PMB_CUDA(h, cudaStreamSynchronize(h->stream));
  for (int i = 0; i < nq; i++) {
    const unsigned st = sth[(size_t)i * 16];
    if (st & PMB_ST_TIMEOUT) return pmb_fail(h, PMB_E_TIMEOUT, "a bounded device wait timed out (batch)");
    const int qi = qidx[i];
    if (st & (PMB_ST_OVERFLOW | PMB_ST_FXRANGE)) {
      if (again) again->push_back(qi);
      if (st & PMB_ST_FXRANGE) {
        DQuery& q = cqs[qi].dq;
        for (int f = 0; f < q.n_fields; f++) {
          DField& fd = q.field[f];
          const unsigned ex = sth[(size_t)i * 16 + 4 + fd.fx_slot];
          if (fd.kind != F_SUM_FX || ex == 0) continue;
          const int e = (int)ex - 1022 + 1;
          if (e > q.fx_e[fd.fx_slot]) {
            fd.fx = (int16_t)(fd.fx - (e - q.fx_e[fd.fx_slot]));
            q.fx_e[fd.fx_slot] = (int16_t)e;
          }
        }
      }
      continue;
    }
    if (tuning) continue;
    pmb_result* r = outs[qi];
    r->n_groups = (int64_t)cnt[1 + i];
    r->capacity = (int64_t)cap[i];
    r->strategy_used = PMB_STRATEGY_GLOBAL_HASH;
    for (int c = 0; c < n_out; c++) {
      r->columns[c].data = out_base + out_off[((size_t)i * n_out + c) * 2];
      r->columns[c].validity = out_base + out_off[((size_t)i * n_out + c) * 2 + 1];
    }
  }
  return PMB_OK;
}

extern "C" int pmb_groupby_batched(pmb_handle* h, const pmb_query* qs, const pmb_column* const* cols,
                                   const int32_t* n_cols, int32_t n_queries, pmb_result** outs) {
  if (!h) return PMB_E_INVALID;
  if (n_queries < 0 || (n_queries > 0 && (!qs || !cols || !n_cols || !outs)))
    return pmb_fail(h, PMB_E_INVALID, "bad batch arguments");
  for (int i = 0; i < n_queries; i++) outs[i] = nullptr;
  if (n_queries == 0) return PMB_OK;
  PMB_CUDA(h, cudaSetDevice(h->device));
  auto fail_all = [&](int rc) {
    for (int i = 0; i < n_queries; i++) {
      pmb_result_free(outs[i]);
      outs[i] = nullptr;
    }
    return rc;
  };
  // host phase timing (PMB_BATCH_TIMING=1 prints it)
  const bool timing = getenv("PMB_BATCH_TIMING") != nullptr;
  auto now = [] { return std::chrono::steady_clock::now(); };
  auto t_prev = now();
  auto phase = [&](const char* name) {
    if (!timing) return;
    const auto t = now();
    fprintf(stderr, "batch %-12s %8.2f ms\n", name, std::chrono::duration<double, std::milli>(t - t_prev).count());
    t_prev = t;
  };
  // compile every query; the batched path takes the queries of query 0's signature
  std::vector<CompiledQuery> cqs(n_queries);
  for (int i = 0; i < n_queries; i++) {
    int rc = pmb_compile_groupby(h, &qs[i], cols[i], n_cols[i], &cqs[i]);
    if (rc) return fail_all(rc);
  }
  phase("compile");
  const std::string sig0 = signature(cqs[0].dq);
  std::vector<int> batch, single;
  for (int i = 0; i < n_queries; i++) {
    const bool ok = cqs[i].dq.key_bits <= 64 && cqs[i].dq.n_rows > 0 && signature(cqs[i].dq) == sig0 &&
                    qs[i].strategy == PMB_STRATEGY_AUTO && qs[i].capacity_hint <= 0 && pmb_jit_enabled(1LL << 40);
    (ok ? batch : single).push_back(i);
  }
  int rc = PMB_OK;
  if (!h->batching || batch.size() < 2 || batch.size() != (size_t)n_queries) {
    // one by one: every call resets the handle's workspace, so only host outputs survive
    for (int i = 0; i < n_queries; i++)
      if (qs[i].output_on_device)
        return fail_all(pmb_fail(h, PMB_E_UNSUPPORTED,
                                 "device outputs need a batch of at least two queries of one signature"));
    for (int i = 0; i < n_queries; i++) {
      rc = pmb_groupby(h, &qs[i], cols[i], n_cols[i], &outs[i]);
      if (rc) return fail_all(rc);
    }
    return PMB_OK;
  }
  {
    rc = pmb_ws_begin(h);
    if (rc) return fail_all(rc);
    pmb_call_begin(h);
    for (int i : batch) {
      outs[i] = pmb_result_new(cqs[i].dq.n_keys + cqs[i].dq.n_aggs);
      if (!outs[i]) return fail_all(pmb_fail(h, PMB_E_OOM, "host allocation failed"));
      const DQuery& q = cqs[i].dq;
      int oc = 0;
      for (int k = 0; k < q.n_keys; k++, oc++) outs[i]->columns[oc].dtype = q.col[q.key[k].col].dtype;
      for (int a = 0; a < q.n_aggs; a++, oc++) outs[i]->columns[oc].dtype = q.agg[a].out_dtype;
      for (int c = 0; c < q.n_cols; c++) {
        rc = pmb_stage_column(h, cols[i][cqs[i].map.user[c]], q.n_rows, &cqs[i].dq.col[c]);
        if (rc) return fail_all(rc);
      }
    }
    const int nb = (int)batch.size();
    phase("stage");
    // 1. per-query sample
    DQuery* d_all = (DQuery*)pmb_ws_alloc(h, sizeof(DQuery) * n_queries);
    BatchSketch* d_sk = (BatchSketch*)pmb_ws_alloc(h, sizeof(BatchSketch) * n_queries);
    if (!d_all || !d_sk) return fail_all(pmb_fail(h, PMB_E_OOM, "workspace exhausted (batch sketch)"));
    std::vector<DQuery> hb_own;
    DQuery* hb = (DQuery*)pmb_host_stage(h, sizeof(DQuery) * nb);
    if (!hb) {
      hb_own.resize(nb);
      hb = hb_own.data();
    }
    for (int j = 0; j < nb; j++) hb[j] = cqs[batch[j]].dq;
    PMB_CUDA(h, cudaMemcpyAsync(d_all, hb, sizeof(DQuery) * nb, cudaMemcpyHostToDevice, h->stream));
    FxColsB fxc;
    memset(&fxc, 0, sizeof(fxc));
    fxc.n = (int)cqs[batch[0]].fx_cols.size();
    for (int f = 0; f < fxc.n; f++) fxc.col[f] = cqs[batch[0]].fx_cols[f];
    const int sk_smem = BS_SLOTS * 12 + 1024 * 4;
    PMB_CUDA(h, cudaFuncSetAttribute(k_batch_sketch, cudaFuncAttributeMaxDynamicSharedMemorySize, sk_smem));
    pmb_kernel_begin(h, "batch_sketch");
    k_batch_sketch<<<nb, BS_NT, sk_smem, h->stream>>>(d_all, d_sk, fxc);
    pmb_kernel_end(h);
    PMB_CUDA(h, cudaGetLastError());
    // the selector's kernels go in before the sketch's readback, whose synchronisation serves both
    const float* sel_out = pmb_selector_batch_launch(h, d_all, nb);
    std::vector<BatchSketch> skb(nb);
    PMB_CUDA(h, cudaMemcpyAsync(skb.data(), d_sk, sizeof(BatchSketch) * nb, cudaMemcpyDeviceToHost, h->stream));
    PMB_CUDA(h, cudaStreamSynchronize(h->stream));
    phase("sketch");
    // 2. estimates (the selector's prediction can only enlarge them) and float-sum ranges
    std::vector<int64_t> nrows(nb), pred(nb, 0);
    for (int j = 0; j < nb; j++) nrows[j] = cqs[batch[j]].dq.n_rows;
    if (sel_out) pmb_selector_batch_groups(sel_out, nb, pred.data(), nrows.data());
    else pmb_selector_predict_batch(h, d_all, nb, pred.data(), nrows.data());
    std::vector<int64_t> est(n_queries, 0);
    std::vector<BatchSketch> sk(n_queries);
    int64_t total_rows = 0;
    for (int j = 0; j < nb; j++) {
      const int i = batch[j];
      sk[i] = skb[j];
      SketchOut so;
      memset(&so, 0, sizeof(so));
      so.samples = skb[j].kept;
      so.distinct = skb[j].distinct;
      so.singletons = skb[j].f1;
      const int64_t neff = skb[j].samples ? (int64_t)((double)cqs[i].dq.n_rows * skb[j].kept / skb[j].samples) : 0;
      est[i] = std::max<int64_t>(pmb_estimate_groups(so, std::max<int64_t>(neff, skb[j].kept)), pred[j]);
      int pbits = 2, tbits = 2;
      while ((1LL << pbits) < cqs[i].dq.n_rows / h->sm_count + 1) pbits++;
      while ((1LL << tbits) < cqs[i].dq.n_rows + 1) tbits++;
      pmb_set_fx(cqs[i].dq, skb[j].fx_expo, 3, pbits + 1, tbits + 1);
      total_rows += cqs[i].dq.n_rows;
    }
    if (timing) {
      int64_t e_sum = 0, p_sum = 0;
      for (int j = 0; j < nb; j++) e_sum += est[batch[j]], p_sum += pred[j];
      fprintf(stderr, "batch estimates: %lld groups in total (selector predictions %lld)\n", (long long)e_sum,
              (long long)p_sum);
    }
    phase("estimates");
    // 3. autotune (first batch of a signature and size class), then the round itself
    int size_class = 0;
    while ((1LL << size_class) < total_rows) size_class++;
    const std::string tkey = sig0 + "#" + std::to_string(size_class) + "#" + std::to_string(nb > 256 ? 1 : 0);
    TuneChoice tc;
    bool have = false;
    {
      std::lock_guard<std::mutex> lock(g_tune_mu);
      auto it = g_tuned.find(tkey);
      if (it != g_tuned.end()) {
        tc = it->second;
        have = true;
      }
    }
    if (!have && !getenv("PMB_NO_AUTOTUNE")) {
      // block size, work-item size (rows of a query per item), unit buffers per warp, warm rule,
      // shared-table capacity (warm slots) and global-table capacity (slots per estimated group);
      // the reference fixes the counterparts (16 partitions, groupby.rs:533; 1024 threadgroup
      // slots, groupby_build_partitioned_build.metal:36-37)
      static const TuneChoice cands[] = {
          {1024, 256, 1, 0, 0, 5},    {1024, 256, 2, 0, 0, 5},    {1024, 256, 2, 1, 0, 5},    {1024, 64, 2, 1, 0, 5},
          {1024, 1024, 2, 1, 0, 5},   {512, 256, 2, 1, 0, 5},     {512, 1024, 2, 1, 0, 5},    {1024, 256, 2, 1, 4096, 5},
          {1024, 256, 2, 1, 1024, 5}, {1024, 256, 2, 1, 0, 3},    {1024, 256, 2, 1, 0, 8}};
      float best = 1e30f;
      for (const TuneChoice& c : cands) {
        float ms = 0;
        const WsMark mark = pmb_ws_mark(h);  // a trial's tables and outputs are given back after it
        rc = batch_round(h, cqs, batch, est, sk, c, true, outs, nullptr, &ms);
        if (rc) return fail_all(rc);
        pmb_ws_release(h, mark);
        if (timing)
          fprintf(stderr, "batch tuning candidate %d threads / %d units / %d buffers / warm rule %d / warm max %d / "
                  "slots x2 %d: %.3f ms\n", c.nt, c.item_units, c.nbuf, c.warm_rule, c.warm_max, c.gslots_x2, ms);
        if (ms < best) {
          best = ms;
          tc = c;
        }
      }
      std::lock_guard<std::mutex> lock(g_tune_mu);
      g_tuned[tkey] = tc;
    }
    if (timing)
      fprintf(stderr, "batch tuning: %d threads, %d units per item, %d buffers, warm rule %d, warm max %d, slots x2 %d\n",
              tc.nt, tc.item_units, tc.nbuf, tc.warm_rule, tc.warm_max, tc.gslots_x2);
    // 4. the rounds: queries grouped by record layout (a query whose float sums would have too few
    //    fraction bits sums them in double-double: another layout); queries that overflowed (3x
    //    table) or left their float-sum range (already widened) run again
    auto to_dd = [&](int i) -> int {
      CompiledQuery& cq = cqs[i];
      bool dd = false;
      for (int f = 0; f < cq.dq.n_fields; f++)
        dd |= cq.dq.field[f].kind == F_SUM_FX && cq.dq.field[f].fx < PMB_FX_MIN_F;
      if (!dd) return PMB_OK;
      for (int f = 0; f < cq.dq.n_fields; f++)
        if (cq.dq.field[f].kind == F_SUM_FX) cq.dd_user_cols.push_back(cq.map.user[cq.dq.field[f].col]);
      return recompile_dd(h, &qs[i], cols[i], n_cols[i], cq);
    };
    phase("autotune");
    std::vector<int> again = batch;
    for (int round = 0; !again.empty() && round < 7; round++) {
      std::map<std::string, std::vector<int>> groups;
      for (int i : again) {
        if (round > 0) est[i] = std::max<int64_t>(est[i] * 3, 1024);
        rc = to_dd(i);
        if (rc) return fail_all(rc);
        groups[signature(cqs[i].dq)].push_back(i);
      }
      std::vector<int> next;
      for (auto& g : groups) {
        rc = batch_round(h, cqs, g.second, est, sk, tc, false, outs, &next, nullptr);
        if (rc) return fail_all(rc);
        if (timing) {
          int64_t rows = 0, e = 0;
          for (int i : g.second) rows += cqs[i].dq.n_rows, e += est[i];
          fprintf(stderr, "batch round %d: %zu queries, %lld rows, %lld estimated groups, %zu to run again\n", round,
                  g.second.size(), (long long)rows, (long long)e, next.size());
        }
      }
      again.swap(next);
    }
    phase("rounds");
    if (!again.empty()) return fail_all(pmb_fail(h, PMB_E_OOM, "batched group-by did not converge"));
    for (int i : batch) {
      rc = pmb_finish_outputs(h, outs[i], qs[i].output_on_device == 0);
      if (rc) return fail_all(rc);
    }
    PMB_CUDA(h, cudaStreamSynchronize(h->stream));
    pmb_call_end(h);
    phase("outputs");
  }
  return PMB_OK;
}
