// pmb_filter.cu — the filter-side operator surface: null-aware compares, Kleene AND/OR,
// stream compaction and the u8 -> u32 prefix sum.
//
// Replaces: cmp_{i64,f64}_* (shaders/cmp_i64.metal:30-85, shaders/cmp_f64.metal:36-180,
// crates/polars-metal-kernels/src/cmp.rs:180-641), bool_and/bool_or
// (shaders/logical_bool.metal:45-125), the 3-pass compaction filter_predicate_to_u8 -> MLX
// cumsum -> filter_scatter_* (shaders/filter_predicate.metal:24-40,
// crates/polars-metal-mlx-sys/cxx/mlx_bridge.cc:59-89, shaders/filter_scatter.metal:52-185,
// crates/polars-metal-kernels/src/pipeline.rs:103-270).
//
// B200 design: predicate bits come from warp ballots (32 rows -> one 32-bit word, no atomics);
// compaction is one pass per column with a decoupled look-back over tiles (Merrill & Garland
// 2016), so there is no materialised keep array, no separate scan kernel and no host round trip.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>

#include "pmb_jit.h"
#include "pmb_plan.h"

namespace {

__host__ __device__ inline int64_t out_min_bytes(int64_t n) {
  int64_t raw = (n + 7) / 8;
  int64_t padded = (raw + 3) & ~3LL;
  return padded < 4 ? 4 : padded;
}

// ----------------------------------------------------------------- predicate -> bitmaps
// One thread per row; each warp writes whole 32-bit words of the (data, validity) outputs.
__global__ void k_pred_bits(const __grid_constant__ DQuery q, unsigned int* __restrict__ out_data,
                            unsigned int* __restrict__ out_valid) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t n_pad = (q.n_rows + 31) / 32 * 32;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n_pad; r += stride) {
    bool valid = false, truth = false;
    if (r < q.n_rows) {
      TileCtx t{nullptr, nullptr, nullptr, 0};
      eval_pred_tf(q, t, r, valid, truth);
    }
    unsigned bv = __ballot_sync(0xffffffffu, valid);
    unsigned bd = __ballot_sync(0xffffffffu, valid && truth);
    if ((threadIdx.x & 31) == 0) {
      out_valid[r >> 5] = bv;
      out_data[r >> 5] = bd;
    }
  }
}

// Kleene logic on bit-packed words (logical_bool.metal truth tables)
__global__ void k_bool_logic(int op, const uint8_t* __restrict__ ld, const uint8_t* __restrict__ lv,
                             const uint8_t* __restrict__ rd, const uint8_t* __restrict__ rv, int64_t n,
                             uint8_t* __restrict__ od, uint8_t* __restrict__ ov) {
  int64_t nb = (n + 7) / 8;
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += stride) {
    unsigned at = ld[b], av = lv[b], bt = rd[b], bv = rv[b];
    at &= av;  // data bits only count where valid
    bt &= bv;
    unsigned af = av & ~at, bf = bv & ~bt;
    unsigned t, f;
    if (op == 0) {
      t = at & bt;
      f = af | bf;
    } else {
      t = at | bt;
      f = af & bf;
    }
    unsigned v = t | f;
    int64_t rem = n - b * 8;
    if (rem < 8) {
      unsigned m = (1u << rem) - 1u;
      v &= m;
      t &= m;
    }
    od[b] = (uint8_t)t;
    ov[b] = (uint8_t)v;
  }
}

// ----------------------------------------------------------------- compaction
// Each tile of TILE rows: keep bits (predicate or bitmap) -> per-warp ballots -> block scan ->
// decoupled look-back for the tile's output base -> scatter values of every column. Output
// validity bits are OR-ed into 32-bit words (a warp's outputs span at most two words).
constexpr int CT_NT = 256;
constexpr int CT_PER = 8;  // rows per thread per tile
constexpr int CT_TILE = CT_NT * CT_PER;

struct CompactParams {
  DQuery q;                     // columns (and predicate when keep_data == nullptr)
  const uint8_t* keep_data;     // bit-packed predicate data or nullptr
  const uint8_t* keep_valid;    // bit-packed predicate validity or nullptr
  unsigned long long* lb;       // look-back states (one per tile)
  unsigned long long* ticket;
  unsigned long long* n_out;
  unsigned int* status;
  int32_t n_out_cols;           // leading columns that are outputs (the rest feed the predicate)
  uint8_t* out_data[PMB_MAX_COLS];
  unsigned int* out_valid[PMB_MAX_COLS];
};

__device__ __forceinline__ void set_bits_two_words(unsigned int* words, int64_t p, int64_t p_first, bool bit) {
  const int64_t w0 = p_first >> 5;
  unsigned m0 = __reduce_or_sync(0xffffffffu, (bit && (p >> 5) == w0) ? (1u << (p & 31)) : 0u);
  unsigned m1 = __reduce_or_sync(0xffffffffu, (bit && (p >> 5) == w0 + 1) ? (1u << (p & 31)) : 0u);
  if ((threadIdx.x & 31) == 0) {
    if (m0) atomicOr(&words[w0], m0);
    if (m1) atomicOr(&words[w0 + 1], m1);
  }
}

__global__ void __launch_bounds__(CT_NT) k_compact(const __grid_constant__ CompactParams P) {
  __shared__ int s_cnt[CT_PER][CT_NT / 32];
  __shared__ int s_off[CT_PER][CT_NT / 32];
  __shared__ long long s_tile;
  __shared__ unsigned long long s_base;
  const DQuery& q = P.q;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_tile = (long long)atomicAdd(P.ticket, 1ULL);
  __syncthreads();
  const long long tile = s_tile;
  const int64_t row0 = tile * CT_TILE;
  TileCtx t{nullptr, nullptr, nullptr, 0};
  bool keep[CT_PER];
  for (int j = 0; j < CT_PER; j++) {
    int64_t r = row0 + (int64_t)j * CT_NT + tid;
    bool k = false;
    if (r < q.n_rows) {
      if (P.keep_data) {
        k = ((P.keep_data[r >> 3] >> (r & 7)) & 1) && (!P.keep_valid || ((P.keep_valid[r >> 3] >> (r & 7)) & 1));
      } else {
        k = eval_keep(q, t, r);
      }
    }
    keep[j] = k;
    unsigned b = __ballot_sync(0xffffffffu, k);
    if (lane == 0) s_cnt[j][warp] = __popc(b);
  }
  __syncthreads();
  if (warp == 0) {
    int acc = 0;
    if (lane == 0) {
      for (int j = 0; j < CT_PER; j++)
        for (int w = 0; w < CT_NT / 32; w++) {
          s_off[j][w] = acc;
          acc += s_cnt[j][w];
        }
    }
    acc = __shfl_sync(0xffffffffu, acc, 0);
    const unsigned long long base = pmb_lookback_warp(P.lb, tile, (unsigned long long)acc, P.status);
    if (lane == 0) {
      s_base = base;
      if (tile == (long long)gridDim.x - 1) *P.n_out = base + acc;
    }
  }
  __syncthreads();
  const unsigned long long base = s_base;
  for (int j = 0; j < CT_PER; j++) {
    unsigned b = __ballot_sync(0xffffffffu, keep[j]);
    if (b == 0) continue;
    int64_t r = row0 + (int64_t)j * CT_NT + tid;
    int64_t p_first = (int64_t)(base + s_off[j][warp]);
    int64_t p = p_first + __popc(b & ((1u << lane) - 1u));
    for (int c = 0; c < P.n_out_cols; c++) {
      const DCol& C = q.col[c];
      uint64_t v = keep[j] ? pmb_load_bits(C.data, C.elem, r) : 0;
      bool valid = keep[j] && pmb_valid_bit(C.valid, r);
      uint8_t* d = P.out_data[c];
      if (keep[j]) {
        switch (C.elem) {
          case 0: break;
          case 1: d[p] = (uint8_t)v; break;
          case 2: reinterpret_cast<uint16_t*>(d)[p] = (uint16_t)v; break;
          case 4: reinterpret_cast<uint32_t*>(d)[p] = (uint32_t)v; break;
          default: reinterpret_cast<uint64_t*>(d)[p] = v; break;
        }
      }
      if (C.elem == 0) set_bits_two_words(reinterpret_cast<unsigned int*>(d), p, p_first, keep[j] && v);
      set_bits_two_words(P.out_valid[c], p, p_first, valid);
    }
  }
}

// ----------------------------------------------------------------- u8 -> u32 inclusive scan
constexpr int SC_NT = 512;  // 8192 rows per tile: one look-back per 8 KB of input
constexpr int SC_PER = 16;
constexpr int SC_TILE = SC_NT * SC_PER;

__global__ void __launch_bounds__(SC_NT) k_cumsum_u8(const uint8_t* __restrict__ in, uint32_t* __restrict__ out,
                                                     int64_t n, unsigned long long* lb, unsigned long long* ticket,
                                                     unsigned int* status) {
  __shared__ uint32_t s_warp[SC_NT / 32];
  __shared__ long long s_tile;
  __shared__ unsigned long long s_base;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_tile = (long long)atomicAdd(ticket, 1ULL);
  __syncthreads();
  const long long tile = s_tile;
  const int64_t r0 = tile * SC_TILE + (int64_t)tid * SC_PER;  // thread-contiguous rows
  uint32_t v[SC_PER];
  uint32_t sum = 0;
  // a whole run of 16 rows at a 16-byte aligned address: one 128-bit load (streaming: read once)
  const bool full = r0 + SC_PER <= n;
  if (full && ((reinterpret_cast<uintptr_t>(in) & 15u) == 0u)) {
    const uint4 w = __ldcs(reinterpret_cast<const uint4*>(in + r0));
    const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int j = 0; j < SC_PER; j++) {
      v[j] = (ws[j >> 2] >> (8 * (j & 3))) & 0xFFu;
      sum += v[j];
    }
  } else {
    for (int j = 0; j < SC_PER; j++) {
      int64_t r = r0 + j;
      v[j] = r < n ? in[r] : 0u;
      sum += v[j];
    }
  }
  // warp inclusive scan of per-thread sums
  uint32_t x = sum;
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    // warp 0: exclusive offsets of the warps' sums, then the tile's look-back with all 32 lanes
    const uint32_t w_sum = lane < SC_NT / 32 ? s_warp[lane] : 0u;
    uint32_t w_inc = w_sum;
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, w_inc, d);
      if (lane >= d) w_inc += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, w_inc, 31);
    __syncwarp();
    if (lane < SC_NT / 32) s_warp[lane] = w_inc - w_sum;
    const unsigned long long base = pmb_lookback_warp(lb, tile, total, status);
    if (lane == 0) s_base = base;
  }
  __syncthreads();
  uint32_t run = (uint32_t)s_base + s_warp[warp] + (x - sum);
#pragma unroll
  for (int j = 0; j < SC_PER; j++) {
    run += v[j];
    v[j] = run;
  }
  if (full && ((reinterpret_cast<uintptr_t>(out) & 15u) == 0u)) {
    // four 128-bit streaming stores (the output is not read again by this kernel)
    uint4* o = reinterpret_cast<uint4*>(out + r0);
#pragma unroll
    for (int j = 0; j < SC_PER / 4; j++) __stcs(o + j, make_uint4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]));
  } else {
    for (int j = 0; j < SC_PER; j++) {
      int64_t r = r0 + j;
      if (r < n) out[r] = v[j];
    }
  }
}

int run_compact(pmb_handle* h, CompiledQuery& cq, const uint8_t* keep_d, const uint8_t* keep_v, int n_out,
                bool to_host, pmb_result** out) {
  DQuery& q = cq.dq;
  const int64_t n = q.n_rows;
  pmb_result* r = pmb_result_new(n_out);
  if (!r) return pmb_fail(h, PMB_E_OOM, "host allocation failed");
  for (int c = 0; c < n_out; c++) r->columns[c].dtype = q.col[c].dtype;
  int64_t tiles = std::max<int64_t>(1, (n + CT_TILE - 1) / CT_TILE);
  CompactParams P;
  memset(&P, 0, sizeof(P));
  P.q = q;
  P.keep_data = keep_d;
  P.keep_valid = keep_v;
  P.n_out_cols = n_out;
  // look-back states for whichever kernel runs (the run-time compiled one has smaller tiles)
  const int64_t lb_tiles = std::max<int64_t>(tiles, (n + JC_TILE_ROWS - 1) / JC_TILE_ROWS);
  P.lb = (unsigned long long*)pmb_ws_alloc(h, (size_t)lb_tiles * 8 + 64);
  unsigned int* status = (unsigned int*)pmb_ws_alloc(h, 64);
  if (!P.lb || !status) {
    pmb_result_free(r);
    return pmb_fail(h, PMB_E_OOM, "workspace exhausted (compaction)");
  }
  P.ticket = P.lb + lb_tiles;
  P.n_out = P.lb + lb_tiles + 1;
  P.status = status;
  cudaMemsetAsync(P.lb, 0, (size_t)lb_tiles * 8 + 64, h->stream);
  cudaMemsetAsync(status, 0, 64, h->stream);
  for (int c = 0; c < n_out; c++) {
    int e = q.col[c].elem;
    size_t db = e ? (size_t)n * e : (size_t)((n + 31) / 32 * 4);
    size_t vb = (size_t)((n + 31) / 32 * 4);
    P.out_data[c] = (uint8_t*)pmb_ws_alloc(h, db + 16);
    P.out_valid[c] = (unsigned int*)pmb_ws_alloc(h, vb + 16);
    if (!P.out_data[c] || !P.out_valid[c]) {
      pmb_result_free(r);
      return pmb_fail(h, PMB_E_OOM, "workspace exhausted (compaction outputs)");
    }
    cudaMemsetAsync(P.out_valid[c], 0, vb + 16, h->stream);
    if (!e) cudaMemsetAsync(P.out_data[c], 0, db + 16, h->stream);
  }
  // a predicate over many rows: the run-time compiled compaction (literal offsets and dtypes)
  cudaKernel_t jk = nullptr;
  if (n > 0 && !keep_d && pmb_jit_enabled(n)) {
    std::string keep_err = h->err;
    if (pmb_jit_compact_kernel(h, cq, n_out, &jk) != PMB_OK) jk = nullptr;  // prebuilt kernel: same results
    h->err = keep_err;
  }
  if (n > 0 && jk) {
    const int64_t jt = (n + JC_TILE_ROWS - 1) / JC_TILE_ROWS;
    if (jt > lb_tiles) {
      pmb_result_free(r);
      return pmb_fail(h, PMB_E_CUDA, "internal: compaction tiles");
    }
    JitCompactParams A;
    memset(&A, 0, sizeof(A));
    for (int c = 0; c < q.n_cols; c++) {
      A.col_data[c] = q.col[c].data;
      A.col_valid[c] = q.col[c].valid;
    }
    A.n_rows = n;
    A.lb = P.lb;
    A.ticket = P.ticket;
    A.n_out = P.n_out;
    A.status = P.status;
    for (int c = 0; c < n_out; c++) {
      A.out_data[c] = P.out_data[c];
      A.out_valid[c] = P.out_valid[c];
    }
    void* args[] = {&A};
    pmb_kernel_begin(h, "compact");
    cudaError_t e = cudaLaunchKernel((const void*)jk, dim3((unsigned)jt), dim3(256), args, 0, h->stream);
    pmb_kernel_end(h);
    if (e != cudaSuccess) {
      pmb_result_free(r);
      return pmb_cuda_check(h, e, "pmb_jit_compact launch");
    }
  } else if (n > 0) {
    pmb_kernel_begin(h, "compact");
    k_compact<<<(unsigned)tiles, CT_NT, 0, h->stream>>>(P);
    pmb_kernel_end(h);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      pmb_result_free(r);
      return pmb_cuda_check(h, e, "k_compact launch");
    }
  }
  cudaMemcpyAsync(h->pinned, status, 4, cudaMemcpyDeviceToHost, h->stream);
  cudaMemcpyAsync(h->pinned + 8, P.n_out, 8, cudaMemcpyDeviceToHost, h->stream);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    pmb_result_free(r);
    return pmb_cuda_check(h, e, "compaction");
  }
  if (*(unsigned int*)h->pinned & PMB_ST_TIMEOUT) {
    pmb_result_free(r);
    return pmb_fail(h, PMB_E_TIMEOUT, "a bounded device wait timed out");
  }
  r->n_groups = n > 0 ? (int64_t) * (unsigned long long*)(h->pinned + 8) : 0;
  for (int c = 0; c < n_out; c++) {
    r->columns[c].data = P.out_data[c];
    r->columns[c].validity = (uint8_t*)P.out_valid[c];
  }
  int rc = pmb_finish_outputs(h, r, to_host);
  if (rc) {
    pmb_result_free(r);
    return rc;
  }
  *out = r;
  return PMB_OK;
}

// copies a caller buffer (host or device) of `bytes` into the workspace
int stage_raw(pmb_handle* h, const void* src, size_t bytes, bool on_device, const uint8_t** out) {
  uint8_t* d = (uint8_t*)pmb_ws_alloc(h, bytes + 16);
  if (!d) return pmb_fail(h, PMB_E_OOM, "workspace exhausted");
  if (bytes) {
    PMB_CUDA(h, cudaMemcpyAsync(d, src, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                h->stream));
    if (!on_device) h->h2d += (int64_t)bytes;
  }
  *out = d;
  return PMB_OK;
}

}  // namespace

extern "C" {

int pmb_compare(pmb_handle* h, const pmb_column* lhs, const pmb_column* rhs, int64_t rhs_i64, double rhs_f64,
                int32_t op, uint8_t* out_data, uint8_t* out_valid, int32_t out_on_device) {
  if (!h) return PMB_E_INVALID;
  if (!lhs || !out_data || !out_valid) return pmb_fail(h, PMB_E_INVALID, "lhs and outputs are required");
  if (op < PMB_CMP_EQ || op > PMB_CMP_GE) return pmb_fail(h, PMB_E_INVALID, "unknown compare op");
  if (lhs->dtype != PMB_I64 && lhs->dtype != PMB_F64)
    return pmb_fail(h, PMB_E_UNSUPPORTED, "compare supports I64 and F64 columns (narrower types widen first)");
  if (rhs && rhs->dtype != lhs->dtype) return pmb_fail(h, PMB_E_INVALID, "compare operands differ in dtype");
  if (rhs && rhs->length != lhs->length) return pmb_fail(h, PMB_E_INVALID, "compare operands differ in length");
  PMB_CUDA(h, cudaSetDevice(h->device));
  int rc = pmb_ws_begin(h);
  if (rc) return rc;
  pmb_call_begin(h);
  // an expression: Compare(Column 0, Column 1 | Literal)
  pmb_column cols[2] = {*lhs, rhs ? *rhs : *lhs};
  pmb_expr_node nodes[3];
  memset(nodes, 0, sizeof(nodes));
  nodes[0].kind = PMB_EXPR_COLUMN;
  nodes[0].column = 0;
  nodes[0].lhs = nodes[0].rhs = -1;
  if (rhs) {
    nodes[1].kind = PMB_EXPR_COLUMN;
    nodes[1].column = 1;
  } else if (lhs->dtype == PMB_I64) {
    nodes[1].kind = PMB_EXPR_LIT_I64;
    nodes[1].lit_i64 = rhs_i64;
  } else {
    nodes[1].kind = PMB_EXPR_LIT_F64;
    nodes[1].lit_f64 = rhs_f64;
  }
  nodes[1].lhs = nodes[1].rhs = -1;
  nodes[2].kind = PMB_EXPR_COMPARE;
  nodes[2].op = op;
  nodes[2].lhs = 0;
  nodes[2].rhs = 1;
  nodes[2].dtype = lhs->dtype;
  pmb_expr e{nodes, 3, 2};
  CompiledQuery cq;
  memset(&cq.dq, 0, sizeof(DQuery));
  rc = pmb_compile_predicate(h, &e, &cq.map, cols, rhs ? 2 : 1, &cq.dq.prog);
  if (rc) return rc;
  const int64_t n = lhs->length;
  cq.dq.n_cols = (int)cq.map.user.size();
  cq.dq.n_rows = n;
  for (int c = 0; c < cq.dq.n_cols; c++) {
    rc = pmb_stage_column(h, cols[cq.map.user[c]], n, &cq.dq.col[c]);
    if (rc) return rc;
  }
  int64_t ob = out_min_bytes(n);
  int64_t words = (n + 31) / 32;
  unsigned int* dd = (unsigned int*)pmb_ws_alloc(h, (size_t)words * 4 + 16);
  unsigned int* dv = (unsigned int*)pmb_ws_alloc(h, (size_t)words * 4 + 16);
  if (!dd || !dv) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (compare)");
  if (n > 0) {
    int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)h->sm_count * 8);
    pmb_kernel_begin(h, "pred_bits");
    k_pred_bits<<<blocks, 256, 0, h->stream>>>(cq.dq, dd, dv);
    pmb_kernel_end(h);
    PMB_CUDA(h, cudaGetLastError());
  }
  cudaMemcpyKind kind = out_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  PMB_CUDA(h, cudaMemsetAsync(dd + words, 0, 16, h->stream));
  PMB_CUDA(h, cudaMemsetAsync(dv + words, 0, 16, h->stream));
  PMB_CUDA(h, cudaMemcpyAsync(out_data, dd, (size_t)ob, kind, h->stream));
  PMB_CUDA(h, cudaMemcpyAsync(out_valid, dv, (size_t)ob, kind, h->stream));
  if (!out_on_device) h->d2h += 2 * ob;
  PMB_CUDA(h, cudaStreamSynchronize(h->stream));
  pmb_call_end(h);
  return PMB_OK;
}

static int bool_logic(pmb_handle* h, int op, const uint8_t* ld, const uint8_t* lv, const uint8_t* rd,
                      const uint8_t* rv, int64_t n, uint8_t* od, uint8_t* ov, int32_t on_device) {
  if (!h) return PMB_E_INVALID;
  if (n < 0 || (n > 0 && (!ld || !lv || !rd || !rv || !od || !ov)))
    return pmb_fail(h, PMB_E_INVALID, "bool logic needs four input bitmaps and two outputs");
  PMB_CUDA(h, cudaSetDevice(h->device));
  int rc = pmb_ws_begin(h);
  if (rc) return rc;
  pmb_call_begin(h);
  size_t nb = (size_t)((n + 7) / 8);
  int64_t ob = out_min_bytes(n);
  const uint8_t *dld, *dlv, *drd, *drv;
  if ((rc = stage_raw(h, ld, nb, on_device, &dld)) || (rc = stage_raw(h, lv, nb, on_device, &dlv)) ||
      (rc = stage_raw(h, rd, nb, on_device, &drd)) || (rc = stage_raw(h, rv, nb, on_device, &drv)))
    return rc;
  uint8_t* dod = (uint8_t*)pmb_ws_alloc(h, (size_t)ob + 16);
  uint8_t* dov = (uint8_t*)pmb_ws_alloc(h, (size_t)ob + 16);
  if (!dod || !dov) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (bool logic)");
  PMB_CUDA(h, cudaMemsetAsync(dod, 0, (size_t)ob, h->stream));
  PMB_CUDA(h, cudaMemsetAsync(dov, 0, (size_t)ob, h->stream));
  if (n > 0) {
    int blocks = (int)std::min<int64_t>(((int64_t)nb + 255) / 256, (int64_t)h->sm_count * 8);
    pmb_kernel_begin(h, "bool_logic");
    k_bool_logic<<<blocks, 256, 0, h->stream>>>(op, dld, dlv, drd, drv, n, dod, dov);
    pmb_kernel_end(h);
    PMB_CUDA(h, cudaGetLastError());
  }
  cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  PMB_CUDA(h, cudaMemcpyAsync(od, dod, (size_t)ob, kind, h->stream));
  PMB_CUDA(h, cudaMemcpyAsync(ov, dov, (size_t)ob, kind, h->stream));
  if (!on_device) h->d2h += 2 * ob;
  PMB_CUDA(h, cudaStreamSynchronize(h->stream));
  pmb_call_end(h);
  return PMB_OK;
}

int pmb_bool_and(pmb_handle* h, const uint8_t* ld, const uint8_t* lv, const uint8_t* rd, const uint8_t* rv, int64_t n,
                 uint8_t* od, uint8_t* ov, int32_t on_device) {
  return bool_logic(h, 0, ld, lv, rd, rv, n, od, ov, on_device);
}

int pmb_bool_or(pmb_handle* h, const uint8_t* ld, const uint8_t* lv, const uint8_t* rd, const uint8_t* rv, int64_t n,
                uint8_t* od, uint8_t* ov, int32_t on_device) {
  return bool_logic(h, 1, ld, lv, rd, rv, n, od, ov, on_device);
}

static int compact_common(pmb_handle* h, const pmb_expr* pred, const uint8_t* pd, const uint8_t* pv, int64_t n_rows,
                          int32_t pred_on_device, const pmb_column* cols, int32_t n_cols, int32_t output_on_device,
                          pmb_result** out) {
  if (!h) return PMB_E_INVALID;
  if (!out) return pmb_fail(h, PMB_E_INVALID, "out is NULL");
  *out = nullptr;
  if (n_cols < 0 || n_cols > PMB_MAX_COLS || (n_cols > 0 && !cols))
    return pmb_fail(h, PMB_E_INVALID, "bad column list (at most 16 columns)");
  PMB_CUDA(h, cudaSetDevice(h->device));
  CompiledQuery cq;
  memset(&cq.dq, 0, sizeof(DQuery));
  for (int c = 0; c < n_cols; c++) {
    if (cols[c].dtype < PMB_BOOL || cols[c].dtype > PMB_F64) return pmb_fail(h, PMB_E_INVALID, "unknown dtype");
    cq.map.user.push_back(c);
  }
  int rc;
  if (pred) {
    rc = pmb_compile_predicate(h, pred, &cq.map, cols, n_cols, &cq.dq.prog);
    if (rc) return rc;
    if (n_cols == 0) return pmb_fail(h, PMB_E_INVALID, "no columns");
    n_rows = cols[0].length;
  }
  for (int c = 0; c < n_cols; c++)
    if (cols[c].length != n_rows) return pmb_fail(h, PMB_E_INVALID, "column length differs from n_rows");
  cq.dq.n_cols = (int)cq.map.user.size();
  cq.dq.n_rows = n_rows;
  rc = pmb_ws_begin(h);
  if (rc) return rc;
  pmb_call_begin(h);
  for (int c = 0; c < cq.dq.n_cols; c++) {
    rc = pmb_stage_column(h, cols[cq.map.user[c]], n_rows, &cq.dq.col[c]);
    if (rc) return rc;
  }
  const uint8_t *kd = nullptr, *kv = nullptr;
  if (!pred) {
    size_t nb = (size_t)((n_rows + 7) / 8);
    if (n_rows > 0 && !pd) return pmb_fail(h, PMB_E_INVALID, "predicate bitmap is NULL");
    if ((rc = stage_raw(h, pd, nb, pred_on_device, &kd))) return rc;
    if (pv && (rc = stage_raw(h, pv, nb, pred_on_device, &kv))) return rc;
  }
  // only the caller's columns are outputs; columns the predicate adds come after them
  rc = run_compact(h, cq, kd, kv, n_cols, output_on_device == 0, out);
  if (rc) return rc;
  pmb_call_end(h);
  return PMB_OK;
}

int pmb_filter_compact(pmb_handle* h, const uint8_t* pred_data, const uint8_t* pred_valid, int64_t n_rows,
                       int32_t pred_on_device, const pmb_column* cols, int32_t n_cols, int32_t output_on_device,
                       pmb_result** out) {
  return compact_common(h, nullptr, pred_data, pred_valid, n_rows, pred_on_device, cols, n_cols, output_on_device, out);
}

int pmb_filter_compact_expr(pmb_handle* h, const pmb_expr* predicate, const pmb_column* cols, int32_t n_cols,
                            int32_t output_on_device, pmb_result** out) {
  if (!predicate) return pmb_fail(h, PMB_E_INVALID, "predicate is NULL");
  return compact_common(h, predicate, nullptr, nullptr, 0, 0, cols, n_cols, output_on_device, out);
}

int pmb_cumsum_u8_to_u32(pmb_handle* h, const uint8_t* in, uint32_t* out, int64_t n, int32_t on_device) {
  if (!h) return PMB_E_INVALID;
  if (n < 0 || (n > 0 && (!in || !out))) return pmb_fail(h, PMB_E_INVALID, "bad cumsum arguments");
  PMB_CUDA(h, cudaSetDevice(h->device));
  int rc = pmb_ws_begin(h);
  if (rc) return rc;
  pmb_call_begin(h);
  const uint8_t* din;
  if ((rc = stage_raw(h, in, (size_t)n, on_device, &din))) return rc;
  uint32_t* dout = on_device ? out : (uint32_t*)pmb_ws_alloc(h, (size_t)n * 4 + 16);
  int64_t tiles = std::max<int64_t>(1, (n + SC_TILE - 1) / SC_TILE);
  unsigned long long* lb = (unsigned long long*)pmb_ws_alloc(h, (size_t)tiles * 8 + 64);
  unsigned int* status = (unsigned int*)pmb_ws_alloc(h, 64);
  if (!dout || !lb || !status) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (cumsum)");
  PMB_CUDA(h, cudaMemsetAsync(lb, 0, (size_t)tiles * 8 + 64, h->stream));
  PMB_CUDA(h, cudaMemsetAsync(status, 0, 64, h->stream));
  if (n > 0) {
    pmb_kernel_begin(h, "cumsum_u8");
    k_cumsum_u8<<<(unsigned)tiles, SC_NT, 0, h->stream>>>(din, dout, n, lb, lb + tiles, status);
    pmb_kernel_end(h);
    PMB_CUDA(h, cudaGetLastError());
  }
  if (!on_device && n > 0) {
    PMB_CUDA(h, cudaMemcpyAsync(out, dout, (size_t)n * 4, cudaMemcpyDeviceToHost, h->stream));
    h->d2h += n * 4;
  }
  PMB_CUDA(h, cudaMemcpyAsync(h->pinned, status, 4, cudaMemcpyDeviceToHost, h->stream));
  PMB_CUDA(h, cudaStreamSynchronize(h->stream));
  pmb_call_end(h);
  if (*(unsigned int*)h->pinned & PMB_ST_TIMEOUT) return pmb_fail(h, PMB_E_TIMEOUT, "a bounded device wait timed out");
  return PMB_OK;
}

}  // extern "C"
