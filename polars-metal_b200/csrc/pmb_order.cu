// pmb_order.cu — the rows of a table sorted by some of its columns, on the device: a Sort over a
// GroupBy, top_k and bottom_k.
//
// The reference sorts on the CPU: its Sort plan runs the inner pipeline, then Polars'
// `df.sort(by, descending, nulls_last)` and the slice (python/polars_metal/_udf.py:684-721); only
// a single non-null Float32 column goes to an MLX sort, reversed and sliced on the host
// (_build_sort_fused, python/polars_metal/_udf.py:724-790). Here every dtype and any number of
// sort columns run on the GPU:
//   1. k_order_range  — per sort column the range of its values in Polars' order (as an unsigned
//                       integer) and its null count;
//   2. the sort columns are packed into keys of one or two 64-bit words: per column a null flag
//                       (when the column has nulls) above (value - min) or (max - value) bits, the
//                       most significant column highest. Columns that do not fit 128 bits go to
//                       further rounds, least significant first; every round is a stable sort of
//                       the previous round's order, so the rounds compose;
//   3. k_order_encode — keys of the rows in the current order, with the digit histograms;
//   4. pmb_sort_pairs — the group-by sort's LSD onesweep passes over the digits that vary;
//   5. k_order_gather — the slice of the sorted rows, a warp per 32 output rows so that each
//                       validity word is one ballot. Integer and Bool sort columns are decoded from
//                       the sorted keys when one round holds them all; the other columns are
//                       gathered by row index, without reading the validity of a column that
//                       k_null_flags found to have no nulls.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "pmb_groupby.h"

namespace {

constexpr int OR_NT = 256;
constexpr int OR_PASSES = 16;   // 8-bit digits of a 128-bit key
constexpr int OR_RADIX = 256;

// Polars' order of a value as an unsigned integer: signed integers with the sign bit flipped;
// floats with -0.0 read as 0.0 and every NaN as one NaN above +inf, negative values' bits
// inverted and non-negative values' sign bit set; unsigned integers and Bool as they are
__device__ __forceinline__ unsigned long long order_key(uint64_t b, int dt) {
  switch (dt) {
    case PMB_I8: return (unsigned long long)(long long)(int8_t)b ^ 0x8000000000000000ULL;
    case PMB_I16: return (unsigned long long)(long long)(int16_t)b ^ 0x8000000000000000ULL;
    case PMB_I32: return (unsigned long long)(long long)(int32_t)b ^ 0x8000000000000000ULL;
    case PMB_I64: return b ^ 0x8000000000000000ULL;
    case PMB_F32: {
      uint32_t x = (uint32_t)b;
      if ((x & 0x7FFFFFFFu) > 0x7F800000u) x = 0x7FC00000u;
      if (x == 0x80000000u) x = 0u;
      return (x & 0x80000000u) ? (unsigned long long)(uint32_t)~x : (unsigned long long)(x | 0x80000000u);
    }
    case PMB_F64: {
      uint64_t x = b;
      if ((x & 0x7FFFFFFFFFFFFFFFULL) > 0x7FF0000000000000ULL) x = 0x7FF8000000000000ULL;
      if (x == 0x8000000000000000ULL) x = 0ULL;
      return (x >> 63) ? ~x : (x | 0x8000000000000000ULL);
    }
    default: return b;
  }
}

struct SortCols {
  int n;
  const uint8_t* data[PMB_MAX_KEYS];
  const uint8_t* valid[PMB_MAX_KEYS];
  int elem[PMB_MAX_KEYS];
  int dtype[PMB_MAX_KEYS];
};

struct OrderRange {
  unsigned long long lo[PMB_MAX_KEYS];
  unsigned long long hi[PMB_MAX_KEYS];
  unsigned long long nulls[PMB_MAX_KEYS];
  unsigned int any[PMB_MAX_KEYS];
};

__device__ __forceinline__ unsigned long long warp_min64(unsigned long long v) {
  for (int o = 16; o; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ unsigned long long warp_max64(unsigned long long v) {
  for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__global__ void __launch_bounds__(OR_NT) k_order_range(const __grid_constant__ SortCols C, int64_t n, OrderRange* out) {
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int c = 0; c < C.n; c++) {
    unsigned long long lo = ~0ULL, hi = 0, nul = 0;
    unsigned any = 0;
    const uint8_t* data = C.data[c];
    const uint8_t* valid = C.valid[c];
    const int elem = C.elem[c], dtype = C.dtype[c];
    // four rows per step, their loads issued together (one row at a time left the kernel latency-bound)
    for (int64_t r0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r0 < n; r0 += 4 * stride) {
      uint64_t b[4];
      bool in[4], v[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int64_t r = r0 + u * stride;
        in[u] = r < n;
        v[u] = in[u] && pmb_valid_bit(valid, r);
        b[u] = in[u] ? pmb_load_bits(data, elem, r) : 0;
      }
#pragma unroll
      for (int u = 0; u < 4; u++) {
        if (in[u] && !v[u]) nul++;
        if (!v[u]) continue;
        const unsigned long long o = order_key(b[u], dtype);
        lo = min(lo, o);
        hi = max(hi, o);
        any = 1;
      }
    }
    lo = warp_min64(lo);
    hi = warp_max64(hi);
    for (int o = 16; o; o >>= 1) nul += __shfl_xor_sync(0xffffffffu, nul, o);
    any = __any_sync(0xffffffffu, any);
    if (lane == 0) {
      if (any) {
        atomicMin(&out->lo[c], lo);
        atomicMax(&out->hi[c], hi);
        atomicOr(&out->any[c], 1u);
      }
      if (nul) atomicAdd(&out->nulls[c], nul);
    }
  }
}

// one round's packed key: per column a null flag (null_off >= 0) and `data_bits` value bits
struct OrderLayout {
  int n;
  int bits;
  int null_off[PMB_MAX_KEYS];
  int data_off[PMB_MAX_KEYS];
  int data_bits[PMB_MAX_KEYS];
  int desc[PMB_MAX_KEYS];
  int nulls_last[PMB_MAX_KEYS];
  unsigned long long lo[PMB_MAX_KEYS];
  unsigned long long hi[PMB_MAX_KEYS];
  const uint8_t* data[PMB_MAX_KEYS];
  const uint8_t* valid[PMB_MAX_KEYS];
  int elem[PMB_MAX_KEYS];
  int dtype[PMB_MAX_KEYS];
};

template <int W>
__device__ __forceinline__ void put_bits(unsigned long long (&k)[W], int off, unsigned long long v, int bits) {
  if (bits == 0) return;
  const int wi = off >> 6, sh = off & 63;
  k[wi] |= v << sh;
  if (W > 1 && sh + bits > 64 && wi + 1 < W) k[wi + 1] |= v >> (64 - sh);
}

template <int W>
__device__ __forceinline__ unsigned key_digit(const unsigned long long (&k)[W], int shift) {
  const int wi = shift >> 6, sh = shift & 63;
  return (unsigned)((k[wi] >> sh) & 0xFFu);  // digits are 8-bit aligned: never across words
}

template <int W>
__global__ void __launch_bounds__(OR_NT) k_order_encode(const __grid_constant__ OrderLayout L, int64_t n,
                                                        const unsigned int* perm, unsigned long long* keys,
                                                        uint64_t cap, unsigned int* idx, int passes,
                                                        unsigned int* hist) {
  __shared__ unsigned int s_hist[OR_PASSES * OR_RADIX];
  for (int i = threadIdx.x; i < passes * OR_RADIX; i += OR_NT) s_hist[i] = 0;
  __syncthreads();
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t pos = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; pos < n; pos += stride) {
    const unsigned r = perm ? perm[pos] : (unsigned)pos;
    unsigned long long k[W];
    for (int i = 0; i < W; i++) k[i] = 0;
    for (int c = 0; c < L.n; c++) {
      const bool v = pmb_valid_bit(L.valid[c], r);
      if (L.null_off[c] >= 0) put_bits<W>(k, L.null_off[c], (L.nulls_last[c] ? !v : v) ? 1ULL : 0ULL, 1);
      if (!v) continue;
      const unsigned long long o = order_key(pmb_load_bits(L.data[c], L.elem[c], r), L.dtype[c]);
      put_bits<W>(k, L.data_off[c], L.desc[c] ? L.hi[c] - o : o - L.lo[c], L.data_bits[c]);
    }
    for (int i = 0; i < W; i++) keys[(uint64_t)i * cap + pos] = k[i];
    idx[pos] = r;
    for (int p = 0; p < passes; p++) atomicAdd(&s_hist[p * OR_RADIX + key_digit<W>(k, 8 * p)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * OR_RADIX; i += OR_NT) {
    const unsigned v = s_hist[i];
    if (v) atomicAdd(&hist[i], v);
  }
}

struct NullFlagCols {
  int n;
  const uint8_t* valid[PMB_MAX_OUT];  // null: no bitmap
};

// flags[c] = 1 when the bitmap of column c has a null among rows [0, n)
__global__ void __launch_bounds__(OR_NT) k_null_flags(const __grid_constant__ NullFlagCols V, int64_t n,
                                                      unsigned int* flags) {
  const int64_t full = n >> 3;
  const int rest = (int)(n & 7);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int c = 0; c < V.n; c++) {
    const uint8_t* v = V.valid[c];
    if (!v) continue;
    bool hole = false;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= full; i += stride) {
      if (i < full) hole |= v[i] != 0xFF;
      else if (rest) hole |= (v[i] & ((1u << rest) - 1u)) != ((1u << rest) - 1u);
    }
    if (__any_sync(0xffffffffu, hole) && (threadIdx.x & 31) == 0) atomicOr(&flags[c], 1u);
  }
}

struct GatherCols {
  int n;
  const uint8_t* data[PMB_MAX_OUT];
  const uint8_t* valid[PMB_MAX_OUT];  // null: every row valid
  int elem[PMB_MAX_OUT];
  int dec[PMB_MAX_OUT];               // >= 0: decoded from the sorted keys, column dec of L
  uint8_t* out_data[PMB_MAX_OUT];
  unsigned int* out_valid[PMB_MAX_OUT];
  const unsigned long long* keys;     // the sorted keys (word-major, stride cap), with dec >= 0
  uint64_t cap;
  int W;
};

template <int W>
__device__ __forceinline__ unsigned long long get_bits(const unsigned long long* keys, uint64_t cap, uint64_t pos,
                                                       int off, int bits) {
  if (bits == 0) return 0;
  const int wi = off >> 6, sh = off & 63;
  unsigned long long v = keys[(uint64_t)wi * cap + pos] >> sh;
  if (W > 1 && sh + bits > 64 && wi + 1 < W) v |= keys[(uint64_t)(wi + 1) * cap + pos] << (64 - sh);
  return bits == 64 ? v : (v & ((1ULL << bits) - 1ULL));
}

// the raw bits of an integer or Bool value from its order key
__device__ __forceinline__ uint64_t from_order_key(unsigned long long o, int dt) {
  switch (dt) {
    case PMB_I8: case PMB_I16: case PMB_I32: case PMB_I64: return o ^ 0x8000000000000000ULL;
    default: return o;
  }
}

constexpr int GU = 4;  // output words a warp fills per iteration: GU independent loads in flight per column

// rows idx[start + p] (start + p without an order) for p < m; a warp fills GU validity words (32
// rows each) per iteration, loading the rows of all GU words before it writes any
template <int W>
__global__ void __launch_bounds__(OR_NT) k_order_gather(const __grid_constant__ GatherCols G,
                                                        const __grid_constant__ OrderLayout L, const unsigned int* idx,
                                                        int64_t start, int64_t m) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x / 32);
  for (int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32 * GU; w0 * 32 < m; w0 += warps * GU) {
    int64_t p[GU], r[GU];
    bool ok[GU];
#pragma unroll
    for (int u = 0; u < GU; u++) {
      p[u] = (w0 + u) * 32 + lane;
      ok[u] = p[u] < m;
      r[u] = ok[u] ? (idx ? (int64_t)idx[start + p[u]] : start + p[u]) : 0;
    }
    for (int c = 0; c < G.n; c++) {
      const int e = G.elem[c];
      const int k = G.dec[c];
      uint64_t b[GU];
      bool v[GU];
      if (k >= 0) {
        // decoded: the null flag and the value field of the sorted key at position start + p
#pragma unroll
        for (int u = 0; u < GU; u++) {
          v[u] = ok[u];
          b[u] = 0;
          if (!ok[u]) continue;
          const uint64_t pos = (uint64_t)(start + p[u]);
          if (L.null_off[k] >= 0) {
            const bool flag = get_bits<W>(G.keys, G.cap, pos, L.null_off[k], 1) != 0;
            v[u] = L.nulls_last[k] ? !flag : flag;
          }
          const unsigned long long f = get_bits<W>(G.keys, G.cap, pos, L.data_off[k], L.data_bits[k]);
          b[u] = v[u] ? from_order_key(L.desc[k] ? L.hi[k] - f : L.lo[k] + f, L.dtype[k]) : 0;
        }
      } else {
        const uint8_t* d = G.data[c];
        switch (e) {
          case 0:
#pragma unroll
            for (int u = 0; u < GU; u++) b[u] = ok[u] ? (uint64_t)((d[r[u] >> 3] >> (r[u] & 7)) & 1u) : 0;
            break;
          case 1:
#pragma unroll
            for (int u = 0; u < GU; u++) b[u] = ok[u] ? (uint64_t)d[r[u]] : 0;
            break;
          case 2:
#pragma unroll
            for (int u = 0; u < GU; u++) b[u] = ok[u] ? (uint64_t)reinterpret_cast<const uint16_t*>(d)[r[u]] : 0;
            break;
          case 4:
#pragma unroll
            for (int u = 0; u < GU; u++) b[u] = ok[u] ? (uint64_t)reinterpret_cast<const uint32_t*>(d)[r[u]] : 0;
            break;
          default:
#pragma unroll
            for (int u = 0; u < GU; u++) b[u] = ok[u] ? reinterpret_cast<const uint64_t*>(d)[r[u]] : 0;
            break;
        }
        const uint8_t* vb = G.valid[c];
#pragma unroll
        for (int u = 0; u < GU; u++) v[u] = ok[u] && (vb == nullptr || ((vb[r[u] >> 3] >> (r[u] & 7)) & 1u));
      }
#pragma unroll
      for (int u = 0; u < GU; u++) {
        if (ok[u]) {
          switch (e) {
            case 0: break;
            case 1: G.out_data[c][p[u]] = (uint8_t)b[u]; break;
            case 2: reinterpret_cast<uint16_t*>(G.out_data[c])[p[u]] = (uint16_t)b[u]; break;
            case 4: reinterpret_cast<uint32_t*>(G.out_data[c])[p[u]] = (uint32_t)b[u]; break;
            default: reinterpret_cast<uint64_t*>(G.out_data[c])[p[u]] = b[u]; break;
          }
        }
        const unsigned vw = __ballot_sync(0xffffffffu, v[u]);
        const unsigned dw = __ballot_sync(0xffffffffu, ok[u] && e == 0 && b[u]);
        if (lane == 0 && (w0 + u) * 32 < m) {
          G.out_valid[c][w0 + u] = vw;
          if (e == 0) reinterpret_cast<unsigned int*>(G.out_data[c])[w0 + u] = dw;
        }
      }
    }
  }
}

int blocks_for(const pmb_handle* h, int64_t threads) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((threads + OR_NT - 1) / OR_NT, (int64_t)h->sm_count * 8));
}

}  // namespace

int pmb_order_columns(pmb_handle* h, const DCol* cols, int n_cols, int64_t n, const pmb_sort_spec& s, pmb_result* r) {
  if (n_cols <= 0 || n_cols > PMB_MAX_OUT || r->n_columns != n_cols)
    return pmb_fail(h, PMB_E_INVALID, "sort: 1 to 32 columns");
  if (s.n_by <= 0 || s.n_by > PMB_MAX_KEYS || !s.by) return pmb_fail(h, PMB_E_INVALID, "sort: 1 to 8 sort columns");
  for (int k = 0; k < s.n_by; k++)
    if (s.by[k] < 0 || s.by[k] >= n_cols) return pmb_fail(h, PMB_E_INVALID, "sort: sort column index out of range");
  if (n > 0xFFFFFFFELL) return pmb_fail(h, PMB_E_UNSUPPORTED, "sort: more than 2^32 - 2 rows");
  for (int c = 0; c < n_cols; c++) r->columns[c].dtype = cols[c].dtype;
  const int nb = s.n_by;
  int desc[PMB_MAX_KEYS], nlast[PMB_MAX_KEYS];
  for (int k = 0; k < nb; k++) {
    desc[k] = s.descending ? (s.descending[k] != 0) : 0;
    nlast[k] = s.nulls_last ? (s.nulls_last[k] != 0) : 0;
  }
  if (s.drop_nulls) nlast[0] = 1;  // the first column's nulls last, then cut off
  // ranges and null counts of the sort columns
  SortCols C;
  memset(&C, 0, sizeof(C));
  C.n = nb;
  for (int k = 0; k < nb; k++) {
    const DCol& d = cols[s.by[k]];
    C.data[k] = d.data;
    C.valid[k] = d.valid;
    C.elem[k] = d.elem;
    C.dtype[k] = d.dtype;
  }
  OrderRange got;
  memset(&got, 0, sizeof(got));
  for (int k = 0; k < PMB_MAX_KEYS; k++) got.lo[k] = ~0ULL;
  // which columns have a null at all (a column without one is gathered without its bitmap)
  unsigned int has_null[PMB_MAX_OUT];
  for (int c = 0; c < n_cols; c++) has_null[c] = cols[c].valid != nullptr;
  if (n > 0) {
    OrderRange* ro = (OrderRange*)pmb_ws_alloc(h, sizeof(OrderRange));
    unsigned int* flags = (unsigned int*)pmb_ws_alloc(h, PMB_MAX_OUT * 4);
    if (!ro || !flags) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (sort ranges)");
    PMB_CUDA(h, cudaMemcpyAsync(ro, &got, sizeof(got), cudaMemcpyHostToDevice, h->stream));
    PMB_CUDA(h, cudaMemsetAsync(flags, 0, PMB_MAX_OUT * 4, h->stream));
    pmb_kernel_begin(h, "order_range");
    k_order_range<<<blocks_for(h, n), OR_NT, 0, h->stream>>>(C, n, ro);
    pmb_kernel_end(h);
    PMB_CUDA(h, cudaGetLastError());
    NullFlagCols V;
    memset(&V, 0, sizeof(V));
    V.n = n_cols;
    for (int c = 0; c < n_cols; c++) V.valid[c] = cols[c].valid;
    pmb_kernel_begin(h, "null_flags");
    k_null_flags<<<blocks_for(h, n / 8 + 1), OR_NT, 0, h->stream>>>(V, n, flags);
    pmb_kernel_end(h);
    PMB_CUDA(h, cudaGetLastError());
    PMB_CUDA(h, cudaMemcpyAsync(&got, ro, sizeof(got), cudaMemcpyDeviceToHost, h->stream));
    PMB_CUDA(h, cudaMemcpyAsync(has_null, flags, (size_t)n_cols * 4, cudaMemcpyDeviceToHost, h->stream));
    PMB_CUDA(h, cudaStreamSynchronize(h->stream));
  }
  // field widths; rounds of at most 128 bits, cut from the least significant column up
  int nbits[PMB_MAX_KEYS], dbits[PMB_MAX_KEYS];
  for (int k = 0; k < nb; k++) {
    nbits[k] = got.nulls[k] ? 1 : 0;
    int b = 0;
    if (got.any[k]) {
      const unsigned long long span = got.hi[k] - got.lo[k];
      while (b < 64 && (span >> b) != 0) b++;
    }
    dbits[k] = b;
  }
  struct Round {
    int first, last, bits;
  };
  std::vector<Round> rounds;  // least significant first
  for (int end = nb - 1; end >= 0;) {
    int first = end, bits = nbits[end] + dbits[end];
    while (first > 0 && bits + nbits[first - 1] + dbits[first - 1] <= 128) {
      first--;
      bits += nbits[first] + dbits[first];
    }
    rounds.push_back({first, end, bits});
    end = first - 1;
  }
  const uint64_t cap = (uint64_t)std::max<int64_t>(n, 1);
  unsigned long long* k0 = (unsigned long long*)pmb_ws_alloc(h, (size_t)2 * cap * 8 + 16);
  unsigned long long* k1 = (unsigned long long*)pmb_ws_alloc(h, (size_t)2 * cap * 8 + 16);
  unsigned int* i0 = (unsigned int*)pmb_ws_alloc(h, (size_t)cap * 4 + 16);
  unsigned int* i1 = (unsigned int*)pmb_ws_alloc(h, (size_t)cap * 4 + 16);
  unsigned int* hist = (unsigned int*)pmb_ws_alloc(h, (size_t)OR_PASSES * OR_RADIX * 4);
  if (!k0 || !k1 || !i0 || !i1 || !hist) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (sort keys)");
  const unsigned int* perm = nullptr;  // the order so far (none: row order)
  std::vector<unsigned int> hh((size_t)OR_PASSES * OR_RADIX);
  OrderLayout L;  // the last round's layout
  memset(&L, 0, sizeof(L));
  int W = 1;
  for (const Round& rd : rounds) {
    if (rd.bits == 0 || n <= 1) continue;  // every key equal: the order stays
    memset(&L, 0, sizeof(L));
    L.n = rd.last - rd.first + 1;
    int off = 0;
    for (int k = rd.last; k >= rd.first; k--) {  // the most significant column highest
      const int i = k - rd.first;
      const DCol& d = cols[s.by[k]];
      L.data[i] = d.data;
      L.valid[i] = d.valid;
      L.elem[i] = d.elem;
      L.dtype[i] = d.dtype;
      L.desc[i] = desc[k];
      L.nulls_last[i] = nlast[k];
      L.lo[i] = got.lo[k];
      L.hi[i] = got.hi[k];
      L.data_off[i] = off;
      L.data_bits[i] = dbits[k];
      off += dbits[k];
      L.null_off[i] = nbits[k] ? off : -1;
      off += nbits[k];
    }
    L.bits = off;
    W = off > 64 ? 2 : 1;
    const int passes = (off + 7) / 8;
    PMB_CUDA(h, cudaMemsetAsync(hist, 0, (size_t)OR_PASSES * OR_RADIX * 4, h->stream));
    pmb_kernel_begin(h, "order_encode");
    if (W == 1) k_order_encode<1><<<blocks_for(h, n), OR_NT, 0, h->stream>>>(L, n, perm, k0, cap, i0, passes, hist);
    else k_order_encode<2><<<blocks_for(h, n), OR_NT, 0, h->stream>>>(L, n, perm, k0, cap, i0, passes, hist);
    pmb_kernel_end(h);
    PMB_CUDA(h, cudaGetLastError());
    PMB_CUDA(h, cudaMemcpyAsync(hh.data(), hist, (size_t)passes * OR_RADIX * 4, cudaMemcpyDeviceToHost, h->stream));
    PMB_CUDA(h, cudaStreamSynchronize(h->stream));
    const int rc = pmb_sort_pairs(h, W, &k0, &k1, &i0, &i1, cap, n, passes, hist, hh.data());
    if (rc) return rc;
    perm = i0;  // the next round reads the rows in this order (and rewrites i0 with the same values)
  }
  // the slice of the sorted rows (rows whose first sort column is null last, when dropped)
  const int64_t total = s.drop_nulls ? n - (int64_t)got.nulls[0] : n;
  const int64_t start = s.offset >= 0 ? std::min<int64_t>(s.offset, total) : std::max<int64_t>(0, total + s.offset);
  const int64_t m = s.limit < 0 ? total - start : std::min<int64_t>(s.limit, total - start);
  GatherCols G;
  memset(&G, 0, sizeof(G));
  G.n = n_cols;
  G.keys = k0;
  G.cap = cap;
  G.W = W;
  for (int c = 0; c < n_cols; c++) G.dec[c] = -1;
  // one round sorted every column: integer and Bool sort columns come back out of the sorted keys
  // (float keys are canonical in the key, -0.0 and NaN payloads, so floats are gathered)
  if (rounds.size() == 1 && perm != nullptr) {
    for (int k = 0; k < nb; k++) {
      const int dt = cols[s.by[k]].dtype;
      if (dt != PMB_F32 && dt != PMB_F64) G.dec[s.by[k]] = k - rounds[0].first;
    }
  }
  const int64_t words = (m + 31) / 32;
  for (int c = 0; c < n_cols; c++) {
    const int e = cols[c].elem;
    const size_t db = e ? (size_t)m * e : (size_t)words * 4;
    G.data[c] = cols[c].data;
    G.valid[c] = has_null[c] ? cols[c].valid : nullptr;
    G.elem[c] = e;
    G.out_data[c] = (uint8_t*)pmb_ws_alloc(h, db + 16);
    G.out_valid[c] = (unsigned int*)pmb_ws_alloc(h, (size_t)words * 4 + 16);
    if (!G.out_data[c] || !G.out_valid[c]) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (sort outputs)");
  }
  if (m > 0) {
    pmb_kernel_begin(h, "order_gather");
    const int gb = blocks_for(h, (words + GU - 1) / GU * 32);
    if (W == 1) k_order_gather<1><<<gb, OR_NT, 0, h->stream>>>(G, L, perm, start, m);
    else k_order_gather<2><<<gb, OR_NT, 0, h->stream>>>(G, L, perm, start, m);
    pmb_kernel_end(h);
    PMB_CUDA(h, cudaGetLastError());
  }
  r->n_groups = m;
  for (int c = 0; c < n_cols; c++) {
    r->columns[c].data = G.out_data[c];
    r->columns[c].validity = (uint8_t*)G.out_valid[c];
    r->columns[c].length = m;
    r->columns[c].on_device = 1;
  }
  return PMB_OK;
}

extern "C" int pmb_sort_columns(pmb_handle* h, const pmb_column* cols, int32_t n_cols, const pmb_sort_spec* spec,
                                int32_t output_on_device, pmb_result** out) {
  if (!h) return PMB_E_INVALID;
  if (!out) return pmb_fail(h, PMB_E_INVALID, "out is NULL");
  *out = nullptr;
  if (!spec || !cols || n_cols <= 0 || n_cols > PMB_MAX_COLS)
    return pmb_fail(h, PMB_E_INVALID, "sort: a spec and 1 to 16 columns are required");
  const int64_t n = cols[0].length;
  for (int c = 0; c < n_cols; c++) {
    if (cols[c].length != n) return pmb_fail(h, PMB_E_INVALID, "sort: columns differ in length");
    if (cols[c].dtype < PMB_BOOL || cols[c].dtype > PMB_F64) return pmb_fail(h, PMB_E_INVALID, "unknown dtype");
  }
  PMB_CUDA(h, cudaSetDevice(h->device));
  int rc = pmb_ws_begin(h);
  if (rc) return rc;
  pmb_call_begin(h);
  DCol d[PMB_MAX_COLS];
  memset(d, 0, sizeof(d));
  for (int c = 0; c < n_cols; c++) {
    rc = pmb_stage_column(h, cols[c], n, &d[c]);
    if (rc) return rc;
  }
  pmb_result* r = pmb_result_new(n_cols);
  if (!r) return pmb_fail(h, PMB_E_OOM, "host allocation failed");
  rc = pmb_order_columns(h, d, n_cols, n, *spec, r);
  if (!rc) rc = pmb_finish_outputs(h, r, output_on_device == 0);
  if (rc) {
    pmb_result_free(r);
    return rc;
  }
  r->strategy_used = PMB_STRATEGY_SORT;
  PMB_CUDA(h, cudaStreamSynchronize(h->stream));
  pmb_call_end(h);
  *out = r;
  return PMB_OK;
}

extern "C" int pmb_groupby_sorted(pmb_handle* h, const pmb_query* q, const pmb_column* cols, int32_t n_cols,
                                  const pmb_sort_spec* spec, pmb_result** out) {
  if (!h) return PMB_E_INVALID;
  if (!out) return pmb_fail(h, PMB_E_INVALID, "out is NULL");
  *out = nullptr;
  if (!q || !spec) return pmb_fail(h, PMB_E_INVALID, "a query and a sort spec are required");
  pmb_query qd = *q;
  qd.output_on_device = 1;
  pmb_result* g = nullptr;
  int rc = pmb_groupby(h, &qd, cols, n_cols, &g);
  if (rc) return rc;
  // the group-by's device columns stay in the workspace; the sort's buffers follow them (no
  // workspace reset), and its launches add to the same call's statistics
  DCol d[PMB_MAX_OUT];
  memset(d, 0, sizeof(d));
  for (int c = 0; c < g->n_columns && c < PMB_MAX_OUT; c++) {
    d[c].data = (const uint8_t*)g->columns[c].data;
    d[c].valid = g->columns[c].validity;
    d[c].dtype = g->columns[c].dtype;
    d[c].elem = pmb_dtype_bytes(g->columns[c].dtype);
  }
  pmb_result* r = pmb_result_new(g->n_columns);
  if (!r) {
    pmb_result_free(g);
    return pmb_fail(h, PMB_E_OOM, "host allocation failed");
  }
  rc = pmb_order_columns(h, d, g->n_columns, g->n_groups, *spec, r);
  r->strategy_used = g->strategy_used;
  r->rehash_count = g->rehash_count;
  r->capacity = g->capacity;
  pmb_result_free(g);
  if (!rc) rc = pmb_finish_outputs(h, r, q->output_on_device == 0);
  if (rc) {
    pmb_result_free(r);
    return rc;
  }
  PMB_CUDA(h, cudaStreamSynchronize(h->stream));
  pmb_call_end(h);
  *out = r;
  return PMB_OK;
}
