// pmb_sort.cu — the sort strategy of the group-by: packed-key LSD radix sort + segmented reduce.
//
// The reference's A2 build sorts (u128 lane, row index) pairs with a stable 16-pass 8-bit LSD
// radix sort, marks segment starts and scans them into group ids on the CPU
// (crates/polars-metal-kernels/src/groupby_build_sort/gpu.rs:24-252,
// shaders/groupby_sort_u128_lane.metal:52-172, shaders/groupby_segments.metal:18-40; CPU
// statement groupby_build_sort/reference.rs:3-35). Here, for B200:
//   1. k_key_range   — per key column the range of its values (as order-preserving u64) and
//                      whether it has nulls; the host packs every key into only its significant
//                      bits (value - min), so most keys fit one 64-bit word and the sort runs
//                      ceil(bits / 8) passes instead of 16;
//   2. k_sort_encode — filter (the query's predicate), packed key + row index, compacted; and the
//                      digit histograms of every pass, in the same read;
//   3. k_sort_pass   — one stable 8-bit LSD pass per digit that is not constant (onesweep style:
//                      warp-level ranking with __match_any_sync, per-digit decoupled look-back
//                      for the tile's global offsets, the tile reordered in shared memory so that
//                      the writes are coalesced);
//   4. k_seg_starts  — segment starts (key differs from its predecessor) compacted in order;
//   5. k_seg_reduce  — one thread per group folds its rows into a group record (the same record
//                      and the same finalisation as the hash path, so both strategies give
//                      identical results, exact float sums included) and writes the output
//                      row; groups of more than 256 rows go to k_seg_reduce_big (one CTA per
//                      group).
// Output groups come out in packed-key order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "pmb_groupby.h"

namespace {

constexpr int ST_NT = 256;              // threads of the sort kernels
constexpr int ST_PER = 16;              // keys per thread in a pass tile
constexpr int ST_TILE = ST_NT * ST_PER;  // 4096 keys per tile
constexpr int RADIX = 256;
constexpr int MAX_PASSES = 16;
constexpr int BIG = 256;                // rows above which a group is reduced by a whole CTA
constexpr int BIG_NT = 128;

// packed-key layout of the sort: per key column an optional null bit, then (value - min) bits
struct SortKeyLayout {
  int n_keys;
  int words;  // 1 or 2
  int bits;   // total
  int col[PMB_MAX_KEYS];
  int null_off[PMB_MAX_KEYS];  // -1: no null bit
  int data_off[PMB_MAX_KEYS];
  int data_bits[PMB_MAX_KEYS];
  unsigned long long lo[PMB_MAX_KEYS];  // order-preserving u64 of the smallest valid value
  int dtype[PMB_MAX_KEYS];
  int elem[PMB_MAX_KEYS];
  const uint8_t* data[PMB_MAX_KEYS];
  const uint8_t* valid[PMB_MAX_KEYS];
};

struct RangeOut {
  unsigned long long lo[PMB_MAX_KEYS];
  unsigned long long hi[PMB_MAX_KEYS];
  unsigned int nulls[PMB_MAX_KEYS];
  unsigned int any[PMB_MAX_KEYS];
};

// order-preserving u64 of a key value: signed integers with the sign bit flipped, everything
// else (unsigned, bool, float bit patterns) as is; grouping only needs equality, the order just
// has to be consistent
__host__ __device__ __forceinline__ bool signed_dt(int dt) {
  return dt == PMB_I8 || dt == PMB_I16 || dt == PMB_I32 || dt == PMB_I64;
}
__device__ __forceinline__ unsigned long long ordered_bits(uint64_t b, int dt) {
  switch (dt) {
    case PMB_I8: return (unsigned long long)((long long)(int8_t)b) ^ 0x8000000000000000ULL;
    case PMB_I16: return (unsigned long long)((long long)(int16_t)b) ^ 0x8000000000000000ULL;
    case PMB_I32: return (unsigned long long)((long long)(int32_t)b) ^ 0x8000000000000000ULL;
    case PMB_I64: return b ^ 0x8000000000000000ULL;
    default: return b;
  }
}
__device__ __forceinline__ uint64_t from_ordered(unsigned long long o, int dt) {
  return signed_dt(dt) ? (o ^ 0x8000000000000000ULL) : o;
}

__global__ void __launch_bounds__(ST_NT) k_key_range(const __grid_constant__ SortKeyLayout L, int64_t n,
                                                     RangeOut* out) {
  unsigned long long lo[PMB_MAX_KEYS], hi[PMB_MAX_KEYS];
  unsigned nul[PMB_MAX_KEYS], any[PMB_MAX_KEYS];
  for (int k = 0; k < L.n_keys; k++) {
    lo[k] = ~0ULL;
    hi[k] = 0;
    nul[k] = any[k] = 0;
  }
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) {
    for (int k = 0; k < L.n_keys; k++) {
      if (!pmb_valid_bit(L.valid[k], r)) {
        nul[k] = 1;
        continue;
      }
      unsigned long long o = ordered_bits(pmb_load_bits(L.data[k], L.elem[k], r), L.dtype[k]);
      lo[k] = o < lo[k] ? o : lo[k];
      hi[k] = o > hi[k] ? o : hi[k];
      any[k] = 1;
    }
  }
  for (int k = 0; k < L.n_keys; k++) {
    for (int o = 16; o; o >>= 1) {
      unsigned long long a = __shfl_xor_sync(0xffffffffu, lo[k], o), b = __shfl_xor_sync(0xffffffffu, hi[k], o);
      lo[k] = a < lo[k] ? a : lo[k];
      hi[k] = b > hi[k] ? b : hi[k];
      nul[k] |= __shfl_xor_sync(0xffffffffu, nul[k], o);
      any[k] |= __shfl_xor_sync(0xffffffffu, any[k], o);
    }
    if ((threadIdx.x & 31) == 0) {
      if (any[k]) {
        atomicMin(&out->lo[k], lo[k]);
        atomicMax(&out->hi[k], hi[k]);
        atomicOr(&out->any[k], 1u);
      }
      if (nul[k]) atomicOr(&out->nulls[k], 1u);
    }
  }
}

template <int W>
struct PKey {
  unsigned long long w[W];
};

template <int W>
__device__ __forceinline__ PKey<W> pack_sort_key(const SortKeyLayout& L, int64_t r) {
  PKey<W> k;
  for (int i = 0; i < W; i++) k.w[i] = 0;
  auto put = [&](int off, unsigned long long v, int bits) {
    if (bits == 0) return;
    const int wi = off >> 6, sh = off & 63;
    k.w[wi] |= v << sh;
    if (W > 1 && sh + bits > 64 && wi + 1 < W) k.w[wi + 1] |= v >> (64 - sh);
  };
  for (int c = 0; c < L.n_keys; c++) {
    if (!pmb_valid_bit(L.valid[c], r)) {
      put(L.null_off[c], 1ULL, 1);
      continue;
    }
    unsigned long long o = ordered_bits(pmb_load_bits(L.data[c], L.elem[c], r), L.dtype[c]);
    put(L.data_off[c], o - L.lo[c], L.data_bits[c]);
  }
  return k;
}

template <int W>
__device__ __forceinline__ unsigned digit_of(const PKey<W>& k, int shift) {
  const int wi = shift >> 6, sh = shift & 63;
  unsigned long long v = k.w[wi] >> sh;
  if (W > 1 && sh > 56 && wi + 1 < W) v |= k.w[wi + 1] << (64 - sh);
  return (unsigned)(v & 0xFF);
}

struct EncodeParams {
  DQuery q;
  SortKeyLayout L;
  int passes;
  int64_t n;
  unsigned long long* keys;  // W words per key, word-major: word i of key j at keys[i * cap + j]
  uint64_t cap;
  unsigned int* idx;
  unsigned long long* lb;      // look-back states, one per tile, zeroed
  unsigned long long* ticket;
  unsigned long long* kept;    // rows that passed the filter
  unsigned int* hist;          // passes x 256
  unsigned int* status;
};

// filter, pack and compact in row order (4096-row tiles, decoupled look-back), with the digit
// histograms of every pass
template <int W>
__global__ void __launch_bounds__(ST_NT) k_sort_encode(const __grid_constant__ EncodeParams E) {
  __shared__ unsigned int s_hist[MAX_PASSES][RADIX];
  __shared__ unsigned int s_cnt[ST_PER][ST_NT / 32];
  __shared__ long long s_tile;
  __shared__ unsigned long long s_base;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < E.passes * RADIX; i += ST_NT) (&s_hist[0][0])[i] = 0;
  if (tid == 0) s_tile = (long long)atomicAdd(E.ticket, 1ULL);
  __syncthreads();
  const long long tile = s_tile;
  const TileCtx t{nullptr, nullptr, nullptr, 0};
  const bool has_pred = E.q.prog.n_ops > 0;
  bool keep[ST_PER];
  for (int j = 0; j < ST_PER; j++) {
    const int64_t r = tile * ST_TILE + (int64_t)j * ST_NT + tid;
    keep[j] = r < E.n && (!has_pred || eval_keep(E.q, t, r));
    const unsigned b = __ballot_sync(0xffffffffu, keep[j]);
    if (lane == 0) s_cnt[j][warp] = __popc(b);
  }
  __syncthreads();
  if (tid == 0) {
    unsigned acc = 0;
    for (int j = 0; j < ST_PER; j++)
      for (int w = 0; w < ST_NT / 32; w++) {
        unsigned c = s_cnt[j][w];
        s_cnt[j][w] = acc;
        acc += c;
      }
    const unsigned long long b = pmb_lookback(E.lb, tile, acc, E.status);
    s_base = b;
    if (tile == (long long)gridDim.x - 1) *E.kept = b + acc;
  }
  __syncthreads();
  for (int j = 0; j < ST_PER; j++) {
    const unsigned b = __ballot_sync(0xffffffffu, keep[j]);
    if (!keep[j]) continue;
    const int64_t r = tile * ST_TILE + (int64_t)j * ST_NT + tid;
    const PKey<W> k = pack_sort_key<W>(E.L, r);
    for (int p = 0; p < E.passes; p++) atomicAdd(&s_hist[p][digit_of<W>(k, 8 * p)], 1u);
    const uint64_t pos = s_base + s_cnt[j][warp] + __popc(b & ((1u << lane) - 1u));
    for (int i = 0; i < W; i++) E.keys[(uint64_t)i * E.cap + pos] = k.w[i];
    E.idx[pos] = (unsigned)r;
  }
  __syncthreads();
  for (int i = tid; i < E.passes * RADIX; i += ST_NT) {
    unsigned v = (&s_hist[0][0])[i];
    if (v) atomicAdd(&E.hist[i], v);
  }
}

struct PassParams {
  const unsigned long long* kin;
  unsigned long long* kout;
  const unsigned int* iin;
  unsigned int* iout;
  uint64_t cap;  // word stride of the key arrays
  int64_t n;
  int shift;
  const unsigned int* hist;      // this pass's 256 digit counts
  unsigned long long* lb;        // n_tiles x 256 look-back states (digit-major), zeroed
  int64_t n_tiles;
  unsigned long long* ticket;
  unsigned int* status;
};

// One stable LSD pass over 8 bits at `shift`.
template <int W>
__global__ void __launch_bounds__(ST_NT) k_sort_pass(const __grid_constant__ PassParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned long long* s_key = reinterpret_cast<unsigned long long*>(smem);       // W x ST_TILE
  unsigned int* s_idx = reinterpret_cast<unsigned int*>(s_key + W * ST_TILE);   // ST_TILE
  __shared__ unsigned int s_whist[ST_NT / 32][RADIX];
  __shared__ unsigned int s_excl[RADIX];      // tile-local exclusive offset of each digit
  __shared__ unsigned long long s_gbase[RADIX];
  __shared__ unsigned int s_scan[ST_NT / 32];
  __shared__ long long s_tile;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_tile = (long long)atomicAdd(P.ticket, 1ULL);
  for (int i = tid; i < (ST_NT / 32) * RADIX; i += ST_NT) (&s_whist[0][0])[i] = 0;
  __syncthreads();
  const long long tile = s_tile;
  const int64_t base = tile * ST_TILE;
  const unsigned lt = (1u << lane) - 1u;
  // warp-striped items: warp w owns tile elements [w*512, w*512+512), item j of lane l is
  // w*512 + j*32 + l. Only the digit and the rank stay in registers; the keys are read again (from
  // L2) when the tile is reordered in shared memory.
  unsigned int rank[ST_PER];
  unsigned short dg[ST_PER];
#pragma unroll
  for (int j = 0; j < ST_PER; j++) {
    const int64_t e = base + warp * (ST_PER * 32) + j * 32 + lane;
    PKey<W> k;
    for (int i = 0; i < W; i++) k.w[i] = e < P.n ? P.kin[(uint64_t)i * P.cap + e] : 0ULL;
    dg[j] = e < P.n ? (unsigned short)digit_of<W>(k, P.shift) : (unsigned short)RADIX;
  }
  // ranks within the warp, in item order (stable): lanes with the same digit in one round are
  // ordered by lane; earlier rounds come first
#pragma unroll
  for (int j = 0; j < ST_PER; j++) {
    const unsigned d = dg[j];
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int leader = __ffs(peers) - 1;
    unsigned old = 0;
    if (d < RADIX && lane == leader) {
      old = s_whist[warp][d];
      s_whist[warp][d] = old + __popc(peers);
    }
    old = __shfl_sync(0xffffffffu, old, leader);
    rank[j] = old + __popc(peers & lt);
    __syncwarp();
  }
  __syncthreads();
  // per digit (thread d): warps' exclusive offsets and the tile's count
  {
    const int d = tid;
    unsigned acc = 0;
    for (int w = 0; w < ST_NT / 32; w++) {
      unsigned c = s_whist[w][d];
      s_whist[w][d] = acc;
      acc += c;
    }
    // tile-local exclusive scan over digits (block scan of one value per thread)
    unsigned x = acc;
    for (int o = 1; o < 32; o <<= 1) {
      unsigned y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_scan[warp] = x;
    __syncthreads();
    if (tid == 0) {
      unsigned a = 0;
      for (int w = 0; w < ST_NT / 32; w++) {
        unsigned c = s_scan[w];
        s_scan[w] = a;
        a += c;
      }
    }
    __syncthreads();
    const unsigned excl = x - acc + s_scan[warp];
    s_excl[d] = excl;
    // global start of this digit: the counts of the digits before it over the whole input
    // (exclusive scan of this pass's histogram), then the earlier tiles (look-back)
    const unsigned hd = P.hist[d];
    unsigned y = hd;
    for (int o = 1; o < 32; o <<= 1) {
      unsigned z = __shfl_up_sync(0xffffffffu, y, o);
      if (lane >= o) y += z;
    }
    __syncthreads();
    if (lane == 31) s_scan[warp] = y;
    __syncthreads();
    if (tid == 0) {
      unsigned a = 0;
      for (int w = 0; w < ST_NT / 32; w++) {
        unsigned c = s_scan[w];
        s_scan[w] = a;
        a += c;
      }
    }
    __syncthreads();
    const unsigned long long gstart = (unsigned long long)(y - hd + s_scan[warp]);
    const unsigned long long pre = pmb_lookback(P.lb + (int64_t)d * P.n_tiles, tile, acc, P.status);
    s_gbase[d] = gstart + pre;
  }
  __syncthreads();
  // reorder the tile in shared memory by digit
#pragma unroll
  for (int j = 0; j < ST_PER; j++) {
    const unsigned d = dg[j];
    if (d < RADIX) {
      const int64_t e = base + warp * (ST_PER * 32) + j * 32 + lane;
      const unsigned lp = s_excl[d] + s_whist[warp][d] + rank[j];
      for (int i = 0; i < W; i++) s_key[i * ST_TILE + lp] = P.kin[(uint64_t)i * P.cap + e];
      s_idx[lp] = P.iin[e];
    }
  }
  __syncthreads();
  const int valid = (int)min((int64_t)ST_TILE, P.n - base);
  for (int i = tid; i < valid; i += ST_NT) {
    PKey<W> k;
    for (int w = 0; w < W; w++) k.w[w] = s_key[w * ST_TILE + i];
    const unsigned d = digit_of<W>(k, P.shift);
    const uint64_t g = s_gbase[d] + (uint64_t)(i - (int)s_excl[d]);
    for (int w = 0; w < W; w++) P.kout[(uint64_t)w * P.cap + g] = k.w[w];
    P.iout[g] = s_idx[i];
  }
}

struct StartsParams {
  const unsigned long long* keys;
  uint64_t cap;
  int64_t n;
  unsigned int* starts;  // n_groups + 1 entries (the last one = n)
  unsigned long long* lb;
  unsigned long long* ticket;
  unsigned long long* n_groups;
  unsigned int* status;
};

template <int W>
__global__ void __launch_bounds__(ST_NT) k_seg_starts(const __grid_constant__ StartsParams S) {
  __shared__ unsigned int s_cnt[ST_PER][ST_NT / 32];
  __shared__ long long s_tile;
  __shared__ unsigned long long s_base;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_tile = (long long)atomicAdd(S.ticket, 1ULL);
  __syncthreads();
  const long long tile = s_tile;
  bool head[ST_PER];
  for (int j = 0; j < ST_PER; j++) {
    const int64_t e = tile * ST_TILE + (int64_t)j * ST_NT + tid;
    bool hd = false;
    if (e < S.n) {
      hd = e == 0;
      for (int w = 0; w < W && !hd; w++) hd = S.keys[(uint64_t)w * S.cap + e] != S.keys[(uint64_t)w * S.cap + e - 1];
    }
    head[j] = hd;
    const unsigned b = __ballot_sync(0xffffffffu, hd);
    if (lane == 0) s_cnt[j][warp] = __popc(b);
  }
  __syncthreads();
  if (tid == 0) {
    unsigned acc = 0;
    for (int j = 0; j < ST_PER; j++)
      for (int w = 0; w < ST_NT / 32; w++) {
        unsigned c = s_cnt[j][w];
        s_cnt[j][w] = acc;
        acc += c;
      }
    const unsigned long long b = pmb_lookback(S.lb, tile, acc, S.status);
    s_base = b;
    if (tile == (long long)gridDim.x - 1) {
      *S.n_groups = b + acc;
      S.starts[b + acc] = (unsigned)S.n;
    }
  }
  __syncthreads();
  for (int j = 0; j < ST_PER; j++) {
    const unsigned b = __ballot_sync(0xffffffffu, head[j]);
    if (head[j]) {
      const int64_t e = tile * ST_TILE + (int64_t)j * ST_NT + tid;
      S.starts[s_base + s_cnt[j][warp] + __popc(b & ((1u << lane) - 1u))] = (unsigned)e;
    }
  }
}

struct ReduceParams {
  DQuery q;
  RecInit ri;
  SortKeyLayout L;
  const unsigned long long* keys;
  uint64_t cap;
  const unsigned int* idx;
  const unsigned int* starts;
  const unsigned long long* n_groups;
  unsigned int* big;             // groups reduced by k_seg_reduce_big
  unsigned long long* big_n;
  unsigned int* status;
  uint8_t* out_data[PMB_MAX_OUT];
  uint8_t* out_valid[PMB_MAX_OUT];
};

__device__ __forceinline__ void store_bits(uint8_t* d, int bytes, int64_t p, uint64_t v) {
  switch (bytes) {
    case 0: break;
    case 1: d[p] = (uint8_t)v; break;
    case 2: reinterpret_cast<uint16_t*>(d)[p] = (uint16_t)v; break;
    case 4: reinterpret_cast<uint32_t*>(d)[p] = (uint32_t)v; break;
    default: reinterpret_cast<uint64_t*>(d)[p] = v; break;
  }
}

// key value of key column c from the packed sort key (false: null)
template <int W>
__device__ __forceinline__ bool unpack_sort_key(const SortKeyLayout& L, const PKey<W>& k, int c, uint64_t& v) {
  auto get = [&](int off, int bits) -> unsigned long long {
    if (bits == 0) return 0ULL;
    const int wi = off >> 6, sh = off & 63;
    unsigned long long x = k.w[wi] >> sh;
    if (W > 1 && sh + bits > 64 && wi + 1 < W) x |= k.w[wi + 1] << (64 - sh);
    return bits == 64 ? x : (x & ((1ULL << bits) - 1ULL));
  };
  if (L.null_off[c] >= 0 && get(L.null_off[c], 1)) return false;
  v = from_ordered(get(L.data_off[c], L.data_bits[c]) + L.lo[c], L.dtype[c]);
  return true;
}

// writes group p's output row from its record; `bitset` chooses how validity / bool bits are set
// (warp-wide for the one-thread-per-group kernel, atomic for the big-group kernel)
template <int W, bool WARP>
__device__ __forceinline__ void write_group(const ReduceParams& R, int64_t p, int64_t p_first, bool have,
                                           const PKey<W>& k, const uint8_t* rec) {
  const DQuery& q = R.q;
  int oc = 0;
  auto setbit = [&](uint8_t* words, bool bit) {
    if (WARP) {
      warp_set_bits(reinterpret_cast<unsigned int*>(words), p, p_first, bit);
    } else if (bit) {
      atomicOr(reinterpret_cast<unsigned int*>(words) + (p >> 5), 1u << (p & 31));
    }
  };
  for (int c = 0; c < q.n_keys; c++, oc++) {
    uint64_t v = 0;
    const bool valid = have && unpack_sort_key<W>(R.L, k, c, v);
    const int dt = R.L.dtype[c];
    if (have) store_bits(R.out_data[oc], pmb_dtype_bytes(dt), p, v);
    if (dt == PMB_BOOL) setbit(R.out_data[oc], have && valid && v);
    setbit(R.out_valid[oc], have && valid);
  }
  for (int a = 0; a < q.n_aggs; a++, oc++) {
    const DAggOut& A = q.agg[a];
    bool valid = true;
    uint64_t bits = 0;
    if (have) finalize_agg(q, A, rec, valid, bits);
    if (have) store_bits(R.out_data[oc], pmb_dtype_bytes(A.out_dtype), p, bits);
    setbit(R.out_valid[oc], have && valid);
  }
}

template <int W, int RW>
__global__ void __launch_bounds__(ST_NT) k_seg_reduce(const __grid_constant__ ReduceParams R) {
  const int64_t ng = (int64_t)*R.n_groups;
  const TileCtx t{nullptr, nullptr, nullptr, 0};
  uint64_t recw[RW];  // the group record, RW >= rec_bytes / 8
  uint8_t* rec = reinterpret_cast<uint8_t*>(recw);
  const int rw = R.q.rec_bytes / 8;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  // every lane of a warp runs the same number of iterations (warp-wide bit setting)
  const int64_t span = (ng + stride - 1) / stride * stride;
  for (int64_t g0 = (int64_t)blockIdx.x * blockDim.x; g0 < span; g0 += stride) {
    const int64_t g = g0 + threadIdx.x;
    const int64_t p_first = g0 + (threadIdx.x & ~31);
    bool have = g < ng;
    PKey<W> k{};
    if (have) {
      const unsigned s = R.starts[g], e = R.starts[g + 1];
      for (int i = 0; i < W; i++) k.w[i] = R.keys[(uint64_t)i * R.cap + s];
      if (e - s > (unsigned)BIG) {
        R.big[atomicAdd(R.big_n, 1ULL)] = (unsigned)g;
        have = false;
      } else {
        for (int w = 0; w < rw; w++) recw[w] = R.ri.w[w];
        for (unsigned i = s; i < e; i++) {
          const int64_t row = R.idx[i];
          fx_range_check(R.q, t, row, R.status);
          apply_row_private(R.q, t, rec, row);
        }
      }
    }
    write_group<W, true>(R, g, p_first, have, k, rec);
  }
}

// groups of more than BIG rows: one CTA each (persistent over the list); thread records are
// merged in shared memory by one thread
template <int W>
__global__ void __launch_bounds__(BIG_NT) k_seg_reduce_big(const __grid_constant__ ReduceParams R) {
  extern __shared__ __align__(16) unsigned char srec[];  // BIG_NT records
  const TileCtx t{nullptr, nullptr, nullptr, 0};
  const int rb = R.q.rec_bytes, rw = rb / 8;
  const unsigned long long nb = *R.big_n;
  uint8_t* mine = srec + (size_t)threadIdx.x * rb;
  for (unsigned long long b = blockIdx.x; b < nb; b += gridDim.x) {
    const unsigned g = R.big[b];
    const unsigned s = R.starts[g], e = R.starts[g + 1];
    for (int w = 0; w < rw; w++) reinterpret_cast<uint64_t*>(mine)[w] = R.ri.w[w];
    for (unsigned i = s + threadIdx.x; i < e; i += BIG_NT) {
      const int64_t row = R.idx[i];
      fx_range_check(R.q, t, row, R.status);
      apply_row_private(R.q, t, mine, row);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int j = 1; j < BIG_NT; j++) merge_private(R.q, srec, srec + (size_t)j * rb);
      PKey<W> k;
      for (int i = 0; i < W; i++) k.w[i] = R.keys[(uint64_t)i * R.cap + s];
      write_group<W, false>(R, g, g, true, k, srec);
    }
    __syncthreads();
  }
}

template <int W>
int run_sort(pmb_handle* h, CompiledQuery& cq, const SortKeyLayout& L, pmb_result* r) {
  DQuery& q = cq.dq;
  const int64_t n = q.n_rows;
  const int passes = std::max(0, (L.bits + 7) / 8);
  const uint64_t cap = (uint64_t)n;
  unsigned long long* k0 = (unsigned long long*)pmb_ws_alloc(h, (size_t)W * cap * 8 + 16);
  unsigned long long* k1 = (unsigned long long*)pmb_ws_alloc(h, (size_t)W * cap * 8 + 16);
  unsigned int* i0 = (unsigned int*)pmb_ws_alloc(h, (size_t)cap * 4 + 16);
  unsigned int* i1 = (unsigned int*)pmb_ws_alloc(h, (size_t)cap * 4 + 16);
  unsigned int* hist = (unsigned int*)pmb_ws_alloc(h, (size_t)MAX_PASSES * RADIX * 4);
  unsigned long long* ctr = (unsigned long long*)pmb_ws_alloc(h, 64);  // kept, ticket, n_groups, big_n
  unsigned int* status = (unsigned int*)pmb_ws_alloc(h, 64);
  const int64_t max_tiles = (n + ST_TILE - 1) / ST_TILE;
  unsigned long long* lb = (unsigned long long*)pmb_ws_alloc(h, (size_t)std::max<int64_t>(max_tiles, 1) * RADIX * 8);
  if (!k0 || !k1 || !i0 || !i1 || !hist || !ctr || !status || !lb)
    return pmb_fail(h, PMB_E_OOM, "workspace exhausted (sort buffers)");
  PMB_CUDA(h, cudaMemsetAsync(hist, 0, (size_t)MAX_PASSES * RADIX * 4, h->stream));
  PMB_CUDA(h, cudaMemsetAsync(ctr, 0, 64, h->stream));
  PMB_CUDA(h, cudaMemsetAsync(status, 0, 64, h->stream));
  {
    EncodeParams E;
    memset(&E, 0, sizeof(E));
    E.q = q;
    E.L = L;
    E.passes = passes;
    E.n = n;
    E.keys = k0;
    E.cap = cap;
    E.idx = i0;
    E.lb = lb;
    E.ticket = ctr + 1;
    E.kept = ctr;
    E.hist = hist;
    E.status = status;
    PMB_CUDA(h, cudaMemsetAsync(lb, 0, (size_t)std::max<int64_t>(max_tiles, 1) * 8, h->stream));
    pmb_kernel_begin(h, "sort_encode");
    k_sort_encode<W><<<(unsigned)std::max<int64_t>(max_tiles, 1), ST_NT, 0, h->stream>>>(E);
    pmb_kernel_end(h);
    PMB_CUDA(h, cudaGetLastError());
  }
  std::vector<unsigned int> hh((size_t)std::max(passes, 1) * RADIX);
  unsigned long long kept = 0;
  unsigned int st0 = 0;
  PMB_CUDA(h, cudaMemcpyAsync(&kept, ctr, 8, cudaMemcpyDeviceToHost, h->stream));
  PMB_CUDA(h, cudaMemcpyAsync(&st0, status, 4, cudaMemcpyDeviceToHost, h->stream));
  if (passes) PMB_CUDA(h, cudaMemcpyAsync(hh.data(), hist, (size_t)passes * RADIX * 4, cudaMemcpyDeviceToHost, h->stream));
  PMB_CUDA(h, cudaStreamSynchronize(h->stream));
  if (st0 & PMB_ST_TIMEOUT) return pmb_fail(h, PMB_E_TIMEOUT, "a bounded device wait timed out (sort)");
  const int64_t m = (int64_t)kept;
  // LSD passes over the digits that are not the same for every key
  const int64_t tiles = (m + ST_TILE - 1) / ST_TILE;
  const size_t pass_smem = (size_t)ST_TILE * (8 * W + 4);
  PMB_CUDA(h, cudaFuncSetAttribute(k_sort_pass<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pass_smem));
  int done = 0;
  for (int p = 0; p < passes && m > 1; p++) {
    bool constant = false;
    for (int d = 0; d < RADIX; d++) constant |= hh[(size_t)p * RADIX + d] == (unsigned)m;
    if (constant) continue;
    PassParams P;
    P.kin = k0;
    P.kout = k1;
    P.iin = i0;
    P.iout = i1;
    P.cap = cap;
    P.n = m;
    P.shift = 8 * p;
    P.hist = hist + (size_t)p * RADIX;
    P.lb = lb;
    P.n_tiles = tiles;
    P.ticket = ctr + 1;
    P.status = status;
    PMB_CUDA(h, cudaMemsetAsync(lb, 0, (size_t)tiles * RADIX * 8, h->stream));
    PMB_CUDA(h, cudaMemsetAsync(ctr + 1, 0, 8, h->stream));
    pmb_kernel_begin(h, "sort_pass");
    k_sort_pass<W><<<(unsigned)tiles, ST_NT, pass_smem, h->stream>>>(P);
    pmb_kernel_end(h);
    PMB_CUDA(h, cudaGetLastError());
    std::swap(k0, k1);
    std::swap(i0, i1);
    done++;
  }
  // segment starts
  unsigned int* starts = (unsigned int*)pmb_ws_alloc(h, (size_t)(m + 2) * 4);
  if (!starts) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (segment starts)");
  unsigned long long ng = 0;
  if (m > 0) {
    StartsParams S;
    S.keys = k0;
    S.cap = cap;
    S.n = m;
    S.starts = starts;
    S.lb = lb;
    S.ticket = ctr + 1;
    S.n_groups = ctr + 2;
    S.status = status;
    PMB_CUDA(h, cudaMemsetAsync(lb, 0, (size_t)tiles * 8, h->stream));
    PMB_CUDA(h, cudaMemsetAsync(ctr + 1, 0, 8, h->stream));
    pmb_kernel_begin(h, "seg_starts");
    k_seg_starts<W><<<(unsigned)tiles, ST_NT, 0, h->stream>>>(S);
    pmb_kernel_end(h);
    PMB_CUDA(h, cudaGetLastError());
    unsigned int st = 0;
    PMB_CUDA(h, cudaMemcpyAsync(&ng, ctr + 2, 8, cudaMemcpyDeviceToHost, h->stream));
    PMB_CUDA(h, cudaMemcpyAsync(&st, status, 4, cudaMemcpyDeviceToHost, h->stream));
    PMB_CUDA(h, cudaStreamSynchronize(h->stream));
    if (st & PMB_ST_TIMEOUT) return pmb_fail(h, PMB_E_TIMEOUT, "a bounded device wait timed out (sort)");
  }
  // outputs
  const int n_out = q.n_keys + q.n_aggs;
  ReduceParams R;
  memset(&R, 0, sizeof(R));
  R.q = q;
  for (size_t w = 0; w < cq.rec_init.size() && w < 48; w++) R.ri.w[w] = cq.rec_init[w];
  R.L = L;
  R.cap = cap;
  R.idx = i0;
  R.starts = starts;
  R.n_groups = ctr + 2;
  R.big = (unsigned int*)pmb_ws_alloc(h, (size_t)(ng + 1) * 4);
  R.big_n = ctr + 3;
  R.status = status;
  if (!R.big) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (big groups)");
  const size_t vbytes = (size_t)((ng + 31) / 32 * 4) + 16;
  for (int c = 0; c < n_out; c++) {
    const int dt = r->columns[c].dtype;
    const size_t db = dt == PMB_BOOL ? vbytes : (size_t)ng * pmb_dtype_bytes(dt) + 16;
    R.out_data[c] = (uint8_t*)pmb_ws_alloc(h, db);
    R.out_valid[c] = (uint8_t*)pmb_ws_alloc(h, vbytes);
    if (!R.out_data[c] || !R.out_valid[c]) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (outputs)");
    PMB_CUDA(h, cudaMemsetAsync(R.out_valid[c], 0, vbytes, h->stream));
    if (dt == PMB_BOOL) PMB_CUDA(h, cudaMemsetAsync(R.out_data[c], 0, vbytes, h->stream));
  }
  for (int attempt = 0; ng > 0; attempt++) {
    R.keys = k0;
    PMB_CUDA(h, cudaMemsetAsync(ctr + 3, 0, 8, h->stream));
    PMB_CUDA(h, cudaMemsetAsync(status, 0, 64, h->stream));
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(((int64_t)ng + ST_NT - 1) / ST_NT, (int64_t)h->sm_count * 16));
    pmb_kernel_begin(h, "seg_reduce");
    if (q.rec_bytes <= 96) k_seg_reduce<W, 12><<<blocks, ST_NT, 0, h->stream>>>(R);
    else if (q.rec_bytes <= 192) k_seg_reduce<W, 24><<<blocks, ST_NT, 0, h->stream>>>(R);
    else k_seg_reduce<W, 48><<<blocks, ST_NT, 0, h->stream>>>(R);
    pmb_kernel_end(h);
    PMB_CUDA(h, cudaGetLastError());
    const size_t big_smem = (size_t)BIG_NT * q.rec_bytes;
    PMB_CUDA(h, cudaFuncSetAttribute(k_seg_reduce_big<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)big_smem));
    pmb_kernel_begin(h, "seg_reduce_big");
    k_seg_reduce_big<W><<<h->sm_count, BIG_NT, big_smem, h->stream>>>(R);
    pmb_kernel_end(h);
    PMB_CUDA(h, cudaGetLastError());
    unsigned int st[12];
    PMB_CUDA(h, cudaMemcpyAsync(st, status, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
    PMB_CUDA(h, cudaStreamSynchronize(h->stream));
    if (st[0] & PMB_ST_TIMEOUT) return pmb_fail(h, PMB_E_TIMEOUT, "a bounded device wait timed out (sort)");
    if (!(st[0] & PMB_ST_FXRANGE)) break;
    // a float sum left its fixed-point range: widen to the largest exponent seen; the sorted
    // order does not depend on it, so only the reduction runs again
    if (attempt >= 4) return pmb_fail(h, PMB_E_CUDA, "float-sum range did not converge");
    for (int i = 0; i < q.n_fields; i++) {
      DField& f = q.field[i];
      if (f.kind != F_SUM_FX || st[4 + f.fx_slot] == 0) continue;
      const int e = (int)st[4 + f.fx_slot] - 1022 + 1;
      if (e > q.fx_e[f.fx_slot]) {
        f.fx = (int16_t)(f.fx - (e - q.fx_e[f.fx_slot]));
        q.fx_e[f.fx_slot] = (int16_t)e;
      }
    }
    if (pmb_fx_to_dd(cq)) return PMB_RETRY_DD;
    R.q = q;
    for (int c = 0; c < n_out; c++) {
      PMB_CUDA(h, cudaMemsetAsync(R.out_valid[c], 0, vbytes, h->stream));
      if (r->columns[c].dtype == PMB_BOOL) PMB_CUDA(h, cudaMemsetAsync(R.out_data[c], 0, vbytes, h->stream));
    }
  }
  r->n_groups = (int64_t)ng;
  r->capacity = 0;
  r->strategy_used = PMB_STRATEGY_SORT;
  for (int c = 0; c < n_out; c++) {
    r->columns[c].data = R.out_data[c];
    r->columns[c].validity = R.out_valid[c];
  }
  (void)done;
  return PMB_OK;
}

}  // namespace

int pmb_groupby_sort(pmb_handle* h, CompiledQuery& cq, pmb_result* r) {
  DQuery& q = cq.dq;
  if (q.n_rows > 0xFFFFFFF0LL) return pmb_fail(h, PMB_E_UNSUPPORTED, "sort strategy: more than 2^32 rows");
  if (q.rec_bytes > 384) return pmb_fail(h, PMB_E_UNSUPPORTED, "sort strategy: group record above 384 bytes");
  SortKeyLayout L;
  memset(&L, 0, sizeof(L));
  L.n_keys = q.n_keys;
  for (int k = 0; k < q.n_keys; k++) {
    const DCol& C = q.col[q.key[k].col];
    L.col[k] = q.key[k].col;
    L.dtype[k] = C.dtype;
    L.elem[k] = C.elem;
    L.data[k] = C.data;
    L.valid[k] = C.valid;
  }
  // value ranges of the key columns
  RangeOut* ro = (RangeOut*)pmb_ws_alloc(h, sizeof(RangeOut));
  if (!ro) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (key ranges)");
  RangeOut init;
  memset(&init, 0, sizeof(init));
  for (int k = 0; k < PMB_MAX_KEYS; k++) init.lo[k] = ~0ULL;
  PMB_CUDA(h, cudaMemcpyAsync(ro, &init, sizeof(init), cudaMemcpyHostToDevice, h->stream));
  {
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((q.n_rows + ST_NT - 1) / ST_NT, (int64_t)h->sm_count * 8));
    pmb_kernel_begin(h, "key_range");
    k_key_range<<<blocks, ST_NT, 0, h->stream>>>(L, q.n_rows, ro);
    pmb_kernel_end(h);
    PMB_CUDA(h, cudaGetLastError());
  }
  RangeOut got;
  PMB_CUDA(h, cudaMemcpyAsync(&got, ro, sizeof(got), cudaMemcpyDeviceToHost, h->stream));
  PMB_CUDA(h, cudaStreamSynchronize(h->stream));
  int off = 0;
  for (int k = 0; k < q.n_keys; k++) {
    L.null_off[k] = -1;
    if (got.nulls[k]) L.null_off[k] = off++;
    int bits = 0;
    if (got.any[k]) {
      L.lo[k] = got.lo[k];
      const unsigned long long span = got.hi[k] - got.lo[k];
      while (bits < 64 && (span >> bits) != 0) bits++;
    }
    L.data_off[k] = off;
    L.data_bits[k] = bits;
    off += bits;
  }
  L.bits = off;
  L.words = off > 64 ? 2 : 1;
  if (off > 128) return pmb_fail(h, PMB_E_UNSUPPORTED, "sort strategy: packed key above 128 bits");
  return L.words == 1 ? run_sort<1>(h, cq, L, r) : run_sort<2>(h, cq, L, r);
}
