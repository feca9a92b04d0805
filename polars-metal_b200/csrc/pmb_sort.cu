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
//   5. with the run-time compiler: k_chunk_bounds cuts the sorted rows at segment starts into
//      work items that fit a shared-memory table, and the partitioned strategy's aggregation
//      (pmb_jit_part_agg, then k_part_finalize) reduces every item's segments there; without it,
//      k_seg_reduce — one thread per group folds its rows into a group record and writes the
//      output row; groups of more than 256 rows go to k_seg_reduce_big (one CTA per group).
// Both use the hash path's records and finalisation, so every strategy gives identical results,
// exact float sums included. The order of the output groups is not specified.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "pmb_groupby.h"
#include "pmb_jit.h"

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
  // one key column at a time with scalar accumulators (per-key arrays indexed at run time would
  // live in local memory); four rows per step, their loads issued together
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int k = 0; k < L.n_keys; k++) {
    unsigned long long lo = ~0ULL, hi = 0;
    unsigned nul = 0, any = 0;
    const uint8_t* data = L.data[k];
    const uint8_t* valid = L.valid[k];
    const int elem = L.elem[k], dtype = L.dtype[k];
    for (int64_t r0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r0 < n; r0 += 4 * stride) {
      uint64_t b[4];
      bool v[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int64_t r = r0 + u * stride;
        v[u] = r < n && pmb_valid_bit(valid, r);
        b[u] = r < n ? pmb_load_bits(data, elem, r) : 0;
        nul |= (r < n && !v[u]) ? 1u : 0u;
      }
#pragma unroll
      for (int u = 0; u < 4; u++) {
        if (!v[u]) continue;
        const unsigned long long o = ordered_bits(b[u], dtype);
        lo = o < lo ? o : lo;
        hi = o > hi ? o : hi;
        any = 1;
      }
    }
    for (int o = 16; o; o >>= 1) {
      const unsigned long long x = __shfl_xor_sync(0xffffffffu, lo, o), y = __shfl_xor_sync(0xffffffffu, hi, o);
      lo = x < lo ? x : lo;
      hi = y > hi ? y : hi;
      nul |= __shfl_xor_sync(0xffffffffu, nul, o);
      any |= __shfl_xor_sync(0xffffffffu, any, o);
    }
    if ((threadIdx.x & 31) == 0) {
      if (any) {
        atomicMin(&out->lo[k], lo);
        atomicMax(&out->hi[k], hi);
        atomicOr(&out->any[k], 1u);
      }
      if (nul) atomicOr(&out->nulls[k], 1u);
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

// hash of a packed key for the partitioned strategy: its top bits are the partition, its low 32
// bits the slot in the partition's shared-memory table
template <int W>
__device__ __forceinline__ unsigned long long part_hash(const PKey<W>& k) {
  unsigned long long h = pmb_fmix64(k.w[0]);
  if (W > 1) h = pmb_fmix64(h ^ (k.w[W - 1] + 0x9E3779B97F4A7C15ULL));
  return h;
}

// digit of a pass: key bits (sort strategy) or hash bits (partitioned strategy)
template <int W>
__device__ __forceinline__ unsigned pass_digit(const PKey<W>& k, int shift, bool hashed) {
  return hashed ? (unsigned)((part_hash<W>(k) >> shift) & 0xFFu) : digit_of<W>(k, shift);
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
  int hashed;                  // digits of the key hash (partitioned strategy)
  int shift0;                  // bit of pass 0's digit; pass p uses shift0 + 8p
  unsigned int* phist;         // partitioned strategy: rows per partition (2^pb counters), or null
  int pb;
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
    for (int p = 0; p < E.passes; p++) atomicAdd(&s_hist[p][pass_digit<W>(k, E.shift0 + 8 * p, E.hashed)], 1u);
    if (E.phist) atomicAdd(&E.phist[part_hash<W>(k) >> (64 - E.pb)], 1u);
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
  int hashed;  // digits of the key hash (partitioned strategy)
};

// One stable LSD pass over 8 bits at `shift`. Look-back states are tile-major (tile * 256 + digit),
// so the 32 digits of a warp read one predecessor's states in one coalesced access. Per-warp digit
// counts are 16-bit (at most 512 keys per warp), which with 4 CTAs per SM keeps the shared memory
// of a CTA under a quarter of the SM's.
template <int W>
__global__ void __launch_bounds__(ST_NT, 4) k_sort_pass(const __grid_constant__ PassParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned long long* s_key = reinterpret_cast<unsigned long long*>(smem);       // W x ST_TILE
  unsigned int* s_idx = reinterpret_cast<unsigned int*>(s_key + W * ST_TILE);   // ST_TILE
  __shared__ unsigned short s_whist[ST_NT / 32][RADIX];
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
    dg[j] = e < P.n ? (unsigned short)pass_digit<W>(k, P.shift, P.hashed) : (unsigned short)RADIX;
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
      s_whist[warp][d] = (unsigned short)(old + __popc(peers));
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
      s_whist[w][d] = (unsigned short)acc;
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
    const unsigned long long pre = pmb_lookback_strided(P.lb + d, tile, RADIX, acc, P.status);
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
    const unsigned d = pass_digit<W>(k, P.shift, P.hashed);
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

// ---------------------------------------------------------------- partitioned strategy
// After the hash-digit passes the kept rows are ordered by partition (the top `pb` bits of the key
// hash), so every group's rows lie inside one partition; the encode pass counted the rows of every
// partition, so their offsets are exact. k_part_agg: persistent CTAs take work items (runs of
// consecutive partitions) and aggregate one partition at a time in a shared-memory table (slot claim by a tag word, records in the global-record layout updated by
// apply_row_shared, values gathered by row index). At the end of each partition the occupied
// slots are compacted and written straight to the output columns (one atomic per partition for
// the output rows; validity words built in shared memory). No global hash table is involved.
constexpr int PA_NT = 1024;
constexpr int PA_R = 2;   // rows per thread and step
constexpr int PA_UC = 4;  // aggregated columns whose loads are issued together

struct PartParams {
  DQuery q;
  RecInit ri;
  SortKeyLayout L;
  const unsigned long long* keys;  // sorted packed keys, word-major (stride cap)
  uint64_t cap;
  const unsigned int* idx;         // their row indices
  int64_t m;                       // kept rows
  int pb;                          // partition bits
  const unsigned long long* pstart;  // 2^pb + 1: first row of every partition
  const unsigned int* items;       // n_items + 1: first partition of every work item (whole partitions
                                   // whose rows, an upper bound of their groups, fit the table)
  int64_t n_items;
  int slots;                       // shared table slots
  int n_out;
  int stage_bytes;                 // one row's aggregated columns, staged per thread
  unsigned int used;               // columns the aggregates read (bit per column)
  int n_used;
  int32_t ucol[PMB_MAX_COLS];      // those columns, in order
  int32_t sdoff[PMB_MAX_COLS];     // a column's value in the stage
  int32_t svoff[PMB_MAX_COLS];     // its validity byte in the stage
  unsigned long long* ticket;
  unsigned long long* n_groups;    // output rows claimed
  int64_t out_cap;
  unsigned int* status;
  uint8_t* out_data[PMB_MAX_OUT];
  uint8_t* out_valid[PMB_MAX_OUT];
};

template <int W>
__device__ __forceinline__ PKey<W> pa_key(const PartParams& A, int64_t i) {
  PKey<W> k;
#pragma unroll
  for (int w = 0; w < W; w++) k.w[w] = A.keys[(uint64_t)w * A.cap + i];
  return k;
}
// shared-memory layout of k_part_agg for `slots` slots
struct PaLayout {
  size_t tag, key, rec, list, vb, db, stage, bytes;
};
__host__ __device__ inline PaLayout pa_layout(int slots, int W, int rec_bytes, int n_out, int stage_bytes) {
  PaLayout o;
  const size_t words = (size_t)slots / 32 + 2;
  o.tag = 0;
  o.key = ((size_t)slots * 4 + 15) & ~(size_t)15;
  o.rec = o.key + (size_t)slots * 8 * W;
  o.list = o.rec + (size_t)slots * rec_bytes;
  o.vb = (o.list + (size_t)slots * 2 + 15) & ~(size_t)15;
  o.db = o.vb + (size_t)n_out * words * 4;
  o.stage = (o.db + (size_t)PMB_MAX_KEYS * words * 4 + 15) & ~(size_t)15;
  o.bytes = o.stage + (size_t)PA_NT * stage_bytes;
  return o;
}

template <int W>
__global__ void __launch_bounds__(PA_NT, 1) k_part_agg(const __grid_constant__ PartParams A) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int S = A.slots, rb = A.q.rec_bytes, rw = rb / 8;
  const PaLayout Ly = pa_layout(S, W, rb, A.n_out, A.stage_bytes);
  unsigned int* tag = reinterpret_cast<unsigned int*>(smem + Ly.tag);  // 0 empty, 1 claimed, 2 key published
  unsigned long long* tkey = reinterpret_cast<unsigned long long*>(smem + Ly.key);  // W x S
  uint8_t* trec = smem + Ly.rec;
  unsigned short* list = reinterpret_cast<unsigned short*>(smem + Ly.list);
  const int nwords = S / 32 + 2;
  unsigned int* vb = reinterpret_cast<unsigned int*>(smem + Ly.vb);  // n_out x nwords
  unsigned int* db = reinterpret_cast<unsigned int*>(smem + Ly.db);  // n_keys x nwords (Bool keys)
  uint8_t* stage = smem + Ly.stage + (size_t)threadIdx.x * A.stage_bytes;
  __shared__ long long s_item;
  __shared__ unsigned long long s_base;
  __shared__ unsigned s_total;  // claimed slots of the current partition
  const int tid = threadIdx.x;
  bool has_fx = false;
  for (int f = 0; f < A.q.n_fields; f++) has_fx |= A.q.field[f].kind == F_SUM_FX;
  for (int i = tid; i < S; i += PA_NT) {
    tag[i] = 0u;
    for (int w = 0; w < rw; w++) reinterpret_cast<uint64_t*>(trec + (size_t)i * rb)[w] = A.ri.w[w];
  }
  for (int i = tid; i < (A.n_out + PMB_MAX_KEYS) * nwords; i += PA_NT) vb[i] = 0u;  // vb and db are adjacent
  if (tid == 0) s_total = 0u;
  for (;;) {
    __syncthreads();
    if (tid == 0) s_item = (long long)atomicAdd(A.ticket, 1ULL);
    __syncthreads();
    const long long it = s_item;
    if (it >= A.n_items) break;
    {
      // the item's partitions: rows [ps, pe)
      const int64_t ps = (int64_t)A.pstart[A.items[it]], pe = (int64_t)A.pstart[A.items[it + 1]];
      for (int64_t b = ps; b < pe; b += (int64_t)PA_NT * PA_R) {
        // PA_R rows per thread; their key and row-index loads go out together
        PKey<W> k[PA_R];
        unsigned slot[PA_R], row[PA_R], probes[PA_R];
        bool pending[PA_R];
        int found[PA_R];
#pragma unroll
        for (int r = 0; r < PA_R; r++) {
          const int64_t i = b + (int64_t)r * PA_NT + tid;
          pending[r] = i < pe;
          found[r] = -1;
          probes[r] = 0;
          slot[r] = 0;
          row[r] = 0;
          if (pending[r]) {
            k[r] = pa_key<W>(A, i);
            row[r] = A.idx[i];
          }
        }
#pragma unroll
        for (int r = 0; r < PA_R; r++)
          if (pending[r]) slot[r] = (unsigned)(((part_hash<W>(k[r]) & 0xFFFFFFFFULL) * (unsigned long long)S) >> 32);
        // find or claim the keys' slots. A claimer publishes its key before the next barrier, so a
        // row that meets a slot being claimed tries that slot again after the barrier instead of
        // waiting for it (a wait could stall on a claimer in its own warp)
        for (int round = 0; round < 64; round++) {
          bool any = false;
#pragma unroll
          for (int r = 0; r < PA_R; r++) {
            while (pending[r]) {
              const unsigned sl = slot[r];
              unsigned tg = *reinterpret_cast<volatile unsigned int*>(&tag[sl]);
              if (tg == 0u) {
                if (atomicCAS(&tag[sl], 0u, 1u) == 0u) {
#pragma unroll
                  for (int w = 0; w < W; w++) tkey[(size_t)w * S + sl] = k[r].w[w];
                  __threadfence_block();
                  *reinterpret_cast<volatile unsigned int*>(&tag[sl]) = 2u;
                  list[atomicAdd(&s_total, 1u)] = (unsigned short)sl;  // the item's groups, in claim order
                  found[r] = (int)sl;
                  pending[r] = false;
                  break;
                }
                tg = *reinterpret_cast<volatile unsigned int*>(&tag[sl]);
              }
              if (tg != 2u) break;  // being claimed: this slot again after the barrier
              __threadfence_block();
              bool eq = true;
#pragma unroll
              for (int w = 0; w < W; w++) eq &= reinterpret_cast<volatile unsigned long long*>(tkey)[(size_t)w * S + sl] == k[r].w[w];
              if (eq) {
                found[r] = (int)sl;
                pending[r] = false;
                break;
              }
              slot[r] = sl + 1 == (unsigned)S ? 0u : sl + 1;
              if (++probes[r] >= (unsigned)S) {
                atomicOr(A.status, PMB_ST_OVERFLOW);  // the item has more groups than the table
                pending[r] = false;
              }
            }
            any |= pending[r];
          }
          if (!__syncthreads_or(any)) break;
        }
        // the rows' aggregated columns: the first PA_UC columns of both rows are loaded together,
        // then every row is staged (one copy of each value) and applied to its record
        uint64_t vals[PA_R][PA_UC];
        unsigned vmask[PA_R];
#pragma unroll
        for (int r = 0; r < PA_R; r++) {
          vmask[r] = 0u;
          if (pending[r]) atomicOr(A.status, PMB_ST_OVERFLOW);
#pragma unroll
          for (int u = 0; u < PA_UC; u++) {
            vals[r][u] = 0;
            if (found[r] >= 0 && u < A.n_used) {
              const DCol& C = A.q.col[A.ucol[u]];
              vals[r][u] = pmb_load_bits(C.data, C.elem, row[r]);
              if (C.valid && pmb_valid_bit(C.valid, row[r])) vmask[r] |= 1u << u;
            }
          }
        }
        auto put = [&](int c, uint64_t v, bool ok) {
          const DCol& C = A.q.col[c];
          uint8_t* d = stage + A.sdoff[c];
          switch (C.elem) {
            case 8: *reinterpret_cast<uint64_t*>(d) = v; break;
            case 4: *reinterpret_cast<uint32_t*>(d) = (uint32_t)v; break;
            case 2: *reinterpret_cast<uint16_t*>(d) = (uint16_t)v; break;
            default: *d = (uint8_t)v; break;
          }
          if (C.valid) stage[A.svoff[c]] = ok ? 1 : 0;
        };
#pragma unroll
        for (int r = 0; r < PA_R; r++) {
          if (found[r] < 0) continue;
#pragma unroll
          for (int u = 0; u < PA_UC; u++)
            if (u < A.n_used) put(A.ucol[u], vals[r][u], (vmask[r] >> u) & 1u);
          for (int u = PA_UC; u < A.n_used; u++) {
            const DCol& C = A.q.col[A.ucol[u]];
            put(A.ucol[u], pmb_load_bits(C.data, C.elem, row[r]), C.valid && pmb_valid_bit(C.valid, row[r]));
          }
          const TileCtx ts{stage, A.sdoff, A.svoff, 0};
          if (has_fx) fx_range_check(A.q, ts, 0, A.status);
          apply_row_shared(A.q, ts, trec + (size_t)found[r] * rb, 0);
        }
      }
      // the partition is complete: its groups (the claimed slots) go to the output
      __syncthreads();
      const unsigned total = s_total;
      if (tid == 0) s_base = total ? atomicAdd(A.n_groups, (unsigned long long)total) : 0ULL;
      __syncthreads();
      const unsigned long long base = s_base, a0 = base & ~31ULL;
      for (unsigned li = tid; li < total; li += PA_NT) {
        const unsigned long long p = base + li;
        if ((int64_t)p >= A.out_cap) {
          atomicOr(A.status, PMB_ST_OVERFLOW);
          continue;
        }
        const int sl = list[li];
        const unsigned rbit = (unsigned)(p - a0);
        PKey<W> k;
#pragma unroll
        for (int w = 0; w < W; w++) k.w[w] = tkey[(size_t)w * S + sl];
        const uint8_t* rec = trec + (size_t)sl * rb;
        int oc = 0;
        for (int c = 0; c < A.q.n_keys; c++, oc++) {
          uint64_t v = 0;
          const bool valid = unpack_sort_key<W>(A.L, k, c, v);
          const int dt = A.L.dtype[c];
          if (dt == PMB_BOOL) {
            if (valid && v) atomicOr(&db[c * nwords + (rbit >> 5)], 1u << (rbit & 31));
          } else {
            store_bits(A.out_data[oc], pmb_dtype_bytes(dt), (int64_t)p, v);
          }
          if (valid) atomicOr(&vb[oc * nwords + (rbit >> 5)], 1u << (rbit & 31));
        }
        for (int ag = 0; ag < A.q.n_aggs; ag++, oc++) {
          const DAggOut& Ag = A.q.agg[ag];
          bool valid = true;
          uint64_t bits = 0;
          finalize_agg(A.q, Ag, rec, valid, bits);
          store_bits(A.out_data[oc], pmb_dtype_bytes(Ag.out_dtype), (int64_t)p, bits);
          if (valid) atomicOr(&vb[oc * nwords + (rbit >> 5)], 1u << (rbit & 31));
        }
      }
      __syncthreads();
      // bitmap words into the outputs, then the table and the bitmaps are reset
      const int nw = total ? (int)((base - a0 + total + 31) / 32) : 0;
      for (int i = tid; i < A.n_out * nw; i += PA_NT) {
        const int oc = i / nw, w = i % nw;
        if ((int64_t)((a0 >> 5) + w) * 32 >= A.out_cap + 32) continue;
        const unsigned v = vb[oc * nwords + w];
        if (v) atomicOr(reinterpret_cast<unsigned int*>(A.out_valid[oc]) + (a0 >> 5) + w, v);
        vb[oc * nwords + w] = 0u;
        if (oc < A.q.n_keys && A.L.dtype[oc] == PMB_BOOL) {
          const unsigned d = db[oc * nwords + w];
          if (d) atomicOr(reinterpret_cast<unsigned int*>(A.out_data[oc]) + (a0 >> 5) + w, d);
          db[oc * nwords + w] = 0u;
        }
      }
      for (unsigned li = tid; li < total; li += PA_NT) {
        const int sl = list[li];
        tag[sl] = 0u;
        for (int w = 0; w < rw; w++) reinterpret_cast<uint64_t*>(trec + (size_t)sl * rb)[w] = A.ri.w[w];
      }
      if (tid == 0) s_total = 0u;  // every thread read it before the s_base barrier
      __syncthreads();
    }
  }
}

// dense groups of the run-time compiled partitioned aggregation (packed keys, global-layout
// records) into the output columns, group g into output row g
struct PartFinParams {
  ReduceParams R;
  const unsigned long long* gkeys;  // word-major, stride gcap
  const uint8_t* grecs;
  uint64_t gcap;
};

template <int W>
__global__ void __launch_bounds__(ST_NT) k_part_finalize(const __grid_constant__ PartFinParams F) {
  const int64_t ng = (int64_t)*F.R.n_groups;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  // every lane of a warp runs the same number of iterations (warp-wide bit setting)
  const int64_t span = (ng + stride - 1) / stride * stride;
  for (int64_t g0 = (int64_t)blockIdx.x * blockDim.x; g0 < span; g0 += stride) {
    const int64_t g = g0 + threadIdx.x;
    const int64_t p_first = g0 + (threadIdx.x & ~31);
    const bool have = g < ng;
    PKey<W> k{};
    if (have)
      for (int w = 0; w < W; w++) k.w[w] = F.gkeys[(uint64_t)w * F.gcap + g];
    write_group<W, true>(F.R, g, p_first, have, k, have ? F.grecs + (uint64_t)g * F.R.q.rec_bytes : nullptr);
  }
}

// the per-thread stage of k_part_agg: the aggregated columns' values (widest first, each aligned
// to its size), then one validity byte per nullable column; returns its bytes (a multiple of 8)
static int pa_stage(const DQuery& q, unsigned* used, int32_t* sdoff, int32_t* svoff) {
  *used = 0;
  for (int f = 0; f < q.n_fields; f++)
    if (q.field[f].kind != F_LEN) *used |= 1u << q.field[f].col;
  int off = 0;
  for (int e = 8; e >= 1; e /= 2)
    for (int c = 0; c < q.n_cols; c++)
      if (((*used >> c) & 1u) && std::max<int>(q.col[c].elem, 1) == e) {
        sdoff[c] = off;
        off += e;
      }
  for (int c = 0; c < q.n_cols; c++)
    if (((*used >> c) & 1u) && q.col[c].valid) svoff[c] = off++;
  return (off + 7) & ~7;
}

// run_part_agg's answer when the sort strategy should reduce its segments itself
constexpr int kSegReduce = -77;

// work-item boundaries for aggregating sorted rows in shared-memory tables: chunk c starts at the
// first segment start at or after c * chunk (m at the end), so no group is cut
__global__ void k_chunk_bounds(const unsigned int* __restrict__ starts, unsigned long long ng, int64_t m, int64_t chunk,
                               int64_t n_chunks, unsigned long long* __restrict__ out) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c > n_chunks) return;
  const int64_t x = c * chunk;
  if (c == n_chunks || x >= m) {
    out[c] = (unsigned long long)m;
    return;
  }
  unsigned long long lo = 0, hi = ng;
  while (lo < hi) {
    const unsigned long long mid = (lo + hi) >> 1;
    if ((int64_t)starts[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  out[c] = lo < ng ? (unsigned long long)starts[lo] : (unsigned long long)m;
}

// float sums that left their fixed-point range: widen to the largest exponent seen (the sorted
// order does not depend on it); true when a column must switch to double-double instead
static bool widen_fx(CompiledQuery& cq, const unsigned int* st) {
  DQuery& q = cq.dq;
  for (int i = 0; i < q.n_fields; i++) {
    DField& f = q.field[i];
    if (f.kind != F_SUM_FX || st[4 + f.fx_slot] == 0) continue;
    const int e = (int)st[4 + f.fx_slot] - 1022 + 1;
    if (e > q.fx_e[f.fx_slot]) {
      f.fx = (int16_t)(f.fx - (e - q.fx_e[f.fx_slot]));
      q.fx_e[f.fx_slot] = (int16_t)e;
    }
  }
  return pmb_fx_to_dd(cq);
}

template <int W>
int run_sort(pmb_handle* h, CompiledQuery& cq, const SortKeyLayout& L, pmb_result* r, int64_t part_groups);

// the aggregation of the partitioned strategy over keys / row indices sorted by partition
template <int W>
int run_part_agg(pmb_handle* h, CompiledQuery& cq, const SortKeyLayout& L, pmb_result* r, const unsigned long long* keys,
                 const unsigned int* idx, uint64_t cap, int64_t m, int pb, const std::vector<unsigned int>& counts,
                 int slots, int64_t groups,
                 unsigned long long* ctr, unsigned int* status, int strategy = PMB_STRATEGY_PARTITIONED) {
  DQuery& q = cq.dq;
  const int n_out = q.n_keys + q.n_aggs;
  PartParams A;
  memset(&A, 0, sizeof(A));
  for (size_t w = 0; w < cq.rec_init.size() && w < 48; w++) A.ri.w[w] = cq.rec_init[w];
  A.L = L;
  A.keys = keys;
  A.cap = cap;
  A.idx = idx;
  A.m = m;
  A.pb = pb;
  // partition offsets, and work items: runs of whole partitions whose rows (an upper bound of
  // their groups) stay within 70% of the table, at least one partition each
  const unsigned long long lim = (unsigned long long)(0.7 * slots);
  std::vector<unsigned long long> pstart(counts.size() + 1, 0);
  std::vector<unsigned int> items(1, 0);
  unsigned long long run = 0;
  for (size_t p = 0; p < counts.size(); p++) {
    pstart[p + 1] = pstart[p] + counts[p];
    if (run > 0 && run + counts[p] > lim) {
      items.push_back((unsigned)p);
      run = 0;
    }
    run += counts[p];
  }
  if (run > 0 || items.size() == 1) items.push_back((unsigned)counts.size());
  if ((int64_t)pstart.back() != m) return pmb_fail(h, PMB_E_CUDA, "partition counts do not add up");
  unsigned long long* d_pstart = (unsigned long long*)pmb_ws_alloc(h, pstart.size() * 8);
  unsigned int* d_items = (unsigned int*)pmb_ws_alloc(h, items.size() * 4);
  if (!d_pstart || !d_items) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (partition offsets)");
  PMB_CUDA(h, cudaMemcpyAsync(d_pstart, pstart.data(), pstart.size() * 8, cudaMemcpyHostToDevice, h->stream));
  PMB_CUDA(h, cudaMemcpyAsync(d_items, items.data(), items.size() * 4, cudaMemcpyHostToDevice, h->stream));
  A.pstart = d_pstart;
  A.items = d_items;
  A.n_items = (int64_t)items.size() - 1;
  A.slots = slots;
  A.n_out = n_out;
  A.stage_bytes = pa_stage(q, &A.used, A.sdoff, A.svoff);
  for (int c = 0; c < q.n_cols; c++)
    if ((A.used >> c) & 1u) A.ucol[A.n_used++] = c;
  A.ticket = ctr + 1;
  A.n_groups = ctr + 2;
  A.status = status;
  const size_t smem = pa_layout(slots, W, q.rec_bytes, n_out, A.stage_bytes).bytes;
  PMB_CUDA(h, cudaFuncSetAttribute(k_part_agg<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int64_t out_cap = std::min<int64_t>(std::max<int64_t>(m, 1), 2 * groups + 65536);
  for (int attempt = 0;; attempt++) {
    if (attempt >= 6) return pmb_fail(h, PMB_E_CUDA, "partitioned strategy did not converge");
    const WsMark mark = pmb_ws_mark(h);
    const size_t vbytes = (size_t)((out_cap + 31) / 32 * 4) + 16;
    for (int c = 0; c < n_out; c++) {
      const int dt = r->columns[c].dtype;
      const size_t dbytes = dt == PMB_BOOL ? vbytes : (size_t)out_cap * pmb_dtype_bytes(dt) + 16;
      A.out_data[c] = (uint8_t*)pmb_ws_alloc(h, dbytes);
      A.out_valid[c] = (uint8_t*)pmb_ws_alloc(h, vbytes);
      if (!A.out_data[c] || !A.out_valid[c]) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (outputs)");
      PMB_CUDA(h, cudaMemsetAsync(A.out_valid[c], 0, vbytes, h->stream));
      if (dt == PMB_BOOL) PMB_CUDA(h, cudaMemsetAsync(A.out_data[c], 0, vbytes, h->stream));
    }
    A.q = q;
    A.out_cap = out_cap;
    PMB_CUDA(h, cudaMemsetAsync(ctr + 1, 0, 16, h->stream));
    PMB_CUDA(h, cudaMemsetAsync(status, 0, 64, h->stream));
    unsigned long long ng = 0;
    unsigned int st[12] = {0};
    // the run-time compiled aggregation writes dense groups that a prebuilt kernel finalises;
    // without NVRTC (or for a signature it cannot take) the prebuilt kernel does both
    JitPlan J;
    cudaKernel_t jk = nullptr;
    if (m > 0 && pmb_jit_enabled(1LL << 40) && pmb_jit_part_kernel(h, cq, W, L.bits < 64, &J, &jk) != PMB_OK) {
      jk = nullptr;  // the prebuilt kernel instead (the compile error stays readable in pmb_last_error)
    }
    unsigned long long* gkeys = nullptr;
    uint8_t* grecs = nullptr;
    if (jk) {
      gkeys = (unsigned long long*)pmb_ws_alloc(h, (size_t)W * out_cap * 8 + 16);
      grecs = (uint8_t*)pmb_ws_alloc(h, (size_t)out_cap * q.rec_bytes + 16);
      if (!gkeys || !grecs) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (groups)");
    }
    if (m > 0) {
      const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(A.n_items, h->sm_count));
      if (jk) {
        JPartH JA;
        memset(&JA, 0, sizeof(JA));
        for (int c = 0; c < q.n_cols; c++) {
          JA.qp.col_data[c] = q.col[c].data;
          JA.qp.col_valid[c] = q.col[c].valid;
        }
        JA.qp.n_rows = q.n_rows;
        JA.qp.status = status;
        for (int f = 0; f < q.n_fields; f++)
          if (q.field[f].kind == F_SUM_FX) {
            JA.qp.fx[q.field[f].fx_slot] = q.field[f].fx;
            JA.qp.fx_e[q.field[f].fx_slot] = q.fx_e[q.field[f].fx_slot];
          }
        JA.keys = keys;
        JA.kcap = cap;
        JA.idx = idx;
        JA.pstart = A.pstart;
        JA.items = A.items;
        JA.n_items = A.n_items;
        JA.slots = slots;
        JA.ticket = A.ticket;
        JA.gkeys = gkeys;
        JA.grecs = grecs;
        JA.gcap = (unsigned long long)out_cap;
        JA.n_groups = A.n_groups;
        const size_t jsmem = (((size_t)slots * 4 + 15) & ~(size_t)15) + (size_t)slots * (8 * W + J.srec + 2);
        PMB_CUDA(h, cudaFuncSetAttribute((const void*)jk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)jsmem));
        void* args[] = {&JA};
        pmb_kernel_begin(h, "part_agg");
        PMB_CUDA(h, cudaLaunchKernel((const void*)jk, dim3(grid), dim3(J.nt), args, jsmem, h->stream));
        pmb_kernel_end(h);
      } else {
        pmb_kernel_begin(h, "part_agg");
        k_part_agg<W><<<grid, PA_NT, smem, h->stream>>>(A);
        pmb_kernel_end(h);
        PMB_CUDA(h, cudaGetLastError());
      }
      PMB_CUDA(h, cudaMemcpyAsync(&ng, ctr + 2, 8, cudaMemcpyDeviceToHost, h->stream));
      PMB_CUDA(h, cudaMemcpyAsync(st, status, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
      PMB_CUDA(h, cudaStreamSynchronize(h->stream));
      if (jk && !(st[0] & (PMB_ST_TIMEOUT | PMB_ST_FXRANGE | PMB_ST_OVERFLOW)) && ng > 0) {
        PartFinParams F;
        memset(&F, 0, sizeof(F));
        F.R.q = q;
        F.R.L = L;
        F.R.n_groups = A.n_groups;
        for (int c = 0; c < n_out; c++) {
          F.R.out_data[c] = A.out_data[c];
          F.R.out_valid[c] = A.out_valid[c];
        }
        F.gkeys = gkeys;
        F.grecs = grecs;
        F.gcap = (uint64_t)out_cap;
        const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(((int64_t)ng + ST_NT - 1) / ST_NT, (int64_t)h->sm_count * 16));
        pmb_kernel_begin(h, "part_finalize");
        k_part_finalize<W><<<blocks, ST_NT, 0, h->stream>>>(F);
        pmb_kernel_end(h);
        PMB_CUDA(h, cudaGetLastError());
      }
    }
    if (st[0] & PMB_ST_TIMEOUT) return pmb_fail(h, PMB_E_TIMEOUT, "a bounded device wait timed out (partitioned)");
    if (st[0] & PMB_ST_FXRANGE) {
      if (widen_fx(cq, st)) return PMB_RETRY_DD;
      pmb_ws_release(h, mark);
      continue;
    }
    if (st[0] & PMB_ST_OVERFLOW) {
      pmb_ws_release(h, mark);
      if ((int64_t)ng > out_cap) {  // more groups than output rows: the exact upper bound next
        out_cap = std::max<int64_t>(m, 1);
        continue;
      }
      // a partition had more groups than its table: the sort strategy instead (the sort's own
      // segment reduce when the caller is the sort)
      if (strategy == PMB_STRATEGY_SORT) return kSegReduce;
      PMB_CUDA(h, cudaMemsetAsync(ctr, 0, 64, h->stream));
      return run_sort<W>(h, cq, L, r, 0);
    }
    r->n_groups = (int64_t)ng;
    r->capacity = out_cap;
    r->strategy_used = strategy;
    for (int c = 0; c < n_out; c++) {
      r->columns[c].data = A.out_data[c];
      r->columns[c].validity = A.out_valid[c];
    }
    return PMB_OK;
  }
}

template <int W>
int run_sort(pmb_handle* h, CompiledQuery& cq, const SortKeyLayout& L, pmb_result* r, int64_t part_groups) {
  DQuery& q = cq.dq;
  const int64_t n = q.n_rows;
  const int n_out = q.n_keys + q.n_aggs;
  // partitioned strategy: the largest shared table that fits, and 2^8 or 2^16 partitions so that
  // a partition holds about a third of a table
  int pb = 0, slots = 0;
  if (part_groups > 0) {
    unsigned used;
    int32_t sd[PMB_MAX_COLS], sv[PMB_MAX_COLS];
    const int stage = pa_stage(q, &used, sd, sv);
    for (slots = 4096; slots >= 256; slots /= 2)
      if (pa_layout(slots, W, q.rec_bytes, n_out, stage).bytes + 2048 <= (size_t)h->max_smem_optin) break;
    if (slots < 256) return pmb_fail(h, PMB_E_UNSUPPORTED, "partitioned strategy: group record too large");
    // twice the estimate: an undersized partition count overflows tables (and falls back to the
    // sort), an oversized one costs one more pass
    pb = 2 * part_groups * 3 / slots + 1 <= 256 ? 8 : 16;
  }
  const int passes = part_groups > 0 ? pb / 8 : std::max(0, (L.bits + 7) / 8);
  const uint64_t cap = (uint64_t)n;
  unsigned long long* k0 = (unsigned long long*)pmb_ws_alloc(h, (size_t)W * cap * 8 + 16);
  unsigned long long* k1 = (unsigned long long*)pmb_ws_alloc(h, (size_t)W * cap * 8 + 16);
  unsigned int* i0 = (unsigned int*)pmb_ws_alloc(h, (size_t)cap * 4 + 16);
  unsigned int* i1 = (unsigned int*)pmb_ws_alloc(h, (size_t)cap * 4 + 16);
  unsigned int* hist = (unsigned int*)pmb_ws_alloc(h, (size_t)MAX_PASSES * RADIX * 4);
  const size_t n_parts = part_groups > 0 ? (size_t)1 << pb : 0;
  unsigned int* phist = n_parts ? (unsigned int*)pmb_ws_alloc(h, n_parts * 4) : nullptr;
  if (n_parts && !phist) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (partition counts)");
  if (n_parts) PMB_CUDA(h, cudaMemsetAsync(phist, 0, n_parts * 4, h->stream));
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
    E.hashed = part_groups > 0;
    E.shift0 = part_groups > 0 ? 64 - pb : 0;
    E.phist = phist;
    E.pb = pb;
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
  std::vector<unsigned int> ph(n_parts);
  if (n_parts) PMB_CUDA(h, cudaMemcpyAsync(ph.data(), phist, n_parts * 4, cudaMemcpyDeviceToHost, h->stream));
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
    P.shift = (part_groups > 0 ? 64 - pb : 0) + 8 * p;
    P.hashed = part_groups > 0;
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
  if (part_groups > 0) return run_part_agg<W>(h, cq, L, r, k0, i0, cap, m, pb, ph, slots, part_groups, ctr, status);
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
  // with the run-time compiler, the sorted rows are cut at segment starts into work items that fit
  // a shared-memory table, and the partitioned strategy's aggregation reduces them (values
  // gathered once per row, records in shared memory); otherwise thread-per-segment reduces below
  if (ng > 0 && pmb_jit_enabled(1LL << 40)) {
    unsigned used;
    int32_t sd[PMB_MAX_COLS], sv[PMB_MAX_COLS];
    const int stage = pa_stage(q, &used, sd, sv);
    int slots = 4096;
    for (; slots >= 256; slots /= 2)
      if (pa_layout(slots, W, q.rec_bytes, n_out, stage).bytes + 2048 <= (size_t)h->max_smem_optin) break;
    if (slots >= 256) {
      const int64_t chunk = (int64_t)(0.7 * slots);
      const int64_t n_chunks = (m + chunk - 1) / chunk;
      unsigned long long* bounds = (unsigned long long*)pmb_ws_alloc(h, (size_t)(n_chunks + 1) * 8);
      if (!bounds) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (segment chunks)");
      pmb_kernel_begin(h, "chunk_bounds");
      k_chunk_bounds<<<(unsigned)((n_chunks + 1 + 255) / 256), 256, 0, h->stream>>>(starts, ng, m, chunk, n_chunks, bounds);
      pmb_kernel_end(h);
      PMB_CUDA(h, cudaGetLastError());
      std::vector<unsigned long long> hb((size_t)n_chunks + 1);
      PMB_CUDA(h, cudaMemcpyAsync(hb.data(), bounds, hb.size() * 8, cudaMemcpyDeviceToHost, h->stream));
      PMB_CUDA(h, cudaStreamSynchronize(h->stream));
      std::vector<unsigned int> counts((size_t)n_chunks);
      for (int64_t c = 0; c < n_chunks; c++) counts[c] = (unsigned)(hb[c + 1] - hb[c]);
      const WsMark mark = pmb_ws_mark(h);
      const int rc = run_part_agg<W>(h, cq, L, r, k0, i0, cap, m, 0, counts, slots, (int64_t)ng, ctr, status,
                                     PMB_STRATEGY_SORT);
      if (rc != kSegReduce) return rc;
      pmb_ws_release(h, mark);
      PMB_CUDA(h, cudaMemcpyAsync(ctr + 2, &ng, 8, cudaMemcpyHostToDevice, h->stream));  // the group count again
    }
  }
  // outputs
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
    if (widen_fx(cq, st)) return PMB_RETRY_DD;
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

int pmb_groupby_sort(pmb_handle* h, CompiledQuery& cq, pmb_result* r, int64_t part_groups) {
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
  return L.words == 1 ? run_sort<1>(h, cq, L, r, part_groups) : run_sort<2>(h, cq, L, r, part_groups);
}

// Stable LSD sort of (key, row index) pairs for callers outside the group-by (the output sort):
// the same onesweep pass kernel, over the 8-bit digits 0 .. n_passes-1 of W-word keys (word-major,
// stride cap). hist_host holds every pass's digit counts of all n keys (also at hist_dev); a digit
// that one value fills is skipped. On return *k and *i are the sorted buffers (the inputs or the
// alternates).
int pmb_sort_pairs(pmb_handle* h, int W, unsigned long long** k, unsigned long long** k_alt, unsigned int** i,
                   unsigned int** i_alt, uint64_t cap, int64_t n, int n_passes, const unsigned int* hist_dev,
                   const unsigned int* hist_host) {
  if (W != 1 && W != 2) return pmb_fail(h, PMB_E_INVALID, "sort: key of 1 or 2 words");
  if (n_passes > MAX_PASSES) return pmb_fail(h, PMB_E_INVALID, "sort: more than 16 digit passes");
  if (n <= 1 || n_passes <= 0) return PMB_OK;
  const int64_t tiles = (n + ST_TILE - 1) / ST_TILE;
  unsigned long long* lb = (unsigned long long*)pmb_ws_alloc(h, (size_t)tiles * RADIX * 8);
  unsigned long long* ticket = (unsigned long long*)pmb_ws_alloc(h, 64);
  unsigned int* status = (unsigned int*)pmb_ws_alloc(h, 64);
  if (!lb || !ticket || !status) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (sort passes)");
  PMB_CUDA(h, cudaMemsetAsync(status, 0, 64, h->stream));
  const size_t pass_smem = (size_t)ST_TILE * (8 * W + 4);
  if (W == 1) PMB_CUDA(h, cudaFuncSetAttribute(k_sort_pass<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pass_smem));
  else PMB_CUDA(h, cudaFuncSetAttribute(k_sort_pass<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pass_smem));
  for (int p = 0; p < n_passes; p++) {
    bool constant = false;
    for (int d = 0; d < RADIX; d++) constant |= hist_host[(size_t)p * RADIX + d] == (unsigned)n;
    if (constant) continue;
    PassParams P;
    P.kin = *k;
    P.kout = *k_alt;
    P.iin = *i;
    P.iout = *i_alt;
    P.cap = cap;
    P.n = n;
    P.shift = 8 * p;
    P.hashed = 0;
    P.hist = hist_dev + (size_t)p * RADIX;
    P.lb = lb;
    P.n_tiles = tiles;
    P.ticket = ticket;
    P.status = status;
    PMB_CUDA(h, cudaMemsetAsync(lb, 0, (size_t)tiles * RADIX * 8, h->stream));
    PMB_CUDA(h, cudaMemsetAsync(ticket, 0, 8, h->stream));
    pmb_kernel_begin(h, "sort_pass");
    if (W == 1) k_sort_pass<1><<<(unsigned)tiles, ST_NT, pass_smem, h->stream>>>(P);
    else k_sort_pass<2><<<(unsigned)tiles, ST_NT, pass_smem, h->stream>>>(P);
    pmb_kernel_end(h);
    PMB_CUDA(h, cudaGetLastError());
    std::swap(*k, *k_alt);
    std::swap(*i, *i_alt);
  }
  unsigned int st = 0;
  PMB_CUDA(h, cudaMemcpyAsync(&st, status, 4, cudaMemcpyDeviceToHost, h->stream));
  PMB_CUDA(h, cudaStreamSynchronize(h->stream));
  if (st & PMB_ST_TIMEOUT) return pmb_fail(h, PMB_E_TIMEOUT, "a bounded device wait timed out (sort)");
  return PMB_OK;
}
