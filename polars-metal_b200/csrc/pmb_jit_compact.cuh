// pmb_jit_compact.cuh — the top-level filter's compaction compiled at run time for one query
// signature (NVRTC): every row's values read once into registers with literal column offsets and
// dtypes (j_cload, generated), its predicate taken from them (j_ckeep), then the kept rows of every
// output column scattered in row order from the same registers (j_cscatter). This text follows
// pmb_device.cuh, the parameter block of pmb_jit_skeleton.cuh and the generated row functions.
//
// Structure (as the prebuilt k_compact, pmb_filter.cu): a CTA takes tiles of JC_TILE rows in
// ticket order; every warp ballots its rows' verdicts, the CTA's warp counts give each warp its
// offset inside the tile, warp 0 looks the tile's output base up with a warp-parallel decoupled
// look-back, then every lane writes its kept rows. Validity (and Bool data) bits are OR-ed into
// 32-bit words; a warp's 32 consecutive outputs span at most two words.

#define JC_NT 256
#define JC_PER 4  // a thread's rows stay in registers from the verdict to the scatter
#define JC_TILE (JC_NT * JC_PER)

struct JCParams {
  const unsigned char* col_data[16];
  const unsigned char* col_valid[16];
  long long n_rows;
  unsigned long long* lb;      // look-back states, one per tile
  unsigned long long* ticket;  // tile ticket
  unsigned long long* n_out;   // rows kept (written by the last tile)
  unsigned int* status;
  unsigned char* out_data[16];
  unsigned int* out_valid[16];
};

__device__ __forceinline__ void jc_set_bits(unsigned int* words, long long p, long long p_first, bool bit) {
  const long long w0 = p_first >> 5;
  const unsigned m0 = __reduce_or_sync(0xffffffffu, (bit && (p >> 5) == w0) ? (1u << (p & 31)) : 0u);
  const unsigned m1 = __reduce_or_sync(0xffffffffu, (bit && (p >> 5) == w0 + 1) ? (1u << (p & 31)) : 0u);
  if ((threadIdx.x & 31) == 0) {
    if (m0) atomicOr(&words[w0], m0);
    if (m1) atomicOr(&words[w0 + 1], m1);
  }
}

// the look-back of pmb_internal.cuh for a whole warp (NVRTC sees only this text)
__device__ __forceinline__ unsigned long long jc_lookback_warp(unsigned long long* status, long long tile,
                                                               unsigned long long count, unsigned int* st) {
  const unsigned long long VAL = (1ULL << 62) - 1;
  const int lane = threadIdx.x & 31;
  if (tile == 0) {
    if (lane == 0) atomicExch(&status[0], (2ULL << 62) | count);
    return 0;
  }
  if (lane == 0) atomicExch(&status[tile], (1ULL << 62) | count);
  unsigned long long excl = 0;
  long long top = tile - 1;
  unsigned spins = 0;
  for (;;) {
    const long long t = top - lane;
    const unsigned long long s = t >= 0 ? *((volatile unsigned long long*)&status[t]) : (2ULL << 62);
    const unsigned flag = (unsigned)(s >> 62);
    const unsigned incl = __ballot_sync(0xffffffffu, flag == 2u), none = __ballot_sync(0xffffffffu, flag == 0u);
    const int first = incl ? __ffs(incl) - 1 : 32;
    const unsigned need = first == 32 ? 0xffffffffu : (0xffffffffu >> (31 - first));
    if (none & need) {
      if (++spins > PMB_SPIN_LIMIT) {
        if (lane == 0) atomicOr(st, PMB_ST_TIMEOUT);
        return 0;
      }
      continue;
    }
    unsigned long long v = lane <= first ? (s & VAL) : 0ULL;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    excl += v;
    if (first < 32) break;
    top -= 32;
  }
  if (lane == 0) atomicExch(&status[tile], (2ULL << 62) | (excl + count));
  return excl;
}

extern "C" __global__ void __launch_bounds__(JC_NT) pmb_jit_compact(const __grid_constant__ JCParams P) {
  __shared__ int s_cnt[JC_PER][JC_NT / 32];
  __shared__ int s_off[JC_PER][JC_NT / 32];
  __shared__ long long s_tile;
  __shared__ unsigned long long s_base;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_tile = (long long)atomicAdd(P.ticket, 1ULL);
  __syncthreads();
  const long long tile = s_tile;
  const long long row0 = tile * JC_TILE;
  unsigned keepm = 0;  // bit j: row row0 + j * JC_NT + tid is kept
  JCRow x[JC_PER];
#pragma unroll
  for (int j = 0; j < JC_PER; j++) {
    const long long r = row0 + (long long)j * JC_NT + tid;
    if (r < P.n_rows) j_cload(P, r, x[j]);
  }
#pragma unroll
  for (int j = 0; j < JC_PER; j++) {
    const long long r = row0 + (long long)j * JC_NT + tid;
    const bool k = r < P.n_rows && j_ckeep(x[j]);
    if (k) keepm |= 1u << j;
    const unsigned b = __ballot_sync(0xffffffffu, k);
    if (lane == 0) s_cnt[j][warp] = __popc(b);
  }
  __syncthreads();
  if (warp == 0) {
    int acc = 0;
    if (lane == 0) {
      for (int j = 0; j < JC_PER; j++)
        for (int w = 0; w < JC_NT / 32; w++) {
          s_off[j][w] = acc;
          acc += s_cnt[j][w];
        }
    }
    acc = __shfl_sync(0xffffffffu, acc, 0);
    const unsigned long long base = jc_lookback_warp(P.lb, tile, (unsigned long long)acc, P.status);
    if (lane == 0) {
      s_base = base;
      if (tile == (long long)gridDim.x - 1) *P.n_out = base + acc;
    }
  }
  __syncthreads();
  const unsigned long long base = s_base;
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int j = 0; j < JC_PER; j++) {
    const bool k = (keepm >> j) & 1u;
    const unsigned b = __ballot_sync(0xffffffffu, k);
    if (b == 0) continue;
    const long long p_first = (long long)(base + (unsigned long long)s_off[j][warp]);
    const long long p = p_first + __popc(b & lt);
    j_cscatter(P, x[j], k, p, p_first);
  }
}
