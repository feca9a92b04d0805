// pmb_jit_part.cuh — the aggregation step of the partitioned strategy, compiled at run time for
// one query signature (follows pmb_jit_skeleton.cuh's parameter block and the generated row
// functions in the same NVRTC source; JP_W, the words of a packed key, and JP_CAS64 are defined
// before it).
//
// Input: the kept rows as packed keys and row indices, ordered by partition (the top bits of the
// key hash), with the first row of every partition; work items are runs of whole partitions whose
// rows fit the shared-memory table. Persistent CTAs take items through a ticket. Per item:
//   1. rows are taken JP_R per thread: the key and row-index loads go out together, the key is
//      found or claimed in the table (one-word keys that cannot equal the all-ones EMPTY marker,
//      JP_CAS64: a CAS on the key word claims and publishes at once, no barrier; otherwise a CAS
//      on the slot's tag word claims, and a row that meets a slot being claimed retries it after
//      the next barrier instead of waiting), the
//      row's aggregated columns are gathered by row index (j_gather) and applied to the slot's
//      record with native 32-bit shared atomics (j_shared);
//   2. the claimed slots (listed in claim order) are written as dense groups: the packed key and
//      the record converted to the global-record layout (j_store_sg), after one atomic per item
//      on the group count; the table is reset for the next item.
// A prebuilt kernel turns the dense groups into the output columns.

struct JPart {
  JParams qp;                         // column pointers, float-sum ranges, status words
  const unsigned long long* keys;     // sorted packed keys, word-major (word w of row i at keys[w * kcap + i])
  unsigned long long kcap;
  const unsigned int* idx;            // row index of every sorted key
  const unsigned long long* pstart;   // first sorted row of every partition (and the end)
  const unsigned int* items;          // first partition of every work item (and the end)
  long long n_items;
  int slots;                          // table slots
  int pad;
  unsigned long long* ticket;
  unsigned long long* gkeys;          // dense groups: packed keys, word-major (stride gcap)
  unsigned char* grecs;               // and their records, J_REC bytes each
  unsigned long long gcap;
  unsigned long long* n_groups;
};

#define JP_R 2

__device__ __forceinline__ unsigned long long jp_hash(const unsigned long long* k) {
  unsigned long long h = pmb_fmix64(k[0]);
  if (JP_W > 1) h = pmb_fmix64(h ^ (k[JP_W - 1] + 0x9E3779B97F4A7C15ULL));
  return h;
}

extern "C" __global__ void __launch_bounds__(J_NT, 1) pmb_jit_part_agg(const __grid_constant__ JPart A) {
  extern __shared__ __align__(16) unsigned char sm[];
  const JParams& P = A.qp;
  const int S = A.slots, tid = threadIdx.x;
  unsigned int* tag = reinterpret_cast<unsigned int*>(sm);  // 0 empty, 1 claimed, 2 key published
  unsigned long long* tkey = reinterpret_cast<unsigned long long*>(sm + ((S * 4 + 15) & ~15));  // JP_W x S
  unsigned char* srec = reinterpret_cast<unsigned char*>(tkey + (size_t)JP_W * S);           // S x J_SREC
  unsigned short* list = reinterpret_cast<unsigned short*>(srec + (size_t)S * J_SREC);       // S
  __shared__ long long s_item;
  __shared__ unsigned long long s_base;
  __shared__ unsigned int s_total;  // claimed slots of the current item
  for (int i = tid; i < S; i += J_NT) {
    tag[i] = 0u;
    if (JP_CAS64) tkey[i] = 0xFFFFFFFFFFFFFFFFULL;
  }
  for (int w = tid; w < S * J_SREC_WORDS; w += J_NT) reinterpret_cast<unsigned int*>(srec)[w] = J_SIDENT[w % J_SREC_WORDS];
  if (tid == 0) s_total = 0u;
  for (;;) {
    __syncthreads();
    if (tid == 0) s_item = (long long)atomicAdd(A.ticket, 1ULL);
    __syncthreads();
    const long long it = s_item;
    if (it >= A.n_items) break;
    const long long ps = (long long)A.pstart[A.items[it]], pe = (long long)A.pstart[A.items[it + 1]];
    for (long long b = ps; b < pe; b += (long long)J_NT * JP_R) {
      unsigned long long k[JP_R][JP_W];
      unsigned slot[JP_R], row[JP_R], probes[JP_R];
      bool pending[JP_R], claimed[JP_R];
      int found[JP_R];
#pragma unroll
      for (int r = 0; r < JP_R; r++) {
        const long long i = b + (long long)r * J_NT + tid;
        pending[r] = i < pe;
        claimed[r] = false;
        found[r] = -1;
        probes[r] = 0;
        slot[r] = 0;
        row[r] = 0;
#pragma unroll
        for (int w = 0; w < JP_W; w++) k[r][w] = pending[r] ? A.keys[(unsigned long long)w * A.kcap + i] : 0ULL;
        if (pending[r]) row[r] = A.idx[i];
      }
#pragma unroll
      for (int r = 0; r < JP_R; r++)
        if (pending[r]) slot[r] = (unsigned)(((jp_hash(k[r]) & 0xFFFFFFFFULL) * (unsigned long long)S) >> 32);
#if JP_CAS64
      // the key word is the claim: no tag, no barrier
#pragma unroll
      for (int r = 0; r < JP_R; r++) {
        while (pending[r]) {
          const unsigned sl = slot[r];
          unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(&tkey[sl]);
          if (cur == 0xFFFFFFFFFFFFFFFFULL) {
            cur = atomicCAS(&tkey[sl], 0xFFFFFFFFFFFFFFFFULL, k[r][0]);
            if (cur == 0xFFFFFFFFFFFFFFFFULL) {
              claimed[r] = true;
              found[r] = (int)sl;
              pending[r] = false;
              break;
            }
          }
          if (cur == k[r][0]) {
            found[r] = (int)sl;
            pending[r] = false;
            break;
          }
          slot[r] = sl + 1 == (unsigned)S ? 0u : sl + 1;
          if (++probes[r] >= (unsigned)S) {
            atomicOr(P.status, PMB_ST_OVERFLOW);  // the item has more groups than the table
            pending[r] = false;
          }
        }
      }
#else
      for (int round = 0; round < 64; round++) {
        bool any = false;
#pragma unroll
        for (int r = 0; r < JP_R; r++) {
          while (pending[r]) {
            const unsigned sl = slot[r];
            unsigned tg = *reinterpret_cast<volatile unsigned int*>(&tag[sl]);
            if (tg == 0u) {
              if (atomicCAS(&tag[sl], 0u, 1u) == 0u) {
#pragma unroll
                for (int w = 0; w < JP_W; w++) tkey[(size_t)w * S + sl] = k[r][w];
                __threadfence_block();
                *reinterpret_cast<volatile unsigned int*>(&tag[sl]) = 2u;
                claimed[r] = true;
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
            for (int w = 0; w < JP_W; w++) eq &= reinterpret_cast<volatile unsigned long long*>(tkey)[(size_t)w * S + sl] == k[r][w];
            if (eq) {
              found[r] = (int)sl;
              pending[r] = false;
              break;
            }
            slot[r] = sl + 1 == (unsigned)S ? 0u : sl + 1;
            if (++probes[r] >= (unsigned)S) {
              atomicOr(P.status, PMB_ST_OVERFLOW);  // the item has more groups than the table
              pending[r] = false;
            }
          }
          any |= pending[r];
        }
        if (!__syncthreads_or(any)) break;
      }
#endif
      // the new groups join the item's list: one shared atomic per warp and row
      {
        const int lane = tid & 31;
#pragma unroll
        for (int r = 0; r < JP_R; r++) {
          const unsigned bl = __ballot_sync(0xffffffffu, claimed[r]);
          unsigned at = 0;
          if (bl && lane == __ffs(bl) - 1) at = atomicAdd(&s_total, (unsigned)__popc(bl));
          at = __shfl_sync(0xffffffffu, at, bl ? __ffs(bl) - 1 : 0);
          if (claimed[r]) list[at + __popc(bl & ((1u << lane) - 1u))] = (unsigned short)found[r];
        }
      }
      JRow rw[JP_R];
#pragma unroll
      for (int r = 0; r < JP_R; r++) {
        if (pending[r]) atomicOr(P.status, PMB_ST_OVERFLOW);
        if (found[r] >= 0) j_gather(P, (long long)row[r], rw[r]);
      }
#pragma unroll
      for (int r = 0; r < JP_R; r++) {
        if (found[r] < 0) continue;
        j_fxcheck(P, rw[r]);
        j_shared(P, srec + (size_t)found[r] * J_SREC, rw[r]);
      }
    }
    // the item is complete: its groups go to the dense group arrays
    __syncthreads();
    const unsigned total = s_total;
    if (tid == 0) s_base = total ? atomicAdd(A.n_groups, (unsigned long long)total) : 0ULL;
    __syncthreads();
    const unsigned long long base = s_base;
    for (unsigned li = tid; li < total; li += J_NT) {
      const int sl = list[li];
      const unsigned long long g = base + li;
      if (g < A.gcap) {
#pragma unroll
        for (int w = 0; w < JP_W; w++) A.gkeys[(unsigned long long)w * A.gcap + g] = tkey[(size_t)w * S + sl];
        j_store_sg(A.grecs + g * J_REC, srec + (size_t)sl * J_SREC);
      } else {
        atomicOr(P.status, PMB_ST_OVERFLOW);
      }
      tag[sl] = 0u;
      if (JP_CAS64) tkey[sl] = 0xFFFFFFFFFFFFFFFFULL;
      for (int w = 0; w < J_SREC_WORDS; w++) reinterpret_cast<unsigned int*>(srec + (size_t)sl * J_SREC)[w] = J_SIDENT[w];
    }
    if (tid == 0) s_total = 0u;  // every thread read it before the s_base barrier
    __syncthreads();
  }
}
