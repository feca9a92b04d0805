// pmb_device.cuh — device helpers shared by the prebuilt kernels and the kernels compiled at
// run time (NVRTC). Only built-in types and intrinsics: no host headers, so NVRTC can compile it.
#pragma once

#ifdef __CUDACC_RTC__
typedef unsigned long long uint64_t;
typedef long long int64_t;
typedef unsigned int uint32_t;
typedef int int32_t;
typedef unsigned short uint16_t;
typedef short int16_t;
typedef unsigned char uint8_t;
typedef signed char int8_t;
#else
#include <stdint.h>
#endif

#define PMB_EMPTY64 0xFFFFFFFFFFFFFFFFULL

// status bits written by kernels into the call's device status word
#define PMB_ST_OVERFLOW 1u  // a hash table ran out of probes / capacity: rehash
#define PMB_ST_TIMEOUT 2u   // a bounded wait gave up
#define PMB_ST_BADARG 4u    // a device-side argument check failed

// bounded spins: iterations before a wait gives up and reports PMB_ST_TIMEOUT
#define PMB_SPIN_LIMIT (1u << 24)

// ----------------------------------------------------------------------------- device helpers
__device__ __forceinline__ uint32_t pmb_smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(pmb_smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(pmb_smem_u32(bar)), "r"(bytes)
               : "memory");
}
// 1-D bulk copy global -> shared (TMA engine), completion counted on `bar`.
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          pmb_smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(pmb_smem_u32(bar))
      : "memory");
}
// L2 eviction policy for inputs that are read once: evict them first, so that the hash tables the
// same kernel updates stay resident in L2
__device__ __forceinline__ uint64_t pmb_policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
// bulk_g2s with an L2 cache policy
__device__ __forceinline__ void bulk_g2s_hint(void* dst, const void* src, uint32_t bytes, uint64_t* bar,
                                              uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          pmb_smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(pmb_smem_u32(bar)), "l"(policy)
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(pmb_smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// try_wait with a suspend-time hint: the thread may sleep up to `ns` nanoseconds for the phase
// instead of spinning, which leaves the issue slots to the warps that have work
__device__ __forceinline__ bool mbar_try_wait_hint(uint64_t* bar, uint32_t parity, uint32_t ns) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(pmb_smem_u32(bar)), "r"(parity), "r"(ns)
      : "memory");
  return ok != 0;
}
// bounded wait; returns false on timeout
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (uint32_t it = 0; it < PMB_SPIN_LIMIT; it++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// bounded wait that sleeps between tests (at most PMB_SPIN_LIMIT tests of at most `ns` each)
__device__ __forceinline__ bool mbar_wait_bounded_sleep(uint64_t* bar, uint32_t parity, uint32_t ns) {
  for (uint32_t it = 0; it < PMB_SPIN_LIMIT; it++)
    if (mbar_try_wait_hint(bar, parity, ns)) return true;
  return false;
}

// MurmurHash3 64-bit finalizer (Appleby, public domain)
// Fire-and-forget updates of global-table records. With PMB_EXPLICIT_RED (the batched kernel's
// source defines it) they are explicit red.global reductions: there the compiler had emitted
// atomics with a return value (104M such L2 sectors for 60M rows) and the explicit form took the
// kernel from 19.0 to 15.2 ms on the 500M-row batch. Elsewhere the compiler already emits
// reductions for unused atomic results, and the hash kernel measured 3% faster with its choice.
#if defined(PMB_EXPLICIT_RED) && PMB_EXPLICIT_RED
__device__ __forceinline__ void pmb_red_add(unsigned long long* p, unsigned long long v) {
  asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "l"(v) : "memory");
}
__device__ __forceinline__ void pmb_red_add(unsigned int* p, unsigned int v) {
  asm volatile("red.relaxed.gpu.global.add.u32 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "r"(v) : "memory");
}
__device__ __forceinline__ void pmb_red_or(unsigned int* p, unsigned int v) {
  asm volatile("red.relaxed.gpu.global.or.b32 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "r"(v) : "memory");
}
__device__ __forceinline__ void pmb_red_or(unsigned long long* p, unsigned long long v) {
  asm volatile("red.relaxed.gpu.global.or.b64 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "l"(v) : "memory");
}
__device__ __forceinline__ void pmb_red_min(long long* p, long long v) {
  asm volatile("red.relaxed.gpu.global.min.s64 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "l"(v) : "memory");
}
__device__ __forceinline__ void pmb_red_max(long long* p, long long v) {
  asm volatile("red.relaxed.gpu.global.max.s64 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "l"(v) : "memory");
}
__device__ __forceinline__ void pmb_red_min(unsigned long long* p, unsigned long long v) {
  asm volatile("red.relaxed.gpu.global.min.u64 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "l"(v) : "memory");
}
__device__ __forceinline__ void pmb_red_max(unsigned long long* p, unsigned long long v) {
  asm volatile("red.relaxed.gpu.global.max.u64 [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "l"(v) : "memory");
}
#else
__device__ __forceinline__ void pmb_red_add(unsigned long long* p, unsigned long long v) { atomicAdd(p, v); }
__device__ __forceinline__ void pmb_red_add(unsigned int* p, unsigned int v) { atomicAdd(p, v); }
__device__ __forceinline__ void pmb_red_or(unsigned int* p, unsigned int v) { atomicOr(p, v); }
__device__ __forceinline__ void pmb_red_or(unsigned long long* p, unsigned long long v) { atomicOr(p, v); }
__device__ __forceinline__ void pmb_red_min(long long* p, long long v) { atomicMin(p, v); }
__device__ __forceinline__ void pmb_red_max(long long* p, long long v) { atomicMax(p, v); }
__device__ __forceinline__ void pmb_red_min(unsigned long long* p, unsigned long long v) { atomicMin(p, v); }
__device__ __forceinline__ void pmb_red_max(unsigned long long* p, unsigned long long v) { atomicMax(p, v); }
#endif

// Global-table records update their 4-byte words (counters, float-sum flags) with 64-bit atomics
// on the 8-byte word that holds them, so that two 4-byte fields sharing a word (a counter in an
// exact float sum's spare word beside its flags) never meet atomics of different sizes.
// Counters stay below 2^32 - 1 (a call has fewer rows), so an add never carries into the other half.
__device__ __forceinline__ void pmb_rec_add32(unsigned char* rec, int off, unsigned int v) {
  pmb_red_add(reinterpret_cast<unsigned long long*>(rec + (off & ~7)), (unsigned long long)v << ((off & 4) ? 32 : 0));
}
__device__ __forceinline__ void pmb_rec_or32(unsigned char* rec, int off, unsigned int v) {
  pmb_red_or(reinterpret_cast<unsigned long long*>(rec + (off & ~7)), (unsigned long long)v << ((off & 4) ? 32 : 0));
}

__host__ __device__ __forceinline__ uint64_t pmb_fmix64(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return k;
}

// a second 32-bit mixer, independent of the key hash (C. Wellons' "lowbias32", public domain):
// the alternative bucket of a two-choice bucketed table
__host__ __device__ __forceinline__ uint32_t pmb_mix32b(uint32_t a) {
  a ^= a >> 16;
  a *= 0x7feb352dU;
  a ^= a >> 15;
  a *= 0x846ca68bU;
  a ^= a >> 16;
  return a;
}
// MurmurHash3 32-bit finalizer (Appleby, public domain)
__host__ __device__ __forceinline__ uint32_t pmb_fmix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x85ebca6bU;
  x ^= x >> 13;
  x *= 0xc2b2ae35U;
  x ^= x >> 16;
  return x;
}

// slot of hash h in a table of `cap` slots, any cap: the high word of h * cap (Lemire's
// multiply-shift range reduction), so capacities need not be powers of two
__device__ __forceinline__ uint64_t pmb_slot(uint64_t h, uint64_t cap) { return __umul64hi(h, cap); }

// Two's complement accumulators of 32-bit words in shared memory, updated with native 32-bit
// atomics (64-bit adds on shared memory are compare-and-swap loops on this GPU). The thread whose
// addition wraps a word adds the carry into the next word, so the words always hold the exact
// total modulo 2^96 (2^64) once all additions are done, in any interleaving.
__device__ __forceinline__ void pmb_s_add96(unsigned* w, unsigned l0, unsigned l1, unsigned l2) {
  unsigned c = 0;
  if (l0) {
    unsigned o = atomicAdd(&w[0], l0);
    c = (o + l0) < o;
  }
  unsigned t1 = l1 + c;
  unsigned c1 = t1 < c;  // l1 = 0xFFFFFFFF with an incoming carry
  if (t1) {
    unsigned o = atomicAdd(&w[1], t1);
    c1 |= (o + t1) < o;
  }
  unsigned t2 = l2 + c1;
  if (t2) atomicAdd(&w[2], t2);
}
__device__ __forceinline__ void pmb_s_add64(unsigned* w, unsigned lo, unsigned hi) {
  unsigned c = 0;
  if (lo) {
    unsigned o = atomicAdd(&w[0], lo);
    c = (o + lo) < o;
  }
  unsigned t = hi + c;
  if (t) atomicAdd(&w[1], t);
}
// d += s for accumulators owned by one thread
__device__ __forceinline__ void pmb_s_fold96(unsigned* d, const unsigned* s) {
  unsigned long long a = (unsigned long long)d[0] + s[0];
  unsigned long long b = (unsigned long long)d[1] + s[1] + (a >> 32);
  d[0] = (unsigned)a;
  d[1] = (unsigned)b;
  d[2] = d[2] + s[2] + (unsigned)(b >> 32);
}
__device__ __forceinline__ void pmb_s_fold64(unsigned* d, const unsigned* s) {
  unsigned long long a = (unsigned long long)d[0] + s[0];
  d[0] = (unsigned)a;
  d[1] = d[1] + s[1] + (unsigned)(a >> 32);
}

// total-order key of a double: monotone in IEEE order for non-NaN values (-0.0 < +0.0)
__device__ __forceinline__ long long pmb_f64_key(double x) {
  long long b = __double_as_longlong(x);
  return b ^ ((b >> 63) & 0x7FFFFFFFFFFFFFFFLL);
}
__device__ __forceinline__ double pmb_f64_from_key(long long k) {
  long long b = k ^ ((k >> 63) & 0x7FFFFFFFFFFFFFFFLL);
  return __longlong_as_double(b);
}

// Exact-to-double-double accumulation: atomicAdd returns the old partial sum, so the rounding
// error of that very addition is recovered with TwoSum (Knuth) and added into the low word.
__device__ __forceinline__ void dd_atomic_add(double* hi, double* lo, double x) {
  double old = atomicAdd(hi, x);
  double s = old + x;
  if (!isfinite(s)) return;
  double bp = s - old;
  double err = (old - (s - bp)) + (x - bp);
  if (err != 0.0) atomicAdd(lo, err);
}

// TwoSum accumulation when one thread owns the record (no atomics)
__device__ __forceinline__ void dd_plain_add(double* hi, double* lo, double x) {
  double old = *hi;
  double s = old + x;
  *hi = s;
  if (!isfinite(s)) return;
  double bp = s - old;
  *lo += (old - (s - bp)) + (x - bp);
}


// ----------------------------------------------------------------------------- exact float sums
// A finite double x is summed as the integer X = trunc(x * 2^F), a two's complement value split
// into 32-bit limbs; integer additions are exact and their order does not matter. F is chosen per
// column so that |x| < 2^(94 - F) and the sums of all rows stay in range; a value outside that
// range is reported (status bit + its exponent) and the call is re-run with a wider range. NaN /
// +inf / -inf are tracked as flag bits beside the sum.
#define PMB_ST_FXRANGE 8u  // a float-sum value exceeded its column's fixed-point range
#define PMB_FX_NAN 1u
#define PMB_FX_PINF 2u
#define PMB_FX_NINF 4u

// biased exponent field of x (0 for zero / subnormal, 2047 for inf / NaN)
__device__ __forceinline__ int pmb_fx_expo(double x) { return (int)((__double_as_longlong(x) >> 52) & 0x7FF); }

// non-finite flag of x (0 for finite values)
__device__ __forceinline__ unsigned pmb_fx_flag(double x) {
  long long b = __double_as_longlong(x);
  if (((b >> 52) & 0x7FF) != 0x7FF) return 0u;
  if (b & 0xFFFFFFFFFFFFFLL) return PMB_FX_NAN;
  return b < 0 ? PMB_FX_NINF : PMB_FX_PINF;
}

// true when the finite x satisfies |x| < 2^E
__device__ __forceinline__ bool pmb_fx_in_range(double x, int E) { return pmb_fx_expo(x) < E + 1023; }

// limbs of trunc(x * 2^F) for a finite x with |x * 2^F| < 2^94
__device__ __forceinline__ void pmb_fx_split(double x, int F, unsigned long long& l0, unsigned long long& l1,
                                             unsigned long long& l2) {
  long long b = __double_as_longlong(x);
  int ex = (int)((b >> 52) & 0x7FF);
  unsigned long long m = (unsigned long long)b & 0xFFFFFFFFFFFFFULL;
  if (ex) m |= 1ULL << 52;
  else ex = 1;
  int sh = ex - 1075 + F;  // X = m * 2^sh, sh <= 41 when x fits
  unsigned long long lo, hi;
  if (sh >= 0) {
    lo = m << sh;
    hi = sh ? (m >> (64 - sh)) : 0ULL;
  } else {
    lo = sh > -64 ? (m >> (-sh)) : 0ULL;
    hi = 0ULL;
  }
  if (b < 0) {  // two's complement negation of the 128-bit (hi, lo)
    lo = ~lo + 1ULL;
    hi = ~hi + (lo == 0ULL ? 1ULL : 0ULL);
  }
  l0 = lo & 0xFFFFFFFFULL;
  l1 = lo >> 32;
  l2 = (unsigned long long)(long long)(int)(unsigned)hi;
}

// The global table keeps an exact float sum in two 64-bit words: the sum of the values' low 32
// bits (unsigned; up to 2^32 additions fit) and the sum of the values shifted right by 32
// (signed), so one value costs two fire-and-forget adds. These are the two words of one value.
__device__ __forceinline__ void pmb_fx_words(double x, int F, unsigned long long& w0, unsigned long long& w1) {
  unsigned long long l0, l1, l2;
  pmb_fx_split(x, F, l0, l1, l2);
  w0 = l0;
  w1 = l1 + (l2 << 32);
}
