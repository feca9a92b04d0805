// pmb_learned.cu — the learned strategy selector: sketch features of a 4096-row key sample, and a
// small MLP (24 -> 64 -> 64 -> 5, fp32, CUDA cores) with hand-written forward, backward and Adam
// kernels. The network is trained on timings and exact group counts that the engine measures on
// synthetic tables (polars_b200/selector.py); its outputs are four strategy scores (shared-memory
// hash, global hash, sort, partitioned) and log2 of the group count. The reference routes by a row threshold and an estimated-cardinality gate
// (crates/polars-metal-core/src/router/cost.rs:35-52, crates/polars-metal-kernels/src/groupby.rs:475-486);
// that plain heuristic (pmb_choose_strategy) stays the fallback.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pmb_groupby.h"

namespace {

constexpr int NF = PMB_SELECTOR_FEATURES;
constexpr int NH = PMB_SELECTOR_HIDDEN;
constexpr int NO = PMB_SELECTOR_OUTPUTS;
constexpr int NS = PMB_SELECTOR_STRATEGIES;  // outputs 0..NS-1: strategy scores; output NS: log2(groups)
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + NH * NF, OFF_W2 = OFF_B1 + NH, OFF_B2 = OFF_W2 + NH * NH,
              OFF_W3 = OFF_B2 + NH, OFF_B3 = OFF_W3 + NO * NH, N_PARAMS = OFF_B3 + NO;
static_assert(N_PARAMS == PMB_SELECTOR_PARAMS, "parameter layout");

constexpr int SAMPLE = 4096;
constexpr int F_NT = 1024;
constexpr int TSLOTS = 8192;  // sample counts: slots (count << 32 | 32-bit key fingerprint), dynamic smem
constexpr int HLL = 256;
constexpr int BUCKETS = 1024;

struct FeatParams {
  DQuery q;
  float* out;  // NF floats
};

__device__ __forceinline__ float lg2p1(double x) { return (float)log2(x + 1.0); }

// sample i of query q (rows evenly spaced over the input): its key hash, never 0, or 0 when the
// filter drops the row or i is past the sample; `nul` tells whether a key column is null there.
// One thread per sample, so the sample's loads are all in flight at once.
__device__ __forceinline__ void sample_one(const DQuery& q, int i, unsigned long long& hv, unsigned char& nul) {
  hv = 0ULL;
  nul = 0;
  const int64_t n = q.n_rows;
  const int m = (int)(n < SAMPLE ? n : SAMPLE);
  if (i >= m) return;
  const TileCtx t{nullptr, nullptr, nullptr, 0};
  const int64_t r = (int64_t)((__int128)i * n / m);  // evenly spaced rows
  if (q.prog.n_ops > 0 && !eval_keep(q, t, r)) return;
  bool anynull = false;
  for (int k = 0; k < q.n_keys; k++) anynull |= !tc_isvalid(q, t, q.key[k].col, r);
  unsigned long long lo, hi = 0;
  if (q.key_bits > 64) {
    Key128 kk = pack_key128(q, t, r);
    lo = kk.lo;
    hi = kk.hi;
  } else {
    lo = pack_key64(q, t, r);
  }
  hv = pmb_fmix64(lo ^ pmb_fmix64(hi + 0x9E3779B97F4A7C15ULL)) | 1ULL;  // never 0 (empty)
  nul = anynull ? 1 : 0;
}

// the features of query q into out[NF] from its samples (hs, ns: SAMPLE entries written by
// sample_one); called by one whole CTA of F_NT threads
__device__ __forceinline__ void features_body(const DQuery& q, const unsigned long long* __restrict__ hs,
                                              const unsigned char* __restrict__ ns, float* out) {
  extern __shared__ unsigned long long s_slot[];  // TSLOTS
  __shared__ unsigned int s_hll[HLL];
  __shared__ unsigned int s_bkt[BUCKETS];
  __shared__ unsigned int s_acc[16];
  const int tid = threadIdx.x;
  for (int i = tid; i < TSLOTS; i += F_NT) s_slot[i] = 0ULL;
  for (int i = tid; i < HLL; i += F_NT) s_hll[i] = 0u;
  for (int i = tid; i < BUCKETS; i += F_NT) s_bkt[i] = 0u;
  if (tid < 16) s_acc[tid] = 0u;
  __syncthreads();
  const int64_t n = q.n_rows;
  const int m = (int)(n < SAMPLE ? n : SAMPLE);
  const bool pred = q.prog.n_ops > 0;
  for (int i = tid; i < m; i += F_NT) {
    const unsigned long long h = hs[i];
    if (h == 0ULL) continue;  // dropped by the filter
    atomicAdd(&s_acc[0], 1u);  // kept
    if (ns[i]) atomicAdd(&s_acc[1], 1u);
    // HyperLogLog register: index from the top 8 bits, rank of the rest
    const unsigned reg = (unsigned)(h >> 56);
    const unsigned rank = (unsigned)__clzll((h << 8) | 0xFFULL) + 1u;
    atomicMax(&s_hll[reg], rank);
    atomicAdd(&s_bkt[(h >> 20) & (BUCKETS - 1)], 1u);
    // exact counts by 32-bit fingerprint (a collision among 4096 samples is rare and only blurs a
    // feature); a slot holds count << 32 | fingerprint
    const unsigned fp = (unsigned)(h >> 32) | 1u;
    unsigned s = (unsigned)(h >> 11) & (TSLOTS - 1);
    for (int p = 0; p < TSLOTS; p++) {
      unsigned long long cur = s_slot[s];
      if (cur == 0ULL) {
        cur = atomicCAS(&s_slot[s], 0ULL, (1ULL << 32) | fp);
        if (cur == 0ULL) break;
      }
      if ((unsigned)cur == fp) {
        atomicAdd(&s_slot[s], 1ULL << 32);
        break;
      }
      s = (s + 1) & (TSLOTS - 1);
    }
  }
  __syncthreads();
  // frequency profile of the sample keys
  for (int i = tid; i < TSLOTS; i += F_NT) {
    const unsigned c = (unsigned)(s_slot[i] >> 32);
    if (!c) continue;
    atomicAdd(&s_acc[2], 1u);  // distinct
    if (c == 1) atomicAdd(&s_acc[3], 1u);
    else if (c == 2) atomicAdd(&s_acc[4], 1u);
    else if (c <= 4) atomicAdd(&s_acc[5], 1u);
    else if (c <= 8) atomicAdd(&s_acc[6], 1u);
    else atomicAdd(&s_acc[7], 1u);
    atomicMax(&s_acc[8], c);
  }
  for (int i = tid; i < BUCKETS; i += F_NT) {
    if (s_bkt[i]) atomicAdd(&s_acc[9], 1u);
    atomicMax(&s_acc[10], s_bkt[i]);
  }
  __syncthreads();
  if (tid == 0) {
    const double kept = s_acc[0], mk = kept > 0 ? kept : 1.0;
    const double d = s_acc[2], f1 = s_acc[3], f2 = s_acc[4];
    // HyperLogLog estimate (Flajolet et al. 2007) with linear counting for small ranges
    double z = 0.0;
    int zeros = 0;
    for (int i = 0; i < HLL; i++) {
      z += ldexp(1.0, -(int)s_hll[i]);
      zeros += s_hll[i] == 0;
    }
    double hll = (0.7213 / (1.0 + 1.079 / HLL)) * HLL * HLL / z;
    if (hll <= 2.5 * HLL && zeros) hll = HLL * log((double)HLL / zeros);
    const double neff = (double)n * (m > 0 ? kept / m : 0.0);
    const double gee = kept > 0 ? sqrt(neff / mk) * f1 + (d - f1) : 0.0;
    const double chao = d + f1 * f1 / (2.0 * (f2 > 0 ? f2 : 1.0));
    float* o = out;
    o[0] = lg2p1((double)n) / 32.f;
    o[1] = q.key_bits / 128.f;
    o[2] = (float)(s_acc[1] / mk);
    o[3] = m > 0 ? (float)(kept / m) : 0.f;
    o[4] = (float)(d / mk);
    o[5] = (float)(f1 / mk);
    o[6] = (float)(f2 / mk);
    o[7] = (float)(s_acc[5] / mk);
    o[8] = (float)(s_acc[6] / mk);
    o[9] = (float)(s_acc[7] / mk);
    o[10] = (float)(s_acc[8] / mk);
    o[11] = s_acc[9] / (float)BUCKETS;
    o[12] = lg2p1(s_acc[10]) / 12.f;
    o[13] = lg2p1(hll) / 13.f;
    o[14] = lg2p1(gee) / 32.f;
    o[15] = lg2p1(chao) / 32.f;
    o[16] = lg2p1(neff) / 32.f;
    o[17] = q.rec_bytes / 256.f;
    o[18] = q.n_fields / 24.f;
    o[19] = q.n_aggs / 24.f;
    o[20] = pred ? 1.f : 0.f;
    o[21] = q.n_keys / 8.f;
    o[22] = (kept > 0 && d == kept) ? 1.f : 0.f;
    o[23] = 1.f;
  }
}

constexpr int SAMPLE_NT = 256;  // threads (samples) per CTA of the sampling kernels

__global__ void __launch_bounds__(SAMPLE_NT) k_feat_sample(const __grid_constant__ FeatParams F,
                                                           unsigned long long* __restrict__ hs,
                                                           unsigned char* __restrict__ ns) {
  const int i = blockIdx.x * SAMPLE_NT + threadIdx.x;
  if (i < SAMPLE) sample_one(F.q, i, hs[i], ns[i]);
}

__global__ void __launch_bounds__(F_NT) k_features(const __grid_constant__ FeatParams F,
                                                   const unsigned long long* __restrict__ hs,
                                                   const unsigned char* __restrict__ ns) {
  features_body(F.q, hs, ns, F.out);
}

// a batch: SAMPLE / SAMPLE_NT sampling CTAs per query, then one feature CTA per query
__global__ void __launch_bounds__(SAMPLE_NT) k_feat_sample_batch(const DQuery* __restrict__ qs,
                                                                 unsigned long long* __restrict__ hs,
                                                                 unsigned char* __restrict__ ns) {
  constexpr int per_q = SAMPLE / SAMPLE_NT;
  const int qi = blockIdx.x / per_q;
  const int i = (blockIdx.x % per_q) * SAMPLE_NT + threadIdx.x;
  sample_one(qs[qi], i, hs[(size_t)qi * SAMPLE + i], ns[(size_t)qi * SAMPLE + i]);
}

__global__ void __launch_bounds__(F_NT) k_features_batch(const DQuery* __restrict__ qs,
                                                         const unsigned long long* __restrict__ hs,
                                                         const unsigned char* __restrict__ ns,
                                                         float* __restrict__ out) {
  const size_t qi = blockIdx.x;
  features_body(qs[qi], hs + qi * SAMPLE, ns + qi * SAMPLE, out + qi * NF);
}

// ---------------------------------------------------------------- MLP (one CTA of 64 threads per sample)
__device__ __forceinline__ void mlp_layers(const float* __restrict__ P, const float* x, float* h1, float* h2,
                                           float* out) {
  const int j = threadIdx.x;
  float a = P[OFF_B1 + j];
  for (int i = 0; i < NF; i++) a = fmaf(P[OFF_W1 + j * NF + i], x[i], a);
  h1[j] = fmaxf(a, 0.f);
  __syncthreads();
  float b = P[OFF_B2 + j];
  for (int k = 0; k < NH; k++) b = fmaf(P[OFF_W2 + j * NH + k], h1[k], b);
  h2[j] = fmaxf(b, 0.f);
  __syncthreads();
  if (j < NO) {
    float c = P[OFF_B3 + j];
    for (int k = 0; k < NH; k++) c = fmaf(P[OFF_W3 + j * NH + k], h2[k], c);
    out[j] = c;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(NH) k_mlp_forward(const float* __restrict__ P, const float* __restrict__ X, int B,
                                                    float* __restrict__ out) {
  __shared__ float x[NF], h1[NH], h2[NH], o[NO];
  const int b = blockIdx.x;
  if (b >= B) return;
  if (threadIdx.x < NF) x[threadIdx.x] = X[(size_t)b * NF + threadIdx.x];
  __syncthreads();
  mlp_layers(P, x, h1, h2, o);
  if (threadIdx.x < NO) out[(size_t)b * NO + threadIdx.x] = o[threadIdx.x];
}

// forward + backward of one sample; parameter gradients accumulate (atomicAdd) into G, scaled 1/B
__global__ void __launch_bounds__(NH) k_mlp_backward(const float* __restrict__ P, const float* __restrict__ X,
                                                     const int* __restrict__ cls, const float* __restrict__ Y,
                                                     const float* __restrict__ SW, int B, float wreg,
                                                     float* __restrict__ G, float* __restrict__ loss) {
  __shared__ float x[NF], h1[NH], h2[NH], o[NO], dout[NO], dh2[NH], dh1[NH];
  const int b = blockIdx.x, j = threadIdx.x;
  if (b >= B) return;
  if (j < NF) x[j] = X[(size_t)b * NF + j];
  __syncthreads();
  mlp_layers(P, x, h1, h2, o);
  const float sw = (SW ? SW[b] : 1.f) / (float)B;
  if (j == 0) {
    // softmax cross-entropy over the strategy scores, squared error of the group-count output
    float mx = o[0];
    for (int k = 1; k < NS; k++) mx = fmaxf(mx, o[k]);
    float e[NS], s = 0.f;
    for (int k = 0; k < NS; k++) {
      e[k] = expf(o[k] - mx);
      s += e[k];
    }
    const int c = cls[b];
    for (int k = 0; k < NS; k++) dout[k] = sw * (e[k] / s - (k == c ? 1.f : 0.f));
    const float r = o[NS] - Y[b];
    dout[NS] = sw * wreg * 2.f * r;
    atomicAdd(loss, sw * (-logf(fmaxf(e[c] / s, 1e-30f)) + wreg * r * r));
  }
  __syncthreads();
  // layer 3
  {
    float g = 0.f;
    for (int k = 0; k < NO; k++) {
      atomicAdd(&G[OFF_W3 + k * NH + j], dout[k] * h2[j]);
      g = fmaf(P[OFF_W3 + k * NH + j], dout[k], g);
    }
    dh2[j] = h2[j] > 0.f ? g : 0.f;
    if (j < NO) atomicAdd(&G[OFF_B3 + j], dout[j]);
  }
  __syncthreads();
  // layer 2: thread j owns row j of W2 (output unit j)
  {
    for (int k = 0; k < NH; k++) atomicAdd(&G[OFF_W2 + j * NH + k], dh2[j] * h1[k]);
    atomicAdd(&G[OFF_B2 + j], dh2[j]);
    float g = 0.f;
    for (int k = 0; k < NH; k++) g = fmaf(P[OFF_W2 + k * NH + j], dh2[k], g);
    dh1[j] = h1[j] > 0.f ? g : 0.f;
  }
  __syncthreads();
  // layer 1
  for (int i = 0; i < NF; i++) atomicAdd(&G[OFF_W1 + j * NF + i], dh1[j] * x[i]);
  atomicAdd(&G[OFF_B1 + j], dh1[j]);
}

__global__ void k_adam(float* __restrict__ P, const float* __restrict__ G, float* __restrict__ M, float* __restrict__ V,
                       int n, float lr, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = G[i];
  const float m = 0.9f * M[i] + 0.1f * g, v = 0.999f * V[i] + 0.001f * g * g;
  M[i] = m;
  V[i] = v;
  P[i] -= lr * (m / c1) / (sqrtf(v / c2) + 1e-8f);
}

// features of a compiled, staged query into device memory
int features_device(pmb_handle* h, const CompiledQuery& cq, float* dev_out) {
  FeatParams F;
  F.q = cq.dq;
  F.out = dev_out;
  const int smem = TSLOTS * 8;
  unsigned long long* hs = (unsigned long long*)pmb_ws_alloc(h, (size_t)SAMPLE * 9);
  if (!hs) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (selector sample)");
  unsigned char* ns = reinterpret_cast<unsigned char*>(hs + SAMPLE);
  PMB_CUDA(h, cudaFuncSetAttribute(k_features, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  pmb_kernel_begin(h, "features");
  k_feat_sample<<<SAMPLE / SAMPLE_NT, SAMPLE_NT, 0, h->stream>>>(F, hs, ns);
  k_features<<<1, F_NT, smem, h->stream>>>(F, hs, ns);
  pmb_kernel_end(h);
  PMB_CUDA(h, cudaGetLastError());
  return PMB_OK;
}

int stage_query(pmb_handle* h, const pmb_query* q, const pmb_column* cols, int32_t n_cols, CompiledQuery* cq) {
  int rc = pmb_compile_groupby(h, q, cols, n_cols, cq);
  if (rc) return rc;
  rc = pmb_ws_begin(h);
  if (rc) return rc;
  h->ptr_ok.clear();  // pointer checks start afresh for this call
  for (int c = 0; c < cq->dq.n_cols; c++) {
    rc = pmb_stage_column(h, cols[cq->map.user[c]], cq->dq.n_rows, &cq->dq.col[c]);
    if (rc) return rc;
  }
  return PMB_OK;
}

}  // namespace

// Group counts predicted by the installed selector for the queries of a batch (device DQuery
// array): out_groups[i] (host) = 2^(output 3), or 0 when unusable; false without a selector.
// group count of query i from the network's outputs o[i * NO ...] (0 when not finite)
static int64_t batch_groups(const float* o, int i, int64_t n_rows) {
  const float g = o[(size_t)i * NO + NS];
  return std::isfinite(g) ? (int64_t)std::min<double>(std::exp2(std::min<double>(std::max<double>(g, 0.0), 40.0)),
                                                      (double)n_rows)
                          : 0;
}

// features and MLP forward of every query of a batch, queued on the stream; the outputs are copied
// into pinned staging, so the caller's next stream synchronisation (the batch sketch's readback)
// serves both. nullptr when no selector is installed or no staging is available yet (then
// pmb_selector_predict_batch runs synchronously).
const float* pmb_selector_batch_launch(pmb_handle* h, const DQuery* d_qs, int nq) {
  if (!h->selector || nq <= 0) return nullptr;
  float* ho = (float*)pmb_host_stage(h, (size_t)nq * NO * sizeof(float));
  if (!ho) return nullptr;
  float* feat = (float*)pmb_ws_alloc(h, (size_t)nq * NF * sizeof(float));
  float* o = (float*)pmb_ws_alloc(h, (size_t)nq * NO * sizeof(float));
  if (!feat || !o) return nullptr;
  const int smem = TSLOTS * 8;
  if (cudaFuncSetAttribute(k_features_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) return nullptr;
  unsigned long long* hs = (unsigned long long*)pmb_ws_alloc(h, (size_t)nq * SAMPLE * 9);
  if (!hs) return nullptr;
  unsigned char* ns = reinterpret_cast<unsigned char*>(hs + (size_t)nq * SAMPLE);
  pmb_kernel_begin(h, "features");
  k_feat_sample_batch<<<nq * (SAMPLE / SAMPLE_NT), SAMPLE_NT, 0, h->stream>>>(d_qs, hs, ns);
  k_features_batch<<<nq, F_NT, smem, h->stream>>>(d_qs, hs, ns, feat);
  pmb_kernel_end(h);
  pmb_kernel_begin(h, "mlp_forward");
  k_mlp_forward<<<nq, NH, 0, h->stream>>>(h->selector, feat, nq, o);
  pmb_kernel_end(h);
  if (cudaGetLastError() != cudaSuccess) return nullptr;
  if (cudaMemcpyAsync(ho, o, (size_t)nq * NO * sizeof(float), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess)
    return nullptr;
  return ho;
}

// the group counts from the staged outputs of pmb_selector_batch_launch, after a synchronisation
void pmb_selector_batch_groups(const float* ho, int nq, int64_t* out_groups, const int64_t* n_rows) {
  for (int i = 0; i < nq; i++) out_groups[i] = batch_groups(ho, i, n_rows[i]);
}

bool pmb_selector_predict_batch(pmb_handle* h, const DQuery* d_qs, int nq, int64_t* out_groups, const int64_t* n_rows) {
  if (!h->selector || nq <= 0) return false;
  float* feat = (float*)pmb_ws_alloc(h, (size_t)nq * NF * sizeof(float));
  float* o = (float*)pmb_ws_alloc(h, (size_t)nq * NO * sizeof(float));
  if (!feat || !o) return false;
  const int smem = TSLOTS * 8;
  if (cudaFuncSetAttribute(k_features_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) return false;
  unsigned long long* hs = (unsigned long long*)pmb_ws_alloc(h, (size_t)nq * SAMPLE * 9);
  if (!hs) return false;
  unsigned char* ns = reinterpret_cast<unsigned char*>(hs + (size_t)nq * SAMPLE);
  pmb_kernel_begin(h, "features");
  k_feat_sample_batch<<<nq * (SAMPLE / SAMPLE_NT), SAMPLE_NT, 0, h->stream>>>(d_qs, hs, ns);
  k_features_batch<<<nq, F_NT, smem, h->stream>>>(d_qs, hs, ns, feat);
  pmb_kernel_end(h);
  pmb_kernel_begin(h, "mlp_forward");
  k_mlp_forward<<<nq, NH, 0, h->stream>>>(h->selector, feat, nq, o);
  pmb_kernel_end(h);
  if (cudaGetLastError() != cudaSuccess) return false;
  std::vector<float> ho((size_t)nq * NO);
  if (cudaMemcpyAsync(ho.data(), o, ho.size() * sizeof(float), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess)
    return false;
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return false;
  for (int i = 0; i < nq; i++) out_groups[i] = batch_groups(ho.data(), i, n_rows[i]);
  return true;
}

// AUTO strategy with the installed selector: false when none is installed or its output is not
// usable (the caller then takes the cardinality heuristic)
// The selector's scores and group count from its outputs (false when unusable)
static bool selector_decode(const float* o, int64_t n_rows, int* strategy, int64_t* groups) {
  for (int k = 0; k < NO; k++)
    if (!std::isfinite(o[k])) return false;
  int best = 0;
  for (int k = 1; k < NS; k++)
    if (o[k] > o[best]) best = k;
  static const int map[NS] = {PMB_STRATEGY_SMEM_HASH, PMB_STRATEGY_GLOBAL_HASH, PMB_STRATEGY_SORT,
                              PMB_STRATEGY_PARTITIONED};
  *strategy = map[best];
  const double g = std::exp2(std::min<double>(std::max<double>(o[NS], 0.0), 40.0));
  *groups = (int64_t)std::min<double>(g, (double)n_rows);
  if (*groups < 1) *groups = 1;
  return true;
}

// pmb_selector_pick in two halves around a synchronisation the caller makes anyway: the launch
// queues the feature and MLP kernels and the copy of the outputs into the handle's pinned staging
// (at PMB_SEL_PINNED_OFF); the read decodes them once the stream has been synchronised.
bool pmb_selector_launch(pmb_handle* h, const CompiledQuery& cq) {
  if (!h->selector || cq.dq.n_rows == 0) return false;
  float* buf = (float*)pmb_ws_alloc(h, (NF + NO) * sizeof(float));
  if (!buf) return false;
  if (features_device(h, cq, buf) != PMB_OK) return false;
  pmb_kernel_begin(h, "mlp_forward");
  k_mlp_forward<<<1, NH, 0, h->stream>>>(h->selector, buf, 1, buf + NF);
  pmb_kernel_end(h);
  if (cudaGetLastError() != cudaSuccess) return false;
  return cudaMemcpyAsync(h->pinned + PMB_SEL_PINNED_OFF, buf + NF, NO * sizeof(float), cudaMemcpyDeviceToHost,
                         h->stream) == cudaSuccess;
}

bool pmb_selector_read(pmb_handle* h, const CompiledQuery& cq, int* strategy, int64_t* groups) {
  float o[NO];
  memcpy(o, h->pinned + PMB_SEL_PINNED_OFF, sizeof(o));
  return selector_decode(o, cq.dq.n_rows, strategy, groups);
}

bool pmb_selector_pick(pmb_handle* h, const CompiledQuery& cq, int* strategy, int64_t* groups) {
  if (!h->selector || cq.dq.n_rows == 0) return false;
  float* buf = (float*)pmb_ws_alloc(h, (NF + NO) * sizeof(float));
  if (!buf) return false;
  if (features_device(h, cq, buf) != PMB_OK) return false;
  pmb_kernel_begin(h, "mlp_forward");
  k_mlp_forward<<<1, NH, 0, h->stream>>>(h->selector, buf, 1, buf + NF);
  pmb_kernel_end(h);
  if (cudaGetLastError() != cudaSuccess) return false;
  float o[NO];
  if (cudaMemcpyAsync(o, buf + NF, sizeof(o), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess) return false;
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return false;
  return selector_decode(o, cq.dq.n_rows, strategy, groups);
}

extern "C" int pmb_selector_features(pmb_handle* h, const pmb_query* q, const pmb_column* cols, int32_t n_cols,
                                     float* out) {
  if (!h) return PMB_E_INVALID;
  if (!out) return pmb_fail(h, PMB_E_INVALID, "out is NULL");
  PMB_CUDA(h, cudaSetDevice(h->device));
  CompiledQuery cq;
  int rc = stage_query(h, q, cols, n_cols, &cq);
  if (rc) return rc;
  float* buf = (float*)pmb_ws_alloc(h, NF * sizeof(float));
  if (!buf) return pmb_fail(h, PMB_E_OOM, "workspace exhausted (features)");
  PMB_CUDA(h, cudaMemsetAsync(buf, 0, NF * sizeof(float), h->stream));
  if (cq.dq.n_rows > 0) {
    rc = features_device(h, cq, buf);
    if (rc) return rc;
  }
  PMB_CUDA(h, cudaMemcpyAsync(out, buf, NF * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  PMB_CUDA(h, cudaStreamSynchronize(h->stream));
  return PMB_OK;
}

extern "C" int pmb_selector_set(pmb_handle* h, const float* params, int32_t n_params) {
  if (!h) return PMB_E_INVALID;
  PMB_CUDA(h, cudaSetDevice(h->device));
  if (!params) {
    if (h->selector) cudaFree(h->selector);
    h->selector = nullptr;
    return PMB_OK;
  }
  if (n_params != N_PARAMS) return pmb_fail(h, PMB_E_INVALID, "selector parameter count mismatch");
  for (int i = 0; i < n_params; i++)
    if (!std::isfinite(params[i])) return pmb_fail(h, PMB_E_INVALID, "selector parameters must be finite");
  if (!h->selector) PMB_CUDA(h, cudaMalloc(&h->selector, N_PARAMS * sizeof(float)));
  PMB_CUDA(h, cudaMemcpyAsync(h->selector, params, N_PARAMS * sizeof(float), cudaMemcpyHostToDevice, h->stream));
  PMB_CUDA(h, cudaStreamSynchronize(h->stream));
  return PMB_OK;
}

extern "C" int pmb_selector_choose(pmb_handle* h, const pmb_query* q, const pmb_column* cols, int32_t n_cols,
                                   int32_t* strategy, int64_t* groups) {
  if (!h) return PMB_E_INVALID;
  if (!strategy || !groups) return pmb_fail(h, PMB_E_INVALID, "strategy / groups is NULL");
  PMB_CUDA(h, cudaSetDevice(h->device));
  CompiledQuery cq;
  int rc = stage_query(h, q, cols, n_cols, &cq);
  if (rc) return rc;
  int s = 0;
  int64_t g = 0;
  // the same decisions as pmb_groupby's AUTO: sample estimate, selector (which can only enlarge
  // the estimate) or heuristic, then the switch to the partitioned strategy
  static thread_local SketchOut sk;
  rc = pmb_groupby_sketch(h, cq, &sk);
  if (rc) return rc;
  const int64_t e = pmb_estimate_groups(sk, cq.dq.n_rows);
  if (pmb_selector_pick(h, cq, &s, &g) &&
      !(pmb_selector_vetoed(cq, sk, s))) {
    g = std::max<int64_t>(e, std::min<int64_t>(g, cq.dq.n_rows));
  } else {
    // the heuristic: cardinality, then the switch to the partitioned strategy (the network
    // scores the partitioned strategy itself)
    g = e;
    s = pmb_choose_strategy(h, cq, sk, g);
    if (pmb_prefer_partitioned(cq, sk, s, g)) s = PMB_STRATEGY_PARTITIONED;
  }
  *strategy = s;
  *groups = g;
  return PMB_OK;
}

extern "C" int pmb_mlp_forward(pmb_handle* h, const float* params, const float* x, int32_t batch, float* out) {
  if (!h) return PMB_E_INVALID;
  if (!params || !x || !out || batch < 0) return pmb_fail(h, PMB_E_INVALID, "bad MLP arguments");
  if (batch == 0) return PMB_OK;
  PMB_CUDA(h, cudaSetDevice(h->device));
  k_mlp_forward<<<batch, NH, 0, h->stream>>>(params, x, batch, out);
  PMB_CUDA(h, cudaGetLastError());
  PMB_CUDA(h, cudaStreamSynchronize(h->stream));
  return PMB_OK;
}

extern "C" int pmb_mlp_gradient(pmb_handle* h, const float* params, const float* x, const int32_t* cls, const float* y,
                                const float* sw, int32_t batch, float wreg, float* grad, float* loss) {
  if (!h) return PMB_E_INVALID;
  if (!params || !x || !cls || !y || !grad || !loss || batch <= 0) return pmb_fail(h, PMB_E_INVALID, "bad MLP arguments");
  PMB_CUDA(h, cudaSetDevice(h->device));
  PMB_CUDA(h, cudaMemsetAsync(grad, 0, N_PARAMS * sizeof(float), h->stream));
  PMB_CUDA(h, cudaMemsetAsync(loss, 0, sizeof(float), h->stream));
  k_mlp_backward<<<batch, NH, 0, h->stream>>>(params, x, cls, y, sw, batch, wreg, grad, loss);
  PMB_CUDA(h, cudaGetLastError());
  PMB_CUDA(h, cudaStreamSynchronize(h->stream));
  return PMB_OK;
}

extern "C" int pmb_mlp_adam_step(pmb_handle* h, float* params, const float* grad, float* m, float* v, int32_t step,
                                 float lr) {
  if (!h) return PMB_E_INVALID;
  if (!params || !grad || !m || !v || step < 1) return pmb_fail(h, PMB_E_INVALID, "bad Adam arguments");
  PMB_CUDA(h, cudaSetDevice(h->device));
  const float c1 = 1.f - std::pow(0.9f, (float)step), c2 = 1.f - std::pow(0.999f, (float)step);
  k_adam<<<(N_PARAMS + 255) / 256, 256, 0, h->stream>>>(params, grad, m, v, N_PARAMS, lr, c1, c2);
  PMB_CUDA(h, cudaGetLastError());
  PMB_CUDA(h, cudaStreamSynchronize(h->stream));
  return PMB_OK;
}
