// pmb_runtime.cu — handle lifetime, device workspace, column staging, results, profiling.
//
// Replaces the reference's Metal runtime pieces for this path: MetalDevice / CommandQueue
// (crates/polars-metal-kernels/src/command.rs:95-231), the Arrow -> device buffer bridge
// (crates/polars-metal-buffer/src/bridge.rs:1-60) and the per-call buffer allocation the
// reference does for every dispatch. Here one handle owns a stream and one growable device
// workspace; each call bump-allocates from it and synchronises once at the end.
#include <cuda_runtime.h>

#include <dlfcn.h>
#include <sys/mman.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <unordered_map>
#include <cstdlib>
#include <cstring>
#include <chrono>
#include <cstdio>
#include <string>

#include "pmb_internal.cuh"

int pmb_fail(pmb_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

int pmb_cuda_check(pmb_handle* h, cudaError_t e, const char* what) {
  std::string m = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return pmb_fail(h, PMB_E_OOM, m);
  return pmb_fail(h, PMB_E_CUDA, m);
}

// ------------------------------------------------------------------ workspace
static void ws_free_all(pmb_handle* h) {
  for (auto& b : h->ws) cudaFree(b.ptr);
  h->ws.clear();
  h->ws_cur = 0;
}

int pmb_ws_begin(pmb_handle* h) {
  if (h->ws.size() > 1) {
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return pmb_cuda_check(h, e, "cudaStreamSynchronize");
    size_t total = 0;
    for (auto& b : h->ws) total += b.cap;
    ws_free_all(h);
    uint8_t* p = nullptr;
    if (cudaMalloc((void**)&p, total) != cudaSuccess) {
      cudaGetLastError();
      return PMB_OK;  // blocks are added again on demand
    }
    h->ws.push_back({p, total, 0});
  }
  for (auto& b : h->ws) b.top = 0;
  h->ws_cur = 0;
  // the staging area grows between calls (the previous call's copies have completed by now)
  if (h->hstage_want > h->hstage_cap) {
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return pmb_cuda_check(h, e, "cudaStreamSynchronize");
    if (h->hstage) cudaFreeHost(h->hstage);
    h->hstage = nullptr;
    h->hstage_cap = 0;
    if (cudaMallocHost((void**)&h->hstage, h->hstage_want) == cudaSuccess) h->hstage_cap = h->hstage_want;
    else cudaGetLastError();
  }
  h->hstage_used = 0;
  h->hstage_want = 0;
  return PMB_OK;
}

void* pmb_host_stage(pmb_handle* h, size_t bytes) {
  const size_t b = (bytes + 255) & ~(size_t)255;
  h->hstage_want += b;
  if (!h->hstage || h->hstage_used + b > h->hstage_cap) return nullptr;
  void* p = h->hstage + h->hstage_used;
  h->hstage_used += b;
  return p;
}

// the allocation position: the current block and its top (blocks after it are empty)
WsMark pmb_ws_mark(const pmb_handle* h) {
  if (h->ws.empty()) return {0, 0};
  return {h->ws_cur + 1, h->ws[h->ws_cur].top};
}

void pmb_ws_release(pmb_handle* h, WsMark m) {
  if (m.blocks == 0) {
    for (auto& b : h->ws) b.top = 0;
    h->ws_cur = 0;
    return;
  }
  h->ws[m.blocks - 1].top = m.top;
  for (size_t i = m.blocks; i < h->ws.size(); i++) h->ws[i].top = 0;
  h->ws_cur = m.blocks - 1;  // the blocks given back are used again before new ones are added
}

void* pmb_ws_alloc(pmb_handle* h, size_t bytes) {
  bytes = pmb_align(bytes ? bytes : 1, 256);
  // bump allocation from the current block on (blocks before it are in use up to their top)
  for (size_t i = h->ws_cur; i < h->ws.size(); i++) {
    auto& b = h->ws[i];
    if (b.top + bytes <= b.cap) {
      void* p = b.ptr + b.top;
      b.top += bytes;
      h->ws_cur = i;
      return p;
    }
  }
  size_t last = h->ws.empty() ? 0 : h->ws.back().cap;
  size_t want = std::max(std::max(bytes, (size_t)64 << 20), last);
  uint8_t* p = nullptr;
  if (cudaMalloc((void**)&p, want) != cudaSuccess) {
    cudaGetLastError();
    if (want == bytes || cudaMalloc((void**)&p, bytes) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    want = bytes;
  }
  h->ws.push_back({p, want, bytes});
  h->ws_cur = h->ws.size() - 1;
  return p;
}

// ------------------------------------------------------------------ profiling
static cudaEvent_t take_event(pmb_handle* h) {
  if (h->event_next == h->event_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    h->event_pool.push_back(e);
  }
  return h->event_pool[h->event_next++];
}

static double host_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void pmb_phase(pmb_handle* h, const char* name) {
  if (!h->phase_timing) return;
  const double t = host_ms();
  h->phases.push_back({name, t - h->phase_t0});
  h->phase_t0 = t;
}

void pmb_call_begin(pmb_handle* h) {
  h->ptr_ok.clear();  // allocation ranges checked in this call (the caller's buffers live through it)
  h->phase_timing = getenv("PMB_CALL_TIMING") != nullptr;
  h->phases.clear();
  if (h->phase_timing) h->phase_t0 = host_ms();
  h->timings.clear();
  h->event_next = 0;
  h->launches = 0;
  h->h2d = h->d2h = 0;
  if (h->profiling) cudaEventRecord(h->call_start, h->stream);
}

void pmb_kernel_begin(pmb_handle* h, const char* name) {
  h->launches++;
  if (!h->profiling) return;
  KernelTiming t;
  t.name = name;
  t.start = take_event(h);
  t.stop = take_event(h);
  cudaEventRecord(t.start, h->stream);
  h->timings.push_back(t);
}

void pmb_kernel_end(pmb_handle* h) {
  if (!h->profiling || h->timings.empty()) return;
  cudaEventRecord(h->timings.back().stop, h->stream);
}

void pmb_call_end(pmb_handle* h) {
  pmb_stats s{};
  s.kernel_launches = h->launches;
  s.h2d_bytes = h->h2d;
  s.d2h_bytes = h->d2h;
  if (h->profiling) {
    cudaEventRecord(h->call_stop, h->stream);
    cudaEventSynchronize(h->call_stop);
    cudaEventElapsedTime(&s.total_ms, h->call_start, h->call_stop);
    for (const KernelTiming& t : h->timings) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, t.start, t.stop);
      int k = 0;
      for (; k < s.n_kernels; k++)
        if (t.name == s.names[k]) break;
      if (k == s.n_kernels) {
        if (s.n_kernels == PMB_MAX_STAT_KERNELS) continue;
        strncpy(s.names[k], t.name.c_str(), 31);
        s.names[k][31] = 0;
        s.n_kernels++;
      }
      s.ms[k] += ms;
      s.launches[k]++;
    }
  }
  h->last_stats = s;
  if (h->phase_timing) {
    pmb_phase(h, "end");
    double total = 0.0;
    for (auto& ph : h->phases) total += ph.second;
    fprintf(stderr, "pmb call %.3f ms host:", total);
    for (auto& ph : h->phases) fprintf(stderr, " %s %.3f", ph.first, ph.second);
    fprintf(stderr, "\n");
  }
}

// ------------------------------------------------------------------ staging kernels
// out bit i = in bit (i + shift), shift in [0, 8); out is zero-padded to whole bytes
__global__ void k_bitmap_shift(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, int64_t n_bits,
                               int shift, int64_t in_bytes) {
  int64_t ob = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t n_out = (n_bits + 7) / 8;
  for (; ob < n_out; ob += (int64_t)gridDim.x * blockDim.x) {
    uint32_t lo = in[ob];
    uint32_t hi = (ob + 1 < in_bytes) ? in[ob + 1] : 0u;
    uint32_t v = ((hi << 8) | lo) >> shift;
    int64_t rem = n_bits - ob * 8;
    if (rem < 8) v &= (1u << rem) - 1u;
    out[ob] = (uint8_t)v;
  }
}

static int launch_shift(pmb_handle* h, const uint8_t* in, uint8_t* out, int64_t n_bits, int shift,
                        int64_t in_bytes) {
  int64_t n_out = (n_bits + 7) / 8;
  if (n_out == 0) return PMB_OK;
  int blocks = (int)std::min<int64_t>((n_out + 255) / 256, 4096);
  pmb_kernel_begin(h, "bitmap_shift");
  k_bitmap_shift<<<blocks, 256, 0, h->stream>>>(in, out, n_bits, shift, in_bytes);
  pmb_kernel_end(h);
  PMB_CUDA(h, cudaGetLastError());
  return PMB_OK;
}

// copies `bytes` into the workspace (H2D when !on_device, D2D otherwise)
static int copy_in(pmb_handle* h, const void* src, size_t bytes, bool on_device, uint8_t** dst) {
  *dst = (uint8_t*)pmb_ws_alloc(h, bytes + 16);
  if (!*dst) return pmb_fail(h, PMB_E_OOM, "workspace exhausted while staging a column");
  if (bytes == 0) return PMB_OK;
  PMB_CUDA(h, cudaMemcpyAsync(*dst, src, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                              h->stream));
  if (!on_device) h->h2d += (int64_t)bytes;
  return PMB_OK;
}

static int stage_bits(pmb_handle* h, const uint8_t* base, int64_t offset, int64_t n, bool on_device,
                      const uint8_t** out) {
  const uint8_t* first = base + offset / 8;
  int shift = (int)(offset % 8);
  int64_t bytes = (n + shift + 7) / 8;
  if (on_device && shift == 0 && ((uintptr_t)first % 16) == 0) {
    *out = first;
    return PMB_OK;
  }
  uint8_t* raw;
  int rc = copy_in(h, first, (size_t)bytes, on_device, &raw);
  if (rc) return rc;
  if (shift == 0) {
    *out = raw;
    return PMB_OK;
  }
  uint8_t* aligned = (uint8_t*)pmb_ws_alloc(h, (size_t)((n + 7) / 8) + 16);
  if (!aligned) return pmb_fail(h, PMB_E_OOM, "workspace exhausted while staging a bitmap");
  rc = launch_shift(h, raw, aligned, n, shift, bytes);
  if (rc) return rc;
  *out = aligned;
  return PMB_OK;
}

// The allocation range of a device pointer (driver's cuMemGetAddressRange, looked up with dlsym
// so the library needs no link-time driver dependency); false when unavailable or not device memory
static bool device_range(const void* p, uintptr_t* base, size_t* size) {
  typedef int (*range_fn)(unsigned long long*, size_t*, unsigned long long);
  static range_fn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    if (void* lib = dlopen("libcuda.so.1", RTLD_NOW | RTLD_LOCAL | RTLD_NOLOAD))
      fn = (range_fn)dlsym(lib, "cuMemGetAddressRange_v2");
  }
  if (!fn) return false;
  unsigned long long b = 0;
  size_t n = 0;
  if (fn(&b, &n, (unsigned long long)(uintptr_t)p) != 0 || n == 0) return false;
  *base = (uintptr_t)b;
  *size = n;
  return true;
}

// A device column's pointer must be memory of the handle's GPU (or pinned host memory). The
// answer is kept per allocation range for the rest of the call, so a batch of thousands of
// columns carved from a few allocations costs a few driver queries.
static int check_device_pointer(pmb_handle* h, const void* p) {
  const uintptr_t a = (uintptr_t)p;
  for (const auto& r : h->ptr_ok)
    if (a >= r.first && a < r.second) return PMB_OK;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return pmb_fail(h, PMB_E_INVALID, "device column pointer is not CUDA memory");
  }
  if (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) {
    if (at.device != h->device)
      return pmb_fail(h, PMB_E_INVALID, "device column lives on GPU " + std::to_string(at.device) +
                                            ", the handle on GPU " + std::to_string(h->device));
    uintptr_t base;
    size_t size;
    if (h->ptr_ok.size() < 64 && device_range(p, &base, &size)) h->ptr_ok.push_back({base, base + size});
    return PMB_OK;
  }
  if (at.type == cudaMemoryTypeHost) return PMB_OK;  // pinned host memory, mapped for the device
  return pmb_fail(h, PMB_E_INVALID, "device column pointer is not CUDA memory (pageable host memory?)");
}

int pmb_stage_column(pmb_handle* h, const pmb_column& c, int64_t n, DCol* out) {
  out->dtype = c.dtype;
  out->elem = pmb_dtype_bytes(c.dtype);
  if (c.offset < 0) return pmb_fail(h, PMB_E_INVALID, "negative column offset");
  if (n > 0 && c.data == nullptr) return pmb_fail(h, PMB_E_INVALID, "column data pointer is NULL");
  bool dev = c.on_device != 0;
  if (dev && n > 0) {
    // a device column must be memory of this handle's GPU: another GPU's buffer would be read
    // through a peer mapping or fault in the kernels, and pageable host memory would fault
    int rc = check_device_pointer(h, c.data);
    if (!rc && c.validity) rc = check_device_pointer(h, c.validity);
    if (rc) return rc;
  }
  if (c.dtype == PMB_BOOL) {
    int rc = stage_bits(h, (const uint8_t*)c.data, c.offset, n, dev, &out->data);
    if (rc) return rc;
  } else {
    const uint8_t* p = (const uint8_t*)c.data + c.offset * out->elem;
    if (dev && ((uintptr_t)p % 16) == 0) {
      out->data = p;
    } else {
      uint8_t* d;
      int rc = copy_in(h, p, (size_t)(n * out->elem), dev, &d);
      if (rc) return rc;
      out->data = d;
    }
  }
  if (c.validity == nullptr) {
    out->valid = nullptr;
  } else {
    int rc = stage_bits(h, c.validity, c.offset, n, dev, &out->valid);
    if (rc) return rc;
  }
  return PMB_OK;
}

// ------------------------------------------------------------------ results
pmb_result* pmb_result_new(int32_t n_columns) {
  pmb_result* r = (pmb_result*)calloc(1, sizeof(pmb_result));
  if (!r) return nullptr;
  r->n_columns = n_columns;
  r->columns = (pmb_out_column*)calloc((size_t)std::max(n_columns, 1), sizeof(pmb_out_column));
  if (!r->columns) {
    free(r);
    return nullptr;
  }
  // columns hold workspace (device) pointers until pmb_finish_outputs copies them to host memory
  // it allocates, so a result freed on an error path before that never frees a device pointer
  for (int32_t c = 0; c < n_columns; c++) r->columns[c].on_device = 1;
  return r;
}

// Host memory for result buffers. Buffers of 1 MB and more come from a process-wide pool of pinned
// (page-locked) blocks that are recycled when results are freed: the copy back from the device then
// runs at the host link's speed into pages that are already resident, instead of through the
// driver's staging into fresh pageable pages that fault on first touch (the hash workload's 46 MB
// result took ~9 ms that way). The pool holds at most PMB_PINNED_POOL_MB (default 1024) megabytes,
// handed out or cached: pinning pages is slow (a batch of 4,096 host results pinned afresh on every
// call ran 1.6x slower than with pageable buffers), so beyond that budget buffers come from malloc,
// and blocks are never unpinned, only reused. A request takes the smallest cached block that holds
// it if that block is at most twice its size. Smaller buffers, and any buffer when pinned memory
// cannot be had, come from malloc. host_release() frees either kind.
namespace {
// the pool's state is never destroyed: a binding may release a buffer from a finalizer that runs
// late in the process's exit, after static objects would have been torn down
struct PinnedPool {
  std::mutex mu;
  std::unordered_map<void*, size_t> size;  // every pinned block handed out or cached
  std::multimap<size_t, void*> free;       // cached blocks by size
  size_t total = 0;                        // bytes of all pinned blocks (handed out or cached)
};
PinnedPool& pool() {
  static PinnedPool* p = new PinnedPool();
  return *p;
}
constexpr size_t POOL_MIN = (size_t)1 << 20;

size_t pool_budget() {
  static size_t cap = [] {
    const char* e = getenv("PMB_PINNED_POOL_MB");
    return (size_t)(e ? std::max(0, atoi(e)) : 1024) << 20;
  }();
  return cap;
}
}  // namespace

static void* host_alloc(size_t bytes) {
  if (bytes >= POOL_MIN) {
    const size_t rounded = (bytes + POOL_MIN - 1) & ~(POOL_MIN - 1);
    PinnedPool& P = pool();
    std::lock_guard<std::mutex> lock(P.mu);
    auto it = P.free.lower_bound(rounded);
    if (it != P.free.end() && it->first <= 2 * rounded) {
      void* p = it->second;
      P.free.erase(it);
      return p;
    }
    void* p = nullptr;
    if (P.total + rounded <= pool_budget()) {
      if (cudaHostAlloc(&p, rounded, cudaHostAllocPortable) == cudaSuccess) {
        P.size[p] = rounded;
        P.total += rounded;
        return p;
      }
      cudaGetLastError();  // no pinned memory: a pageable buffer works the same, only slower
    }
  }
  return malloc(bytes ? bytes : 1);
}

void host_release(void* p) {
  if (!p) return;
  {
    PinnedPool& P = pool();
    std::lock_guard<std::mutex> lock(P.mu);
    auto it = P.size.find(p);
    if (it != P.size.end()) {
      P.free.emplace(it->second, p);
      return;
    }
  }
  free(p);
}

static size_t bitmap_bytes(int64_t n) {
  size_t b = (size_t)((n + 7) / 8);
  b = (b + 3) & ~(size_t)3;
  return b < 4 ? 4 : b;
}

int pmb_finish_outputs(pmb_handle* h, pmb_result* r, bool to_host) {
  int64_t n = r->n_groups;
  for (int c = 0; c < r->n_columns; c++) {
    pmb_out_column& oc = r->columns[c];
    oc.length = n;
    if (!to_host) {
      oc.on_device = 1;
      continue;
    }
    size_t db = oc.dtype == PMB_BOOL ? bitmap_bytes(n) : (size_t)n * pmb_dtype_bytes(oc.dtype);
    size_t vb = bitmap_bytes(n);
    void* hd = host_alloc(db);
    uint8_t* hv = (uint8_t*)host_alloc(vb);
    if (!hd || !hv) {
      host_release(hd);
      host_release(hv);
      return pmb_fail(h, PMB_E_OOM, "host output allocation failed");
    }
    // the copies below fill every byte but the padding of the bitmaps, which is zeroed here
    size_t copy_d = oc.dtype == PMB_BOOL ? (size_t)((n + 7) / 8) : db;
    if (n == 0) copy_d = 0;
    memset((uint8_t*)hd + copy_d, 0, (db ? db : 1) - copy_d);
    memset(hv + (size_t)((n + 7) / 8), 0, vb - (size_t)((n + 7) / 8));
    if (n > 0) {
      PMB_CUDA(h, cudaMemcpyAsync(hd, oc.data, copy_d, cudaMemcpyDeviceToHost, h->stream));
      PMB_CUDA(h, cudaMemcpyAsync(hv, oc.validity, (size_t)((n + 7) / 8), cudaMemcpyDeviceToHost, h->stream));
      h->d2h += (int64_t)(copy_d + (size_t)((n + 7) / 8));
    }
    oc.data = hd;
    oc.validity = hv;
    oc.on_device = 0;
  }
  if (to_host) PMB_CUDA(h, cudaStreamSynchronize(h->stream));
  return PMB_OK;
}

// ------------------------------------------------------------------ C ABI
extern "C" {

const char* pmb_version(void) { return "pmb 0.1.0 (sm_100a)"; }

int pmb_open(pmb_handle** out, int32_t device, uint64_t workspace_bytes) {
  if (!out) return PMB_E_INVALID;
  *out = nullptr;
  pmb_handle* h = new pmb_handle();
  h->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) {
    delete h;
    return PMB_E_CUDA;
  }
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) {
    delete h;
    return PMB_E_CUDA;
  }
  if (prop.major < 10) {
    delete h;
    return PMB_E_UNSUPPORTED;  // built for sm_100a only
  }
  h->sm_count = prop.multiProcessorCount;
  h->max_smem_optin = (int)prop.sharedMemPerBlockOptin;
  if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&h->call_start) != cudaSuccess || cudaEventCreate(&h->call_stop) != cudaSuccess ||
      cudaMallocHost((void**)&h->pinned, 65536) != cudaSuccess) {
    pmb_close(h);
    return PMB_E_CUDA;
  }
  h->stream = h->own_stream;
  if (workspace_bytes) {
    uint8_t* p = nullptr;
    if (cudaMalloc((void**)&p, workspace_bytes) != cudaSuccess) {
      cudaGetLastError();
      pmb_close(h);
      return PMB_E_OOM;
    }
    h->ws.push_back({p, (size_t)workspace_bytes, 0});
  }
  *out = h;
  return PMB_OK;
}

void pmb_close(pmb_handle* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  ws_free_all(h);
  if (h->pinned) cudaFreeHost(h->pinned);
  if (h->hstage) cudaFreeHost(h->hstage);
  if (h->selector) cudaFree(h->selector);
  for (cudaEvent_t e : h->event_pool) cudaEventDestroy(e);
  if (h->call_start) cudaEventDestroy(h->call_start);
  if (h->call_stop) cudaEventDestroy(h->call_stop);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
}

const char* pmb_last_error(const pmb_handle* h) { return h ? h->err.c_str() : "null handle"; }

int pmb_set_stream(pmb_handle* h, void* stream) {
  if (!h) return PMB_E_INVALID;
  h->stream = stream ? (cudaStream_t)stream : h->own_stream;
  return PMB_OK;
}

int pmb_set_profiling(pmb_handle* h, int32_t enabled) {
  if (!h) return PMB_E_INVALID;
  h->profiling = enabled != 0;
  return PMB_OK;
}

int pmb_set_batching(pmb_handle* h, int32_t enabled) {
  if (!h) return PMB_E_INVALID;
  h->batching = enabled != 0;
  return PMB_OK;
}

int pmb_last_stats(const pmb_handle* h, pmb_stats* out) {
  if (!h || !out) return PMB_E_INVALID;
  *out = h->last_stats;
  return PMB_OK;
}

void pmb_result_free(pmb_result* r) {
  if (!r) return;
  for (int c = 0; c < r->n_columns; c++) {
    if (!r->columns[c].on_device) {
      host_release(r->columns[c].data);
      host_release(r->columns[c].validity);
    }
  }
  free(r->columns);
  free(r);
}

int64_t pmb_results_pack(pmb_result* const* rs, int32_t n, uint64_t* words, int64_t cap_words) {
  if (n < 0 || (n > 0 && (!rs || !words))) return -1;
  int64_t w = 0;
  for (int32_t i = 0; i < n; i++) {
    const pmb_result* r = rs[i];
    const int32_t nc = r ? r->n_columns : 0;
    if (w + 4 + 4 * (int64_t)nc > cap_words) return -1;
    words[w++] = r ? (uint64_t)r->n_groups : 0;
    words[w++] = (uint64_t)(uint32_t)nc | ((uint64_t)(uint32_t)(r ? r->strategy_used : 0) << 32);
    words[w++] = r ? (uint64_t)(uint32_t)r->rehash_count : 0;
    words[w++] = r ? (uint64_t)r->capacity : 0;
    for (int32_t c = 0; c < nc; c++) {
      const pmb_out_column& o = r->columns[c];
      words[w++] = (uint64_t)(uintptr_t)o.data;
      words[w++] = (uint64_t)(uintptr_t)o.validity;
      words[w++] = (uint64_t)o.length;
      words[w++] = (uint64_t)(uint32_t)o.dtype | ((uint64_t)(uint32_t)o.on_device << 32);
    }
  }
  return w;
}

void pmb_host_buffer_free(void* p) { host_release(p); }

void pmb_results_free(pmb_result* const* rs, int32_t n) {
  if (!rs) return;
  for (int32_t i = 0; i < n; i++) pmb_result_free(rs[i]);
}

}  // extern "C"
