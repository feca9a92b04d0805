// pmb_noalloc.cu — the u8 -> u32 inclusive prefix sum for callers that cannot allocate.
//
// pmb_cumsum_u8_to_u32 (pmb_filter.cu) takes its look-back scratch from the handle's workspace,
// which grows with cudaMalloc. Some callers may not allocate device memory at all: a host
// framework that has reserved the device's memory for its own pool (an allocation would fail
// or fragment that pool), or a latency-critical loop where cudaMalloc / cudaFree would
// synchronise the whole device. This file gives them one entry point that allocates nothing:
// the caller passes device input and output, and the scratch (the tile states of the
// decoupled look-back and a status word) lives in the fixed-size array below.
//
// The array is a file-scope __device__ variable: every GPU that loads this library holds it
// until the process exits. Host code cannot use its name as a device address (it is a host-side
// stand-in), so the first call on each device looks the address up with cudaGetSymbolAddress,
// with that device current, and later calls reuse it. All calls share the array and it keeps the
// previous call's contents, so each call clears what must start at zero; calls whose work
// overlaps on the GPU (other streams, other host threads) would race on it.
#include <cuda_runtime.h>

#include <mutex>

#include "pmb_internal.cuh"

namespace {

constexpr int NA_NT = 256;
constexpr int NA_PER = 16;
constexpr int NA_TILE = NA_NT * NA_PER;                 // rows per tile
constexpr int64_t NA_MAX_TILES = PMB_NOALLOC_MAX_ROWS / NA_TILE;
// tile states + tile ticket + status word, in 8-byte words
constexpr int64_t NA_SCRATCH_WORDS = NA_MAX_TILES + 2;

static __device__ __align__(256) unsigned long long g_noalloc_scratch[NA_SCRATCH_WORDS];

std::mutex g_mu;
void* g_scratch_addr[64] = {nullptr};  // device address of the array, per device ordinal

// Same single-pass decoupled look-back scan as pmb_filter.cu's k_cumsum_u8; the scratch words
// come in as a pointer: [0, tiles) tile states, [tiles] ticket, [tiles + 1] status.
__global__ void __launch_bounds__(NA_NT) k_cumsum_u8_noalloc(const uint8_t* __restrict__ in,
                                                             uint32_t* __restrict__ out, int64_t n,
                                                             unsigned long long* scratch, int64_t tiles) {
  __shared__ uint32_t s_warp[NA_NT / 32];
  __shared__ long long s_tile;
  __shared__ unsigned long long s_base;
  unsigned long long* lb = scratch;
  unsigned long long* ticket = scratch + tiles;
  unsigned int* status = reinterpret_cast<unsigned int*>(scratch + tiles + 1);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_tile = (long long)atomicAdd(ticket, 1ULL);
  __syncthreads();
  const long long tile = s_tile;
  const int64_t r0 = tile * NA_TILE + (int64_t)tid * NA_PER;
  uint32_t v[NA_PER];
  uint32_t sum = 0;
  for (int j = 0; j < NA_PER; j++) {
    int64_t r = r0 + j;
    v[j] = r < n ? in[r] : 0u;
    sum += v[j];
  }
  uint32_t x = sum;
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (tid == 0) {
    uint32_t acc = 0;
    for (int w = 0; w < NA_NT / 32; w++) {
      uint32_t t = s_warp[w];
      s_warp[w] = acc;
      acc += t;
    }
    s_base = pmb_lookback(lb, tile, acc, status);
  }
  __syncthreads();
  uint32_t run = (uint32_t)s_base + s_warp[warp] + (x - sum);
  for (int j = 0; j < NA_PER; j++) {
    run += v[j];
    int64_t r = r0 + j;
    if (r < n) out[r] = run;
  }
}

}  // namespace

extern "C" int pmb_cumsum_u8_to_u32_noalloc(const uint8_t* in, uint32_t* out, int64_t n, void* cuda_stream) {
  if (n < 0 || n > PMB_NOALLOC_MAX_ROWS) return PMB_E_INVALID;  // beyond the fixed scratch
  if (n == 0) return PMB_OK;
  if (!in || !out) return PMB_E_INVALID;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return PMB_E_CUDA;
  void* scratch = nullptr;
  {
    // set-up, once per device, with that device current
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
      if (cudaGetSymbolAddress(&g_scratch_addr[dev], g_noalloc_scratch) != cudaSuccess) {
        g_scratch_addr[dev] = nullptr;
        cudaGetLastError();
        return PMB_E_CUDA;
      }
    }
    scratch = g_scratch_addr[dev];
  }
  cudaStream_t s = (cudaStream_t)cuda_stream;
  const int64_t tiles = (n + NA_TILE - 1) / NA_TILE;
  unsigned long long* words = (unsigned long long*)scratch;
  // the previous call's tile states, ticket and status are still there: clear this call's part
  if (cudaMemsetAsync(words, 0, (size_t)tiles * 8, s) != cudaSuccess) return PMB_E_CUDA;
  if (cudaMemsetAsync(words + NA_MAX_TILES, 0, 16, s) != cudaSuccess) return PMB_E_CUDA;
  k_cumsum_u8_noalloc<<<(unsigned)tiles, NA_NT, 0, s>>>(in, out, n, words, NA_MAX_TILES);
  if (cudaGetLastError() != cudaSuccess) return PMB_E_CUDA;
  // the status word says whether a bounded wait gave up (read into host stack memory)
  unsigned int status = 0;
  if (cudaMemcpyAsync(&status, words + NA_MAX_TILES + 1, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return PMB_E_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return PMB_E_CUDA;
  return (status & PMB_ST_TIMEOUT) ? PMB_E_TIMEOUT : PMB_OK;
}
