// dtmx_noalloc.cu -- NaN/Inf count over caller-owned device arrays that
// allocates no device memory.
//
// Who needs this: a caller whose device memory is owned by another allocator
// that has reserved the whole pool (so a cudaMalloc of its own would fail or
// fragment that pool), or a watchdog/health-check thread that must not call
// cudaMalloc/cudaFree (they take the allocator's locks and can synchronise
// the device).  Such a caller passes its own device arrays in and gets a host
// count back; the scratch the reduction needs is a fixed array below.
//
// Scratch: g_partial holds one count per block of DTMX_NOALLOC_BLOCK_ELEMS
// elements plus the final total.  It is a file-scope __device__ array, so every
// GPU that loads this library holds it (DTMX_NOALLOC_MAX_BLOCKS + 1 eight-byte
// words, 32 KiB) until the process exits.  Each field is cut into its own
// blocks (the last one partial), so the limit is on the block count:
// nfields * ceil(nelem / DTMX_NOALLOC_BLOCK_ELEMS) <= DTMX_NOALLOC_MAX_BLOCKS.
// Every call overwrites the entries it uses and the total, so nothing carries
// over from the previous call; two calls whose kernels overlap on the GPU
// (different host threads, same device) race on it.
#include <cuda_runtime.h>
#include <cstdint>

#include "dtmx.h"

namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 16;
constexpr long long kBlockElems = (long long)kThreads * kPerThread;   // 4096 elements per block
static_assert(kBlockElems == DTMX_NOALLOC_BLOCK_ELEMS, "block size of the header");
constexpr int kMaxBlocks = DTMX_NOALLOC_MAX_BLOCKS;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned long long g_partial[kMaxBlocks + 1];

// Device address of g_partial per device, looked up on the first call made
// with that device current.
unsigned long long* g_scratch[kMaxDevices] = {};

__global__ void count_blocks(const float* __restrict__ data, long long nelem, int block_base,
                             unsigned long long* partial) {
  __shared__ unsigned int warp_sum[kThreads / 32];
  const long long start = (long long)blockIdx.x * kBlockElems;
  unsigned int cnt = 0;
#pragma unroll
  for (int q = 0; q < kPerThread; q++) {
    const long long e = start + (long long)q * kThreads + threadIdx.x;
    if (e < nelem && !isfinite(data[e])) cnt++;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int w = 0; w < kThreads / 32; w++) t += warp_sum[w];
    partial[block_base + blockIdx.x] = t;     // overwritten on every call: no clearing needed
  }
}

__global__ void sum_blocks(unsigned long long* partial, int nblocks) {
  __shared__ unsigned long long s[kThreads];
  unsigned long long t = 0;
  for (int b = threadIdx.x; b < nblocks; b += kThreads) t += partial[b];
  s[threadIdx.x] = t;
  __syncthreads();
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[kMaxBlocks] = s[0];   // the total slot, written every call
}

}  // namespace

extern "C" int dtmx_count_nonfinite_noalloc(const float* const* d_fields, int nfields, int64_t nelem,
                                            int64_t* count_out) {
  if (!d_fields || nfields < 1 || nelem < 0 || !count_out) return DTMX_ERR_INVALID;
  // blocks per field, rounded up per field; divided before any product, so no overflow
  const long long per_field = nelem / kBlockElems + (nelem % kBlockElems != 0);
  if (per_field > kMaxBlocks / nfields) return DTMX_ERR_TOO_LARGE;
  for (int f = 0; f < nfields; f++)
    if (!d_fields[f] && nelem > 0) return DTMX_ERR_INVALID;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return DTMX_ERR_NODEVICE;
  if (dev < 0 || dev >= kMaxDevices) return DTMX_ERR_UNSUPPORTED;
  if (!g_scratch[dev]) {
    // set-up on the first call on this device, with this device current
    void* q = nullptr;
    if (cudaGetSymbolAddress(&q, g_partial) != cudaSuccess || !q) return DTMX_ERR_CUDA;
    g_scratch[dev] = static_cast<unsigned long long*>(q);
  }
  unsigned long long* partial = g_scratch[dev];
  int base = 0;
  for (int f = 0; f < nfields && per_field > 0; f++) {
    count_blocks<<<(unsigned)per_field, kThreads>>>(d_fields[f], nelem, base, partial);
    base += (int)per_field;
  }
  sum_blocks<<<1, kThreads>>>(partial, base);
  if (cudaGetLastError() != cudaSuccess) return DTMX_ERR_CUDA;
  unsigned long long total = 0;
  if (cudaMemcpy(&total, partial + kMaxBlocks, sizeof(total), cudaMemcpyDeviceToHost) != cudaSuccess)
    return DTMX_ERR_CUDA;
  *count_out = (int64_t)total;
  return DTMX_OK;
}
