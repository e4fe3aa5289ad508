// Memory-system probe: the random-access ceilings that bound the engine's kernels.
//
// The level kernels of the GST engine are not streaming kernels: every relaxation reads
// the 32-byte distance row (or one 8-byte state cell) of a random target vertex and
// updates it with an atomic.  The streaming copy bandwidth of the device is therefore
// not what they can reach; the random-sector rate is.  This probe measures
// it on the device the engine runs on: uniformly random 32-byte row gathers from an
// array far larger than the L2 (the DRAM-bound case), the same from an array the L2
// holds, and random 4-byte atomicMin reductions.  It allocates its array itself (this
// is a diagnostic, not a solve path).
#include <algorithm>
#include <cstdint>

#include <cuda_runtime.h>

#include "gst.h"

namespace {

__device__ __forceinline__ uint64_t probe_mix(uint64_t x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdull;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ull;
  x ^= x >> 33;
  return x;
}

// iters x 4 independent random 32-byte rows per thread (two 16-byte loads each)
__global__ void probe_gather32(const uint4* __restrict__ a, uint64_t nrows, uint64_t iters,
                               uint32_t* out) {
  const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  uint32_t acc = 0;
  for (uint64_t i = 0; i < iters; i++) {
    uint4 r[4], s[4];
#pragma unroll
    for (int x = 0; x < 4; x++) {
      const uint64_t idx = probe_mix(t * 1315423911ull + i * 4 + x) % nrows;
      r[x] = __ldcg(a + 2 * idx);
      s[x] = __ldcg(a + 2 * idx + 1);
    }
#pragma unroll
    for (int x = 0; x < 4; x++) acc ^= r[x].x ^ s[x].w;
  }
  out[t] = acc;
}

// iters x 4 random 4-byte atomicMin reductions per thread
__global__ void probe_red32(uint32_t* a, uint64_t n, uint64_t iters) {
  const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  for (uint64_t i = 0; i < iters; i++) {
#pragma unroll
    for (int x = 0; x < 4; x++) {
      const uint64_t idx = probe_mix(t * 2654435761ull + i * 4 + x) % n;
      atomicMin(a + idx, (uint32_t)(i + x));
    }
  }
}

}  // namespace

extern "C" gst_status gst_probe_random_access(int32_t device, int64_t bytes, double* gather_dram,
                                              double* gather_l2, double* red_dram) {
  if (bytes < (int64_t)(256 << 20) || !gather_dram || !gather_l2 || !red_dram) return GST_BAD_INPUT;
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess)
    return GST_DEVICE_ERROR;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int blocks = sms * 8, threads = 256;
  const uint64_t nthreads = (uint64_t)blocks * threads;
  uint4* a = nullptr;
  uint32_t* out = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  gst_status st = GST_OK;
  float ms = 0;
  if (cudaMalloc(&a, (size_t)bytes) != cudaSuccess || cudaMalloc(&out, nthreads * 4) != cudaSuccess ||
      cudaMemset(a, 0x7f, (size_t)bytes) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
      cudaEventCreate(&e1) != cudaSuccess) {
    st = GST_DEVICE_ERROR;
  } else {
    const uint64_t iters = 16;  // x 4 accesses per thread
    const uint64_t n = nthreads * iters * 4;
    const uint64_t rows_big = (uint64_t)bytes / 32, rows_l2 = (uint64_t)(32 << 20) / 32;
    double best[3] = {0, 0, 0};
    for (int rep = 0; rep < 3; rep++) {
      cudaEventRecord(e0);
      probe_gather32<<<blocks, threads>>>(a, rows_big, iters, out);
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      cudaEventElapsedTime(&ms, e0, e1);
      best[0] = std::max(best[0], n / (ms * 1e-3));
      cudaEventRecord(e0);
      probe_gather32<<<blocks, threads>>>(a, rows_l2, iters, out);
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      cudaEventElapsedTime(&ms, e0, e1);
      best[1] = std::max(best[1], n / (ms * 1e-3));
      cudaEventRecord(e0);
      probe_red32<<<blocks, threads>>>((uint32_t*)a, (uint64_t)bytes / 4, iters);
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      cudaEventElapsedTime(&ms, e0, e1);
      best[2] = std::max(best[2], n / (ms * 1e-3));
    }
    if (cudaGetLastError() != cudaSuccess) st = GST_DEVICE_ERROR;
    *gather_dram = best[0];
    *gather_l2 = best[1];
    *red_dram = best[2];
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (out) cudaFree(out);
  if (a) cudaFree(a);
  cudaSetDevice(prev);
  return st;
}
