// Integer-pipe throughput probe: the denominator of the DP kernels'
// integer-ALU roofline, measured on the device in use.
//
// The DP recurrences are 32-bit adds and maxes (the per-cell count is
// 6 + 5 x predecessors). Three kernels time the three forms the kernels
// issue them in: a plain add (add.s32), a plain max (max.s32) and the DPX
// fused add-max (__viaddmax_s32, two operations per instruction). Each
// thread runs 8 independent dependency chains so that issue, not latency,
// bounds the loop; the grid fills every SM to its thread limit. The rates
// are operations per second (an add-max counts as two).
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/minipoa_b200.h"

namespace poa {
namespace {

constexpr int PROBE_ITERS = 2048;
constexpr int PROBE_THREADS = 256;

__global__ void __launch_bounds__(PROBE_THREADS) k_probe_add(int32_t *sink, int32_t seed) {
  int32_t a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = seed + int32_t(threadIdx.x) * (k + 1);
  const int32_t b = seed ^ 0x55;
  for (int it = 0; it < PROBE_ITERS; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) asm volatile("add.s32 %0, %0, %1;" : "+r"(a[k]) : "r"(b));
  }
  int32_t x = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) x ^= a[k];
  if (x == seed) sink[threadIdx.x] = x;  // keeps the chains live
}

__global__ void __launch_bounds__(PROBE_THREADS) k_probe_max(int32_t *sink, int32_t seed) {
  int32_t a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = seed + int32_t(threadIdx.x) * (k + 1);
  int32_t b = seed ^ 0x55;
  for (int it = 0; it < PROBE_ITERS; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) asm volatile("max.s32 %0, %0, %1;" : "+r"(a[k]) : "r"(b));
  }
  int32_t x = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) x ^= a[k];
  if (x == seed) sink[threadIdx.x] = x;
}

__global__ void __launch_bounds__(PROBE_THREADS) k_probe_addmax(int32_t *sink, int32_t seed) {
  int32_t a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = seed + int32_t(threadIdx.x) * (k + 1);
  const int32_t e = -(seed & 7) - 1;
  for (int it = 0; it < PROBE_ITERS; ++it) {
    // chain k folds its neighbour in: a[k] = max(a[k] + e, a[k+1]); every
    // result feeds the next iteration, so no operation can be hoisted
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = __viaddmax_s32(a[k], e, a[(k + 1) & 7]);
  }
  int32_t x = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) x ^= a[k];
  if (x == seed) sink[threadIdx.x] = x;
}

}  // namespace
}  // namespace poa

extern "C" int poa_probe_int_peak(int32_t device, double *out_ops_per_s) {
  using namespace poa;
  if (!out_ops_per_s) return POA_ERR_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return POA_ERR_CUDA;
  int sms = 0, max_threads = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
      cudaDeviceGetAttribute(&max_threads, cudaDevAttrMaxThreadsPerMultiProcessor, device) != cudaSuccess)
    return POA_ERR_CUDA;
  const int blocks = sms * (max_threads / PROBE_THREADS);
  int32_t *sink = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = POA_OK;
  if (cudaMalloc(&sink, PROBE_THREADS * sizeof(int32_t)) != cudaSuccess) return POA_ERR_ALLOC;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    rc = POA_ERR_CUDA;
  }
  // per form: instructions per thread per launch x operations per instruction
  const double per_thread[3] = {double(PROBE_ITERS) * 8, double(PROBE_ITERS) * 8, double(PROBE_ITERS) * 8 * 2};
  for (int form = 0; form < 3 && rc == POA_OK; ++form) {
    float best = 0;
    for (int rep = 0; rep < 4 && rc == POA_OK; ++rep) {  // the first launch warms up
      cudaEventRecord(e0, st);
      if (form == 0) k_probe_add<<<blocks, PROBE_THREADS, 0, st>>>(sink, 12345 + rep);
      if (form == 1) k_probe_max<<<blocks, PROBE_THREADS, 0, st>>>(sink, 12345 + rep);
      if (form == 2) k_probe_addmax<<<blocks, PROBE_THREADS, 0, st>>>(sink, 12345 + rep);
      cudaEventRecord(e1, st);
      if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
        rc = POA_ERR_CUDA;
        break;
      }
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 0 && (best == 0 || ms < best)) best = ms;
    }
    out_ops_per_s[form] = best > 0 ? double(blocks) * PROBE_THREADS * per_thread[form] / (best / 1e3) : 0.0;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  cudaFree(sink);
  return rc;
}
