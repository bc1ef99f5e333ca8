// Throughput probe of shared-memory atomics (no counterpart in the reference).
//
// The pair kernel accumulates its histograms with shared-memory atomics (five
// FP64 sums and a 32-bit count per run of pairs); the benchmark reports the
// shared-atomic term of its bound against a rate measured here on the same
// GPU: every CTA of a one-wave grid adds into a histogram of `nb` bins in
// shared memory, each thread `iters` times, at addresses that are distinct
// within a warp (mode 0), drawn from a fixed pseudo-random bin sequence (mode
// 1), or with 32-bit integer adds at distinct addresses (mode 2).
#include <cuda_runtime.h>
#include <stdint.h>

#include "lya_internal.cuh"

namespace {

constexpr int PROBE_THREADS = 512;
constexpr int PROBE_BINS = 2500;

template <int MODE>
__global__ void __launch_bounds__(PROBE_THREADS, 1) k_probe_atomics(int iters, double* __restrict__ sink) {
  __shared__ double h[PROBE_BINS];
  __shared__ unsigned int c[PROBE_BINS];
  for (int i = threadIdx.x; i < PROBE_BINS; i += blockDim.x) { h[i] = 0.0; c[i] = 0u; }
  __syncthreads();
  // distinct addresses within a warp (lane-strided), or a linear-congruential bin sequence
  unsigned int x = 2654435761u * (blockIdx.x * PROBE_THREADS + threadIdx.x + 1u);
  int b = (threadIdx.x * 37) % PROBE_BINS;
  const double v = 1.0 + threadIdx.x * 1e-3;
  for (int it = 0; it < iters; ++it) {
    if (MODE == 1) {
      x = x * 1664525u + 1013904223u;
      b = (int)((x >> 8) % PROBE_BINS);
    }
    if (MODE < 2) atomicAdd(&h[b], v); else atomicAdd(&c[b], 1u);
    if (MODE != 1) { b += 97; if (b >= PROBE_BINS) b -= PROBE_BINS; }
  }
  __syncthreads();
  double s = 0.0;
  for (int i = threadIdx.x; i < PROBE_BINS; i += blockDim.x) s += h[i] + (double)c[i];
  if (s == -1.0) sink[0] = s;   // keeps the adds; never true
}

}  // namespace

extern "C" int lya_probe_smem_atomics(int device, double* rates) {
  if (!rates) return lya_fail(nullptr, LYA_ERR_ARG, "lya_probe_smem_atomics: rates is NULL");
  cudaError_t e = cudaSetDevice(device);
  int sms = 0;
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaEvent_t a = nullptr, b = nullptr;
  if (e == cudaSuccess) e = cudaEventCreate(&a);
  if (e == cudaSuccess) e = cudaEventCreate(&b);
  const int iters = 4096;
  for (int mode = 0; mode < 3 && e == cudaSuccess; ++mode) {
    float best = 1e30f;
    for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep) {
      e = cudaEventRecord(a, 0);
      if (mode == 0) k_probe_atomics<0><<<sms, PROBE_THREADS>>>(iters, nullptr);
      if (mode == 1) k_probe_atomics<1><<<sms, PROBE_THREADS>>>(iters, nullptr);
      if (mode == 2) k_probe_atomics<2><<<sms, PROBE_THREADS>>>(iters, nullptr);
      if (e == cudaSuccess) e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaEventRecord(b, 0);
      if (e == cudaSuccess) e = cudaEventSynchronize(b);
      float ms = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
      if (e == cudaSuccess && rep > 0 && ms < best) best = ms;   // the first run warms up
    }
    if (e == cudaSuccess) rates[mode] = (double)sms * PROBE_THREADS * iters / (best * 1e-3);
  }
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  if (e != cudaSuccess) return lya_fail(nullptr, LYA_ERR_CUDA, "lya_probe_smem_atomics: %s", cudaGetErrorString(e));
  return LYA_OK;
}
