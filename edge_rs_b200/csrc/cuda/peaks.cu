// Microbenchmark of the FP64 FMA pipe, the roofline the fit kernel is held to
// (its work is FP64 FMAs, adds, multiplies and divisions; no tensor core or
// HBM stream bounds it). Every thread runs 8 independent FMA chains so the
// pipe, not the dependency latency, sets the rate; the grid is sized to keep
// every SM full.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "../host/export.hpp"

namespace {

constexpr int kChains = 8;

__global__ void fma_chains(double* out, int iters, double b, double c) {
  double a[kChains];
#pragma unroll
  for (int i = 0; i < kChains; ++i) a[i] = threadIdx.x * 1e-9 + i;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < kChains; ++i) a[i] = __fma_rn(a[i], b, c);
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < kChains; ++i) s += a[i];
  if (s == 12345.678) out[threadIdx.x] = s;  // keeps the chains alive
}

}  // namespace

// Measured FP64 FMA throughput of the current device in TFLOP/s (2 flops per
// FMA), best of `repeats` timed launches after one warm-up. Returns a
// negative value on a CUDA error.
NB_API double nb_measure_fp64_tflops(int repeats) {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1.0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1.0;
  double* out = nullptr;
  if (cudaMalloc(&out, 1024 * sizeof(double)) != cudaSuccess) return -1.0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int threads = 256, blocks = sms * 8, iters = 1 << 14;
  const double flops = 2.0 * kChains * static_cast<double>(iters) * threads * blocks;
  double best = 0.0;
  for (int r = 0; r <= repeats; ++r) {
    cudaEventRecord(e0);
    fma_chains<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
    cudaEventRecord(e1);
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      best = -1.0;
      break;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0 && ms > 0.0f) best = std::max(best, flops / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  return best;
}
