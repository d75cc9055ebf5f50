// Widens the positive counts the upload moved as floats (whole counts below
// 2^24, exact in a float) into the double array the kernels read.
#include <cuda_runtime.h>

#include "pml_device.cuh"

namespace nebula {
namespace device {
namespace {

__global__ void widen_counts_kernel(const float* __restrict__ src, double* __restrict__ dst, size_t n) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    dst[i] = static_cast<double>(src[i]);
}

}  // namespace

int widen_counts(const float* src, double* dst, size_t n, void* stream) {
  if (n == 0) return cudaSuccess;
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const size_t blocks = (n + 255) / 256;
  const int grid = static_cast<int>(blocks < static_cast<size_t>(8 * sms) ? blocks : static_cast<size_t>(8 * sms));
  widen_counts_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(src, dst, n);
  return cudaGetLastError();
}

}  // namespace device
}  // namespace nebula
