// The request ring's self-check kernel: one-warp CTAs take tickets with
// ring_next, answer each EchoRequest with echo_of and publish it with
// ring_publish, the same protocol the persistent fit and stage-one kernels
// run (ring_device.cuh). The host side is nb_ring_check_cuda.
#include <cuda_runtime.h>

#include "pml_device.cuh"
#include "ring_device.cuh"

namespace nebula {
namespace device {
namespace {

__global__ void __launch_bounds__(32) ring_echo_kernel(RingView ring, EchoResult* results, long long* done) {
  __shared__ EchoRequest req;
  for (;;) {
    const long long t = ring_next(ring, &req, nullptr);
    if (t < 0) return;  // stopped, or the wait for work ran out (status word set)
    if (threadIdx.x == 0) results[t & ring.mask] = echo_of(req, t);
    ring_publish(done + (t & ring.mask), t);
  }
}

}  // namespace

int launch_ring_echo(const RingView& ring, EchoResult* results, long long* done, int ctas, void* stream) {
  if (ctas < 1 || ring.request_bytes != static_cast<int>(sizeof(EchoRequest))) return cudaErrorInvalidValue;
  ring_echo_kernel<<<ctas, 32, 0, static_cast<cudaStream_t>(stream)>>>(ring, results, done);
  return cudaGetLastError();
}

}  // namespace device
}  // namespace nebula
