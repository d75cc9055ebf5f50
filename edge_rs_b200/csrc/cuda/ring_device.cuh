// Device side of the request rings (the protocol is stated beside RingView
// in pml_device.cuh). Waiting clusters poll device words in L2; one waiting
// warp at a time, the holder of the ring's lock, reads the host's `posted`
// counter across the bus and copies the newly posted requests into the
// device ring before advancing `forwarded`.
#pragma once

#include <cstdint>

#include "pml_device.cuh"

namespace nebula {
namespace device {

constexpr int kMaxForward = 256;  // requests one lock hold forwards at most

__device__ __forceinline__ unsigned long long ld_relaxed_gpu(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_acquire_gpu(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed_sys(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.sys.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_acquire_sys(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.sys.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_relaxed_sys(const int* p) {
  int v;
  asm volatile("ld.relaxed.sys.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_acquire_sys(const int* p) {
  int v;
  asm volatile("ld.acquire.sys.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ bool try_lock(unsigned long long* p) {
  unsigned long long old;
  asm volatile("atom.acquire.gpu.global.cas.b64 %0, [%1], %2, %3;"
               : "=l"(old)
               : "l"(p), "l"(0ull), "l"(1ull)
               : "memory");
  return old == 0ull;
}
__device__ __forceinline__ void unlock(unsigned long long* p) {
  asm volatile("st.release.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(0ull) : "memory");
}

__device__ __forceinline__ long long ring_clock_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// By the 32 lanes of the lock holder's warp: forwards the requests posted
// since `forwarded` (at most kMaxForward) into the device ring, publishes the
// new `forwarded`, sets `stopped` when the host has stopped and everything is
// forwarded, and releases the lock. Returns how many requests it forwarded.
__device__ __forceinline__ int ring_forward(const RingView& r, unsigned lane) {
  unsigned long long* w = r.words;
  unsigned long long f = 0, p = 0;
  int stop = 0;
  if (lane == 0) {
    f = ld_relaxed_gpu(w + kForwarded);  // written only under the lock
    // the stop word first: the host stores `posted` before it, so once stop
    // is seen the `posted` read after it is final
    stop = ld_relaxed_sys(r.stop);
    if (stop) stop = ld_acquire_sys(r.stop);
    p = ld_relaxed_sys(r.posted);
    if (p > f) p = ld_acquire_sys(r.posted);  // orders the request reads below after it
    if (p < f) p = f;
    if (p > f + kMaxForward) {
      p = f + kMaxForward;
      stop = 0;  // more to forward first
    }
  }
  f = __shfl_sync(0xffffffffu, f, 0);
  p = __shfl_sync(0xffffffffu, p, 0);
  stop = __shfl_sync(0xffffffffu, stop, 0);
  __syncwarp();
  const long long words = r.request_bytes / 8;
  const long long total = static_cast<long long>(p - f) * words;
  for (long long base = 0; base < total; base += 32 * 4) {
    unsigned long long v[4];
    long long at[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const long long idx = base + u * 32 + lane;
      const long long ticket = static_cast<long long>(f) + idx / words;
      at[u] = idx < total ? ((ticket & r.mask) * words + idx % words) : -1;
      if (at[u] >= 0) v[u] = ld_relaxed_sys(reinterpret_cast<const unsigned long long*>(r.host_ring) + at[u]);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (at[u] >= 0) reinterpret_cast<unsigned long long*>(r.ring)[at[u]] = v[u];
  }
  __threadfence();
  __syncwarp();
  if (lane == 0) {
    if (p > f) st_release_gpu(w + kForwarded, p);
    if (stop) st_release_gpu(w + kStopped, 1ull);
    unlock(w + kLock);
  }
  return static_cast<int>(p - f);
}

// By the 32 lanes of one warp (converged): takes the next ticket, waits for
// its request and copies it into dst (shared memory, r.request_bytes); returns
// the ticket, or -1 once nothing more will be posted or the wait ran out
// (then *status = 1). *wait_ns (lane 0): global-timer ns from taking the
// ticket to holding its request.
__device__ __forceinline__ long long ring_next(const RingView& r, void* dst, long long* wait_ns) {
  const unsigned lane = threadIdx.x & 31u;
  unsigned long long* w = r.words;
  long long t = 0, t0 = 0;
  if (lane == 0) {
    t = static_cast<long long>(atomicAdd(w + kTaken, 1ull));
    t0 = ring_clock_ns();
  }
  t = __shfl_sync(0xffffffffu, t, 0);
  unsigned int pause = 128;
  for (;;) {
    int action = 0;  // 0 back off, 1 ready, 2 holds the lock, 3 exit
    if (lane == 0) {
      if (static_cast<long long>(ld_relaxed_gpu(w + kForwarded)) > t) {
        ld_acquire_gpu(w + kForwarded);
        action = 1;
      } else if (ld_relaxed_gpu(w + kStopped) != 0) {
        ld_acquire_gpu(w + kStopped);  // `forwarded` is final now
        action = static_cast<long long>(ld_relaxed_gpu(w + kForwarded)) > t ? 1 : 3;
      } else if (ring_clock_ns() - t0 > r.idle_ns) {
        *reinterpret_cast<volatile int*>(r.status) = 1;
        __threadfence_system();
        action = 3;
      } else if (try_lock(w + kLock)) {
        action = 2;
      }
    }
    action = __shfl_sync(0xffffffffu, action, 0);
    if (action == 1) break;
    if (action == 3) return -1;
    if (action == 2 && ring_forward(r, lane) > 0) {
      pause = 128;
      continue;  // its own ticket may be among them
    }
    __nanosleep(pause);
    if (pause < 2048) pause *= 2;
  }
  const int words = r.request_bytes / 8;
  const unsigned long long* src =
      reinterpret_cast<const unsigned long long*>(r.ring + static_cast<size_t>(t & r.mask) * r.request_bytes);
  __syncwarp();
  for (int i = static_cast<int>(lane); i < words; i += 32) static_cast<unsigned long long*>(dst)[i] = __ldcg(src + i);
  __syncwarp();
  if (wait_ns && lane == 0) *wait_ns = ring_clock_ns() - t0;
  return t;
}

// After every thread of the CTA has written its part of a result into mapped
// memory: fence them to system scope, then (thread 0) publish done = t + 1.
__device__ __forceinline__ void ring_publish(long long* done, long long t) {
  __threadfence_system();
  __syncthreads();
  if (threadIdx.x == 0) *reinterpret_cast<volatile long long*>(done) = t + 1;
}

}  // namespace device
}  // namespace nebula
