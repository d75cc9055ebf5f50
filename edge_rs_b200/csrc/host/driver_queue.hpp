// Host side of a persistent kernel's request ring (the protocol is stated
// beside device::RingView in ../cuda/pml_device.cuh). What the host and the
// running kernel exchange lives in pinned host memory mapped into the
// device's address space: requests and the `posted` counter go one way,
// results, done flags and the status word the other. No copy engine and no
// stream order is involved, so the ring works whether or not other GPU work
// can run beside the kernel (a profiler that serialises launches,
// CUDA_LAUNCH_BLOCKING), and requests may be posted before the launch.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <functional>
#include <memory>
#include <mutex>
#include <string>

#include "../cuda/pml_device.cuh"

namespace nebula {

class RequestQueue {
 public:
  // Device pointers a persistent kernel takes (see RingView, FitQueue).
  struct View {
    device::RingView ring;
    void* results;
    long long* done;
  };

  // request_bytes, result_bytes: one ticket's request and result; capacity:
  // tickets in the ring, a power of two. Nothing is allocated before prepare().
  RequestQueue(size_t request_bytes, size_t result_bytes, size_t capacity);
  ~RequestQueue();
  RequestQueue(const RequestQueue&) = delete;
  RequestQueue& operator=(const RequestQueue&) = delete;

  // Restarts the tickets at zero (the device-side counters are reset on
  // `stream`). Requests may be posted from here on.
  void prepare(cudaStream_t stream);
  // Calls launch(view) to start the persistent kernel on `stream`, between
  // two events that time it. Under a profiler that serialises launches this
  // returns only once the kernel has ended, so the threads that post, read
  // results and finally call request_stop() must be running already.
  void launch(cudaStream_t stream, const std::function<cudaError_t(const View&)>& launch);
  // Copies n requests into the ring (safe from several host threads; one at
  // a time) and returns the first one's ticket. A slot is reused only once
  // the result of the ticket it last held has been read (consumed()); post
  // waits for that (bounded), try_post returns -1 instead and posts nothing.
  // A thread that reads results itself must use try_post: it could otherwise
  // wait on a result only it would read.
  long long post(const void* requests, size_t n);
  long long try_post(const void* requests, size_t n);
  // The caller has read ticket's result: its slot may take a new ticket.
  void consumed(long long ticket);
  bool done(long long ticket) const;
  const void* result(long long ticket) const;
  // True from prepare() until the launched kernel has ended.
  bool running();
  // Tells clusters waiting for work to exit once no ticket is left (any
  // thread, any number of times).
  void request_stop() noexcept;
  // request_stop(), then waits for the kernel; NB_ERR_GPU if a wait ran out.
  // abort(): the same without throwing.
  void stop();
  void abort() noexcept;
  // Throws NB_ERR_GPU describing the queue's state (`what` happened).
  [[noreturn]] void failure(const char* what);
  double device_ms() const { return device_ms_; }
  size_t capacity() const { return capacity_; }
  // How long a cluster waits for its ticket's request before it sets the
  // status word and exits (default 5 s); takes effect at the next launch.
  void set_idle_ns(long long ns) { idle_ns_ = ns; }

 private:
  enum State : int { kIdle = 0, kPrepared = 1, kLaunched = 2 };
  void stop_impl(bool check);
  long long post_impl(const void* requests, size_t n, bool wait);
  bool slot_free(long long ticket) const;
  size_t request_bytes_, result_bytes_, capacity_;
  unsigned long long* d_words_ = nullptr;  // device: the ring's counters (kRingWords)
  char* d_ring_ = nullptr;                 // device: forwarded requests
  char* h_ring_ = nullptr;                 // mapped: requests, slot for slot
  unsigned long long* h_posted_ = nullptr; // mapped: tickets below it are posted
  int* h_stop_ = nullptr;       // mapped: nonzero once no ticket will be posted
  int* h_status_ = nullptr;     // mapped: 1 once a cluster's wait ran out
  char* h_results_ = nullptr;   // mapped
  long long* h_done_ = nullptr; // mapped
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  std::atomic<long long> next_{0};
  std::unique_ptr<std::atomic<long long>[]> consumed_;  // per slot: last ticket read + 1
  std::mutex post_mu_;
  std::atomic<int> state_{kIdle};
  int device_ = -1;
  double device_ms_ = 0.0;
  long long idle_ns_;
};

}  // namespace nebula
