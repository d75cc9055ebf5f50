// Host side of a persistent kernel's request ring (the protocol is stated in
// ../cuda/pml_device.cuh, FitQueue): requests and their sequence numbers go
// into device memory by copies on one stream, results and done flags come back
// through host memory mapped into the device's address space.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <functional>
#include <memory>
#include <mutex>
#include <string>

namespace nebula {

class RequestQueue {
 public:
  // Device pointers a persistent kernel takes (see FitQueue).
  struct View {
    const void* ring;
    const long long* seq;
    const int* stop;
    unsigned long long* taken;
    void* results;
    long long* done;
    int* status;
    long long mask;
    long long idle_ns;
  };

  // request_bytes, result_bytes: one ticket's request and result; capacity:
  // tickets in the ring, a power of two. Nothing is allocated before start().
  RequestQueue(size_t request_bytes, size_t result_bytes, size_t capacity);
  ~RequestQueue();
  RequestQueue(const RequestQueue&) = delete;
  RequestQueue& operator=(const RequestQueue&) = delete;

  // Restarts the tickets at zero and calls launch(view) to start the
  // persistent kernel on `stream` (after the resets, which run on it).
  void start(cudaStream_t stream, const std::function<cudaError_t(const View&)>& launch);
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
  bool running();
  // Tells waiting clusters to exit and waits for the kernel; NB_ERR_GPU if a
  // wait ran out. abort(): the same without throwing.
  void stop();
  void abort() noexcept;
  // Throws NB_ERR_GPU describing the queue's state (`what` happened).
  [[noreturn]] void failure(const char* what);
  double device_ms() const { return device_ms_; }
  size_t capacity() const { return capacity_; }

 private:
  void stop_impl(bool check);
  void copy_range(void* dst, const void* src, size_t elem, long long first, size_t n);
  long long post_impl(const void* requests, size_t n, bool wait);
  bool slot_free(long long ticket) const;
  size_t request_bytes_, result_bytes_, capacity_;
  char* d_ring_ = nullptr;
  long long* d_seq_ = nullptr;
  int* d_stop_ = nullptr;
  unsigned long long* d_taken_ = nullptr;
  int* d_status_ = nullptr;
  char* h_ring_ = nullptr;      // pinned staging, slot for slot
  long long* h_seq_ = nullptr;  // pinned staging, slot for slot
  int* h_one_ = nullptr;        // pinned: 1
  char* h_results_ = nullptr;   // mapped
  long long* h_done_ = nullptr; // mapped
  cudaStream_t post_stream_ = nullptr;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr, ready_ = nullptr;
  std::atomic<long long> next_{0};
  std::unique_ptr<std::atomic<long long>[]> consumed_;  // per slot: last ticket read + 1
  std::mutex post_mu_;
  bool running_ = false;
  int device_ = -1;
  double device_ms_ = 0.0;
};

}  // namespace nebula
