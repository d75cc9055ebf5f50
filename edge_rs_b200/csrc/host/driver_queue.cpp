// Host side of the persistent kernels' request rings (driver_queue.hpp).
#include "driver_queue.hpp"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <thread>
#include <vector>

#include "common.hpp"

namespace nebula {
namespace {

constexpr long long kIdleNs = 30000000000LL;  // longest wait of a cluster for work: 30 s

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) fail(NB_ERR_GPU, std::string(what) + ": " + cudaGetErrorString(e));
}

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// A ring's buffers, stream and events. Pinned and mapped host memory is slow
// to allocate and to free, so a ring's set goes back to a process-wide pool
// when the ring is destroyed and the next ring of the same shape on the same
// device takes it (the memory is held until the process exits).
struct RingSet {
  int device;
  size_t request_bytes, result_bytes, capacity;
  char* d_ring;
  long long* d_seq;
  int* d_stop;
  unsigned long long* d_taken;
  int* d_status;
  char* h_ring;
  long long* h_seq;
  int* h_one;
  char* h_results;
  long long* h_done;
  cudaStream_t post_stream;
  cudaEvent_t ev0, ev1, ready;
};

std::mutex& pool_mutex() {
  static std::mutex mu;
  return mu;
}
std::vector<RingSet>& ring_pool() {
  static std::vector<RingSet>* pool = new std::vector<RingSet>();  // kept until exit
  return *pool;
}

}  // namespace

RequestQueue::RequestQueue(size_t request_bytes, size_t result_bytes, size_t capacity)
    : request_bytes_(request_bytes), result_bytes_(result_bytes), capacity_(capacity) {}

RequestQueue::~RequestQueue() {
  abort();
  if (!d_ring_) return;
  cudaStreamSynchronize(post_stream_);
  std::lock_guard<std::mutex> lock(pool_mutex());
  ring_pool().push_back(RingSet{device_, request_bytes_, result_bytes_, capacity_, d_ring_, d_seq_, d_stop_,
                                d_taken_, d_status_, h_ring_, h_seq_, h_one_, h_results_, h_done_, post_stream_,
                                ev0_, ev1_, ready_});
}

void RequestQueue::start(cudaStream_t stream, const std::function<cudaError_t(const View&)>& launch) {
  if (running_) fail(NB_ERR_GPU, "the work queue is already running");
  const size_t cap = capacity_;
  if (!d_ring_) {
    check(cudaGetDevice(&device_), "cudaGetDevice");
    std::lock_guard<std::mutex> lock(pool_mutex());
    std::vector<RingSet>& pool = ring_pool();
    for (size_t i = 0; i < pool.size(); ++i) {
      const RingSet& r = pool[i];
      if (r.device != device_ || r.request_bytes != request_bytes_ || r.result_bytes != result_bytes_ ||
          r.capacity != cap)
        continue;
      d_ring_ = r.d_ring;
      d_seq_ = r.d_seq;
      d_stop_ = r.d_stop;
      d_taken_ = r.d_taken;
      d_status_ = r.d_status;
      h_ring_ = r.h_ring;
      h_seq_ = r.h_seq;
      h_one_ = r.h_one;
      h_results_ = r.h_results;
      h_done_ = r.h_done;
      post_stream_ = r.post_stream;
      ev0_ = r.ev0;
      ev1_ = r.ev1;
      ready_ = r.ready;
      pool.erase(pool.begin() + static_cast<long>(i));
      break;
    }
  }
  if (!d_ring_) {
    check(cudaEventCreate(&ev0_), "event");
    check(cudaEventCreate(&ev1_), "event");
    check(cudaEventCreateWithFlags(&ready_, cudaEventDisableTiming), "event");
    check(cudaStreamCreateWithFlags(&post_stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    check(cudaMalloc(reinterpret_cast<void**>(&d_ring_), cap * request_bytes_), "cudaMalloc");
    check(cudaMalloc(reinterpret_cast<void**>(&d_seq_), cap * sizeof(long long)), "cudaMalloc");
    check(cudaMalloc(reinterpret_cast<void**>(&d_stop_), sizeof(int)), "cudaMalloc");
    check(cudaMalloc(reinterpret_cast<void**>(&d_taken_), sizeof(unsigned long long)), "cudaMalloc");
    check(cudaMalloc(reinterpret_cast<void**>(&d_status_), sizeof(int)), "cudaMalloc");
    check(cudaMallocHost(reinterpret_cast<void**>(&h_ring_), cap * request_bytes_), "cudaMallocHost");
    check(cudaMallocHost(reinterpret_cast<void**>(&h_seq_), cap * sizeof(long long)), "cudaMallocHost");
    check(cudaMallocHost(reinterpret_cast<void**>(&h_one_), sizeof(int)), "cudaMallocHost");
    *h_one_ = 1;
    check(cudaHostAlloc(reinterpret_cast<void**>(&h_results_), cap * result_bytes_, cudaHostAllocMapped),
          "cudaHostAlloc");
    check(cudaHostAlloc(reinterpret_cast<void**>(&h_done_), cap * sizeof(long long), cudaHostAllocMapped),
          "cudaHostAlloc");
  }
  // tickets restart at zero: no stale sequence number or done flag may match one
  std::memset(h_done_, 0, cap * sizeof(long long));
  if (!consumed_) consumed_.reset(new std::atomic<long long>[cap]);
  for (size_t i = 0; i < cap; ++i) consumed_[i].store(0);
  next_.store(0);
  check(cudaMemsetAsync(d_seq_, 0xff, cap * sizeof(long long), stream), "memset");
  check(cudaMemsetAsync(d_stop_, 0, sizeof(int), stream), "memset");
  check(cudaMemsetAsync(d_taken_, 0, sizeof(unsigned long long), stream), "memset");
  check(cudaMemsetAsync(d_status_, 0, sizeof(int), stream), "memset");
  check(cudaEventRecord(ready_, stream), "event");
  check(cudaStreamWaitEvent(post_stream_, ready_, 0), "stream wait");  // posts follow the resets
  View v{};
  v.ring = d_ring_;
  v.seq = d_seq_;
  v.stop = d_stop_;
  v.taken = d_taken_;
  void* dev_ptr = nullptr;
  check(cudaHostGetDevicePointer(&dev_ptr, h_results_, 0), "mapped results");
  v.results = dev_ptr;
  check(cudaHostGetDevicePointer(&dev_ptr, h_done_, 0), "mapped flags");
  v.done = static_cast<long long*>(dev_ptr);
  v.status = d_status_;
  v.mask = static_cast<long long>(cap - 1);
  v.idle_ns = kIdleNs;
  check(cudaEventRecord(ev0_, stream), "event");
  check(launch(v), "queue kernel launch");
  check(cudaEventRecord(ev1_, stream), "event");
  running_ = true;
}

void RequestQueue::copy_range(void* dst, const void* src, size_t elem, long long first, size_t n) {
  const long long mask = static_cast<long long>(capacity_ - 1);
  size_t copied = 0;
  while (copied < n) {
    const size_t slot = static_cast<size_t>((first + static_cast<long long>(copied)) & mask);
    const size_t len = std::min(n - copied, capacity_ - slot);
    check(cudaMemcpyAsync(static_cast<char*>(dst) + slot * elem, static_cast<const char*>(src) + slot * elem,
                          len * elem, cudaMemcpyHostToDevice, post_stream_),
          "queue copy");
    copied += len;
  }
}

long long RequestQueue::post(const void* requests, size_t n) { return post_impl(requests, n, true); }

long long RequestQueue::try_post(const void* requests, size_t n) { return post_impl(requests, n, false); }

void RequestQueue::consumed(long long ticket) {
  if (ticket >= 0) consumed_[ticket & static_cast<long long>(capacity_ - 1)].store(ticket + 1, std::memory_order_release);
}

// Ticket t may take its slot once the slot's previous ticket, t - capacity,
// has been read.
bool RequestQueue::slot_free(long long t) const {
  const long long cap = static_cast<long long>(capacity_);
  return t < cap || consumed_[t & (cap - 1)].load(std::memory_order_acquire) == t - cap + 1;
}

long long RequestQueue::post_impl(const void* requests, size_t n, bool wait) {
  if (n == 0) return next_.load();
  if (n > capacity_ / 2) fail(NB_ERR_GPU, "too many requests in one post");
  // One post at a time through one stream: copies from several streams into
  // neighbouring ring slots lost updates.
  std::lock_guard<std::mutex> lock(post_mu_);
  const long long first = next_.load();
  const long long cap = static_cast<long long>(capacity_);
  const long long mask = cap - 1;
  for (size_t i = 0; i < n; ++i) {
    const long long t = first + static_cast<long long>(i);
    if (slot_free(t)) continue;
    if (!wait) return -1;
    // the slot's previous result has not been read yet: wait for it (bounded)
    const auto t0 = std::chrono::steady_clock::now();
    while (!slot_free(t)) {
      if (!running()) failure("ended with work pending");
      if (ms_since(t0) > 60000.0) failure("made no progress for 60 s");
      std::this_thread::yield();
    }
  }
  next_.store(first + static_cast<long long>(n));
  const char* src = static_cast<const char*>(requests);
  for (size_t i = 0; i < n; ++i) {
    const long long t = first + static_cast<long long>(i);
    std::memcpy(h_ring_ + static_cast<size_t>(t & mask) * request_bytes_, src + i * request_bytes_,
                request_bytes_);
    h_seq_[t & mask] = t;
  }
  // the requests, then (later on the same stream) their sequence numbers
  copy_range(d_ring_, h_ring_, request_bytes_, first, n);
  copy_range(d_seq_, h_seq_, sizeof(long long), first, n);
  return first;
}

bool RequestQueue::done(long long ticket) const {
  if (ticket < 0) return false;  // not posted yet
  long long& flag = h_done_[ticket & static_cast<long long>(capacity_ - 1)];
  return std::atomic_ref<long long>(flag).load(std::memory_order_acquire) == ticket + 1;
}

const void* RequestQueue::result(long long ticket) const {
  return h_results_ + static_cast<size_t>(ticket & static_cast<long long>(capacity_ - 1)) * result_bytes_;
}

bool RequestQueue::running() {
  const cudaError_t e = cudaEventQuery(ev1_);
  if (e == cudaErrorNotReady) return true;
  check(e, "queue kernel");
  return false;
}

void RequestQueue::stop_impl(bool check_status) {
  if (!running_) return;
  running_ = false;
  const cudaError_t e1 = cudaMemcpyAsync(d_stop_, h_one_, sizeof(int), cudaMemcpyHostToDevice, post_stream_);
  const cudaError_t e2 = cudaEventSynchronize(ev1_);
  int status = 0;
  const cudaError_t e3 = cudaMemcpy(&status, d_status_, sizeof(int), cudaMemcpyDeviceToHost);
  cudaStreamSynchronize(post_stream_);
  if (!check_status) return;
  check(e1, "stop copy");
  check(e2, "queue kernel");
  check(e3, "queue status");
  float ms = 0.0f;
  check(cudaEventElapsedTime(&ms, ev0_, ev1_), "event time");
  device_ms_ += ms;
  if (status != 0) fail(NB_ERR_GPU, "a queue cluster waited more than 30 s for work");
}

void RequestQueue::stop() { stop_impl(true); }

void RequestQueue::abort() noexcept {
  try {
    stop_impl(false);
  } catch (...) {
  }
}

void RequestQueue::failure(const char* what) {
  int status = -1;
  cudaMemcpy(&status, d_status_, sizeof(int), cudaMemcpyDeviceToHost);
  unsigned long long taken = 0;
  cudaMemcpy(&taken, d_taken_, sizeof(taken), cudaMemcpyDeviceToHost);
  fail(NB_ERR_GPU, std::string("the queue kernel ") + what + " (tickets posted " + std::to_string(next_.load()) +
                       ", taken " + std::to_string(taken) +
                       (status == 1 ? ", a cluster waited more than 30 s for work)" : ")"));
}

}  // namespace nebula
