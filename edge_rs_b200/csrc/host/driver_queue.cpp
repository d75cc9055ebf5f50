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

// Longest wait of a cluster for its ticket: 5 s. Tickets are posted as
// results come back, so a cluster waits at most about as long as the
// longest fit in flight (milliseconds); a ring that stalls fails within
// seconds instead of holding every SM.
constexpr long long kIdleNs = 5000000000LL;
constexpr double kHostWaitMs = 60000.0;  // a post's wait for a slot to be read

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) fail(NB_ERR_GPU, std::string(what) + ": " + cudaGetErrorString(e));
}

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

template <typename T>
T* device_view(T* host) {
  void* p = nullptr;
  check(cudaHostGetDevicePointer(&p, host, 0), "mapped pointer");
  return static_cast<T*>(p);
}

// A ring's buffers and events. Pinned and mapped host memory is slow to
// allocate and to free, so a ring's set goes back to a process-wide pool when
// the ring is destroyed and the next ring of the same shape on the same
// device takes it (the memory is held until the process exits).
struct RingSet {
  int device;
  size_t request_bytes, result_bytes, capacity;
  unsigned long long* d_words;
  char* d_ring;
  char* h_ring;
  unsigned long long* h_posted;
  int* h_stop;
  int* h_status;
  char* h_results;
  long long* h_done;
  cudaEvent_t ev0, ev1;
};

std::mutex& pool_mutex() {
  static std::mutex mu;
  return mu;
}
std::vector<RingSet>& ring_pool() {
  static std::vector<RingSet>* pool = new std::vector<RingSet>();  // kept until exit
  return *pool;
}

void* mapped_alloc(size_t bytes) {
  void* p = nullptr;
  check(cudaHostAlloc(&p, bytes, cudaHostAllocMapped), "cudaHostAlloc");
  return p;
}

}  // namespace

RequestQueue::RequestQueue(size_t request_bytes, size_t result_bytes, size_t capacity)
    : request_bytes_(request_bytes), result_bytes_(result_bytes), capacity_(capacity), idle_ns_(kIdleNs) {}

static std::string idle_text(long long ns) {
  return ns % 1000000000LL == 0 ? std::to_string(ns / 1000000000LL) + " s" : std::to_string(ns / 1000000LL) + " ms";
}

RequestQueue::~RequestQueue() {
  abort();
  if (!h_ring_) return;
  std::lock_guard<std::mutex> lock(pool_mutex());
  ring_pool().push_back(RingSet{device_, request_bytes_, result_bytes_, capacity_, d_words_, d_ring_, h_ring_,
                                h_posted_, h_stop_, h_status_, h_results_, h_done_, ev0_, ev1_});
}

void RequestQueue::prepare(cudaStream_t stream) {
  if (state_.load() != kIdle) fail(NB_ERR_GPU, "the work queue is already running");
  const size_t cap = capacity_;
  if (!h_ring_) {
    check(cudaGetDevice(&device_), "cudaGetDevice");
    std::lock_guard<std::mutex> lock(pool_mutex());
    std::vector<RingSet>& pool = ring_pool();
    for (size_t i = 0; i < pool.size(); ++i) {
      const RingSet& r = pool[i];
      if (r.device != device_ || r.request_bytes != request_bytes_ || r.result_bytes != result_bytes_ ||
          r.capacity != cap)
        continue;
      d_words_ = r.d_words;
      d_ring_ = r.d_ring;
      h_ring_ = r.h_ring;
      h_posted_ = r.h_posted;
      h_stop_ = r.h_stop;
      h_status_ = r.h_status;
      h_results_ = r.h_results;
      h_done_ = r.h_done;
      ev0_ = r.ev0;
      ev1_ = r.ev1;
      pool.erase(pool.begin() + static_cast<long>(i));
      break;
    }
  }
  if (!h_ring_) {
    check(cudaEventCreate(&ev0_), "event");
    check(cudaEventCreate(&ev1_), "event");
    check(cudaMalloc(reinterpret_cast<void**>(&d_words_), device::kRingWords * sizeof(unsigned long long)),
          "cudaMalloc");
    check(cudaMalloc(reinterpret_cast<void**>(&d_ring_), cap * request_bytes_), "cudaMalloc");
    h_ring_ = static_cast<char*>(mapped_alloc(cap * request_bytes_));
    // posted, stop and status, a cache line apart
    char* words = static_cast<char*>(mapped_alloc(3 * 64));
    h_posted_ = reinterpret_cast<unsigned long long*>(words);
    h_stop_ = reinterpret_cast<int*>(words + 64);
    h_status_ = reinterpret_cast<int*>(words + 128);
    h_results_ = static_cast<char*>(mapped_alloc(cap * result_bytes_));
    h_done_ = static_cast<long long*>(mapped_alloc(cap * sizeof(long long)));
  }
  // tickets restart at zero: no stale done flag may match one (the kernel is
  // not running, and its launch orders these stores before any of its loads)
  std::memset(h_done_, 0, cap * sizeof(long long));
  std::atomic_ref<unsigned long long>(*h_posted_).store(0);
  std::atomic_ref<int>(*h_stop_).store(0);
  std::atomic_ref<int>(*h_status_).store(0);
  if (!consumed_) consumed_.reset(new std::atomic<long long>[cap]);
  for (size_t i = 0; i < cap; ++i) consumed_[i].store(0);
  next_.store(0);
  check(cudaMemsetAsync(d_words_, 0, device::kRingWords * sizeof(unsigned long long), stream), "memset");
  state_.store(kPrepared);
}

void RequestQueue::launch(cudaStream_t stream, const std::function<cudaError_t(const View&)>& launch_fn) {
  if (state_.load() != kPrepared) fail(NB_ERR_GPU, "the work queue was not prepared");
  View v{};
  v.ring.host_ring = device_view(h_ring_);
  v.ring.posted = device_view(h_posted_);
  v.ring.stop = device_view(h_stop_);
  v.ring.status = device_view(h_status_);
  v.ring.ring = d_ring_;
  v.ring.words = d_words_;
  v.ring.mask = static_cast<long long>(capacity_ - 1);
  v.ring.idle_ns = idle_ns_;
  v.ring.request_bytes = static_cast<int>(request_bytes_);
  v.results = device_view(h_results_);
  v.done = device_view(h_done_);
  check(cudaEventRecord(ev0_, stream), "event");
  check(launch_fn(v), "queue kernel launch");
  check(cudaEventRecord(ev1_, stream), "event");
  state_.store(kLaunched);
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
  std::lock_guard<std::mutex> lock(post_mu_);  // tickets are handed out in order
  const long long first = next_.load();
  const long long mask = static_cast<long long>(capacity_) - 1;
  for (size_t i = 0; i < n; ++i) {
    const long long t = first + static_cast<long long>(i);
    if (slot_free(t)) continue;
    if (!wait) return -1;
    // the slot's previous result has not been read yet: wait for it (bounded)
    const auto t0 = std::chrono::steady_clock::now();
    while (!slot_free(t)) {
      if (!running()) failure("ended with work pending");
      if (ms_since(t0) > kHostWaitMs) failure("made no progress for 60 s");
      std::this_thread::yield();
    }
  }
  next_.store(first + static_cast<long long>(n));
  // the requests, then the released count: the warp that acquires `posted`
  // reads the requests stored before it (the device reads this memory
  // coherently)
  const char* src = static_cast<const char*>(requests);
  for (size_t i = 0; i < n; ++i) {
    const long long t = first + static_cast<long long>(i);
    std::memcpy(h_ring_ + static_cast<size_t>(t & mask) * request_bytes_, src + i * request_bytes_,
                request_bytes_);
  }
  std::atomic_ref<unsigned long long>(*h_posted_)
      .store(static_cast<unsigned long long>(first) + n, std::memory_order_release);
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
  const int s = state_.load();
  if (s == kPrepared) return true;  // launched soon (or now, by another thread)
  if (s != kLaunched) return false;
  const cudaError_t e = cudaEventQuery(ev1_);
  if (e == cudaErrorNotReady) return true;
  check(e, "queue kernel");
  return false;
}

void RequestQueue::request_stop() noexcept {
  if (h_stop_) std::atomic_ref<int>(*h_stop_).store(1, std::memory_order_release);
}

void RequestQueue::stop_impl(bool check_status) {
  const int s = state_.exchange(kIdle);
  if (s == kIdle) return;
  request_stop();
  if (s != kLaunched) return;  // never launched: nothing to wait for
  const cudaError_t e = cudaEventSynchronize(ev1_);
  const int status = std::atomic_ref<int>(*h_status_).load(std::memory_order_acquire);
  if (!check_status) return;
  check(e, "queue kernel");
  float ms = 0.0f;
  check(cudaEventElapsedTime(&ms, ev0_, ev1_), "event time");
  device_ms_ += ms;
  if (status != 0) fail(NB_ERR_GPU, "a queue cluster waited more than " + idle_text(idle_ns_) + " for work");
}

void RequestQueue::stop() { stop_impl(true); }

void RequestQueue::abort() noexcept {
  try {
    stop_impl(false);
  } catch (...) {
  }
}

void RequestQueue::failure(const char* what) {
  const int status = h_status_ ? std::atomic_ref<int>(*h_status_).load(std::memory_order_acquire) : 0;
  std::string taken = "unknown while the kernel runs";
  if (state_.load() == kLaunched && cudaEventQuery(ev1_) == cudaSuccess) {
    unsigned long long n = 0;
    if (cudaMemcpy(&n, d_words_ + device::kTaken, sizeof(n), cudaMemcpyDeviceToHost) == cudaSuccess)
      taken = std::to_string(n);
  }
  fail(NB_ERR_GPU, std::string("the queue kernel ") + what + " (tickets posted " + std::to_string(next_.load()) +
                       ", taken " + taken +
                       (status == 1 ? ", a cluster waited more than " + idle_text(idle_ns_) + " for work)" : ")"));
}

}  // namespace nebula
