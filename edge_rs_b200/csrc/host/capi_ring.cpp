// C-ABI of the request ring's self-check, nb_ring_check_cuda: the ring that
// feeds the persistent kernels (RequestQueue, driver_queue.cpp; the device
// side in ring_device.cuh) driven end to end with an echo kernel
// (ring_check.cu). One host thread posts, another reads and checks every
// result in ticket order, as the drivers' threads do. With no
// requests the kernel is not stopped, so its bounded wait for work runs out:
// the CTAs set the status word and return, and the call reports NB_ERR_GPU
// with no fault and the context intact.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <exception>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/nebula_cuda.h"
#include "common.hpp"
#include "driver_queue.hpp"
#include "export.hpp"

namespace {

using nebula::device::EchoRequest;
using nebula::device::EchoResult;
using Clock = std::chrono::steady_clock;

void write_err(char* err, size_t len, const std::string& msg) {
  if (!err || len == 0) return;
  const size_t n = std::min(len - 1, msg.size());
  std::memcpy(err, msg.data(), n);
  err[n] = 0;
}

double ms_since(Clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

// splitmix64: distinct, well-mixed request words per ticket
unsigned long long mix(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

EchoRequest request_of(unsigned long long i) { return EchoRequest{i, mix(3 * i), mix(3 * i + 1), mix(3 * i + 2)}; }

}  // namespace

NB_API int32_t nb_ring_check_cuda(uint64_t n_requests, uint32_t capacity, uint32_t ctas, uint32_t idle_ms,
                                  uint64_t* mismatches, char* err, size_t err_len) {
  using namespace nebula;
  if (mismatches) *mismatches = 0;
  if (capacity < 2 || (capacity & (capacity - 1)) != 0 || ctas < 1 || ctas > 65535) {
    write_err(err, err_len, "capacity must be a power of two >= 2 and ctas in [1, 65535]");
    return NB_ERR_INVALID_ARGUMENT;
  }
  cudaStream_t stream = nullptr;
  if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) {
    write_err(err, err_len, "cudaStreamCreate failed");
    return NB_ERR_GPU;
  }
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } stream_guard{stream};
  try {
    RequestQueue q(sizeof(EchoRequest), sizeof(EchoResult), capacity);
    if (idle_ms > 0) q.set_idle_ns(static_cast<long long>(idle_ms) * 1000000LL);
    struct QueueGuard {
      RequestQueue& q;
      ~QueueGuard() { q.abort(); }
    } queue_guard{q};
    q.prepare(stream);
    std::atomic<bool> abort{false};
    std::exception_ptr poster_err;
    // the poster starts before the launch, as the drivers' do
    std::thread poster([&] {
      try {
        const uint64_t chunk = std::min<uint64_t>(capacity / 2 > 0 ? capacity / 2 : 1, 256);
        std::vector<EchoRequest> buf;
        for (uint64_t first = 0; first < n_requests && !abort.load(); first += chunk) {
          const uint64_t n = std::min(chunk, n_requests - first);
          buf.resize(n);
          for (uint64_t i = 0; i < n; ++i) buf[i] = request_of(first + i);
          q.post(buf.data(), n);
        }
      } catch (...) {
        poster_err = std::current_exception();
        abort.store(true);
      }
    });
    // the reader too starts before the launch: under a profiler that
    // serialises launches, the launch returns only once the kernel has ended
    std::atomic<uint64_t> bad{0};
    std::exception_ptr reader_err;
    std::thread reader([&] {
      try {
        auto last = Clock::now();
        for (uint64_t t = 0; t < n_requests && !abort.load(); ++t) {
          const long long ticket = static_cast<long long>(t);
          while (!q.done(ticket)) {
            if (abort.load()) return;
            if (!q.running()) q.failure("ended with work pending");
            if (ms_since(last) > 10000.0) q.failure("made no progress for 10 s");
            std::this_thread::yield();
          }
          const EchoResult want = device::echo_of(request_of(t), ticket);
          if (std::memcmp(q.result(ticket), &want, sizeof(want)) != 0) bad.fetch_add(1);
          q.consumed(ticket);
          last = Clock::now();
        }
      } catch (...) {
        reader_err = std::current_exception();
        abort.store(true);
        q.request_stop();
      }
    });
    try {
      q.launch(stream, [&](const RequestQueue::View& v) {
        return static_cast<cudaError_t>(device::launch_ring_echo(v.ring, static_cast<EchoResult*>(v.results),
                                                                 v.done, static_cast<int>(ctas), stream));
      });
      if (n_requests == 0) {
        // nothing is posted and no stop is requested: the kernel ends only
        // when its wait for work runs out (bounded here too)
        const double limit_ms = (idle_ms > 0 ? idle_ms : 5000.0) + 10000.0;
        const auto t0 = Clock::now();
        while (q.running() && ms_since(t0) < limit_ms) std::this_thread::sleep_for(std::chrono::milliseconds(1));
        if (q.running()) {
          q.stop();
          fail(NB_ERR_GPU, "the echo kernel did not end by itself");
        }
      }
    } catch (...) {
      abort.store(true);
      q.request_stop();
      reader.join();
      poster.join();
      throw;
    }
    reader.join();
    poster.join();
    if (reader_err) std::rethrow_exception(reader_err);
    if (poster_err) std::rethrow_exception(poster_err);
    q.stop();  // NB_ERR_GPU if a CTA's wait ran out
    if (mismatches) *mismatches = bad.load();
    return NB_OK;
  } catch (const NbError& e) {
    write_err(err, err_len, e.message);
    return e.code;
  } catch (const std::exception& e) {
    write_err(err, err_len, e.what());
    return NB_ERR_GPU;
  }
}
