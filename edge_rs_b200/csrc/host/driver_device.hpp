// The product driver's resident device state and per-round launch.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <memory>
#include <mutex>
#include <vector>

#include "../cuda/pml_device.cuh"
#include "../cuda/ptmg_device.cuh"
#include "common.hpp"
#include "driver_queue.hpp"

namespace nebula {

// Owns one call's device copy of the design, offsets and kept genes' counts,
// and runs batches of inner fits on them.
//
// Batches go through lanes: each lane has its own stream, request/result
// buffers and work-queue counter, so batches of different lanes run on the
// device concurrently (a lane's kernel fills the SMs another lane's kernel
// leaves idle) while the host prepares the next batch of another lane.
class DeviceFitter {
 public:
  static constexpr int kDefaultLanes = 8;
  static constexpr int kMaxLanes = 64;

  // tables: use the zero-count tables where they apply (zero_tables.hpp)
  DeviceFitter(const Prepared& prep, const std::vector<GeneCounts>& genes, int device, int lanes = 1,
               bool tables = true);
  ~DeviceFitter();
  DeviceFitter(const DeviceFitter&) = delete;
  DeviceFitter& operator=(const DeviceFitter&) = delete;

  // Runs one batch on lane 0 and waits; the returned results (pinned host
  // memory) stay valid until lane 0's next batch.
  const device::FitResult* run(const std::vector<device::FitRequest>& reqs);
  // Queues one batch on `lane` and returns at once; collect() waits for it
  // and returns its results, valid until the lane's next submit().
  void submit(int lane, const std::vector<device::FitRequest>& reqs);
  const device::FitResult* collect(int lane);
  // True once the lane's batch has finished (collect() will not wait).
  bool ready(int lane);

  // Streaming mode: one persistent launch serves requests posted while it
  // runs (device::FitQueue). queue_prepare resets the ring (requests may be
  // posted from then on); queue_launch starts the kernel with `cluster` CTAs
  // per request (under a profiler that serialises launches it returns only
  // when the kernel has ended, so the threads that post and read results
  // run before it and one of them calls queue_request_stop when the work is
  // done); queue_post (safe from several host threads) stores a batch of
  // requests into the mapped ring and returns the first one's ticket;
  // queue_done / queue_result read a ticket's result from host memory the
  // kernel writes; queue_stop tells idle clusters to exit, waits for the
  // kernel and reports a timed-out wait as NB_ERR_GPU.
  static constexpr int kMaxPosters = 8;
  struct Tally {
    uint64_t requests = 0, sweeps = 0, cell_visits = 0, sparse_visits = 0, slot_cycles = 0, h2d = 0, d2h = 0;
    int64_t first_ns = INT64_MAX, last_ns = INT64_MIN;  // earliest fit start, latest fit end
    int64_t wait_ns = 0;  // the clusters' waits for their tickets' requests
  };
  void queue_prepare();
  void queue_launch(int cluster);
  void queue_request_stop() noexcept { fitq_.request_stop(); }
  long long queue_post(const device::FitRequest* reqs, size_t n, int poster, Tally* tally);
  bool queue_done(long long ticket) const;
  const device::FitResult& queue_result(long long ticket) const;
  // The caller has read ticket's result (RequestQueue::consumed).
  void queue_consumed(long long ticket) { fitq_.consumed(ticket); }
  void queue_account(long long ticket, int gene, Tally* tally) const;
  void add_tally(const Tally& t);
  bool queue_running();
  void queue_stop();
  // queue_stop without throwing, for unwinding
  void queue_abort() noexcept;
  // Throws NB_ERR_GPU describing the queue's state.
  [[noreturn]] void queue_failure(const char* what);
  // CTAs per request for a stage with `requests` requests in flight.
  int cluster_for(size_t requests) const;
  // Fits the streaming kernel runs at once with `cluster` CTAs per fit.
  int resident_fits(int cluster) const { return queue_clusters_[cluster]; }
  // Stage one in streaming mode (device::PtmgQueue), the same protocol as
  // the fit queue below; a result is ptmg_stride() doubles.
  void ptmg_queue_prepare(size_t capacity);
  void ptmg_queue_launch();
  void ptmg_request_stop() noexcept;
  // Posts from a thread that reads no results (RequestQueue::post).
  long long ptmg_post(const device::PtmgRequest* reqs, size_t n);
  void ptmg_consumed(long long ticket);
  bool ptmg_done(long long ticket) const;
  const double* ptmg_result(long long ticket) const;
  bool ptmg_running();
  void ptmg_stop();
  void ptmg_abort() noexcept;
  [[noreturn]] void ptmg_failure(const char* what);
  size_t ptmg_stride() const;

  double device_ms() const { return device_ms_; }
  uint64_t launches() const { return launches_; }
  uint64_t requests() const { return requests_; }
  uint64_t sweeps() const { return sweeps_; }
  uint64_t cell_visits() const { return cell_visits_; }
  uint64_t sparse_visits() const { return sparse_visits_; }
  uint64_t slot_cycles() const { return slot_cycles_; }
  // Zero-count groups the sweeps look up (0: every cell is swept).
  size_t tabled_groups() const { return tabled_groups_; }
  // The run has zero-count tables (whether or not the sweeps use them):
  // stage one then descends by L-BFGS-B alone, as the reference does.
  bool design_tabled() const { return design_tabled_; }
  // Device time from the first fit's start to the last fit's end since the
  // last reset_counters, in ms (0 before any fit).
  double ticket_wait_ms() const { return wait_ns_ / 1e6; }
  double busy_span_ms() const { return last_ns_ > first_ns_ ? (last_ns_ - first_ns_) / 1e6 : 0.0; }
  // CTAs the streaming kernel launches with `cluster` CTAs per fit.
  int queue_grid(int cluster) const { return queue_clusters_[cluster] * cluster; }
  int grid() const { return grid_; }
  int lanes() const { return static_cast<int>(lanes_.size()); }
  uint64_t h2d_bytes() const { return h2d_bytes_; }
  uint64_t d2h_bytes() const { return d2h_bytes_; }
  void reset_counters();
  // Brackets a step with events: begin_step orders every lane after it,
  // end_step joins every lane and returns the device time between the two in
  // milliseconds.
  void begin_step();
  double end_step();

 private:
  struct Lane {
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int32_t* h_header = nullptr;  // pinned: request count and queue counter
    int32_t* d_counter = nullptr;  // [0] request count, [1] work-queue counter
    device::FitRequest* d_req = nullptr;
    device::FitResult* d_res = nullptr;
    device::FitRequest* h_req = nullptr;
    device::FitResult* h_res = nullptr;
    size_t capacity = 0;
    size_t pending = 0;  // requests of the batch in flight
  };
  void reserve(Lane& lane, size_t n);
  void ensure_lane(Lane& lane);
  RequestQueue fitq_{sizeof(device::FitRequest), sizeof(device::FitResult), 16384};
  std::unique_ptr<RequestQueue> ptmgq_;
  void ensure_ptmg_scratch();
  int queue_clusters_[device::kMaxCluster + 1] = {};
  cudaStream_t stream_ = nullptr;
  cudaEvent_t step0_ = nullptr, step1_ = nullptr;
  std::vector<Lane> lanes_;
  std::vector<uint64_t> gene_nnz_;
  size_t n_cells_ = 0;
  size_t dense_cells_ = 0;  // cells a sweep's dense part visits
  device::GeneData data_{};
  device::FitControl ctl_{};
  std::vector<void*> pooled_;  // stream-ordered allocations from the device's memory pool
  size_t tabled_groups_ = 0;
  bool design_tabled_ = false;
  int grid_ = 0;
  int max_clusters_[device::kMaxCluster + 1] = {};  // resident clusters per cluster size
  // stage-one buffers
  double* d_scratch_ = nullptr;
  int pgrid_ = 0;
  double device_ms_ = 0.0;
  uint64_t launches_ = 0, requests_ = 0, sweeps_ = 0, cell_visits_ = 0, sparse_visits_ = 0, slot_cycles_ = 0;
  int64_t first_ns_ = INT64_MAX, last_ns_ = INT64_MIN;
  int64_t wait_ns_ = 0;
  uint64_t h2d_bytes_ = 0, d2h_bytes_ = 0;
};

struct Session;

int32_t run_nebula_device(const nb_csr* counts, const uint64_t* subject_id, const double* design,
                          uint32_t n_coef, const double* offset, const nb_params* params,
                          const nb_options* options, nb_fit* out, nb_stats* stats, char* err,
                          size_t err_len);

}  // namespace nebula
