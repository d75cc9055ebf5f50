// nebula_sparse_cuda: the drop-in for nebula_sparse (src/sc/nebula.rs:434-445)
// with every penalised inner fit on the GPU.
//
// Covers the reference's device path (src/gpu/stage_two.rs:281-320 fit_all,
// :362-544 search_all) and the two stages around it. Stage one's cell passes
// and every inner fit of stages two and three run in persistent launches fed
// by device request rings (driver_queue.hpp); host worker threads own
// disjoint sets of genes, step each gene's search (Newton for stage one,
// BOBYQA for stage two) as soon as its points return, and post the gene's
// next points. No gene waits for another. The host only steps the searches
// and assembles the objective from the scalars each device fit returns.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <chrono>
#include <cstring>
#include <exception>
#include <limits>
#include <memory>
#include <mutex>
#include <thread>

#include "../cuda/pml_device.cuh"
#include "common.hpp"
#include "driver_device.hpp"
#include "export.hpp"
#include "search.hpp"
#include "stage_one.hpp"
#include "warm_start.hpp"
#include "zero_tables.hpp"

namespace nebula {
namespace {

using Clock = std::chrono::steady_clock;
double ms_since(Clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) fail(NB_ERR_GPU, std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename F>
void parallel_for(size_t n, int threads, F&& f) {
  int nt = threads > 0 ? threads : static_cast<int>(std::thread::hardware_concurrency());
  nt = std::max(1, std::min<int>(nt, static_cast<int>(n)));
  std::atomic<size_t> next{0};
  std::mutex err_mu;
  std::optional<std::pair<size_t, NbError>> first_err;
  auto worker = [&]() {
    for (;;) {
      size_t i = next.fetch_add(1);
      if (i >= n) return;
      try {
        f(i);
      } catch (const NbError& e) {
        std::lock_guard<std::mutex> lock(err_mu);
        if (!first_err || i < first_err->first) first_err = std::make_pair(i, e);
      }
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
  worker();
  for (auto& th : pool) th.join();
  if (first_err) throw first_err->second;
}

// The per-call arrays come from the device's default memory pool in stream
// order and go back to it in stream order when the call ends. The pool keeps
// what is freed (release threshold raised once per device), so a later call
// takes its arrays from it instead of allocating, and no call waits for a
// synchronous free at its end.
void keep_pool_memory() {
  static std::atomic<bool> done[64];
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= 64 || done[dev].exchange(true)) return;
  cudaMemPool_t pool = nullptr;
  cuda_check(cudaDeviceGetDefaultMemPool(&pool, dev), "default memory pool");
  uint64_t keep = UINT64_MAX;
  cuda_check(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "memory pool threshold");
}

// Pinned host buffers for the upload's staging, kept in a process-wide pool:
// pinned memory is slow to allocate and free, and a copy from it runs
// asynchronously at the link's speed (a pageable source goes through the
// driver's bounce buffers). A call takes one buffer (grown when too small)
// and returns it once its copies have completed. Held until the process exits.
class PinnedStage {
 public:
  explicit PinnedStage(size_t bytes) {
    {
      std::lock_guard<std::mutex> lock(mu());
      if (!pool().empty()) {
        buf_ = pool().back();
        pool().pop_back();
      }
    }
    if (buf_.second < bytes) {
      if (buf_.first) cudaFreeHost(buf_.first);
      buf_ = {nullptr, 0};
      cuda_check(cudaMallocHost(&buf_.first, bytes), "cudaMallocHost");
      buf_.second = bytes;
    }
  }
  ~PinnedStage() {
    std::lock_guard<std::mutex> lock(mu());
    pool().push_back(buf_);
  }
  PinnedStage(const PinnedStage&) = delete;
  PinnedStage& operator=(const PinnedStage&) = delete;
  char* data() const { return static_cast<char*>(buf_.first); }

 private:
  static std::mutex& mu() {
    static std::mutex m;
    return m;
  }
  static std::vector<std::pair<void*, size_t>>& pool() {
    static auto* p = new std::vector<std::pair<void*, size_t>>();
    return *p;
  }
  std::pair<void*, size_t> buf_{nullptr, 0};
};

template <typename T>
T* pool_alloc(size_t n, cudaStream_t stream, std::vector<void*>* pooled) {
  T* d = nullptr;
  cuda_check(cudaMallocAsync(reinterpret_cast<void**>(&d), std::max<size_t>(n, 1) * sizeof(T), stream),
             "cudaMallocAsync");
  pooled->push_back(d);
  return d;
}

template <typename T>
T* device_copy(const T* host, size_t n, cudaStream_t stream, std::vector<void*>* pooled) {
  T* d = pool_alloc<T>(n, stream, pooled);
  if (n) cuda_check(cudaMemcpyAsync(d, host, n * sizeof(T), cudaMemcpyHostToDevice, stream), "H2D copy");
  return d;
}

}  // namespace

// ---------------------------------------------------------------------------
// Resident device copy of one call's inputs, and the per-round launch.

DeviceFitter::DeviceFitter(const Prepared& prep, const std::vector<GeneCounts>& genes, int device, int lanes,
                           bool tables)
    : lanes_(static_cast<size_t>(std::max(1, std::min(lanes, kMaxLanes)))) {
  const Shared& sh = prep.shared;
  if (device >= 0) cuda_check(cudaSetDevice(device), "cudaSetDevice");
  cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  keep_pool_memory();
  const int K = sh.n_subjects;
  const size_t G = genes.size();
  std::vector<uint64_t> gene_ptr(G + 1, 0);
  for (size_t g = 0; g < G; ++g) gene_ptr[g + 1] = gene_ptr[g] + genes[g].cells.size();
  const size_t nnz = gene_ptr[G];
  // the kept genes' entries, concatenated on all host threads straight into
  // pinned staging (every element is written once), and the design and
  // offsets beside them, so that every large copy runs asynchronously
  const size_t nz = std::max<size_t>(nnz, 1);
  const size_t nd = sh.design.size(), no = sh.log_offset.size();
  PinnedStage stage((nz + nd + no) * sizeof(double) + nz * sizeof(uint32_t));
  double* const counts_h = reinterpret_cast<double*>(stage.data());
  // whole counts below 2^24 travel as floats (exact), half the bytes, and
  // are widened to doubles on the device
  bool small_whole = true;
  for (const GeneCounts& gc : genes) small_whole = small_whole && gc.small_whole;
  float* const countsf_h = reinterpret_cast<float*>(counts_h);
  double* const design_h = counts_h + nz;
  double* const offset_h = design_h + nd;
  uint32_t* const cells_h = reinterpret_cast<uint32_t*>(offset_h + no);
  std::vector<double> totals(G * K);
  std::vector<uint64_t> runs(G * (K + 1));
  // the sweep's fixed cell ranges and, per gene, the first positive entry at
  // or after each range boundary (absolute positions)
  constexpr int R = device::kRanges;
  std::vector<uint32_t> rcells(R + 1);
  for (int v = 0; v <= R; ++v) rcells[v] = static_cast<uint32_t>(sh.n_cells * static_cast<size_t>(v) / R);
  std::vector<uint64_t> rpos(G * (R + 1));
  // zero-count tables (the reference's ZeroCells, nebula.rs:641), built once
  // for the call when enough cells share their subject's design rows, on
  // their own thread while the others fill the staging; whether the run is
  // tabled decides stage one's descent (L-BFGS-B), so it is found even when
  // the sweeps are asked to visit every cell
  zero::Tables zt;
  bool tabled = false;
  std::exception_ptr tables_err;
  std::thread tables_thread([&] {
    try {
      tabled = zero::build_tables(sh.design.data(), sh.log_offset.data(), sh.fid.data(), K, sh.n_coef, &zt);
    } catch (...) {
      tables_err = std::current_exception();
    }
  });
  struct JoinAtExit {
    std::thread& t;
    ~JoinAtExit() {
      if (t.joinable()) t.join();
    }
  } join_tables{tables_thread};
  parallel_for(G + 1, 0, [&](size_t g) {
    if (g == G) {
      std::copy(sh.design.begin(), sh.design.end(), design_h);
      std::copy(sh.log_offset.begin(), sh.log_offset.end(), offset_h);
      return;
    }
    const GeneCounts& gc = genes[g];
    std::copy(gc.cells.begin(), gc.cells.end(), cells_h + gene_ptr[g]);
    if (small_whole) {
      float* dst = countsf_h + gene_ptr[g];
      for (size_t i = 0; i < gc.counts.size(); ++i) dst[i] = static_cast<float>(gc.counts[i]);
    } else {
      std::copy(gc.counts.begin(), gc.counts.end(), counts_h + gene_ptr[g]);
    }
    std::copy(prep.totals.begin() + prep.kept[g] * K, prep.totals.begin() + (prep.kept[g] + 1) * K,
              totals.begin() + g * K);
    // positive_runs (pml.rs:1155-1160) as absolute positions
    for (int s = 0; s <= K; ++s) {
      uint64_t b = sh.fid[s];
      auto it = std::lower_bound(gc.cells.begin(), gc.cells.end(), b,
                                 [](uint32_t c, uint64_t v) { return c < v; });
      runs[g * (K + 1) + s] = gene_ptr[g] + static_cast<uint64_t>(it - gc.cells.begin());
    }
    for (int v = 0; v <= R; ++v) {
      auto it = std::lower_bound(gc.cells.begin(), gc.cells.end(), rcells[v]);
      rpos[g * (R + 1) + v] = gene_ptr[g] + static_cast<uint64_t>(it - gc.cells.begin());
    }
  });
  gene_nnz_.resize(G);
  for (size_t g = 0; g < G; ++g) gene_nnz_[g] = genes[g].cells.size();
  n_cells_ = sh.n_cells;
  dense_cells_ = sh.n_cells;
  std::vector<uint32_t> fid(sh.fid.begin(), sh.fid.end());
  data_.n_varying = device::varying_columns(sh.design.data(), sh.n_coef, sh.fid.data(), K, data_.varying);
  // stage one's warp ranges, as many as its CTA has warps
  const int pw = device::ptmg_warps(sh.n_coef, data_.n_varying);
  std::vector<uint32_t> wcells(static_cast<size_t>(pw) + 1);
  for (int w = 0; w <= pw; ++w) wcells[w] = static_cast<uint32_t>(sh.n_cells * static_cast<size_t>(w) / pw);

  // the small pageable arrays first: a copy from pageable memory returns only
  // once the stream's earlier copies are done, so issued after the large
  // pinned ones it would wait for them
  data_.fid = device_copy(fid.data(), fid.size(), stream_, &pooled_);
  data_.gene_ptr = device_copy(gene_ptr.data(), gene_ptr.size(), stream_, &pooled_);
  data_.runs = device_copy(runs.data(), runs.size(), stream_, &pooled_);
  data_.totals = device_copy(totals.data(), totals.size(), stream_, &pooled_);
  data_.warp_cells = device_copy(wcells.data(), wcells.size(), stream_, &pooled_);
  data_.range_cells = device_copy(rcells.data(), rcells.size(), stream_, &pooled_);
  data_.range_pos = device_copy(rpos.data(), rpos.size(), stream_, &pooled_);
  data_.design = device_copy(design_h, nd, stream_, &pooled_);
  data_.log_offset = device_copy(offset_h, no, stream_, &pooled_);
  data_.cells = device_copy(cells_h, nnz, stream_, &pooled_);
  if (small_whole && nnz > 0) {
    const float* countsf_d = device_copy(countsf_h, nnz, stream_, &pooled_);
    double* counts_d = pool_alloc<double>(nnz, stream_, &pooled_);
    cuda_check(static_cast<cudaError_t>(device::widen_counts(countsf_d, counts_d, nnz, stream_)), "widen counts");
    data_.counts = counts_d;
  } else {
    data_.counts = device_copy(counts_h, nnz, stream_, &pooled_);
  }
  h2d_bytes_ = (sh.design.size() + sh.log_offset.size() + (small_whole ? 0 : nnz) + totals.size()) * sizeof(double) +
               (small_whole ? nnz : 0) * sizeof(float) +
               (fid.size() + nnz + wcells.size() + rcells.size()) * sizeof(uint32_t) +
               (gene_ptr.size() + runs.size() + rpos.size()) * sizeof(uint64_t);
  tables_thread.join();
  if (tables_err) std::rethrow_exception(tables_err);
  design_tabled_ = tabled;
  {
    if (tables && design_tabled_) {
      std::vector<uint64_t> lpos(R + 1);
      for (int v = 0; v <= R; ++v)
        lpos[v] = static_cast<uint64_t>(std::lower_bound(zt.loose.begin(), zt.loose.end(), rcells[v]) -
                                        zt.loose.begin());
      data_.tabled = 1;
      data_.zgroups = device_copy(zt.groups.data(), zt.groups.size(), stream_, &pooled_);
      data_.zsubject = device_copy(zt.subject_groups.data(), zt.subject_groups.size(), stream_, &pooled_);
      data_.zindex = device_copy(zt.index.data(), zt.index.size(), stream_, &pooled_);
      data_.zpanels = device_copy(zt.panels.data(), zt.panels.size(), stream_, &pooled_);
      data_.loose = device_copy(zt.loose.data(), zt.loose.size(), stream_, &pooled_);
      data_.subject_loose = device_copy(zt.subject_loose.data(), zt.subject_loose.size(), stream_, &pooled_);
      data_.loose_pos = device_copy(lpos.data(), lpos.size(), stream_, &pooled_);
      tabled_groups_ = zt.groups.size();
      dense_cells_ = zt.loose.size();
      h2d_bytes_ += zt.groups.size() * sizeof(zero::Group) + zt.panels.size() * sizeof(double) +
                    (zt.subject_groups.size() + zt.index.size() + zt.loose.size() + zt.subject_loose.size()) *
                        sizeof(uint32_t) +
                    lpos.size() * sizeof(uint64_t);
    }
  }
  data_.n_cells = static_cast<int32_t>(sh.n_cells);
  data_.n_subjects = K;
  data_.n_coef = sh.n_coef;
  {
    // per gene two (beta, log_w) slots for warm inner starts
    const size_t doubles = std::max<size_t>(G, 1) * 2 * static_cast<size_t>(sh.n_coef + K);
    data_.warm_state = pool_alloc<double>(doubles, stream_, &pooled_);
  }
  ctl_.eps = sh.params.eps;
  ctl_.max_iter = kPmlMaxIter;
  ctl_.max_backtrack = kPmlMaxBacktrack;

  int sms = 0, dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attribute");
  int per_sm = device::fit_blocks_per_sm(K, sh.n_coef, data_.n_varying);
  if (per_sm <= 0)
    fail(NB_ERR_UNSUPPORTED, "the fit kernel cannot be resident with " + std::to_string(K) +
                                 " subjects and " + std::to_string(sh.n_coef) + " columns");
  grid_ = per_sm * sms;
  for (int c = 2; c <= device::kMaxCluster; c *= 2)
    max_clusters_[c] = device::fit_max_clusters(K, sh.n_coef, data_.n_varying, c);
  for (int c = 1; c <= device::kMaxCluster; c *= 2)
    queue_clusters_[c] = device::fit_queue_max_clusters(K, sh.n_coef, data_.n_varying, c);
  cuda_check(cudaEventCreate(&step0_), "event");
  cuda_check(cudaEventCreate(&step1_), "event");
  // the pinned staging goes back to its pool when this returns
  cuda_check(cudaStreamSynchronize(stream_), "upload");
}

void DeviceFitter::reset_counters() {
  device_ms_ = 0.0;
  launches_ = requests_ = sweeps_ = cell_visits_ = sparse_visits_ = slot_cycles_ = h2d_bytes_ = d2h_bytes_ = 0;
  first_ns_ = INT64_MAX;
  last_ns_ = INT64_MIN;
  wait_ns_ = 0;
}

void DeviceFitter::begin_step() {
  cuda_check(cudaEventRecord(step0_, stream_), "event");
  for (Lane& lane : lanes_)
    if (lane.stream) cuda_check(cudaStreamWaitEvent(lane.stream, step0_, 0), "stream wait");
}

// A batch lane's stream, events and counters, made on its first use (only
// the kernel-level entry runs batches); the lane's work follows stream_'s.
void DeviceFitter::ensure_lane(Lane& lane) {
  if (lane.stream) return;
  cuda_check(cudaStreamCreateWithFlags(&lane.stream, cudaStreamNonBlocking), "cudaStreamCreate");
  cuda_check(cudaEventCreate(&lane.ev0), "event");
  cuda_check(cudaEventCreate(&lane.ev1), "event");
  lane.d_counter = pool_alloc<int32_t>(2, stream_, &pooled_);
  cuda_check(cudaMallocHost(reinterpret_cast<void**>(&lane.h_header), 2 * sizeof(int32_t)), "cudaMallocHost");
  cuda_check(cudaEventRecord(lane.ev0, stream_), "event");
  cuda_check(cudaStreamWaitEvent(lane.stream, lane.ev0, 0), "stream wait");
}

double DeviceFitter::end_step() {
  for (Lane& lane : lanes_) {
    if (!lane.stream) continue;
    cuda_check(cudaEventRecord(lane.ev1, lane.stream), "event");
    cuda_check(cudaStreamWaitEvent(stream_, lane.ev1, 0), "stream wait");
  }
  cuda_check(cudaEventRecord(step1_, stream_), "event");
  cuda_check(cudaEventSynchronize(step1_), "event");
  float ms = 0.0f;
  cuda_check(cudaEventElapsedTime(&ms, step0_, step1_), "event time");
  return ms;
}

void DeviceFitter::ensure_ptmg_scratch() {
  if (d_scratch_) return;
  const int K = data_.n_subjects;
  pgrid_ = device::ptmg_resident_ctas(K, data_.n_coef, data_.n_varying);
  if (pgrid_ <= 0)
    fail(NB_ERR_UNSUPPORTED, "the stage-one kernel cannot be resident with " + std::to_string(K) + " subjects");
  d_scratch_ = pool_alloc<double>(
      static_cast<size_t>(pgrid_) * device::ptmg_scratch_doubles(K, data_.n_coef, data_.n_varying), stream_,
      &pooled_);
}

size_t DeviceFitter::ptmg_stride() const {
  return static_cast<size_t>(2 + device::ptmg_width_of(data_.n_coef)) * static_cast<size_t>(data_.n_subjects);
}

void DeviceFitter::ptmg_queue_prepare(size_t capacity) {
  ensure_ptmg_scratch();
  if (!ptmgq_ || ptmgq_->capacity() != capacity)
    ptmgq_ = std::make_unique<RequestQueue>(sizeof(device::PtmgRequest), ptmg_stride() * sizeof(double), capacity);
  ptmgq_->prepare(stream_);
}

void DeviceFitter::ptmg_queue_launch() {
  ptmgq_->launch(stream_, [&](const RequestQueue::View& v) {
    device::PtmgQueue pq{};
    pq.ring = v.ring;
    pq.results = static_cast<double*>(v.results);
    pq.result_stride = static_cast<long long>(ptmg_stride());
    pq.done = v.done;
    return static_cast<cudaError_t>(device::launch_ptmg_queue(data_, pq, d_scratch_, pgrid_, stream_));
  });
  ++launches_;
}

void DeviceFitter::ptmg_request_stop() noexcept {
  if (ptmgq_) ptmgq_->request_stop();
}

long long DeviceFitter::ptmg_post(const device::PtmgRequest* reqs, size_t n) { return ptmgq_->post(reqs, n); }
void DeviceFitter::ptmg_consumed(long long ticket) { ptmgq_->consumed(ticket); }
bool DeviceFitter::ptmg_done(long long ticket) const { return ptmgq_->done(ticket); }
const double* DeviceFitter::ptmg_result(long long ticket) const {
  return static_cast<const double*>(ptmgq_->result(ticket));
}
bool DeviceFitter::ptmg_running() { return ptmgq_->running(); }
void DeviceFitter::ptmg_stop() { ptmgq_->stop(); }
void DeviceFitter::ptmg_abort() noexcept {
  if (ptmgq_) ptmgq_->abort();
}
void DeviceFitter::ptmg_failure(const char* what) { ptmgq_->failure(what); }


DeviceFitter::~DeviceFitter() {
  fitq_.abort();
  ptmg_abort();
  for (Lane& lane : lanes_) {
    if (lane.stream) cudaStreamSynchronize(lane.stream);
    if (lane.d_req) cudaFree(lane.d_req);
    if (lane.d_res) cudaFree(lane.d_res);
    if (lane.h_req) cudaFreeHost(lane.h_req);
    if (lane.h_res) cudaFreeHost(lane.h_res);
    if (lane.h_header) cudaFreeHost(lane.h_header);
    if (lane.ev0) cudaEventDestroy(lane.ev0);
    if (lane.ev1) cudaEventDestroy(lane.ev1);
    if (lane.stream) cudaStreamDestroy(lane.stream);
  }
  for (void* p : pooled_) cudaFreeAsync(p, stream_);  // back to the device's pool
  if (step0_) cudaEventDestroy(step0_);
  if (step1_) cudaEventDestroy(step1_);
  if (stream_) cudaStreamDestroy(stream_);
}

void DeviceFitter::reserve(Lane& lane, size_t n) {
  if (n <= lane.capacity) return;
  size_t cap = std::max<size_t>(n, lane.capacity * 2);
  if (lane.d_req) cudaFree(lane.d_req);
  if (lane.d_res) cudaFree(lane.d_res);
  if (lane.h_req) cudaFreeHost(lane.h_req);
  if (lane.h_res) cudaFreeHost(lane.h_res);
  cuda_check(cudaMalloc(reinterpret_cast<void**>(&lane.d_req), cap * sizeof(device::FitRequest)), "cudaMalloc");
  cuda_check(cudaMalloc(reinterpret_cast<void**>(&lane.d_res), cap * sizeof(device::FitResult)), "cudaMalloc");
  cuda_check(cudaMallocHost(reinterpret_cast<void**>(&lane.h_req), cap * sizeof(device::FitRequest)),
             "cudaMallocHost");
  cuda_check(cudaMallocHost(reinterpret_cast<void**>(&lane.h_res), cap * sizeof(device::FitResult)),
             "cudaMallocHost");
  lane.capacity = cap;
}

void DeviceFitter::submit(int lane_index, const std::vector<device::FitRequest>& reqs) {
  Lane& lane = lanes_[lane_index];
  ensure_lane(lane);
  const size_t n = reqs.size();
  lane.pending = n;
  if (n == 0) return;
  reserve(lane, n);
  std::memcpy(lane.h_req, reqs.data(), n * sizeof(device::FitRequest));
  lane.h_header[0] = static_cast<int32_t>(n);
  lane.h_header[1] = 0;
  cuda_check(cudaMemcpyAsync(lane.d_req, lane.h_req, n * sizeof(device::FitRequest), cudaMemcpyHostToDevice,
                             lane.stream),
             "request copy");
  cuda_check(cudaMemcpyAsync(lane.d_counter, lane.h_header, 2 * sizeof(int32_t), cudaMemcpyHostToDevice,
                             lane.stream),
             "count copy");
  cuda_check(cudaEventRecord(lane.ev0, lane.stream), "event");
  // Spread each request over a cluster of CTAs when the requests in flight
  // leave SM slots idle: the largest power of two (up to kMaxCluster) with
  // requests x cluster within the resident CTA slots.
  size_t in_flight = n;
  for (const Lane& other : lanes_)
    if (&other != &lane) in_flight += other.pending;
  int cluster = 1;
  while (cluster < device::kMaxCluster && in_flight * static_cast<size_t>(cluster) * 2 <= static_cast<size_t>(grid_) &&
         max_clusters_[cluster * 2] > 0)
    cluster *= 2;
  int grid = static_cast<int>(std::min<size_t>(grid_, n));
  if (cluster > 1) grid = static_cast<int>(std::min<size_t>(max_clusters_[cluster], n)) * cluster;
  cuda_check(static_cast<cudaError_t>(device::launch_fit(data_, ctl_, lane.d_req, lane.d_res, lane.d_counter,
                                                          lane.d_counter + 1, grid, cluster, lane.stream)),
             "fit kernel launch");
  cuda_check(cudaEventRecord(lane.ev1, lane.stream), "event");
  cuda_check(cudaMemcpyAsync(lane.h_res, lane.d_res, n * sizeof(device::FitResult), cudaMemcpyDeviceToHost,
                             lane.stream),
             "result copy");
  ++launches_;
  requests_ += n;
  h2d_bytes_ += n * sizeof(device::FitRequest) + 2 * sizeof(int32_t);
  d2h_bytes_ += n * sizeof(device::FitResult);
}

const device::FitResult* DeviceFitter::collect(int lane_index) {
  Lane& lane = lanes_[lane_index];
  const size_t n = lane.pending;
  if (n == 0) return nullptr;
  cuda_check(cudaStreamSynchronize(lane.stream), "fit kernel");
  float ms = 0.0f;
  cuda_check(cudaEventElapsedTime(&ms, lane.ev0, lane.ev1), "event time");
  device_ms_ += ms;
  for (size_t i = 0; i < n; ++i) {
    const uint64_t sw = static_cast<uint64_t>(lane.h_res[i].sweeps);
    sweeps_ += sw;
    cell_visits_ += sw * (dense_cells_ + gene_nnz_[lane.h_req[i].gene]);
    sparse_visits_ += sw * gene_nnz_[lane.h_req[i].gene];
    slot_cycles_ += static_cast<uint64_t>(lane.h_res[i].cycles);
  }
  lane.pending = 0;
  return lane.h_res;
}

// ---------------------------------------------------------------------------
// Streaming mode.

int DeviceFitter::cluster_for(size_t requests) const {
  // Spread each fit over more CTAs while each CTA keeps at least 25,000 cells
  // per sweep, so a sweep's fixed costs (the cluster barrier, the combine, the
  // Newton step every CTA repeats) stay small; beyond two CTAs only while the
  // requests times the cluster stay within eight times the resident CTA
  // slots, where the searches that finish last would otherwise run on a few
  // SMs. The count is the design's cells even under zero-count tables, whose
  // sweeps visit far fewer: their steps are bound by the chains of
  // evaluations, and a fit spread wider ends sooner (500 genes x 100,000
  // cells, categorical: 77 ms a step at 4 CTAs per fit, 92 at 2, 119 at 1).
  // The sessions' tuning picked 4, 2, 2 and 2 CTAs for 500 x 100,000 (p = 4),
  // 4,000 x 50,000 (p = 8), 2,000 x 200,000 (p = 8) and 20,000 x 100,000
  // (p = 4), which this rule gives.
  int cluster = 1;
  while (cluster < device::kMaxCluster && queue_clusters_[cluster * 2] > 0 &&
         n_cells_ >= static_cast<size_t>(cluster) * 2 * 25000 &&
         (cluster < 2 || requests * static_cast<size_t>(cluster) * 2 <= 8 * static_cast<size_t>(grid_)))
    cluster *= 2;
  return cluster;
}

void DeviceFitter::queue_prepare() { fitq_.prepare(stream_); }

void DeviceFitter::queue_launch(int cluster) {
  if (cluster < 1 || cluster > device::kMaxCluster || queue_clusters_[cluster] <= 0)
    fail(NB_ERR_GPU, "no resident cluster of " + std::to_string(cluster) + " fit CTAs");
  const int grid = queue_clusters_[cluster] * cluster;
  fitq_.launch(stream_, [&](const RequestQueue::View& v) {
    device::FitQueue fq{};
    fq.ring = v.ring;
    fq.results = static_cast<device::FitResult*>(v.results);
    fq.done = v.done;
    return static_cast<cudaError_t>(device::launch_fit_queue(data_, ctl_, fq, grid, cluster, stream_));
  });
  ++launches_;
}

long long DeviceFitter::queue_post(const device::FitRequest* reqs, size_t n, int poster, Tally* tally) {
  (void)poster;
  const long long first = fitq_.post(reqs, n);
  tally->h2d += n * (sizeof(device::FitRequest) + sizeof(long long));
  return first;
}

bool DeviceFitter::queue_done(long long ticket) const { return fitq_.done(ticket); }

const device::FitResult& DeviceFitter::queue_result(long long ticket) const {
  return *static_cast<const device::FitResult*>(fitq_.result(ticket));
}

void DeviceFitter::queue_account(long long ticket, int gene, Tally* tally) const {
  const device::FitResult& r = queue_result(ticket);
  ++tally->requests;
  tally->d2h += sizeof(device::FitResult) + sizeof(long long);
  if (r.status != 0) return;
  const uint64_t sw = static_cast<uint64_t>(r.sweeps);
  tally->sweeps += sw;
  tally->cell_visits += sw * (dense_cells_ + gene_nnz_[static_cast<size_t>(gene)]);
  tally->sparse_visits += sw * gene_nnz_[static_cast<size_t>(gene)];
  tally->slot_cycles += static_cast<uint64_t>(r.cycles);
  tally->first_ns = std::min<int64_t>(tally->first_ns, r.start_ns);
  tally->wait_ns += r.wait_ns;
  tally->last_ns = std::max<int64_t>(tally->last_ns, r.end_ns);
}

void DeviceFitter::add_tally(const Tally& t) {
  requests_ += t.requests;
  sweeps_ += t.sweeps;
  cell_visits_ += t.cell_visits;
  sparse_visits_ += t.sparse_visits;
  slot_cycles_ += t.slot_cycles;
  h2d_bytes_ += t.h2d;
  d2h_bytes_ += t.d2h;
  first_ns_ = std::min(first_ns_, t.first_ns);
  wait_ns_ += t.wait_ns;
  last_ns_ = std::max(last_ns_, t.last_ns);
}

bool DeviceFitter::queue_running() { return fitq_.running(); }

void DeviceFitter::queue_stop() {
  const double before = fitq_.device_ms();
  fitq_.stop();
  device_ms_ += fitq_.device_ms() - before;
}

void DeviceFitter::queue_abort() noexcept { fitq_.abort(); }

void DeviceFitter::queue_failure(const char* what) { fitq_.failure(what); }

bool DeviceFitter::ready(int lane_index) {
  const cudaError_t e = cudaStreamQuery(lanes_[lane_index].stream);
  if (e == cudaErrorNotReady) return false;
  cuda_check(e, "fit kernel");
  return true;
}

const device::FitResult* DeviceFitter::run(const std::vector<device::FitRequest>& reqs) {
  submit(0, reqs);
  return collect(0);
}

// ---------------------------------------------------------------------------

namespace {

// Admission order of stage two's requests: a warm search takes about this
// share of the plain search's evaluations (c1, initial radius 0.03), and a
// cold fit about this many warm fits' sweeps.
constexpr double kWarmEvaluationShare = 0.62;
constexpr double kColdFitCost = 1.5;

// Default initial trust radius of a warm search, as a fraction of NLopt's.
// On 500 genes x 100,000 cells (stage one's start within about 1%) it cuts
// the search's evaluations by 38% against the full radius; on genes drawn
// with sigma^2 and phi LogNormal sd 1.0 (starts off by about 10%) by 32%,
// with the warm search ending worse than the cold one on 1 of 200 genes
// (2 of 200 at the full radius). Smaller radii gain nothing more there.
constexpr double kWarmRadius = 0.03;

struct GeneTask {
  std::unique_ptr<StageTwoSearch> search;
  VarianceObjective objective;
  std::optional<std::optional<std::pair<std::vector<double>, bool>>> refit;
};

void write_err(char* err, size_t len, const std::string& msg) {
  if (!err || len == 0) return;
  size_t n = std::min(len - 1, msg.size());
  std::memcpy(err, msg.data(), n);
  err[n] = 0;
}

}  // namespace

// One call's validated inputs, stage-one plans and resident device copy.
struct Session {
  Prepared prep;
  std::vector<GeneCounts> genes;
  std::vector<GenePlan> plans;
  std::unique_ptr<DeviceFitter> fitter;
  nb_options opt{};
  double ms_prepare = 0.0, ms_stage_one = 0.0, ms_upload = 0.0;
  // autotuning of the CTAs per fit: the first calls of a session try the
  // candidates in turn (the results do not depend on the choice) and later
  // calls take the fastest
  std::vector<int> tune_candidates;
  std::vector<double> tune_ms;
  int tuned = 0;
  // the warm-start network's outputs per kept gene (mlp::kOut each), computed
  // on the session's first fit; empty until then
  std::vector<float> net_y;
};

int choose_cluster(Session& ss, size_t G) {
  const int forced = ss.opt.cluster;
  if (forced == 1 || forced == 2 || forced == 4 || forced == 8) return forced;
  if (ss.tuned > 0) return ss.tuned;
  if (ss.tune_candidates.empty()) {
    const int guess = ss.fitter->cluster_for(G);
    for (int c : {guess, guess * 2, guess / 2})
      if (c >= 1 && c <= device::kMaxCluster &&
          std::find(ss.tune_candidates.begin(), ss.tune_candidates.end(), c) == ss.tune_candidates.end())
        ss.tune_candidates.push_back(c);
  }
  return ss.tune_candidates[ss.tune_ms.size()];
}

// `ms`: the call's persistent launch alone (its device time), so a first
// call's one-off host work (the network's outputs, the ring's pinned
// buffers) does not count against the first candidate. A neighbour replaces
// the guess only when it is at least 2% faster: one call per candidate is a
// noisy sample, and the guess is right on the configurations measured.
void record_cluster(Session& ss, int cluster, double ms) {
  if (ss.tuned > 0 || ss.tune_candidates.empty() || ss.opt.cluster != 0) return;
  if (ss.tune_candidates[ss.tune_ms.size()] != cluster) return;
  ss.tune_ms.push_back(ms);
  if (ss.tune_ms.size() == ss.tune_candidates.size()) {
    size_t best = 0;
    for (size_t i = 1; i < ss.tune_ms.size(); ++i)
      if (ss.tune_ms[i] < ss.tune_ms[best] && ss.tune_ms[i] < 0.98 * ss.tune_ms[0]) best = i;
    ss.tuned = ss.tune_candidates[best];
  }
}

// borrow_counts: the genes view the caller's CSR rows instead of copying
// them (a one-shot call, whose caller keeps its arrays for the call); a
// session kept across calls holds its own copy.
std::unique_ptr<Session> create_session(const nb_csr* counts, const uint64_t* subject_id, const double* design,
                                        uint32_t n_coef, const double* offset, const nb_params* params,
                                        const nb_options* options, bool borrow_counts) {
  auto t0 = Clock::now();
  auto ss = std::make_unique<Session>();
  ss->opt.device = -1;
  ss->opt.audit_percent = 5;
  if (options) ss->opt = *options;
  if (n_coef > static_cast<uint32_t>(device::kMaxCoef))
    fail(NB_ERR_UNSUPPORTED, "the device path takes at most 8 design columns");
  ss->prep = prepare(counts, subject_id, design, n_coef, offset, params);
  const Shared& sh = ss->prep.shared;
  const size_t G = ss->prep.kept.size();
  ss->genes.resize(G);
  parallel_for(G, ss->opt.host_threads,
               [&](size_t g) { ss->genes[g] = positive_indices(ss->prep.counts, ss->prep.kept[g], borrow_counts); });
  ss->ms_prepare = ms_since(t0);
  auto t2 = Clock::now();
  ss->fitter = std::make_unique<DeviceFitter>(ss->prep, ss->genes, ss->opt.device, 1, ss->opt.dense_sweep == 0);
  ss->ms_upload = ms_since(t2);
  // stage one (nebula.rs:812-901): every gene's projected Newton at its own
  // pace through one persistent launch of marginal-likelihood cell passes;
  // host worker threads own the genes, assemble value, gradient and Hessian
  // from a finished pass and post the gene's next point
  auto t1 = Clock::now();
  const int nb = sh.n_coef, K = sh.n_subjects, np = nb + 2;
  const size_t stride = ss->fitter->ptmg_stride();
  std::vector<std::unique_ptr<MarginalSearch>> search(G);
  std::vector<std::vector<double>> xy(G);
  std::vector<long long> ticket(G, -1);
  ss->plans.resize(G);
  size_t capacity = 256;
  while (capacity < 2 * G && capacity < 4096) capacity *= 2;
  const int hw = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
  const int workers = std::max(1, std::min<int>({ss->opt.host_threads > 0 ? ss->opt.host_threads : 2 * hw, 32,
                                                 static_cast<int>(std::max<size_t>(G, 1))}));
  std::atomic<bool> abort{false};
  std::mutex err_mu;
  std::optional<NbError> first_err;
  auto request_of = [&](size_t g) {
    const double* x = search[g]->ask();
    Terms t(x[nb], x[nb + 1]);
    device::PtmgRequest r{};
    r.gene = static_cast<int32_t>(g);
    r.alpha = t.alpha;
    r.lambda = t.lambda;
    r.gamma = t.gamma;
    for (int j = 0; j < nb; ++j) r.beta[j] = x[j];
    return r;
  };
  // Workers queue their genes' next requests here; one poster thread posts
  // each drain as one batch (the workers never wait on the copies, and the
  // batches grow while a post is under way), as in stages two and three.
  std::mutex queue_mu;
  std::vector<device::PtmgRequest> queued;
  std::vector<size_t> queued_genes;
  std::atomic<int> workers_left{workers};
  auto poster = [&]() {
    struct StopAtEnd {  // every ticket has been read, or the stage failed
      DeviceFitter& f;
      ~StopAtEnd() { f.ptmg_request_stop(); }
    } stop_at_end{*ss->fitter};
    std::vector<device::PtmgRequest> batch;
    std::vector<size_t> genes;
    try {
      while (!abort.load(std::memory_order_relaxed)) {
        bool idle = false;
        {
          std::lock_guard<std::mutex> lock(queue_mu);
          batch.swap(queued);
          genes.swap(queued_genes);
          idle = batch.empty() && workers_left.load() == 0;
        }
        if (idle) return;
        if (batch.empty()) {
          std::this_thread::yield();
          continue;
        }
        // chunks of at most a quarter of the ring; the owning workers read the
        // tickets with acquire loads
        for (size_t at = 0; at < batch.size();) {
          const size_t n = std::min(batch.size() - at, capacity / 4);
          const long long first = ss->fitter->ptmg_post(batch.data() + at, n);
          for (size_t k = 0; k < n; ++k)
            std::atomic_ref<long long>(ticket[genes[at + k]]).store(first + static_cast<long long>(k),
                                                                    std::memory_order_release);
          at += n;
        }
        batch.clear();
        genes.clear();
      }
    } catch (const NbError& e) {
      std::lock_guard<std::mutex> lock(err_mu);
      if (!first_err) first_err = e;
      abort.store(true);
    } catch (const std::exception& e) {
      std::lock_guard<std::mutex> lock(err_mu);
      if (!first_err) first_err = NbError{NB_ERR_GPU, e.what()};
      abort.store(true);
    }
  };
  auto worker = [&](int w) {
    struct Leave {
      std::atomic<int>& left;
      ~Leave() { left.fetch_sub(1); }
    } leave{workers_left};
    try {
      std::vector<size_t> waiting, owners;
      std::vector<device::PtmgRequest> box;
      auto post = [&]() {
        if (box.empty()) return;
        std::lock_guard<std::mutex> lock(queue_mu);
        queued.insert(queued.end(), box.begin(), box.end());
        queued_genes.insert(queued_genes.end(), owners.begin(), owners.end());
        box.clear();
        owners.clear();
      };
      for (size_t g = static_cast<size_t>(w); g < G; g += static_cast<size_t>(workers)) {
        std::vector<double> start, lower, upper;
        marginal_box(sh, ss->genes[g], &start, &lower, &upper);
        search[g] = std::make_unique<MarginalSearch>(start, lower, upper, nb, ss->fitter->design_tabled());
        xy[g] = positive_xy(sh, ss->genes[g]);
        box.push_back(request_of(g));
        owners.push_back(g);
        waiting.push_back(g);
        post();
      }
      std::vector<double> grad(np), hess(static_cast<size_t>(np) * np), x(np);
      auto last_progress = Clock::now();
      while (!waiting.empty() && !abort.load(std::memory_order_relaxed)) {
        bool progressed = false;
        for (size_t i = 0; i < waiting.size();) {
          const size_t g = waiting[i];
          if (!ss->fitter->ptmg_done(std::atomic_ref<long long>(ticket[g]).load(std::memory_order_acquire))) {
            ++i;
            continue;
          }
          progressed = true;
          const double* r = ss->fitter->ptmg_result(ticket[g]);
          PtmgSums sums;
          sums.cumsumxtb.assign(r, r + K);
          sums.ylin.assign(r + K, r + 2 * K);
          sums.sums.assign(r + 2 * K, r + stride);
          ss->fitter->ptmg_consumed(ticket[g]);
          ticket[g] = -1;
          MarginalGene mg{&sh, &ss->genes[g], &ss->prep.totals[ss->prep.kept[g] * K], xy[g].data()};
          x.assign(search[g]->ask(), search[g]->ask() + np);
          const double f = ptmg_assemble(mg, x.data(), sums, grad.data(), hess.data());
          search[g]->tell(f, grad.data(), hess.data());
          if (search[g]->done()) {
            ss->plans[g] = plan_from(sh, ss->genes[g], search[g]->best(), search[g]->failed());
            waiting[i] = waiting.back();
            waiting.pop_back();
            continue;
          }
          box.push_back(request_of(g));
          owners.push_back(g);
          ++i;
        }
        post();
        if (progressed) {
          last_progress = Clock::now();
        } else {
          if (!ss->fitter->ptmg_running()) ss->fitter->ptmg_failure("ended with work pending");
          if (ms_since(last_progress) > 60000.0) ss->fitter->ptmg_failure("made no progress for 60 s");
          std::this_thread::yield();
        }
      }
    } catch (const NbError& e) {
      std::lock_guard<std::mutex> lock(err_mu);
      if (!first_err) first_err = e;
      abort.store(true);
    } catch (const std::exception& e) {
      std::lock_guard<std::mutex> lock(err_mu);
      if (!first_err) first_err = NbError{NB_ERR_GPU, e.what()};
      abort.store(true);
    }
  };
  {
    struct QueueGuard {
      DeviceFitter& f;
      ~QueueGuard() { f.ptmg_abort(); }
    } guard{*ss->fitter};
    // The ring is ready before the kernel starts and every thread that posts
    // or reads results runs before the launch: a profiler that serialises
    // launches returns from it only once the kernel has ended, which the
    // poster's stop request at the end of the work allows.
    ss->fitter->ptmg_queue_prepare(capacity);
    std::thread post_thread(poster);
    std::vector<std::thread> pool;
    for (int w = 0; w < workers; ++w) pool.emplace_back(worker, w);
    try {
      ss->fitter->ptmg_queue_launch();
    } catch (...) {
      abort.store(true);
      for (auto& th : pool) th.join();
      post_thread.join();
      throw;
    }
    for (auto& th : pool) th.join();
    post_thread.join();
    if (first_err) throw *first_err;
    ss->fitter->ptmg_stop();
  }
  ss->ms_stage_one = ms_since(t1);
  return ss;
}

// Starts of the warm-started searches: the caller's points (warm_start 2) or
// the network's prediction from the genes' features (warm_start 1); a
// non-finite or non-positive start falls back to stage one's.
// The warm-start network's outputs for every kept gene (cached in the
// session): log-corrections of stage one's (sigma, gamma) and the log of the
// plain search's evaluation count.
const std::vector<float>& network_outputs(Session& ss) {
  const Shared& sh = ss.prep.shared;
  const size_t G = ss.genes.size();
  const int K = sh.n_subjects;
  if (ss.net_y.size() == G * mlp::kOut) return ss.net_y;
  std::vector<float> features(G * mlp::kIn), y(G * mlp::kOut);
  parallel_for(G, ss.opt.host_threads, [&](size_t g) {
    warm_features(sh, ss.genes[g], &ss.prep.totals[ss.prep.kept[g] * K], ss.plans[g], &features[g * mlp::kIn]);
  });
  const float* params = ss.opt.mlp_weights ? ss.opt.mlp_weights : builtin_mlp_params();
  char err[256] = {};
  if (G > 0) {
    const int32_t rc = nb_mlp_predict_cuda(params, features.data(), G, y.data(), err, sizeof(err));
    if (rc != NB_OK) fail(rc, std::string("warm-start network: ") + err);
  }
  ss.net_y = std::move(y);
  return ss.net_y;
}

void warm_starts(Session& ss, std::vector<std::array<double, 2>>* point) {
  const size_t G = ss.genes.size();
  for (size_t g = 0; g < G; ++g) (*point)[g] = {ss.plans[g].sigma, ss.plans[g].gamma};
  auto accept = [&](size_t g, double sigma, double gamma) {
    if (std::isfinite(sigma) && sigma > 0.0) (*point)[g][0] = sigma;
    if (std::isfinite(gamma) && gamma > 0.0) (*point)[g][1] = gamma;
  };
  if (ss.opt.warm_start == 3) return;  // stage one's starts, warm inner fits only
  if (ss.opt.warm_start == 2) {
    if (!ss.opt.warm_points) fail(NB_ERR_INVALID_ARGUMENT, "warm_start 2 needs warm_points");
    for (size_t g = 0; g < G; ++g) {
      const size_t in = ss.prep.kept[g];
      accept(g, ss.opt.warm_points[2 * in], ss.opt.warm_points[2 * in + 1]);
    }
    return;
  }
  const std::vector<float>& y = network_outputs(ss);
  // Corrections smaller than about twice the network's held-out error
  // (log-ratio 0.07) are dropped: stage one's start is then as good.
  constexpr double kGate = 0.07;
  auto gate = [&](double d) { return std::fabs(d) > kGate ? std::clamp(d, -10.0, 10.0) : 0.0; };
  for (size_t g = 0; g < G; ++g) {
    const double d0 = gate(static_cast<double>(y[g * mlp::kOut + 0]));
    const double d1 = gate(static_cast<double>(y[g * mlp::kOut + 1]));
    accept(g, ss.plans[g].sigma * std::exp(d0), ss.plans[g].gamma * std::exp(d1));
  }
}

// Stages two and three on the resident data, into `out`.
void fit_session(Session& ss, nb_fit* out, nb_stats* stats) {
  const Shared& sh = ss.prep.shared;
  const size_t G = ss.genes.size();
  DeviceFitter& fitter = *ss.fitter;
  // the network's outputs (computed on a session's first fit) before the
  // step's clock starts: the cluster tuning compares the first calls' steps
  network_outputs(ss);
  fitter.reset_counters();
  fitter.begin_step();
  // Stages two and three through one persistent launch: every gene's search
  // runs at its own pace. When all of a gene's pending points have come
  // back, the host steps its search and posts the next points, or, once the
  // search is done, the gene's final fit (nebula.rs:948-967). No gene waits
  // for another, and a gene's sequence of evaluations is that of the
  // reference's search. The genes are dealt to host worker threads, each of
  // which builds its genes' searches and steps them.
  auto t2 = Clock::now();
  // Warm start (nb_options.warm_start): each search starts from a predicted
  // or given point; an audit sample of the genes also runs cold (a twin task
  // G + a for gene audit_of[a]) and keeps the cold result where the warm
  // search's best objective is worse.
  const int warm = (ss.opt.warm_start >= 1 && ss.opt.warm_start <= 3) ? ss.opt.warm_start : 0;
  std::vector<std::array<double, 2>> warm_point(G);
  if (warm) warm_starts(ss, &warm_point);
  // the plain search's predicted evaluation count per gene (the network's
  // third output), for the order in which requests are admitted
  std::vector<double> budget(G);
  {
    const std::vector<float>& y = network_outputs(ss);
    for (size_t g = 0; g < G; ++g) budget[g] = std::exp(std::clamp(static_cast<double>(y[g * mlp::kOut + 2]), 0.0, 8.0));
  }
  // The warm search's initial trust radius, a fraction of NLopt's.
  const double radius = ss.opt.warm_radius > 0.0 ? std::min(ss.opt.warm_radius, 1.0) : kWarmRadius;
  std::vector<size_t> audit_of;
  std::vector<long long> twin(G, -1);
  if (warm) {
    const uint32_t share = static_cast<uint32_t>(std::clamp(ss.opt.audit_percent, 0, 100));
    for (size_t g = 0; g < G; ++g) {
      const uint32_t h = static_cast<uint32_t>((static_cast<uint64_t>(g) * 2654435761ULL) >> 7) % 100u;
      if (ss.plans[g].refit != Refit::None && h < share) {
        twin[g] = static_cast<long long>(G + audit_of.size());
        audit_of.push_back(g);
      }
    }
  }
  const size_t T = G + audit_of.size();
  auto gene_of = [&](size_t v) { return v < G ? v : audit_of[v - G]; };
  std::vector<GeneTask> tasks(T);
  std::vector<int> evaluations(G, 0);
  std::vector<char> warm_done(G, 0), cold_done(G, 0), parked(T, 0);
  std::vector<double> warm_best(G), cold_best(G);
  std::vector<std::optional<std::optional<std::pair<std::vector<double>, bool>>>> cold_refit(G);
  std::atomic<uint64_t> refit_cold{0};
  struct Slot {
    double subject, cell;
    int ticket;  // index into the gene's tickets, -1 when the point is outside the domain
  };
  struct Flight {
    std::vector<long long> tickets;
    std::vector<Slot> slots;
    bool final_fit = false;
    int anchor = -1;  // warm start: index of the ticket whose iterate is stored
  };
  // Warm inner starts (warm mode, searched genes, not the audit twins): the
  // first point of each step of a gene's search stores its final (beta,
  // log_w) in slot (step & 1); every point of the next step starts its
  // Newton loop there instead of at (beta_start, 0). A step reads only the
  // slot the previous step wrote, so concurrent points never race.
  std::vector<int> wstep(G, 0);
  std::vector<std::array<char, 2>> wvalid(G, std::array<char, 2>{0, 0});
  std::vector<Flight> flight(T);
  std::vector<double> sigma(G), gamma(G);
  std::vector<int> conv(G);
  std::vector<FinalFit> finals(G);
  // a worker's requests of one pass, posted together; owners[k] = (gene,
  // index of the gene's ticket) for outbox[k]
  struct Outbox {
    std::vector<device::FitRequest> reqs;
    std::vector<std::pair<size_t, size_t>> owners;
  };
  auto plan_points = [&](size_t v, Outbox* box) {
    const size_t g = gene_of(v);
    GeneTask& t = tasks[v];
    Flight& f = flight[v];
    f.slots.clear();
    f.tickets.clear();
    f.anchor = -1;
    const bool inner_warm = warm && v < G && ss.opt.cold_inner == 0;
    const int wb = wstep[g] & 1;
    const bool can_read = inner_warm && wvalid[g][1 - wb];
    for (const auto& point : t.search->ask()) {
      double subject = 0.0, cell = 0.0;
      std::vector<double> beta;
      Slot slot{0.0, 0.0, -1};
      if (t.objective.request(point, ss.plans[g].beta_start, &subject, &cell, &beta)) {
        device::FitRequest r{};
        r.gene = static_cast<int32_t>(g);
        r.ord = t.search->order();
        r.reml = sh.params.reml ? 1 : 0;
        r.subject = subject;
        r.cell = cell;
        for (int j = 0; j < sh.n_coef; ++j) r.beta[j] = beta[j];
        if (inner_warm) {
          r.flags = (wb ? device::kWarmBuffer : 0) | (can_read ? device::kWarmRead : 0);
          if (f.anchor < 0) {
            r.flags |= device::kWarmWrite;
            f.anchor = static_cast<int>(f.tickets.size());
          }
        }
        slot = Slot{subject, cell, static_cast<int>(f.tickets.size())};
        box->owners.emplace_back(v, f.tickets.size());
        box->reqs.push_back(r);
        f.tickets.push_back(-1);
      }
      f.slots.push_back(slot);
    }
  };
  auto plan_final = [&](size_t g, Outbox* box) {
    apply_refit(ss.plans[g], tasks[g].refit, &sigma[g], &gamma[g], &conv[g]);
    device::FitRequest r{};
    r.gene = static_cast<int32_t>(g);
    r.ord = 1;
    r.reml = sh.params.reml ? 1 : 0;
    r.subject = sigma[g];
    r.cell = gamma[g];
    for (int j = 0; j < sh.n_coef; ++j) r.beta[j] = ss.plans[g].beta_start[j];
    r.beta[sh.intercept] -= sigma[g] / 2.0;
    Flight& f = flight[g];
    f.final_fit = true;
    f.tickets.assign(1, -1);
    box->owners.emplace_back(g, 0);
    box->reqs.push_back(r);
  };
  const int hw = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
  // Twice as many workers as hardware threads: a worker mostly polls for
  // results and yields, and more of them turn results around sooner (on 16
  // threads, warm c1: 6267 genes/s with 16 workers, 7061 with 32).
  const int workers = std::max(1, std::min<int>({ss.opt.host_threads > 0 ? ss.opt.host_threads : 2 * hw, 32,
                                                 static_cast<int>(std::max<size_t>(G, 1))}));
  const int cluster = choose_cluster(ss, G);
  std::vector<DeviceFitter::Tally> tallies(workers + 1);  // the workers', then the poster's
  std::vector<uint64_t> steps(workers, 0);
  std::atomic<bool> abort{false};
  std::mutex err_mu;
  std::optional<NbError> first_err;
  // Admission. A gene's search is a chain of dependent evaluations, so the
  // step ends when the longest chains do. Requests in the ring are served
  // in ticket order, so posting every ready request at once would advance
  // all genes at the same slow pace and leave the long chains for last with
  // the SMs idle. Instead at most `cap` requests are in flight (5/4 of the
  // fits the kernel runs at once); the others wait in a heap keyed by their
  // task's predicted remaining work (longest first: the cold audit searches,
  // then the genes the network predicts to need the most evaluations, the
  // final fits last). The results do not depend on the order. On c1 (500
  // genes x 100,000 cells) a cap of twice the resident fits gave 7,500 warm
  // and 3,870 plain genes/s, 5/4 of them 7,650 and 4,100: fewer genes' entries
  // are live in L2 at once, and more of the waiting requests are ordered by
  // the heap instead of the ring.
  struct Entry {
    double priority;
    uint64_t order;
    size_t v;
    std::vector<device::FitRequest> reqs;
  };
  auto entry_less = [](const Entry& a, const Entry& b) {
    return a.priority < b.priority || (a.priority == b.priority && a.order > b.order);
  };
  std::mutex gate_mu;
  std::vector<Entry> heap;
  uint64_t gate_order = 0;
  long long in_flight = 0;
  const long long cap = 5 * static_cast<long long>(std::max(1, fitter.resident_fits(cluster))) / 4;
  // predicted remaining evaluations of task v, in units of a warm fit
  auto remaining = [&](size_t v) {
    const bool cold = !(warm && v < G);
    const double predicted = budget[gene_of(v)] * (cold ? 1.0 : kWarmEvaluationShare);
    const double done = static_cast<double>(tasks[v].search->evaluations());
    return std::max(predicted - done, 1.0) * (cold ? kColdFitCost : 1.0) + 1.0;
  };
  // Workers queue their ready requests here (`released` of theirs have been
  // consumed since their last call); the poster thread below posts them.
  auto post = [&](Outbox* box, long long released, int, DeviceFitter::Tally*) {
    std::lock_guard<std::mutex> lock(gate_mu);
    in_flight -= released;
    for (size_t k = 0; k < box->reqs.size();) {
      Entry e;
      e.v = box->owners[k].first;
      e.order = gate_order++;
      e.priority = flight[e.v].final_fit ? 1.0 : remaining(e.v);
      for (; k < box->reqs.size() && box->owners[k].first == e.v; ++k) e.reqs.push_back(box->reqs[k]);
      heap.push_back(std::move(e));
      std::push_heap(heap.begin(), heap.end(), entry_less);
    }
    box->reqs.clear();
    box->owners.clear();
  };
  // One poster thread drains the heap while room remains and posts each
  // drain as one batch outside the lock, so workers never wait on the copies
  // and the batches grow while a post is under way (posting from every
  // worker held the lock for half of the step, one or two requests a post).
  std::atomic<int> workers_left{0};
  auto poster = [&](DeviceFitter::Tally* tally) {
    struct StopAtEnd {  // every ticket has been read, or the stage failed
      DeviceFitter& f;
      ~StopAtEnd() { f.queue_request_stop(); }
    } stop_at_end{fitter};
    std::vector<device::FitRequest> batch;
    std::vector<std::pair<size_t, size_t>> owners;
    try {
      while (!abort.load(std::memory_order_relaxed)) {
        batch.clear();
        owners.clear();
        bool idle = false;
        {
          std::lock_guard<std::mutex> lock(gate_mu);
          while (!heap.empty()) {
            const long long n = static_cast<long long>(heap.front().reqs.size());
            if (in_flight > 0 && in_flight + n > cap) break;
            std::pop_heap(heap.begin(), heap.end(), entry_less);
            Entry e = std::move(heap.back());
            heap.pop_back();
            for (size_t k = 0; k < e.reqs.size(); ++k) {
              batch.push_back(e.reqs[k]);
              owners.emplace_back(e.v, k);
            }
            in_flight += n;
            if (batch.size() >= 4096) break;
          }
          idle = batch.empty() && heap.empty() && workers_left.load() == 0;
        }
        if (idle) return;
        if (batch.empty()) {
          std::this_thread::yield();
          continue;
        }
        const long long first = fitter.queue_post(batch.data(), batch.size(), 0, tally);
        // the owning workers read the tickets with acquire loads
        for (size_t k = 0; k < owners.size(); ++k)
          std::atomic_ref<long long>(flight[owners[k].first].tickets[owners[k].second])
              .store(first + static_cast<long long>(k), std::memory_order_release);
      }
    } catch (const NbError& e) {
      std::lock_guard<std::mutex> lock(err_mu);
      if (!first_err) first_err = e;
      abort.store(true);
    } catch (const std::exception& e) {
      std::lock_guard<std::mutex> lock(err_mu);
      if (!first_err) first_err = NbError{NB_ERR_GPU, e.what()};
      abort.store(true);
    }
  };
  auto worker = [&](int w) {
    struct Leave {
      std::atomic<int>& left;
      ~Leave() { left.fetch_sub(1); }
    } leave{workers_left};
    try {
      DeviceFitter::Tally* tally = &tallies[w];
      Outbox box;
      std::vector<size_t> waiting;
      std::vector<size_t> mine;
      for (size_t g = static_cast<size_t>(w); g < G; g += static_cast<size_t>(workers)) mine.push_back(g);
      if (warm == 1)  // the searches predicted to take longest first
        std::stable_sort(mine.begin(), mine.end(), [&](size_t a, size_t b) { return budget[a] > budget[b]; });
      auto start_search = [&](size_t v, bool use_warm) {
        const size_t g = gene_of(v);
        const GenePlan& plan = ss.plans[g];
        std::optional<double> fixed_cell;
        std::vector<double> start;
        if (plan.refit == Refit::Both) {
          start = {plan.sigma, plan.gamma};
          if (use_warm) start = {warm_point[g][0], warm_point[g][1]};
        } else {
          start = {use_warm ? warm_point[g][0] : plan.sigma};
          fixed_cell = plan.gamma;
        }
        std::vector<double> lower, upper;
        variance_bounds(sh.params, fixed_cell.has_value(), &lower, &upper);
        for (size_t d = 0; d < start.size(); ++d) start[d] = std::clamp(start[d], lower[d], upper[d]);
        tasks[v].search = std::make_unique<StageTwoSearch>(start, lower, upper, plan.ord, use_warm ? radius : 1.0);
        tasks[v].objective = VarianceObjective::make(sh, ss.genes[g], fixed_cell);
        plan_points(v, &box);
        waiting.push_back(v);
      };
      for (size_t g : mine) {
        if (ss.plans[g].refit != Refit::None) {
          start_search(g, warm != 0);
          if (twin[g] >= 0) start_search(static_cast<size_t>(twin[g]), false);
        } else {
          plan_final(g, &box);
          waiting.push_back(g);
        }
        post(&box, 0, w, tally);  // every gene's first request as soon as it is planned
      }
      post(&box, 0, w, tally);
      auto last_progress = Clock::now();
      while (!waiting.empty() && !abort.load(std::memory_order_relaxed)) {
        bool progressed = false;
        long long released = 0;  // this pass's consumed requests
        for (size_t i = 0; i < waiting.size();) {
          const size_t g = waiting[i];
          if (parked[g]) {
            ++i;
            continue;
          }
          Flight& f = flight[g];
          // a gene planned earlier in this pass (an audited gene whose cold
          // twin just finished) holds tickets of -1 until the pass posts them
          bool ready = true;
          for (size_t k = f.tickets.size(); k > 0 && ready; --k) {
            const long long t = std::atomic_ref<long long>(f.tickets[k - 1]).load(std::memory_order_acquire);
            ready = t >= 0 && fitter.queue_done(t);
          }
          if (!ready) {
            ++i;
            continue;
          }
          progressed = true;
          ++steps[w];
          released += static_cast<long long>(f.tickets.size());
          if (f.final_fit) {
            fitter.queue_account(f.tickets[0], static_cast<int>(g), tally);
            const device::FitResult& r = fitter.queue_result(f.tickets[0]);
            if (r.status != 0) fail(NB_ERR_INVALID_ARGUMENT, "opt_pml rejected the final variance components");
            FinalFit& ff = finals[g];
            ff.beta.assign(r.beta, r.beta + sh.n_coef);
            ff.information.resize(static_cast<size_t>(sh.n_coef) * sh.n_coef);
            for (int a = 0; a < sh.n_coef; ++a)
              for (int b = 0; b < sh.n_coef; ++b)
                ff.information[a * sh.n_coef + b] = r.information[a * sh.n_coef + b];
            ff.log_likelihood = r.log_likelihood;
            ff.iterations = r.iterations;
            ff.backtracks = r.backtracks;
            fitter.queue_consumed(f.tickets[0]);
            waiting[i] = waiting.back();
            waiting.pop_back();
            continue;
          }
          GeneTask& t = tasks[g];
          const size_t gene = gene_of(g);
          std::vector<double> values(f.slots.size(), std::numeric_limits<double>::infinity());
          for (size_t p = 0; p < f.slots.size(); ++p) {
            const Slot& sl = f.slots[p];
            if (sl.ticket < 0) continue;
            const long long ticket = f.tickets[static_cast<size_t>(sl.ticket)];
            fitter.queue_account(ticket, static_cast<int>(gene), tally);
            const device::FitResult& r = fitter.queue_result(ticket);
            if (r.status != 0) continue;
            InnerFit fit{r.log_likelihood, r.log_likelihood_prev, r.log_det, r.second_order};
            values[p] = t.objective.assemble(sl.subject, sl.cell, fit, t.objective.tail(sl.cell));
          }
          if (warm && g < G) {
            const int wb = wstep[g] & 1;
            wvalid[g][wb] = f.anchor >= 0 && fitter.queue_result(f.tickets[static_cast<size_t>(f.anchor)]).status == 0;
            ++wstep[g];
          }
          for (long long t : f.tickets) fitter.queue_consumed(t);
          t.search->tell(values);
          if (t.search->done()) {
            t.refit = t.search->result();
            const double best = t.search->best_value();
            if (g < G) evaluations[g] = t.search->evaluations();
            t.search.reset();
            // the audit: both searches of a twinned gene must be done
            auto decide_and_finish = [&](size_t h) {
              const bool warm_ok = tasks[h].refit.has_value() && tasks[h].refit->has_value();
              const bool cold_ok = cold_refit[h].has_value() && cold_refit[h]->has_value();
              if (cold_ok && (!warm_ok || cold_best[h] < warm_best[h] - 1e-9 * std::fabs(cold_best[h]))) {
                tasks[h].refit = cold_refit[h];
                refit_cold.fetch_add(1);
              }
              parked[h] = 0;
              plan_final(h, &box);
            };
            if (g >= G) {  // a cold twin
              cold_refit[gene] = t.refit;
              cold_best[gene] = best;
              cold_done[gene] = 1;
              waiting[i] = waiting.back();
              waiting.pop_back();
              if (warm_done[gene]) decide_and_finish(gene);
              continue;
            }
            warm_best[g] = best;
            warm_done[g] = 1;
            if (twin[g] < 0 || cold_done[g]) {
              if (twin[g] < 0) plan_final(g, &box);
              else decide_and_finish(g);
            } else {
              parked[g] = 1;  // waits for its cold twin
            }
          } else {
            plan_points(g, &box);
          }
          ++i;
        }
        if (released > 0 || !box.reqs.empty()) post(&box, released, w, tally);
        if (progressed) {
          last_progress = Clock::now();
        } else {
          if (!fitter.queue_running()) fitter.queue_failure("ended with work pending");
          if (ms_since(last_progress) > 60000.0) fitter.queue_failure("made no progress for 60 s");
          std::this_thread::yield();
        }
      }
    } catch (const NbError& e) {
      std::lock_guard<std::mutex> lock(err_mu);
      if (!first_err) first_err = e;
      abort.store(true);
    } catch (const std::exception& e) {
      std::lock_guard<std::mutex> lock(err_mu);
      if (!first_err) first_err = NbError{NB_ERR_GPU, e.what()};
      abort.store(true);
    }
  };
  {
    struct QueueGuard {
      DeviceFitter& f;
      ~QueueGuard() { f.queue_abort(); }
    } guard{fitter};
    // as in stage one: the posting and reading threads run before the launch
    fitter.queue_prepare();
    workers_left.store(workers);
    std::thread post_thread(poster, &tallies[workers]);
    std::vector<std::thread> pool;
    for (int w = 0; w < workers; ++w) pool.emplace_back(worker, w);
    try {
      fitter.queue_launch(cluster);
    } catch (...) {
      abort.store(true);
      for (auto& th : pool) th.join();
      post_thread.join();
      throw;
    }
    for (auto& th : pool) th.join();
    post_thread.join();
    if (first_err) throw *first_err;
    fitter.queue_stop();
  }
  for (const auto& tl : tallies) fitter.add_tally(tl);
  uint64_t rounds = 0;
  for (uint64_t n : steps) rounds += n;
  const double ms_stage_two = ms_since(t2);
  auto t3 = Clock::now();
  std::vector<GeneOutcome> outcomes(G);
  for (size_t g = 0; g < G; ++g) outcomes[g] = finish_gene(sh, sigma[g], gamma[g], conv[g], finals[g]);
  if (ss.opt.evaluations)
    for (size_t g = 0; g < G; ++g) ss.opt.evaluations[g] = evaluations[g];
  const double ms_stage_three = ms_since(t3);
  const double ms_step = fitter.end_step();
  record_cluster(ss, cluster, fitter.device_ms());
  assemble_fit(sh, outcomes, ss.prep.kept, out);
  if (stats) {
    stats->rounds = rounds;
    stats->requests = fitter.requests();
    stats->sweeps = fitter.sweeps();
    stats->cell_visits = fitter.cell_visits();
    stats->sparse_visits = fitter.sparse_visits();
    stats->fit_slots = static_cast<uint64_t>(fitter.queue_grid(cluster));
    stats->slot_cycles = fitter.slot_cycles();
    stats->cluster = static_cast<uint64_t>(cluster);
    stats->audited = audit_of.size();
    stats->refit_cold = refit_cold.load();
    stats->gpu_launches = fitter.launches();
    stats->ms_prepare = ss.ms_prepare;
    stats->ms_upload = ss.ms_upload;
    stats->ms_busy_span = fitter.busy_span_ms();
    stats->ms_ticket_wait = fitter.ticket_wait_ms();
    stats->zero_groups = fitter.tabled_groups();
    stats->ms_stage_one = ss.ms_stage_one;
    stats->ms_stage_two = ms_stage_two;
    stats->ms_stage_three = ms_stage_three;
    stats->ms_device = fitter.device_ms();
    stats->ms_step_device = ms_step;
    stats->h2d_bytes = fitter.h2d_bytes();
    stats->d2h_bytes = fitter.d2h_bytes();
  }
}

int32_t run_nebula_device(const nb_csr* counts, const uint64_t* subject_id, const double* design,
                          uint32_t n_coef, const double* offset, const nb_params* params,
                          const nb_options* options, nb_fit* out, nb_stats* stats, char* err,
                          size_t err_len) {
  const auto t_start = Clock::now();
  try {
    if (!out) fail(NB_ERR_INVALID_ARGUMENT, "out is null");
    std::unique_ptr<Session> ss = create_session(counts, subject_id, design, n_coef, offset, params, options, true);
    const uint64_t upload = ss->fitter->h2d_bytes();
    if (stats) *stats = nb_stats{};
    fit_session(*ss, out, stats);
    if (stats) {
      stats->h2d_bytes += upload;
      stats->ms_total = ms_since(t_start);
    }
    return NB_OK;
  } catch (const NbError& e) {
    write_err(err, err_len, e.message);
    return e.code;
  }
}

}  // namespace nebula

struct nb_session {
  std::unique_ptr<nebula::Session> impl;
};

NB_API int32_t nb_session_create(const nb_csr* counts, const uint64_t* subject_id, const double* design,
                                 uint32_t n_coef, const double* offset_or_null, const nb_params* params_or_null,
                                 const nb_options* options, nb_session** out, char* err, size_t err_len) {
  try {
    if (!out) nebula::fail(NB_ERR_INVALID_ARGUMENT, "out is null");
    auto s = std::make_unique<nb_session>();
    s->impl = nebula::create_session(counts, subject_id, design, n_coef, offset_or_null, params_or_null, options,
                                     false);
    *out = s.release();
    return NB_OK;
  } catch (const nebula::NbError& e) {
    nebula::write_err(err, err_len, e.message);
    return e.code;
  }
}

NB_API int32_t nb_session_features(nb_session* session, float* features, double* stage_one, uint64_t* n_kept,
                                   char* err, size_t err_len) {
  try {
    if (!session || !session->impl) nebula::fail(NB_ERR_INVALID_ARGUMENT, "null session");
    nebula::Session& ss = *session->impl;
    const nebula::Shared& sh = ss.prep.shared;
    const size_t G = ss.genes.size();
    const int K = sh.n_subjects;
    if (n_kept) *n_kept = G;
    for (size_t g = 0; g < G; ++g) {
      if (features)
        nebula::warm_features(sh, ss.genes[g], &ss.prep.totals[ss.prep.kept[g] * K], ss.plans[g],
                              features + g * nebula::mlp::kIn);
      if (stage_one) {
        stage_one[2 * g] = ss.plans[g].sigma;
        stage_one[2 * g + 1] = ss.plans[g].gamma;
      }
    }
    return NB_OK;
  } catch (const nebula::NbError& e) {
    nebula::write_err(err, err_len, e.message);
    return e.code;
  }
}

NB_API int32_t nb_session_fit(nb_session* session, nb_fit* out, nb_stats* stats, char* err, size_t err_len) {
  try {
    if (!session || !out) nebula::fail(NB_ERR_INVALID_ARGUMENT, "null session or output");
    if (stats) *stats = nb_stats{};
    nebula::fit_session(*session->impl, out, stats);
    if (stats) {
      stats->ms_prepare = session->impl->ms_prepare;
      stats->ms_stage_one = session->impl->ms_stage_one;
    }
    return NB_OK;
  } catch (const nebula::NbError& e) {
    nebula::write_err(err, err_len, e.message);
    return e.code;
  }
}

NB_API void nb_session_free(nb_session* session) { delete session; }

NB_API void nb_params_default(nb_params* p) {
  if (!p) return;
  nebula::Params d;
  p->min_subject = d.min0;
  p->min_cell = d.min1;
  p->max_subject = d.max0;
  p->max_cell = d.max1;
  p->method = d.method;
  p->cutoff_cell = d.cutoff_cell;
  p->kappa = d.kappa;
  p->cpc = d.cpc;
  p->mincp = d.mincp;
  p->min_subjects = d.min_subjects;
  p->reml = d.reml ? 1 : 0;
  p->eps = d.eps;
}

NB_API int32_t nebula_sparse_cuda(const nb_csr* counts, const uint64_t* subject_id, const double* design,
                                  uint32_t n_coef, const double* offset_or_null,
                                  const nb_params* params_or_null, nb_fit* out, char* err, size_t err_len) {
  return nebula::run_nebula_device(counts, subject_id, design, n_coef, offset_or_null, params_or_null,
                                   nullptr, out, nullptr, err, err_len);
}

NB_API int32_t nebula_sparse_cuda_ex(const nb_csr* counts, const uint64_t* subject_id, const double* design,
                                     uint32_t n_coef, const double* offset_or_null,
                                     const nb_params* params_or_null, const nb_options* options, nb_fit* out,
                                     nb_stats* stats, char* err, size_t err_len) {
  return nebula::run_nebula_device(counts, subject_id, design, n_coef, offset_or_null, params_or_null, options,
                                   out, stats, err, err_len);
}

// opt_pml (src/sc/pml.rs:468-508) for a batch of variance points of one
// gene, on the device; the batched twin of the reference's device entry
// (src/gpu/nebula_gpu.rs:466-594 opt_pml_batch). scalars_out per request:
// log_likelihood, log_likelihood_prev, log_det, second_order; ints_out:
// status (0 ok, 1 rejected arguments), iterations, backtracks, sweeps.
NB_API int32_t nb_opt_pml_cuda(const double* design, const double* offset, uint64_t n_cells, uint32_t n_beta,
                               const double* counts, const uint32_t* cells, uint64_t n_pos,
                               const uint64_t* subject_start, uint32_t k, const double* subject_total,
                               uint32_t n_requests, const double* beta_init, const double* subject,
                               const double* cell, const int32_t* ord, int32_t reml, double eps,
                               double* beta_out, double* information_out, double* scalars_out,
                               int32_t* ints_out, char* err, size_t err_len) {
  using namespace nebula;
  try {
    if (n_beta == 0 || n_beta > static_cast<uint32_t>(device::kMaxCoef))
      fail(NB_ERR_UNSUPPORTED, "the device path takes 1 to 8 design columns");
    if (k == 0 || n_cells == 0) fail(NB_ERR_MUST_BE_POSITIVE, "need cells and subjects");
    if (subject_start[0] != 0 || subject_start[k] != n_cells)
      fail(NB_ERR_INVALID_ARGUMENT, "subject_start must run from 0 to n_cells");
    for (uint32_t s = 0; s < k; ++s)
      if (subject_start[s] >= subject_start[s + 1])
        fail(NB_ERR_SUBJECTS_NOT_CONTIGUOUS, "empty or unordered subject block");
    for (uint64_t i = 0; i < n_pos; ++i)
      if (cells[i] >= n_cells || (i > 0 && cells[i] <= cells[i - 1]))
        fail(NB_ERR_INVALID_ARGUMENT, "Cell indices must be strictly increasing and in range.");
    Prepared prep;
    Shared& sh = prep.shared;
    sh.design.assign(design, design + n_cells * n_beta);
    sh.log_offset.assign(offset, offset + n_cells);
    sh.fid.assign(subject_start, subject_start + k + 1);
    sh.n_cells = n_cells;
    sh.n_coef = static_cast<int>(n_beta);
    sh.n_subjects = static_cast<int>(k);
    sh.params.eps = eps;
    prep.totals.assign(subject_total, subject_total + k);
    prep.kept = {0};
    std::vector<GeneCounts> genes(1);
    genes[0].own(cells, counts, n_pos);
    DeviceFitter fitter(prep, genes, -1);
    std::vector<device::FitRequest> reqs(n_requests);
    for (uint32_t q = 0; q < n_requests; ++q) {
      device::FitRequest& r = reqs[q];
      r = device::FitRequest{};
      r.gene = 0;
      r.ord = ord ? ord[q] : 1;
      r.reml = reml;
      r.subject = subject[q];
      r.cell = cell[q];
      for (uint32_t j = 0; j < n_beta; ++j) r.beta[j] = beta_init[q * n_beta + j];
    }
    const device::FitResult* res = fitter.run(reqs);
    for (uint32_t q = 0; q < n_requests; ++q) {
      const device::FitResult& r = res[q];
      for (uint32_t j = 0; j < n_beta; ++j) beta_out[q * n_beta + j] = r.beta[j];
      for (uint32_t j = 0; j < n_beta * n_beta; ++j) information_out[q * n_beta * n_beta + j] = r.information[j];
      scalars_out[q * 4 + 0] = r.log_likelihood;
      scalars_out[q * 4 + 1] = r.log_likelihood_prev;
      scalars_out[q * 4 + 2] = r.log_det;
      scalars_out[q * 4 + 3] = r.second_order;
      ints_out[q * 4 + 0] = r.status;
      ints_out[q * 4 + 1] = r.iterations;
      ints_out[q * 4 + 2] = r.backtracks;
      ints_out[q * 4 + 3] = r.sweeps;
    }
    return NB_OK;
  } catch (const NbError& e) {
    if (err && err_len) {
      size_t n = std::min(err_len - 1, e.message.size());
      std::memcpy(err, e.message.data(), n);
      err[n] = 0;
    }
    return e.code;
  }
}
