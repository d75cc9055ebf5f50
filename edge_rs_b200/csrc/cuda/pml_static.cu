// nb_opt_pml_cuda_noalloc: the batched inner fit of nb_opt_pml_cuda for
// callers that cannot allocate device memory.
//
// Who needs it: a host program that hands this library device buffers it
// already owns and must not have the library allocate behind its back — an
// engine whose device memory belongs to its own pool or arena (a caching
// allocator, a fixed HBM budget per tenant), a real-time loop where a
// cudaMalloc's implicit device synchronisation would stall other streams, or
// a plugin loaded into a process that forbids allocation after start-up.
// nb_opt_pml_cuda copies host arrays into device memory it allocates per
// call; this entry point takes device pointers for every input and output
// and keeps its working memory (the fit kernel's request and result records,
// the per-subject layout it derives, the work-queue counter) in one
// file-scope device array of fixed size instead.
//
// Limits: that array is kNoAllocScratchBytes = 2 MiB per device, loaded with
// the library's module and held by every GPU that loads it until the process
// exits. A call takes at most kNoAllocMaxRequests = 2048 requests and
// kNoAllocMaxSubjects = 8192 subjects; larger calls are refused with
// NB_ERR_INVALID_ARGUMENT before anything is launched.
//
// Sharing: every call on a device uses the same array, and the array keeps
// the last call's contents; each call rewrites the words that must start at
// zero (queue counter, validation flags) before its kernels read them. Calls
// whose GPU work overlaps — issued from several host threads, on any streams
// — race on the array and corrupt each other's results: issue them one at a
// time per device.
//
// Set-up: the first call on a device (the calling thread's current device)
// looks up the array's device address with cudaGetSymbolAddress and the SM
// count, and caches both for that device for the life of the process; calls
// after a cudaDeviceReset of that device are not supported (the module's
// array may then sit elsewhere). Every call is blocking (it reads a status
// word back and synchronises its stream before returning), so no call can be
// made while a stream is being captured.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <mutex>
#include <string>

#include "../host/common.hpp"
#include "../host/export.hpp"
#include "pml_device.cuh"

namespace nebula {
namespace device {
namespace {

constexpr uint32_t kNoAllocMaxRequests = 2048;
constexpr uint32_t kNoAllocMaxSubjects = 8192;
constexpr size_t kNoAllocScratchBytes = size_t{2} << 20;
constexpr size_t kScratchAlign = 256;
constexpr int kMaxDevices = 64;
constexpr int kStageThreads = 256;

// Validation flags the staging kernel raises (the checks nb_opt_pml_cuda
// makes on the host).
enum : int32_t { kBadSubjectRange = 1, kBadSubjectBlock = 2, kBadCells = 4 };

constexpr size_t round_up(size_t bytes) { return (bytes + kScratchAlign - 1) / kScratchAlign * kScratchAlign; }

// Byte offsets of one call's regions inside the array.
struct Layout {
  size_t header;      // int32 [0] request count, [1] work-queue counter, [2] validation flags
  size_t fid;         // uint32 (k + 1) subject boundaries
  size_t runs;        // uint64 (k + 1) first positive entry of each subject
  size_t gene_ptr;    // uint64 2
  size_t warp_cells;  // uint32 kWarps + 1
  size_t range_cells; // uint32 kRanges + 1
  size_t range_pos;   // uint64 kRanges + 1
  size_t requests;    // FitRequest n
  size_t results;     // FitResult n
  size_t end;
};

constexpr Layout layout_for(size_t k, size_t n) {
  Layout l{};
  l.header = 0;
  l.fid = l.header + round_up(4 * sizeof(int32_t));
  l.runs = l.fid + round_up((k + 1) * sizeof(uint32_t));
  l.gene_ptr = l.runs + round_up((k + 1) * sizeof(uint64_t));
  l.warp_cells = l.gene_ptr + round_up(2 * sizeof(uint64_t));
  l.range_cells = l.warp_cells + round_up((kWarps + 1) * sizeof(uint32_t));
  l.range_pos = l.range_cells + round_up((kRanges + 1) * sizeof(uint32_t));
  l.requests = l.range_pos + round_up((kRanges + 1) * sizeof(uint64_t));
  l.results = l.requests + round_up(n * sizeof(FitRequest));
  l.end = l.results + round_up(n * sizeof(FitResult));
  return l;
}

static_assert(layout_for(kNoAllocMaxSubjects, kNoAllocMaxRequests).end <= kNoAllocScratchBytes,
              "the largest accepted call must fit the no-allocation scratch array");

}  // namespace
}  // namespace device
}  // namespace nebula

// The shared working memory. In host code this name is only a handle for
// cudaGetSymbolAddress, never a device address.
static __device__ __align__(256) unsigned char nb_noalloc_scratch[nebula::device::kNoAllocScratchBytes];

namespace nebula {
namespace device {
namespace {

// Checks the subject blocks and positive cells, marks the design columns
// that vary within a subject (header[3], one bit per column), and writes the
// derived per-subject layout and the request records into the scratch array.
__global__ void stage_noalloc(unsigned char* scratch, Layout L, const double* design,
                              const uint64_t* subject_start, uint32_t k,
                              uint64_t n_cells, const uint32_t* cells, uint64_t n_pos, uint32_t n_req,
                              uint32_t n_beta, const double* beta_init, const double* subject, const double* cell,
                              const int32_t* ord, int32_t reml) {
  int32_t* header = reinterpret_cast<int32_t*>(scratch + L.header);
  uint32_t* fid = reinterpret_cast<uint32_t*>(scratch + L.fid);
  uint64_t* runs = reinterpret_cast<uint64_t*>(scratch + L.runs);
  uint64_t* gene_ptr = reinterpret_cast<uint64_t*>(scratch + L.gene_ptr);
  uint32_t* warp_cells = reinterpret_cast<uint32_t*>(scratch + L.warp_cells);
  uint32_t* range_cells = reinterpret_cast<uint32_t*>(scratch + L.range_cells);
  uint64_t* range_pos = reinterpret_cast<uint64_t*>(scratch + L.range_pos);
  FitRequest* reqs = reinterpret_cast<FitRequest*>(scratch + L.requests);
  const uint64_t tid = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;

  for (uint64_t i = tid; i < n_pos; i += stride) {
    const uint32_t c = cells[i];
    if (c >= n_cells || (i > 0 && c <= cells[i - 1])) atomicOr(&header[2], kBadCells);
  }
  for (uint64_t r = tid; r < n_cells; r += stride) {
    // the subject block holding cell r: the last s with subject_start[s] <= r
    uint64_t lo = 0, hi = k;
    while (lo < hi) {
      const uint64_t mid = lo + (hi - lo + 1) / 2;
      if (subject_start[mid] <= r) lo = mid; else hi = mid - 1;
    }
    const uint64_t first = subject_start[lo];
    if (first >= r) continue;  // r starts its block (or the blocks are malformed)
    for (uint32_t j = 0; j < n_beta; ++j)
      if (design[r * n_beta + j] != design[first * n_beta + j]) atomicOr(&header[3], 1 << j);
  }
  for (uint64_t s = tid; s <= k; s += stride) {
    const uint64_t b = subject_start[s];
    if ((s == 0 && b != 0) || (s == k && b != n_cells)) atomicOr(&header[2], kBadSubjectRange);
    if (s < k && b >= subject_start[s + 1]) atomicOr(&header[2], kBadSubjectBlock);
    fid[s] = static_cast<uint32_t>(b);
    // positive_runs (pml.rs:1155-1160): first positive entry at or after b
    uint64_t lo = 0, hi = n_pos;
    while (lo < hi) {
      const uint64_t mid = lo + (hi - lo) / 2;
      if (cells[mid] < b) lo = mid + 1; else hi = mid;
    }
    runs[s] = lo;
  }
  for (uint64_t q = tid; q < n_req; q += stride) {
    FitRequest r{};
    r.gene = 0;
    r.ord = ord ? ord[q] : 1;
    r.reml = reml;
    r.subject = subject[q];
    r.cell = cell[q];
    for (uint32_t j = 0; j < n_beta; ++j) r.beta[j] = beta_init[q * n_beta + j];
    reqs[q] = r;
  }
  if (tid <= static_cast<uint64_t>(kWarps)) warp_cells[tid] = static_cast<uint32_t>(n_cells * tid / kWarps);
  for (uint64_t v = tid; v <= static_cast<uint64_t>(kRanges); v += stride) {
    // the sweep's cell ranges and the first positive entry at or after each boundary
    const uint64_t b = n_cells * v / kRanges;
    range_cells[v] = static_cast<uint32_t>(b);
    uint64_t lo = 0, hi = n_pos;
    while (lo < hi) {
      const uint64_t mid = lo + (hi - lo) / 2;
      if (cells[mid] < b) lo = mid + 1; else hi = mid;
    }
    range_pos[v] = lo;
  }
  if (tid == 0) {
    gene_ptr[0] = 0;
    gene_ptr[1] = n_pos;
    header[0] = static_cast<int32_t>(n_req);
    header[1] = 0;
  }
}

// Copies the fit records into the caller's output arrays (the layout of
// nb_opt_pml_cuda).
__global__ void unpack_noalloc(const FitResult* res, uint32_t n_req, uint32_t n_beta, double* beta_out,
                               double* information_out, double* scalars_out, int32_t* ints_out) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n_req) return;
  const FitResult& r = res[q];
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

struct DeviceSlot {
  unsigned char* scratch;
  int sms;
};
std::mutex g_slots_mu;
DeviceSlot g_slots[kMaxDevices];

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) fail(NB_ERR_GPU, std::string(what) + ": " + cudaGetErrorString(e));
}

void write_err(char* err, size_t len, const std::string& msg) {
  if (!err || len == 0) return;
  const size_t n = std::min(len - 1, msg.size());
  std::memcpy(err, msg.data(), n);
  err[n] = 0;
}

// The array's address and the SM count on the current device, looked up
// once per device.
DeviceSlot slot_for_current_device() {
  int dev = 0;
  check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) fail(NB_ERR_GPU, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_slots_mu);
  DeviceSlot& s = g_slots[dev];
  if (!s.scratch) {
    void* ptr = nullptr;
    check(cudaGetSymbolAddress(&ptr, nb_noalloc_scratch), "cudaGetSymbolAddress of the scratch array");
    int sms = 0;
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    s.sms = sms;
    s.scratch = static_cast<unsigned char*>(ptr);
  }
  return s;
}

}  // namespace
}  // namespace device
}  // namespace nebula

NB_API int32_t nb_opt_pml_cuda_noalloc(const double* design, const double* offset, uint64_t n_cells,
                                       uint32_t n_beta, const double* counts, const uint32_t* cells,
                                       uint64_t n_pos, const uint64_t* subject_start, uint32_t k,
                                       const double* subject_total, uint32_t n_requests, const double* beta_init,
                                       const double* subject, const double* cell, const int32_t* ord,
                                       int32_t reml, double eps, double* beta_out, double* information_out,
                                       double* scalars_out, int32_t* ints_out, void* stream, char* err,
                                       size_t err_len) {
  using namespace nebula;
  using namespace nebula::device;
  try {
    if (n_beta == 0 || n_beta > static_cast<uint32_t>(kMaxCoef))
      fail(NB_ERR_UNSUPPORTED, "the device path takes 1 to 8 design columns");
    if (k == 0 || n_cells == 0) fail(NB_ERR_MUST_BE_POSITIVE, "need cells and subjects");
    if (n_cells > static_cast<uint64_t>(INT_MAX)) fail(NB_ERR_INVALID_ARGUMENT, "too many cells for the device path");
    if (n_requests > kNoAllocMaxRequests)
      fail(NB_ERR_INVALID_ARGUMENT, "nb_opt_pml_cuda_noalloc takes at most " + std::to_string(kNoAllocMaxRequests) +
                                        " requests per call (fixed 2 MiB scratch array); got " +
                                        std::to_string(n_requests));
    if (k > kNoAllocMaxSubjects)
      fail(NB_ERR_INVALID_ARGUMENT, "nb_opt_pml_cuda_noalloc takes at most " + std::to_string(kNoAllocMaxSubjects) +
                                        " subjects (fixed 2 MiB scratch array); got " + std::to_string(k));
    if (!design || !offset || !subject_start || !subject_total || (n_pos && (!counts || !cells)))
      fail(NB_ERR_INVALID_ARGUMENT, "null input array");
    if (n_requests == 0) return NB_OK;
    if (!beta_init || !subject || !cell || !beta_out || !information_out || !scalars_out || !ints_out)
      fail(NB_ERR_INVALID_ARGUMENT, "null request or output array");

    const DeviceSlot slot = slot_for_current_device();
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const Layout L = layout_for(k, n_requests);
    unsigned char* base = slot.scratch;
    int32_t* header = reinterpret_cast<int32_t*>(base + L.header);

    check(cudaMemsetAsync(header, 0, 4 * sizeof(int32_t), st), "clearing the scratch header");
    uint64_t items = n_pos;
    if (k + uint64_t{1} > items) items = k + uint64_t{1};
    if (n_requests > items) items = n_requests;
    if (static_cast<uint64_t>(kRanges) + 1 > items) items = kRanges + 1;
    if (n_cells > items) items = n_cells;
    uint64_t blocks = (items + kStageThreads - 1) / kStageThreads;
    const uint64_t max_blocks = static_cast<uint64_t>(slot.sms) * 8;
    if (blocks > max_blocks) blocks = max_blocks;
    stage_noalloc<<<static_cast<unsigned>(blocks), kStageThreads, 0, st>>>(
        base, L, design, subject_start, k, n_cells, cells, n_pos, n_requests, n_beta, beta_init, subject, cell, ord,
        reml);
    check(cudaGetLastError(), "staging launch");
    int32_t flags_mask[2] = {0, 0};  // validation flags, varying columns
    check(cudaMemcpyAsync(flags_mask, header + 2, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, st),
          "validation flags");
    check(cudaStreamSynchronize(st), "staging");
    const int32_t flags = flags_mask[0];
    if (flags & kBadSubjectRange) fail(NB_ERR_INVALID_ARGUMENT, "subject_start must run from 0 to n_cells");
    if (flags & kBadSubjectBlock) fail(NB_ERR_SUBJECTS_NOT_CONTIGUOUS, "empty or unordered subject block");
    if (flags & kBadCells)
      fail(NB_ERR_INVALID_ARGUMENT, "Cell indices must be strictly increasing and in range.");

    GeneData data{};
    data.design = design;
    data.log_offset = offset;
    data.fid = reinterpret_cast<const uint32_t*>(base + L.fid);
    data.gene_ptr = reinterpret_cast<const uint64_t*>(base + L.gene_ptr);
    data.cells = cells;
    data.counts = counts;
    data.runs = reinterpret_cast<const uint64_t*>(base + L.runs);
    data.totals = subject_total;
    data.warp_cells = reinterpret_cast<const uint32_t*>(base + L.warp_cells);
    data.range_cells = reinterpret_cast<const uint32_t*>(base + L.range_cells);
    data.range_pos = reinterpret_cast<const uint64_t*>(base + L.range_pos);
    data.n_cells = static_cast<int32_t>(n_cells);
    data.n_subjects = static_cast<int32_t>(k);
    data.n_coef = static_cast<int32_t>(n_beta);
    data.n_varying = 0;
    for (uint32_t j = 0; j < n_beta; ++j)
      if (flags_mask[1] & (1 << j)) data.varying[data.n_varying++] = static_cast<int32_t>(j);
    const int per_sm = fit_blocks_per_sm(static_cast<int>(k), static_cast<int>(n_beta), data.n_varying);
    if (per_sm <= 0)
      fail(NB_ERR_UNSUPPORTED, "the fit kernel cannot be resident with " + std::to_string(k) + " subjects and " +
                                   std::to_string(n_beta) + " columns");
    FitControl ctl{};
    ctl.eps = eps;
    ctl.max_iter = kPmlMaxIter;
    ctl.max_backtrack = kPmlMaxBacktrack;
    FitResult* results = reinterpret_cast<FitResult*>(base + L.results);
    const int launched = launch_fit(data, ctl, reinterpret_cast<const FitRequest*>(base + L.requests), results,
                                    header, header + 1, per_sm * slot.sms, 1, st);
    check(static_cast<cudaError_t>(launched), "fit kernel launch");
    unpack_noalloc<<<(n_requests + kStageThreads - 1) / kStageThreads, kStageThreads, 0, st>>>(
        results, n_requests, n_beta, beta_out, information_out, scalars_out, ints_out);
    check(cudaGetLastError(), "unpack launch");
    check(cudaStreamSynchronize(st), "fit");
    return NB_OK;
  } catch (const NbError& e) {
    nebula::device::write_err(err, err_len, e.message);
    return e.code;
  }
}
