// Layout shared by the host driver and the batched inner-fit kernel.
//
// The kernel runs the reference's penalised NB-gamma inner fit (opt_pml,
// src/sc/pml.rs:1614-1800) for a batch of requests, one (gene, sigma, gamma)
// point each, in FP64 throughout: the profile objective the stage-two search
// compares must agree with the CPU path to ~1e-12 so that BOBYQA, whose
// resolution is ~1e-6, retraces the same points.
#pragma once

#include <cstddef>
#include <cstdint>

#include "../host/zero_group.hpp"

namespace nebula {
namespace device {

constexpr int kMaxCoef = 8;        // the device path's width cap (pml_kernel.rs:1208-1212)
constexpr int kThreads = 256;      // threads per fit CTA
constexpr int kWarps = kThreads / 32;
constexpr int kRanges = 64;        // fixed cell ranges of a sweep's summation tree
constexpr int kMaxCluster = 8;     // CTAs one request may be spread over

// One inner fit to run.
struct alignas(16) FitRequest {
  int32_t gene;       // row of the resident CSR (kept genes, in kept order)
  int32_t ord;        // Laplace order (1, 2 or 3)
  int32_t reml;       // add log|det(information)| to the log-determinant
  int32_t flags;      // warm inner starts (kWarm*); 0 = the reference's cold start
  double subject;     // nebula's sigma[0] = log(1 + sigma^2)
  double cell;        // NB size gamma
  double beta[kMaxCoef];  // starting fixed effects (log_w starts at zero)
};

// What one inner fit hands back (PmlResult, pml.rs:288-326).
struct alignas(16) FitResult {
  double log_likelihood, log_likelihood_prev, log_det, second_order;
  double beta[kMaxCoef];
  double information[kMaxCoef * kMaxCoef];
  int32_t iterations, backtracks, sweeps, status;  // status 0 ok, 1 rejected arguments
  int64_t cycles;  // SM clock cycles the request held its CTAs (summed over the cluster)
  int64_t start_ns, end_ns;  // global timer when the fit began and ended
  int64_t wait_ns;  // streaming mode: how long the cluster waited for this ticket's request
};

// FitRequest.flags: start the Newton loop from the gene's stored (beta,
// log_w) in buffer 1 - kWarmBuffer instead of (beta, 0); store the final
// (beta, log_w) into buffer kWarmBuffer.
constexpr int32_t kWarmRead = 1;
constexpr int32_t kWarmWrite = 2;
constexpr int32_t kWarmBuffer = 4;

// Resident per-call data, device pointers.
struct GeneData {
  const double* design;      // n_cells x n_coef, centred, row-major
  const double* log_offset;  // n_cells
  const uint32_t* fid;       // n_subjects + 1
  const uint64_t* gene_ptr;  // n_genes + 1 into cells/counts
  const uint32_t* cells;     // positive entries' cells, increasing per gene
  const double* counts;      // positive counts
  const uint64_t* runs;      // n_genes x (n_subjects + 1): first positive entry of each subject
  const double* totals;      // n_genes x n_subjects count totals
  const uint32_t* warp_cells;  // ptmg_warps + 1 boundaries of stage one's warp ranges
  const uint32_t* range_cells; // kRanges + 1 boundaries of the sweep's cell ranges
  const uint64_t* range_pos;   // n_genes x (kRanges + 1): first positive entry at or after each boundary
  double* warm_state;          // n_genes x 2 x (n_coef + n_subjects), or null
  int32_t n_cells;
  int32_t n_subjects;
  int32_t n_coef;
  // The columns that vary within some subject, increasing (the reference's
  // cell_level_columns, ptmg.rs:1962-2005); every other column is constant
  // within each subject, and a sweep applies its share per subject instead
  // of per cell.
  int32_t n_varying;
  int32_t varying[kMaxCoef];
  // Zero-count tables (zero_group.hpp) when the design is categorical enough
  // (zero_tables.hpp): a sweep's dense part then visits only the loose cells,
  // and each subject's tabled groups add their looked-up sums.
  int32_t tabled;
  const zero::Group* zgroups;     // subject by subject
  const uint32_t* zsubject;       // n_subjects + 1 into zgroups
  const uint32_t* zindex;         // per base panel: first panel, depth
  const double* zpanels;          // zero::kPanelDoubles per panel
  const uint32_t* loose;          // cells in no tabled group, ascending
  const uint32_t* subject_loose;  // n_subjects + 1 into loose
  const uint64_t* loose_pos;      // kRanges + 1: first loose entry at or after each range boundary
};

// The columns of a row-major n_cells x n_coef design that take more than one
// value within some subject (subjects are the contiguous blocks between
// fid[s] and fid[s + 1]); writes them increasing into `out` and returns how
// many there are.
template <typename Boundary>
inline int varying_columns(const double* design, int n_coef, const Boundary* fid, int n_subjects, int32_t* out) {
  int n = 0;
  for (int j = 0; j < n_coef; ++j) {
    bool varies = false;
    for (int s = 0; s < n_subjects && !varies; ++s) {
      if (fid[s] >= fid[s + 1]) continue;
      const double first = design[static_cast<size_t>(fid[s]) * n_coef + j];
      for (size_t i = static_cast<size_t>(fid[s]) + 1; i < static_cast<size_t>(fid[s + 1]); ++i)
        if (design[i * n_coef + j] != first) {
          varies = true;
          break;
        }
    }
    if (varies) out[n++] = j;
  }
  return n;
}

struct FitControl {
  double eps;
  int32_t max_iter;
  int32_t max_backtrack;
};

// Shared-memory bytes one fit CTA needs for n_subjects, n_coef columns and
// n_varying of them varying within subjects.
size_t fit_smem_bytes(int n_subjects, int n_coef, int n_varying);

// Launches the persistent fit kernel over *n_requests (read on the device)
// requests; `counter` must be zeroed before each launch (work queue).
// `grid` CTAs, in thread-block clusters of `cluster` (1, 2, 4 or 8; grid a
// multiple of it), loop over the queue, each cluster taking one request at a
// time and sharing its sweeps. Returns cudaError_t as int.
int launch_fit(const GeneData& data, const FitControl& ctl, const FitRequest* requests,
               FitResult* results, const int32_t* n_requests, int32_t* counter, int grid,
               int cluster, void* stream);

// Streaming mode: one persistent launch serves requests the host posts while
// it runs, through a request ring (ring_device.cuh).
// - The host stores ticket t's request in host_ring[t & mask] and then
//   releases `posted` = t + 1 (tickets are posted in order). Both are host
//   memory mapped into the device's address space, so posting needs no copy
//   engine and works while launches are serialised.
// - A cluster takes the next ticket off words[kTaken] and waits until
//   words[kForwarded] > t, polling L2 only. One waiting warp at a time (the
//   holder of words[kLock]) reads `posted` across the bus and forwards the
//   newly posted requests into the device ring; the rest never touch host
//   memory, so a hundred idle clusters add no bus traffic that the result
//   writes and their fences would queue behind.
// - The cluster reads its request from the device ring, runs it, writes the
//   result into results[t & mask] (mapped) and then done[t & mask] = t + 1.
// - *stop != 0 (mapped) means nothing more will be posted: the lock holder
//   that has forwarded everything sets words[kStopped], and clusters waiting
//   on a ticket nobody will post exit. A wait that runs out (idle_ns by the
//   global timer) sets *status = 1 (mapped) and exits too.
struct RingView {
  const char* host_ring;             // mapped: requests as posted
  const unsigned long long* posted;  // mapped: tickets below it are posted
  const int* stop;                   // mapped
  int* status;                       // mapped
  char* ring;                        // device: forwarded requests
  unsigned long long* words;         // device: kRingWords counters, zeroed before the launch
  long long mask;                    // ring capacity - 1 (a power of two)
  long long idle_ns;
  int request_bytes;                 // a multiple of 8
};
constexpr int kTaken = 0, kForwarded = 1, kLock = 2, kStopped = 3, kRingWords = 4;

struct FitQueue {
  RingView ring;
  FitResult* results;  // mapped
  long long* done;     // mapped
};

int launch_fit_queue(const GeneData& data, const FitControl& ctl, const FitQueue& queue, int grid, int cluster,
                     void* stream);

// The ring's self-check (ring_check.cu): one-warp CTAs serve tickets with
// the same ring_next / ring_publish as the persistent kernels and answer
// each EchoRequest with its EchoResult.
struct EchoRequest {
  unsigned long long tag, a, b, c;
};
struct EchoResult {
  unsigned long long tag, mixed, folded, ticket;
};
__host__ __device__ inline EchoResult echo_of(const EchoRequest& q, long long ticket) {
  const unsigned long long t = static_cast<unsigned long long>(ticket);
  return EchoResult{q.tag, q.a * 0x9E3779B97F4A7C15ull + q.b, q.c ^ (t * 0xD1B54A32D192ED03ull), t};
}
int launch_ring_echo(const RingView& ring, EchoResult* results, long long* done, int ctas, void* stream);

// dst[i] = src[i] for n counts uploaded as floats (upload.cu).
int widen_counts(const float* src, double* dst, size_t n, void* stream);

// Clusters of `cluster` CTAs the streaming kernel can keep resident at once.
int fit_queue_max_clusters(int n_subjects, int n_coef, int n_varying, int cluster);

// CTAs per SM the fit kernel can keep resident for this shape.
int fit_blocks_per_sm(int n_subjects, int n_coef, int n_varying);

// Clusters of `cluster` CTAs the fit kernel can keep resident at once (0 if
// none fits).
int fit_max_clusters(int n_subjects, int n_coef, int n_varying, int cluster);

}  // namespace device
}  // namespace nebula
