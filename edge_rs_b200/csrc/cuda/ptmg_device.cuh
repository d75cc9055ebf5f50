// Layout shared by the host driver and the stage-one kernel (ptmg_eval.cu).
#pragma once

#include <cstddef>
#include <cstdint>

#include "pml_device.cuh"

namespace nebula {
namespace device {

// One marginal-likelihood evaluation at [beta, sigma, phi]; alpha, lambda
// and gamma are the host's Terms of (sigma, phi).
struct alignas(16) PtmgRequest {
  int32_t gene;
  int32_t pad;
  double alpha, lambda, gamma;
  double beta[kMaxCoef];
};

// Per request the kernel writes (2 + ptmg_width_of(n_coef)) * n_subjects
// doubles: cumsumxtb (K), ylin (K), then K rows of the pass-two sums.
int ptmg_width_of(int n_coef);
// Scratch doubles per CTA, and CTAs per SM, for n_coef columns of which
// n_varying vary within subjects (GeneData.n_varying).
size_t ptmg_scratch_doubles(int n_subjects, int n_coef, int n_varying);
int ptmg_blocks_per_sm(int n_subjects, int n_coef, int n_varying);

// Streaming mode for stage one: the request-ring protocol of FitQueue
// (pml_device.cuh) with PtmgRequests and results of result_stride doubles
// each in host-mapped memory; one CTA per request, `grid` CTAs each owning
// its row of `scratch`.
struct PtmgQueue {
  const PtmgRequest* ring;
  const long long* seq;
  const int* stop;
  unsigned long long* taken;
  double* results;
  long long result_stride;
  long long* done;
  int* status;
  long long mask;
  long long idle_ns;
};

int launch_ptmg_queue(const GeneData& d, const PtmgQueue& queue, double* scratch, int grid, void* stream);

}  // namespace device
}  // namespace nebula
