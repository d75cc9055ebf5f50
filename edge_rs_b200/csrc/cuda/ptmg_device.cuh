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

// Warps of a stage-one CTA, and so the ranges of its summation tree (the
// cells cut into this many equal contiguous ranges, warp_cells): 16 (one
// 512-thread CTA per SM) for designs of at most 4 columns with at most one
// varying within subjects, whose per-thread state fits in 128 registers;
// otherwise 8 (256 threads), where a thread needs up to 224. An SM holds 16
// or 8 warps either way, but with 16 in one CTA each request is served by
// twice the warps, so a gene's chain of Newton points runs about twice as
// fast; stage one is bound by its longest chain.
constexpr int ptmg_warps(int n_coef, int n_varying) { return n_coef <= 4 && n_varying <= 1 ? 16 : 8; }
constexpr int kMaxPtmgWarps = 16;

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
  RingView ring;
  double* results;
  long long result_stride;
  long long* done;
};

int launch_ptmg_queue(const GeneData& d, const PtmgQueue& queue, double* scratch, int grid, void* stream);

}  // namespace device
}  // namespace nebula
