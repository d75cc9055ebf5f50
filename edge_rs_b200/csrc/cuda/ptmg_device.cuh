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

// Warps serving one stage-one request, and so the ranges of its summation
// tree (the cells cut into this many equal contiguous ranges, warp_cells):
// 16 for designs of at most 4 columns with at most one varying within
// subjects, whose per-thread state fits in 128 registers; otherwise 8, where
// a thread needs up to 224. The warps form a cluster of CTAs of four warps
// each on as many SMs (ptmg_impl.cuh), so one request has the FP64 pipes of
// 4 (or 2) SMs: stage one is bound by its longest gene's chain of dependent
// Newton points, and a point now takes a fraction of one SM's time.
constexpr int ptmg_warps(int n_coef, int n_varying) { return n_coef <= 4 && n_varying <= 1 ? 16 : 8; }
constexpr int kMaxPtmgWarps = 16;

// Per request the kernel writes (2 + ptmg_width_of(n_coef)) * n_subjects
// doubles: cumsumxtb (K), ylin (K), then K rows of the pass-two sums.
int ptmg_width_of(int n_coef);
// Scratch doubles per CTA (a cluster uses its first CTA's share), and the
// CTAs the stage-one kernel keeps resident at once (whole clusters of
// ptmg_warps / 4 CTAs of four warps), for n_coef columns of which n_varying
// vary within subjects (GeneData.n_varying).
size_t ptmg_scratch_doubles(int n_subjects, int n_coef, int n_varying);
int ptmg_resident_ctas(int n_subjects, int n_coef, int n_varying);

// Streaming mode for stage one: the request-ring protocol of FitQueue
// (pml_device.cuh) with PtmgRequests and results of result_stride doubles
// each in host-mapped memory; one cluster per request, `grid` CTAs (whole
// clusters), each cluster owning its first CTA's row of `scratch`.
struct PtmgQueue {
  RingView ring;
  double* results;
  long long result_stride;
  long long* done;
};

int launch_ptmg_queue(const GeneData& d, const PtmgQueue& queue, double* scratch, int grid, void* stream);

}  // namespace device
}  // namespace nebula
