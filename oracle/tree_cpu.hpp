// ORACLE — test infrastructure only. The summation trees the CPU oracle shares
// with the CUDA kernels, restated on the CPU: tree_sums for stage one's cell
// passes (ptmg_eval.cu), range_sums for the inner fit's sweep (pml_fit.cu).
#pragma once

#include <algorithm>
#include <cstddef>
#include <vector>

#include "pml_cpu.hpp"

namespace oracle {

// Warps of the stage-one kernel's request (ptmg_warps, ptmg_device.cuh): 16
// for designs of at most 4 columns with at most one varying within subjects,
// else 8.
constexpr int kLanes = 32;
inline int stage_one_warps(int n_beta, int n_varying) { return n_beta <= 4 && n_varying <= 1 ? 16 : 8; }

struct Tree {
  int nv;
  std::vector<double> lanes, next;  // kLanes x nv each
  explicit Tree(int n) : nv(n), lanes(static_cast<size_t>(kLanes) * n, 0.0), next(lanes.size()) {}
  double* lane(int l) { return &lanes[static_cast<size_t>(l) * nv]; }
  void clear() { std::fill(lanes.begin(), lanes.end(), 0.0); }
  void reduce(double* out) {
    for (int off = 16; off > 0; off >>= 1) {
      for (int l = 0; l < kLanes; ++l) {
        const double* a = &lanes[static_cast<size_t>(l) * nv];
        const double* b = &lanes[static_cast<size_t>(l ^ off) * nv];
        double* o = &next[static_cast<size_t>(l) * nv];
        for (int v = 0; v < nv; ++v) o[v] = a[v] + b[v];
      }
      lanes.swap(next);
    }
    for (int v = 0; v < nv; ++v) out[v] = lanes[v];
  }
};

inline int subject_of(const PmlData& d, size_t c) {
  int s = 0;
  while (d.subject_start[s + 1] <= c) ++s;
  return s;
}

// The segment tree both kernels sum in. The cells are cut into `ranges`
// equal contiguous ranges (range v = [N v / ranges, N (v + 1) / ranges)).
// Within a range, each subject segment is summed by kLanes strided partials,
// first over the segment's cells (dense: lane l takes cells c0 + l,
// c0 + l + kLanes, ...) and then, continuing the same partials, over the
// positive entries whose cells fall in the segment (sparse: lane l takes
// entries p0 + l, p0 + l + kLanes, ...); the partials are combined by the
// butterfly v[l] += v[l ^ off] for off = 16, 8, 4, 2, 1 into the segment's
// piece (lane 0's value). A subject's total is 0 + the pieces of the
// non-empty ranges that meet it, in range order. With zero-count tables
// (`zeros`, the fit's sweeps only) the dense part visits only the segment's
// loose cells, lane l taking loose entries q0 + l, q0 + l + kLanes, ... (the
// tabled groups are added per subject by the caller). Returns per-subject
// totals, K x nv.
template <typename Dense, typename Sparse>
std::vector<double> segment_sums(const PmlData& d, int ranges, const nebula::zero::Tables* zeros, int nv,
                                 Dense cell, Sparse pos) {
  const int k = d.k;
  auto start = [&](int v) { return d.n_cells * static_cast<size_t>(v) / static_cast<size_t>(ranges); };
  std::vector<double> pieces(static_cast<size_t>(k + ranges) * nv, 0.0);
  Tree tree(nv);
  auto first_entry = [&](size_t c) {
    return static_cast<size_t>(std::lower_bound(d.cells, d.cells + d.n_pos, c,
                                                [](uint32_t x, size_t v) { return x < v; }) -
                               d.cells);
  };
  for (int v = 0; v < ranges; ++v) {
    const size_t a = start(v), b = start(v + 1);
    if (a >= b) continue;
    int s = subject_of(d, a);
    size_t pa = first_entry(a);
    for (size_t c0 = a; c0 < b; ++s) {
      const size_t s_end = std::min<size_t>(b, d.subject_start[s + 1]);
      const size_t p_end = first_entry(s_end);
      tree.clear();
      if (zeros) {
        const std::vector<uint32_t>& loose = zeros->loose;
        const size_t q0 = static_cast<size_t>(std::lower_bound(loose.begin(), loose.end(), c0) - loose.begin());
        const size_t q1 = static_cast<size_t>(std::lower_bound(loose.begin(), loose.end(), s_end) - loose.begin());
        for (int l = 0; l < kLanes; ++l)
          for (size_t q = q0 + l; q < q1; q += kLanes) cell(tree.lane(l), loose[q], s);
      } else {
        for (int l = 0; l < kLanes; ++l)
          for (size_t r = c0 + l; r < s_end; r += kLanes) cell(tree.lane(l), r, s);
      }
      for (int l = 0; l < kLanes; ++l)
        for (size_t i = pa + l; i < p_end; i += kLanes) pos(tree.lane(l), i, s);
      tree.reduce(&pieces[static_cast<size_t>(s + v) * nv]);
      pa = p_end;
      c0 = s_end;
    }
  }
  std::vector<double> total(static_cast<size_t>(k) * nv);
  for (int s = 0; s < k; ++s) {
    for (int x = 0; x < nv; ++x) {
      double t = 0.0;
      for (int v = 0; v < ranges; ++v) {
        const size_t a = start(v), b = start(v + 1);
        if (a < b && a < d.subject_start[s + 1] && b > d.subject_start[s])
          t += pieces[static_cast<size_t>(s + v) * nv + x];
      }
      total[static_cast<size_t>(s) * nv + x] = t;
    }
  }
  return total;
}

// Stage one's per-subject sums (ptmg_eval.cu): the segment tree over as many
// ranges as the kernel's request has warps (stage_one_warps), every cell swept.
template <typename Dense, typename Sparse>
std::vector<double> tree_sums(const PmlData& d, int nv, int warps, Dense cell, Sparse pos) {
  return segment_sums(d, warps, nullptr, nv, cell, pos);
}

// The fit kernel's tree (pml_fit.cu): the segment tree over kRanges ranges,
// with the run's zero-count tables where it has them. The tree does not
// depend on how many warps or CTAs share the ranges.
constexpr int kRanges = 64;

template <typename Dense, typename Sparse>
std::vector<double> range_sums(const PmlData& d, int nv, Dense cell, Sparse pos) {
  return segment_sums(d, kRanges, d.zeros, nv, cell, pos);
}

}  // namespace oracle
