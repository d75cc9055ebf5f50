// ORACLE — test infrastructure only. The summation trees the CPU oracle shares
// with the CUDA kernels, restated on the CPU: tree_sums for stage one's cell
// passes (ptmg_eval.cu), range_sums for the inner fit's sweep (pml_fit.cu).
#pragma once

#include <algorithm>
#include <cstddef>
#include <vector>

#include "pml_cpu.hpp"

namespace oracle {

// The summation tree of stage one's per-subject sums, so that the oracle and
// the CUDA kernel agree bit for bit. Dense part: the cells
// are cut into `warps` equal contiguous ranges, as many as the kernel's CTA has
// warps (stage_one_warps); within a range each subject
// piece is summed by kLanes strided partial sums (lane l takes cells
// c0 + l, c0 + l + kLanes, ...), which are then combined by the butterfly
// v[l] += v[l ^ off] for off = 16, 8, 4, 2, 1 (lane 0's value is kept).
// Sparse part: each subject's positive entries the same way. A subject's total
// is 0 + its dense pieces in range order + its sparse piece.
constexpr int kLanes = 32;

// Warps of the stage-one kernel's CTA (ptmg_warps, ptmg_device.cuh): 16 for
// designs of at most 4 columns with at most one varying within subjects,
// else 8.
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

inline size_t warp_start(const PmlData& d, int w, int warps) {
  return d.n_cells * static_cast<size_t>(w) / static_cast<size_t>(warps);
}

inline int subject_of(const PmlData& d, size_t c) {
  int s = 0;
  while (d.subject_start[s + 1] <= c) ++s;
  return s;
}

// Runs `cell(lane_acc, r, s)` over every cell (dense) and `pos(lane_acc, i, s)`
// over every positive entry (sparse) through the tree; returns per-subject
// totals, K x nv.
template <typename Dense, typename Sparse>
std::vector<double> tree_sums(const PmlData& d, const std::vector<size_t>& run, int nv, int warps, Dense cell,
                              Sparse pos) {
  const int k = d.k;
  std::vector<double> dense(static_cast<size_t>(k + warps) * nv, 0.0), sparse(static_cast<size_t>(k) * nv, 0.0);
  Tree tree(nv);
  for (int w = 0; w < warps; ++w) {
    const size_t c_begin = warp_start(d, w, warps), c_end = warp_start(d, w + 1, warps);
    if (c_begin >= c_end) continue;
    int s = subject_of(d, c_begin);
    for (size_t c0 = c_begin; c0 < c_end; ++s) {
      const size_t s_end = std::min<size_t>(c_end, d.subject_start[s + 1]);
      tree.clear();
      for (int l = 0; l < kLanes; ++l)
        for (size_t r = c0 + l; r < s_end; r += kLanes) cell(tree.lane(l), r, s);
      tree.reduce(&dense[static_cast<size_t>(s + w) * nv]);
      c0 = s_end;
    }
  }
  for (int s = 0; s < k; ++s) {
    tree.clear();
    for (int l = 0; l < kLanes; ++l)
      for (size_t i = run[s] + l; i < run[s + 1]; i += kLanes) pos(tree.lane(l), i, s);
    tree.reduce(&sparse[static_cast<size_t>(s) * nv]);
  }
  std::vector<double> total(static_cast<size_t>(k) * nv);
  for (int s = 0; s < k; ++s) {
    for (int v = 0; v < nv; ++v) {
      double t = 0.0;
      for (int w = 0; w < warps; ++w)
        if (warp_start(d, w, warps) < d.subject_start[s + 1] && warp_start(d, w + 1, warps) > d.subject_start[s])
          t += dense[static_cast<size_t>(s + w) * nv + v];
      t += sparse[static_cast<size_t>(s) * nv + v];
      total[static_cast<size_t>(s) * nv + v] = t;
    }
  }
  return total;
}

// The fit kernel's tree (pml_fit.cu). The cells are cut into kRanges equal
// contiguous ranges (range v = [N v / kRanges, N (v + 1) / kRanges)). Within a
// range, each subject segment is summed by kLanes strided partials, first
// over the segment's cells (dense: lane l takes cells c0 + l, c0 + l + kLanes,
// ...) and then, continuing the same partials, over the positive entries
// whose cells fall in the segment (sparse: lane l takes entries p0 + l,
// p0 + l + kLanes, ...); the partials are butterflied as above into the
// segment's piece. A subject's total is 0 + the pieces of the non-empty
// ranges that meet it, in range order. The tree does not depend on how many
// warps or CTAs share the ranges. With zero-count tables (d.zeros) the dense
// part visits only the segment's loose cells, lane l taking loose entries
// q0 + l, q0 + l + kLanes, ... (the tabled groups are added per subject by
// the caller).
constexpr int kRanges = 64;

inline size_t range_start(const PmlData& d, int v) { return d.n_cells * static_cast<size_t>(v) / kRanges; }

template <typename Dense, typename Sparse>
std::vector<double> range_sums(const PmlData& d, int nv, Dense cell, Sparse pos) {
  const int k = d.k;
  std::vector<double> pieces(static_cast<size_t>(k + kRanges) * nv, 0.0);
  Tree tree(nv);
  auto first_entry = [&](size_t c) {
    return static_cast<size_t>(std::lower_bound(d.cells, d.cells + d.n_pos, c,
                                                [](uint32_t x, size_t v) { return x < v; }) -
                               d.cells);
  };
  for (int v = 0; v < kRanges; ++v) {
    const size_t a = range_start(d, v), b = range_start(d, v + 1);
    if (a >= b) continue;
    int s = subject_of(d, a);
    size_t pa = first_entry(a);
    for (size_t c0 = a; c0 < b; ++s) {
      const size_t s_end = std::min<size_t>(b, d.subject_start[s + 1]);
      const size_t p_end = first_entry(s_end);
      tree.clear();
      if (d.zeros) {
        const std::vector<uint32_t>& loose = d.zeros->loose;
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
      for (int v = 0; v < kRanges; ++v) {
        const size_t a = range_start(d, v), b = range_start(d, v + 1);
        if (a < b && a < d.subject_start[s + 1] && b > d.subject_start[s])
          t += pieces[static_cast<size_t>(s + v) * nv + x];
      }
      total[static_cast<size_t>(s) * nv + x] = t;
    }
  }
  return total;
}

}  // namespace oracle
