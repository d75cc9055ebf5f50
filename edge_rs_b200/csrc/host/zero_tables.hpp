// Zero-count tables for a run (the reference's ZeroCells, src/sc/zeros.rs):
// the cells of each subject are grouped by their design row, every group of at
// least kMinGroupCells cells gets the piecewise Chebyshev tables of
// zero_group.hpp, and the rest are loose cells a sweep visits one by one.
// When fewer than half of the cells would be tabled (a continuous cell-level
// column leaves one cell per group), there are no tables and every sweep visits
// every cell (zeros.rs:219-282).
//
// The construction follows zeros.rs:284-445: each base panel of width 4 in
// s = ln(tau) is halved (up to six times) until the last two Chebyshev
// coefficients of all six forms are below 1e-14 plus 32 ulps of the form's
// size; the coefficients come from the values at the 17 Chebyshev-Lobatto
// nodes, and the sums at a node are compensated (Neumaier) sums over the
// group's distinct offsets. It runs once per call on the host, and the FP64
// CPU oracle builds its tables with this same code, so both evaluate the same
// coefficients.
#pragma once

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <thread>
#include <utility>
#include <vector>

#include "zero_group.hpp"

namespace nebula {
namespace zero {

constexpr double kNoiseUlps = 32.0;
constexpr int kMaxDepth = 6;
constexpr double kPanelTol = 1e-14;
constexpr double kTailDepth = 40.0;
constexpr size_t kMinGroupCells = 32;
constexpr double kMinTabledShare = 0.5;

struct Tables {
  std::vector<Group> groups;             // subject by subject, by first cell within a subject
  std::vector<uint32_t> subject_groups;  // n_subjects + 1 into groups
  std::vector<uint32_t> loose;           // cells in no tabled group, ascending
  std::vector<uint32_t> subject_loose;   // n_subjects + 1 into loose
  std::vector<uint32_t> index;           // per base panel: first panel, depth
  std::vector<double> panels;            // kPanelDoubles per panel
};

namespace detail {

struct Compensated {  // Neumaier's summation
  double sum = 0.0, carry = 0.0;
  void add(double x) {
    const double t = sum + x;
    if (std::fabs(sum) >= std::fabs(x)) carry += (sum - t) + x;
    else carry += (x - t) + sum;
    sum = t;
  }
  double total() const { return sum + carry; }
};

// The six sums at s over the group's distinct ln O with their multiplicities.
inline void direct_sums(const std::vector<std::pair<double, double>>& distinct, double s, double* out) {
  Compensated acc[kForms];
  for (const auto& [l, m] : distinct) {
    const double v = std::exp(s + l);
    const double w = 1.0 / (1.0 + v);
    const double u = v * w;
    const double uw = u * w;
    acc[0].add(m * std::log1p(v));
    acc[1].add(m * u);
    acc[2].add(m * uw);
    acc[3].add(m * (uw * (w - u)));
    acc[4].add(m * (uw * (w * w - 4.0 * u * w + u * u)));
    acc[5].add(m * (uw * (w * w * w - 11.0 * w * w * u + 11.0 * w * u * u - u * u * u)));
  }
  for (int f = 0; f < kForms; ++f) out[f] = acc[f].total();
}

// Chebyshev coefficients from the values at the Lobatto nodes cos(pi j / N).
inline void chebyshev(const double* values, double* c) {
  const double n = kDegree;
  const double pi = 3.14159265358979323846;
  for (int k = 0; k <= kDegree; ++k) {
    double acc = 0.0;
    for (int j = 0; j <= kDegree; ++j) {
      const double weight = (j == 0 || j == kDegree) ? 0.5 : 1.0;
      acc += weight * values[j] * std::cos(pi * static_cast<double>(j * k) / n);
    }
    c[k] = 2.0 * acc / n;
  }
  c[0] *= 0.5;
  c[kDegree] *= 0.5;
}

// One panel's coefficients (kPanelDoubles) and whether every form converged.
inline bool fit_panel(const std::vector<std::pair<double, double>>& distinct, double left, double width,
                      double* panel) {
  double values[kForms][kPoints];
  const double pi = 3.14159265358979323846;
  for (int j = 0; j < kPoints; ++j) {
    const double x = std::cos(pi * static_cast<double>(j) / kDegree);
    double sums[kForms];
    direct_sums(distinct, left + 0.5 * width * (x + 1.0), sums);
    for (int f = 0; f < 3; ++f) values[f][j] = std::log(sums[f]);
    for (int f = 3; f < kForms; ++f) values[f][j] = sums[f] / sums[2];
  }
  bool ok = true;
  for (int f = 0; f < kForms; ++f) {
    double* c = panel + f * kPoints;
    chebyshev(values[f], c);
    double size = 0.0;
    for (int j = 0; j < kPoints; ++j) size = std::max(size, std::fabs(values[f][j]));
    const double tail = std::fabs(c[kDegree - 1]) + std::fabs(c[kDegree]);
    ok = ok && tail <= kPanelTol + kNoiseUlps * 2.220446049250313e-16 * size;
  }
  return ok;
}

// Sorts 64-bit keys (least significant 16-bit digit first; a pass whose
// digit is the same in every key is skipped). The table bound only needs
// equal keys next to each other; a comparison sort of 100,000 keys took
// 5 ms of a call.
inline void radix_sort(std::vector<uint64_t>& keys, std::vector<uint64_t>& tmp) {
  const size_t n = keys.size();
  if (n < 2) return;
  tmp.resize(n);
  std::vector<size_t> count(size_t{1} << 16);
  for (int shift = 0; shift < 64; shift += 16) {
    std::fill(count.begin(), count.end(), 0);
    for (uint64_t k : keys) ++count[(k >> shift) & 0xffff];
    if (count[(keys[0] >> shift) & 0xffff] == n) continue;
    size_t sum = 0;
    for (size_t& c : count) {
      const size_t t = c;
      c = sum;
      sum += t;
    }
    for (uint64_t k : keys) tmp[count[(k >> shift) & 0xffff]++] = k;
    keys.swap(tmp);
  }
}

// One group's sums and panels; its base panels' (first, depth) entries use
// panel numbers local to the group (0, 1, ...).
struct Built {
  Group group{};
  std::vector<uint32_t> index;
  std::vector<double> panels;
};

inline Built build_group(int64_t row, std::vector<double> log_o) {
  Built b;
  std::sort(log_o.begin(), log_o.end());
  std::vector<std::pair<double, double>> distinct;
  for (double l : log_o) {
    if (!distinct.empty() && distinct.back().first == l) distinct.back().second += 1.0;
    else distinct.emplace_back(l, 1.0);
  }
  Group& g = b.group;
  g.row = row;
  g.n = static_cast<double>(log_o.size());
  g.s_lo = -kTailDepth - log_o.back();
  g.s_hi = kTailDepth - log_o.front();
  g.n_base = static_cast<int32_t>(std::ceil((g.s_hi - g.s_lo) / kBaseWidth));
  Compensated so, sio, slo;
  for (double l : log_o) {
    so.add(std::exp(l));
    sio.add(std::exp(-l));
    slo.add(l);
  }
  g.sum_o = so.total();
  g.sum_inv_o = sio.total();
  g.sum_log_o = slo.total();
  std::vector<double> trial;
  for (int base = 0; base < g.n_base; ++base) {
    const double left = g.s_lo + static_cast<double>(base) * kBaseWidth;
    int depth = 0;
    for (;; ++depth) {
      const int parts = 1 << depth;
      const double width = kBaseWidth / parts;
      trial.assign(static_cast<size_t>(parts) * kPanelDoubles, 0.0);
      bool ok = true;
      for (int p = 0; p < parts; ++p)
        ok = fit_panel(distinct, left + p * width, width, &trial[static_cast<size_t>(p) * kPanelDoubles]) && ok;
      if (ok || depth == kMaxDepth) break;
    }
    b.index.push_back(static_cast<uint32_t>(b.panels.size() / kPanelDoubles));
    b.index.push_back(static_cast<uint32_t>(depth));
    b.panels.insert(b.panels.end(), trial.begin(), trial.end());
  }
  return b;
}

}  // namespace detail

// Groups the cells and tabulates every group large enough; false (and no
// tables) when under kMinTabledShare of the cells would be covered. fid holds
// the n_subjects + 1 subject boundaries of the row-major n_cells x n_coef
// design; threads 0 = all hardware threads.
inline bool build_tables(const double* design, const double* log_offset, const uint64_t* fid, int n_subjects,
                         int n_coef, Tables* out, int threads = 0) {
  const size_t n_cells = static_cast<size_t>(fid[n_subjects]);
  // A cell can sit in a tabled group only if its value in every column occurs
  // at least kMinGroupCells times; counting the values of the columns that
  // vary within some subject bounds the tabled cells from above, and a
  // continuous column ends the build here without grouping the rows.
  {
    std::vector<uint64_t> bits(n_cells), tmp;
    for (int j = 0; j < n_coef; ++j) {
      bool varies = false;
      for (int s = 0; s < n_subjects && !varies; ++s)
        for (uint64_t r = fid[s] + 1; r < fid[s + 1] && !varies; ++r)
          varies = std::memcmp(&design[r * n_coef + j], &design[fid[s] * n_coef + j], sizeof(double)) != 0;
      if (!varies) continue;
      for (size_t r = 0; r < n_cells; ++r) std::memcpy(&bits[r], &design[r * n_coef + j], sizeof(double));
      detail::radix_sort(bits, tmp);
      size_t coverable = 0;
      for (size_t a = 0, b; a < n_cells; a = b) {
        for (b = a + 1; b < n_cells && bits[b] == bits[a];) ++b;
        if (b - a >= kMinGroupCells) coverable += b - a;
      }
      if (static_cast<double>(coverable) < kMinTabledShare * static_cast<double>(n_cells)) return false;
    }
  }
  std::vector<std::vector<uint32_t>> members;  // tabled groups, subject by subject
  Tables t;
  t.subject_groups.assign(static_cast<size_t>(n_subjects) + 1, 0);
  t.subject_loose.assign(static_cast<size_t>(n_subjects) + 1, 0);
  size_t tabled = 0;
  for (int s = 0; s < n_subjects; ++s) {
    std::map<std::vector<uint64_t>, std::vector<uint32_t>> by_row;
    std::vector<uint64_t> key(static_cast<size_t>(n_coef));
    for (uint64_t r = fid[s]; r < fid[s + 1]; ++r) {
      for (int j = 0; j < n_coef; ++j) std::memcpy(&key[j], &design[r * n_coef + j], sizeof(double));
      by_row[key].push_back(static_cast<uint32_t>(r));
    }
    std::vector<std::vector<uint32_t>> kept;
    std::vector<uint32_t> loose;
    for (auto& [k, cells] : by_row) {
      if (cells.size() >= kMinGroupCells) {
        tabled += cells.size();
        kept.push_back(std::move(cells));
      } else {
        loose.insert(loose.end(), cells.begin(), cells.end());
      }
    }
    std::sort(kept.begin(), kept.end(), [](const auto& a, const auto& b) { return a[0] < b[0]; });
    for (auto& c : kept) members.push_back(std::move(c));
    t.subject_groups[s + 1] = static_cast<uint32_t>(members.size());
    std::sort(loose.begin(), loose.end());
    t.loose.insert(t.loose.end(), loose.begin(), loose.end());
    t.subject_loose[s + 1] = static_cast<uint32_t>(t.loose.size());
  }
  if (static_cast<double>(tabled) < kMinTabledShare * static_cast<double>(n_cells)) return false;

  std::vector<detail::Built> built(members.size());
  std::atomic<size_t> next{0};
  auto work = [&]() {
    for (size_t i; (i = next.fetch_add(1)) < members.size();) {
      std::vector<double> logs;
      logs.reserve(members[i].size());
      for (uint32_t r : members[i]) logs.push_back(log_offset[r]);
      built[i] = detail::build_group(members[i][0], std::move(logs));
    }
  };
  int nt = threads > 0 ? threads : static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
  nt = std::max(1, std::min<int>(nt, static_cast<int>(members.size())));
  std::vector<std::thread> pool;
  for (int i = 1; i < nt; ++i) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();

  for (detail::Built& b : built) {
    const uint32_t panel0 = static_cast<uint32_t>(t.panels.size() / kPanelDoubles);
    b.group.index = static_cast<int32_t>(t.index.size() / 2);
    for (size_t i = 0; i < b.index.size(); i += 2) {
      t.index.push_back(panel0 + b.index[i]);
      t.index.push_back(b.index[i + 1]);
    }
    t.panels.insert(t.panels.end(), b.panels.begin(), b.panels.end());
    t.groups.push_back(b.group);
  }
  *out = std::move(t);
  return true;
}

}  // namespace zero
}  // namespace nebula
