// One zero-count group's table as the fit kernel and the host read it, and
// its evaluation (host and device). The tables are built by zero_tables.hpp.
//
// Within a subject, the cells that share a design row differ only in their
// offset O. At a count of zero every per-cell term a sweep sums is a function
// of v = tau * O, with tau = exp(x'beta + log_w) / gamma shared by the group.
// So each of the six sums below is a function of s = ln(tau) alone, fixed for
// the whole run, and is tabulated once (src/sc/zeros.rs:1-28):
//   L = sum ln(1 + v)           A = sum v / (1 + v)         B = sum v / (1 + v)^2
//   C = sum u w (w - u)          D = sum u w (w^2 - 4 u w + u^2)
//   E = sum u w (w^3 - 11 w^2 u + 11 w u^2 - u^3)     (w = 1/(1+v), u = v w)
// Each is a piecewise Chebyshev series of degree 16 in s; L, A and B are
// stored as logs, C, D and E as ratios to B. Outside [s_lo, s_hi] every v is
// below e^-40 or above e^40 and closed forms in the group's offset sums
// stand in (zeros.rs:146-215).
#pragma once

#include <cstdint>

#include "nbmath.hpp"

namespace nebula {
namespace zero {

constexpr int kForms = 6;
constexpr int kDegree = 16;
constexpr int kPoints = kDegree + 1;
constexpr int kPanelDoubles = kForms * kPoints;
constexpr double kBaseWidth = 4.0;

struct Group {
  double n;          // cells
  double sum_o;      // sum O, for the small-v side
  double sum_inv_o;  // sum 1/O, for the large-v side
  double sum_log_o;  // sum ln O, for the large-v side
  double s_lo, s_hi; // the tabulated range of s
  int64_t row;       // a member cell: its design row is the group's
  int32_t index;     // the group's first base panel in the index table
  int32_t n_base;    // base panels of width kBaseWidth from s_lo
};

// sum_k c_k T_k(x) by Clenshaw's recurrence.
NB_HD double clenshaw(const double* c, double x) {
  const double two_x = 2.0 * x;
  double b1 = 0.0, b2 = 0.0;
  for (int k = kDegree; k >= 1; --k) {
    const double b0 = nb_fma(two_x, b1, c[k]) - b2;
    b2 = b1;
    b1 = b0;
  }
  return nb_fma(x, b1, c[0]) - b2;
}

// m consecutive sums starting at sum `from` (0 = L ... 5 = E) at s into out;
// asking for C, D or E needs B (2) in the same call. `index` holds per base
// panel its first panel and its depth (the base panel is split into 2^depth
// equal panels); `panels` holds kPanelDoubles coefficients per panel.
NB_HD void eval(const Group& g, const uint32_t* index, const double* panels, double s, int from, int m,
                double* out) {
  if (!(s == s)) {  // NaN
    for (int j = 0; j < m; ++j) out[j] = s;
    return;
  }
  if (s < g.s_lo) {  // every sum is sum v to first order
    const double v = nb_exp(s) * g.sum_o;
    for (int j = 0; j < m; ++j) out[j] = v;
    return;
  }
  if (s > g.s_hi) {
    const double r = nb_exp(-s) * g.sum_inv_o;
    for (int j = 0; j < m; ++j) {
      const int f = from + j;
      out[j] = f == 0 ? (g.n * s + g.sum_log_o) + r : f == 1 ? g.n - r : (f == 2 || f == 4) ? r : -r;
    }
    return;
  }
  const double pos = (s - g.s_lo) / kBaseWidth;
  int base = static_cast<int>(pos);
  if (base > g.n_base - 1) base = g.n_base - 1;
  const uint32_t first = index[2 * (g.index + base)];
  const uint32_t depth = index[2 * (g.index + base) + 1];
  const double parts = static_cast<double>(1u << depth);
  double within = (pos - static_cast<double>(base)) * parts;
  if (within < 0.0) within = 0.0;
  if (within > parts - 1e-9) within = parts - 1e-9;
  const int sub = static_cast<int>(within);
  const double x = 2.0 * (within - static_cast<double>(sub)) - 1.0;
  const double* panel = panels + static_cast<size_t>(first + static_cast<uint32_t>(sub)) * kPanelDoubles;
  double b_value = 0.0;
  for (int j = 0; j < m; ++j) {
    const int f = from + j;
    const double v = clenshaw(panel + f * kPoints, x);
    out[j] = f < 3 ? nb_exp(v) : v;
    if (f == 2) b_value = out[j];
  }
  for (int j = 0; j < m; ++j)
    if (from + j >= 3) out[j] *= b_value;
}

}  // namespace zero
}  // namespace nebula
