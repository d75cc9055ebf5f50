// glm_sc_test (src/sc/test.rs:96-200): Wald test of a contrast c per gene,
// effect c'beta, variance c'Vc with the full packed covariance (A19),
// p = chisq_sf(z^2, 1), Benjamini-Hochberg FDR (src/numeric/stats.rs:40-61).
//
// chisq_sf(x, 1) = Q(1/2, x/2) = erfc(sqrt(x/2)); the reference evaluates the
// regularised upper incomplete gamma (dist.rs:162-173, 737-746), the same
// function. log p is kept in log space past erfc's underflow with the
// asymptotic series of erfc (Abramowitz and Stegun 7.1.23).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "common.hpp"
#include "export.hpp"

namespace {

double log_erfc(double x) {
  double p = std::erfc(x);
  if (p > 1e-300) return std::log(p);
  // x > ~26: erfc(x) = exp(-x^2) / (x sqrt(pi)) * (1 - 1/(2x^2) + 3/(4x^4) - 15/(8x^6) + ...)
  const double u = 1.0 / (2.0 * x * x);
  const double series = 1.0 - u * (1.0 - 3.0 * u * (1.0 - 5.0 * u * (1.0 - 7.0 * u)));
  return -x * x - std::log(x * std::sqrt(M_PI)) + std::log(series);
}

void write_err(char* err, size_t len, const std::string& msg) {
  if (!err || len == 0) return;
  size_t n = std::min(len - 1, msg.size());
  std::memcpy(err, msg.data(), n);
  err[n] = 0;
}

bool total_greater(double a, double b) {  // p[b].total_cmp(&p[a]) as an ordering
  int64_t ia, ib;
  std::memcpy(&ia, &a, 8);
  std::memcpy(&ib, &b, 8);
  ia ^= static_cast<int64_t>(static_cast<uint64_t>(ia >> 63) >> 1);
  ib ^= static_cast<int64_t>(static_cast<uint64_t>(ib >> 63) >> 1);
  return ia > ib;
}

}  // namespace

NB_API int32_t nb_glm_sc_test(const double* coefficients, const double* covariance, uint64_t n_genes,
                              uint64_t n_coef, const double* contrast, double* log_fc, double* se, double* z,
                              double* p_value, double* log_p_value, double* fdr, char* err, size_t err_len) {
  if (n_genes == 0 || n_coef == 0) {
    write_err(err, err_len, "fit dimensions must be positive");
    return NB_ERR_MUST_BE_POSITIVE;
  }
  if (!coefficients || !covariance || !contrast) {
    write_err(err, err_len, "null input");
    return NB_ERR_INVALID_ARGUMENT;
  }
  bool all_zero = true;
  for (uint64_t j = 0; j < n_coef; ++j) all_zero = all_zero && contrast[j] == 0.0;
  if (all_zero) {
    write_err(err, err_len, "contrast is entirely zero");
    return NB_ERR_INVALID_ARGUMENT;
  }
  const uint64_t packed = n_coef * (n_coef + 1) / 2;
  std::vector<double> p(n_genes);
  for (uint64_t g = 0; g < n_genes; ++g) {
    const double* beta = coefficients + g * n_coef;
    const double* cov = covariance + g * packed;
    double effect = 0.0;
    for (uint64_t j = 0; j < n_coef; ++j) effect += beta[j] * contrast[j];
    double variance = 0.0;
    for (uint64_t i = 0; i < n_coef; ++i) {
      if (contrast[i] == 0.0) continue;
      for (uint64_t j = 0; j < n_coef; ++j) {
        if (contrast[j] == 0.0) continue;
        uint64_t lo = std::min(i, j), hi = std::max(i, j);
        variance += contrast[i] * contrast[j] * cov[hi * (hi + 1) / 2 + lo];
      }
    }
    double error = variance > 0.0 ? std::sqrt(variance) : 0.0;
    double statistic = error > 0.0 ? effect / error : 0.0;
    double pv = 1.0, lp = 0.0;
    if (error > 0.0) {
      double x = std::fabs(statistic) / std::sqrt(2.0);
      double stat2 = statistic * statistic;
      if (stat2 <= 0.0) {
        pv = 1.0;
      } else if (std::isinf(stat2)) {
        pv = 0.0;
        lp = -std::numeric_limits<double>::infinity();
      } else {
        pv = std::erfc(x);
        lp = log_erfc(x);
      }
    }
    if (log_fc) log_fc[g] = effect;
    if (se) se[g] = error;
    if (z) z[g] = statistic;
    if (p_value) p_value[g] = pv;
    if (log_p_value) log_p_value[g] = lp;
    p[g] = pv;
  }
  if (fdr) {
    std::vector<size_t> order(n_genes);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return total_greater(p[a], p[b]); });
    double running = std::numeric_limits<double>::infinity();
    const double n = static_cast<double>(n_genes);
    for (size_t j = 0; j < n_genes; ++j) {
      size_t idx = order[j];
      double rank = static_cast<double>(n_genes - j);
      running = std::min(running, n / rank * p[idx]);
      fdr[idx] = std::min(running, 1.0);
    }
  }
  return NB_OK;
}
