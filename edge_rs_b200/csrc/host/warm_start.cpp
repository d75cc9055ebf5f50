// Features of the warm-start network and its built-in parameters.
#include "warm_start.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "export.hpp"

namespace nebula {

void warm_features(const Shared& sh, const GeneCounts& gc, const double* subject_totals, const GenePlan& plan,
                   float* out) {
  const double n = static_cast<double>(sh.n_cells);
  const int k = sh.n_subjects;
  double s1 = 0.0, s2 = 0.0, top = 0.0;
  for (double y : gc.counts) {
    s1 += y;
    s2 += y * y;
    top = std::max(top, y);
  }
  const double nnz = static_cast<double>(gc.counts.size());
  const double mean = s1 / n;
  const double var = std::max(s2 / n - mean * mean, 0.0);
  double lm = 0.0, lm2 = 0.0;
  for (int s = 0; s < k; ++s) {
    const double cells = static_cast<double>(sh.fid[s + 1] - sh.fid[s]);
    const double v = std::log((subject_totals[s] + 0.5) / cells);
    lm += v;
    lm2 += v * v;
  }
  lm /= k;
  lm2 = std::max(lm2 / k - lm * lm, 0.0);
  const double f[mlp::kIn] = {std::log(mean + 1e-12),
                              std::log(var + 1e-12),
                              1.0 - nnz / n,
                              std::log(std::max(plan.sigma, 1e-12)),
                              std::log(std::max(plan.gamma, 1e-12)),
                              std::log1p(top),
                              nnz > 0 ? static_cast<double>(gc.n_one) / nnz : 0.0,
                              lm2,
                              std::log(n / k),
                              std::log(static_cast<double>(k)),
                              static_cast<double>(plan.ord),
                              nnz > 0 ? std::log(s1 / nnz) : 0.0};
  for (int i = 0; i < mlp::kIn; ++i) out[i] = static_cast<float>(f[i]);
}

const float* builtin_mlp_params() {
  static const float kParams[mlp::kParams] = {
#include "warm_start_weights.inc"
  };
  return kParams;
}

}  // namespace nebula

// The built-in network's parameters (NB_MLP_PARAMS floats).
NB_API void nb_mlp_builtin(float* params) {
  std::memcpy(params, nebula::builtin_mlp_params(), sizeof(float) * nebula::mlp::kParams);
}
