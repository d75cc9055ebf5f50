// Stage one, shared by the device driver and the CPU oracle: assembly of the
// marginal likelihood from per-subject sums, the projected-Newton minimiser as
// a coroutine, and the stage-two plan.
//
// Follows src/sc/ptmg.rs (Terms 288-348, gamma_terms 404-474, Subjects
// 712-761, gradient_parts 796-850, finish_gradient 865-880, the Hessian
// assembly 1123-1250) and src/sc/nebula.rs (plan_gene 812-901,
// minimise_marginal 1075-1112, descend_marginal 1132-1170, bound_restart
// 1190-1202, newton_marginal 1225-1325, cholesky_solve 2077-2095,
// design_cv ptmg.rs:1888-1944).
//
// Two departures, both in how the reference's quantities are summed, not in
// what they are: the per-cell sums are split into a dense part at a count of
// zero plus what the positive counts add (every per-cell term is affine in
// the count), and the reference's three x x' e blocks enter the Hessian only
// as bp ymm_d - bg ym + bgte ym^2 per subject, so the cell pass sums
// x x' e and x x' e ym (ym g e/w - g) directly. A descent is the reference's:
// the exact-Hessian projected Newton on a dense run, L-BFGS-B (lbfgsb.hpp)
// where the run is tabled or the Newton stalls or does not improve, and the
// start kept when that fails too (nebula.rs:1132-1170). Its value and
// gradient come from the dense sums even on a tabled run, where the
// reference reads its zero-count tables; the two agree to rounding.
#include "stage_one.hpp"

#include <algorithm>
#include <cmath>
#include <limits>

#include "lbfgsb.hpp"
#include "special.hpp"

namespace nebula {
namespace {

constexpr double kBetaBound = 100.0;           // nebula.rs:68
constexpr double kHighOrderCountCutoff = 3.0;  // nebula.rs:81
constexpr int kHighOrder = 3;                  // nebula.rs:84
constexpr double kKappaFloor = 20.0;           // nebula.rs:96
constexpr double kKappaSigmaNumerator = 8.0;   // nebula.rs:99
constexpr double kFtolAbs = 1e-6;              // nebula.rs:127
constexpr double kPgtol = 1e-7;                // nebula.rs:130
constexpr int kNewtonMaxIter = 50;             // nebula.rs:134
constexpr double kArmijo = 1e-4;               // nebula.rs:137
constexpr int kMaxHalvings = 40;               // nebula.rs:140
constexpr double kShift = 1e-8;                // nebula.rs:145
constexpr int kRestarts = 3;                   // nebula.rs:153
constexpr double kRestartGain = 1e-6;          // nebula.rs:161
constexpr int kLbfgsbMaxIter = 300;            // nebula.rs:164
constexpr int kLbfgsbMaxLineSearch = 40;       // nebula.rs:167
constexpr int kUnrolled = 8;                   // pml.rs:1165

struct GammaTerms {
  double subject_value = 0, subject_digamma = 0, subject_trigamma = 0;
  double cell_value = 0, cell_digamma = 0, cell_trigamma = 0;
};

// gamma_terms at Hessian order (ptmg.rs:404-474).
GammaTerms gamma_terms(const MarginalGene& g, double alpha, double gamma) {
  GammaTerms out;
  const int k = g.sh->n_subjects;
  double n_positive = 0, ln_sum = 0, di_sum = 0, tri_sum = 0;
  for (int s = 0; s < k; ++s) {
    double total = g.totals[s];
    if (total > 0.0) {
      n_positive += 1.0;
      ln_sum += ln_gamma(total + alpha);
      di_sum += digamma(total + alpha);
      tri_sum += trigamma(total + alpha);
    }
  }
  out.subject_value = ln_sum - n_positive * ln_gamma(alpha);
  out.subject_digamma = di_sum - n_positive * digamma(alpha);
  out.subject_trigamma = tri_sum - n_positive * trigamma(alpha);
  // one term per distinct count (the reference walks every count, ptmg.rs:443-458)
  const double n_one = static_cast<double>(g.gc->n_one), n_two = static_cast<double>(g.gc->n_two);
  double n_big = 0, ln_big = 0, di_big = 0, tri_big = 0;
  for (size_t i = 0; i < g.gc->big_values.size(); ++i) {
    const double y = g.gc->big_values[i], m = g.gc->big_mult[i];
    n_big += m;
    ln_big += m * ln_gamma(y + gamma);
    di_big += m * digamma(y + gamma);
    tri_big += m * trigamma(y + gamma);
  }
  double n_small = n_one + n_two;
  out.cell_value = ln_big - n_big * ln_gamma(gamma) + n_small * std::log(gamma) + n_two * std::log(gamma + 1.0);
  out.cell_digamma = di_big - n_big * digamma(gamma) + n_small / gamma + n_two / (gamma + 1.0);
  out.cell_trigamma = tri_big - n_big * trigamma(gamma) - n_small / (gamma * gamma) -
                      n_two / ((gamma + 1.0) * (gamma + 1.0));
  return out;
}

bool all_finite(double f, const std::vector<double>& g, const std::vector<double>& h) {
  if (!std::isfinite(f)) return false;
  for (double v : g)
    if (!std::isfinite(v)) return false;
  for (double v : h)
    if (!std::isfinite(v)) return false;
  return true;
}

bool bound_restart(const std::vector<double>& best, const std::vector<double>& start,
                   const std::vector<double>& lower, const std::vector<double>& upper,
                   std::vector<double>* out) {
  *out = best;
  bool moved = false;
  for (size_t j = 0; j < best.size(); ++j) {
    for (double bound : {lower[j], upper[j]}) {
      if (best[j] == bound && start[j] != bound && bound * start[j] > 0.0) {
        (*out)[j] = std::sqrt(bound * start[j]);
        moved = true;
      }
    }
  }
  return moved;
}

}  // namespace

Terms::Terms(double sigma, double phi) {
  double exps = std::exp(sigma);
  double exps_m1 = exps - 1.0;
  exps_s = std::sqrt(exps);
  alpha = 1.0 / exps_m1;
  lambda = alpha / exps_s;
  double exps_sq = exps_m1 * exps_m1;
  gamma = phi;
  log_lambda = std::log(lambda);
  log_gamma = std::log(phi);
  alpha_pr = -exps / exps_sq;
  lambda_pr = (1.0 - 3.0 * exps) / (2.0 * exps_s * exps_sq);
  alpha_dpr = 2.0 * exps * exps / (exps_sq * exps_m1) - exps / exps_sq;
  lambda_dpr = -3.0 * exps / (2.0 * exps_s * exps_sq) + (3.0 * exps - 1.0) / (4.0 * exps_s * exps_sq) +
               (3.0 * exps - 1.0) * exps_s / (exps_sq * exps_m1);
}

double ptmg_assemble(const MarginalGene& g, const double* params, const PtmgSums& S, double* grad_out,
                     double* hess_out) {
  const Shared& sh = *g.sh;
  const int nb = sh.n_coef, k = sh.n_subjects, np = nb + 2, W = ptmg_width(nb), T = nb * (nb + 1) / 2;
  const Terms t(params[nb], params[nb + 1]);
  const double gamma = t.gamma;
  auto at = [&](int s, int v) { return S.sums[static_cast<size_t>(s) * W + v]; };
  const int o_xf = kPtmgScalars, o_d41 = o_xf + nb, o_t1 = o_d41 + nb, o_t2 = o_t1 + nb, o_bp = o_t2 + nb,
            o_bq = o_bp + T;

  // the linear-predictor part (ptmg.rs:661-708)
  double total = 0.0;
  for (int s = 0; s < k; ++s) total += S.ylin[s];
  // Subjects::new (ptmg.rs:739-760)
  std::vector<double> mustar_log(k), ymustar(k), ymumustar(k), imustar(k);
  for (int s = 0; s < k; ++s) {
    double ystar = g.totals[s] + t.alpha;
    double mu = S.cumsumxtb[s] + t.lambda;
    double log_mu = std::log(mu);
    mustar_log[s] = log_mu;
    ymustar[s] = ystar / mu;
    ymumustar[s] = ystar / mu / mu;
    imustar[s] = 1.0 / mu;
    total -= ystar * log_mu;
  }
  total += static_cast<double>(k) * t.alpha * t.log_lambda;
  total += static_cast<double>(sh.n_cells) * t.gamma * t.log_gamma;
  // the cell pass (ptmg.rs:926-966, 1381-1428), per subject
  double slpey = 0, gstar_sum = 0, sum_tempa = 0, sum_gt = 0;
  std::vector<double> d42c(k), hb2_f(k), b2f(k);
  for (int s = 0; s < k; ++s) {
    total += at(s, 0);
    total -= at(s, 2);
    slpey += at(s, 1);
    gstar_sum += at(s, 3);
    sum_tempa += at(s, 4);
    sum_gt += at(s, 5);
    d42c[s] = at(s, 6) - S.cumsumxtb[s];
    hb2_f[s] = at(s, 7);
    b2f[s] = at(s, 8);
  }
  // gradient_parts (ptmg.rs:796-850)
  const double n_cells = static_cast<double>(sh.n_cells);
  std::vector<double> ymm_d(k), gradient(np, 0.0);
  for (int s = 0; s < k; ++s) ymm_d[s] = ymumustar[s] * d42c[s];
  for (int j = 0; j < nb; ++j) {
    double acc = 0.0;
    for (int s = 0; s < k; ++s) acc += at(s, o_xf + j) * ymm_d[s] - at(s, o_d41 + j) * ymustar[s];
    gradient[j] = acc;
  }
  for (int j = 0; j < nb; ++j) gradient[j] += g.xy[j];
  double sum_log_mu = 0.0, sum_ym = 0.0;
  for (int s = 0; s < k; ++s) sum_log_mu += mustar_log[s];
  for (int s = 0; s < k; ++s) sum_ym += ymustar[s];
  double ldm = t.log_lambda * static_cast<double>(k) - sum_log_mu;
  double adlmy = t.exps_s * static_cast<double>(k) - sum_ym;
  std::vector<double> hbl0(k);
  for (int s = 0; s < k; ++s) hbl0[s] = d42c[s] * imustar[s];
  double dbim = 0.0, sum_ymm_d = 0.0;
  for (int s = 0; s < k; ++s) dbim += hbl0[s];
  for (int s = 0; s < k; ++s) sum_ymm_d += ymm_d[s];
  gradient[nb] = -t.alpha_pr * dbim + t.lambda_pr * sum_ymm_d + t.alpha_pr * ldm + t.lambda_pr * adlmy;
  gradient[nb + 1] = t.log_gamma * n_cells + n_cells - slpey - gstar_sum;
  double value = -total;
  for (auto& v : gradient) v = -v;

  // Hessian in log-likelihood sign (ptmg.rs:1123-1240)
  std::vector<double> hessian(static_cast<size_t>(np) * np, 0.0);
  double lam_ratio = t.lambda_pr / t.lambda;
  double hes_sigma = (t.alpha_dpr * t.log_lambda + 2.0 * t.alpha_pr * lam_ratio - t.alpha * lam_ratio * lam_ratio +
                      t.alpha / t.lambda * t.lambda_dpr) *
                     static_cast<double>(k);
  double sum_hbl0_imu = 0, sum_ymmd_imu = 0;
  for (int s = 0; s < k; ++s) sum_hbl0_imu += hbl0[s] * imustar[s];
  for (int s = 0; s < k; ++s) sum_ymmd_imu += ymm_d[s] * imustar[s];
  hes_sigma -= dbim * t.alpha_dpr - 2.0 * t.alpha_pr * t.lambda_pr * sum_hbl0_imu - t.lambda_dpr * sum_ymm_d +
               2.0 * t.lambda_pr * t.lambda_pr * sum_ymmd_imu;
  double s_imu = 0, s_mlog = 0, s_ym = 0, s_ymm = 0;
  for (int s = 0; s < k; ++s) s_imu += imustar[s];
  for (int s = 0; s < k; ++s) s_mlog += mustar_log[s];
  for (int s = 0; s < k; ++s) s_ym += ymustar[s];
  for (int s = 0; s < k; ++s) s_ymm += ymumustar[s];
  hes_sigma -= 2.0 * t.alpha_pr * t.lambda_pr * s_imu + t.alpha_dpr * s_mlog + t.lambda_dpr * s_ym -
               t.lambda_pr * t.lambda_pr * s_ymm;
  std::vector<double> hes_sigma_beta(nb, 0.0);
  for (int j = 0; j < nb; ++j) {
    double d41_imu = 0, d41_ymm = 0, xf_hbl_imu = 0, xf_hbl_ymm = 0;
    for (int s = 0; s < k; ++s) {
      d41_imu += at(s, o_d41 + j) * imustar[s];
      d41_ymm += at(s, o_d41 + j) * ymumustar[s];
      xf_hbl_imu += at(s, o_xf + j) * hbl0[s] * imustar[s];
      xf_hbl_ymm += at(s, o_xf + j) * hbl0[s] * ymumustar[s];
    }
    hes_sigma_beta[j] =
        -t.alpha_pr * d41_imu + t.lambda_pr * d41_ymm - (-t.alpha_pr * xf_hbl_imu + 2.0 * t.lambda_pr * xf_hbl_ymm);
  }
  std::vector<double> apm(k);
  for (int s = 0; s < k; ++s) apm[s] = t.alpha_pr * imustar[s] - t.lambda_pr * ymumustar[s];
  double hes_gamma = n_cells / gamma - 2.0 * sum_tempa + sum_gt;
  std::vector<double> hes_gamma_beta(nb, 0.0);
  for (int j = 0; j < nb; ++j) {
    double a = 0, b = 0;
    for (int s = 0; s < k; ++s) {
      a += at(s, o_t1 + j) * ymustar[s];
      b += at(s, o_xf + j) * hb2_f[s] * ymumustar[s];
    }
    hes_gamma_beta[j] = a - b;
  }
  double hes_sigma_gamma = 0;
  for (int s = 0; s < k; ++s) hes_sigma_gamma += apm[s] * hb2_f[s];
  for (int j = 0; j < nb; ++j) {
    double a = 0, b = 0;
    for (int s = 0; s < k; ++s) {
      a += at(s, o_t2 + j) * apm[s] * ymustar[s];
      b += at(s, o_xf + j) * apm[s] * b2f[s] * ymumustar[s];
    }
    hes_sigma_beta[j] += a - b;
  }
  {
    double acc = 0;
    for (int s = 0; s < k; ++s) acc += b2f[s] * apm[s] * apm[s];
    hes_sigma += acc;
  }
  std::vector<double> ymuymuimu(k), b2f_scaled(k), ymmd_imu(k);
  for (int s = 0; s < k; ++s) {
    ymuymuimu[s] = ymustar[s] * ymustar[s] * imustar[s];
    b2f_scaled[s] = b2f[s] * ymuymuimu[s] * imustar[s];
    ymmd_imu[s] = ymm_d[s] * imustar[s];
  }
  int tri = 0;
  for (int p = 0; p < nb; ++p) {
    for (int q = p; q < nb; ++q, ++tri) {
      double acc = 0.0;
      for (int s = 0; s < k; ++s) {
        acc += at(s, o_bq + tri);
        acc += ymm_d[s] * at(s, o_bp + tri);
      }
      for (int s = 0; s < k; ++s) {
        double xf_p = at(s, o_xf + p), xf_q = at(s, o_xf + q);
        acc += (at(s, o_d41 + p) * xf_q + at(s, o_d41 + q) * xf_p) * ymumustar[s];
        acc -= ymuymuimu[s] * (at(s, o_t2 + p) * xf_q + at(s, o_t2 + q) * xf_p);
        double cross = xf_p * xf_q;
        acc -= cross * ymumustar[s];
        acc += b2f_scaled[s] * cross;
        acc -= 2.0 * cross * ymmd_imu[s];
      }
      hessian[p * np + q] = acc;
      hessian[q * np + p] = acc;
    }
  }
  hessian[nb * np + nb] = hes_sigma;
  hessian[(nb + 1) * np + nb + 1] = hes_gamma;
  hessian[nb * np + nb + 1] = hes_sigma_gamma;
  hessian[(nb + 1) * np + nb] = hes_sigma_gamma;
  for (int j = 0; j < nb; ++j) {
    hessian[nb * np + j] = hes_sigma_beta[j];
    hessian[j * np + nb] = hes_sigma_beta[j];
    hessian[(nb + 1) * np + j] = hes_gamma_beta[j];
    hessian[j * np + nb + 1] = hes_gamma_beta[j];
  }
  for (auto& h : hessian) h = -h;
  // the gamma-function terms of R/ptmg.R (ptmg.rs:1242-1248)
  GammaTerms extra = gamma_terms(g, t.alpha, gamma);
  value = value - extra.subject_value - extra.cell_value;
  gradient[nb] -= t.alpha_pr * extra.subject_digamma;
  gradient[nb + 1] -= extra.cell_digamma;
  hessian[nb * np + nb] -= t.alpha_dpr * extra.subject_digamma + t.alpha_pr * t.alpha_pr * extra.subject_trigamma;
  hessian[(nb + 1) * np + nb + 1] -= extra.cell_trigamma;
  if (grad_out)
    for (int j = 0; j < np; ++j) grad_out[j] = gradient[j];
  if (hess_out)
    for (int j = 0; j < np * np; ++j) hess_out[j] = hessian[j];
  return value;
}

std::vector<double> positive_xy(const Shared& sh, const GeneCounts& gc) {
  const int nb = sh.n_coef;
  std::vector<double> xy(nb, 0.0);
  for (size_t i = 0; i < gc.counts.size(); ++i) {
    const double* row = &sh.design[static_cast<size_t>(gc.cells[i]) * nb];
    for (int j = 0; j < nb; ++j) xy[j] += row[j] * gc.counts[i];
  }
  return xy;
}

bool cholesky_solve(const std::vector<double>& a, int n, const std::vector<double>& b, std::vector<double>* x) {
  std::vector<double> l = a;
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j <= i; ++j) {
      double sum = l[i * n + j];
      for (int kk = 0; kk < j; ++kk) sum -= l[i * n + kk] * l[j * n + kk];
      if (i == j) {
        if (sum <= 0.0 || std::isnan(sum)) return false;
        l[i * n + j] = std::sqrt(sum);
      } else {
        l[i * n + j] = sum / l[j * n + j];
      }
    }
  }
  for (int i = 0; i < n; ++i)
    if (!std::isfinite(l[i * n + i])) return false;
  *x = b;
  std::vector<double>& v = *x;
  for (int i = 0; i < n; ++i) {
    double sum = v[i];
    for (int kk = 0; kk < i; ++kk) sum -= l[i * n + kk] * v[kk];
    v[i] = sum / l[i * n + i];
  }
  for (int i = n - 1; i >= 0; --i) {
    double sum = v[i];
    for (int kk = i + 1; kk < n; ++kk) sum -= l[kk * n + i] * v[kk];
    v[i] = sum / l[i * n + i];
  }
  for (double e : v)
    if (!std::isfinite(e)) return false;
  return true;
}

// ---------------------------------------------------------------------------
// minimise_marginal as a coroutine (nebula.rs:1075-1325)

MarginalSearch::MarginalSearch(std::vector<double> start, std::vector<double> lower, std::vector<double> upper,
                               int nb, bool tabled)
    : start_(std::move(start)), lower_(std::move(lower)), upper_(std::move(upper)),
      n_(static_cast<int>(start_.size())), nb_(nb), tabled_(tabled) {
  g_.assign(n_, 0.0);
  h_.assign(static_cast<size_t>(n_) * n_, 0.0);
  task_ = run();
}

MarginalSearch::~MarginalSearch() {
  if (task_.h) task_.h.destroy();
}

MarginalSearch::Eval MarginalSearch::evaluate(const std::vector<double>& x) {
  x_ = x;
  waiting_ = true;
  ++evaluations_;
  return Eval{this};
}

void MarginalSearch::tell(double f, const double* g, const double* h) {
  if (!waiting_) return;
  f_ = f;
  for (int j = 0; j < n_; ++j) g_[j] = g[j];
  for (int j = 0; j < n_ * n_; ++j) h_[j] = h[j];
  waiting_ = false;
  task_.h.resume();
}

MarginalSearch::Task MarginalSearch::run() {
  const int n = n_;
  const bool speculative = nb_ <= kUnrolled;
  std::vector<double> x0(n);
  for (int j = 0; j < n; ++j) x0[j] = std::clamp(start_[j], lower_[j], upper_[j]);
  co_await evaluate(x0);
  const double f0 = f_;
  if (!std::isfinite(f0)) {
    best_ = x0;
    failed_ = true;
    co_return;
  }
  std::vector<double> xs = x0, best, last, anchor = x0, x, g, h, xt, gt, ht, d, step_free, rhs, block;
  double fs = f0, best_f = 0.0, f = 0.0, ft = 0.0;
  for (int attempt = 0; attempt <= kRestarts; ++attempt) {
    if (attempt > 0) {  // restart off a bound the previous start was inside
      std::vector<double> x1;
      if (!bound_restart(last, anchor, lower_, upper_, &x1)) break;
      co_await evaluate(x1);
      if (!std::isfinite(f_)) break;
      xs = x1;
      fs = f_;
    }
    // descend_marginal (nebula.rs:1132-1170): projected Newton from (xs, fs)
    // on a dense run (1225-1325), L-BFGS-B where that is not taken or fails
    int status = tabled_ ? 2 : 0;  // 0 running, 1 converged, 2 stalled or not run
    if (!tabled_) {
      x = xs;
      co_await evaluate(x);
      f = f_;
      g = g_;
      h = h_;
      if (!all_finite(f, g, h)) status = 2;
    }
    for (int it = 0; status == 0 && it < kNewtonMaxIter; ++it) {
      double projected = 0.0;
      for (int i = 0; i < n; ++i)
        projected = std::fmax(projected, std::fabs(std::clamp(x[i] - g[i], lower_[i], upper_[i]) - x[i]));
      if (projected < kPgtol) {
        status = 1;
        break;
      }
      std::vector<int> free;
      for (int i = 0; i < n; ++i)
        if (!((x[i] <= lower_[i] && g[i] > 0.0) || (x[i] >= upper_[i] && g[i] < 0.0))) free.push_back(i);
      const int m = static_cast<int>(free.size());
      rhs.assign(m, 0.0);
      for (int p = 0; p < m; ++p) rhs[p] = -g[free[p]];
      double largest = 0.0;
      for (int i : free) largest = std::fmax(largest, std::fabs(h[i * n + i]));
      double shift = 0.0;
      bool factored = false;
      for (;;) {
        block.assign(static_cast<size_t>(m) * m, 0.0);
        for (int p = 0; p < m; ++p) {
          for (int q = 0; q < m; ++q) block[p * m + q] = h[free[p] * n + free[q]];
          block[p * m + p] += shift;
        }
        if (cholesky_solve(block, m, rhs, &step_free)) {
          factored = true;
          break;
        }
        shift = shift == 0.0 ? kShift * std::fmax(largest, 1.0) : shift * 10.0;
        if (!std::isfinite(shift)) break;
      }
      if (!factored) {
        status = 2;
        break;
      }
      d.assign(n, 0.0);
      for (int p = 0; p < m; ++p) d[free[p]] = step_free[p];
      double alpha = 1.0;
      bool accepted = false;
      xt.assign(n, 0.0);
      for (int hv = 0; hv < kMaxHalvings; ++hv) {
        for (int i = 0; i < n; ++i) xt[i] = std::clamp(x[i] + alpha * d[i], lower_[i], upper_[i]);
        double decrease = 0.0;
        for (int i = 0; i < n; ++i) decrease += g[i] * (xt[i] - x[i]);
        co_await evaluate(xt);
        ft = f_;
        const bool ok = speculative ? all_finite(ft, g_, h_) : std::isfinite(ft);
        if (ok && ft <= f + kArmijo * decrease) {
          accepted = true;
          gt = g_;
          ht = h_;
          break;
        }
        alpha *= 0.5;
      }
      if (!accepted) {
        status = 2;
        break;
      }
      if ((f - ft) <= kFtolAbs) {
        x = xt;
        f = ft;
        status = 1;
        break;
      }
      // a wide design takes the Hessian at the accepted point only; the
      // evaluations here always carry it, so only its finiteness is new
      if (!speculative && !all_finite(ft, gt, ht)) {
        status = 2;
        break;
      }
      x = xt;
      f = ft;
      g = gt;
      h = ht;
    }
    std::vector<double> xd = xs;
    double fd = fs;
    if (status == 1 && f < fs) {
      xd = x;
      fd = f;
    } else {
      // the quasi-Newton, its ftol relative to the start's objective so that
      // its stop is nebula's absolute eps (nebula.rs:1146-1168)
      LbfgsbParams lp;
      lp.ftol = kFtolAbs / std::fmax(std::fabs(fs), 1.0);
      lp.pgtol = kPgtol;
      lp.max_iter = kLbfgsbMaxIter;
      lp.max_line_search = kLbfgsbMaxLineSearch;
      Lbfgsb quasi(xs, lower_, upper_, lp);
      std::vector<double> xq(n);
      while (const double* q = quasi.ask()) {
        xq.assign(q, q + n);
        co_await evaluate(xq);
        quasi.tell(f_, g_.data());
      }
      if (quasi.f() < fs) {
        xd = quasi.x();
        fd = quasi.f();
      }
    }
    if (attempt == 0) {
      best = xd;
      best_f = fd;
    } else if (fd < best_f - kRestartGain) {
      best = xd;
      best_f = fd;
    }
    last = xd;
    anchor = xs;
  }
  best_ = best;
  failed_ = false;
  co_return;
}

void marginal_box(const Shared& sh, const GeneCounts& gc, std::vector<double>* start, std::vector<double>* lower,
                  std::vector<double>* upper) {
  const int nc = sh.n_coef;
  const Params& p = sh.params;
  start->assign(nc + 2, 0.0);
  lower->assign(nc + 2, -kBetaBound);
  upper->assign(nc + 2, kBetaBound);
  (*start)[sh.intercept] = std::log(gc.mean_count) - sh.log_mean_offset;
  (*start)[nc] = 1.0;
  (*start)[nc + 1] = 1.0;
  (*lower)[nc] = p.min0;
  (*lower)[nc + 1] = p.min1;
  (*upper)[nc] = p.max0;
  (*upper)[nc + 1] = p.max1;
}

GenePlan plan_from(const Shared& sh, const GeneCounts& gc, const std::vector<double>& x, bool failed) {
  const int nc = sh.n_coef;
  const Params& p = sh.params;
  GenePlan plan;
  plan.ord = gc.mean_count * sh.cells_per_subject < kHighOrderCountCutoff ? kHighOrder : 1;
  plan.convergence = failed ? 0 : kConvSuccess;
  plan.sigma = x[nc];
  plan.gamma = x[nc + 1];
  plan.beta_start.assign(nc, 0.0);
  plan.beta_start[sh.intercept] = std::log(gc.mean_count) - sh.log_mean_offset;
  if (sh.method == NB_METHOD_HL) {
    plan.refit = Refit::Both;
    return plan;
  }
  double cv2p;
  if (sh.cell_columns.empty()) {
    cv2p = sh.cv2;
  } else {  // design_cv (ptmg.rs:1888-1944)
    std::vector<double> mu(sh.n_cells);
    for (size_t i = 0; i < sh.n_cells; ++i) {
      double eta = sh.log_offset[i];
      for (int c : sh.cell_columns) eta += sh.design[i * nc + c] * x[c];
      mu[i] = std::exp(eta);
    }
    double mean = 0.0;
    for (double v : mu) mean += v;
    mean /= static_cast<double>(sh.n_cells);
    if (mean <= 0.0) {
      cv2p = 0.0;
    } else {
      double ss = 0.0;
      for (double v : mu) ss += (v - mean) * (v - mean);
      cv2p = ss / static_cast<double>(sh.n_cells) / (mean * mean);
    }
  }
  double gni = sh.cells_per_subject * plan.gamma;
  if (gni < p.cutoff_cell || plan.convergence == 0 || std::isnan(cv2p)) {
    plan.refit = Refit::Both;
  } else {
    double kappa_obs = gni / (1.0 + cv2p);
    bool weak = kappa_obs < kKappaFloor || (kappa_obs < p.kappa && plan.sigma < kKappaSigmaNumerator / kappa_obs);
    plan.refit = weak ? Refit::SubjectOnly : Refit::None;
  }
  return plan;
}

}  // namespace nebula
