// Stage one: the Poisson-gamma marginal likelihood over [beta, sigma, phi]
// and its projected-Newton minimiser, then the plan for stage two.
//
// Follows src/sc/ptmg.rs (Terms 288-348, gamma_terms 404-474,
// linear_predictor 661-708, Subjects 712-761, gradient_parts 796-850,
// finish_gradient 865-880, evaluate 898-973, evaluate_hessian 999-1251,
// hessian_subject 1310-1440) and src/sc/nebula.rs (plan_gene 812-901,
// minimise_marginal 1075-1112, descend_marginal 1132-1170, bound_restart
// 1190-1202, newton_marginal 1225-1325, cholesky_solve 2077-2095,
// design_cv ptmg.rs:1888-1944).
//
// Dense designs only: the reference switches categorical designs to
// zero-count tables and L-BFGS-B (nebula.rs:1141-1169); here every design
// takes the exact-Hessian projected Newton, and a Newton search that fails
// keeps its start, as descend_marginal does when L-BFGS-B fails too.
#include <algorithm>
#include <cmath>
#include <limits>

#include "common.hpp"
#include "special.hpp"
#include "stage_one.hpp"

namespace nebula {
namespace {

constexpr double kBetaBound = 100.0;             // nebula.rs:68
constexpr double kHighOrderCountCutoff = 3.0;    // nebula.rs:81
constexpr int kHighOrder = 3;                    // nebula.rs:84
constexpr double kKappaFloor = 20.0;             // nebula.rs:96
constexpr double kKappaSigmaNumerator = 8.0;     // nebula.rs:99
constexpr double kFtolAbs = 1e-6;                // nebula.rs:127
constexpr double kPgtol = 1e-7;                  // nebula.rs:130
constexpr int kNewtonMaxIter = 50;               // nebula.rs:134
constexpr double kArmijo = 1e-4;                 // nebula.rs:137
constexpr int kMaxHalvings = 40;                 // nebula.rs:140
constexpr double kShift = 1e-8;                  // nebula.rs:145
constexpr int kRestarts = 3;                     // nebula.rs:153
constexpr double kRestartGain = 1e-6;            // nebula.rs:161
constexpr int kUnrolled = 8;                     // pml.rs:1165

struct Terms {  // ptmg.rs:288-348
  double exps_s, alpha, lambda, gamma, log_lambda, log_gamma, alpha_pr, lambda_pr, alpha_dpr,
      lambda_dpr;
  Terms(double sigma, double phi) {
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
};

enum class Order { Value, Gradient, Hessian };

struct GammaTerms {
  double subject_value = 0, subject_digamma = 0, subject_trigamma = 0;
  double cell_value = 0, cell_digamma = 0, cell_trigamma = 0;
};

GammaTerms gamma_terms(const PtmgGene& g, double alpha, double gamma, Order order) {
  GammaTerms out;
  double n_positive = 0, ln_sum = 0, di_sum = 0, tri_sum = 0;
  for (int s = 0; s < g.k; ++s) {
    double total = g.subject_totals[s];
    if (total > 0.0) {
      n_positive += 1.0;
      ln_sum += ln_gamma(total + alpha);
      if (order != Order::Value) di_sum += digamma(total + alpha);
      if (order == Order::Hessian) tri_sum += trigamma(total + alpha);
    }
  }
  out.subject_value = ln_sum - n_positive * ln_gamma(alpha);
  if (order != Order::Value) out.subject_digamma = di_sum - n_positive * digamma(alpha);
  if (order == Order::Hessian) out.subject_trigamma = tri_sum - n_positive * trigamma(alpha);
  double n_one = 0, n_two = 0, n_big = 0, ln_big = 0, di_big = 0, tri_big = 0;
  for (size_t i = 0; i < g.n_pos; ++i) {
    double y = g.counts[i];
    if (y == 1.0) {
      n_one += 1.0;
    } else if (y == 2.0) {
      n_two += 1.0;
    } else {
      n_big += 1.0;
      ln_big += ln_gamma(y + gamma);
      if (order != Order::Value) di_big += digamma(y + gamma);
      if (order == Order::Hessian) tri_big += trigamma(y + gamma);
    }
  }
  double n_small = n_one + n_two;
  out.cell_value = ln_big - n_big * ln_gamma(gamma) + n_small * std::log(gamma) +
                   n_two * std::log(gamma + 1.0);
  if (order != Order::Value)
    out.cell_digamma = di_big - n_big * digamma(gamma) + n_small / gamma + n_two / (gamma + 1.0);
  if (order == Order::Hessian)
    out.cell_trigamma = tri_big - n_big * trigamma(gamma) - n_small / (gamma * gamma) -
                        n_two / ((gamma + 1.0) * (gamma + 1.0));
  return out;
}

// exp(eta) per cell and its subject sums; returns sum y*eta (ptmg.rs:661-708).
double linear_predictor(PtmgGene& g, const double* beta) {
  const int nb = g.nb;
  const bool wide = nb > kUnrolled;
  double total = 0.0;
  for (int s = 0; s < g.k; ++s) {
    double csx = 0.0;
    for (size_t i = g.fid[s]; i < g.fid[s + 1]; ++i) {
      const double* row = g.design + i * nb;
      double eta;
      if (wide) {
        double xb = 0.0;
        for (int j = 0; j < nb; ++j) xb += row[j] * beta[j];
        eta = g.log_offset[i] + xb;
      } else {
        eta = g.log_offset[i];
        for (int j = 0; j < nb; ++j) eta += row[j] * beta[j];
      }
      double y = g.y_cell[i];
      if (y != 0.0) total += eta * y;
      double e = std::exp(eta);
      g.extb[i] = e;
      csx += e;
    }
    g.cumsumxtb[s] = csx;
  }
  return total;
}

struct Subjects {  // ptmg.rs:712-761
  std::vector<double> mustar_log, ymustar, ymumustar, imustar;
  Subjects(const PtmgGene& g, const Terms& t, double* total) {
    const int k = g.k;
    mustar_log.resize(k);
    ymustar.resize(k);
    ymumustar.resize(k);
    imustar.resize(k);
    for (int s = 0; s < k; ++s) {
      double ystar = g.subject_totals[s] + t.alpha;
      double mu = g.cumsumxtb[s] + t.lambda;
      double log_mu = std::log(mu);
      mustar_log[s] = log_mu;
      ymustar[s] = ystar / mu;
      ymumustar[s] = ystar / mu / mu;
      imustar[s] = 1.0 / mu;
      *total -= ystar * log_mu;
    }
    *total += static_cast<double>(k) * t.alpha * t.log_lambda;
    *total += static_cast<double>(g.n_cells) * t.gamma * t.log_gamma;
  }
};

struct GradientParts {
  std::vector<double> gradient, ymm_d, hbl0;
  double dbim = 0, sum_ymm_d = 0;
};

GradientParts gradient_parts(const PtmgGene& g, const Terms& t, const Subjects& sub,
                             const std::vector<double>& xexb_f, const std::vector<double>& dbeta_41,
                             const std::vector<double>& d42c, double slpey, double gstar_sum) {
  const int nb = g.nb, k = g.k;
  const double n_cells = static_cast<double>(g.n_cells);
  GradientParts p;
  p.ymm_d.resize(k);
  for (int s = 0; s < k; ++s) p.ymm_d[s] = sub.ymumustar[s] * d42c[s];
  p.gradient.assign(nb + 2, 0.0);
  for (int j = 0; j < nb; ++j) {
    double acc = 0.0;
    for (int s = 0; s < k; ++s) acc += xexb_f[s * nb + j] * p.ymm_d[s] - dbeta_41[s * nb + j] * sub.ymustar[s];
    p.gradient[j] = acc;
  }
  for (size_t i = 0; i < g.n_pos; ++i) {
    const double* row = g.design + static_cast<size_t>(g.cells[i]) * nb;
    for (int j = 0; j < nb; ++j) p.gradient[j] += row[j] * g.counts[i];
  }
  double sum_log_mu = 0.0, sum_ym = 0.0;
  for (int s = 0; s < k; ++s) sum_log_mu += sub.mustar_log[s];
  for (int s = 0; s < k; ++s) sum_ym += sub.ymustar[s];
  double ldm = t.log_lambda * static_cast<double>(k) - sum_log_mu;
  double adlmy = t.exps_s * static_cast<double>(k) - sum_ym;
  p.hbl0.resize(k);
  for (int s = 0; s < k; ++s) p.hbl0[s] = d42c[s] * sub.imustar[s];
  for (int s = 0; s < k; ++s) p.dbim += p.hbl0[s];
  for (int s = 0; s < k; ++s) p.sum_ymm_d += p.ymm_d[s];
  p.gradient[nb] = -t.alpha_pr * p.dbim + t.lambda_pr * p.sum_ymm_d + t.alpha_pr * ldm + t.lambda_pr * adlmy;
  p.gradient[nb + 1] = t.log_gamma * n_cells + n_cells - slpey - gstar_sum;
  return p;
}

}  // namespace

PtmgGene::PtmgGene(const Shared& sh, const GeneCounts& gc, const double* totals)
    : design(sh.design.data()), log_offset(sh.log_offset.data()), fid(sh.fid.data()),
      n_cells(sh.n_cells), nb(sh.n_coef), k(sh.n_subjects), counts(gc.counts.data()),
      cells(gc.cells.data()), n_pos(gc.counts.size()), subject_totals(totals),
      y_cell(sh.n_cells, 0.0), extb(sh.n_cells, 0.0), cumsumxtb(sh.n_subjects, 0.0) {
  for (size_t i = 0; i < n_pos; ++i) y_cell[cells[i]] = counts[i];
}

// Value and gradient in one pass (evaluate, ptmg.rs:898-973).
double ptmg_value_gradient(PtmgGene& g, const double* params, double* grad_out) {
  const int nb = g.nb, k = g.k;
  Terms t(params[nb], params[nb + 1]);
  const double gamma = t.gamma;
  double total = linear_predictor(g, params);
  Subjects sub(g, t, &total);
  std::vector<double> xexb_f(static_cast<size_t>(k) * nb, 0.0), dbeta_41(static_cast<size_t>(k) * nb, 0.0),
      d42c(k, 0.0);
  double slpey = 0.0, gstar_sum = 0.0;
  for (int s = 0; s < k; ++s) {
    double ym = sub.ymustar[s];
    double acc = 0.0;
    double* xf = &xexb_f[static_cast<size_t>(s) * nb];
    double* d41 = &dbeta_41[static_cast<size_t>(s) * nb];
    for (size_t i = g.fid[s]; i < g.fid[s + 1]; ++i) {
      double e = g.extb[i];
      double we = ym * e;
      double w = we + gamma;
      double log_w = std::log(w);
      double inv_w = 1.0 / w;
      total += we;
      total -= (gamma + g.y_cell[i]) * log_w;
      slpey += log_w;
      double gg = (gamma + g.y_cell[i]) * inv_w;
      gstar_sum += gg;
      const double* row = g.design + i * nb;
      for (int j = 0; j < nb; ++j) {
        double v = row[j] * e;
        xf[j] += v;
        d41[j] += gg * v;
      }
      acc += gg * e;
    }
    d42c[s] = acc - g.cumsumxtb[s];
  }
  GradientParts parts = gradient_parts(g, t, sub, xexb_f, dbeta_41, d42c, slpey, gstar_sum);
  // finish_gradient (ptmg.rs:865-880)
  for (auto& v : parts.gradient) v = -v;
  GammaTerms extra = gamma_terms(g, t.alpha, t.gamma, Order::Gradient);
  double value = -total - extra.subject_value - extra.cell_value;
  parts.gradient[nb] -= t.alpha_pr * extra.subject_digamma;
  parts.gradient[nb + 1] -= extra.cell_digamma;
  for (int j = 0; j < nb + 2; ++j) grad_out[j] = parts.gradient[j];
  return value;
}

// Value, gradient and Hessian in one pass (evaluate_hessian, ptmg.rs:999-1251).
double ptmg_value_gradient_hessian(PtmgGene& g, const double* params, double* grad_out,
                                   double* hess_out) {
  const int nb = g.nb, k = g.k, nn = nb * nb, np = nb + 2;
  Terms t(params[nb], params[nb + 1]);
  const double gamma = t.gamma;
  double total = linear_predictor(g, params);
  Subjects sub(g, t, &total);
  const bool wide = nb > kUnrolled;
  const size_t kb = static_cast<size_t>(k) * nb;
  std::vector<double> xexb_f(kb, 0.0), dbeta_41(kb, 0.0), tmp1_f(kb, 0.0), tmp2_f(kb, 0.0);
  std::vector<double> block_plain(wide ? 0 : static_cast<size_t>(k) * nn, 0.0);
  std::vector<double> block_g(block_plain.size(), 0.0), block_gte(block_plain.size(), 0.0);
  std::vector<double> cell_terms(wide ? 2 * g.n_cells : 0, 0.0);
  std::vector<double> hb2_f(k, 0.0), b2f(k, 0.0), d42c(k, 0.0);
  double slpey = 0, gstar_sum = 0, sum_tempa = 0, sum_gt = 0;
  for (int s = 0; s < k; ++s) {
    double ym = sub.ymustar[s];
    double acc = 0, hb2 = 0, b2 = 0;
    double* xf = &xexb_f[static_cast<size_t>(s) * nb];
    double* d41 = &dbeta_41[static_cast<size_t>(s) * nb];
    double* t1 = &tmp1_f[static_cast<size_t>(s) * nb];
    double* t2 = &tmp2_f[static_cast<size_t>(s) * nb];
    double* bp = wide ? nullptr : &block_plain[static_cast<size_t>(s) * nn];
    double* bg = wide ? nullptr : &block_g[static_cast<size_t>(s) * nn];
    double* bgte = wide ? nullptr : &block_gte[static_cast<size_t>(s) * nn];
    for (size_t i = g.fid[s]; i < g.fid[s + 1]; ++i) {
      double e = g.extb[i];
      double y = g.y_cell[i];
      double we = ym * e;
      double w = we + gamma;
      double log_w = std::log(w);
      double inv_w = 1.0 / w;
      total += we;
      total -= (gamma + y) * log_w;
      slpey += log_w;
      double gg = (gamma + y) * inv_w;
      gstar_sum += gg;
      double gt = gg * inv_w;
      double gte = gt * e;
      sum_tempa += inv_w;
      sum_gt += gt;
      acc += gg * e;
      hb2 += gte - e * inv_w;
      b2 += gte * e;
      double f1 = gt - inv_w;
      const double* row = g.design + i * nb;
      if (wide) {
        cell_terms[2 * i] = gg * e;
        cell_terms[2 * i + 1] = gte * e;
      }
      for (int a = 0; a < nb; ++a) {
        double xe = row[a] * e;
        xf[a] += xe;
        d41[a] += gg * xe;
        t1[a] += xe * f1;
        t2[a] += xe * gte;
        if (!wide) {
          for (int b = a; b < nb; ++b) {
            double c = xe * row[b];
            bp[a * nb + b] += c;
            bg[a * nb + b] += c * gg;
            bgte[a * nb + b] += c * gte;
          }
        }
      }
    }
    hb2_f[s] = hb2;
    b2f[s] = b2;
    d42c[s] = acc - g.cumsumxtb[s];
  }
  GradientParts parts = gradient_parts(g, t, sub, xexb_f, dbeta_41, d42c, slpey, gstar_sum);
  double value = -total;
  std::vector<double>& gradient = parts.gradient;
  for (auto& v : gradient) v = -v;
  const auto& ymustar = sub.ymustar;
  const auto& ymumustar = sub.ymumustar;
  const auto& imustar = sub.imustar;
  const auto& ymm_d = parts.ymm_d;
  const auto& hbl0 = parts.hbl0;
  std::vector<double> hessian(static_cast<size_t>(np) * np, 0.0);
  double lam_ratio = t.lambda_pr / t.lambda;
  double hes_sigma = (t.alpha_dpr * t.log_lambda + 2.0 * t.alpha_pr * lam_ratio - t.alpha * lam_ratio * lam_ratio +
                      t.alpha / t.lambda * t.lambda_dpr) *
                     static_cast<double>(k);
  double sum_hbl0_imu = 0, sum_ymmd_imu = 0;
  for (int s = 0; s < k; ++s) sum_hbl0_imu += hbl0[s] * imustar[s];
  for (int s = 0; s < k; ++s) sum_ymmd_imu += ymm_d[s] * imustar[s];
  hes_sigma -= parts.dbim * t.alpha_dpr - 2.0 * t.alpha_pr * t.lambda_pr * sum_hbl0_imu -
               t.lambda_dpr * parts.sum_ymm_d + 2.0 * t.lambda_pr * t.lambda_pr * sum_ymmd_imu;
  double s_imu = 0, s_mlog = 0, s_ym = 0, s_ymm = 0;
  for (int s = 0; s < k; ++s) s_imu += imustar[s];
  for (int s = 0; s < k; ++s) s_mlog += sub.mustar_log[s];
  for (int s = 0; s < k; ++s) s_ym += ymustar[s];
  for (int s = 0; s < k; ++s) s_ymm += ymumustar[s];
  hes_sigma -= 2.0 * t.alpha_pr * t.lambda_pr * s_imu + t.alpha_dpr * s_mlog + t.lambda_dpr * s_ym -
               t.lambda_pr * t.lambda_pr * s_ymm;
  std::vector<double> hes_sigma_beta(nb, 0.0);
  for (int j = 0; j < nb; ++j) {
    double d41_imu = 0, d41_ymm = 0, xf_hbl_imu = 0, xf_hbl_ymm = 0;
    for (int s = 0; s < k; ++s) {
      d41_imu += dbeta_41[s * nb + j] * imustar[s];
      d41_ymm += dbeta_41[s * nb + j] * ymumustar[s];
      xf_hbl_imu += xexb_f[s * nb + j] * hbl0[s] * imustar[s];
      xf_hbl_ymm += xexb_f[s * nb + j] * hbl0[s] * ymumustar[s];
    }
    hes_sigma_beta[j] = -t.alpha_pr * d41_imu + t.lambda_pr * d41_ymm -
                        (-t.alpha_pr * xf_hbl_imu + 2.0 * t.lambda_pr * xf_hbl_ymm);
  }
  std::vector<double> apm(k);
  for (int s = 0; s < k; ++s) apm[s] = t.alpha_pr * imustar[s] - t.lambda_pr * ymumustar[s];
  double hes_gamma = static_cast<double>(g.n_cells) / gamma - 2.0 * sum_tempa + sum_gt;
  std::vector<double> hes_gamma_beta(nb, 0.0);
  for (int j = 0; j < nb; ++j) {
    double a = 0, b = 0;
    for (int s = 0; s < k; ++s) {
      a += tmp1_f[s * nb + j] * ymustar[s];
      b += xexb_f[s * nb + j] * hb2_f[s] * ymumustar[s];
    }
    hes_gamma_beta[j] = a - b;
  }
  double hes_sigma_gamma = 0;
  for (int s = 0; s < k; ++s) hes_sigma_gamma += apm[s] * hb2_f[s];
  for (int j = 0; j < nb; ++j) {
    double a = 0, b = 0;
    for (int s = 0; s < k; ++s) {
      a += tmp2_f[s * nb + j] * apm[s] * ymustar[s];
      b += xexb_f[s * nb + j] * apm[s] * b2f[s] * ymumustar[s];
    }
    hes_sigma_beta[j] += a - b;
  }
  {
    double acc = 0;
    for (int s = 0; s < k; ++s) acc += b2f[s] * apm[s] * apm[s];
    hes_sigma += acc;
  }
  std::vector<double> ymu2(k), ymuymuimu(k), b2f_scaled(k), ymmd_imu(k);
  for (int s = 0; s < k; ++s) {
    ymu2[s] = ymustar[s] * ymustar[s];
    ymuymuimu[s] = ymu2[s] * imustar[s];
    b2f_scaled[s] = b2f[s] * ymuymuimu[s] * imustar[s];
    ymmd_imu[s] = ymm_d[s] * imustar[s];
  }
  std::vector<double> gram;
  if (wide) {  // the three blocks folded into one X' diag(w) X
    gram.assign(static_cast<size_t>(nb) * nb, 0.0);
    for (int s = 0; s < k; ++s) {
      double ym = ymustar[s];
      for (size_t i = g.fid[s]; i < g.fid[s + 1]; ++i) {
        double wt = g.extb[i] * ymm_d[s] - ym * cell_terms[2 * i] + ym * ym * cell_terms[2 * i + 1];
        const double* row = g.design + i * nb;
        for (int p = 0; p < nb; ++p)
          for (int q = p; q < nb; ++q) gram[p * nb + q] += wt * row[p] * row[q];
      }
    }
  }
  for (int p = 0; p < nb; ++p) {
    for (int q = p; q < nb; ++q) {
      double acc = 0.0;
      if (wide) {
        acc += gram[p * nb + q];
      } else {
        for (int s = 0; s < k; ++s) {
          size_t at = static_cast<size_t>(s) * nn + p * nb + q;
          acc -= block_g[at] * ymustar[s];
          acc += block_gte[at] * ymu2[s];
          acc += ymm_d[s] * block_plain[at];
        }
      }
      for (int s = 0; s < k; ++s) {
        double xf_p = xexb_f[s * nb + p], xf_q = xexb_f[s * nb + q];
        acc += (dbeta_41[s * nb + p] * xf_q + dbeta_41[s * nb + q] * xf_p) * ymumustar[s];
        acc -= ymuymuimu[s] * (tmp2_f[s * nb + p] * xf_q + tmp2_f[s * nb + q] * xf_p);
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
  GammaTerms extra = gamma_terms(g, t.alpha, gamma, Order::Hessian);
  value = value - extra.subject_value - extra.cell_value;
  gradient[nb] -= t.alpha_pr * extra.subject_digamma;
  gradient[nb + 1] -= extra.cell_digamma;
  hessian[nb * np + nb] -= t.alpha_dpr * extra.subject_digamma + t.alpha_pr * t.alpha_pr * extra.subject_trigamma;
  hessian[(nb + 1) * np + nb + 1] -= extra.cell_trigamma;
  for (int j = 0; j < np; ++j) grad_out[j] = gradient[j];
  for (int j = 0; j < np * np; ++j) hess_out[j] = hessian[j];
  return value;
}

// Lower Cholesky that also rejects an infinite pivot (nebula.rs:2077-2095,
// linalg.rs:30-75).
bool cholesky_solve(const std::vector<double>& a, int n, const std::vector<double>& b,
                    std::vector<double>* x) {
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

namespace {

bool all_finite(double f, const std::vector<double>& g, const std::vector<double>& h) {
  if (!std::isfinite(f)) return false;
  for (double v : g)
    if (!std::isfinite(v)) return false;
  for (double v : h)
    if (!std::isfinite(v)) return false;
  return true;
}

// Projected Newton inside the box (nebula.rs:1225-1325). False on a stall.
bool newton_marginal(PtmgGene& gene, const std::vector<double>& x0, const std::vector<double>& lower,
                     const std::vector<double>& upper, std::vector<double>* x_out, double* f_out) {
  const int n = static_cast<int>(x0.size());
  std::vector<double> x = x0, g(n), h(static_cast<size_t>(n) * n);
  double f = ptmg_value_gradient_hessian(gene, x.data(), g.data(), h.data());
  if (!all_finite(f, g, h)) return false;
  const bool speculative = gene.nb <= kUnrolled;
  std::vector<double> gt(n), ht(static_cast<size_t>(n) * n);
  for (int it = 0; it < kNewtonMaxIter; ++it) {
    double projected = 0.0;
    for (int i = 0; i < n; ++i)
      projected = std::fmax(projected, std::fabs(std::clamp(x[i] - g[i], lower[i], upper[i]) - x[i]));
    if (projected < kPgtol) {
      *x_out = x;
      *f_out = f;
      return true;
    }
    std::vector<int> free;
    for (int i = 0; i < n; ++i)
      if (!((x[i] <= lower[i] && g[i] > 0.0) || (x[i] >= upper[i] && g[i] < 0.0))) free.push_back(i);
    const int m = static_cast<int>(free.size());
    std::vector<double> rhs(m);
    for (int p = 0; p < m; ++p) rhs[p] = -g[free[p]];
    double largest = 0.0;
    for (int i : free) largest = std::fmax(largest, std::fabs(h[i * n + i]));
    double shift = 0.0;
    std::vector<double> step_free;
    for (;;) {
      std::vector<double> block(static_cast<size_t>(m) * m, 0.0);
      for (int p = 0; p < m; ++p) {
        for (int q = 0; q < m; ++q) block[p * m + q] = h[free[p] * n + free[q]];
        block[p * m + p] += shift;
      }
      if (cholesky_solve(block, m, rhs, &step_free)) break;
      shift = shift == 0.0 ? kShift * std::fmax(largest, 1.0) : shift * 10.0;
      if (!std::isfinite(shift)) return false;
    }
    std::vector<double> d(n, 0.0);
    for (int p = 0; p < m; ++p) d[free[p]] = step_free[p];
    double alpha = 1.0;
    bool accepted = false, have_derivs = false;
    std::vector<double> xt(n);
    double ft = 0.0;
    for (int hv = 0; hv < kMaxHalvings; ++hv) {
      for (int i = 0; i < n; ++i) xt[i] = std::clamp(x[i] + alpha * d[i], lower[i], upper[i]);
      double decrease = 0.0;
      for (int i = 0; i < n; ++i) decrease += g[i] * (xt[i] - x[i]);
      bool ok;
      if (speculative) {
        ft = ptmg_value_gradient_hessian(gene, xt.data(), gt.data(), ht.data());
        ok = all_finite(ft, gt, ht);
        have_derivs = ok;
      } else {
        ft = ptmg_value_gradient(gene, xt.data(), gt.data());
        ok = std::isfinite(ft);
        have_derivs = false;
      }
      if (ok && ft <= f + kArmijo * decrease) {
        accepted = true;
        break;
      }
      alpha *= 0.5;
    }
    if (!accepted) return false;
    if ((f - ft) <= kFtolAbs) {
      *x_out = xt;
      *f_out = ft;
      return true;
    }
    if (!have_derivs) {
      ft = ptmg_value_gradient_hessian(gene, xt.data(), gt.data(), ht.data());
      if (!all_finite(ft, gt, ht)) return false;
    }
    x = xt;
    f = ft;
    g = gt;
    h = ht;
  }
  return false;
}

void descend_marginal(PtmgGene& gene, const std::vector<double>& x0, double f0,
                      const std::vector<double>& lower, const std::vector<double>& upper,
                      std::vector<double>* x_out, double* f_out) {
  std::vector<double> x;
  double f;
  if (newton_marginal(gene, x0, lower, upper, &x, &f) && f < f0) {
    *x_out = x;
    *f_out = f;
    return;
  }
  *x_out = x0;
  *f_out = f0;
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

// minimise_marginal (nebula.rs:1075-1112): the best point and whether every
// attempt failed.
std::vector<double> minimise_marginal(PtmgGene& gene, const std::vector<double>& start,
                                      const std::vector<double>& lower,
                                      const std::vector<double>& upper, bool* failed) {
  const size_t n = start.size();
  std::vector<double> x0(n), grad(n);
  for (size_t j = 0; j < n; ++j) x0[j] = std::clamp(start[j], lower[j], upper[j]);
  double f0 = ptmg_value_gradient(gene, x0.data(), grad.data());
  if (!std::isfinite(f0)) {
    *failed = true;
    return x0;
  }
  std::vector<double> best;
  double best_f;
  descend_marginal(gene, x0, f0, lower, upper, &best, &best_f);
  std::vector<double> last = best, anchor = x0;
  for (int r = 0; r < kRestarts; ++r) {
    std::vector<double> x1;
    if (!bound_restart(last, anchor, lower, upper, &x1)) break;
    double f1 = ptmg_value_gradient(gene, x1.data(), grad.data());
    if (!std::isfinite(f1)) break;
    std::vector<double> x;
    double f;
    descend_marginal(gene, x1, f1, lower, upper, &x, &f);
    if (f < best_f - kRestartGain) {
      best = x;
      best_f = f;
    }
    last = x;
    anchor = x1;
  }
  *failed = false;
  return best;
}

// plan_gene (nebula.rs:812-901).
GenePlan plan_gene(const Shared& sh, const GeneCounts& gc, const double* totals) {
  const int nc = sh.n_coef;
  const Params& p = sh.params;
  GenePlan plan;
  plan.ord = gc.mean_count * sh.cells_per_subject < kHighOrderCountCutoff ? kHighOrder : 1;
  PtmgGene gene(sh, gc, totals);
  double log_mean_count = std::log(gc.mean_count);
  std::vector<double> start(nc + 2, 0.0), lower(nc + 2, -kBetaBound), upper(nc + 2, kBetaBound);
  start[sh.intercept] = log_mean_count - sh.log_mean_offset;
  start[nc] = 1.0;
  start[nc + 1] = 1.0;
  lower[nc] = p.min0;
  lower[nc + 1] = p.min1;
  upper[nc] = p.max0;
  upper[nc + 1] = p.max1;
  bool failed = false;
  std::vector<double> x = minimise_marginal(gene, start, lower, upper, &failed);
  plan.convergence = failed ? 0 : kConvSuccess;
  plan.sigma = x[nc];
  plan.gamma = x[nc + 1];
  plan.beta_start.assign(nc, 0.0);
  plan.beta_start[sh.intercept] = log_mean_count - sh.log_mean_offset;
  if (sh.method == NB_METHOD_HL) {
    plan.refit = Refit::Both;
  } else {
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
  }
  return plan;
}

}  // namespace nebula
