// ORACLE — test infrastructure only (see pml_cpu.hpp). FP64 restatement of
// the reference's opt_pml, one gene at a time. Its sums follow a fixed tree
// (see tree_sums) and its exp/log are nbmath.hpp's, so that the CUDA kernel,
// which takes the same tree and the same functions, agrees with it bit for
// bit; against the R goldens the association of the sums does not matter at
// their 1e-11 tolerance.
#include "pml_cpu.hpp"

#include "nbmath.hpp"
#include "tree_cpu.hpp"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <limits>

namespace oracle {
namespace {

constexpr double kGradientTolerance = 0.01;  // pml.rs:67
constexpr double kStepCutoff = 40.0;         // pml.rs:74
constexpr double kEigenCutoff = 1e-8;        // pml.rs:80
constexpr int kJacobiSweeps = 30;            // pml.rs:86

struct Penalty {  // pml.rs:347-412
  Prior kind;
  double alpha, lambda;
  double accumulate(double ll, const std::vector<double>& log_w, const std::vector<double>& w) const {
    if (kind == Prior::Gamma) {
      double sl = 0.0, sw = 0.0;
      for (double l : log_w) sl += l;
      for (double x : w) sw += x;
      return ll + (alpha * sl - lambda * sw);
    }
    double quad = 0.0;
    for (double l : log_w) quad += l * l;
    return ll - quad / alpha / 2.0 - static_cast<double>(log_w.size()) / 2.0 * std::log(alpha);
  }
  double gradient(double log_w_s, double w_s) const {
    return kind == Prior::Gamma ? alpha - lambda * w_s : -log_w_s / alpha;
  }
  double curvature(double w_s) const { return kind == Prior::Gamma ? lambda * w_s : 1.0 / alpha; }
};

struct Sweep {  // pml.rs:1171-1210
  double ll = 0;
  std::vector<double> w, db, dw, vw, vwb, vb;
  void init(int nb, int k) {
    w.assign(k, 0);
    db.assign(nb, 0);
    dw.assign(k, 0);
    vw.assign(k, 0);
    vwb.assign(static_cast<size_t>(k) * nb, 0);
    vb.assign(static_cast<size_t>(nb) * nb, 0);
  }
};

}  // namespace

// Start of each subject's run of positive counts (pml.rs:1155-1160).
std::vector<size_t> positive_runs(const PmlData& d) {
  std::vector<size_t> run(d.k + 1);
  for (int s = 0; s <= d.k; ++s) {
    uint64_t b = d.subject_start[s];
    run[s] = static_cast<size_t>(std::lower_bound(d.cells, d.cells + d.n_pos, b,
                                                  [](uint32_t c, uint64_t v) { return c < v; }) -
                                 d.cells);
  }
  return run;
}

// The design columns that take more than one value within some subject (the
// reference's cell_level_columns, ptmg.rs:1962-2005), increasing; vpos[a] is
// column a's index among them, or -1 for a column constant within every
// subject. A sweep sums only the varying columns per cell and applies each
// constant column's share per subject.
Split split_columns(const PmlData& d) {
  Split sp;
  sp.vpos.assign(d.n_beta, -1);
  for (int j = 0; j < d.n_beta; ++j) {
    bool varies = false;
    for (int s = 0; s < d.k && !varies; ++s) {
      if (d.subject_start[s] >= d.subject_start[s + 1]) continue;
      const double first = d.design[d.subject_start[s] * d.n_beta + j];
      for (size_t r = d.subject_start[s] + 1; r < d.subject_start[s + 1] && !varies; ++r)
        varies = d.design[r * d.n_beta + j] != first;
    }
    if (varies) {
      sp.vpos[j] = static_cast<int>(sp.varying.size());
      sp.varying.push_back(j);
    }
  }
  return sp;
}

// Subject s's design row (its constant columns' values); zeros for a subject
// without cells.
std::vector<double> subject_row(const PmlData& d, int s) {
  std::vector<double> x(d.n_beta, 0.0);
  if (d.subject_start[s] < d.subject_start[s + 1])
    for (int a = 0; a < d.n_beta; ++a) x[a] = d.design[d.subject_start[s] * d.n_beta + a];
  return x;
}

// Per subject, the constant columns' share of eta (cs, in column order) and
// cs + log_w.
void constant_shares(const PmlData& d, const Split& sp, const std::vector<double>& beta,
                     const std::vector<double>& log_w, std::vector<double>* cs, std::vector<double>* csl) {
  cs->assign(d.k, 0.0);
  csl->assign(d.k, 0.0);
  for (int s = 0; s < d.k; ++s) {
    const std::vector<double> x = subject_row(d, s);
    double c = 0.0;
    for (int a = 0; a < d.n_beta; ++a)
      if (sp.vpos[a] < 0) c = nebula::nb_fma(x[a], beta[a], c);
    (*cs)[s] = c;
    (*csl)[s] = c + log_w[s];
  }
}

// Cell r's varying design values, and eta over them continuing from `start`.
int varying_row(const PmlData& d, const Split& sp, size_t r, double* x) {
  const int nv = static_cast<int>(sp.varying.size());
  for (int j = 0; j < nv; ++j) x[j] = d.design[r * d.n_beta + sp.varying[j]];
  return nv;
}
double varying_eta(const Split& sp, const double* x, const std::vector<double>& beta, double start) {
  double eta = start;
  for (size_t j = 0; j < sp.varying.size(); ++j) eta = nebula::nb_fma(x[j], beta[sp.varying[j]], eta);
  return eta;
}

namespace {

// Slot layout of a per-subject partial: resid, weight, sum ln t, sum y eta,
// sum y ln t, X'd (nb), sum p x (nb), sum p x x' (upper triangle).
enum { kResid = 0, kWeight = 1, kSumLog = 2, kLinear = 3, kWlog = 4, kScore = 5 };

// The fold of pml.rs:1469-1489 over the varying columns (nb of them): d
// into the gradient, p into the curvature.
void fold(double* acc, const double* x, int nb, double dd, double p) {
  acc[kResid] += dd;
  acc[kWeight] += p;
  double* score = acc + kScore;
  double* first = score + nb;
  double* second = first + nb;
  int t = 0;
  for (int a = 0; a < nb; ++a) {
    score[a] = nebula::nb_fma(x[a], dd, score[a]);
    double pa = p * x[a];
    first[a] += pa;
    for (int b = a; b < nb; ++b) {
      second[t] = nebula::nb_fma(pa, x[b], second[t]);
      ++t;
    }
  }
}

// sweep_width (pml.rs:1419-1590): each subject is a dense part over every cell
// at a count of zero, then a sparse part adding what the positive counts
// change.
void sweep(const PmlData& d, const std::vector<double>& beta, const std::vector<double>& log_w,
           double gamma, const Penalty& pen, Sweep& out) {
  const int nb = d.n_beta, k = d.k, T = nb * (nb + 1) / 2, nv = 5 + 2 * nb + T;
  const Split sp = split_columns(d);
  const int nr = static_cast<int>(sp.varying.size());
  const int nsr = 5 + 2 * nr + nr * (nr + 1) / 2;  // reduced slot: the varying columns only
  std::vector<double> cs, csl;
  constant_shares(d, sp, beta, log_w, &cs, &csl);
  auto dense = [&](double* acc, size_t r, int s) {
    double x[kMaxRow];
    varying_row(d, sp, r, x);
    double e = nebula::nb_exp_tab(varying_eta(sp, x, beta, d.offset[r] + csl[s]), &nebula::kNbTables);
    double t = e + gamma;
    acc[kSumLog] += nebula::nb_log_tab(t, &nebula::kNbTables);
    double inv = 1.0 / t;
    double u = e * inv;
    fold(acc, x, nr, -gamma * u, (gamma * u) * inv);
  };
  auto sparse = [&](double* acc, size_t i, int s) {
    size_t c = d.cells[i];
    double y = d.counts[i];
    double x[kMaxRow];
    varying_row(d, sp, c, x);
    double eta = varying_eta(sp, x, beta, d.offset[c] + cs[s]);
    double e = nebula::nb_exp_tab(eta + log_w[s], &nebula::kNbTables);
    double t = e + gamma;
    acc[kLinear] = nebula::nb_fma(eta, y, acc[kLinear]);
    acc[kWlog] = nebula::nb_fma(y, nebula::nb_log_tab(t, &nebula::kNbTables), acc[kWlog]);
    double inv = 1.0 / t;
    double u = e * inv;
    fold(acc, x, nr, y * (1.0 - u), (y * u) * inv);
  };
  std::vector<double> red = range_sums(d, nsr, dense, sparse);
  // each tabled group's cells at a count of zero (pml.rs:1515-1526): with
  // s = ln tau, sum ln t = n ln gamma + L, sum d = -gamma A, sum p = B
  if (d.zeros) {
    const double ln_gamma = nebula::nb_log(gamma);
    for (int s = 0; s < k; ++s) {
      double* R = &red[static_cast<size_t>(s) * nsr];
      for (uint32_t g = d.zeros->subject_groups[s]; g < d.zeros->subject_groups[s + 1]; ++g) {
        const nebula::zero::Group& G = d.zeros->groups[g];
        double x[kMaxRow];
        varying_row(d, sp, static_cast<size_t>(G.row), x);
        const double log_tau = varying_eta(sp, x, beta, csl[s] - ln_gamma);
        double f[3];
        nebula::zero::eval(G, d.zeros->index.data(), d.zeros->panels.data(), log_tau, 0, 3, f);
        R[kSumLog] += G.n * ln_gamma + f[0];
        fold(R, x, nr, -gamma * f[1], f[2]);
      }
    }
  }
  // every column's sums per subject: a constant column a's are its value
  // times the matching sums without it
  std::vector<double> tot(static_cast<size_t>(k) * nv);
  for (int s = 0; s < k; ++s) {
    const double* R = &red[static_cast<size_t>(s) * nsr];
    const std::vector<double> X = subject_row(d, s);
    double* F = &tot[static_cast<size_t>(s) * nv];
    for (int x = 0; x < kScore; ++x) F[x] = R[x];
    for (int a = 0; a < nb; ++a) {
      const int va = sp.vpos[a];
      F[kScore + a] = va >= 0 ? R[kScore + va] : X[a] * R[kResid];
      F[kScore + nb + a] = va >= 0 ? R[kScore + nr + va] : X[a] * R[kWeight];
    }
    int t = 0;
    for (int a = 0; a < nb; ++a)
      for (int b = a; b < nb; ++b, ++t) {
        const int va = sp.vpos[a], vb = sp.vpos[b];
        double v;
        if (va >= 0 && vb >= 0) v = R[kScore + 2 * nr + va * nr - va * (va - 1) / 2 + (vb - va)];
        else if (vb >= 0) v = X[a] * R[kScore + nr + vb];
        else if (va >= 0) v = X[b] * R[kScore + nr + va];
        else v = X[a] * (X[b] * R[kWeight]);
        F[kScore + 2 * nb + t] = v;
      }
  }
  std::vector<double> llv(k);
  for (int s = 0; s < k; ++s) {
    const double* S = &tot[static_cast<size_t>(s) * nv];
    const double lw = log_w[s];
    const double w_s = nebula::nb_exp(lw);
    llv[s] = S[kLinear] + lw * d.subject_total[s] - gamma * S[kSumLog] - S[kWlog];
    out.w[s] = w_s;
    out.dw[s] = S[kResid] + pen.gradient(lw, w_s);
    out.vw[s] = gamma * S[kWeight] + pen.curvature(w_s);
    for (int a = 0; a < nb; ++a) out.vwb[static_cast<size_t>(s) * nb + a] = gamma * S[kScore + nb + a];
  }
  for (int a = 0; a < nb; ++a) {
    double acc = 0.0;
    for (int s = 0; s < k; ++s) acc += tot[static_cast<size_t>(s) * nv + kScore + a];
    out.db[a] = acc;
  }
  int t = 0;
  for (int a = 0; a < nb; ++a) {
    for (int b = a; b < nb; ++b, ++t) {
      double acc = 0.0;
      for (int s = 0; s < k; ++s) acc += gamma * tot[static_cast<size_t>(s) * nv + kScore + 2 * nb + t];
      out.vb[a * nb + b] = acc;
      out.vb[b * nb + a] = acc;
    }
  }
  double ll = 0.0;
  for (int s = 0; s < k; ++s) ll += llv[s];
  out.ll = pen.accumulate(ll, log_w, out.w);
}

// Pivoted LDL' solve in place, Eigen's LDLT as nebula calls it (pml.rs:1940-2021).
void ldlt_solve(std::vector<double>& a, std::vector<double>& b, int n) {
  std::vector<int> perm(n);
  std::vector<double> tmp(n);
  for (int step = 0; step < n; ++step) {
    int pivot = step;
    double best = std::fabs(a[step * n + step]);
    for (int i = step + 1; i < n; ++i) {
      double v = std::fabs(a[i * n + i]);
      if (v > best) {
        best = v;
        pivot = i;
      }
    }
    perm[step] = pivot;
    if (pivot != step) {
      for (int j = 0; j < step; ++j) std::swap(a[step * n + j], a[pivot * n + j]);
      for (int i = pivot + 1; i < n; ++i) std::swap(a[i * n + step], a[i * n + pivot]);
      std::swap(a[step * n + step], a[pivot * n + pivot]);
      for (int i = step + 1; i < pivot; ++i) std::swap(a[i * n + step], a[pivot * n + i]);
    }
    if (step > 0) {
      for (int j = 0; j < step; ++j) tmp[j] = a[j * n + j] * a[step * n + j];
      double acc = 0.0;
      for (int j = 0; j < step; ++j) acc += a[step * n + j] * tmp[j];
      a[step * n + step] -= acc;
      for (int i = step + 1; i < n; ++i) {
        double acc2 = 0.0;
        for (int j = 0; j < step; ++j) acc2 += a[i * n + j] * tmp[j];
        a[i * n + step] -= acc2;
      }
    }
    double dd = a[step * n + step];
    if (dd != 0.0)
      for (int i = step + 1; i < n; ++i) a[i * n + step] /= dd;
  }
  for (int step = 0; step < n; ++step) std::swap(b[step], b[perm[step]]);
  for (int i = 0; i < n; ++i) {
    double acc = b[i];
    for (int j = 0; j < i; ++j) acc -= a[i * n + j] * b[j];
    b[i] = acc;
  }
  for (int i = 0; i < n; ++i) {
    double dd = a[i * n + i];
    b[i] = std::fabs(dd) > DBL_MIN ? b[i] / dd : 0.0;
  }
  for (int i = n - 1; i >= 0; --i) {
    double acc = b[i];
    for (int j = i + 1; j < n; ++j) acc -= a[j * n + i] * b[j];
    b[i] = acc;
  }
  for (int step = n - 1; step >= 0; --step) std::swap(b[step], b[perm[step]]);
}

// Partial-pivot LU determinant, a product as in the C++ (pml.rs:2036-2069).
double determinant(std::vector<double> a, int n) {
  double det = 1.0;
  for (int step = 0; step < n; ++step) {
    int pivot = step;
    double best = std::fabs(a[step * n + step]);
    for (int i = step + 1; i < n; ++i) {
      double v = std::fabs(a[i * n + step]);
      if (v > best) {
        best = v;
        pivot = i;
      }
    }
    if (pivot != step) {
      for (int j = 0; j < n; ++j) std::swap(a[step * n + j], a[pivot * n + j]);
      det = -det;
    }
    double dd = a[step * n + step];
    det *= dd;
    if (dd == 0.0) return 0.0;
    for (int i = step + 1; i < n; ++i) {
      double factor = a[i * n + step] / dd;
      a[i * n + step] = factor;
      for (int j = step + 1; j < n; ++j) a[i * n + j] -= factor * a[step * n + j];
    }
  }
  return det;
}

// Higher-order Laplace terms at the final iterate (pml.rs:1828-1919).
double laplace_correction(const PmlData& d, const std::vector<double>& beta, const std::vector<double>& log_w,
                          const std::vector<double>& w_cur, double gamma,
                          double lambda, int ord) {
  const bool high = ord > 2;
  auto terms = [&](double e, double scale, double* acc) {
    double t = e + gamma;
    double inv = 1.0 / t;
    double p2 = (e * inv) * inv, p3 = p2 * inv, p4 = p3 * inv, p5 = p4 * inv, e2 = e * e;
    acc[0] += scale * p2;
    acc[1] += scale * (p3 * (gamma - e));
    acc[2] += scale * (p4 * (gamma * gamma + e2 - (4.0 * gamma) * e));
    acc[3] += scale * (p5 * (gamma * gamma * gamma - (11.0 * gamma * gamma) * e + (11.0 * gamma) * e2 - e2 * e));
  };
  const Split sp = split_columns(d);
  std::vector<double> cs, csl;
  constant_shares(d, sp, beta, log_w, &cs, &csl);
  auto dense = [&](double* acc, size_t r, int s) {
    double x[kMaxRow];
    varying_row(d, sp, r, x);
    terms(nebula::nb_exp_tab(varying_eta(sp, x, beta, d.offset[r] + csl[s]), &nebula::kNbTables), gamma, acc);
  };
  auto sparse = [&](double* acc, size_t i, int s) {
    double x[kMaxRow];
    varying_row(d, sp, d.cells[i], x);
    const double eta = varying_eta(sp, x, beta, d.offset[d.cells[i]] + cs[s]);
    terms(nebula::nb_exp_tab(eta + log_w[s], &nebula::kNbTables), d.counts[i], acc);
  };
  std::vector<double> tot = range_sums(d, 4, dense, sparse);
  // each tabled group's B, C, D and E (pml.rs:1875-1885)
  if (d.zeros) {
    const double ln_gamma = nebula::nb_log(gamma);
    for (int s = 0; s < d.k; ++s) {
      for (uint32_t g = d.zeros->subject_groups[s]; g < d.zeros->subject_groups[s + 1]; ++g) {
        const nebula::zero::Group& G = d.zeros->groups[g];
        double x[kMaxRow];
        varying_row(d, sp, static_cast<size_t>(G.row), x);
        const double log_tau = varying_eta(sp, x, beta, csl[s] - ln_gamma);
        double f[4];
        nebula::zero::eval(G, d.zeros->index.data(), d.zeros->panels.data(), log_tau, 2, 4, f);
        for (int j = 0; j < 4; ++j) tot[static_cast<size_t>(s) * 4 + j] += f[j];
      }
    }
  }
  double third_acc = 0, fourth_acc = 0, fifth_acc = 0;
  for (int s = 0; s < d.k; ++s) {
    const double* S = &tot[static_cast<size_t>(s) * 4];
    double prior = lambda * w_cur[s];
    double vw = gamma * S[0] + prior;
    double third = gamma * S[1] + prior;
    third_acc += third * third / (vw * vw * vw);
    if (high) {
      double fourth = gamma * S[2] + prior;
      double fifth = gamma * S[3] + prior;
      double vs = vw * vw;
      fourth_acc += fourth / vs;
      fifth_acc += fifth * third / (vs * vs);
    }
  }
  double second = 5.0 * third_acc / 24.0;
  if (high) {
    second -= fourth_acc / 8.0;
    second += 7.0 * fifth_acc / 48.0;
  }
  return second;
}

}  // namespace

double min_eigenvalue(const double* m, int n) {  // pml.rs:2084-2134
  if (n == 0) return std::numeric_limits<double>::quiet_NaN();
  if (n == 1) return m[0];
  std::vector<double> a(m, m + n * n);
  double frob = 0.0;
  for (double v : a) frob += v * v;
  double tol = std::max(frob * DBL_EPSILON * DBL_EPSILON, DBL_MIN);
  for (int sweep_i = 0; sweep_i < kJacobiSweeps; ++sweep_i) {
    double off = 0.0;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) off += a[p * n + q] * a[p * n + q];
    if (off <= tol) break;
    for (int p = 0; p < n; ++p) {
      for (int q = p + 1; q < n; ++q) {
        double apq = a[p * n + q];
        if (apq == 0.0) continue;
        double theta = (a[q * n + q] - a[p * n + p]) / (2.0 * apq);
        double t = std::copysign(1.0, theta) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double c = 1.0 / std::sqrt(t * t + 1.0);
        double s = t * c;
        for (int r = 0; r < n; ++r) {
          double arp = a[r * n + p], arq = a[r * n + q];
          a[r * n + p] = c * arp - s * arq;
          a[r * n + q] = s * arp + c * arq;
        }
        for (int r = 0; r < n; ++r) {
          double apr = a[p * n + r], aqr = a[q * n + r];
          a[p * n + r] = c * apr - s * aqr;
          a[q * n + r] = s * apr + c * aqr;
        }
      }
    }
  }
  double mn = std::numeric_limits<double>::infinity();
  for (int i = 0; i < n; ++i) mn = std::fmin(mn, a[i * n + i]);
  return mn;
}

int check_convergence(const PmlResult& r, const PmlParams& p, bool at_bound, int initial) {
  int code = initial;
  if (code == 1) {
    if (at_bound) code = -60;
    else if (std::isnan(r.log_likelihood)) code = -30;
    else if (r.iterations == p.max_iter) code = -20;
    else if (r.backtracks == p.max_backtrack + 1) code = -10;
    else if (r.backtracks == p.max_backtrack + 2) code = -40;
    else code = 1;
  }
  int nb = static_cast<int>(r.beta.size());
  if (nb > 1 && min_eigenvalue(r.information.data(), nb) < kEigenCutoff) code = -25;
  return code;
}

bool opt_pml(const PmlData& d, const double* beta_init, const double* log_w_init, double subject,
             double gamma, const PmlParams& params, Prior prior, PmlResult* out) {
  Penalty pen{prior, 0.0, 0.0};
  if (prior == Prior::Gamma) {  // gamma_penalty (pml.rs:432-441)
    double exps = nebula::nb_exp(subject);
    if (!(std::isfinite(exps) && exps > 1.0)) return false;
    pen.alpha = 1.0 / (exps - 1.0);
    pen.lambda = 1.0 / (std::sqrt(exps) * (exps - 1.0));
  } else {
    if (!(std::isfinite(subject) && subject > 0.0)) return false;
    pen.alpha = subject;
  }
  if (!(std::isfinite(gamma) && gamma > 0.0)) return false;
  if (d.n_beta < 1 || d.n_beta > kMaxRow) return false;
  const int nb = d.n_beta, k = d.k;
  std::vector<double> beta(beta_init, beta_init + nb);
  std::vector<double> log_w(k, 0.0);
  if (log_w_init) log_w.assign(log_w_init, log_w_init + k);
  Sweep cur, trial;
  cur.init(nb, k);
  trial.init(nb, k);
  std::vector<double> vw_step(k, 0), vb2(nb * nb, 0), step_beta(nb), step_log_w(k), dwvw(k);
  std::vector<double> damp_beta(nb), damp_log_w(k), new_beta(nb), new_log_w(k);
  int sweeps = 0;
  sweep(d, beta, log_w, gamma, pen, cur);
  ++sweeps;
  double ll = cur.ll, ll_prev = 0.0, likdif = 0.0;
  int step = 0, backtracks = 0;
  while (step == 0 || (likdif > params.eps && step < params.max_iter)) {
    ++step;
    std::fill(damp_beta.begin(), damp_beta.end(), 1.0);
    std::fill(damp_log_w.begin(), damp_log_w.end(), 1.0);
    vw_step = cur.vw;
    for (int s = 0; s < k; ++s) dwvw[s] = cur.dw[s] / cur.vw[s];
    for (int a = 0; a < nb; ++a) {
      for (int b = a; b < nb; ++b) {
        double acc = 0.0;
        for (int s = 0; s < k; ++s) acc += cur.vwb[s * nb + a] * cur.vwb[s * nb + b] / cur.vw[s];
        double v = cur.vb[a * nb + b] - acc;
        vb2[a * nb + b] = v;
        vb2[b * nb + a] = v;
      }
    }
    for (int j = 0; j < nb; ++j) {
      double acc = 0.0;
      for (int s = 0; s < k; ++s) acc += cur.vwb[s * nb + j] * dwvw[s];
      step_beta[j] = cur.db[j] - acc;
    }
    std::vector<double> factor = vb2;
    ldlt_solve(factor, step_beta, nb);
    for (int s = 0; s < k; ++s) {
      double acc = 0.0;
      for (int j = 0; j < nb; ++j) acc += cur.vwb[s * nb + j] * step_beta[j];
      step_log_w[s] = dwvw[s] - acc / cur.vw[s];
    }
    for (int j = 0; j < nb; ++j) new_beta[j] = beta[j] + step_beta[j];
    for (int s = 0; s < k; ++s) new_log_w[s] = log_w[s] + step_log_w[s];
    ll_prev = ll;
    sweep(d, new_beta, new_log_w, gamma, pen, trial);
    ++sweeps;
    ll = trial.ll;
    likdif = ll - ll_prev;
    backtracks = 0;
    double min_step = kStepCutoff;
    while (likdif < 0.0 || std::isinf(ll)) {
      ++backtracks;
      min_step /= 2.0;
      if (backtracks > params.max_backtrack) {
        likdif = 0.0;
        ll = ll_prev;
        double gb = 0.0, gw = 0.0;
        for (double v : cur.db) gb = std::fmax(gb, std::fabs(v));
        for (double v : cur.dw) gw = std::fmax(gw, std::fabs(v));
        if (gb > kGradientTolerance || gw > kGradientTolerance) ++backtracks;
        break;
      }
      for (int j = 0; j < nb; ++j) {
        double dd = step_beta[j];
        if (dd < kStepCutoff && dd > -kStepCutoff) {
          damp_beta[j] /= 2.0;
          new_beta[j] = beta[j] + dd * damp_beta[j];
        } else if (dd > 0.0) {
          new_beta[j] = beta[j] + min_step;
        } else {
          new_beta[j] = beta[j] - min_step;
        }
      }
      for (int s = 0; s < k; ++s) {
        double dd = step_log_w[s];
        if (dd < kStepCutoff && dd > -kStepCutoff) {
          damp_log_w[s] /= 2.0;
          new_log_w[s] = log_w[s] + dd * damp_log_w[s];
        } else if (dd > 0.0) {
          new_log_w[s] = log_w[s] + min_step;
        } else {
          new_log_w[s] = log_w[s] - min_step;
        }
      }
      sweep(d, new_beta, new_log_w, gamma, pen, trial);
      ++sweeps;
      ll = trial.ll;
      likdif = ll - ll_prev;
    }
    beta = new_beta;
    log_w = new_log_w;
    std::swap(cur, trial);
  }
  double log_det = 0.0;
  for (int s = 0; s < k; ++s) log_det += nebula::nb_log(std::fabs(vw_step[s]));
  if (params.reml) log_det += nebula::nb_log(std::fabs(determinant(vb2, nb)));
  double second = 0.0;
  if (prior == Prior::Gamma && params.ord > 1) {
    second = laplace_correction(d, beta, log_w, cur.w, gamma, pen.lambda, params.ord);
    ++sweeps;
  }
  out->beta = beta;
  out->log_w = log_w;
  out->information = vb2;
  out->log_likelihood = ll;
  out->log_likelihood_prev = ll_prev;
  out->log_det = log_det;
  out->second_order = second;
  out->iterations = step;
  out->backtracks = backtracks;
  out->sweeps = sweeps;
  out->convergence = check_convergence(*out, params, false, 1);
  return true;
}

double pml_objective_gradient(const PmlData& d, const double* beta, const double* log_w,
                              double subject, double gamma, double* gradient) {
  Penalty pen{Prior::Gamma, subject, subject};  // nebula's Gamma(alpha, alpha) reading
  const int nb = d.n_beta, k = d.k;
  std::vector<double> b(beta, beta + nb), lw(log_w, log_w + k);
  Sweep cur;
  cur.init(nb, k);
  sweep(d, b, lw, gamma, pen, cur);
  for (int j = 0; j < nb; ++j) gradient[j] = -cur.db[j];
  for (int s = 0; s < k; ++s) gradient[nb + s] = -cur.dw[s];
  return -cur.ll;
}

}  // namespace oracle
