// Stage-two search, profile objective, stage-three finish and assembly; see
// search.hpp for the reference lines each piece follows.
#include "search.hpp"

#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <limits>

#include "special.hpp"
#include "stage_one.hpp"

namespace nebula {

namespace {

constexpr double kVarianceXatol = 1e-7;        // nebula.rs:173
constexpr double kVarianceFatol = 1e-7;        // nebula.rs:176
constexpr int kVarianceMaxIter = 500;          // nebula.rs:179
constexpr double kPolishWidths[3] = {1e-2, 3e-3, 1e-3};  // nebula.rs:106
constexpr double kPolishFloor[2] = {1e-5, 1e-4};         // nebula.rs:112
constexpr double kPolishMaxStep = 2.0;                   // nebula.rs:118
constexpr double kBoundSlack = 1.0 + 1e-4;               // nebula.rs:92
constexpr double kNmStep = 0.05;          // optimise.rs:40
constexpr double kNmZeroStep = 0.00025;   // optimise.rs:45
constexpr double kNmCollapsedUlps = 16.0; // optimise.rs:56

// f64::total_cmp as a strict weak order.
bool total_less(double a, double b) {
  int64_t ia, ib;
  std::memcpy(&ia, &a, 8);
  std::memcpy(&ib, &b, 8);
  ia ^= static_cast<int64_t>(static_cast<uint64_t>(ia >> 63) >> 1);
  ib ^= static_cast<int64_t>(static_cast<uint64_t>(ib >> 63) >> 1);
  return ia < ib;
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

// Reverse-communicated Nelder-Mead, scipy's scheme as the reference steps it
// (src/numeric/optimise.rs:390-678).
class NelderMead {
 public:
  NelderMead(const std::vector<double>& x0, double xatol, double fatol, int max_iter)
      : xatol_(xatol), fatol_(fatol), max_iter_(max_iter), n_(static_cast<int>(x0.size())) {
    simplex_.push_back(x0);
    for (int i = 0; i < n_; ++i) {
      std::vector<double> v = x0;
      if (v[i] != 0.0) v[i] *= 1.0 + kNmStep;
      else v[i] = kNmZeroStep;
      simplex_.push_back(v);
    }
    values_.assign(n_ + 1, 0.0);
    order_.resize(n_ + 1);
    for (int i = 0; i <= n_; ++i) order_[i] = i;
    pending_ = simplex_[0];
    centroid_.assign(n_, 0.0);
    reflected_.assign(n_, 0.0);
  }
  const std::vector<double>* ask() const { return phase_ == Phase::Done ? nullptr : &pending_; }
  struct Result {
    std::vector<double> x;
    double f;
  };
  Result result() const { return {simplex_[order_[0]], values_[order_[0]]}; }
  void tell(double value) {
    const int n = n_;
    switch (phase_) {
      case Phase::Init:
        values_[init_] = value;
        if (init_ < n) {
          ++init_;
          pending_ = simplex_[init_];
        } else {
          begin_iteration();
        }
        break;
      case Phase::Reflect: {
        f_reflected_ = value;
        if (value < values_[best_]) {
          for (int j = 0; j < n; ++j) pending_[j] = centroid_[j] + 2.0 * (centroid_[j] - simplex_[worst_][j]);
          phase_ = Phase::Expand;
        } else if (value < values_[second_worst_]) {
          simplex_[worst_] = reflected_;
          values_[worst_] = value;
          begin_iteration();
        } else {
          inside_ = value >= values_[worst_];
          for (int j = 0; j < n; ++j)
            pending_[j] = inside_ ? centroid_[j] - 0.5 * (centroid_[j] - simplex_[worst_][j])
                                  : centroid_[j] + 0.5 * (centroid_[j] - simplex_[worst_][j]);
          phase_ = Phase::Contract;
        }
        break;
      }
      case Phase::Expand:
        if (value < f_reflected_) {
          simplex_[worst_] = pending_;
          values_[worst_] = value;
        } else {
          simplex_[worst_] = reflected_;
          values_[worst_] = f_reflected_;
        }
        begin_iteration();
        break;
      case Phase::Contract: {
        bool accept = inside_ ? value < values_[worst_] : value <= f_reflected_;
        if (accept) {
          simplex_[worst_] = pending_;
          values_[worst_] = value;
          begin_iteration();
        } else {
          shrink_vertex(1);
        }
        break;
      }
      case Phase::Shrink:
        values_[order_[shrink_pos_]] = value;
        if (shrink_pos_ < n) shrink_vertex(shrink_pos_ + 1);
        else begin_iteration();
        break;
      case Phase::Done:
        break;
    }
  }

 private:
  enum class Phase { Init, Reflect, Expand, Contract, Shrink, Done };
  void sort_order() {
    std::stable_sort(order_.begin(), order_.end(),
                     [this](int a, int b) { return total_less(values_[a], values_[b]); });
  }
  void shrink_vertex(int pos) {
    int i = order_[pos];
    for (int j = 0; j < n_; ++j) {
      double anchor = simplex_[best_][j];
      simplex_[i][j] = anchor + 0.5 * (simplex_[i][j] - anchor);
    }
    pending_ = simplex_[i];
    shrink_pos_ = pos;
    phase_ = Phase::Shrink;
  }
  void begin_iteration() {
    const int n = n_;
    if (next_iter_ >= max_iter_) {
      sort_order();
      phase_ = Phase::Done;
      return;
    }
    ++next_iter_;
    sort_order();
    best_ = order_[0];
    worst_ = order_[n];
    second_worst_ = order_[n - 1];
    double spread_x = 0.0, spread_f = 0.0;
    for (int p = 1; p <= n; ++p) {
      int i = order_[p];
      double m = 0.0;
      for (int j = 0; j < n; ++j) m = std::fmax(m, std::fabs(simplex_[i][j] - simplex_[best_][j]));
      spread_x = std::fmax(spread_x, m);
      spread_f = std::fmax(spread_f, std::fabs(values_[i] - values_[best_]));
    }
    double scale = DBL_MIN;
    for (double v : simplex_[best_]) scale = std::fmax(scale, std::fabs(v));
    bool collapsed = spread_x <= kNmCollapsedUlps * DBL_EPSILON * scale;
    if (collapsed || (spread_x <= xatol_ && spread_f <= fatol_)) {
      sort_order();
      phase_ = Phase::Done;
      return;
    }
    std::fill(centroid_.begin(), centroid_.end(), 0.0);
    for (int p = 0; p < n; ++p)
      for (int j = 0; j < n; ++j) centroid_[j] += simplex_[order_[p]][j];
    for (int j = 0; j < n; ++j) centroid_[j] /= static_cast<double>(n);
    for (int j = 0; j < n; ++j) reflected_[j] = centroid_[j] + (centroid_[j] - simplex_[worst_][j]);
    pending_ = reflected_;
    phase_ = Phase::Reflect;
  }

  double xatol_, fatol_;
  int max_iter_, n_;
  std::vector<std::vector<double>> simplex_;
  std::vector<double> values_;
  std::vector<int> order_;
  int next_iter_ = 0, init_ = 0, shrink_pos_ = 0;
  Phase phase_ = Phase::Init;
  std::vector<double> pending_, centroid_, reflected_;
  double f_reflected_ = 0.0;
  bool inside_ = false;
  int best_ = 0, worst_ = 0, second_worst_ = 0;
};

// ------------------------------------------------------------------------
// StageTwoSearch (nebula.rs:1607-1951)

StageTwoSearch::StageTwoSearch(const std::vector<double>& start, const std::vector<double>& lower,
                               const std::vector<double>& upper, int ord, double radius_scale)
    : lower_(lower), upper_(upper), start_(start), order_(ord), radius_scale_(radius_scale) {
  begin_pass();
}

StageTwoSearch::~StageTwoSearch() = default;

std::vector<double> StageTwoSearch::clamped(const std::vector<double>& x) const {
  std::vector<double> out(x.size());
  for (size_t j = 0; j < x.size(); ++j) out[j] = std::clamp(x[j], lower_[j], upper_[j]);
  return out;
}

void StageTwoSearch::begin_pass() {
  invalid_ = false;
  restarted_ = false;
  pinned_.reset();
  simplex_.reset();
  failed_ = false;
  if (start_.size() == 2) {
    std::vector<double> x0 = clamped(start_);
    bobyqa_ = std::make_unique<Bobyqa>(x0.data(), lower_.data(), upper_.data(), 2, 1e-6, 1000, radius_scale_);
    radius_scale_ = 1.0;
    if (!bobyqa_->ok()) {
      bobyqa_.reset();
      end_pass(std::nullopt);
      return;
    }
    stage_ = Stage::Bobyqa;
    ask_bobyqa();
    return;
  }
  stage_ = Stage::Start;
  asked_ = {clamped(start_)};
}

void StageTwoSearch::ask_bobyqa() {
  const double* x = bobyqa_->ask();
  if (x) {
    asked_ = {std::vector<double>(x, x + bobyqa_->n())};
    return;
  }
  BobyqaResult r = bobyqa_->result();
  bobyqa_.reset();
  failed_ = r.status == BobyqaStatus::RoundoffLimited;
  end_pass(r.x);
}

void StageTwoSearch::end_pass(std::optional<std::vector<double>> found) {
  if ((found.has_value() && !invalid_) || order_ == 1) {
    found_ = std::move(found);
    stage_ = Stage::Done;
    asked_.clear();
  } else {
    order_ = 1;
    begin_pass();
  }
}

void StageTwoSearch::ask_simplex() {
  const std::vector<double>* x = simplex_->ask();
  if (x) {
    asked_ = {clamped(*x)};
    return;
  }
  NelderMead::Result r = simplex_->result();
  std::vector<double> best = clamped(r.x);
  std::vector<double> x0;
  if (!restarted_ && bound_restart(best, clamped(start_), lower_, upper_, &x0)) {
    restarted_ = true;
    pinned_ = std::make_pair(best, r.f);
    simplex_ = std::make_unique<NelderMead>(x0, kVarianceXatol, kVarianceFatol, kVarianceMaxIter);
    ask_simplex();
    return;
  }
  if (pinned_.has_value()) {
    auto first = std::move(*pinned_);
    pinned_.reset();
    if (first.second <= r.f) best = first.first;
  }
  best_ = best;
  simplex_.reset();
  stage_ = Stage::Check;
  asked_ = {best};
}

void StageTwoSearch::begin_polish() {
  if (width_ == 3) {
    std::vector<double> best = std::move(best_);
    best_.clear();
    end_pass(best);
    return;
  }
  const double width = kPolishWidths[width_];
  const size_t n = best_.size();
  const std::vector<double>& x = best_;
  std::vector<double> step(n);
  for (size_t j = 0; j < n; ++j) step[j] = std::fmax(width * std::fabs(x[j]), kPolishFloor[j]);
  std::vector<std::array<double, 3>> nodes(n);
  for (size_t j = 0; j < n; ++j) {
    if (x[j] - step[j] < lower_[j]) nodes[j] = {0.0, 1.0, 2.0};
    else if (x[j] + step[j] > upper_[j]) nodes[j] = {-2.0, -1.0, 0.0};
    else nodes[j] = {-1.0, 0.0, 1.0};
  }
  size_t n_points = 1;
  for (size_t j = 0; j < n; ++j) n_points *= 3;
  offsets_.clear();
  asked_.clear();
  for (size_t point = 0; point < n_points; ++point) {
    std::vector<double> u(n);
    size_t rest = point;
    for (size_t j = 0; j < n; ++j) {
      double node = nodes[j][rest % 3];
      rest /= 3;
      double p = std::clamp(x[j] + node * step[j], lower_[j], upper_[j]);
      u[j] = (p - x[j]) / step[j];
    }
    std::vector<double> q(n);
    for (size_t j = 0; j < n; ++j) q[j] = x[j] + u[j] * step[j];
    asked_.push_back(q);
    offsets_.push_back(u);
  }
  step_ = step;
  stage_ = Stage::Polish;
}

std::optional<std::vector<double>> StageTwoSearch::fit_polish(const std::vector<double>& values) const {
  const std::vector<double>& x = best_;
  const int n = static_cast<int>(x.size());
  const int n_terms = 1 + 2 * n + n * (n - 1) / 2;
  std::vector<double> rows;
  for (const auto& u : offsets_) {
    rows.push_back(1.0);
    for (double v : u) rows.push_back(v);
    for (double v : u) rows.push_back(0.5 * v * v);
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) rows.push_back(u[i] * u[j]);
  }
  std::vector<double> normal(static_cast<size_t>(n_terms) * n_terms, 0.0), rhs(n_terms, 0.0);
  for (size_t point = 0; point < values.size(); ++point) {
    const double* row = &rows[point * n_terms];
    double f = values[point];
    for (int a = 0; a < n_terms; ++a) {
      rhs[a] += row[a] * f;
      for (int b = 0; b < n_terms; ++b) normal[a * n_terms + b] += row[a] * row[b];
    }
  }
  std::vector<double> coefficients;
  if (!cholesky_solve(normal, n_terms, rhs, &coefficients)) return std::nullopt;
  std::vector<double> hessian(static_cast<size_t>(n) * n, 0.0), negated(n);
  for (int j = 0; j < n; ++j) hessian[j * n + j] = coefficients[1 + n + j];
  int cross = 1 + 2 * n;
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) {
      hessian[i * n + j] = coefficients[cross];
      hessian[j * n + i] = coefficients[cross];
      ++cross;
    }
  for (int j = 0; j < n; ++j) negated[j] = -coefficients[1 + j];
  std::vector<double> delta;
  if (!cholesky_solve(hessian, n, negated, &delta)) return std::nullopt;
  for (double d : delta)
    if (!std::isfinite(d) || std::fabs(d) > kPolishMaxStep) return std::nullopt;
  std::vector<double> out(n);
  for (int j = 0; j < n; ++j) out[j] = std::clamp(x[j] + delta[j] * step_[j], lower_[j], upper_[j]);
  return out;
}

void StageTwoSearch::tell(const std::vector<double>& values) {
  evaluations_ += static_cast<int>(values.size());
  for (double v : values) {
    if (!std::isfinite(v)) invalid_ = true;
    else if (v < best_value_) best_value_ = v;
  }
  switch (stage_) {
    case Stage::Start:
      if (!std::isfinite(values[0])) {
        end_pass(std::nullopt);
        return;
      }
      simplex_ = std::make_unique<NelderMead>(clamped(start_), kVarianceXatol, kVarianceFatol,
                                              kVarianceMaxIter);
      stage_ = Stage::NelderMead;
      ask_simplex();
      break;
    case Stage::NelderMead:
      simplex_->tell(values[0]);
      ask_simplex();
      break;
    case Stage::Check:
      if (!std::isfinite(values[0])) {
        end_pass(std::nullopt);
        return;
      }
      width_ = 0;
      begin_polish();
      break;
    case Stage::Polish: {
      bool finite = true;
      for (double v : values) finite = finite && std::isfinite(v);
      if (finite) {
        auto next = fit_polish(values);
        if (next) best_ = *next;
      }
      ++width_;
      begin_polish();
      break;
    }
    case Stage::Bobyqa:
      if (!std::isfinite(values[0])) {
        end_pass(std::nullopt);
        return;
      }
      bobyqa_->tell(values[0]);
      ask_bobyqa();
      break;
    case Stage::Done:
      break;
  }
}

std::optional<std::pair<std::vector<double>, bool>> StageTwoSearch::result() const {
  if (!found_) return std::nullopt;
  return std::make_pair(*found_, failed_);
}

// ------------------------------------------------------------------------
// VarianceObjective (nebula.rs:1365-1505, variance_objective 2031-2059)

VarianceObjective VarianceObjective::make(const Shared& sh, const GeneCounts& gc,
                                          std::optional<double> fixed_cell) {
  VarianceObjective o;
  o.intercept = sh.intercept;
  o.n_cells = static_cast<double>(sh.n_cells);
  o.n_subjects = static_cast<double>(sh.n_subjects);
  o.n_positive = static_cast<double>(gc.counts.size());
  o.n_one = static_cast<double>(gc.n_one);
  o.n_two = static_cast<double>(gc.n_two);
  o.fixed_cell = fixed_cell;
  std::vector<double> values;
  for (double y : gc.counts)
    if (y != 1.0 && y != 2.0) values.push_back(y);
  std::sort(values.begin(), values.end(), total_less);
  for (double y : values) {
    if (!o.histogram.empty() && o.histogram.back().first == y) o.histogram.back().second += 1.0;
    else o.histogram.emplace_back(y, 1.0);
  }
  return o;
}

bool VarianceObjective::request(const std::vector<double>& x, const std::vector<double>& beta_start,
                                double* subject, double* cell, std::vector<double>* beta) const {
  *subject = x[0];
  *cell = fixed_cell ? *fixed_cell : x[1];
  if (!(std::isfinite(*subject) && *subject > 0.0 && std::isfinite(*cell) && *cell > 0.0)) return false;
  *beta = beta_start;
  (*beta)[intercept] -= *subject / 2.0;
  return true;
}

double VarianceObjective::tail(double cell) const {
  double t = 0.0;
  for (const auto& [y, m] : histogram) t += m * ln_gamma(y + cell);
  return t;
}

double VarianceObjective::assemble(double subject, double cell, const InnerFit& fit, double tail) const {
  if (fit.second_order < -1.0) return std::numeric_limits<double>::infinity();
  double exps = std::exp(subject);
  double alpha = 1.0 / (exps - 1.0);
  double lambda = 1.0 / (std::sqrt(exps) * (exps - 1.0));
  double base = std::isnan(fit.log_likelihood) ? fit.log_likelihood_prev : fit.log_likelihood;
  double ll = base + n_cells * cell * std::log(cell) + n_subjects * alpha * std::log(lambda) -
              n_subjects * ln_gamma(alpha);
  ll += tail - (n_positive - n_one - n_two) * ln_gamma(cell) + (n_one + n_two) * std::log(cell) +
        n_two * std::log(cell + 1.0);
  ll += -0.5 * fit.log_det + std::log(1.0 + fit.second_order);
  return std::isfinite(ll) ? -ll : std::numeric_limits<double>::infinity();
}

void variance_bounds(const Params& p, bool fixed_cell, std::vector<double>* lower,
                     std::vector<double>* upper) {
  if (fixed_cell) {
    *lower = {p.min0};
    *upper = {p.max0};
  } else {
    *lower = {p.min0, p.min1};
    *upper = {p.max0, p.max1};
  }
}

void apply_refit(const GenePlan& plan,
                 const std::optional<std::optional<std::pair<std::vector<double>, bool>>>& refit,
                 double* sigma, double* gamma, int* convergence) {
  *sigma = plan.sigma;
  *gamma = plan.gamma;
  *convergence = plan.convergence;
  if ((plan.refit == Refit::Both || plan.refit == Refit::SubjectOnly) && refit.has_value()) {
    const auto& found = *refit;
    if (found.has_value()) {
      *sigma = found->first[0];
      if (plan.refit == Refit::Both) *gamma = found->first[1];
      *convergence = found->second ? kConvOuterFailed : kConvSuccess;
    } else {
      *convergence = kConvOuterFailed;
    }
  }
}

// ------------------------------------------------------------------------
// Stage three (nebula.rs:918-1000)

double min_eigenvalue(const double* m, int n) {  // cyclic Jacobi, pml.rs:2084-2134
  if (n == 0) return std::numeric_limits<double>::quiet_NaN();
  if (n == 1) return m[0];
  std::vector<double> a(m, m + n * n);
  double frob = 0.0;
  for (double v : a) frob += v * v;
  double tol = std::fmax(frob * DBL_EPSILON * DBL_EPSILON, DBL_MIN);
  for (int it = 0; it < 30; ++it) {
    double off = 0.0;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) off += a[p * n + q] * a[p * n + q];
    if (off <= tol) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        double apq = a[p * n + q];
        if (apq == 0.0) continue;
        double theta = (a[q * n + q] - a[p * n + p]) / (2.0 * apq);
        double t = std::copysign(1.0, theta) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
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
  double mn = std::numeric_limits<double>::infinity();
  for (int i = 0; i < n; ++i) mn = std::fmin(mn, a[i * n + i]);
  return mn;
}

namespace {

// Lower Cholesky factor rejecting non-positive, NaN or infinite pivots
// (cholesky_factor, nebula.rs:2077-2081).
bool cholesky_factor(std::vector<double>& l, int n) {
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) {
      double sum = l[i * n + j];
      for (int k = 0; k < j; ++k) sum -= l[i * n + k] * l[j * n + k];
      if (i == j) {
        if (sum <= 0.0 || std::isnan(sum)) return false;
        l[i * n + j] = std::sqrt(sum);
      } else {
        l[i * n + j] = sum / l[j * n + j];
      }
    }
  for (int i = 0; i < n; ++i)
    if (!std::isfinite(l[i * n + i])) return false;
  return true;
}

bool cholesky_inverse(const std::vector<double>& a, int n, std::vector<double>* inv) {
  std::vector<double> l = a;
  if (!cholesky_factor(l, n)) return false;
  inv->assign(static_cast<size_t>(n) * n, 0.0);
  std::vector<double> col(n);
  for (int j = 0; j < n; ++j) {
    std::fill(col.begin(), col.end(), 0.0);
    col[j] = 1.0;
    for (int i = 0; i < n; ++i) {
      double sum = col[i];
      for (int k = 0; k < i; ++k) sum -= l[i * n + k] * col[k];
      col[i] = sum / l[i * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
      double sum = col[i];
      for (int k = i + 1; k < n; ++k) sum -= l[k * n + i] * col[k];
      col[i] = sum / l[i * n + i];
    }
    for (double v : col)
      if (!std::isfinite(v)) return false;
    for (int i = 0; i < n; ++i) (*inv)[i * n + j] = col[i];
  }
  return true;
}

}  // namespace

GeneOutcome finish_gene(const Shared& sh, double sigma, double gamma, int convergence,
                        const FinalFit& fit) {
  const Params& p = sh.params;
  const int nc = sh.n_coef;
  bool at_bound = sigma == p.max0 || gamma == p.min1;
  // check_convergence (pml.rs:1111-1139) with the final fit's max_iter
  int code = convergence;
  if (code == kConvSuccess) {
    if (at_bound) code = kConvAtBound;
    else if (std::isnan(fit.log_likelihood)) code = kConvNotFinite;
    else if (fit.iterations == kPmlMaxIter) code = kConvMaxIter;
    else if (fit.backtracks == kPmlMaxBacktrack + 1) code = kConvCriticalPoint;
    else if (fit.backtracks == kPmlMaxBacktrack + 2) code = kConvStalled;
    else code = kConvSuccess;
  }
  if (nc > 1 && min_eigenvalue(fit.information.data(), nc) < 1e-8) code = kConvSingular;
  GeneOutcome out;
  out.beta = fit.beta;
  const size_t packed = packed_len(nc);
  std::vector<double> inverse;
  if (code != kConvSingular && cholesky_inverse(fit.information, nc, &inverse)) {
    out.covariance.assign(packed, 0.0);
    for (int j = 0; j < nc; ++j)
      for (int i = 0; i <= j; ++i) out.covariance[j * (j + 1) / 2 + i] = inverse[i * nc + j];
    out.se.resize(nc);
    for (int j = 0; j < nc; ++j) out.se[j] = std::sqrt(inverse[j * nc + j]);
  } else {
    code = kConvSingular;
    out.covariance.assign(packed, std::numeric_limits<double>::quiet_NaN());
    out.se.assign(nc, std::numeric_limits<double>::quiet_NaN());
  }
  out.subject = sigma;
  out.cell = 1.0 / gamma;
  out.convergence = code;
  return out;
}

void assemble_fit(const Shared& sh, const std::vector<GeneOutcome>& outcomes,
                  const std::vector<size_t>& kept, nb_fit* out) {
  const int nc = sh.n_coef;
  std::vector<double> scale = sh.sds;
  scale[sh.intercept] = 1.0;
  const size_t packed = packed_len(nc);
  for (size_t g = 0; g < outcomes.size(); ++g) {
    const GeneOutcome& o = outcomes[g];
    for (int j = 0; j < nc; ++j) {
      if (out->coefficients) out->coefficients[g * nc + j] = o.beta[j] / scale[j];
      if (out->se) out->se[g * nc + j] = o.se[j] / scale[j];
    }
    if (out->covariance) {
      size_t idx = 0;
      for (int j = 0; j < nc; ++j)
        for (int i = 0; i <= j; ++i, ++idx)
          out->covariance[g * packed + idx] = o.covariance[j * (j + 1) / 2 + i] / (scale[i] * scale[j]);
    }
    if (out->subject_overdispersion) out->subject_overdispersion[g] = o.subject;
    if (out->cell_overdispersion) out->cell_overdispersion[g] = o.cell;
    if (out->convergence) out->convergence[g] = o.convergence;
    if (out->sigma_at_bound) out->sigma_at_bound[g] = o.subject <= sh.params.min0 * kBoundSlack ? 1 : 0;
    if (out->gene_index) out->gene_index[g] = kept[g];
  }
  out->n_kept = outcomes.size();
  out->n_coef = static_cast<uint64_t>(nc);
}

}  // namespace nebula
