// L-BFGS-B in reverse communication (lbfgsb.hpp), following
// src/numeric/lbfgsb.rs: the correction memory and its compact form
// (Memory, 130-314), solve_dense (317-361), the generalised Cauchy point
// (cauchy_point, 400-494), the subspace minimisation (subspace_minimise,
// 528-626), the feasible-step cap (max_feasible_step, 641-652), the
// strong-Wolfe line search with its bisecting zoom (line_search 675-779,
// zoom 801-849) and the driver (minimise, 876-1019). Every sum runs in the
// reference's order with separate multiplies and adds, so iterates agree
// with it to the last digit given the same objective values.
#include "lbfgsb.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <string>
#include <utility>

#include "common.hpp"

namespace nebula {
namespace {

constexpr double kWolfeC1 = 1e-4;         // lbfgsb.rs:29
constexpr double kWolfeC2 = 0.9;          // lbfgsb.rs:34
constexpr double kCurvatureEps = 2.2e-16; // lbfgsb.rs:40
constexpr double kMaxStep = 1e3;          // lbfgsb.rs:45
constexpr double kEpsilon = std::numeric_limits<double>::epsilon();
constexpr double kInf = std::numeric_limits<double>::infinity();

double dot(const std::vector<double>& a, const std::vector<double>& b) {
  double acc = 0.0;
  for (size_t i = 0; i < a.size(); ++i) acc += a[i] * b[i];
  return acc;
}

// The correction pairs, oldest first, and theta (B = theta I - W M W').
struct Memory {
  std::vector<std::vector<double>> s, y;
  double theta = 1.0;
  size_t limit;
  explicit Memory(size_t l) : limit(l) {}
  int k() const { return static_cast<int>(s.size()); }
  void reset() {
    s.clear();
    y.clear();
    theta = 1.0;
  }
  // Admits (s, y) unless its curvature is too small; evicts the oldest pair
  // when full.
  bool push(std::vector<double> sv, std::vector<double> yv) {
    const double sy = dot(sv, yv);
    const double yy = dot(yv, yv);
    if (sy <= kCurvatureEps * yy || yy <= 0.0) return false;
    if (s.size() == limit) {
      s.erase(s.begin());
      y.erase(y.begin());
    }
    theta = yy / sy;
    s.push_back(std::move(sv));
    y.push_back(std::move(yv));
    return true;
  }
  // W[i, j], W = [Y, theta S].
  double w(int i, int j) const {
    const int kk = k();
    return j < kk ? y[j][i] : theta * s[j - kk][i];
  }
  std::vector<double> wt_dot(const std::vector<double>& v) const {
    const int kk = k();
    std::vector<double> out(2 * kk, 0.0);
    for (int j = 0; j < 2 * kk; ++j) {
      double acc = 0.0;
      for (size_t i = 0; i < v.size(); ++i) acc += w(static_cast<int>(i), j) * v[i];
      out[j] = acc;
    }
    return out;
  }
  // M^{-1} = [[-D, L'], [L, theta S'S]], row-major 2k x 2k.
  std::vector<double> middle() const {
    const int kk = k(), dim = 2 * kk;
    std::vector<double> m(static_cast<size_t>(dim) * dim, 0.0);
    for (int i = 0; i < kk; ++i) m[i * dim + i] = -dot(s[i], y[i]);
    for (int i = 0; i < kk; ++i)
      for (int j = 0; j < kk; ++j)
        if (i > j) {
          const double sy = dot(s[i], y[j]);
          m[(kk + i) * dim + j] = sy;
          m[j * dim + (kk + i)] = sy;
        }
    for (int i = 0; i < kk; ++i)
      for (int j = 0; j < kk; ++j) m[(kk + i) * dim + (kk + j)] = theta * dot(s[i], s[j]);
    return m;
  }
  // M v, by solving M^{-1} z = v.
  bool apply_m(const std::vector<double>& v, std::vector<double>* out) const {
    const int dim = 2 * k();
    if (dim == 0) {
      out->clear();
      return true;
    }
    return lbfgsb_solve_dense(middle(), v, dim, out);
  }
};

struct CauchyPoint {
  std::vector<double> x;
  std::vector<char> free;
  std::vector<double> c;  // W' (xcp - x)
};

// Algorithm CP of Byrd, Lu, Nocedal and Zhu: walks the projected steepest
// descent path's segments until the one holding the model's minimiser.
bool cauchy_point(const std::vector<double>& x, const std::vector<double>& g, const std::vector<double>& lower,
                  const std::vector<double>& upper, const Memory& mem, CauchyPoint* out) {
  const int n = static_cast<int>(x.size());
  const int k = mem.k();
  std::vector<double> t(n, kInf), d(n, 0.0);
  for (int i = 0; i < n; ++i) {
    if (g[i] < 0.0 && std::isfinite(upper[i])) {
      t[i] = (x[i] - upper[i]) / g[i];
    } else if (g[i] > 0.0 && std::isfinite(lower[i])) {
      t[i] = (x[i] - lower[i]) / g[i];
    }
    d[i] = t[i] == 0.0 ? 0.0 : -g[i];
  }
  std::vector<double> xcp = x;
  std::vector<char> free(n);
  for (int i = 0; i < n; ++i) free[i] = t[i] > 0.0;
  std::vector<int> order;
  for (int i = 0; i < n; ++i)
    if (t[i] > 0.0 && std::isfinite(t[i])) order.push_back(i);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return t[a] < t[b]; });

  std::vector<double> c(2 * k, 0.0);
  std::vector<double> p = mem.wt_dot(d);
  double dd = 0.0;
  for (double v : d) dd += v * v;
  double f_prime = -dd;
  std::vector<double> mp, mc, mwb;
  if (!mem.apply_m(p, &mp)) return false;
  double f_double = -mem.theta * f_prime - dot(p, mp);
  const double f_double_initial = std::fmax(f_double, kEpsilon);
  f_double = std::fmax(f_double, kEpsilon);
  double dt_min = -f_prime / f_double;
  double t_old = 0.0;
  size_t cursor = 0;
  std::vector<double> wb(2 * k);
  while (cursor < order.size()) {
    const int b = order[cursor];
    const double t_b = t[b];
    const double dt = t_b - t_old;
    if (dt_min < dt) break;
    xcp[b] = d[b] > 0.0 ? upper[b] : lower[b];
    const double zb = xcp[b] - x[b];
    free[b] = 0;
    for (int j = 0; j < 2 * k; ++j) c[j] += dt * p[j];
    const double gb = g[b];
    for (int j = 0; j < 2 * k; ++j) wb[j] = mem.w(b, j);
    if (!mem.apply_m(c, &mc) || !mem.apply_m(p, &mp) || !mem.apply_m(wb, &mwb)) return false;
    f_prime += dt * f_double + gb * gb + mem.theta * gb * zb - gb * dot(wb, mc);
    f_double += -mem.theta * gb * gb - 2.0 * gb * dot(wb, mp) - gb * gb * dot(wb, mwb);
    f_double = std::fmax(f_double, kEpsilon * f_double_initial);
    for (int j = 0; j < 2 * k; ++j) p[j] += gb * wb[j];
    d[b] = 0.0;
    dt_min = -f_prime / f_double;
    t_old = t_b;
    ++cursor;
  }
  dt_min = std::fmax(dt_min, 0.0);
  const double t_final = t_old + dt_min;
  for (int i = 0; i < n; ++i)
    if (free[i] && t[i] >= t_final) xcp[i] = x[i] + t_final * d[i];
  for (int j = 0; j < 2 * k; ++j) c[j] += dt_min * p[j];
  out->x = std::move(xcp);
  out->free = std::move(free);
  out->c = std::move(c);
  return true;
}

// The quadratic model's minimiser over the free variables from the Cauchy
// point (Sherman-Morrison-Woodbury on the compact form), truncated to the box.
bool subspace_minimise(const std::vector<double>& x, const std::vector<double>& g,
                       const std::vector<double>& lower, const std::vector<double>& upper, const CauchyPoint& cp,
                       const Memory& mem, std::vector<double>* out) {
  const int n = static_cast<int>(x.size());
  const int k = mem.k();
  if (k == 0) {
    *out = cp.x;
    return true;
  }
  std::vector<int> free;
  for (int i = 0; i < n; ++i)
    if (cp.free[i]) free.push_back(i);
  if (free.empty()) {
    *out = cp.x;
    return true;
  }
  const int dim = 2 * k;
  const double theta = mem.theta;
  std::vector<double> mc;
  if (!mem.apply_m(cp.c, &mc)) return false;
  std::vector<double> r(free.size()), wi(dim);
  for (size_t slot = 0; slot < free.size(); ++slot) {
    const int i = free[slot];
    for (int j = 0; j < dim; ++j) wi[j] = mem.w(i, j);
    r[slot] = g[i] + theta * (cp.x[i] - x[i]) - dot(wi, mc);
  }
  std::vector<double> v(dim, 0.0);
  for (int j = 0; j < dim; ++j) {
    double acc = 0.0;
    for (size_t slot = 0; slot < free.size(); ++slot) acc += mem.w(free[slot], j) * r[slot];
    v[j] = acc;
  }
  std::vector<double> mv;
  if (!mem.apply_m(v, &mv)) return false;
  std::vector<double> wtw(static_cast<size_t>(dim) * dim, 0.0);
  for (int a = 0; a < dim; ++a)
    for (int b = 0; b < dim; ++b) {
      double acc = 0.0;
      for (int i : free) acc += mem.w(i, a) * mem.w(i, b);
      wtw[a * dim + b] = acc;
    }
  std::vector<double> n_mat(static_cast<size_t>(dim) * dim, 0.0), col(dim), m_col;
  for (int b = 0; b < dim; ++b) {
    for (int a = 0; a < dim; ++a) col[a] = wtw[a * dim + b];
    if (!mem.apply_m(col, &m_col)) return false;
    for (int a = 0; a < dim; ++a) n_mat[a * dim + b] = -m_col[a] / theta;
  }
  for (int a = 0; a < dim; ++a) n_mat[a * dim + a] += 1.0;
  std::vector<double> sol;
  if (!lbfgsb_solve_dense(n_mat, mv, dim, &sol)) return false;
  std::vector<double> d(free.size());
  for (size_t slot = 0; slot < free.size(); ++slot) {
    double acc = 0.0;
    for (int j = 0; j < dim; ++j) acc += mem.w(free[slot], j) * sol[j];
    d[slot] = -(r[slot] / theta + acc / (theta * theta));
  }
  double alpha = 1.0;
  for (size_t slot = 0; slot < free.size(); ++slot) {
    const int i = free[slot];
    if (d[slot] > 0.0 && std::isfinite(upper[i])) {
      alpha = std::fmin(alpha, (upper[i] - cp.x[i]) / d[slot]);
    } else if (d[slot] < 0.0 && std::isfinite(lower[i])) {
      alpha = std::fmin(alpha, (lower[i] - cp.x[i]) / d[slot]);
    }
  }
  alpha = std::clamp(alpha, 0.0, 1.0);
  *out = cp.x;
  for (size_t slot = 0; slot < free.size(); ++slot) {
    const int i = free[slot];
    (*out)[i] = std::clamp(cp.x[i] + alpha * d[slot], lower[i], upper[i]);
  }
  return true;
}

double max_feasible_step(const std::vector<double>& x, const std::vector<double>& dir,
                         const std::vector<double>& lower, const std::vector<double>& upper) {
  double step = kInf;
  for (size_t i = 0; i < x.size(); ++i) {
    if (dir[i] > 0.0 && std::isfinite(upper[i])) {
      step = std::fmin(step, (upper[i] - x[i]) / dir[i]);
    } else if (dir[i] < 0.0 && std::isfinite(lower[i])) {
      step = std::fmin(step, (lower[i] - x[i]) / dir[i]);
    }
  }
  return std::fmax(step, 0.0);
}

double projected_gradient_norm(const std::vector<double>& x, const std::vector<double>& g,
                               const std::vector<double>& lower, const std::vector<double>& upper) {
  double norm = 0.0;
  for (size_t i = 0; i < x.size(); ++i)
    norm = std::fmax(norm, std::fabs(std::clamp(x[i] - g[i], lower[i], upper[i]) - x[i]));
  return norm;
}

}  // namespace

bool lbfgsb_solve_dense(const std::vector<double>& a, const std::vector<double>& b, int dim,
                        std::vector<double>* out) {
  std::vector<double> m = a;
  std::vector<double> x = b;
  for (int col = 0; col < dim; ++col) {
    int pivot = col;
    double best = std::fabs(m[col * dim + col]);
    for (int row = col + 1; row < dim; ++row) {
      const double v = std::fabs(m[row * dim + col]);
      if (v > best) {
        best = v;
        pivot = row;
      }
    }
    if (best < 1e-300) return false;
    if (pivot != col) {
      for (int j = 0; j < dim; ++j) std::swap(m[col * dim + j], m[pivot * dim + j]);
      std::swap(x[col], x[pivot]);
    }
    const double diag = m[col * dim + col];
    for (int row = col + 1; row < dim; ++row) {
      const double factor = m[row * dim + col] / diag;
      if (factor == 0.0) continue;
      for (int j = col; j < dim; ++j) m[row * dim + j] -= factor * m[col * dim + j];
      x[row] -= factor * x[col];
    }
  }
  for (int col = dim - 1; col >= 0; --col) {
    double acc = x[col];
    for (int j = col + 1; j < dim; ++j) acc -= m[col * dim + j] * x[j];
    x[col] = acc / m[col * dim + col];
  }
  *out = std::move(x);
  return true;
}

Lbfgsb::Lbfgsb(const std::vector<double>& x0, std::vector<double> lower, std::vector<double> upper,
               const LbfgsbParams& params)
    : x0_(x0), lower_(std::move(lower)), upper_(std::move(upper)), params_(params),
      n_(static_cast<int>(x0.size())) {
  if (n_ == 0) fail(NB_ERR_MUST_BE_POSITIVE, "x0.len() must be positive");
  if (lower_.size() != x0.size())
    fail(NB_ERR_LENGTH_MISMATCH, "lower: expected " + std::to_string(n_) + ", got " + std::to_string(lower_.size()));
  if (upper_.size() != x0.size())
    fail(NB_ERR_LENGTH_MISMATCH, "upper: expected " + std::to_string(n_) + ", got " + std::to_string(upper_.size()));
  for (int i = 0; i < n_; ++i)
    if (lower_[i] > upper_[i])
      fail(NB_ERR_INVALID_BOUNDS, "bound " + std::to_string(i) + ": lower " + std::to_string(lower_[i]) +
                                      " above upper " + std::to_string(upper_[i]));
  if (params_.memory <= 0) fail(NB_ERR_MUST_BE_POSITIVE, "memory must be positive");
  g_eval_.assign(n_, 0.0);
  task_ = run();
}

Lbfgsb::~Lbfgsb() {
  if (task_.h) task_.h.destroy();
}

Lbfgsb::Eval Lbfgsb::evaluate(const std::vector<double>& x) {
  x_eval_ = x;
  waiting_ = true;
  return Eval{};
}

void Lbfgsb::tell(double f, const double* g) {
  if (!waiting_) return;
  f_eval_ = f;
  for (int i = 0; i < n_; ++i) g_eval_[i] = g[i];
  waiting_ = false;
  task_.h.resume();
}

// minimise (lbfgsb.rs:876-1019), with line_search and zoom inlined: each
// objective evaluation suspends the coroutine until tell().
Lbfgsb::Task Lbfgsb::run() {
  const int n = n_;
  const std::vector<double>& lo = lower_;
  const std::vector<double>& hi = upper_;
  std::vector<double> x(n);
  for (int i = 0; i < n; ++i) x[i] = std::clamp(x0_[i], lo[i], hi[i]);
  co_await evaluate(x);
  double f = f_eval_;
  std::vector<double> grad = g_eval_;
  int evaluations = 1;
  Memory mem(static_cast<size_t>(params_.memory));
  LbfgsbStatus status = LbfgsbStatus::MaxIterations;
  int iterations = 0;
  std::vector<double> direction(n), point(n), target;
  CauchyPoint cp;
  for (int iter = 0; iter < params_.max_iter; ++iter) {
    iterations = iter + 1;
    if (projected_gradient_norm(x, grad, lo, hi) <= params_.pgtol) {
      status = LbfgsbStatus::GradientTolerance;
      break;
    }
    // the Cauchy point, then the subspace step; projected steepest descent
    // when either meets a singular middle matrix
    const bool have = cauchy_point(x, grad, lo, hi, mem, &cp) && subspace_minimise(x, grad, lo, hi, cp, mem, &target);
    bool all_zero = true;
    for (int i = 0; i < n; ++i) {
      direction[i] = have ? target[i] - x[i] : std::clamp(x[i] - grad[i], lo[i], hi[i]) - x[i];
      all_zero = all_zero && direction[i] == 0.0;
    }
    if (all_zero) {
      status = LbfgsbStatus::GradientTolerance;
      break;
    }

    // line_search (lbfgsb.rs:675-779): strong Wolfe, doubling out to the
    // feasible step, then zoom's bisection (801-849)
    bool found = false;
    std::vector<double> x_new, g_new;
    double f_new = 0.0;
    int used = 0;
    const double slope0 = dot(grad, direction);
    const double step_max = std::fmin(max_feasible_step(x, direction, lo, hi), kMaxStep);
    if (slope0 < 0.0 && step_max > 0.0) {
      const int max_evals = params_.max_line_search;
      double alpha_prev = 0.0, f_prev = f, alpha = std::fmin(1.0, step_max);
      bool have_best = false;
      std::vector<double> best_x, best_g;
      double best_f = 0.0;
      // zoom's bracket, when the search hands over to it
      bool zoom = false;
      double z_lo = 0.0, z_flo = 0.0, z_hi = 0.0;
      for (int iteration = 0; iteration < max_evals; ++iteration) {
        for (int i = 0; i < n; ++i) point[i] = std::clamp(x[i] + alpha * direction[i], lo[i], hi[i]);
        co_await evaluate(point);
        const double ft = f_eval_;
        ++used;
        if (!std::isfinite(ft)) {
          alpha *= 0.5;
          if (alpha < 1e-20) break;
          continue;
        }
        const bool sufficient = ft <= f + kWolfeC1 * alpha * slope0;
        if (!sufficient || (iteration > 0 && ft >= f_prev)) {
          zoom = true;
          z_lo = alpha_prev;
          z_flo = f_prev;
          z_hi = alpha;
          break;
        }
        const double slope = dot(g_eval_, direction);
        if (std::fabs(slope) <= -kWolfeC2 * slope0) {
          found = true;
          x_new = point;
          f_new = ft;
          g_new = g_eval_;
          break;
        }
        if (slope >= 0.0) {
          zoom = true;
          z_lo = alpha;
          z_flo = ft;
          z_hi = alpha_prev;
          break;
        }
        if (alpha >= step_max) {  // on the boundary, still descending: the answer
          found = true;
          x_new = point;
          f_new = ft;
          g_new = g_eval_;
          break;
        }
        have_best = true;
        best_x = point;
        best_f = ft;
        best_g = g_eval_;
        alpha_prev = alpha;
        f_prev = ft;
        alpha = std::fmin(alpha * 2.0, step_max);
      }
      if (zoom) {
        const int budget = max_evals - used;
        for (int it = 0; it < budget; ++it) {
          const double a = 0.5 * (z_lo + z_hi);
          if (std::fabs(z_hi - z_lo) < 1e-16) break;
          for (int i = 0; i < n; ++i) point[i] = std::clamp(x[i] + a * direction[i], lo[i], hi[i]);
          co_await evaluate(point);
          const double ft = f_eval_;
          ++used;
          if (!std::isfinite(ft) || ft > f + kWolfeC1 * a * slope0 || ft >= z_flo) {
            z_hi = a;
            continue;
          }
          const double slope = dot(g_eval_, direction);
          if (std::fabs(slope) <= -kWolfeC2 * slope0) {
            found = true;
            x_new = point;
            f_new = ft;
            g_new = g_eval_;
            break;
          }
          if (slope * (z_hi - z_lo) >= 0.0) z_hi = z_lo;
          z_lo = a;
          z_flo = ft;
        }
      } else if (!found && have_best) {
        found = true;
        x_new = best_x;
        f_new = best_f;
        g_new = best_g;
      }
    }
    if (!found) {
      // a stalled line search is usually the model's fault: drop the pairs
      // and retry from projected steepest descent, then give up
      if (mem.k() > 0) {
        mem.reset();
        continue;
      }
      status = LbfgsbStatus::LineSearchFailed;
      break;
    }
    evaluations += used;
    std::vector<double> s(n), y(n);
    for (int i = 0; i < n; ++i) {
      s[i] = x_new[i] - x[i];
      y[i] = g_new[i] - grad[i];
    }
    mem.push(std::move(s), std::move(y));
    const double reduction = f - f_new;
    const double scale = std::fmax(std::fmax(std::fabs(f), std::fabs(f_new)), 1.0);
    x = x_new;
    f = f_new;
    grad = g_new;
    if (reduction <= params_.ftol * scale) {
      status = LbfgsbStatus::ObjectiveTolerance;
      break;
    }
  }
  x_ = std::move(x);
  f_ = f;
  g_ = std::move(grad);
  iterations_ = iterations;
  evaluations_ = evaluations;
  status_ = status;
  co_return;
}

}  // namespace nebula
