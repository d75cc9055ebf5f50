// Stage one: the Poisson-gamma marginal likelihood over [beta, sigma, phi]
// (src/sc/ptmg.rs) and its minimiser, the projected Newton with L-BFGS-B
// behind it (src/sc/nebula.rs minimise_marginal 1075-1112, descend_marginal
// 1132-1170, newton_marginal 1225-1325), then the plan for stage two
// (plan_gene 812-901).
//
// An evaluation is split in two: per-subject sums over the cells (on the
// device for the product, on the CPU for the oracle, both with the same
// summation tree) and the assembly of value, gradient and Hessian from those
// sums (here, shared). The minimiser is a coroutine that asks for evaluations,
// so every gene's search can advance in lockstep with one batched launch per
// round.
#pragma once

#include <coroutine>
#include <vector>

#include "common.hpp"

namespace nebula {

// Per-subject sums of one evaluation at params = [beta, sigma, phi].
// Pass one: cumsumxtb = sum exp(eta) and ylin = sum y eta (positive cells).
// Pass two, with ym = (cumsumy + alpha) / (cumsumxtb + lambda) per subject,
// w = ym e + gamma and g = (gamma + y) / w per cell, the kPtmgScalars sums
//   we, ln w, (gamma + y) ln w, g, 1/w, g/w, g e, g e/w - e/w, g e^2/w
// then x e, g x e, x e (g/w - 1/w), x e g e/w (n_coef each) and the two
// triangles x x' e and x x' e ym (ym g e/w - g).
constexpr int kPtmgScalars = 9;
inline int ptmg_width(int nb) { return kPtmgScalars + 4 * nb + nb * (nb + 1); }

struct PtmgSums {
  std::vector<double> cumsumxtb, ylin;  // K each
  std::vector<double> sums;             // K x ptmg_width(nb)
};

// The scalars every kernel derives from (sigma, phi) (ptmg.rs:288-348).
struct Terms {
  double exps_s, alpha, lambda, gamma, log_lambda, log_gamma, alpha_pr, lambda_pr, alpha_dpr, lambda_dpr;
  Terms(double sigma, double phi);
};

// One gene as stage one reads it.
struct MarginalGene {
  const Shared* sh;
  const GeneCounts* gc;
  const double* totals;  // cumsumy, K
  const double* xy;      // sum over positive cells of x y, n_coef (positive_xy)
};

// sum_i x_i y_i over a gene's positive cells, the count part of the
// fixed-effect gradient (ptmg.rs:825-830); independent of the parameters.
std::vector<double> positive_xy(const Shared& sh, const GeneCounts& gc);

// Value, gradient and row-major Hessian of the negative marginal
// log-likelihood from the per-subject sums (ptmg.rs:739-880, 999-1251).
double ptmg_assemble(const MarginalGene& g, const double* params, const PtmgSums& sums, double* grad,
                     double* hess);

// Reverse-communication minimise_marginal: ask() gives the point to evaluate
// (null when done), tell() its value, gradient and Hessian (any may be
// non-finite). `tabled`: the run has zero-count tables (the reference's
// `zeros` is Some), so every descent is the quasi-Newton L-BFGS-B; otherwise
// the projected Newton runs first and L-BFGS-B takes over where it fails or
// does not improve (descend_marginal, nebula.rs:1132-1170).
class MarginalSearch {
 public:
  MarginalSearch(std::vector<double> start, std::vector<double> lower, std::vector<double> upper, int nb,
                 bool tabled = false);
  ~MarginalSearch();
  MarginalSearch(const MarginalSearch&) = delete;
  MarginalSearch& operator=(const MarginalSearch&) = delete;
  const double* ask() const { return waiting_ ? x_.data() : nullptr; }
  void tell(double f, const double* g, const double* h);
  bool done() const { return !waiting_; }
  // The best point and whether every attempt failed (nebula's is_conv).
  const std::vector<double>& best() const { return best_; }
  bool failed() const { return failed_; }
  int evaluations() const { return evaluations_; }

 private:
  struct Task {
    struct promise_type {
      Task get_return_object() { return Task{std::coroutine_handle<promise_type>::from_promise(*this)}; }
      std::suspend_never initial_suspend() noexcept { return {}; }
      std::suspend_always final_suspend() noexcept { return {}; }
      void return_void() {}
      void unhandled_exception() {}
    };
    std::coroutine_handle<promise_type> h;
  };
  struct Eval {
    MarginalSearch* self;
    bool await_ready() const noexcept { return false; }
    void await_suspend(std::coroutine_handle<>) noexcept {}
    void await_resume() const noexcept {}
  };
  Eval evaluate(const std::vector<double>& x);
  Task run();

  std::vector<double> start_, lower_, upper_;
  int n_, nb_;
  bool tabled_;
  std::vector<double> x_;
  double f_ = 0.0;
  std::vector<double> g_, h_;
  bool waiting_ = false;
  std::vector<double> best_;
  bool failed_ = false;
  int evaluations_ = 0;
  Task task_{};
};

// The bounds and start of stage one for a gene (nebula.rs:837-848).
void marginal_box(const Shared& sh, const GeneCounts& gc, std::vector<double>* start,
                  std::vector<double>* lower, std::vector<double>* upper);

// plan_gene (nebula.rs:812-901) from the finished search.
GenePlan plan_from(const Shared& sh, const GeneCounts& gc, const std::vector<double>& x, bool failed);

bool cholesky_solve(const std::vector<double>& a, int n, const std::vector<double>& b,
                    std::vector<double>* x);

}  // namespace nebula
