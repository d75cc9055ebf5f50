// Box-constrained limited-memory BFGS as the reference runs it for stage one
// (src/numeric/lbfgsb.rs: Byrd, Lu, Nocedal and Zhu 1995 with the compact
// representation B = theta I - W M W', the generalised Cauchy point and the
// direct primal subspace minimisation, and a bisecting strong-Wolfe line
// search in place of the Fortran's dcsrch), restated in reverse
// communication: ask() gives the point whose value and gradient the search
// needs next, tell() hands them in. The stage-one search uses it for tabled
// designs and when its projected Newton fails (src/sc/nebula.rs:1132-1170).
#pragma once

#include <coroutine>
#include <vector>

namespace nebula {

// LbfgsbParams (lbfgsb.rs:52-78); the defaults are scipy's, ftol NEBULA's.
struct LbfgsbParams {
  int memory = 10;
  double ftol = 1e-6;
  double pgtol = 1e-5;
  int max_iter = 200;
  int max_line_search = 20;
};

// LbfgsbStatus (lbfgsb.rs:86-101).
enum class LbfgsbStatus { GradientTolerance = 0, ObjectiveTolerance = 1, MaxIterations = 2, LineSearchFailed = 3 };

class Lbfgsb {
 public:
  // minimise's argument checks (lbfgsb.rs:894-921) throw NbError:
  // NB_ERR_MUST_BE_POSITIVE for an empty start or zero memory,
  // NB_ERR_LENGTH_MISMATCH, NB_ERR_INVALID_BOUNDS for lower > upper.
  Lbfgsb(const std::vector<double>& x0, std::vector<double> lower, std::vector<double> upper,
         const LbfgsbParams& params);
  ~Lbfgsb();
  Lbfgsb(const Lbfgsb&) = delete;
  Lbfgsb& operator=(const Lbfgsb&) = delete;

  // The point to evaluate next, or null once the search has stopped.
  const double* ask() const { return waiting_ ? x_eval_.data() : nullptr; }
  // The objective and gradient at the point ask() gave (either may be
  // non-finite; a non-finite value is a failed evaluation).
  void tell(double f, const double* g);
  bool done() const { return !waiting_; }

  // LbfgsbResult (lbfgsb.rs:107-120), valid once done().
  const std::vector<double>& x() const { return x_; }
  double f() const { return f_; }
  const std::vector<double>& gradient() const { return g_; }
  int iterations() const { return iterations_; }
  int evaluations() const { return evaluations_; }
  LbfgsbStatus status() const { return status_; }

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
    bool await_ready() const noexcept { return false; }
    void await_suspend(std::coroutine_handle<>) noexcept {}
    void await_resume() const noexcept {}
  };
  Eval evaluate(const std::vector<double>& x);
  Task run();

  std::vector<double> x0_, lower_, upper_;
  LbfgsbParams params_;
  int n_ = 0;
  std::vector<double> x_eval_, g_eval_;
  double f_eval_ = 0.0;
  bool waiting_ = false;
  std::vector<double> x_, g_;
  double f_ = 0.0;
  int iterations_ = 0, evaluations_ = 0;
  LbfgsbStatus status_ = LbfgsbStatus::MaxIterations;
  Task task_{};
};

// solve_dense (lbfgsb.rs:317-361): Gaussian elimination with partial
// pivoting of a row-major dim x dim system; false when a pivot is below
// 1e-300.
bool lbfgsb_solve_dense(const std::vector<double>& a, const std::vector<double>& b, int dim,
                        std::vector<double>* x);

}  // namespace nebula
