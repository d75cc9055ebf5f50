// Powell's BOBYQA (bound-constrained derivative-free minimisation) with the
// set-up NLopt 2.7.1 wraps around it: the default initial step, the rescaling
// that equalises those steps, rhobeg from the step and rhoend = xtol_rel *
// rhobeg. For the same objective values it asks for the same points, in the
// same order, as nloptr::bobyqa (the reference pins this against nloptr traces:
// src/numeric/bobyqa.rs:2926-2972, tests/data/e2e/bobyqa_*.csv).
//
// The objective is reverse-communicated. The search runs as a C++20 coroutine
// that suspends wherever Powell's code calls CALFUN (PRELIM, the trust-region
// step and RESCUE), so thousands of per-gene searches can wait on one batched
// device launch. `ask()` gives the pending point, `tell()` its value.
//
// Reference: src/numeric/bobyqa.rs:318-560 (set-up, ask/tell/result),
// :641-1547 (bobyqb), :1581-1986 (rescue), :2007-2423 (trsbox),
// :2438-2710 (altmov), :2722-2788 (update).
#pragma once

#include <coroutine>
#include <vector>

namespace nebula {

enum class BobyqaStatus : int {
  Running = 0,
  XtolReached = 4,      // NLopt XTOL_REACHED
  MaxevalReached = 5,   // NLopt MAXEVAL_REACHED
  Success = 1,          // NLopt SUCCESS
  RoundoffLimited = -4  // NLopt ROUNDOFF_LIMITED
};

struct BobyqaResult {
  std::vector<double> x;
  double f;
  int evaluations;
  BobyqaStatus status;
};

class Bobyqa {
 public:
  // Sets the search up as nlopt_optimize + bobyqa do. `ok()` is false when the
  // box is too narrow for the initial radius (NLopt refuses it).
  //
  // `radius_scale` < 1 starts the trust region at that fraction of NLopt's
  // initial radius while rhoend stays xtol_rel times the unscaled radius: a
  // search from a start already close to the optimum skips the coarse radii
  // and ends at the same final resolution. 1 is NLopt's search exactly.
  Bobyqa(const double* x0, const double* lower, const double* upper, int n,
         double xtol_rel = 1e-6, int maxeval = 1000, double radius_scale = 1.0);
  ~Bobyqa();
  Bobyqa(const Bobyqa&) = delete;
  Bobyqa& operator=(const Bobyqa&) = delete;

  bool ok() const { return ok_; }
  // The point awaiting a value, on the caller's scale, or nullptr when done.
  const double* ask() const;
  void tell(double value);
  bool done() const;
  BobyqaResult result() const;
  int n() const { return n_; }

 private:
  struct Task {
    struct promise_type {
      Task get_return_object() {
        return Task{std::coroutine_handle<promise_type>::from_promise(*this)};
      }
      std::suspend_never initial_suspend() noexcept { return {}; }
      std::suspend_always final_suspend() noexcept { return {}; }
      void return_void() {}
      void unhandled_exception() {}
    };
    std::coroutine_handle<promise_type> h;
  };
  // Suspends until tell() supplies the value at x_ (already rescaled into
  // pending_ by request()).
  struct Eval {
    Bobyqa* self;
    bool await_ready() const noexcept { return false; }
    void await_suspend(std::coroutine_handle<>) noexcept {}
    double await_resume() const noexcept { return self->f_; }
  };
  Eval request();
  bool stop_evals() const { return maxeval_ > 0 && nevals_ >= maxeval_; }
  Task run();

  // index helpers, one-based (k, j) into column-major arrays
  int ix(int k, int j) const { return (k - 1) + (j - 1) * npt_; }
  int ib(int k, int j) const { return (k - 1) + (j - 1) * ndim_; }
  int iz(int k, int j) const { return (k - 1) + (j - 1) * npt_; }

  bool ok_ = true;
  int n_ = 0, npt_ = 0, ndim_ = 0;
  std::vector<double> s_;        // NLopt rescaling: the search works in x / s
  std::vector<double> xl_, xu_;  // rescaled bounds, one-based
  double rhobeg_ = 0, rhoend_ = 0;
  int maxeval_ = 0, nevals_ = 0;
  std::vector<double> x_;        // point under evaluation, rescaled, one-based
  std::vector<double> pending_;  // the same point on the caller's scale
  double f_ = 0;
  bool waiting_ = false;
  BobyqaStatus rc_ = BobyqaStatus::Running;
  double minf_ = 0;
  std::vector<double> xbest_;
  std::vector<double> sl0_, su0_;  // initial sl/su computed in the constructor
  Task task_{};
};

}  // namespace nebula
