// Stage two's search over the variance components and the profile objective
// it minimises, plus stage three's finishing arithmetic and the final
// unscaling. Shared by the device driver (which batches every gene's pending
// evaluation into one launch) and the CPU oracle (which evaluates each point
// as it is asked for).
//
// Reference: src/sc/nebula.rs StageTwoSearch 1568-1951, VarianceObjective
// 1365-1505, variance_bounds 2003-2015, finish_gene 918-1000,
// cholesky_inverse 2107-2122, assemble 2233-2277; src/gpu/stage_two.rs
// count_histogram / histogram_tail 746-766.
#pragma once

#include <memory>
#include <optional>
#include <limits>
#include <vector>

#include "bobyqa.hpp"
#include "common.hpp"

namespace nebula {

class NelderMead;  // the one-component simplex of NEBULA-LN's restricted refit

// Reverse-communication stage-two search (nebula.rs:1568-1951). Two
// components run BOBYQA from the clamped start; a rejected evaluation at a
// raised Laplace order restarts the pass at order one. One component runs
// the clamped start, a bounded Nelder-Mead (restarted once off a bound), the
// clamped minimiser once more, and three quadratic polish stencils.
class StageTwoSearch {
 public:
  // `radius_scale` < 1 narrows the first BOBYQA pass's initial trust region
  // (Bobyqa's radius_scale) for a start believed close to the optimum; a
  // restarted pass uses the full radius.
  StageTwoSearch(const std::vector<double>& start, const std::vector<double>& lower,
                 const std::vector<double>& upper, int ord, double radius_scale = 1.0);
  ~StageTwoSearch();
  int order() const { return order_; }
  bool done() const { return stage_ == Stage::Done; }
  // The points awaiting values (one for BOBYQA, 3^n for a polish stencil).
  const std::vector<std::vector<double>>& ask() const { return asked_; }
  void tell(const std::vector<double>& values);
  // The minimiser and whether the optimiser reported failure; nullopt if the
  // search was abandoned.
  std::optional<std::pair<std::vector<double>, bool>> result() const;
  int evaluations() const { return evaluations_; }
  // The smallest finite objective value told so far (+inf if none).
  double best_value() const { return best_value_; }

 private:
  enum class Stage { Start, NelderMead, Check, Polish, Bobyqa, Done };
  std::vector<double> clamped(const std::vector<double>& x) const;
  void begin_pass();
  void ask_bobyqa();
  void end_pass(std::optional<std::vector<double>> found);
  void ask_simplex();
  void begin_polish();
  std::optional<std::vector<double>> fit_polish(const std::vector<double>& values) const;

  std::vector<double> lower_, upper_, start_;
  int order_;
  double radius_scale_ = 1.0;
  bool invalid_ = false;
  Stage stage_ = Stage::Start;
  std::vector<std::vector<double>> asked_;
  std::unique_ptr<Bobyqa> bobyqa_;
  std::unique_ptr<NelderMead> simplex_;
  std::vector<double> best_;
  size_t width_ = 0;
  std::vector<double> step_;
  std::vector<std::vector<double>> offsets_;
  std::optional<std::vector<double>> found_;
  bool restarted_ = false;
  std::optional<std::pair<std::vector<double>, double>> pinned_;
  bool failed_ = false;
  int evaluations_ = 0;
  double best_value_ = std::numeric_limits<double>::infinity();
};

// The profile objective of one gene at one Laplace order
// (nebula.rs:1365-1505 VarianceObjective).
struct VarianceObjective {
  int intercept = 0;
  double n_cells = 0, n_subjects = 0;
  double n_positive = 0, n_one = 0, n_two = 0;
  std::optional<double> fixed_cell;
  // Distinct counts other than one and two with their multiplicities
  // (stage_two.rs:746-761).
  std::vector<std::pair<double, double>> histogram;

  static VarianceObjective make(const Shared& sh, const GeneCounts& gc, std::optional<double> fixed_cell);
  // Resolves x into (subject, cell, beta_init); false where the objective is
  // infinite without a fit (nebula.rs:1404-1416).
  bool request(const std::vector<double>& x, const std::vector<double>& beta_start, double* subject,
               double* cell, std::vector<double>* beta) const;
  // sum lgamma(y + cell) over the positive counts other than one and two,
  // one lgamma per distinct count (stage_two.rs:764-766).
  double tail(double cell) const;
  // The negated profile log-likelihood (nebula.rs:1452-1477).
  double assemble(double subject, double cell, const InnerFit& fit, double tail) const;
};

// The box the search runs in (nebula.rs:2003-2015).
void variance_bounds(const Params& p, bool fixed_cell, std::vector<double>* lower,
                     std::vector<double>* upper);

// Applies the stage-two result to the plan: the final (sigma, gamma) and the
// convergence code carried into stage three (nebula.rs:925-946).
void apply_refit(const GenePlan& plan, const std::optional<std::optional<std::pair<std::vector<double>, bool>>>& refit,
                 double* sigma, double* gamma, int* convergence);

// Stage three's finish from the final inner fit (nebula.rs:969-999).
GeneOutcome finish_gene(const Shared& sh, double sigma, double gamma, int convergence,
                        const FinalFit& fit);

double min_eigenvalue(const double* a, int n);

// Unscales and packs the outcomes into the caller's nb_fit (nebula.rs:2233-2277).
void assemble_fit(const Shared& sh, const std::vector<GeneOutcome>& outcomes,
                  const std::vector<size_t>& kept, nb_fit* out);

}  // namespace nebula
