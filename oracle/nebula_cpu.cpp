// ORACLE — test infrastructure only. The reference's CPU nebula_sparse
// (src/sc/nebula.rs:434-473 fit_genes, 1014-1033 fit_gene, 1972-1991
// refine_variance): each gene runs stage one, then stage two with every
// objective evaluation an FP64 CPU opt_pml (pml_cpu.cpp) evaluated as soon as
// the search asks, then the stage-three fit; genes run in parallel over host
// threads like rayon's par_iter. Used by the tests as the parity reference
// for nebula_sparse_cuda and by bench.py as the timed CPU baseline.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>
#include <thread>

#include "common.hpp"
#include "pml_cpu.hpp"
#include "ptmg_cpu.hpp"
#include "search.hpp"
#include "special.hpp"
#include "stage_one.hpp"

#define ORACLE_API extern "C" __attribute__((visibility("default")))

namespace {

using namespace nebula;

oracle::PmlData pml_view(const Shared& sh, const GeneCounts& gc, const double* totals,
                         const zero::Tables* zeros) {
  return oracle::PmlData{sh.design.data(), sh.log_offset.data(), sh.n_cells, sh.n_coef,
                         gc.counts.data(), gc.cells.data(), gc.counts.size(), sh.fid.data(),
                         sh.n_subjects, totals, zeros};
}

struct GeneStats {
  long evaluations = 0, sweeps = 0;
};

GeneOutcome fit_gene_cpu(const Shared& sh, const CsrView& csr, const std::vector<double>& totals,
                         size_t g, const zero::Tables* zeros, GeneStats* stats) {
  const int k = sh.n_subjects;
  const double* tot = &totals[g * k];
  GeneCounts gc = positive_indices(csr, g);
  int marginal_evaluations = 0;
  GenePlan plan = oracle::plan_gene(sh, gc, tot, &marginal_evaluations, zeros != nullptr);
  oracle::PmlData data = pml_view(sh, gc, tot, zeros);
  std::optional<std::optional<std::pair<std::vector<double>, bool>>> refit;
  if (plan.refit != Refit::None) {
    std::optional<double> fixed_cell;
    std::vector<double> start;
    if (plan.refit == Refit::Both) {
      start = {plan.sigma, plan.gamma};
    } else {
      start = {plan.sigma};
      fixed_cell = plan.gamma;
    }
    std::vector<double> lower, upper;
    variance_bounds(sh.params, fixed_cell.has_value(), &lower, &upper);
    StageTwoSearch search(start, lower, upper, plan.ord);
    VarianceObjective objective = VarianceObjective::make(sh, gc, fixed_cell);
    while (!search.done()) {
      const auto& points = search.ask();
      std::vector<double> values;
      values.reserve(points.size());
      for (const auto& x : points) {
        double subject, cell;
        std::vector<double> beta;
        double v = std::numeric_limits<double>::infinity();
        if (objective.request(x, plan.beta_start, &subject, &cell, &beta)) {
          oracle::PmlParams p;
          p.reml = sh.params.reml;
          p.eps = sh.params.eps;
          p.ord = search.order();
          oracle::PmlResult r;
          if (oracle::opt_pml(data, beta.data(), nullptr, subject, cell, p, oracle::Prior::Gamma, &r)) {
            InnerFit fit{r.log_likelihood, r.log_likelihood_prev, r.log_det, r.second_order};
            // the lgamma tail over distinct counts (stage_two.rs:746-766), which the
            // reference pins to the per-count sum of nebula.rs:1429-1437 at 1e-14
            v = objective.assemble(subject, cell, fit, objective.tail(cell));
            stats->sweeps += r.sweeps;
          }
        }
        ++stats->evaluations;
        values.push_back(v);
      }
      search.tell(values);
    }
    refit = search.result();
  }
  double sigma, gamma;
  int convergence;
  apply_refit(plan, refit, &sigma, &gamma, &convergence);
  // stage three (nebula.rs:948-967)
  oracle::PmlParams p;
  p.reml = sh.params.reml;
  p.eps = sh.params.eps;
  p.ord = 1;
  std::vector<double> beta_start = plan.beta_start;
  beta_start[sh.intercept] -= sigma / 2.0;
  oracle::PmlResult r;
  if (!oracle::opt_pml(data, beta_start.data(), nullptr, sigma, gamma, p, oracle::Prior::Gamma, &r))
    fail(NB_ERR_INVALID_ARGUMENT, "opt_pml rejected the final variance components");
  stats->sweeps += r.sweeps;
  FinalFit ff{r.beta, r.information, r.log_likelihood, r.iterations, r.backtracks};
  return finish_gene(sh, sigma, gamma, convergence, ff);
}

void write_err(char* err, size_t len, const std::string& msg) {
  if (!err || len == 0) return;
  size_t n = std::min(len - 1, msg.size());
  std::memcpy(err, msg.data(), n);
  err[n] = 0;
}

}  // namespace

// The CPU nebula_sparse over `threads` host threads (0 = all cores).
// work_out (may be null): evaluations, sweeps, genes.
ORACLE_API int32_t oracle_nebula_sparse(const nb_csr* counts, const uint64_t* subject_id,
                                        const double* design, uint32_t n_coef,
                                        const double* offset, const nb_params* params,
                                        int32_t threads, nb_fit* out, int64_t* work_out,
                                        char* err, size_t err_len) {
  try {
    Prepared prep = prepare(counts, subject_id, design, n_coef, offset, params);
    const size_t n = prep.kept.size();
    // the run's zero-count tables, built once (nebula.rs:641, zeros.rs:219)
    const Shared& sh = prep.shared;
    zero::Tables tables;
    const bool tabled = zero::build_tables(sh.design.data(), sh.log_offset.data(), sh.fid.data(), sh.n_subjects,
                                           sh.n_coef, &tables, threads);
    std::vector<GeneOutcome> outcomes(n);
    std::vector<GeneStats> stats(n);
    std::vector<int> failed(n, 0);
    std::vector<NbError> errors(n);
    int nt = threads > 0 ? threads : static_cast<int>(std::thread::hardware_concurrency());
    nt = std::max(1, std::min<int>(nt, static_cast<int>(n)));
    std::atomic<size_t> next{0};
    auto worker = [&]() {
      for (;;) {
        size_t i = next.fetch_add(1);
        if (i >= n) return;
        try {
          outcomes[i] = fit_gene_cpu(prep.shared, prep.counts, prep.totals, prep.kept[i],
                                     tabled ? &tables : nullptr, &stats[i]);
        } catch (const NbError& e) {
          failed[i] = 1;
          errors[i] = e;
        }
      }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    for (size_t i = 0; i < n; ++i)
      if (failed[i]) throw errors[i];
    assemble_fit(prep.shared, outcomes, prep.kept, out);
    if (work_out) {
      int64_t ev = 0, sw = 0;
      for (const auto& s : stats) {
        ev += s.evaluations;
        sw += s.sweeps;
      }
      work_out[0] = ev;
      work_out[1] = sw;
      work_out[2] = static_cast<int64_t>(n);
    }
    return NB_OK;
  } catch (const NbError& e) {
    write_err(err, err_len, e.message);
    return e.code;
  }
}
