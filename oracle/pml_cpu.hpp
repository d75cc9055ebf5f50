// ORACLE — test infrastructure only. A plain FP64 CPU restatement of the
// reference's penalised NB-gamma inner fit (opt_pml), used by tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg to check and time
// the CUDA path. Nothing in the product links or calls it.
//
// Follows src/sc/pml.rs of edge-rs 0.4.0: optimise 1614-1800, sweep_width
// 1419-1590 (dense sweep, no zero-count tables), laplace_correction
// 1828-1919, ldlt_solve 1940-2021, determinant 2036-2069, min_eigenvalue
// 2084-2134, check_convergence 1111-1139.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include "zero_tables.hpp"

namespace oracle {

// Widest design the oracle's per-cell row buffers hold (the reference's CPU
// path has no width cap; its e2e sets reach 13 columns).
constexpr int kMaxRow = 64;

// One gene in the layout of PmlData (pml.rs:122-136).
struct PmlData {
  const double* design;  // row-major n_cells x n_beta
  const double* offset;  // log offset per cell
  size_t n_cells;
  int n_beta;
  const double* counts;      // positive counts, increasing cell order
  const uint32_t* cells;     // their cells
  size_t n_pos;
  const uint64_t* subject_start;  // k + 1 boundaries
  int k;
  const double* subject_total;    // k
  // the run's zero-count tables (zeros.rs), or null to sweep every cell
  const nebula::zero::Tables* zeros = nullptr;
};

// The design columns that vary within some subject (increasing) and each
// column's index among them (-1 for one constant within every subject); the
// sweeps sum only the varying columns per cell (pml_cpu.cpp, ptmg_cpu.cpp).
struct Split {
  std::vector<int> varying, vpos;
};
Split split_columns(const PmlData& d);
// Subject s's design row (zeros for a subject without cells).
std::vector<double> subject_row(const PmlData& d, int s);
// Cell r's varying design values into x; returns how many.
int varying_row(const PmlData& d, const Split& sp, size_t r, double* x);

struct PmlParams {
  bool reml = false;
  double eps = 1e-6;
  int ord = 1;
  int max_iter = 50;
  int max_backtrack = 10;
};

struct PmlResult {
  std::vector<double> beta, log_w, information;
  double log_likelihood = 0, log_likelihood_prev = 0, log_det = 0, second_order = 0;
  int convergence = 1, iterations = 0, backtracks = 0;
  int sweeps = 0;  // cell passes, for the work model
};

enum class Prior { Gamma, LogNormal };

// opt_pml (pml.rs:468) with the gamma prior, or opt_pml_nbm (pml.rs:528) with
// the log-normal one. log_w_init may be null (zeros). Returns false on the
// argument errors the reference reports (non-positive gamma or subject).
bool opt_pml(const PmlData& data, const double* beta_init, const double* log_w_init,
             double subject, double cell, const PmlParams& params, Prior prior, PmlResult* out);

double min_eigenvalue(const double* a, int n);

// Start of each subject's run of positive counts (pml.rs:1155-1160).
std::vector<size_t> positive_runs(const PmlData& d);
int check_convergence(const PmlResult& r, const PmlParams& p, bool at_bound, int initial);

// pml_log_likelihood_gradient (pml.rs:573-615): the negated objective and
// gradient at a point, with nebula's Gamma(alpha, alpha) reading of `subject`.
double pml_objective_gradient(const PmlData& data, const double* beta, const double* log_w,
                              double subject, double cell, double* gradient);

}  // namespace oracle
