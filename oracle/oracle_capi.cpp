// ORACLE — test infrastructure only. C-ABI the tests and the CPU-baseline leg
// of bench.py load with ctypes. Never linked by the product library.
#include <cstdint>
#include <vector>

#include "common.hpp"
#include "lbfgsb.hpp"
#include "nbmath.hpp"
#include "pml_cpu.hpp"

#define ORACLE_API extern "C" __attribute__((visibility("default")))

// scalars_out: log_likelihood, log_likelihood_prev, log_det, second_order
// ints_out: convergence, iterations, backtracks, sweeps
ORACLE_API int32_t oracle_opt_pml(const double* design, const double* offset, uint64_t n_cells,
                                  uint32_t n_beta, const double* counts, const uint32_t* cells,
                                  uint64_t n_pos, const uint64_t* subject_start, uint32_t k,
                                  const double* subject_total, const double* beta_init,
                                  const double* log_w_init, double subject, double cell,
                                  int32_t reml, double eps, int32_t ord, int32_t max_iter,
                                  int32_t prior_lognormal, int32_t tabled, double* beta_out, double* log_w_out,
                                  double* information_out, double* scalars_out,
                                  int32_t* ints_out) {
  oracle::PmlData d{design, offset, n_cells, static_cast<int>(n_beta), counts, cells, n_pos,
                    subject_start, static_cast<int>(k), subject_total};
  // the zero-count tables of this design and these offsets, when they apply
  nebula::zero::Tables tables;
  if (tabled && nebula::zero::build_tables(design, offset, subject_start, static_cast<int>(k), static_cast<int>(n_beta),
                                           &tables))
    d.zeros = &tables;
  oracle::PmlParams p;
  p.reml = reml != 0;
  p.eps = eps;
  p.ord = ord;
  p.max_iter = max_iter;
  oracle::PmlResult r;
  if (!oracle::opt_pml(d, beta_init, log_w_init, subject, cell, p,
                       prior_lognormal ? oracle::Prior::LogNormal : oracle::Prior::Gamma, &r))
    return 4;
  for (uint32_t j = 0; j < n_beta; ++j) beta_out[j] = r.beta[j];
  for (uint32_t s = 0; s < k; ++s) log_w_out[s] = r.log_w[s];
  for (uint32_t j = 0; j < n_beta * n_beta; ++j) information_out[j] = r.information[j];
  scalars_out[0] = r.log_likelihood;
  scalars_out[1] = r.log_likelihood_prev;
  scalars_out[2] = r.log_det;
  scalars_out[3] = r.second_order;
  ints_out[0] = r.convergence;
  ints_out[1] = r.iterations;
  ints_out[2] = r.backtracks;
  ints_out[3] = r.sweeps;
  return 0;
}

ORACLE_API double oracle_pml_objective_gradient(const double* design, const double* offset,
                                                uint64_t n_cells, uint32_t n_beta,
                                                const double* counts, const uint32_t* cells,
                                                uint64_t n_pos, const uint64_t* subject_start,
                                                uint32_t k, const double* subject_total,
                                                const double* beta, const double* log_w,
                                                double subject, double cell, double* gradient) {
  oracle::PmlData d{design, offset, n_cells, static_cast<int>(n_beta), counts, cells, n_pos,
                    subject_start, static_cast<int>(k), subject_total};
  return oracle::pml_objective_gradient(d, beta, log_w, subject, cell, gradient);
}

ORACLE_API double oracle_min_eigenvalue(const double* a, uint32_t n) {
  return oracle::min_eigenvalue(a, static_cast<int>(n));
}

// The shared exp/log of nbmath.hpp over an array, for their accuracy tests:
// which = 0 nb_exp, 1 nb_log, 2 nb_exp_tab, 3 nb_log_tab.
ORACLE_API void oracle_nbmath(int32_t which, const double* x, double* out, uint64_t n) {
  for (uint64_t i = 0; i < n; ++i) {
    switch (which) {
      case 0: out[i] = nebula::nb_exp(x[i]); break;
      case 1: out[i] = nebula::nb_log(x[i]); break;
      case 2: out[i] = nebula::nb_exp_tab(x[i], &nebula::kNbTables); break;
      default: out[i] = nebula::nb_log_tab(x[i], &nebula::kNbTables); break;
    }
  }
}

// The zero-count tables (zero_tables.hpp) of one group holding every cell of
// log offsets log_o (n >= 32), evaluated at s[0..m): out[i * count + j] is sum
// `from + j` (0 = L ... 5 = E) at s[i]; range_out = {s_lo, s_hi}. Returns 0,
// or 1 when no tables were built.
ORACLE_API int32_t oracle_zero_eval(const double* log_o, uint64_t n, const double* s, uint64_t m, int32_t from,
                                    int32_t count, double* out, double* range_out) {
  std::vector<double> design(n, 1.0);
  const uint64_t fid[2] = {0, n};
  nebula::zero::Tables t;
  if (!nebula::zero::build_tables(design.data(), log_o, fid, 1, 1, &t) || t.groups.size() != 1) return 1;
  for (uint64_t i = 0; i < m; ++i)
    nebula::zero::eval(t.groups[0], t.index.data(), t.panels.data(), s[i], from, count, out + i * count);
  range_out[0] = t.groups[0].s_lo;
  range_out[1] = t.groups[0].s_hi;
  return 0;
}

// How build_tables groups a design: returns the number of tabled groups (-1
// when no tables are built); rows_out (n_cells) gets each group's design row
// cell, loose_out (n_cells) the loose cells, *n_loose their number.
ORACLE_API int32_t oracle_zero_groups(const double* design, const double* log_offset, const uint64_t* subject_start,
                                      uint32_t k, uint32_t n_coef, int64_t* rows_out, uint32_t* loose_out,
                                      uint64_t* n_loose) {
  nebula::zero::Tables t;
  if (!nebula::zero::build_tables(design, log_offset, subject_start, static_cast<int>(k), static_cast<int>(n_coef),
                                  &t))
    return -1;
  for (size_t g = 0; g < t.groups.size(); ++g) rows_out[g] = t.groups[g].row;
  for (size_t i = 0; i < t.loose.size(); ++i) loose_out[i] = t.loose[i];
  *n_loose = t.loose.size();
  return static_cast<int32_t>(t.groups.size());
}

// The stage-one quasi-Newton (lbfgsb.hpp) on an objective the caller
// evaluates: fg(x, n, grad_out, ctx) returns the value at x and writes the
// gradient. x_out (n) and *f_out receive the result, ints_out its status
// (LbfgsbStatus), iterations and evaluations. Returns 0, or the NB_ERR_* code
// of a rejected argument (its message into err).
typedef double (*oracle_fg)(const double* x, uint32_t n, double* grad, void* ctx);
ORACLE_API int32_t oracle_lbfgsb(oracle_fg fg, void* ctx, const double* x0, uint32_t n, const double* lower,
                                 uint32_t n_lower, const double* upper, uint32_t n_upper, int32_t memory,
                                 double ftol, double pgtol, int32_t max_iter, int32_t max_line_search,
                                 double* x_out, double* f_out, int32_t* ints_out, char* err, uint64_t err_len) {
  try {
    nebula::LbfgsbParams p;
    p.memory = memory;
    p.ftol = ftol;
    p.pgtol = pgtol;
    p.max_iter = max_iter;
    p.max_line_search = max_line_search;
    nebula::Lbfgsb search(std::vector<double>(x0, x0 + n), std::vector<double>(lower, lower + n_lower),
                          std::vector<double>(upper, upper + n_upper), p);
    std::vector<double> g(n);
    while (const double* x = search.ask()) {
      const double f = fg(x, n, g.data(), ctx);
      search.tell(f, g.data());
    }
    for (uint32_t i = 0; i < n; ++i) x_out[i] = search.x()[i];
    *f_out = search.f();
    ints_out[0] = static_cast<int32_t>(search.status());
    ints_out[1] = search.iterations();
    ints_out[2] = search.evaluations();
    return 0;
  } catch (const nebula::NbError& e) {
    if (err && err_len) {
      const size_t m = std::min<size_t>(err_len - 1, e.message.size());
      for (size_t i = 0; i < m; ++i) err[i] = e.message[i];
      err[m] = 0;
    }
    return e.code;
  }
}

// solve_dense of the quasi-Newton (lbfgsb.rs:317-361); returns 0, or 1 when a
// pivot underflows.
ORACLE_API int32_t oracle_lbfgsb_solve_dense(const double* a, const double* b, uint32_t dim, double* x_out) {
  std::vector<double> x;
  if (!nebula::lbfgsb_solve_dense(std::vector<double>(a, a + dim * dim), std::vector<double>(b, b + dim),
                                  static_cast<int>(dim), &x))
    return 1;
  for (uint32_t i = 0; i < dim; ++i) x_out[i] = x[i];
  return 0;
}
