// Stage one (the marginal likelihood) and the stage-two plan; see
// stage_one.cpp for the reference lines each piece follows.
#pragma once

#include <vector>

#include "common.hpp"

namespace nebula {

// One gene in the layout the marginal-likelihood kernels read (ptmg.rs:75-91
// GeneData plus the PtmgScratch buffers, ptmg.rs:217-275).
struct PtmgGene {
  const double* design;
  const double* log_offset;
  const uint64_t* fid;
  size_t n_cells;
  int nb, k;
  const double* counts;
  const uint32_t* cells;
  size_t n_pos;
  const double* subject_totals;
  std::vector<double> y_cell, extb, cumsumxtb;
  PtmgGene(const Shared& sh, const GeneCounts& gc, const double* totals);
};

// Negative marginal log-likelihood and gradient at [beta, sigma, phi]
// (nebula:::ptmg_ll_der, ptmg.rs:568).
double ptmg_value_gradient(PtmgGene& g, const double* params, double* grad);
// ... and the Hessian, row-major (n_coef+2)^2 (ptmg.rs:615).
double ptmg_value_gradient_hessian(PtmgGene& g, const double* params, double* grad,
                                   double* hess);

std::vector<double> minimise_marginal(PtmgGene& gene, const std::vector<double>& start,
                                      const std::vector<double>& lower,
                                      const std::vector<double>& upper, bool* failed);

GenePlan plan_gene(const Shared& sh, const GeneCounts& gc, const double* totals);

bool cholesky_solve(const std::vector<double>& a, int n, const std::vector<double>& b,
                    std::vector<double>* x);

}  // namespace nebula
