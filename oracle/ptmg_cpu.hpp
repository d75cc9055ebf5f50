// ORACLE — test infrastructure only. Stage one on the CPU (see ptmg_cpu.cpp).
#pragma once

#include "common.hpp"
#include "pml_cpu.hpp"
#include "stage_one.hpp"

namespace oracle {

// The per-subject sums of one marginal-likelihood evaluation.
nebula::PtmgSums ptmg_sums(const PmlData& d, const double* beta, double alpha, double lambda, double gamma);

// plan_gene (nebula.rs:812-901) with every evaluation on the CPU; `tabled`:
// the run has zero-count tables, so stage one descends by L-BFGS-B alone.
nebula::GenePlan plan_gene(const nebula::Shared& sh, const nebula::GeneCounts& gc, const double* totals,
                           int* evaluations, bool tabled = false);

}  // namespace oracle
