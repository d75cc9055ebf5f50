// Inputs and outputs of the warm-start network (mlp_layout.hpp): the
// summary features of a kept gene and the stage-two start they predict.
#pragma once

#include <vector>

#include "common.hpp"
#include "mlp_layout.hpp"

namespace nebula {

// The 12 features of one gene, in order: log mean count per cell, log
// variance of the counts per cell, zero fraction, log stage-one sigma, log
// stage-one gamma, log(1 + largest count), share of positive counts equal to
// one, variance over subjects of log((total + 1/2) / cells), log cells per
// subject, log subjects, stage one's Laplace order, log mean positive count.
void warm_features(const Shared& sh, const GeneCounts& gc, const double* subject_totals, const GenePlan& plan,
                   float* out);

// The built-in network (trained by edge_rs_b200/warm_start.py on plain fits
// of synthetic genes; mlp::kParams floats).
const float* builtin_mlp_params();

}  // namespace nebula
