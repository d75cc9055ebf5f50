// Entry points of one (n_coef, n_varying) instantiation of stage one's
// kernel (ptmg_impl.cuh), gathered per column count in ptmg_nb<NB>.cu and
// dispatched by ptmg_eval.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

#include "ptmg_device.cuh"

namespace nebula {
namespace device {

struct PtmgOps {
  int (*launch)(const GeneData& d, const PtmgQueue& qu, double* scratch, int grid, cudaStream_t stream);
  int (*resident)(int K);  // CTAs resident at once (whole clusters)
  size_t (*scratch)(int K);
};

PtmgOps ptmg_ops_nb1(int n_varying);
PtmgOps ptmg_ops_nb2(int n_varying);
PtmgOps ptmg_ops_nb3(int n_varying);
PtmgOps ptmg_ops_nb4(int n_varying);
PtmgOps ptmg_ops_nb5(int n_varying);
PtmgOps ptmg_ops_nb6(int n_varying);
PtmgOps ptmg_ops_nb7(int n_varying);
PtmgOps ptmg_ops_nb8(int n_varying);

}  // namespace device
}  // namespace nebula
