// Entry points of one (n_coef, n_varying) instantiation of the fit kernels
// (pml_fit_impl.cuh), gathered per column count in pml_fit_nb<NB>.cu and
// dispatched by pml_fit.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

#include "pml_device.cuh"

namespace nebula {
namespace device {

struct FitOps {
  size_t (*smem)(int K);
  int (*launch)(const GeneData& d, const FitControl& ctl, const FitRequest* req, FitResult* res,
                const int32_t* n_req, int32_t* counter, int grid, int cluster, cudaStream_t stream);
  int (*launch_queue)(const GeneData& d, const FitControl& ctl, const FitQueue& qu, int grid, int cluster,
                      cudaStream_t stream);
  int (*blocks)(int K);
  int (*clusters)(int K, int cluster);
  int (*queue_clusters)(int K, int cluster);
};

// The instantiation for NB columns of which n_varying vary within subjects
// (0 <= n_varying <= NB); all null outside that range.
FitOps fit_ops_nb1(int n_varying);
FitOps fit_ops_nb2(int n_varying);
FitOps fit_ops_nb3(int n_varying);
FitOps fit_ops_nb4(int n_varying);
FitOps fit_ops_nb5(int n_varying);
FitOps fit_ops_nb6(int n_varying);
FitOps fit_ops_nb7(int n_varying);
FitOps fit_ops_nb8(int n_varying);

}  // namespace device
}  // namespace nebula
