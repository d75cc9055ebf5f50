// Dispatch of the fit kernels (pml_fit_impl.cuh) by design width and by how
// many columns vary within subjects (GeneData.n_varying).
#include "pml_device.cuh"
#include "pml_fit_ops.cuh"

namespace nebula {
namespace device {
namespace {

FitOps ops(int n_coef, int n_varying) {
  switch (n_coef) {
    case 1: return fit_ops_nb1(n_varying);
    case 2: return fit_ops_nb2(n_varying);
    case 3: return fit_ops_nb3(n_varying);
    case 4: return fit_ops_nb4(n_varying);
    case 5: return fit_ops_nb5(n_varying);
    case 6: return fit_ops_nb6(n_varying);
    case 7: return fit_ops_nb7(n_varying);
    case 8: return fit_ops_nb8(n_varying);
    default: return FitOps{};
  }
}

}  // namespace

size_t fit_smem_bytes(int n_subjects, int n_coef, int n_varying) {
  const FitOps o = ops(n_coef, n_varying);
  return o.smem ? o.smem(n_subjects) : 0;
}

int fit_blocks_per_sm(int n_subjects, int n_coef, int n_varying) {
  const FitOps o = ops(n_coef, n_varying);
  return o.blocks ? o.blocks(n_subjects) : 0;
}

int fit_max_clusters(int n_subjects, int n_coef, int n_varying, int cluster) {
  const FitOps o = ops(n_coef, n_varying);
  return o.clusters ? o.clusters(n_subjects, cluster) : 0;
}

int fit_queue_max_clusters(int n_subjects, int n_coef, int n_varying, int cluster) {
  const FitOps o = ops(n_coef, n_varying);
  return o.queue_clusters ? o.queue_clusters(n_subjects, cluster) : 0;
}

int launch_fit(const GeneData& d, const FitControl& ctl, const FitRequest* req, FitResult* res,
               const int32_t* n_req, int32_t* counter, int grid, int cluster, void* stream) {
  const FitOps o = ops(d.n_coef, d.n_varying);
  if (!o.launch) return cudaErrorInvalidValue;
  return o.launch(d, ctl, req, res, n_req, counter, grid, cluster, static_cast<cudaStream_t>(stream));
}

int launch_fit_queue(const GeneData& d, const FitControl& ctl, const FitQueue& qu, int grid, int cluster,
                     void* stream) {
  const FitOps o = ops(d.n_coef, d.n_varying);
  if (!o.launch_queue) return cudaErrorInvalidValue;
  return o.launch_queue(d, ctl, qu, grid, cluster, static_cast<cudaStream_t>(stream));
}

}  // namespace device
}  // namespace nebula
