// Dispatch of stage one's kernel (ptmg_impl.cuh) by design width and by how
// many columns vary within subjects (GeneData.n_varying).
#include "ptmg_device.cuh"
#include "ptmg_ops.cuh"

namespace nebula {
namespace device {
namespace {

PtmgOps ops(int n_coef, int n_varying) {
  switch (n_coef) {
    case 1: return ptmg_ops_nb1(n_varying);
    case 2: return ptmg_ops_nb2(n_varying);
    case 3: return ptmg_ops_nb3(n_varying);
    case 4: return ptmg_ops_nb4(n_varying);
    case 5: return ptmg_ops_nb5(n_varying);
    case 6: return ptmg_ops_nb6(n_varying);
    case 7: return ptmg_ops_nb7(n_varying);
    case 8: return ptmg_ops_nb8(n_varying);
    default: return PtmgOps{};
  }
}

}  // namespace

int launch_ptmg_queue(const GeneData& d, const PtmgQueue& queue, double* scratch, int grid, void* stream) {
  const PtmgOps o = ops(d.n_coef, d.n_varying);
  if (!o.launch) return cudaErrorInvalidValue;
  return o.launch(d, queue, scratch, grid, static_cast<cudaStream_t>(stream));
}

int ptmg_resident_ctas(int n_subjects, int n_coef, int n_varying) {
  const PtmgOps o = ops(n_coef, n_varying);
  return o.resident ? o.resident(n_subjects) : 0;
}

size_t ptmg_scratch_doubles(int n_subjects, int n_coef, int n_varying) {
  const PtmgOps o = ops(n_coef, n_varying);
  return o.scratch ? o.scratch(n_subjects) : 0;
}

int ptmg_width_of(int n_coef) { return 9 + 4 * n_coef + n_coef * (n_coef + 1); }

}  // namespace device
}  // namespace nebula
