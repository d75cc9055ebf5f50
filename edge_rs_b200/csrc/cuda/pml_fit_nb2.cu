// The fit kernels for 2 design column(s), one instantiation per count of
// columns that vary within subjects (pml_fit_impl.cuh).
#include "pml_fit_impl.cuh"

namespace nebula {
namespace device {

FitOps fit_ops_nb2(int n_varying) { return ops_for<2>(n_varying); }

}  // namespace device
}  // namespace nebula
