// Stage one's kernel for 2 design column(s), one instantiation per count
// of columns that vary within subjects (ptmg_impl.cuh).
#include "ptmg_impl.cuh"

namespace nebula {
namespace device {

PtmgOps ptmg_ops_nb2(int n_varying) { return ptmg_ops_for<2>(n_varying); }

}  // namespace device
}  // namespace nebula
