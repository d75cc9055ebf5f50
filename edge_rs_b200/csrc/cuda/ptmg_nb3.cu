// Stage one's kernel for 3 design column(s), one instantiation per count
// of columns that vary within subjects (ptmg_impl.cuh).
#include "ptmg_impl.cuh"

namespace nebula {
namespace device {

PtmgOps ptmg_ops_nb3(int n_varying) { return ptmg_ops_for<3>(n_varying); }

}  // namespace device
}  // namespace nebula
