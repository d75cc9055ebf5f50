// Device copy of the tables of nb_exp_tab / nb_log_tab (nbmath.hpp); kernels
// copy it into shared memory once per CTA and pass that copy.
#pragma once

#include "../host/nbmath.hpp"

namespace nebula {

static __device__ const NbTableData kNbTablesDevice = {
#include "../host/nbmath_tables.inc"
};

// Copies the tables into `dst` (shared memory) with every thread of the CTA;
// the caller synchronises before use.
__device__ __forceinline__ void nb_load_tables(NbTableData* dst) {
  const double* src = reinterpret_cast<const double*>(&kNbTablesDevice);
  double* out = reinterpret_cast<double*>(dst);
  for (int i = threadIdx.x; i < kNbTableDoubles; i += blockDim.x) out[i] = src[i];
}

}  // namespace nebula
