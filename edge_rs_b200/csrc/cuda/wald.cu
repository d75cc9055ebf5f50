// glm_sc_test on the device (src/sc/test.rs:96-200): the Wald test of a
// contrast c per gene, effect c'beta, variance c'Vc from the packed
// covariance, p = chisq_sf(z^2, 1) = erfc(|z| / sqrt 2), log p kept in log
// space past erfc's underflow, and the Benjamini-Hochberg FDR
// (src/numeric/stats.rs:40-61) over all genes. The same arithmetic as the
// host nb_glm_sc_test (capi_wald.cpp) in the same order; erfc and log are
// CUDA's, so p-values agree with the host's to a few ulps.
//
// BH: p-values sorted decreasing (a stable radix sort of their total-order
// keys, ties kept in gene order as the host's stable sort keeps them), the
// running minimum of n / rank * p by an inclusive scan, then scattered back.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>

#include "nebula_cuda.h"
#include "../host/export.hpp"

namespace {

constexpr int kMaxContrast = 8;

struct Contrast {
  double c[kMaxContrast];
  int n;
};

__device__ double log_erfc(double x) {
  const double p = erfc(x);
  if (p > 1e-300) return log(p);
  // x > ~26: erfc(x) = exp(-x^2) / (x sqrt(pi)) (1 - 1/(2x^2) + 3/(4x^4) - 15/(8x^6) + ...)
  const double u = 1.0 / (2.0 * x * x);
  const double series = 1.0 - u * (1.0 - 3.0 * u * (1.0 - 5.0 * u * (1.0 - 7.0 * u)));
  return -x * x - log(x * sqrt(3.14159265358979323846)) + log(series);
}

// Order-preserving map of a double onto an unsigned key (the total order
// f64::total_cmp sorts by).
__device__ __forceinline__ unsigned long long total_key(double v) {
  long long i = __double_as_longlong(v);
  i ^= static_cast<long long>(static_cast<unsigned long long>(i >> 63) >> 1);
  return static_cast<unsigned long long>(i) ^ 0x8000000000000000ULL;
}

__global__ void wald_genes(const double* __restrict__ beta, const double* __restrict__ cov, uint64_t n_genes,
                           Contrast ct, double* log_fc, double* se, double* z, double* p_value,
                           double* log_p_value, unsigned long long* keys, uint32_t* index) {
  const uint64_t g = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (g >= n_genes) return;
  const int n = ct.n;
  const double* b = beta + g * n;
  const double* v = cov + g * static_cast<uint64_t>(n * (n + 1) / 2);
  double effect = 0.0;
  for (int j = 0; j < n; ++j) effect += b[j] * ct.c[j];
  double variance = 0.0;
  for (int i = 0; i < n; ++i) {
    if (ct.c[i] == 0.0) continue;
    for (int j = 0; j < n; ++j) {
      if (ct.c[j] == 0.0) continue;
      const int lo = i < j ? i : j, hi = i < j ? j : i;
      variance += ct.c[i] * ct.c[j] * v[hi * (hi + 1) / 2 + lo];
    }
  }
  const double error = variance > 0.0 ? sqrt(variance) : 0.0;
  const double statistic = error > 0.0 ? effect / error : 0.0;
  double pv = 1.0, lp = 0.0;
  if (error > 0.0) {
    const double x = fabs(statistic) / sqrt(2.0);
    const double stat2 = statistic * statistic;
    if (stat2 <= 0.0) {
      pv = 1.0;
    } else if (isinf(stat2)) {
      pv = 0.0;
      lp = -INFINITY;
    } else {
      pv = erfc(x);
      lp = log_erfc(x);
    }
  }
  if (log_fc) log_fc[g] = effect;
  if (se) se[g] = error;
  if (z) z[g] = statistic;
  if (p_value) p_value[g] = pv;
  if (log_p_value) log_p_value[g] = lp;
  if (keys) {
    keys[g] = total_key(pv);
    index[g] = static_cast<uint32_t>(g);
  }
}

// rank j of the decreasing order: n / (n - j) * p
__global__ void bh_terms(const unsigned long long* __restrict__ sorted_keys, uint64_t n_genes, double* terms) {
  const uint64_t j = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (j >= n_genes) return;
  long long i = static_cast<long long>(sorted_keys[j] ^ 0x8000000000000000ULL);
  i ^= static_cast<long long>(static_cast<unsigned long long>(i >> 63) >> 1);
  const double p = __longlong_as_double(i);
  const double n = static_cast<double>(n_genes);
  terms[j] = n / static_cast<double>(n_genes - j) * p;
}

__global__ void bh_scatter(const double* __restrict__ running, const uint32_t* __restrict__ order, uint64_t n_genes,
                           double* fdr) {
  const uint64_t j = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (j >= n_genes) return;
  fdr[order[j]] = fmin(running[j], 1.0);
}

struct MinOp {
  __device__ double operator()(double a, double b) const { return fmin(a, b); }
};

void write_err(char* err, size_t len, const std::string& msg) {
  if (!err || len == 0) return;
  const size_t n = msg.size() < len - 1 ? msg.size() : len - 1;
  std::memcpy(err, msg.data(), n);
  err[n] = 0;
}

}  // namespace

NB_API int32_t nb_glm_sc_test_cuda(const double* coefficients, const double* covariance, uint64_t n_genes,
                                   uint64_t n_coef, const double* contrast, double* log_fc, double* se, double* z,
                                   double* p_value, double* log_p_value, double* fdr, void* stream, char* err,
                                   size_t err_len) {
  if (n_genes == 0 || n_coef == 0) {
    write_err(err, err_len, "fit dimensions must be positive");
    return NB_ERR_MUST_BE_POSITIVE;
  }
  if (!coefficients || !covariance || !contrast) {
    write_err(err, err_len, "null input");
    return NB_ERR_INVALID_ARGUMENT;
  }
  if (n_coef > static_cast<uint64_t>(kMaxContrast)) {
    write_err(err, err_len, "the device Wald test takes at most 8 coefficients");
    return NB_ERR_UNSUPPORTED;
  }
  if (n_genes >= (1ULL << 32)) {
    write_err(err, err_len, "too many genes for one call");
    return NB_ERR_INVALID_ARGUMENT;
  }
  Contrast ct{};
  ct.n = static_cast<int>(n_coef);
  bool all_zero = true;
  for (uint64_t j = 0; j < n_coef; ++j) {
    ct.c[j] = contrast[j];
    all_zero = all_zero && contrast[j] == 0.0;
  }
  if (all_zero) {
    write_err(err, err_len, "contrast is entirely zero");
    return NB_ERR_INVALID_ARGUMENT;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  auto gpu_fail = [&](cudaError_t e, const char* what) {
    write_err(err, err_len, std::string(what) + ": " + cudaGetErrorString(e));
    return NB_ERR_GPU;
  };
  const int threads = 256;
  const unsigned blocks = static_cast<unsigned>((n_genes + threads - 1) / threads);
  // BH works on sortable keys of every gene's p-value
  unsigned long long *keys = nullptr, *keys_sorted = nullptr;
  uint32_t *index = nullptr, *order = nullptr;
  double *terms = nullptr, *running = nullptr;
  void* temp = nullptr;
  size_t temp_bytes = 0;
  cudaError_t e = cudaSuccess;
  auto release = [&]() {
    for (void* ptr : {static_cast<void*>(keys), static_cast<void*>(keys_sorted), static_cast<void*>(index),
                      static_cast<void*>(order), static_cast<void*>(terms), static_cast<void*>(running), temp})
      if (ptr) cudaFreeAsync(ptr, st);
  };
  if (fdr) {
    const size_t n = static_cast<size_t>(n_genes);
    if ((e = cudaMallocAsync(reinterpret_cast<void**>(&keys), n * 8, st)) != cudaSuccess ||
        (e = cudaMallocAsync(reinterpret_cast<void**>(&keys_sorted), n * 8, st)) != cudaSuccess ||
        (e = cudaMallocAsync(reinterpret_cast<void**>(&index), n * 4, st)) != cudaSuccess ||
        (e = cudaMallocAsync(reinterpret_cast<void**>(&order), n * 4, st)) != cudaSuccess ||
        (e = cudaMallocAsync(reinterpret_cast<void**>(&terms), n * 8, st)) != cudaSuccess ||
        (e = cudaMallocAsync(reinterpret_cast<void**>(&running), n * 8, st)) != cudaSuccess) {
      release();
      return gpu_fail(e, "device memory");
    }
  }
  wald_genes<<<blocks, threads, 0, st>>>(coefficients, covariance, n_genes, ct, log_fc, se, z, p_value, log_p_value,
                                         keys, index);
  if ((e = cudaGetLastError()) != cudaSuccess) {
    release();
    return gpu_fail(e, "Wald kernel");
  }
  if (fdr) {
    const int n = static_cast<int>(n_genes);
    size_t sort_bytes = 0, scan_bytes = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, sort_bytes, keys, keys_sorted, index, order, n, 0, 64, st);
    cub::DeviceScan::InclusiveScan(nullptr, scan_bytes, terms, running, MinOp{}, n, st);
    temp_bytes = sort_bytes > scan_bytes ? sort_bytes : scan_bytes;
    if ((e = cudaMallocAsync(&temp, temp_bytes, st)) != cudaSuccess) {
      release();
      return gpu_fail(e, "device memory");
    }
    if ((e = cub::DeviceRadixSort::SortPairsDescending(temp, temp_bytes, keys, keys_sorted, index, order, n, 0, 64,
                                                        st)) != cudaSuccess) {
      release();
      return gpu_fail(e, "sort");
    }
    bh_terms<<<blocks, threads, 0, st>>>(keys_sorted, n_genes, terms);
    if ((e = cub::DeviceScan::InclusiveScan(temp, temp_bytes, terms, running, MinOp{}, n, st)) != cudaSuccess) {
      release();
      return gpu_fail(e, "scan");
    }
    bh_scatter<<<blocks, threads, 0, st>>>(running, order, n_genes, fdr);
    if ((e = cudaGetLastError()) != cudaSuccess) {
      release();
      return gpu_fail(e, "BH kernels");
    }
  }
  release();
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return gpu_fail(e, "Wald test");
  return NB_OK;
}
