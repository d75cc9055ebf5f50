// The Hessian contraction of the inner fit on the tensor cores, and the
// precision it costs. Every Newton step of the penalised NB-gamma fit
// (src/sc/pml.rs:1419-1590, sweep_width) accumulates
//     S_r = sum over cells c of w_rc x_c x_c'   (p x p, p(p+1)/2 distinct)
// for each request r; over a batch of R requests that is the dense product
// W [R x N] . KR [N x p(p+1)/2] of the requests' cell weights with the
// Khatri-Rao square of the shared design (the reference's fused gradient and
// curvature assembly, src/gpu/pml_kernel.rs:350-515).
//
// nb_contract_krx_cuda evaluates that product four ways:
//   0 FP64 on CUDA cores (the reference's arithmetic),
//   1 FP32 on CUDA cores (FP32 inputs and accumulation),
//   2 TF32 on the tensor cores (tcgen05.mma kind::tf32, FP32 accumulation
//     in tensor memory),
//   3 split BF16 on the tensor cores: w = w_hi + w_lo and kr = kr_hi + kr_lo
//     in BF16, S = hi.hi + hi.lo + lo.hi (three tcgen05.mma kind::f16 per
//     K step, FP32 accumulation in tensor memory).
// The tensor-core kernel is hand-written sm_100a: one CTA per split of the
// cells, M = 128 requests by N = 48 (the 36 products padded) accumulated in
// 64 tensor-memory columns, operands staged by the CTA's threads into shared
// memory in the no-swizzle K-major core-matrix layout and issued by one
// thread; each CTA's FP32 partial sums are added in FP64 afterwards.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "nebula_cuda.h"
#include "../host/export.hpp"

namespace {

constexpr int kM = 128;        // requests per tile (the MMA's M)
constexpr int kN = 48;         // Khatri-Rao columns, padded (the MMA's N; p <= 8 gives 36)
constexpr int kTmemCols = 64;  // tensor-memory columns allocated (a power of two >= kN)
constexpr int kThreads = 128;  // four warps: one per 32-lane quarter of tensor memory
constexpr int kRowBytes = 128; // bytes of one operand row per K tile (64 BF16 or 32 TF32 values)
constexpr long long kWaitLimit = 2000000;  // mbarrier polls before a CTA gives up (about a second)

// ---------------------------------------------------------------- operands

// Khatri-Rao rows, transposed: kr[j][c] = x_c[a] x_c[b] for the j-th pair
// a <= b (j = b (b + 1) / 2 + a, the packing of NebulaFit's covariance), zero
// for j >= p(p+1)/2.
__global__ void khatri_rao(const double* __restrict__ x, uint64_t n_cells, int p, double* kr) {
  const uint64_t c = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  if (c >= n_cells) return;
  const int pairs = p * (p + 1) / 2;
  for (int b = 0; b < p; ++b)
    for (int a = 0; a <= b; ++a) kr[static_cast<uint64_t>(b * (b + 1) / 2 + a) * n_cells + c] = x[c * p + a] * x[c * p + b];
  for (int j = pairs; j < kN; ++j) kr[static_cast<uint64_t>(j) * n_cells + c] = 0.0;
}

// FP64 rows (stride ld) into BF16 hi and lo (hi = rn(v), lo = rn(v - hi))
// or FP32 (TF32 reads the top 19 bits), rows padded with zeros to n_pad.
__global__ void split_rows(const double* __restrict__ src, uint64_t rows, uint64_t cols, uint64_t ld,
                           uint64_t n_pad, __nv_bfloat16* hi, __nv_bfloat16* lo, float* f32) {
  const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
  const uint64_t r = i / n_pad, c = i - r * n_pad;
  if (r >= rows) return;
  const double v = c < cols ? src[r * ld + c] : 0.0;
  if (hi) {
    const __nv_bfloat16 h = __double2bfloat16(v);
    hi[i] = h;
    lo[i] = __double2bfloat16(v - static_cast<double>(__bfloat162float(h)));
  }
  if (f32) f32[i] = static_cast<float>(v);
}

// ------------------------------------------------------------ tensor cores

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, no swizzle, K-major: 8-row x 16-byte core
// matrices, row groups `sbo` bytes apart, K chunks `lbo` bytes apart.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = static_cast<uint64_t>((addr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
  d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
  d |= 1ull << 46;  // descriptor version of sm_100; base offset 0, layout SWIZZLE_NONE (0)
  return d;
}

// Instruction descriptor: FP32 accumulator, A and B in BF16 (kind::f16) or
// TF32 (kind::tf32), both K-major, N = kN, M = kM.
template <bool TF32>
__device__ __forceinline__ uint32_t instr_desc() {
  const uint32_t fmt = TF32 ? 2u : 1u;
  return (1u << 4) | (fmt << 7) | (fmt << 10) | (static_cast<uint32_t>(kN >> 3) << 17) |
         (static_cast<uint32_t>(kM >> 4) << 24);
}

template <bool TF32>
__device__ __forceinline__ void mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  if constexpr (TF32) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
  } else {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
  }
}

__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity) {
  for (long long i = 0; i < kWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

constexpr int kStages = 4;  // operand tiles in flight per CTA

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// One CTA: requests 0..kM-1 against the Khatri-Rao rows 0..kN-1 over the
// K tiles [t0, t1) of kRowBytes per row; FP32 partial sums into
// partial[blockIdx.x][kM][kN]. Operands are row-major in global memory,
// `row_bytes` apart: A (requests) a_hi / a_lo, B (pairs) b_hi / b_lo (the
// lo halves unused for TF32). kStages tiles are in flight: the threads copy
// tile i + kStages - 1 (cp.async) while the tensor cores multiply tile i;
// a stage is refilled once the MMAs that read it have completed (its
// mbarrier). *status = 1 if a wait ran out.
template <bool TF32>
__global__ void __launch_bounds__(kThreads, 1)
    contract_tc(const char* __restrict__ a_hi, const char* __restrict__ a_lo, const char* __restrict__ b_hi,
                const char* __restrict__ b_lo, uint64_t row_bytes, uint64_t tiles, uint64_t tiles_per_cta,
                float* partial, int* status) {
  extern __shared__ __align__(1024) unsigned char smem[];
  constexpr uint32_t kLboA = (kM / 8) * 128, kLboB = (kN / 8) * 128;
  constexpr uint32_t kABytes = kM * kRowBytes, kBBytes = kN * kRowBytes;
  constexpr uint32_t kStageBytes = (TF32 ? 1 : 2) * (kABytes + kBBytes);
  __shared__ __align__(8) unsigned long long mbar[kStages];
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint64_t t0 = blockIdx.x * tiles_per_cta;
  const uint64_t t1 = t0 + tiles_per_cta < tiles ? t0 + tiles_per_cta : tiles;
  const uint64_t n_tiles = t1 > t0 ? t1 - t0 : 0;
  const uint32_t base = smem_u32(smem);
  // stage s: A hi, B hi, then (split BF16) A lo, B lo
  auto a_at = [&](int st, int lo) { return base + st * kStageBytes + (lo ? kABytes + kBBytes : 0); };
  auto b_at = [&](int st, int lo) { return base + st * kStageBytes + kABytes + (lo ? kABytes + kBBytes : 0); };
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int st = 0; st < kStages; ++st)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[st])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = instr_desc<TF32>();
  // copies tile t0 + i into stage i % kStages (16-byte chunk c of a row's
  // tile is K chunk c: row group (row / 8) at 128-byte steps, K chunks kLbo apart)
  auto load = [&](uint64_t i) {
    if (i < n_tiles) {
      const int st = static_cast<int>(i % kStages);
      const uint64_t k_off = (t0 + i) * kRowBytes;
      for (int c = tid; c < kM * 8; c += kThreads) {
        const int m = c >> 3, kc = c & 7;
        const uint32_t dst = static_cast<uint32_t>(kc) * kLboA + static_cast<uint32_t>(m >> 3) * 128 + (m & 7) * 16;
        const uint64_t src = static_cast<uint64_t>(m) * row_bytes + k_off + kc * 16;
        cp_async16(a_at(st, 0) + dst, a_hi + src);
        if (!TF32) cp_async16(a_at(st, 1) + dst, a_lo + src);
      }
      for (int c = tid; c < kN * 8; c += kThreads) {
        const int n = c >> 3, kc = c & 7;
        const uint32_t dst = static_cast<uint32_t>(kc) * kLboB + static_cast<uint32_t>(n >> 3) * 128 + (n & 7) * 16;
        const uint64_t src = static_cast<uint64_t>(n) * row_bytes + k_off + kc * 16;
        cp_async16(b_at(st, 0) + dst, b_hi + src);
        if (!TF32) cp_async16(b_at(st, 1) + dst, b_lo + src);
      }
    }
    cp_async_commit();  // one group per tile, empty past the end
  };
  for (int i = 0; i < kStages - 1; ++i) load(static_cast<uint64_t>(i));
  uint32_t uses[kStages] = {};  // completed MMA groups per stage: the parity to wait for
  bool ok = true;
  uint64_t issued = 0;  // tiles whose MMAs have been issued
  for (uint64_t i = 0; i < n_tiles; ++i) {
    const int st = static_cast<int>(i % kStages);
    // the stage that tile i + kStages - 1 refills last held tile i - 1
    if (i > 0) {
      const int prev = static_cast<int>((i - 1) % kStages);
      ok = __syncthreads_and(mbar_wait(smem_u32(&mbar[prev]), uses[prev] & 1u)) != 0;
      if (!ok) break;
      ++uses[prev];
    }
    load(i + kStages - 1);
    cp_async_wait<kStages - 1>();  // this thread's copies of tile i have landed
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      // four MMA K steps of two 16-byte chunks each (16 BF16 or 8 TF32 values)
#pragma unroll
      for (int step = 0; step < 4; ++step) {
        const uint32_t acc = (i == 0 && step == 0) ? 0u : 1u;
        const uint64_t da_hi = smem_desc(a_at(st, 0) + 2 * step * kLboA, kLboA, 128);
        const uint64_t db_hi = smem_desc(b_at(st, 0) + 2 * step * kLboB, kLboB, 128);
        mma<TF32>(tmem, da_hi, db_hi, idesc, acc);
        if (!TF32) {
          const uint64_t da_lo = smem_desc(a_at(st, 1) + 2 * step * kLboA, kLboA, 128);
          const uint64_t db_lo = smem_desc(b_at(st, 1) + 2 * step * kLboB, kLboB, 128);
          mma<TF32>(tmem, da_hi, db_lo, idesc, 1u);
          mma<TF32>(tmem, da_lo, db_hi, idesc, 1u);
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&mbar[st]))
                   : "memory");
    }
    issued = i + 1;
  }
  cp_async_wait<0>();
  // the last tile's MMAs (or, after a failed wait, the ones in flight: once more, bounded)
  if (issued > 0) {
    const int last = static_cast<int>((issued - 1) % kStages);
    const bool done = mbar_wait(smem_u32(&mbar[last]), uses[last] & 1u);
    ok = __syncthreads_and(ok && done) != 0;
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  __syncthreads();
  float* out = partial + static_cast<uint64_t>(blockIdx.x) * kM * kN;
  const int row = warp * 32 + lane;
  if (!ok) {
    if (tid == 0) atomicExch(status, 1);
  } else if (n_tiles == 0) {
    for (int c = 0; c < kN; ++c) out[row * kN + c] = 0.0f;
  } else {
    // each warp reads its 32 lanes (rows) of the accumulator, 16 columns at a time
#pragma unroll
    for (int c0 = 0; c0 < kN; c0 += 16) {
      uint32_t r[16];
      const uint32_t addr = tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c0);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(addr)
          : "memory");
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int i = 0; i < 16; ++i) out[row * kN + c0 + i] = __uint_as_float(r[i]);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

// -------------------------------------------------------------- CUDA cores

// One thread per request over the cells [c0, c1) of this CTA's split:
// acc[j] += w_rc * kr_jc in T (FP64: w and the exact FP64 product x_a x_b;
// FP32: both rounded to FP32, FP32 fused multiply-adds), then the partial
// sums per CTA.
template <typename T>
__global__ void __launch_bounds__(kM)
    contract_cc(const T* __restrict__ w, const T* __restrict__ kr, uint64_t n_cells, uint64_t ld, int n_req,
                int pairs, uint64_t cells_per_cta, double* partial) {
  const int r = threadIdx.x;
  const uint64_t c0 = blockIdx.x * cells_per_cta;
  const uint64_t c1 = c0 + cells_per_cta < n_cells ? c0 + cells_per_cta : n_cells;
  T acc[kN];
#pragma unroll
  for (int j = 0; j < kN; ++j) acc[j] = T(0);
  if (r < n_req) {
    const T* wr = w + static_cast<uint64_t>(r) * ld;
    for (uint64_t c = c0; c < c1; ++c) {
      const T wc = wr[c];
#pragma unroll
      for (int j = 0; j < kN; ++j)
        if (j < pairs) acc[j] = fma(wc, __ldg(kr + static_cast<uint64_t>(j) * ld + c), acc[j]);
    }
  }
  double* out = partial + static_cast<uint64_t>(blockIdx.x) * kM * kN + static_cast<uint64_t>(r) * kN;
#pragma unroll
  for (int j = 0; j < kN; ++j) out[j] = static_cast<double>(acc[j]);
}

// S[r][j] = sum over the CTAs' partials, in CTA order, in FP64.
template <typename P>
__global__ void reduce_partials(const P* __restrict__ partial, int ctas, int n_req, int pairs, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_req * pairs) return;
  const int r = i / pairs, j = i - r * pairs;
  double s = 0.0;
  for (int b = 0; b < ctas; ++b) s += static_cast<double>(partial[(static_cast<uint64_t>(b) * kM + r) * kN + j]);
  out[i] = s;
}

void write_err(char* err, size_t len, const std::string& msg) {
  if (!err || len == 0) return;
  const size_t n = msg.size() < len - 1 ? msg.size() : len - 1;
  std::memcpy(err, msg.data(), n);
  err[n] = 0;
}

}  // namespace

// Variants: 0 FP64 CUDA cores, 1 FP32 CUDA cores, 2 TF32 tensor cores,
// 3 split-BF16 tensor cores. design: device n_cells x n_coef (FP64,
// row-major); weights: device n_requests x n_cells (FP64); out: device
// n_requests x n_coef (n_coef + 1) / 2, entry b (b + 1) / 2 + a holding
// sum_c w_rc x_ca x_cb (a <= b). ms_out (host, may be NULL): [0] device time
// of the contraction kernel, [1] with the operand conversions.
NB_API int32_t nb_contract_krx_cuda(int32_t variant, const double* design, uint64_t n_cells, uint32_t n_coef,
                                    const double* weights, uint32_t n_requests, double* out, double* ms_out,
                                    void* stream, char* err, size_t err_len) {
  if (variant < 0 || variant > 3) {
    write_err(err, err_len, "variant must be 0 (FP64), 1 (FP32), 2 (TF32) or 3 (split BF16)");
    return NB_ERR_INVALID_ARGUMENT;
  }
  if (!design || !weights || !out) {
    write_err(err, err_len, "null input");
    return NB_ERR_INVALID_ARGUMENT;
  }
  if (n_cells == 0 || n_coef == 0 || n_requests == 0) {
    write_err(err, err_len, "dimensions must be positive");
    return NB_ERR_MUST_BE_POSITIVE;
  }
  if (n_coef > 8 || n_requests > static_cast<uint32_t>(kM)) {
    write_err(err, err_len, "at most 8 columns and 128 requests per call");
    return NB_ERR_UNSUPPORTED;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int p = static_cast<int>(n_coef), pairs = p * (p + 1) / 2, nr = static_cast<int>(n_requests);
  const bool tc = variant >= 2, tf32 = variant == 2;
  // cells padded to whole K tiles (64 BF16 or 32 TF32 values of 128 bytes)
  const uint64_t kt = tf32 ? 32 : 64;
  const uint64_t n_pad = (n_cells + kt - 1) / kt * kt;
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) {
    write_err(err, err_len, std::string("device: ") + cudaGetErrorString(e));
    return NB_ERR_GPU;
  }
  const int ctas = sms;
  std::vector<void*> owned;
  auto alloc = [&](size_t bytes) -> void* {
    void* ptr = nullptr;
    if (e == cudaSuccess) e = cudaMallocAsync(&ptr, bytes, st);
    if (ptr) owned.push_back(ptr);
    return ptr;
  };
  auto release = [&]() {
    for (void* ptr : owned) cudaFreeAsync(ptr, st);
  };
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
  for (auto& x : ev)
    if (e == cudaSuccess) e = cudaEventCreate(&x);
  double* kr = static_cast<double*>(alloc(static_cast<size_t>(kN) * n_cells * 8));
  double* partial64 = tc ? nullptr : static_cast<double*>(alloc(static_cast<size_t>(ctas) * kM * kN * 8));
  float* partial32 = tc ? static_cast<float*>(alloc(static_cast<size_t>(ctas) * kM * kN * 4)) : nullptr;
  int* status = static_cast<int*>(alloc(sizeof(int)));
  __nv_bfloat16 *a_hi = nullptr, *a_lo = nullptr, *b_hi = nullptr, *b_lo = nullptr;
  float *a32 = nullptr, *b32 = nullptr;
  if (variant == 3) {
    a_hi = static_cast<__nv_bfloat16*>(alloc(static_cast<size_t>(kM) * n_pad * 2));
    a_lo = static_cast<__nv_bfloat16*>(alloc(static_cast<size_t>(kM) * n_pad * 2));
    b_hi = static_cast<__nv_bfloat16*>(alloc(static_cast<size_t>(kN) * n_pad * 2));
    b_lo = static_cast<__nv_bfloat16*>(alloc(static_cast<size_t>(kN) * n_pad * 2));
  } else if (variant != 0) {
    a32 = static_cast<float*>(alloc(static_cast<size_t>(kM) * n_pad * 4));
    b32 = static_cast<float*>(alloc(static_cast<size_t>(kN) * n_pad * 4));
  }
  if (e != cudaSuccess) {
    release();
    for (auto& x : ev)
      if (x) cudaEventDestroy(x);
    write_err(err, err_len, std::string("device memory: ") + cudaGetErrorString(e));
    return NB_ERR_GPU;
  }
  const int th = 256;
  e = cudaMemsetAsync(status, 0, sizeof(int), st);
  if (e == cudaSuccess) e = cudaEventRecord(ev[0], st);
  khatri_rao<<<static_cast<unsigned>((n_cells + th - 1) / th), th, 0, st>>>(design, n_cells, p, kr);
  if (variant >= 1) {
    // requests beyond n_requests are zero rows of the 128-row tile
    const uint64_t na = static_cast<uint64_t>(kM) * n_pad, nb = static_cast<uint64_t>(kN) * n_pad;
    if (e == cudaSuccess) e = cudaMemsetAsync(variant == 3 ? static_cast<void*>(a_hi) : static_cast<void*>(a32), 0,
                                               na * (variant == 3 ? 2 : 4), st);
    if (variant == 3 && e == cudaSuccess) e = cudaMemsetAsync(a_lo, 0, na * 2, st);
    split_rows<<<static_cast<unsigned>((static_cast<uint64_t>(nr) * n_pad + th - 1) / th), th, 0, st>>>(
        weights, nr, n_cells, n_cells, n_pad, a_hi, a_lo, a32);
    split_rows<<<static_cast<unsigned>((nb + th - 1) / th), th, 0, st>>>(kr, kN, n_cells, n_cells, n_pad, b_hi,
                                                                          b_lo, b32);
  }
  if (e == cudaSuccess) e = cudaEventRecord(ev[1], st);
  if (tc) {
    const uint64_t tiles = n_pad / kt;
    const uint64_t per = (tiles + ctas - 1) / ctas;
    const size_t smem = static_cast<size_t>(kStages) * (tf32 ? 1 : 2) * (kM + kN) * kRowBytes;
    const char* ah = tf32 ? reinterpret_cast<const char*>(a32) : reinterpret_cast<const char*>(a_hi);
    const char* al = tf32 ? nullptr : reinterpret_cast<const char*>(a_lo);
    const char* bh = tf32 ? reinterpret_cast<const char*>(b32) : reinterpret_cast<const char*>(b_hi);
    const char* bl = tf32 ? nullptr : reinterpret_cast<const char*>(b_lo);
    const uint64_t row_bytes = n_pad * (tf32 ? 4 : 2);
    if (tf32) {
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(contract_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
      if (e == cudaSuccess)
        contract_tc<true><<<ctas, kThreads, smem, st>>>(ah, al, bh, bl, row_bytes, tiles, per, partial32, status);
    } else {
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(contract_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
      if (e == cudaSuccess)
        contract_tc<false><<<ctas, kThreads, smem, st>>>(ah, al, bh, bl, row_bytes, tiles, per, partial32, status);
    }
  } else {
    const uint64_t per = (n_cells + ctas - 1) / ctas;
    if (variant == 0)
      contract_cc<double><<<ctas, kM, 0, st>>>(weights, kr, n_cells, n_cells, nr, pairs, per, partial64);
    else
      contract_cc<float><<<ctas, kM, 0, st>>>(a32, b32, n_cells, n_pad, nr, pairs, per, partial64);
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaEventRecord(ev[2], st);
  const int nt = nr * pairs;
  if (tc)
    reduce_partials<float><<<(nt + th - 1) / th, th, 0, st>>>(partial32, ctas, nr, pairs, out);
  else
    reduce_partials<double><<<(nt + th - 1) / th, th, 0, st>>>(partial64, ctas, nr, pairs, out);
  int h_status = 0;
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_status, status, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  float t_kernel = 0.0f, t_total = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t_kernel, ev[1], ev[2]);
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t_total, ev[0], ev[2]);
  release();
  for (auto& x : ev)
    if (x) cudaEventDestroy(x);
  if (e != cudaSuccess) {
    write_err(err, err_len, std::string("contraction: ") + cudaGetErrorString(e));
    return NB_ERR_GPU;
  }
  if (h_status != 0) {
    write_err(err, err_len, "a tensor-core CTA's wait for its MMAs ran out");
    return NB_ERR_GPU;
  }
  if (ms_out) {
    ms_out[0] = t_kernel;
    ms_out[1] = t_total;
  }
  return NB_OK;
}
