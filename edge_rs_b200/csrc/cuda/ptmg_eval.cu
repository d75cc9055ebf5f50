// Stage one's cell passes on the device: per-subject sums of the Poisson-gamma
// marginal likelihood (src/sc/ptmg.rs linear_predictor 661-708, the cell loop
// of evaluate 926-966 and hessian_subject 1381-1428) for a batch of
// (gene, [beta, sigma, phi]) requests. The host assembles value, gradient and
// Hessian from them (stage_one.cpp ptmg_assemble).
//
// Pass one sums exp(eta) per subject over every cell and y eta over the
// positive ones (two accumulators, so the dense and sparse halves stay apart).
// Pass two, with ym = (cumsumy + alpha) / (cumsumxtb + lambda) per subject,
// sums the nine scalars, the x-weighted vectors and the two triangles of
// stage_one.hpp, split into the value at a count of zero (dense, every cell)
// plus what each positive count adds (sparse); every per-cell term is affine
// in the count.
//
// The summation tree, the exp/log (nbmath.hpp) and the fused multiply-adds
// (written explicitly; the file is compiled with -fmad=false) are those of the
// CPU oracle (oracle/ptmg_cpu.cpp), so the two agree bit for bit. One
// persistent launch serves the whole stage: each CTA claims the next ticket
// of the device request ring, waits (bounded) for the host to post it, and
// writes its result to host-mapped memory; the warp slots live in a per-CTA
// global scratch region (L2-resident).
#include <cuda_runtime.h>

#include <cstdint>

#include "../host/nbmath.hpp"
#include "ptmg_device.cuh"

namespace nebula {
namespace device {
namespace {

template <int NB>
struct PDims {
  static constexpr int T = NB * (NB + 1) / 2;
  static constexpr int W = 9 + 4 * NB + 2 * T;
  static constexpr int kXf = 9, kD41 = kXf + NB, kT1 = kD41 + NB, kT2 = kT1 + NB, kBp = kT2 + NB, kBq = kBp + T;
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

template <int NV>
__device__ __forceinline__ void reduce_to(const double* acc, double* slot, int lane) {
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double s = warp_sum(acc[v]);
    if (lane == 0) slot[v] = s;
  }
}

template <int NB>
__device__ __forceinline__ void load_row(const double* __restrict__ design, int r, double* x) {
  const double* row = design + static_cast<size_t>(r) * NB;
#pragma unroll
  for (int j = 0; j < NB; ++j) x[j] = __ldg(row + j);
}

template <int NB>
__device__ __forceinline__ double eta_of(const double* x, const double* beta, double off) {
  double eta = off;
#pragma unroll
  for (int j = 0; j < NB; ++j) eta = nb_fma(x[j], beta[j], eta);
  return eta;
}

__device__ __forceinline__ int subject_of(const uint32_t* fid, int K, int c) {
  int lo = 0, hi = K;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (fid[mid] <= static_cast<uint32_t>(c)) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Pass two's dense (count zero) contribution of one cell.
template <int NB>
__device__ __forceinline__ void dense_two(double* acc, const double* x, double e, double ym, double gamma) {
  using D = PDims<NB>;
  const double we = ym * e;
  const double w = we + gamma;
  const double lw = nb_log(w);
  const double iw = 1.0 / w;
  const double gg = gamma * iw;
  const double gt = gg * iw;
  const double gte = gt * e;
  acc[0] += we;
  acc[1] += lw;
  acc[2] = nb_fma(gamma, lw, acc[2]);
  acc[3] += gg;
  acc[4] += iw;
  acc[5] += gt;
  acc[6] = nb_fma(gg, e, acc[6]);
  acc[7] += gte - e * iw;
  acc[8] = nb_fma(gte, e, acc[8]);
  const double f1 = gt - iw;
  const double q = ym * (ym * gte - gg);
  int t = 0;
#pragma unroll
  for (int a = 0; a < NB; ++a) {
    const double xe = x[a] * e;
    acc[D::kXf + a] += xe;
    acc[D::kD41 + a] = nb_fma(gg, xe, acc[D::kD41 + a]);
    acc[D::kT1 + a] = nb_fma(xe, f1, acc[D::kT1 + a]);
    acc[D::kT2 + a] = nb_fma(xe, gte, acc[D::kT2 + a]);
#pragma unroll
    for (int b = a; b < NB; ++b) {
      const double c = xe * x[b];
      acc[D::kBp + t] += c;
      acc[D::kBq + t] = nb_fma(c, q, acc[D::kBq + t]);
      ++t;
    }
  }
}

// What a positive count y adds to a cell's pass-two contribution.
template <int NB>
__device__ __forceinline__ void sparse_two(double* acc, const double* x, double e, double y, double ym,
                                           double gamma) {
  using D = PDims<NB>;
  const double w = ym * e + gamma;
  const double lw = nb_log(w);
  const double iw = 1.0 / w;
  const double gg = y * iw;
  const double gt = gg * iw;
  const double gte = gt * e;
  acc[2] = nb_fma(y, lw, acc[2]);
  acc[3] += gg;
  acc[5] += gt;
  acc[6] = nb_fma(gg, e, acc[6]);
  acc[7] += gte;
  acc[8] = nb_fma(gte, e, acc[8]);
  const double q = ym * (ym * gte - gg);
  int t = 0;
#pragma unroll
  for (int a = 0; a < NB; ++a) {
    const double xe = x[a] * e;
    acc[D::kD41 + a] = nb_fma(gg, xe, acc[D::kD41 + a]);
    acc[D::kT1 + a] = nb_fma(xe, gt, acc[D::kT1 + a]);
    acc[D::kT2 + a] = nb_fma(xe, gte, acc[D::kT2 + a]);
#pragma unroll
    for (int b = a; b < NB; ++b) {
      const double c = xe * x[b];
      acc[D::kBq + t] = nb_fma(c, q, acc[D::kBq + t]);
      ++t;
    }
  }
}

// One pass through the tree: dense pieces into slots[(s + warp) * stride],
// sparse pieces into slots[(K + kWarps + s) * stride], then per subject
// out[s * out_stride + v] = 0 + dense pieces (warp order) + sparse piece.
template <int NB, int PASS, int NV>
__device__ void tree_pass(const GeneData& d, const uint32_t* fid, const uint32_t* wcells, int gene,
                          const double* beta, const double* ym, double gamma, double* slots, int stride,
                          double* out, int out_stride) {
  const int K = d.n_subjects;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c_begin = static_cast<int>(wcells[warp]), c_end = static_cast<int>(wcells[warp + 1]);
  if (c_begin < c_end) {
    int s = subject_of(fid, K, c_begin);
    for (int c0 = c_begin; c0 < c_end; ++s) {
      const int s_end = min(c_end, static_cast<int>(fid[s + 1]));
      double acc[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) acc[v] = 0.0;
      const double yms = PASS == 2 ? ym[s] : 0.0;
      for (int r = c0 + lane; r < s_end; r += 32) {
        double x[NB];
        load_row<NB>(d.design, r, x);
        const double e = nb_exp(eta_of<NB>(x, beta, __ldg(d.log_offset + r)));
        if constexpr (PASS == 1) acc[0] += e;
        else dense_two<NB>(acc, x, e, yms, gamma);
      }
      reduce_to<NV>(acc, slots + (s + warp) * stride, lane);
      c0 = s_end;
    }
  }
  const uint64_t* runs = d.runs + static_cast<size_t>(gene) * (K + 1);
  for (int s = warp; s < K; s += kWarps) {
    const uint64_t p0 = runs[s], p1 = runs[s + 1];
    double acc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] = 0.0;
    const double yms = PASS == 2 ? ym[s] : 0.0;
    for (uint64_t p = p0 + lane; p < p1; p += 32) {
      const int c = static_cast<int>(__ldg(d.cells + p));
      const double y = __ldg(d.counts + p);
      double x[NB];
      load_row<NB>(d.design, c, x);
      const double eta = eta_of<NB>(x, beta, __ldg(d.log_offset + c));
      if constexpr (PASS == 1) acc[1] = nb_fma(eta, y, acc[1]);
      else sparse_two<NB>(acc, x, nb_exp(eta), y, yms, gamma);
    }
    reduce_to<NV>(acc, slots + (K + kWarps + s) * stride, lane);
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < K * NV; idx += blockDim.x) {
    const int s = idx / NV, v = idx - s * NV;
    const uint32_t a0 = fid[s], a1 = fid[s + 1];
    double total = 0.0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w)
      if (wcells[w] < a1 && wcells[w + 1] > a0) total += slots[(s + w) * stride + v];
    total += slots[(K + kWarps + s) * stride + v];
    out[s * out_stride + v] = total;
  }
  __syncthreads();
}

// Shared-memory and scratch views of one stage-one CTA.
struct PtmgCta {
  double* ym;        // K
  double* p1;        // K x 2: cumsumxtb, ylin
  uint32_t* fid;     // K + 1
  uint32_t* wcells;  // kWarps + 1
  double* slots;     // this CTA's scratch rows
};

template <int NB>
__device__ PtmgCta ptmg_setup(const GeneData& d, double* smem, double* scratch) {
  using D = PDims<NB>;
  const int K = d.n_subjects;
  PtmgCta c;
  c.ym = smem;
  c.p1 = c.ym + K;
  c.fid = reinterpret_cast<uint32_t*>(c.p1 + 2 * K);
  c.wcells = c.fid + K + 1;
  for (int i = threadIdx.x; i <= K; i += blockDim.x) c.fid[i] = d.fid[i];
  if (threadIdx.x <= kWarps) c.wcells[threadIdx.x] = d.warp_cells[threadIdx.x];
  c.slots = scratch + static_cast<size_t>(blockIdx.x) * (2 * K + kWarps) * D::W;
  return c;
}

// Both passes of one request into `out` ((2 + W) K doubles).
template <int NB>
__device__ void ptmg_one(const GeneData& d, const PtmgCta& c, const PtmgRequest& req, double* beta_sm, double* out) {
  using D = PDims<NB>;
  const int K = d.n_subjects;
  const int tid = threadIdx.x;
  if (tid < NB) beta_sm[tid] = req.beta[tid];
  __syncthreads();
  double beta[NB];
#pragma unroll
  for (int j = 0; j < NB; ++j) beta[j] = beta_sm[j];
  tree_pass<NB, 1, 2>(d, c.fid, c.wcells, req.gene, beta, c.ym, req.gamma, c.slots, D::W, c.p1, 2);
  const double* tot = d.totals + static_cast<size_t>(req.gene) * K;
  for (int s = tid; s < K; s += blockDim.x) {
    c.ym[s] = (__ldg(tot + s) + req.alpha) / (c.p1[2 * s] + req.lambda);
    out[s] = c.p1[2 * s];          // cumsumxtb
    out[K + s] = c.p1[2 * s + 1];  // ylin
  }
  __syncthreads();
  tree_pass<NB, 2, D::W>(d, c.fid, c.wcells, req.gene, beta, c.ym, req.gamma, c.slots, D::W, out + 2 * K, D::W);
}

__device__ __forceinline__ long long global_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Streaming mode: one persistent launch for stage one, the request-ring
// protocol of FitQueue (pml_device.cuh) with one CTA per request.
template <int NB>
__global__ void __launch_bounds__(kThreads, 1) ptmg_queue_kernel(GeneData d, PtmgQueue qu, double* scratch) {
  extern __shared__ __align__(16) double smem[];
  const PtmgCta c = ptmg_setup<NB>(d, smem, scratch);
  __shared__ long long next_ticket;
  __shared__ double beta_sm[kMaxCoef];
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) {
      const long long t = static_cast<long long>(atomicAdd(qu.taken, 1ull));
      const volatile long long* seq = qu.seq + (t & qu.mask);
      const volatile int* stop = qu.stop;
      const long long t0 = global_ns();
      unsigned int pause = 128;
      long long got = -1;
      for (;;) {
        if (*seq == t) {
          got = t;
          break;
        }
        if (*stop != 0) break;
        if (global_ns() - t0 > qu.idle_ns) {
          atomicExch(qu.status, 1);
          break;
        }
        __nanosleep(pause);
        if (pause < 2048) pause *= 2;
      }
      next_ticket = got;
    }
    __syncthreads();
    const long long t = next_ticket;
    if (t < 0) break;
    PtmgRequest req;
    {
      const int4* src = reinterpret_cast<const int4*>(qu.ring + (t & qu.mask));
      int4* dst = reinterpret_cast<int4*>(&req);
#pragma unroll
      for (int i = 0; i < static_cast<int>(sizeof(PtmgRequest) / 16); ++i) dst[i] = __ldcg(src + i);
    }
    ptmg_one<NB>(d, c, req, beta_sm, qu.results + (t & qu.mask) * qu.result_stride);
    // every thread's result writes reach host memory before the flag
    __threadfence_system();
    __syncthreads();
    if (threadIdx.x == 0) reinterpret_cast<volatile long long*>(qu.done)[t & qu.mask] = t + 1;
  }
}

template <int NB>
int launch_queue_nb(const GeneData& d, const PtmgQueue& qu, double* scratch, int grid, cudaStream_t stream) {
  const size_t smem = ptmg_smem_bytes(d.n_subjects);
  cudaError_t e = cudaFuncSetAttribute(ptmg_queue_kernel<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  ptmg_queue_kernel<NB><<<grid, kThreads, smem, stream>>>(d, qu, scratch);
  return cudaGetLastError();
}

}  // namespace

int launch_ptmg_queue(const GeneData& d, const PtmgQueue& queue, double* scratch, int grid, void* stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  switch (d.n_coef) {
    case 1: return launch_queue_nb<1>(d, queue, scratch, grid, s);
    case 2: return launch_queue_nb<2>(d, queue, scratch, grid, s);
    case 3: return launch_queue_nb<3>(d, queue, scratch, grid, s);
    case 4: return launch_queue_nb<4>(d, queue, scratch, grid, s);
    case 5: return launch_queue_nb<5>(d, queue, scratch, grid, s);
    case 6: return launch_queue_nb<6>(d, queue, scratch, grid, s);
    case 7: return launch_queue_nb<7>(d, queue, scratch, grid, s);
    case 8: return launch_queue_nb<8>(d, queue, scratch, grid, s);
    default: return cudaErrorInvalidValue;
  }
}

size_t ptmg_smem_bytes(int n_subjects) {
  return static_cast<size_t>(3 * n_subjects) * 8 + (n_subjects + 1 + kWarps + 1) * 4 + 16;
}

int ptmg_width_of(int n_coef) { return 9 + 4 * n_coef + n_coef * (n_coef + 1); }

size_t ptmg_scratch_doubles(int n_subjects, int n_coef) {
  return static_cast<size_t>(2 * n_subjects + kWarps) * ptmg_width_of(n_coef);
}

}  // namespace device
}  // namespace nebula
