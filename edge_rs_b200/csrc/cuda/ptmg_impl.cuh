// Stage one's cell passes on the device: per-subject sums of the Poisson-gamma
// marginal likelihood (src/sc/ptmg.rs linear_predictor 661-708, the cell loop
// of evaluate 926-966 and hessian_subject 1381-1428) for a stream of
// (gene, [beta, sigma, phi]) requests. The host assembles value, gradient and
// Hessian from them (stage_one.cpp ptmg_assemble). Instantiated per design
// width NB and count NV of the columns that vary within subjects
// (ptmg_nb<NB>.cu); ptmg_eval.cu dispatches.
//
// Pass one sums exp(eta) per subject over every cell and y eta over the
// positive ones (two accumulators, so the dense and sparse halves stay apart).
// Pass two, with ym = (cumsumy + alpha) / (cumsumxtb + lambda) per subject,
// sums the nine scalars, the x-weighted vectors and the two triangles of
// stage_one.hpp, split into the value at a count of zero (dense, every cell)
// plus what each positive count adds (sparse); every per-cell term is affine
// in the count.
//
// The cells' sums run over the NV varying columns only. eta starts from the
// offset plus the subject's constant share (the subject-constant columns
// times beta, once per subject and request), and pass two keeps, beside the
// nine scalars, sum e and sum e q (dense and sparse q alike) and the vector
// sum x e q over the varying columns: a constant column a's sums are then its
// value times a scalar sum (sum x_a e = x_a sum e, sum x_a gg e = x_a acc[6],
// ...), and the subject's full row of stage_one.hpp is expanded before it is
// written (expand_two).
//
// The summation tree, the exp/log (nbmath.hpp) and the fused multiply-adds
// (written explicitly; compiled with -fmad=false) are those of the CPU oracle
// (oracle/ptmg_cpu.cpp), so the two agree bit for bit. One persistent launch
// serves the whole stage: each CTA claims the next ticket of the request
// ring (host memory mapped into the device), waits (bounded) for the host to
// post it, and writes its result to host-mapped memory; the warp slots and the subjects' reduced
// sums live in a per-cluster global scratch region (L2-resident).
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../host/nbmath.hpp"
#include "nbmath_device.cuh"
#include "ptmg_device.cuh"
#include "ptmg_ops.cuh"
#include "ring_device.cuh"

namespace nebula {
namespace device {
namespace {

namespace cg = cooperative_groups;

// The full per-subject row of pass two (stage_one.hpp).
template <int NB>
struct PDims {
  static constexpr int T = NB * (NB + 1) / 2;
  static constexpr int W = 9 + 4 * NB + 2 * T;
  static constexpr int kXf = 9, kD41 = kXf + NB, kT1 = kD41 + NB, kT2 = kT1 + NB, kBp = kT2 + NB, kBq = kBp + T;
};

// The reduced row over NV varying columns: the nine scalars, sum e, sum e q,
// the vectors Xf, D41, T1, T2, Eq and the triangles Bp, Bq.
template <int NV>
struct RDims {
  static constexpr int T = NV * (NV + 1) / 2;
  static constexpr int kE = 9, kEq = 10;
  static constexpr int kXf = 11, kD41 = kXf + NV, kT1 = kD41 + NV, kT2 = kT1 + NV, kQv = kT2 + NV;
  static constexpr int kBp = kQv + NV, kBq = kBp + T;
  static constexpr int W = kBq + T;
};

// A request's W warp ranges are served by a thread-block cluster of W / 4
// CTAs of four warps each (ptmg_cluster), spread over as many SMs: CTA rank r
// takes ranges [4 r, 4 r + 4). The tree, and so every sum, is the same as
// one CTA of W warps would take.
constexpr int kPtmgCtaWarps = 4;
constexpr int kPtmgCtaThreads = kPtmgCtaWarps * 32;
constexpr int ptmg_cluster(int nb, int nv) { return ptmg_warps(nb, nv) / kPtmgCtaWarps; }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

template <int N>
__device__ __forceinline__ void reduce_to(const double* acc, double* slot, int lane) {
#pragma unroll
  for (int v = 0; v < N; ++v) {
    double s = warp_sum(acc[v]);
    if (lane == 0) slot[v] = s;
  }
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

// The varying design values of cell r and eta over them from `start`.
template <int NB, int NV>
__device__ __forceinline__ void varying_row(const double* __restrict__ design, const int* vc, int r, double* x) {
  const double* row = design + static_cast<size_t>(r) * NB;
#pragma unroll
  for (int j = 0; j < NV; ++j) x[j] = __ldg(row + vc[j]);
}

template <int NV>
__device__ __forceinline__ double eta_from(const double* x, const double* beta, double start) {
  double eta = start;
#pragma unroll
  for (int j = 0; j < NV; ++j) eta = nb_fma(x[j], beta[j], eta);
  return eta;
}

// Pass two's dense (count zero) contribution of one cell.
template <int NV>
__device__ __forceinline__ void dense_two(double* acc, const double* x, double e, double ym, double gamma,
                                          const NbTableData* tab) {
  using D = RDims<NV>;
  const double we = ym * e;
  const double w = we + gamma;
  const double lw = nb_log_tab(w, tab);
  const double iw = nb_recip(w);
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
  acc[D::kE] += e;
  acc[D::kEq] = nb_fma(e, q, acc[D::kEq]);
  int t = 0;
#pragma unroll
  for (int a = 0; a < NV; ++a) {
    const double xe = x[a] * e;
    acc[D::kXf + a] += xe;
    acc[D::kD41 + a] = nb_fma(gg, xe, acc[D::kD41 + a]);
    acc[D::kT1 + a] = nb_fma(xe, f1, acc[D::kT1 + a]);
    acc[D::kT2 + a] = nb_fma(xe, gte, acc[D::kT2 + a]);
    acc[D::kQv + a] = nb_fma(xe, q, acc[D::kQv + a]);
#pragma unroll
    for (int b = a; b < NV; ++b) {
      const double c = xe * x[b];
      acc[D::kBp + t] += c;
      acc[D::kBq + t] = nb_fma(c, q, acc[D::kBq + t]);
      ++t;
    }
  }
}

// What a positive count y adds to a cell's pass-two contribution.
template <int NV>
__device__ __forceinline__ void sparse_two(double* acc, const double* x, double e, double y, double ym,
                                           double gamma, const NbTableData* tab) {
  using D = RDims<NV>;
  const double w = ym * e + gamma;
  const double lw = nb_log_tab(w, tab);
  const double iw = nb_recip(w);
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
  acc[D::kEq] = nb_fma(e, q, acc[D::kEq]);
  int t = 0;
#pragma unroll
  for (int a = 0; a < NV; ++a) {
    const double xe = x[a] * e;
    acc[D::kD41 + a] = nb_fma(gg, xe, acc[D::kD41 + a]);
    acc[D::kT1 + a] = nb_fma(xe, gt, acc[D::kT1 + a]);
    acc[D::kT2 + a] = nb_fma(xe, gte, acc[D::kT2 + a]);
    acc[D::kQv + a] = nb_fma(xe, q, acc[D::kQv + a]);
#pragma unroll
    for (int b = a; b < NV; ++b) {
      const double cc = xe * x[b];
      acc[D::kBq + t] = nb_fma(cc, q, acc[D::kBq + t]);
      ++t;
    }
  }
}

// Shared-memory and scratch views of one stage-one CTA.
struct PtmgCta {
  const NbTableData* tab;  // exp/log tables (nbmath.hpp), shared memory
  double* ym;        // K
  double* p1;        // K x 2: cumsumxtb, ylin
  double* cs;        // K: the constant columns' share of eta for this request
  uint32_t* fid;     // K + 1
  uint32_t* wcells;  // ptmg_warps + 1
  int32_t* vpos;     // kMaxCoef: each column's index among the varying ones, or -1
  double* slots;     // the cluster's scratch: warp and subject pieces
  double* reduced;   // the cluster's scratch: K reduced pass-two rows
  int rank, size;    // this CTA's place in its cluster
};

__device__ __forceinline__ void cluster_sync(const PtmgCta& c) {
  if (c.size > 1) cg::this_cluster().sync();  // barrier.cluster: release / acquire at cluster scope
  else __syncthreads();
}

// One pass through the segment tree: warp w of the request sums its cell
// range [wcells[w], wcells[w + 1]) one subject segment at a time, first the
// segment's cells (dense, at a count of zero) and then, into the same
// partials, the positive entries whose cells fall in the segment (sparse),
// into slots[(s + w) * stride]; then per subject
// out[s * out_stride + v] = 0 + the pieces of the warps that meet it, in warp
// order, by every CTA of the cluster (`all_combine`) or by rank 0 alone.
// Lanes take two cells (r, r + 32) or entries per iteration; each lane's
// partials still take them in its sequential order. The warp ranges are
// every (64 / W)-th of the fit's 64 cell ranges, so their first positive
// entries are the gene's range_pos there.
template <int NB, int NV, int PASS, int N>
__device__ void tree_pass(const GeneData& d, const PtmgCta& c, int gene, const double* beta, double gamma,
                          const int* vc, int stride, double* out, int out_stride, bool all_combine) {
  const int K = d.n_subjects;
  constexpr int W = ptmg_warps(NB, NV);
  static_assert(kRanges % W == 0, "warp ranges are unions of the fit's cell ranges");
  constexpr int kStep = kRanges / W;
  const int warp = c.rank * kPtmgCtaWarps + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  constexpr int NX = NV > 0 ? NV : 1;
  const int c_begin = static_cast<int>(c.wcells[warp]), c_end = static_cast<int>(c.wcells[warp + 1]);
  if (c_begin < c_end) {
    const uint64_t* runs = d.runs + static_cast<size_t>(gene) * (K + 1);
    const uint64_t* rpos = d.range_pos + static_cast<size_t>(gene) * (kRanges + 1);
    uint64_t pa = rpos[warp * kStep];
    const uint64_t p_last = rpos[(warp + 1) * kStep];
    int s = subject_of(c.fid, K, c_begin);
    for (int c0 = c_begin; c0 < c_end; ++s) {
      const int s_end = min(c_end, static_cast<int>(c.fid[s + 1]));
      const uint64_t p_end = s_end == c_end ? p_last : runs[s + 1];
      double acc[N];
#pragma unroll
      for (int v = 0; v < N; ++v) acc[v] = 0.0;
      const double yms = PASS == 2 ? c.ym[s] : 0.0;
      const double cs = c.cs[s];
      // each lane's next two rows and offsets are loaded one iteration
      // ahead, so their latency overlaps the current cells' arithmetic
      int r = c0 + lane;
      double xa[NX], xb[NX], oa = 0.0, ob = 0.0;
      if (r < s_end) {
        const int rb = r + 32 < s_end ? r + 32 : r;
        varying_row<NB, NV>(d.design, vc, r, xa);
        varying_row<NB, NV>(d.design, vc, rb, xb);
        oa = __ldg(d.log_offset + r);
        ob = __ldg(d.log_offset + rb);
      }
      for (; r < s_end; r += 64) {
        const bool has_b = r + 32 < s_end;
        const int rn = r + 64 < s_end ? r + 64 : r;
        const int rnb = rn + 32 < s_end ? rn + 32 : rn;
        double xna[NX], xnb[NX];
        varying_row<NB, NV>(d.design, vc, rn, xna);
        varying_row<NB, NV>(d.design, vc, rnb, xnb);
        const double ona = __ldg(d.log_offset + rn), onb = __ldg(d.log_offset + rnb);
        const double ea = nb_exp_tab(eta_from<NV>(xa, beta, oa + cs), c.tab);
        const double eb = nb_exp_tab(eta_from<NV>(xb, beta, ob + cs), c.tab);
        if constexpr (PASS == 1) {
          acc[0] += ea;
          if (has_b) acc[0] += eb;
        } else {
          dense_two<NV>(acc, xa, ea, yms, gamma, c.tab);
          if (has_b) dense_two<NV>(acc, xb, eb, yms, gamma, c.tab);
        }
#pragma unroll
        for (int j = 0; j < NV; ++j) {
          xa[j] = xna[j];
          xb[j] = xnb[j];
        }
        oa = ona;
        ob = onb;
      }
      // the segment's positive entries, continuing the same partials
      for (uint64_t p = pa + lane; p < p_end; p += 64) {
        const bool has_b = p + 32 < p_end;
        const uint64_t pb = has_b ? p + 32 : p;
        const int ca = static_cast<int>(__ldg(d.cells + p)), cb = static_cast<int>(__ldg(d.cells + pb));
        const double ya = __ldg(d.counts + p), yb = __ldg(d.counts + pb);
        double xca[NX], xcb[NX];
        varying_row<NB, NV>(d.design, vc, ca, xca);
        varying_row<NB, NV>(d.design, vc, cb, xcb);
        const double eta_a = eta_from<NV>(xca, beta, __ldg(d.log_offset + ca) + cs);
        const double eta_b = eta_from<NV>(xcb, beta, __ldg(d.log_offset + cb) + cs);
        if constexpr (PASS == 1) {
          acc[1] = nb_fma(eta_a, ya, acc[1]);
          if (has_b) acc[1] = nb_fma(eta_b, yb, acc[1]);
        } else {
          sparse_two<NV>(acc, xca, nb_exp_tab(eta_a, c.tab), ya, yms, gamma, c.tab);
          if (has_b) sparse_two<NV>(acc, xcb, nb_exp_tab(eta_b, c.tab), yb, yms, gamma, c.tab);
        }
      }
      reduce_to<N>(acc, c.slots + (s + warp) * stride, lane);
      pa = p_end;
      c0 = s_end;
    }
  }
  cluster_sync(c);  // every CTA's pieces are in the scratch (read past L1)
  if (all_combine || c.rank == 0) {
    for (int idx = threadIdx.x; idx < K * N; idx += blockDim.x) {
      const int s = idx / N, v = idx - s * N;
      const uint32_t a0 = c.fid[s], a1 = c.fid[s + 1];
      double total = 0.0;
#pragma unroll
      for (int w = 0; w < W; ++w)
        if (c.wcells[w] < a1 && c.wcells[w + 1] > a0) total += __ldcg(c.slots + (s + w) * stride + v);
      out[s * out_stride + v] = total;
    }
  }
  cluster_sync(c);  // no CTA refills the pieces before every combine has read them
}

// Subject s's full pass-two row (PDims<NB>) from its reduced one, element x.
template <int NB, int NV>
__device__ __forceinline__ double expand_two(const double* R, const double* X, const int32_t* vpos, int x) {
  using F = PDims<NB>;
  using D = RDims<NV>;
  if (x < F::kXf) return R[x];
  if (x < F::kBp) {
    const int part = (x - F::kXf) / NB, a = (x - F::kXf) - part * NB, va = vpos[a];
    const int from[4] = {D::kXf, D::kD41, D::kT1, D::kT2};
    const int scalar[4] = {D::kE, 6, 7, 8};
    return va >= 0 ? R[from[part] + va] : X[a] * R[scalar[part]];
  }
  const bool q = x >= F::kBq;
  int a = 0, rem = x - (q ? F::kBq : F::kBp);
  while (rem >= NB - a) {
    rem -= NB - a;
    ++a;
  }
  const int b = a + rem, va = vpos[a], vb = vpos[b];
  const int vec = q ? D::kQv : D::kXf;
  if (va >= 0 && vb >= 0) return R[(q ? D::kBq : D::kBp) + va * NV - va * (va - 1) / 2 + (vb - va)];
  if (vb >= 0) return X[a] * R[vec + vb];
  if (va >= 0) return X[b] * R[vec + va];
  return X[a] * (X[b] * R[q ? D::kEq : D::kE]);
}

template <int NB, int NV>
__device__ PtmgCta ptmg_setup(const GeneData& d, double* smem, double* scratch) {
  const int K = d.n_subjects;
  constexpr int W = ptmg_warps(NB, NV);
  PtmgCta c;
  NbTableData* tab = reinterpret_cast<NbTableData*>(smem);
  nb_load_tables(tab);  // first used after the request loop's opening cluster barrier
  c.tab = tab;
  c.ym = smem + kNbTableDoubles;
  c.p1 = c.ym + K;
  c.cs = c.p1 + 2 * K;
  c.fid = reinterpret_cast<uint32_t*>(c.cs + K);
  c.wcells = c.fid + K + 1;
  c.vpos = reinterpret_cast<int32_t*>(c.wcells + W + 1);
  for (int i = threadIdx.x; i <= K; i += blockDim.x) c.fid[i] = d.fid[i];
  if (threadIdx.x <= W) c.wcells[threadIdx.x] = d.warp_cells[threadIdx.x];
  if (threadIdx.x < NB) {
    int pos = -1;
    for (int j = 0; j < NV; ++j)
      if (d.varying[j] == static_cast<int>(threadIdx.x)) pos = j;
    c.vpos[threadIdx.x] = pos;
  }
  c.size = ptmg_cluster(NB, NV);
  c.rank = c.size > 1 ? static_cast<int>(cg::this_cluster().block_rank()) : 0;
  // per cluster: the K + W segment pieces, then the K reduced rows
  const size_t per_cta = static_cast<size_t>(2 * K + W) * RDims<NV>::W;
  c.slots = scratch + static_cast<size_t>(blockIdx.x / c.size) * per_cta;
  c.reduced = c.slots + static_cast<size_t>(K + W) * RDims<NV>::W;
  return c;
}

// Both passes of one request into `out` ((2 + W) K doubles).
template <int NB, int NV>
__device__ void ptmg_one(const GeneData& d, const PtmgCta& c, const PtmgRequest& req, double* beta_sm, double* out) {
  using F = PDims<NB>;
  using D = RDims<NV>;
  constexpr int NX = NV > 0 ? NV : 1;
  const int K = d.n_subjects;
  const int tid = threadIdx.x;
  if (tid < NB) beta_sm[tid] = req.beta[tid];
  __syncthreads();
  // the constant columns' share of eta per subject, in column order
  for (int s = tid; s < K; s += blockDim.x) {
    double v = 0.0;
    if (c.fid[s] < c.fid[s + 1]) {
      const double* row = d.design + static_cast<size_t>(c.fid[s]) * NB;
#pragma unroll
      for (int a = 0; a < NB; ++a)
        if (c.vpos[a] < 0) v = nb_fma(__ldg(row + a), beta_sm[a], v);
    }
    c.cs[s] = v;
  }
  int vc[NX];
  double beta[NX];
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    vc[j] = d.varying[j];
    beta[j] = beta_sm[vc[j]];
  }
  __syncthreads();
  tree_pass<NB, NV, 1, 2>(d, c, req.gene, beta, req.gamma, vc, D::W, c.p1, 2, true);
  const double* tot = d.totals + static_cast<size_t>(req.gene) * K;
  for (int s = tid; s < K; s += blockDim.x) {
    c.ym[s] = (__ldg(tot + s) + req.alpha) / (c.p1[2 * s] + req.lambda);
    if (c.rank == 0) {
      out[s] = c.p1[2 * s];          // cumsumxtb
      out[K + s] = c.p1[2 * s + 1];  // ylin
    }
  }
  __syncthreads();
  tree_pass<NB, NV, 2, D::W>(d, c, req.gene, beta, req.gamma, vc, D::W, c.reduced, D::W, false);
  if (c.rank != 0) return;  // rank 0 writes the result
  // every subject's full row, the constant columns' sums from the scalars
  for (int idx = tid; idx < K * F::W; idx += blockDim.x) {
    const int s = idx / F::W, x = idx - s * F::W;
    double X[NB];
    const bool has = c.fid[s] < c.fid[s + 1];
    const double* row = d.design + static_cast<size_t>(has ? c.fid[s] : 0) * NB;
#pragma unroll
    for (int a = 0; a < NB; ++a) X[a] = has ? __ldg(row + a) : 0.0;
    out[2 * K + idx] = expand_two<NB, NV>(c.reduced + static_cast<size_t>(s) * D::W, X, c.vpos, x);
  }
}

// Streaming mode: one persistent launch for stage one, the request-ring
// protocol of FitQueue (pml_device.cuh) with one cluster per request: rank
// 0's first warp takes the ticket and hands it and the request to the other
// CTAs, every CTA sweeps its ranges, rank 0 writes the result.
template <int NB, int NV>
__global__ void __launch_bounds__(kPtmgCtaThreads, ptmg_cluster(NB, NV))
    ptmg_queue_kernel(GeneData d, PtmgQueue qu, double* scratch) {
  extern __shared__ __align__(16) double smem[];
  const PtmgCta c = ptmg_setup<NB, NV>(d, smem, scratch);
  __shared__ long long next_ticket;
  __shared__ PtmgRequest next_req;
  __shared__ double beta_sm[kMaxCoef];
  for (;;) {
    cluster_sync(c);  // nobody still reads the previous ticket and request
    if (c.rank == 0 && threadIdx.x < 32) {
      const long long got = ring_next(qu.ring, &next_req, nullptr);
      if (threadIdx.x == 0) next_ticket = got;
      if (c.size > 1) {
        cg::cluster_group cluster = cg::this_cluster();
        constexpr int kWords = static_cast<int>(sizeof(PtmgRequest) / 8);
        const unsigned long long* mine = reinterpret_cast<const unsigned long long*>(&next_req);
        for (int r = 1; r < c.size; ++r) {
          if (threadIdx.x == 0) *cluster.map_shared_rank(&next_ticket, r) = got;
          if (static_cast<int>(threadIdx.x) < kWords && got >= 0)
            cluster.map_shared_rank(reinterpret_cast<unsigned long long*>(&next_req), r)[threadIdx.x] =
                mine[threadIdx.x];
        }
      }
    }
    cluster_sync(c);
    const long long t = next_ticket;
    if (t < 0) break;
    const PtmgRequest req = next_req;
    ptmg_one<NB, NV>(d, c, req, beta_sm, qu.results + (t & qu.ring.mask) * qu.result_stride);
    if (c.rank == 0) ring_publish(qu.done + (t & qu.ring.mask), t);
  }
  cluster_sync(c);  // no CTA leaves while another may still write its shared memory
}

inline size_t smem_bytes(int K) {
  return static_cast<size_t>(kNbTableDoubles + 4 * K) * 8 + (K + 1 + kMaxPtmgWarps + 1 + kMaxCoef) * 4 + 16;
}

template <int NB, int NV>
cudaLaunchConfig_t ptmg_config(int grid, size_t smem, cudaStream_t stream, cudaLaunchAttribute* attr) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid, 1, 1);
  cfg.blockDim = dim3(kPtmgCtaThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = ptmg_cluster(NB, NV);
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

template <int NB, int NV>
int launch_queue_nb(const GeneData& d, const PtmgQueue& qu, double* scratch, int grid, cudaStream_t stream) {
  const size_t smem = smem_bytes(d.n_subjects);
  cudaError_t e = cudaFuncSetAttribute(ptmg_queue_kernel<NB, NV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  if (grid % ptmg_cluster(NB, NV) != 0) return cudaErrorInvalidValue;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = ptmg_config<NB, NV>(grid, smem, stream, attr);
  return cudaLaunchKernelEx(&cfg, ptmg_queue_kernel<NB, NV>, d, qu, scratch);
}

// CTAs the kernel keeps resident at once: whole clusters.
template <int NB, int NV>
int resident_nb(int K) {
  const size_t smem = smem_bytes(K);
  if (cudaFuncSetAttribute(ptmg_queue_kernel<NB, NV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(smem)) != cudaSuccess)
    return 0;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = ptmg_config<NB, NV>(ptmg_cluster(NB, NV), smem, nullptr, attr);
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, ptmg_queue_kernel<NB, NV>, &cfg) != cudaSuccess) return 0;
  return clusters * ptmg_cluster(NB, NV);
}

template <int NB, int NV>
size_t scratch_nb(int K) {
  return static_cast<size_t>(2 * K + ptmg_warps(NB, NV)) * RDims<NV>::W;
}

template <int NB, int NV = 0>
PtmgOps ptmg_ops_for(int n_varying) {
  if constexpr (NV > NB) {
    return PtmgOps{};
  } else {
    if (n_varying == NV) return PtmgOps{&launch_queue_nb<NB, NV>, &resident_nb<NB, NV>, &scratch_nb<NB, NV>};
    return ptmg_ops_for<NB, NV + 1>(n_varying);
  }
}

}  // namespace
}  // namespace device
}  // namespace nebula
