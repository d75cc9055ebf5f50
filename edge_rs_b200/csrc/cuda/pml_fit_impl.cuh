// Batched penalised NB-gamma inner fit (the reference's opt_pml,
// src/sc/pml.rs:1614-1800) on sm_100a, FP64 throughout.
//
// fit_one runs the whole Newton loop of one (gene, sigma, gamma) request:
// sweep, Schur complement, pivoted LDL' solve, backtracking, log-determinant
// and the higher-order Laplace pass. Two kernels drive it: fit_kernel (batch:
// persistent clusters over an atomic counter of a request array) and
// fit_queue_kernel (one persistent launch per call, fed by the host through
// a device ring of requests with per-slot sequence numbers). Either runs a
// request on a cluster of 1, 2, 4 or 8 CTAs that share its sweeps.
//
// A sweep (pml.rs:1419-1590) splits each subject into a dense part over every
// cell at a count of zero and a sparse part over the gene's positive counts.
// The cells are cut into kRanges fixed ranges; each subject segment of a
// range is one piece, summed by a warp's lanes over its cells and then its
// positive entries and butterfly-reduced into a shared-memory slot; a combine
// step sums each subject's pieces in range order, reading other CTAs' pieces
// through distributed shared memory. No atomics, and the tree does not depend
// on the launch shape, so results are bitwise reproducible.
//
// The per-request scalars (Newton state, step sizes, loop flags) live in
// shared memory and are written by thread 0 between barriers, so every
// thread of the CTA takes the same branches. Every loop is bounded by
// max_iter Newton steps of at most max_backtrack + 1 trial sweeps: nothing
// waits on anything.
//
// The arithmetic is that of the FP64 CPU oracle operation for operation: the
// same exp/log (nbmath.hpp), fused multiply-adds only where written (the
// file is compiled with -fmad=false), and the same summation tree, so the
// two agree bit for bit and the stage-two search retraces the same points.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cfloat>
#include <cstdint>

#include "nbmath_device.cuh"
#include "pml_device.cuh"
#include "pml_fit_ops.cuh"
#include "ring_device.cuh"

namespace cg = cooperative_groups;

namespace nebula {
namespace device {
namespace {

constexpr double kStepCutoff = 40.0;        // pml.rs:74
constexpr double kGradientTolerance = 0.01; // pml.rs:67

// Slot layout of one per-subject partial: resid, weight, sum ln t,
// sum y*eta, sum y ln t, X'd (NB), sum p x (NB), sum p x x' (upper, NB(NB+1)/2).
enum : int { kResid = 0, kWeight = 1, kSumLog = 2, kLinear = 3, kWlog = 4, kScore = 5 };
template <int NB>
struct Dims {
  static constexpr int T = NB * (NB + 1) / 2;
  static constexpr int NS = 5 + 2 * NB + T;
  static constexpr int kFirst = kScore + NB;
  static constexpr int kSecond = kFirst + NB;
};
constexpr int kLaplaceSums = 4;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// Reduced per-cell slot of a sweep over NV varying design columns: resid,
// weight, sum ln t, sum y*eta, sum y ln t, then over the varying columns only
// X'd (NV), sum p x (NV) and sum p x x' (upper, NV(NV+1)/2). The subject-
// constant columns' shares are applied per subject after the combine
// (expand_slot).
template <int NV>
struct Reduced {
  static constexpr int kFirst = kScore + NV;
  static constexpr int kSecond = kFirst + NV;
  static constexpr int NS = kSecond + NV * (NV + 1) / 2;
  static constexpr int NP = NS > kLaplaceSums ? NS : kLaplaceSums;  // piece stride (fit or Laplace sums)
};

// Shared-memory carve-up for one CTA (all offsets in doubles).
template <int NB, int NV>
struct Smem {
  static constexpr int NP = Reduced<NV>::NP;
  int K;
  NbTableData* tab;      // exp/log tables (nbmath.hpp)
  double* pieces[2];     // (K + kRanges) x NP each: one sweep's (subject, range) pieces, by sweep parity
  double* rtot;          // K x NP, per-subject reduced totals after the combine
  double* totals;        // K x NS (Dims<NB>), per-subject totals over every column
  double* sw[2];         // two sweeps: w K, dw K, vw K, vwb K*NB, db NB, vb NB*NB, ll 1
  double* beta;          // NB
  double* log_w;         // K
  double* new_beta;      // NB
  double* new_log_w;     // K
  double* step_beta;     // NB
  double* step_log_w;    // K
  double* dwvw;          // K
  double* damp_beta;     // NB
  double* damp_log_w;    // K
  double* vw_step;       // K
  double* vb2;           // NB*NB
  double* factor;        // NB*NB
  double* llv;           // K (per-subject log-likelihood terms)
  double* sc;            // 16 scalars
  double* xs;            // K x NB: each subject's design row (its constant columns' values)
  double* cs;            // K: the constant columns' share of eta this sweep
  double* csl;           // K: cs + log_w
  uint64_t* rpos;        // kRanges + 1: the request's gene's range_pos row
  uint64_t* runs;        // K + 1: the request's gene's first positive entry per subject
  uint32_t* fid;         // K + 1
  uint32_t* rcells;      // kRanges + 1
  int32_t* vlo;          // K: first range meeting each subject
  int32_t* vhi;          // K: last range meeting each subject
  int32_t* vpos;         // NB: each column's index among the varying columns, or -1

  __host__ __device__ static size_t sweep_doubles(int K) { return 3 * K + K * NB + NB + NB * NB + 1; }
  __host__ __device__ static size_t doubles(int K) {
    return (size_t)kNbTableDoubles + (size_t)(3 * K + 2 * kRanges) * NP +
           (size_t)K * Dims<NB>::NS + 2 * sweep_doubles(K) + 4 * NB + 7 * K + 2 * NB * NB + 16 +
           (size_t)K * NB + 2 * K + (kRanges + 1) + (K + 1);
  }
  __host__ __device__ static size_t bytes(int K) {
    return doubles(K) * 8 + (size_t)(K + 1 + kRanges + 1 + 2 * K + NB) * 4 + 16;
  }

  __device__ void carve(double* base, int K_) {
    K = K_;
    double* p = base;
    tab = reinterpret_cast<NbTableData*>(p);
    p += kNbTableDoubles;
    pieces[0] = p;
    p += (K + kRanges) * NP;
    pieces[1] = p;
    p += (K + kRanges) * NP;
    rtot = p;
    p += K * NP;
    totals = p;
    p += K * Dims<NB>::NS;
    sw[0] = p;
    p += sweep_doubles(K);
    sw[1] = p;
    p += sweep_doubles(K);
    beta = p; p += NB;
    log_w = p; p += K;
    new_beta = p; p += NB;
    new_log_w = p; p += K;
    step_beta = p; p += NB;
    step_log_w = p; p += K;
    dwvw = p; p += K;
    damp_beta = p; p += NB;
    damp_log_w = p; p += K;
    vw_step = p; p += K;
    vb2 = p; p += NB * NB;
    factor = p; p += NB * NB;
    llv = p; p += K;
    sc = p; p += 16;
    xs = p; p += K * NB;
    cs = p; p += K;
    csl = p; p += K;
    rpos = reinterpret_cast<uint64_t*>(p);
    p += kRanges + 1;
    runs = reinterpret_cast<uint64_t*>(p);
    p += K + 1;
    fid = reinterpret_cast<uint32_t*>(p);
    rcells = fid + K + 1;
    vlo = reinterpret_cast<int32_t*>(rcells + kRanges + 1);
    vhi = vlo + K;
    vpos = vhi + K;
  }
};

// Views into one sweep's storage.
template <int NB>
struct SweepView {
  double *w, *dw, *vw, *vwb, *db, *vb, *ll;
  __device__ SweepView(double* p, int K) {
    w = p;
    dw = p + K;
    vw = p + 2 * K;
    vwb = p + 3 * K;
    db = vwb + K * NB;
    vb = db + NB;
    ll = vb + NB * NB;
  }
};

// Scalar slots in Smem::sc.
enum : int {
  kLl = 0, kLlPrev = 1, kLikdif = 2, kMinStep = 3, kStep = 4, kBacktracks = 5, kStop = 6,
  kSweeps = 7, kAlpha = 8, kLambda = 9, kGamma = 10, kLogDet = 11, kSecond = 12, kCur = 13
};

__device__ __forceinline__ int subject_of(const uint32_t* fid, int K, int c) {
  int lo = 0, hi = K;  // fid[lo] <= c < fid[hi]
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (fid[mid] <= static_cast<uint32_t>(c)) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Per-cell fold (pml.rs:1469-1489) into the register accumulator, over the
// varying columns only (Reduced<NV> layout).
template <int NV>
__device__ __forceinline__ void fold(double* acc, const double* x, double d, double p) {
  acc[kResid] += d;
  acc[kWeight] += p;
  int t = 0;
#pragma unroll
  for (int a = 0; a < NV; ++a) {
    acc[kScore + a] = nb_fma(x[a], d, acc[kScore + a]);
    double pa = p * x[a];
    acc[Reduced<NV>::kFirst + a] += pa;
#pragma unroll
    for (int b = a; b < NV; ++b) {
      acc[Reduced<NV>::kSecond + t] = nb_fma(pa, x[b], acc[Reduced<NV>::kSecond + t]);
      ++t;
    }
  }
}

// The four per-cell Laplace sums (pml.rs:1842-1856, 1863-1868, 1893-1899),
// each term scaled by gamma (dense) or the count (sparse).
__device__ __forceinline__ void laplace_terms(double* acc, double e, double t, double gamma, double scale) {
  const double inv = nb_recip(t);
  const double p2 = (e * inv) * inv, p3 = p2 * inv, p4 = p3 * inv, p5 = p4 * inv, e2 = e * e;
  acc[0] += scale * p2;
  acc[1] += scale * (p3 * (gamma - e));
  acc[2] += scale * (p4 * (gamma * gamma + e2 - (4.0 * gamma) * e));
  acc[3] += scale * (p5 * (gamma * gamma * gamma - (11.0 * gamma * gamma) * e + (11.0 * gamma) * e2 - e2 * e));
}

// eta over the varying columns, continuing from `start` (the offset plus
// the subject's constant share).
template <int NV>
__device__ __forceinline__ double linear_eta(const double* x, const double* beta, double start) {
  double eta = start;
#pragma unroll
  for (int j = 0; j < NV; ++j) eta = nb_fma(x[j], beta[j], eta);
  return eta;
}

template <int NV>
__device__ __forceinline__ void reduce_to(double* acc, double* slot, int lane) {
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double s = warp_sum(acc[v]);
    if (lane == 0) slot[v] = s;
  }
}

// Which CTA of its cluster this is, and how many CTAs share each request.
struct Cluster {
  int rank, size;
};

__device__ __forceinline__ void cluster_barrier(const Cluster& cl) {
  if (cl.size > 1) cg::this_cluster().sync();
  else __syncthreads();
}

// One sweep's per-subject sums into sm.rtot (Reduced<NV> slots). Mode 0:
// the fit sums of sweep_width; mode 1: the four Laplace sums
// (pml.rs:1842-1899).
//
// eta splits into the subject-constant columns' share, summed once per
// subject (cs, and csl = cs + log_w for the dense cells), and the varying
// columns, summed per cell from it: dense cells take exp(off + csl + x_v b_v),
// positive entries eta = off + cs + x_v b_v and exp(eta + log_w).
//
// The cells are cut into kRanges fixed ranges; the cluster's CTAs split the
// ranges (rank r takes kRanges / size consecutive ones) and a CTA's warps
// take its ranges in turn. Within a range, each subject segment is one
// piece: lanes stride the segment's cells at a count of zero (dense), then,
// into the same partials, the gene's positive entries in the segment
// (sparse, what each count changes), then the warp butterfly-reduces the
// partials into the piece's slot (subject + range, unique because both
// advance together). After a cluster barrier every CTA combines, per
// subject and in range order, the pieces of the ranges that meet it, reading
// other CTAs' pieces through distributed shared memory. The pieces are
// double-buffered by sweep parity, so the next sweep's writes never race this
// combine and one barrier per sweep suffices.
template <int NB, int NV, int MODE>
__device__ void sweep_sums(const GeneData& d, Smem<NB, NV>& sm, const double* beta_sm, const double* log_w,
                           double gamma, int parity, const Cluster& cl) {
  constexpr int NPV = MODE == 0 ? Reduced<NV>::NS : kLaplaceSums;
  constexpr int NP = Smem<NB, NV>::NP;
  constexpr int NX = NV > 0 ? NV : 1;  // array extent
  const int K = sm.K;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const NbTableData* tab = sm.tab;
  double* pieces = sm.pieces[parity];
  // the constant columns' share of eta, per subject, in column order
  for (int s = threadIdx.x; s < K; s += blockDim.x) {
    double c = 0.0;
#pragma unroll
    for (int a = 0; a < NB; ++a)
      if (sm.vpos[a] < 0) c = nb_fma(sm.xs[s * NB + a], beta_sm[a], c);
    sm.cs[s] = c;
    sm.csl[s] = c + log_w[s];
  }
  int vc[NX];
  double beta[NX];
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    vc[j] = d.varying[j];
    beta[j] = beta_sm[vc[j]];
  }
  __syncthreads();

  const int per_cta = kRanges / cl.size;
  for (int v = cl.rank * per_cta + warp; v < (cl.rank + 1) * per_cta; v += kWarps) {
    const int a = static_cast<int>(sm.rcells[v]), b = static_cast<int>(sm.rcells[v + 1]);
    if (a >= b) continue;
    int s = subject_of(sm.fid, K, a);
    uint64_t pa = sm.rpos[v];
    const uint64_t pv_end = sm.rpos[v + 1];
    for (int c0 = a; c0 < b; ++s) {
      const int s_end = min(b, static_cast<int>(sm.fid[s + 1]));
      const uint64_t p_end = min(sm.runs[s + 1], pv_end);
      const double lw = log_w[s];
      const double cs = sm.cs[s], csl = sm.csl[s];
      double acc[NPV];
#pragma unroll
      for (int x = 0; x < NPV; ++x) acc[x] = 0.0;
      // dense: two cells (r and r + 32) per iteration; their exp/log/division
      // chains interleave, and each accumulator still takes cell r before
      // cell r + 32, the order of the lane's sequential sum. The cells'
      // varying design values and offsets are read straight from L2 (the
      // other resident warps hide the latency): staging the next iteration's
      // rows in shared memory with cp.async cost more issue slots than it
      // saved (warm c1 65.1 against 62.8-63.4 ms a step).
      if (d.tabled) {
        // zero-count tables: the dense part visits the segment's loose cells
        // only, two per iteration like the positive entries below
        const uint64_t q_begin = max(static_cast<uint64_t>(__ldg(d.subject_loose + s)), __ldg(d.loose_pos + v));
        const uint64_t q_end = min(static_cast<uint64_t>(__ldg(d.subject_loose + s + 1)), __ldg(d.loose_pos + v + 1));
        for (uint64_t q = q_begin + lane; q < q_end; q += 64) {
          const bool has_b = q + 32 < q_end;
          const int ca = static_cast<int>(__ldg(d.loose + q)), cb = static_cast<int>(__ldg(d.loose + (has_b ? q + 32 : q)));
          double xa[NX], xb[NX];
#pragma unroll
          for (int j = 0; j < NV; ++j) {
            xa[j] = __ldg(d.design + static_cast<size_t>(ca) * NB + vc[j]);
            xb[j] = __ldg(d.design + static_cast<size_t>(cb) * NB + vc[j]);
          }
          const double ea = nb_exp_tab(linear_eta<NV>(xa, beta, __ldg(d.log_offset + ca) + csl), tab);
          const double eb = nb_exp_tab(linear_eta<NV>(xb, beta, __ldg(d.log_offset + cb) + csl), tab);
          const double ta = ea + gamma, tb = eb + gamma;
          if (MODE == 0) {
            const double la = nb_log_tab(ta, tab), lb = nb_log_tab(tb, tab);
            const double inva = nb_recip(ta), invb = nb_recip(tb);
            const double ua = ea * inva, ub = eb * invb;
            acc[kSumLog] += la;
            fold<NV>(acc, xa, -gamma * ua, (gamma * ua) * inva);
            if (has_b) {
              acc[kSumLog] += lb;
              fold<NV>(acc, xb, -gamma * ub, (gamma * ub) * invb);
            }
          } else {
            laplace_terms(acc, ea, ta, gamma, gamma);
            if (has_b) laplace_terms(acc, eb, tb, gamma, gamma);
          }
        }
      } else {
        for (int r = c0 + lane; r < s_end; r += 64) {
          const bool has_b = r + 32 < s_end;
          const int rb = has_b ? r + 32 : r;
          double xa[NX], xb[NX];
#pragma unroll
          for (int j = 0; j < NV; ++j) {
            xa[j] = __ldg(d.design + static_cast<size_t>(r) * NB + vc[j]);
            xb[j] = __ldg(d.design + static_cast<size_t>(rb) * NB + vc[j]);
          }
          const double offa = __ldg(d.log_offset + r), offb = __ldg(d.log_offset + rb);
          const double ea = nb_exp_tab(linear_eta<NV>(xa, beta, offa + csl), tab);
          const double eb = nb_exp_tab(linear_eta<NV>(xb, beta, offb + csl), tab);
          const double ta = ea + gamma, tb = eb + gamma;
          if (MODE == 0) {
            const double la = nb_log_tab(ta, tab), lb = nb_log_tab(tb, tab);
            const double inva = nb_recip(ta), invb = nb_recip(tb);
            const double ua = ea * inva, ub = eb * invb;
            acc[kSumLog] += la;
            fold<NV>(acc, xa, -gamma * ua, (gamma * ua) * inva);
            if (has_b) {
              acc[kSumLog] += lb;
              fold<NV>(acc, xb, -gamma * ub, (gamma * ub) * invb);
            }
          } else {
            laplace_terms(acc, ea, ta, gamma, gamma);
            if (has_b) laplace_terms(acc, eb, tb, gamma, gamma);
          }
        }
      }
      // sparse: the segment's positive entries, into the same partials
      for (uint64_t p = pa + lane; p < p_end; p += 64) {
        const bool has_b = p + 32 < p_end;
        const uint64_t pb = has_b ? p + 32 : p;
        const int ca = static_cast<int>(__ldg(d.cells + p)), cb = static_cast<int>(__ldg(d.cells + pb));
        const double ya = __ldg(d.counts + p), yb = __ldg(d.counts + pb);
        double xa[NX], xb[NX];
#pragma unroll
        for (int j = 0; j < NV; ++j) {
          xa[j] = __ldg(d.design + static_cast<size_t>(ca) * NB + vc[j]);
          xb[j] = __ldg(d.design + static_cast<size_t>(cb) * NB + vc[j]);
        }
        const double eta_a = linear_eta<NV>(xa, beta, __ldg(d.log_offset + ca) + cs);
        const double eta_b = linear_eta<NV>(xb, beta, __ldg(d.log_offset + cb) + cs);
        const double ea = nb_exp_tab(eta_a + lw, tab), eb = nb_exp_tab(eta_b + lw, tab);
        const double ta = ea + gamma, tb = eb + gamma;
        if (MODE == 0) {
          const double la = nb_log_tab(ta, tab), lb = nb_log_tab(tb, tab);
          const double inva = nb_recip(ta), invb = nb_recip(tb);
          const double ua = ea * inva, ub = eb * invb;
          acc[kLinear] = nb_fma(eta_a, ya, acc[kLinear]);
          acc[kWlog] = nb_fma(ya, la, acc[kWlog]);
          fold<NV>(acc, xa, ya * (1.0 - ua), (ya * ua) * inva);
          if (has_b) {
            acc[kLinear] = nb_fma(eta_b, yb, acc[kLinear]);
            acc[kWlog] = nb_fma(yb, lb, acc[kWlog]);
            fold<NV>(acc, xb, yb * (1.0 - ub), (yb * ub) * invb);
          }
        } else {
          laplace_terms(acc, ea, ta, gamma, ya);
          if (has_b) laplace_terms(acc, eb, tb, gamma, yb);
        }
      }
      reduce_to<NPV>(acc, pieces + (s + v) * NP, lane);
      pa = p_end;
      c0 = s_end;
    }
  }
  cluster_barrier(cl);
  // combine: per subject, the pieces of the non-empty ranges that meet it, in range order
  for (int idx = threadIdx.x; idx < K * NPV; idx += blockDim.x) {
    const int s = idx / NPV, x = idx - s * NPV;
    double total = 0.0;
    for (int v = sm.vlo[s]; v <= sm.vhi[s]; ++v) {
      if (sm.rcells[v] >= sm.rcells[v + 1]) continue;
      const double* src = pieces + (s + v) * NP + x;
      const int owner = v / per_cta;
      if (owner != cl.rank) src = cg::this_cluster().map_shared_rank(src, owner);
      total += *src;
    }
    sm.rtot[s * NP + x] = total;
  }
  __syncthreads();
  if (d.tabled) {
    // each tabled group's cells at a count of zero, per subject in group
    // order (pml.rs:1515-1526, 1875-1885): with s = ln tau, sum ln t =
    // n ln gamma + L, sum d = -gamma A, sum p = B; the Laplace pass adds B..E
    const double ln_gamma = nb_log(gamma);
    for (int s = threadIdx.x; s < K; s += blockDim.x) {
      double* R = sm.rtot + s * NP;
      const uint32_t g_end = __ldg(d.zsubject + s + 1);
      for (uint32_t g = __ldg(d.zsubject + s); g < g_end; ++g) {
        const zero::Group G = d.zgroups[g];
        double xg[NX];
#pragma unroll
        for (int j = 0; j < NV; ++j) xg[j] = __ldg(d.design + static_cast<size_t>(G.row) * NB + vc[j]);
        const double log_tau = linear_eta<NV>(xg, beta, sm.csl[s] - ln_gamma);
        if (MODE == 0) {
          double f[3];
          zero::eval(G, d.zindex, d.zpanels, log_tau, 0, 3, f);
          R[kSumLog] += G.n * ln_gamma + f[0];
          fold<NV>(R, xg, -gamma * f[1], f[2]);
        } else {
          double f[4];
          zero::eval(G, d.zindex, d.zpanels, log_tau, 2, 4, f);
#pragma unroll
          for (int j = 0; j < 4; ++j) R[j] += f[j];
        }
      }
    }
    __syncthreads();
  }
}

// Slot x of subject s over every column (Dims<NB> layout) from its reduced
// totals: a constant column a's sums are its value times the matching sum
// without it (sum d x_a = x_a sum d, sum p x_a x_b = x_a sum p x_b, ...).
template <int NB, int NV>
__device__ __forceinline__ double expand_slot(const Smem<NB, NV>& sm, int s, int x) {
  const double* R = sm.rtot + s * Smem<NB, NV>::NP;
  const double* X = sm.xs + s * NB;
  if (x < kScore) return R[x];
  if (x < Dims<NB>::kFirst) {
    const int a = x - kScore, va = sm.vpos[a];
    return va >= 0 ? R[kScore + va] : X[a] * R[kResid];
  }
  if (x < Dims<NB>::kSecond) {
    const int a = x - Dims<NB>::kFirst, va = sm.vpos[a];
    return va >= 0 ? R[Reduced<NV>::kFirst + va] : X[a] * R[kWeight];
  }
  int a = 0, rem = x - Dims<NB>::kSecond;
  while (rem >= NB - a) {
    rem -= NB - a;
    ++a;
  }
  const int b = a + rem, va = sm.vpos[a], vb = sm.vpos[b];
  if (va >= 0 && vb >= 0) return R[Reduced<NV>::kSecond + va * NV - va * (va - 1) / 2 + (vb - va)];
  if (vb >= 0) return X[a] * R[Reduced<NV>::kFirst + vb];
  if (va >= 0) return X[b] * R[Reduced<NV>::kFirst + va];
  return X[a] * (X[b] * R[kWeight]);
}

// A full sweep into `out` (pml.rs:1564-1589).
template <int NB, int NV>
__device__ void sweep(const GeneData& d, Smem<NB, NV>& sm, int gene, const double* beta, const double* log_w,
                      SweepView<NB> out, int& parity, const Cluster& cl) {
  const int K = sm.K;
  const double gamma = sm.sc[kGamma], alpha = sm.sc[kAlpha], lambda = sm.sc[kLambda];
  sweep_sums<NB, NV, 0>(d, sm, beta, log_w, gamma, parity, cl);
  parity ^= 1;
  const double* tot = d.totals + static_cast<size_t>(gene) * K;
  const int tid = threadIdx.x;
  for (int idx = tid; idx < K * Dims<NB>::NS; idx += blockDim.x) {
    const int s = idx / Dims<NB>::NS;
    sm.totals[idx] = expand_slot<NB, NV>(sm, s, idx - s * Dims<NB>::NS);
  }
  __syncthreads();
  for (int s = tid; s < K; s += blockDim.x) {
    const double* T = sm.totals + s * Dims<NB>::NS;
    const double lw = log_w[s];
    const double w_s = nb_exp(lw);
    sm.llv[s] = T[kLinear] + lw * __ldg(tot + s) - gamma * T[kSumLog] - T[kWlog];
    out.w[s] = w_s;
    out.dw[s] = T[kResid] + (alpha - lambda * w_s);
    out.vw[s] = gamma * T[kWeight] + lambda * w_s;
#pragma unroll
    for (int a = 0; a < NB; ++a) out.vwb[s * NB + a] = gamma * T[Dims<NB>::kFirst + a];
  }
  __syncthreads();
  // sums over subjects in subject order, as the CPU path adds them
  if (tid < NB) {
    double acc = 0.0;
    for (int s = 0; s < K; ++s) acc += sm.totals[s * Dims<NB>::NS + kScore + tid];
    out.db[tid] = acc;
  } else if (tid < NB + Dims<NB>::T) {
    const int t = tid - NB;
    int a = 0, rem = t;
    while (rem >= NB - a) {
      rem -= NB - a;
      ++a;
    }
    const int b = a + rem;
    double acc = 0.0;
    for (int s = 0; s < K; ++s) acc += gamma * sm.totals[s * Dims<NB>::NS + Dims<NB>::kSecond + t];
    out.vb[a * NB + b] = acc;
    out.vb[b * NB + a] = acc;
  } else if (tid == 64) {
    double ll = 0.0, sl = 0.0, sw = 0.0;
    for (int s = 0; s < K; ++s) ll += sm.llv[s];
    for (int s = 0; s < K; ++s) sl += log_w[s];
    for (int s = 0; s < K; ++s) sw += out.w[s];
    *out.ll = ll + (alpha * sl - lambda * sw);
  }
  if (tid == 0) sm.sc[kSweeps] += 1.0;
  __syncthreads();
}

// Pivoted LDL' solve, Eigen's LDLT as nebula calls it (pml.rs:1940-2021).
template <int NB>
__device__ void ldlt_solve(double* a, double* b) {
  int perm[NB];
  double tmp[NB];
  for (int step = 0; step < NB; ++step) {
    int pivot = step;
    double best = fabs(a[step * NB + step]);
    for (int i = step + 1; i < NB; ++i) {
      double v = fabs(a[i * NB + i]);
      if (v > best) {
        best = v;
        pivot = i;
      }
    }
    perm[step] = pivot;
    if (pivot != step) {
      for (int j = 0; j < step; ++j) {
        double t = a[step * NB + j];
        a[step * NB + j] = a[pivot * NB + j];
        a[pivot * NB + j] = t;
      }
      for (int i = pivot + 1; i < NB; ++i) {
        double t = a[i * NB + step];
        a[i * NB + step] = a[i * NB + pivot];
        a[i * NB + pivot] = t;
      }
      double t = a[step * NB + step];
      a[step * NB + step] = a[pivot * NB + pivot];
      a[pivot * NB + pivot] = t;
      for (int i = step + 1; i < pivot; ++i) {
        double u = a[i * NB + step];
        a[i * NB + step] = a[pivot * NB + i];
        a[pivot * NB + i] = u;
      }
    }
    if (step > 0) {
      for (int j = 0; j < step; ++j) tmp[j] = a[j * NB + j] * a[step * NB + j];
      double acc = 0.0;
      for (int j = 0; j < step; ++j) acc += a[step * NB + j] * tmp[j];
      a[step * NB + step] -= acc;
      for (int i = step + 1; i < NB; ++i) {
        double acc2 = 0.0;
        for (int j = 0; j < step; ++j) acc2 += a[i * NB + j] * tmp[j];
        a[i * NB + step] -= acc2;
      }
    }
    double dd = a[step * NB + step];
    if (dd != 0.0)
      for (int i = step + 1; i < NB; ++i) a[i * NB + step] /= dd;
  }
  for (int step = 0; step < NB; ++step) {
    double t = b[step];
    b[step] = b[perm[step]];
    b[perm[step]] = t;
  }
  for (int i = 0; i < NB; ++i) {
    double acc = b[i];
    for (int j = 0; j < i; ++j) acc -= a[i * NB + j] * b[j];
    b[i] = acc;
  }
  for (int i = 0; i < NB; ++i) {
    double dd = a[i * NB + i];
    b[i] = fabs(dd) > DBL_MIN ? b[i] / dd : 0.0;
  }
  for (int i = NB - 1; i >= 0; --i) {
    double acc = b[i];
    for (int j = i + 1; j < NB; ++j) acc -= a[j * NB + i] * b[j];
    b[i] = acc;
  }
  for (int step = NB - 1; step >= 0; --step) {
    double t = b[step];
    b[step] = b[perm[step]];
    b[perm[step]] = t;
  }
}

// Determinant by partial-pivot LU, a product as the C++ takes it (pml.rs:2036-2069).
template <int NB>
__device__ double determinant(double* a) {
  double det = 1.0;
  for (int step = 0; step < NB; ++step) {
    int pivot = step;
    double best = fabs(a[step * NB + step]);
    for (int i = step + 1; i < NB; ++i) {
      double v = fabs(a[i * NB + step]);
      if (v > best) {
        best = v;
        pivot = i;
      }
    }
    if (pivot != step) {
      for (int j = 0; j < NB; ++j) {
        double t = a[step * NB + j];
        a[step * NB + j] = a[pivot * NB + j];
        a[pivot * NB + j] = t;
      }
      det = -det;
    }
    double dd = a[step * NB + step];
    det *= dd;
    if (dd == 0.0) return 0.0;
    for (int i = step + 1; i < NB; ++i) {
      double f = a[i * NB + step] / dd;
      a[i * NB + step] = f;
      for (int j = step + 1; j < NB; ++j) a[i * NB + j] -= f * a[step * NB + j];
    }
  }
  return det;
}

__device__ __forceinline__ long long global_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// One inner fit (optimise, pml.rs:1614-1800) by the calling cluster: every
// CTA of the cluster runs it in step (each sweep shared over the cluster's
// CTAs) and rank 0 writes the result to `out`.
template <int NB, int NV>
__device__ void fit_one(const GeneData& d, const FitControl& ctl, Smem<NB, NV>& sm, const FitRequest& req,
                        FitResult* out, const Cluster& cl, int& parity, long long t_start) {
  const int K = sm.K;
  const int tid = threadIdx.x;
  const int gene = req.gene;
  const long long ns_start = global_ns();

  // gamma_penalty (pml.rs:432-441) and the argument checks of optimise
  const double exps = nb_exp(req.subject);
  const bool bad = !(isfinite(exps) && exps > 1.0) || !(isfinite(req.cell) && req.cell > 0.0);
  if (bad) {
    if (tid == 0 && cl.rank == 0) {
      out->status = 1;
      out->iterations = 0;
      out->sweeps = 0;
      out->cycles = 0;
      out->start_ns = ns_start;
      out->end_ns = global_ns();
    }
    return;
  }
  if (tid == 0) {
    sm.sc[kAlpha] = 1.0 / (exps - 1.0);
    sm.sc[kLambda] = 1.0 / (sqrt(exps) * (exps - 1.0));
    sm.sc[kGamma] = req.cell;
    sm.sc[kSweeps] = 0.0;
  }
  // warm inner start: the gene's stored iterate (read past L1; another
  // cluster wrote it in an earlier step of the gene's search)
  const size_t warm_stride = static_cast<size_t>(NB + K);
  const bool warm_read = d.warm_state && (req.flags & kWarmRead);
  const double* warm_src =
      warm_read ? d.warm_state + (static_cast<size_t>(gene) * 2 + ((req.flags & kWarmBuffer) ? 0 : 1)) * warm_stride
                : nullptr;
  if (tid < NB) sm.beta[tid] = warm_read ? __ldcg(warm_src + tid) : req.beta[tid];
  for (int s = tid; s < K; s += blockDim.x) sm.log_w[s] = warm_read ? __ldcg(warm_src + NB + s) : 0.0;
  for (int i = tid; i <= kRanges; i += blockDim.x)
    sm.rpos[i] = d.range_pos[static_cast<size_t>(gene) * (kRanges + 1) + i];
  for (int i = tid; i <= K; i += blockDim.x) sm.runs[i] = d.runs[static_cast<size_t>(gene) * (K + 1) + i];
  __syncthreads();

  int cur = 0;  // index of the current sweep buffer (every thread tracks it identically)
  sweep<NB, NV>(d, sm, gene, sm.beta, sm.log_w, SweepView<NB>(sm.sw[cur], K), parity, cl);
  if (tid == 0) {
    sm.sc[kLl] = *SweepView<NB>(sm.sw[cur], K).ll;
    sm.sc[kLlPrev] = 0.0;
    sm.sc[kLikdif] = 0.0;
    sm.sc[kStep] = 0.0;
    sm.sc[kBacktracks] = 0.0;
  }
  __syncthreads();

  for (;;) {
    const double step = sm.sc[kStep];
    // A warm-started fit takes at least two Newton steps: the log-determinant
    // comes from the previous iterate's vw (pml.rs:1767-1777), which after a
    // single step would still be the stored start.
    const double min_steps = warm_read ? 2.0 : 1.0;
    const bool go = step < min_steps || (sm.sc[kLikdif] > ctl.eps && step < static_cast<double>(ctl.max_iter));
    __syncthreads();
    if (!go) break;
    SweepView<NB> c(sm.sw[cur], K);
    SweepView<NB> tr(sm.sw[cur ^ 1], K);
    if (tid == 0) sm.sc[kStep] = step + 1.0;
    // Schur complement of the random-effect block and the step (pml.rs:1660-1710)
    for (int s = tid; s < K; s += blockDim.x) {
      sm.vw_step[s] = c.vw[s];
      sm.dwvw[s] = c.dw[s] / c.vw[s];
      sm.damp_log_w[s] = 1.0;
    }
    if (tid < NB) sm.damp_beta[tid] = 1.0;
    __syncthreads();
    if (tid < Dims<NB>::T) {
      int a = 0, rem = tid;
      while (rem >= NB - a) {
        rem -= NB - a;
        ++a;
      }
      const int b = a + rem;
      double acc = 0.0;
      for (int s = 0; s < K; ++s) acc += c.vwb[s * NB + a] * c.vwb[s * NB + b] / c.vw[s];
      const double v = c.vb[a * NB + b] - acc;
      sm.vb2[a * NB + b] = v;
      sm.vb2[b * NB + a] = v;
      sm.factor[a * NB + b] = v;
      sm.factor[b * NB + a] = v;
    } else if (tid >= 64 && tid < 64 + NB) {
      const int j = tid - 64;
      double acc = 0.0;
      for (int s = 0; s < K; ++s) acc += c.vwb[s * NB + j] * sm.dwvw[s];
      sm.step_beta[j] = c.db[j] - acc;
    }
    __syncthreads();
    if (tid == 0) ldlt_solve<NB>(sm.factor, sm.step_beta);
    __syncthreads();
    for (int s = tid; s < K; s += blockDim.x) {
      double acc = 0.0;
#pragma unroll
      for (int j = 0; j < NB; ++j) acc += c.vwb[s * NB + j] * sm.step_beta[j];
      sm.step_log_w[s] = sm.dwvw[s] - acc / c.vw[s];
      sm.new_log_w[s] = sm.log_w[s] + sm.step_log_w[s];
    }
    if (tid < NB) sm.new_beta[tid] = sm.beta[tid] + sm.step_beta[tid];
    if (tid == 0) sm.sc[kLlPrev] = sm.sc[kLl];
    __syncthreads();
    sweep<NB, NV>(d, sm, gene, sm.new_beta, sm.new_log_w, tr, parity, cl);
    if (tid == 0) {
      sm.sc[kLl] = *tr.ll;
      sm.sc[kLikdif] = sm.sc[kLl] - sm.sc[kLlPrev];
      sm.sc[kBacktracks] = 0.0;
      sm.sc[kMinStep] = kStepCutoff;
      sm.sc[kStop] = 0.0;
    }
    __syncthreads();
    // backtracking (pml.rs:1716-1760)
    for (;;) {
      const double ll = sm.sc[kLl];
      const bool again = sm.sc[kLikdif] < 0.0 || isinf(ll);
      __syncthreads();
      if (!again) break;
      if (tid == 0) {
        const double bt = sm.sc[kBacktracks] + 1.0;
        sm.sc[kBacktracks] = bt;
        sm.sc[kMinStep] = sm.sc[kMinStep] / 2.0;
        if (bt > static_cast<double>(ctl.max_backtrack)) {
          sm.sc[kLikdif] = 0.0;
          sm.sc[kLl] = sm.sc[kLlPrev];
          double gb = 0.0, gw = 0.0;
          for (int j = 0; j < NB; ++j) gb = fmax(gb, fabs(c.db[j]));
          for (int s = 0; s < K; ++s) gw = fmax(gw, fabs(c.dw[s]));
          if (gb > kGradientTolerance || gw > kGradientTolerance) sm.sc[kBacktracks] = bt + 1.0;
          sm.sc[kStop] = 1.0;
        }
      }
      __syncthreads();
      if (sm.sc[kStop] != 0.0) break;
      const double min_step = sm.sc[kMinStep];
      if (tid < NB) {
        const double dd = sm.step_beta[tid];
        if (dd < kStepCutoff && dd > -kStepCutoff) {
          sm.damp_beta[tid] /= 2.0;
          sm.new_beta[tid] = sm.beta[tid] + dd * sm.damp_beta[tid];
        } else if (dd > 0.0) {
          sm.new_beta[tid] = sm.beta[tid] + min_step;
        } else {
          sm.new_beta[tid] = sm.beta[tid] - min_step;
        }
      }
      for (int s = tid; s < K; s += blockDim.x) {
        const double dd = sm.step_log_w[s];
        if (dd < kStepCutoff && dd > -kStepCutoff) {
          sm.damp_log_w[s] /= 2.0;
          sm.new_log_w[s] = sm.log_w[s] + dd * sm.damp_log_w[s];
        } else if (dd > 0.0) {
          sm.new_log_w[s] = sm.log_w[s] + min_step;
        } else {
          sm.new_log_w[s] = sm.log_w[s] - min_step;
        }
      }
      __syncthreads();
      sweep<NB, NV>(d, sm, gene, sm.new_beta, sm.new_log_w, tr, parity, cl);
      if (tid == 0) {
        sm.sc[kLl] = *tr.ll;
        sm.sc[kLikdif] = sm.sc[kLl] - sm.sc[kLlPrev];
      }
      __syncthreads();
    }
    // accept the trial point as the new iterate
    if (tid < NB) sm.beta[tid] = sm.new_beta[tid];
    for (int s = tid; s < K; s += blockDim.x) sm.log_w[s] = sm.new_log_w[s];
    cur ^= 1;
    __syncthreads();
  }

  // log-determinant from the previous iterate's vw (pml.rs:1767-1777)
  if (tid == 0) {
    double log_det = 0.0;
    for (int s = 0; s < K; ++s) log_det += nb_log(fabs(sm.vw_step[s]));
    if (req.reml) {
      for (int i = 0; i < NB * NB; ++i) sm.factor[i] = sm.vb2[i];
      log_det += nb_log(fabs(determinant<NB>(sm.factor)));
    }
    sm.sc[kLogDet] = log_det;
    sm.sc[kSecond] = 0.0;
  }
  __syncthreads();
  // higher-order Laplace correction at the final iterate (pml.rs:1828-1919)
  if (req.ord > 1) {
    SweepView<NB> c(sm.sw[cur], K);
    sweep_sums<NB, NV, 1>(d, sm, sm.beta, sm.log_w, sm.sc[kGamma], parity, cl);
    parity ^= 1;
    if (tid == 0) {
      const double gamma = sm.sc[kGamma], lambda = sm.sc[kLambda];
      const bool high = req.ord > 2;
      double third_acc = 0.0, fourth_acc = 0.0, fifth_acc = 0.0;
      for (int s = 0; s < K; ++s) {
        const double* S = sm.rtot + s * Smem<NB, NV>::NP;
        const double prior = lambda * c.w[s];
        const double vw = gamma * S[0] + prior;
        const double third = gamma * S[1] + prior;
        third_acc += third * third / (vw * vw * vw);
        if (high) {
          const double fourth = gamma * S[2] + prior;
          const double fifth = gamma * S[3] + prior;
          const double vs = vw * vw;
          fourth_acc += fourth / vs;
          fifth_acc += fifth * third / (vs * vs);
        }
      }
      double second = 5.0 * third_acc / 24.0;
      if (high) {
        second -= fourth_acc / 8.0;
        second += 7.0 * fifth_acc / 48.0;
      }
      sm.sc[kSecond] = second;
      sm.sc[kSweeps] += 1.0;
    }
    __syncthreads();
  }
  if (cl.rank != 0) return;  // rank 0 of the cluster writes the result
  if (d.warm_state && (req.flags & kWarmWrite)) {
    double* dst = d.warm_state + (static_cast<size_t>(gene) * 2 + ((req.flags & kWarmBuffer) ? 1 : 0)) * warm_stride;
    if (tid < NB) __stcg(dst + tid, sm.beta[tid]);
    for (int s = tid; s < K; s += blockDim.x) __stcg(dst + NB + s, sm.log_w[s]);
  }
  if (tid < NB) out->beta[tid] = sm.beta[tid];
  for (int i = tid; i < NB * NB; i += blockDim.x) out->information[i] = sm.vb2[i];
  if (tid == 0) {
    out->log_likelihood = sm.sc[kLl];
    out->log_likelihood_prev = sm.sc[kLlPrev];
    out->log_det = sm.sc[kLogDet];
    out->second_order = sm.sc[kSecond];
    out->iterations = static_cast<int32_t>(sm.sc[kStep]);
    out->backtracks = static_cast<int32_t>(sm.sc[kBacktracks]);
    out->sweeps = static_cast<int32_t>(sm.sc[kSweeps]);
    out->status = 0;
    out->cycles = (clock64() - t_start) * cl.size;  // every CTA of the cluster was busy
    out->start_ns = ns_start;
    out->end_ns = global_ns();
  }
}

// Per-CTA set-up shared by both kernels: tables, subject boundaries, the
// cell ranges and the ranges meeting each subject, the cluster coordinates.
template <int NB, int NV>
__device__ Cluster setup_cta(const GeneData& d, Smem<NB, NV>& sm) {
  const int K = sm.K;
  const int tid = threadIdx.x;
  nb_load_tables(sm.tab);
  for (int i = tid; i <= K; i += blockDim.x) sm.fid[i] = d.fid[i];
  for (int i = tid; i <= kRanges; i += blockDim.x) sm.rcells[i] = d.range_cells[i];
  __syncthreads();
  // the ranges that meet each subject: vlo = first with end > fid[s],
  // vhi = last with start < fid[s + 1]
  for (int s = tid; s < K; s += blockDim.x) {
    int lo = 0;
    while (lo < kRanges - 1 && sm.rcells[lo + 1] <= sm.fid[s]) ++lo;
    int hi = kRanges - 1;
    while (hi > 0 && sm.rcells[hi] >= sm.fid[s + 1]) --hi;
    sm.vlo[s] = lo;
    sm.vhi[s] = hi;
  }
  // each subject's design row (the constant columns' values) and each
  // column's place among the varying ones
  for (int i = tid; i < K * NB; i += blockDim.x) {
    const int s = i / NB;
    sm.xs[i] = sm.fid[s] < sm.fid[s + 1] ? d.design[static_cast<size_t>(sm.fid[s]) * NB + (i - s * NB)] : 0.0;
  }
  if (tid < NB) {
    int pos = -1;
    for (int j = 0; j < NV; ++j)
      if (d.varying[j] == tid) pos = j;
    sm.vpos[tid] = pos;
  }
  Cluster cl;
  cg::cluster_group cluster = cg::this_cluster();
  cl.rank = static_cast<int>(cluster.block_rank());
  cl.size = static_cast<int>(cluster.num_blocks());
  return cl;
}

// CTAs per SM the fit kernels are compiled for. With at most one varying
// column (4 columns or fewer) the per-cell state is small enough for 80
// registers, and three CTAs per SM hide more of the FP64 latency than the
// spills cost (measured: 3220 against 2996 plain genes/s on 500 genes x
// 100,000 cells, 4 columns of which 1 varies).
constexpr int min_blocks(int nb, int nv) { return nb <= 4 && nv <= 1 ? 3 : (nb <= 4 ? 2 : 1); }

// Batch mode: *n_requests requests in device memory, taken off an atomic
// counter one per cluster.
template <int NB, int NV>
__global__ void __launch_bounds__(kThreads, min_blocks(NB, NV)) fit_kernel(GeneData d, FitControl ctl,
                                                       const FitRequest* __restrict__ requests,
                                                       FitResult* __restrict__ results,
                                                       const int32_t* __restrict__ n_requests,
                                                       int32_t* __restrict__ counter) {
  extern __shared__ __align__(16) double smem_raw[];
  Smem<NB, NV> sm;
  sm.carve(smem_raw, d.n_subjects);
  const Cluster cl = setup_cta<NB, NV>(d, sm);
  const int tid = threadIdx.x;
  __shared__ int next_req;
  const int total = *n_requests;
  int parity = 0;  // sweep parity of the pieces buffers, identical in every thread of the cluster

  for (;;) {
    // one request per cluster: rank 0 takes it off the queue and hands it to
    // every CTA; the first barrier keeps it from overwriting a value a CTA
    // has not read yet
    cluster_barrier(cl);
    if (cl.rank == 0 && tid == 0) {
      const int taken = atomicAdd(counter, 1);
      if (cl.size == 1) {
        next_req = taken;
      } else {
        cg::cluster_group cluster = cg::this_cluster();
        for (int r = 0; r < cl.size; ++r) *cluster.map_shared_rank(&next_req, r) = taken;
      }
    }
    cluster_barrier(cl);
    const int q = next_req;
    if (q >= total) break;
    const FitRequest req = requests[q];
    fit_one<NB, NV>(d, ctl, sm, req, results + q, cl, parity, clock64());
  }
}

// Streaming mode (FitQueue): one persistent launch for a whole stage.
template <int NB, int NV>
__global__ void __launch_bounds__(kThreads, min_blocks(NB, NV)) fit_queue_kernel(GeneData d, FitControl ctl,
                                                             FitQueue qu) {
  extern __shared__ __align__(16) double smem_raw[];
  Smem<NB, NV> sm;
  sm.carve(smem_raw, d.n_subjects);
  const Cluster cl = setup_cta<NB, NV>(d, sm);
  const int tid = threadIdx.x;
  __shared__ long long next_ticket;  // the ticket to run, or -1 to exit
  __shared__ FitRequest next_req;    // its request
  int parity = 0;
  long long wait_ns = 0;             // rank 0's thread 0: the last ticket's wait

  for (;;) {
    // rank 0's first warp takes a ticket, waits for its request and hands
    // ticket and request to every CTA of the cluster; the first barrier keeps
    // it from overwriting what a CTA has not read yet
    cluster_barrier(cl);
    if (cl.rank == 0 && tid < 32) {
      long long waited = 0;
      const long long got = ring_next(qu.ring, &next_req, &waited);
      if (tid == 0) {
        wait_ns = waited;
        next_ticket = got;
      }
      if (cl.size > 1) {
        cg::cluster_group cluster = cg::this_cluster();
        constexpr int kWords = static_cast<int>(sizeof(FitRequest) / 8);
        const unsigned long long* mine = reinterpret_cast<const unsigned long long*>(&next_req);
        for (int r = 1; r < cl.size; ++r) {
          if (tid == 0) *cluster.map_shared_rank(&next_ticket, r) = got;
          if (tid < kWords && got >= 0)
            cluster.map_shared_rank(reinterpret_cast<unsigned long long*>(&next_req), r)[tid] = mine[tid];
        }
      }
    }
    cluster_barrier(cl);
    const long long t = next_ticket;
    if (t < 0) break;
    const FitRequest req = next_req;
    fit_one<NB, NV>(d, ctl, sm, req, qu.results + (t & qu.ring.mask), cl, parity, clock64());
    if (cl.rank == 0) {  // rank 0 wrote the result
      if (tid == 0) qu.results[t & qu.ring.mask].wait_ns = wait_ns;
      ring_publish(qu.done + (t & qu.ring.mask), t);
    }
  }
}

template <int NB, int NV>
size_t smem_for(int K) {
  return Smem<NB, NV>::bytes(K);
}

// Opts the kernel into the dynamic shared memory one CTA needs; the
// attribute may not exceed the per-block opt-in limit less the kernel's
// static shared memory. The attribute only grows: the largest size set so
// far, per device.
inline cudaError_t configure_kernel(const void* kernel, size_t smem, std::atomic<int>* configured) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const bool cached = dev >= 0 && dev < 64;
  if (cached && configured[dev].load() >= static_cast<int>(smem)) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e == cudaSuccess && cached) {
    int seen = configured[dev].load();
    while (seen < static_cast<int>(smem) && !configured[dev].compare_exchange_weak(seen, static_cast<int>(smem))) {
    }
  }
  return e;
}

template <int NB, int NV>
cudaError_t configure_queue_nb(size_t smem) {
  static std::atomic<int> configured[64];
  return configure_kernel(reinterpret_cast<const void*>(fit_queue_kernel<NB, NV>), smem, configured);
}

template <int NB, int NV>
cudaError_t configure_nb(size_t smem) {
  static std::atomic<int> configured[64];
  return configure_kernel(reinterpret_cast<const void*>(fit_kernel<NB, NV>), smem, configured);
}

inline cudaLaunchConfig_t cluster_config(int grid, size_t smem, cudaStream_t stream, cudaLaunchAttribute* attr,
                                         int cluster) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid, 1, 1);
  cfg.blockDim = dim3(kThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

template <int NB, int NV>
int launch_nb(const GeneData& d, const FitControl& ctl, const FitRequest* req, FitResult* res,
              const int32_t* n_req, int32_t* counter, int grid, int cluster, cudaStream_t stream) {
  const size_t smem = Smem<NB, NV>::bytes(d.n_subjects);
  cudaError_t e = configure_nb<NB, NV>(smem);
  if (e != cudaSuccess) return e;
  if (cluster <= 1) {
    fit_kernel<NB, NV><<<grid, kThreads, smem, stream>>>(d, ctl, req, res, n_req, counter);
    return cudaGetLastError();
  }
  if (cluster > kMaxCluster || (cluster & (cluster - 1)) != 0 || grid % cluster != 0) return cudaErrorInvalidValue;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = cluster_config(grid, smem, stream, attr, cluster);
  return cudaLaunchKernelEx(&cfg, fit_kernel<NB, NV>, d, ctl, req, res, n_req, counter);
}

template <int NB, int NV>
int launch_queue_nb(const GeneData& d, const FitControl& ctl, const FitQueue& qu, int grid, int cluster,
                    cudaStream_t stream) {
  const size_t smem = Smem<NB, NV>::bytes(d.n_subjects);
  cudaError_t e = configure_queue_nb<NB, NV>(smem);
  if (e != cudaSuccess) return e;
  if (cluster < 1 || cluster > kMaxCluster || (cluster & (cluster - 1)) != 0 || grid % cluster != 0)
    return cudaErrorInvalidValue;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = cluster_config(grid, smem, stream, attr, cluster);
  return cudaLaunchKernelEx(&cfg, fit_queue_kernel<NB, NV>, d, ctl, qu);
}

template <int NB, int NV>
int blocks_nb(int K) {
  int blocks = 0;
  const size_t smem = Smem<NB, NV>::bytes(K);
  if (configure_nb<NB, NV>(smem) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fit_kernel<NB, NV>, kThreads, smem) != cudaSuccess)
    return 0;
  return blocks;
}

template <int NB, int NV>
int clusters_nb(int K, int cluster) {
  const size_t smem = Smem<NB, NV>::bytes(K);
  if (configure_nb<NB, NV>(smem) != cudaSuccess) return 0;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = cluster_config(cluster, smem, nullptr, attr, cluster);
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, fit_kernel<NB, NV>, &cfg) != cudaSuccess) return 0;
  return n;
}

template <int NB, int NV>
int queue_clusters_nb(int K, int cluster) {
  const size_t smem = Smem<NB, NV>::bytes(K);
  if (configure_queue_nb<NB, NV>(smem) != cudaSuccess) return 0;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = cluster_config(cluster, smem, nullptr, attr, cluster);
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, fit_queue_kernel<NB, NV>, &cfg) != cudaSuccess) return 0;
  return n;
}

template <int NB, int NV>
FitOps make_ops() {
  return FitOps{&smem_for<NB, NV>, &launch_nb<NB, NV>, &launch_queue_nb<NB, NV>,
                &blocks_nb<NB, NV>, &clusters_nb<NB, NV>, &queue_clusters_nb<NB, NV>};
}

// The instantiations for NB columns, by how many of them vary within subjects.
template <int NB, int NV = 0>
FitOps ops_for(int n_varying) {
  if constexpr (NV > NB) {
    return FitOps{};
  } else {
    if (n_varying == NV) return make_ops<NB, NV>();
    return ops_for<NB, NV + 1>(n_varying);
  }
}

}  // namespace
}  // namespace device
}  // namespace nebula
