// ORACLE — test infrastructure only. Stage one's per-subject cell sums on the
// CPU (the reference's ptmg.rs linear_predictor 661-708 and the cell loops of
// evaluate 926-966 / hessian_subject 1381-1428), in the summation tree and
// with the exp/log and fused multiply-adds the device kernel ptmg_eval.cu
// uses, so the two agree bit for bit; plus stage one driven by the CPU.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "nbmath.hpp"
#include "pml_cpu.hpp"
#include "ptmg_cpu.hpp"
#include "stage_one.hpp"
#include "tree_cpu.hpp"

namespace oracle {
namespace {

using nebula::nb_fma;

// the table-driven exp and log the kernel calls (its shared-memory copy of
// the same tables)
double cell_exp(double x) { return nebula::nb_exp_tab(x, &nebula::kNbTables); }
double cell_log(double x) { return nebula::nb_log_tab(x, &nebula::kNbTables); }


}  // namespace

nebula::PtmgSums ptmg_sums(const PmlData& d, const double* beta, double alpha, double lambda, double gamma) {
  const int nb = d.n_beta, k = d.k, T = nb * (nb + 1) / 2, W = nebula::ptmg_width(nb);
  const int kXf = 9, kD41 = kXf + nb, kT1 = kD41 + nb, kT2 = kT1 + nb, kBp = kT2 + nb, kBq = kBp + T;
  // the per-cell sums run over the varying columns (ptmg_impl.cuh): the
  // reduced row holds the nine scalars, sum e, sum e q, the vectors Xf, D41,
  // T1, T2, Eq over the varying columns and the triangles Bp, Bq
  const Split sp = split_columns(d);
  const int nv = static_cast<int>(sp.varying.size()), tv = nv * (nv + 1) / 2;
  const int rE = 9, rEq = 10, rXf = 11, rD41 = rXf + nv, rT1 = rD41 + nv, rT2 = rT1 + nv, rQv = rT2 + nv;
  const int rBp = rQv + nv, rBq = rBp + tv, RW = rBq + tv;
  const int warps = stage_one_warps(nb, nv);  // the kernel's warp ranges
  std::vector<double> cs(k), bv(nv);
  for (int j = 0; j < nv; ++j) bv[j] = beta[sp.varying[j]];
  for (int s = 0; s < k; ++s) {  // the constant columns' share of eta, in column order
    const std::vector<double> row = subject_row(d, s);
    double c = 0.0;
    for (int a = 0; a < nb; ++a)
      if (sp.vpos[a] < 0) c = nb_fma(row[a], beta[a], c);
    cs[s] = c;
  }
  auto eta_at = [&](size_t r, int s, double* x) {
    varying_row(d, sp, r, x);
    double eta = d.offset[r] + cs[s];
    for (int j = 0; j < nv; ++j) eta = nb_fma(x[j], bv[j], eta);
    return eta;
  };
  nebula::PtmgSums out;
  // pass one: sum e over every cell, sum y eta over the positive ones
  auto dense1 = [&](double* acc, size_t r, int s) {
    double x[kMaxRow];
    acc[0] += cell_exp(eta_at(r, s, x));
  };
  auto sparse1 = [&](double* acc, size_t i, int s) {
    double x[kMaxRow];
    acc[1] = nb_fma(eta_at(d.cells[i], s, x), d.counts[i], acc[1]);
  };
  std::vector<double> p1 = tree_sums(d, 2, warps, dense1, sparse1);
  out.cumsumxtb.resize(k);
  out.ylin.resize(k);
  std::vector<double> ym(k);
  for (int s = 0; s < k; ++s) {
    out.cumsumxtb[s] = p1[2 * s];
    out.ylin[s] = p1[2 * s + 1];
    ym[s] = (d.subject_total[s] + alpha) / (p1[2 * s] + lambda);
  }
  // pass two
  auto dense2 = [&](double* acc, size_t r, int s) {
    double x[kMaxRow];
    const double e = cell_exp(eta_at(r, s, x));
    const double yms = ym[s];
    const double we = yms * e;
    const double w = we + gamma;
    const double lw = cell_log(w);
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
    const double q = yms * (yms * gte - gg);
    acc[rE] += e;
    acc[rEq] = nb_fma(e, q, acc[rEq]);
    int t = 0;
    for (int a = 0; a < nv; ++a) {
      const double xe = x[a] * e;
      acc[rXf + a] += xe;
      acc[rD41 + a] = nb_fma(gg, xe, acc[rD41 + a]);
      acc[rT1 + a] = nb_fma(xe, f1, acc[rT1 + a]);
      acc[rT2 + a] = nb_fma(xe, gte, acc[rT2 + a]);
      acc[rQv + a] = nb_fma(xe, q, acc[rQv + a]);
      for (int b = a; b < nv; ++b) {
        const double c = xe * x[b];
        acc[rBp + t] += c;
        acc[rBq + t] = nb_fma(c, q, acc[rBq + t]);
        ++t;
      }
    }
  };
  auto sparse2 = [&](double* acc, size_t i, int s) {
    double x[kMaxRow];
    const double y = d.counts[i];
    const double e = cell_exp(eta_at(d.cells[i], s, x));
    const double yms = ym[s];
    const double w = yms * e + gamma;
    const double lw = cell_log(w);
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
    const double q = yms * (yms * gte - gg);
    acc[rEq] = nb_fma(e, q, acc[rEq]);
    int t = 0;
    for (int a = 0; a < nv; ++a) {
      const double xe = x[a] * e;
      acc[rD41 + a] = nb_fma(gg, xe, acc[rD41 + a]);
      acc[rT1 + a] = nb_fma(xe, gt, acc[rT1 + a]);
      acc[rT2 + a] = nb_fma(xe, gte, acc[rT2 + a]);
      acc[rQv + a] = nb_fma(xe, q, acc[rQv + a]);
      for (int b = a; b < nv; ++b) {
        const double cc = xe * x[b];
        acc[rBq + t] = nb_fma(cc, q, acc[rBq + t]);
        ++t;
      }
    }
  };
  const std::vector<double> red = tree_sums(d, RW, warps, dense2, sparse2);
  // every subject's full row: a constant column's sums are its value times a
  // scalar sum (sum x_a e = x_a sum e, sum x_a gg e = x_a acc[6], ...)
  out.sums.assign(static_cast<size_t>(k) * W, 0.0);
  for (int s = 0; s < k; ++s) {
    const double* R = &red[static_cast<size_t>(s) * RW];
    const std::vector<double> X = subject_row(d, s);
    double* F = &out.sums[static_cast<size_t>(s) * W];
    for (int x = 0; x < kXf; ++x) F[x] = R[x];
    const int from[4] = {rXf, rD41, rT1, rT2}, scalar[4] = {rE, 6, 7, 8}, block[4] = {kXf, kD41, kT1, kT2};
    for (int part = 0; part < 4; ++part)
      for (int a = 0; a < nb; ++a) {
        const int va = sp.vpos[a];
        F[block[part] + a] = va >= 0 ? R[from[part] + va] : X[a] * R[scalar[part]];
      }
    for (int qpart = 0; qpart < 2; ++qpart) {
      const int base = qpart ? rBq : rBp, vec = qpart ? rQv : rXf, sc = qpart ? rEq : rE;
      int t = 0;
      for (int a = 0; a < nb; ++a)
        for (int b = a; b < nb; ++b, ++t) {
          const int va = sp.vpos[a], vb = sp.vpos[b];
          double v;
          if (va >= 0 && vb >= 0) v = R[base + va * nv - va * (va - 1) / 2 + (vb - va)];
          else if (vb >= 0) v = X[a] * R[vec + vb];
          else if (va >= 0) v = X[b] * R[vec + va];
          else v = X[a] * (X[b] * R[sc]);
          F[(qpart ? kBq : kBp) + t] = v;
        }
    }
  }
  return out;
}

nebula::GenePlan plan_gene(const nebula::Shared& sh, const nebula::GeneCounts& gc, const double* totals,
                           int* evaluations, bool tabled) {
  PmlData d{sh.design.data(), sh.log_offset.data(), sh.n_cells, sh.n_coef, gc.counts.data(), gc.cells.data(),
            gc.counts.size(), sh.fid.data(), sh.n_subjects, totals};
  const std::vector<double> xy = nebula::positive_xy(sh, gc);
  nebula::MarginalGene mg{&sh, &gc, totals, xy.data()};
  std::vector<double> start, lower, upper;
  nebula::marginal_box(sh, gc, &start, &lower, &upper);
  nebula::MarginalSearch search(start, lower, upper, sh.n_coef, tabled);
  const int np = sh.n_coef + 2;
  std::vector<double> g(np), h(static_cast<size_t>(np) * np);
  while (const double* x = search.ask()) {
    nebula::Terms t(x[sh.n_coef], x[sh.n_coef + 1]);
    nebula::PtmgSums sums = ptmg_sums(d, x, t.alpha, t.lambda, t.gamma);
    double f = nebula::ptmg_assemble(mg, x, sums, g.data(), h.data());
    search.tell(f, g.data(), h.data());
  }
  if (evaluations) *evaluations = search.evaluations();
  return nebula::plan_from(sh, gc, search.best(), search.failed());
}

}  // namespace oracle

#define ORACLE_API extern "C" __attribute__((visibility("default")))

// Value, gradient and Hessian of the marginal negative log-likelihood at
// params = [beta, sigma, phi] (nebula:::ptmg_ll_der_hes, ptmg.rs:615).
ORACLE_API double oracle_ptmg_eval(const double* design, const double* log_offset, uint64_t n_cells,
                                   uint32_t n_coef, const double* counts, const uint32_t* cells, uint64_t n_pos,
                                   const uint64_t* fid, uint32_t k, const double* totals, const double* params,
                                   double* grad, double* hess) {
  nebula::Shared sh;
  sh.design.assign(design, design + n_cells * n_coef);
  sh.log_offset.assign(log_offset, log_offset + n_cells);
  sh.fid.assign(fid, fid + k + 1);
  sh.n_cells = n_cells;
  sh.n_coef = static_cast<int>(n_coef);
  sh.n_subjects = static_cast<int>(k);
  nebula::GeneCounts gc;
  gc.own(cells, counts, n_pos);
  for (double y : gc.counts) {  // the tallies positive_indices keeps (ptmg.rs:1708-1719)
    if (y == 1.0) {
      ++gc.n_one;
    } else if (y == 2.0) {
      ++gc.n_two;
    } else {
      size_t i = 0;
      while (i < gc.big_values.size() && gc.big_values[i] < y) ++i;
      if (i < gc.big_values.size() && gc.big_values[i] == y) {
        gc.big_mult[i] += 1.0;
      } else {
        gc.big_values.insert(gc.big_values.begin() + i, y);
        gc.big_mult.insert(gc.big_mult.begin() + i, 1.0);
      }
    }
  }
  oracle::PmlData d{sh.design.data(), sh.log_offset.data(), n_cells, static_cast<int>(n_coef), gc.counts.data(),
                    gc.cells.data(), n_pos, sh.fid.data(), static_cast<int>(k), totals};
  const std::vector<double> xy = nebula::positive_xy(sh, gc);
  nebula::MarginalGene mg{&sh, &gc, totals, xy.data()};
  nebula::Terms t(params[n_coef], params[n_coef + 1]);
  nebula::PtmgSums sums = oracle::ptmg_sums(d, params, t.alpha, t.lambda, t.gamma);
  return nebula::ptmg_assemble(mg, params, sums, grad, hess);
}
