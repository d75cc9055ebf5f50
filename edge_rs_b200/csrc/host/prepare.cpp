// Input validation and the per-run preprocessing of nebula_sparse_with
// (src/sc/nebula.rs:512-657): CSR checks (src/utils/sparse.rs:89-160),
// subject_boundaries (nebula.rs:2138-2154), offset_summary
// (ptmg.rs:1827-1868), centre_design (ptmg.rs:1748-1797),
// cell_level_columns (ptmg.rs:1962-2005), cumsum_y (ptmg.rs:1596-1644), the
// LN->HL override (nebula.rs:612-617) and the expression filter
// (nebula.rs:621-639).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <sstream>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "common.hpp"

namespace nebula {
namespace {

// Runs f(begin, end) over [0, n) in contiguous blocks on the host's threads
// when `parallel` (else as one block); true when every block returned true.
template <typename F>
bool all_blocks(size_t n, bool parallel, F&& f) {
  const size_t hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t blocks = parallel ? std::min<size_t>({hw, 64, std::max<size_t>(n, 1)}) : 1;
  if (blocks == 1) return f(size_t{0}, n);
  std::atomic<bool> ok{true};
  std::vector<std::thread> pool;
  for (size_t b = 0; b < blocks; ++b)
    pool.emplace_back([&, b] {
      if (!f(n * b / blocks, n * (b + 1) / blocks)) ok.store(false);
    });
  for (auto& t : pool) t.join();
  return ok.load();
}

}  // namespace

void fail(int32_t code, const std::string& message) { throw NbError{code, message}; }

Params Params::from(const nb_params* p) {
  Params out;
  if (!p) return out;
  out.min0 = p->min_subject;
  out.min1 = p->min_cell;
  out.max0 = p->max_subject;
  out.max1 = p->max_cell;
  out.method = p->method;
  out.cutoff_cell = p->cutoff_cell;
  out.kappa = p->kappa;
  out.cpc = p->cpc;
  out.mincp = p->mincp;
  out.min_subjects = p->min_subjects;
  out.reml = p->reml != 0;
  out.eps = p->eps;
  return out;
}

void Params::validate() const {
  const double lo[2] = {min0, min1}, hi[2] = {max0, max1};
  for (int i = 0; i < 2; ++i) {
    if (!(std::isfinite(lo[i]) && lo[i] > 0.0))
      fail(NB_ERR_MUST_BE_POSITIVE, "min." + std::to_string(i) + " must be positive");
    if (!(std::isfinite(hi[i]) && hi[i] > lo[i]))
      fail(NB_ERR_INVALID_BOUNDS, "bounds of component " + std::to_string(i) + " are invalid");
  }
  if (!(std::isfinite(eps) && eps > 0.0)) fail(NB_ERR_MUST_BE_POSITIVE, "eps must be positive");
  if (mincp == 0) fail(NB_ERR_MUST_BE_POSITIVE, "mincp must be positive");
  if (method != NB_METHOD_LN && method != NB_METHOD_HL)
    fail(NB_ERR_INVALID_ARGUMENT, "method must be LN or HL");
}

namespace {

// Checks the CSR structure; returns whether every stored value is a
// non-negative finite number (found in the same pass as the index check and
// reported by the caller after the checks that come before it).
bool validate_csr(const nb_csr* c) {
  if (!c) fail(NB_ERR_INVALID_ARGUMENT, "counts is null");
  if (c->format != NB_CSR)
    fail(NB_ERR_MALFORMED_SPARSE, "nebula_sparse needs gene-major counts in CSR form.");
  if (c->n_genes == 0 || c->n_cells == 0) {
    std::ostringstream m;
    m << "empty counts: " << c->n_genes << " genes, " << c->n_cells << " samples";
    fail(NB_ERR_EMPTY_COUNTS, m.str());
  }
  if (!c->indptr || (c->nnz > 0 && (!c->indices || !c->data)))
    fail(NB_ERR_MALFORMED_SPARSE, "null CSR arrays");
  if (c->indptr[0] != 0) fail(NB_ERR_MALFORMED_SPARSE, "indptr must start at 0");
  for (uint64_t g = 0; g < c->n_genes; ++g)
    if (c->indptr[g + 1] < c->indptr[g]) fail(NB_ERR_MALFORMED_SPARSE, "indptr is not non-decreasing");
  if (c->indptr[c->n_genes] != c->nnz)
    fail(NB_ERR_MALFORMED_SPARSE, "indptr does not end at the number of stored values");
  std::atomic<bool> finite{true};
  const bool in_range = all_blocks(c->nnz, c->nnz >= (size_t{1} << 20), [&](size_t a, size_t b) {
    bool ok = true, fin = true;
    for (size_t i = a; i < b; ++i) {
      ok &= c->indices[i] < c->n_cells;
      const double v = c->data[i];
      fin &= std::isfinite(v) && v >= 0.0;
    }
    if (!fin) finite.store(false);
    return ok;
  });
  if (!in_range) fail(NB_ERR_MALFORMED_SPARSE, "cell index out of range");
  return finite.load();
}

}  // namespace

Prepared prepare(const nb_csr* counts, const uint64_t* subject_id, const double* design,
                 uint32_t n_coef, const double* offset, const nb_params* params_in) {
  Params params = Params::from(params_in);
  params.validate();
  const bool finite = validate_csr(counts);
  const size_t n_cells = counts->n_cells;
  const size_t n_genes = counts->n_genes;
  if (n_cells < 2) fail(NB_ERR_INVALID_ARGUMENT, "NEBULA needs more than one cell in the count matrix.");
  if (n_coef == 0) fail(NB_ERR_MUST_BE_POSITIVE, "n_coef must be positive");
  if (!finite) fail(NB_ERR_INVALID_ARGUMENT, "The counts hold a value that is not a non-negative finite number.");
  if (!design) fail(NB_ERR_SHAPE_MISMATCH, "design is null");
  if (!subject_id) fail(NB_ERR_LENGTH_MISMATCH, "subject_id is null");

  Prepared out;
  out.counts = CsrView{counts->n_genes, counts->n_cells, counts->nnz, counts->indptr,
                       counts->indices, counts->data};
  Shared& sh = out.shared;
  sh.params = params;
  sh.n_cells = n_cells;
  sh.n_coef = static_cast<int>(n_coef);

  // subject_boundaries (nebula.rs:2138-2154)
  sh.fid.push_back(0);
  {
    std::unordered_set<uint64_t> seen{subject_id[0]};
    for (size_t i = 1; i < n_cells; ++i) {
      if (subject_id[i] != subject_id[i - 1]) {
        if (seen.count(subject_id[i]))
          fail(NB_ERR_SUBJECTS_NOT_CONTIGUOUS,
               "subject " + std::to_string(subject_id[i]) + " is not contiguous");
        seen.insert(subject_id[i]);
        sh.fid.push_back(i);
      }
    }
    sh.fid.push_back(n_cells);
  }
  sh.n_subjects = static_cast<int>(sh.fid.size()) - 1;
  if (sh.n_subjects < 2)
    fail(NB_ERR_TOO_FEW_SUBJECTS, "need at least 2 subjects, got " + std::to_string(sh.n_subjects));

  // offsets (nebula.rs:569-580, offset_summary ptmg.rs:1827-1868)
  if (offset) {
    for (size_t i = 0; i < n_cells; ++i)
      if (!(std::isfinite(offset[i]) && offset[i] > 0.0))
        fail(NB_ERR_MUST_BE_POSITIVE, "offset must be positive");
  }
  double mean_offset = 1.0;
  if (offset) {
    double s = 0.0;
    for (size_t i = 0; i < n_cells; ++i) s += offset[i];
    mean_offset = s / static_cast<double>(n_cells);
  }
  double cv = 0.0;
  if (mean_offset > 0.0) {
    double ss = 0.0;
    for (size_t i = 0; i < n_cells; ++i) {
      double v = (offset ? offset[i] : 1.0) - mean_offset;
      ss += v * v;
    }
    cv = std::sqrt(ss / static_cast<double>(n_cells)) / mean_offset;
  }
  sh.log_offset.resize(n_cells);
  all_blocks(n_cells, n_cells >= (size_t{1} << 15), [&](size_t a, size_t b) {
    for (size_t i = a; i < b; ++i) sh.log_offset[i] = std::log(offset ? offset[i] : 1.0);
    return true;
  });
  sh.log_mean_offset = std::log(mean_offset);
  sh.cv2 = cv * cv;

  // centre_design (ptmg.rs:1748-1797), in row-major passes over the design;
  // each column's sums still take its cells in order
  const int nc = sh.n_coef;
  std::vector<double> mean(nc, 0.0), var(nc, 0.0);
  for (size_t i = 0; i < n_cells; ++i) {
    const double* row = design + i * nc;
    for (int j = 0; j < nc; ++j)
      if (!std::isfinite(row[j])) fail(NB_ERR_INVALID_ARGUMENT, "design holds a non-finite value.");
  }
  for (size_t i = 0; i < n_cells; ++i) {
    const double* row = design + i * nc;
    for (int j = 0; j < nc; ++j) mean[j] += row[j];
  }
  for (int j = 0; j < nc; ++j) mean[j] /= static_cast<double>(n_cells);
  sh.design.resize(n_cells * nc);
  for (size_t i = 0; i < n_cells; ++i) {
    const double* row = design + i * nc;
    double* out_row = &sh.design[i * nc];
    for (int j = 0; j < nc; ++j) {
      const double d = row[j] - mean[j];
      out_row[j] = d;
      var[j] += d * d;
    }
  }
  // per column: 0 scaled by its sd, 1 a constant column set to one (the
  // intercept), 2 a zero vector (refused below)
  std::vector<int> mode(nc, 0);
  sh.sds.assign(nc, 0.0);
  for (int j = 0; j < nc; ++j) {
    const double sd = std::sqrt(var[j] / static_cast<double>(n_cells));
    if (sd > 0.0) {
      sh.sds[j] = sd;
    } else if (design[j] != 0.0) {
      sh.sds[j] = sd;
      mode[j] = 1;
    } else {
      sh.sds[j] = -1.0;
      mode[j] = 2;
    }
  }
  for (size_t i = 0; i < n_cells; ++i) {
    double* out_row = &sh.design[i * nc];
    for (int j = 0; j < nc; ++j) {
      if (mode[j] == 0) out_row[j] /= sh.sds[j];
      else if (mode[j] == 1) out_row[j] = 1.0;
    }
  }
  for (int j = 0; j < nc; ++j)
    if (sh.sds[j] < 0.0) fail(NB_ERR_INVALID_ARGUMENT, "Some predictors are a zero vector.");
  {
    int n_const = 0;
    for (int j = 0; j < nc; ++j)
      if (sh.sds[j] == 0.0) {
        ++n_const;
        sh.intercept = j;
      }
    if (n_const == 0) fail(NB_ERR_MISSING_INTERCEPT, "the design has no intercept");
    if (n_const > 1) fail(NB_ERR_INVALID_ARGUMENT, "More than one predictor has zero variation.");
  }

  // cell_level_columns (ptmg.rs:1962-2005)
  for (int j = 0; j < nc; ++j) {
    bool varies = false;
    for (int s = 0; s < sh.n_subjects && !varies; ++s) {
      double first = sh.design[sh.fid[s] * nc + j];
      for (size_t i = sh.fid[s]; i < sh.fid[s + 1]; ++i)
        if (sh.design[i * nc + j] != first) {
          varies = true;
          break;
        }
    }
    if (varies) sh.cell_columns.push_back(j);
  }

  // cumsum_y (ptmg.rs:1596-1644)
  const int k = sh.n_subjects;
  std::vector<int> subject_of(n_cells);
  for (int s = 0; s < k; ++s)
    for (size_t i = sh.fid[s]; i < sh.fid[s + 1]; ++i) subject_of[i] = s;
  out.totals.assign(n_genes * k, 0.0);
  // each gene's row on its own, in entry order; blocks of genes run in
  // parallel. Cells come in increasing order (checked later), so the
  // subject advances with them; a cell before the current subject (an
  // unsorted row) looks its subject up
  all_blocks(n_genes, counts->nnz >= (size_t{1} << 20), [&](size_t a, size_t b) {
    for (size_t g = a; g < b; ++g) {
      double* row = &out.totals[g * k];
      int s = 0;
      for (uint32_t e = counts->indptr[g]; e < counts->indptr[g + 1]; ++e) {
        double v = counts->data[e];
        if (v > 0.0) {
          const uint64_t c = counts->indices[e];
          if (c < sh.fid[s]) s = subject_of[c];
          while (c >= sh.fid[s + 1]) ++s;
          row[s] += v;
        }
      }
    }
    return true;
  });

  sh.cells_per_subject = static_cast<double>(n_cells) / static_cast<double>(k);
  sh.method = sh.cells_per_subject < 30.0 ? NB_METHOD_HL : params.method;

  // expression filter (nebula.rs:621-639)
  for (size_t g = 0; g < n_genes; ++g) {
    const double* row = &out.totals[g * k];
    double total = 0.0;
    for (int s = 0; s < k; ++s) total += row[s];
    size_t stored = counts->indptr[g + 1] - counts->indptr[g];
    bool pooled = total / static_cast<double>(n_cells) > params.cpc && stored >= params.mincp;
    if (!pooled) continue;
    if (params.min_subjects != 0) {
      uint64_t expressed = 0;
      for (int s = 0; s < k; ++s)
        if (row[s] / static_cast<double>(sh.fid[s + 1] - sh.fid[s]) > params.cpc) ++expressed;
      if (expressed < params.min_subjects) continue;
    }
    out.kept.push_back(g);
  }
  if (out.kept.empty())
    fail(NB_ERR_NO_GENES_AFTER_FILTERING, "no genes left after filtering " + std::to_string(n_genes));
  return out;
}

GeneCounts positive_indices(const CsrView& csr, size_t gene, bool borrow) {
  GeneCounts out;
  const uint32_t e0 = csr.indptr[gene], e1 = csr.indptr[gene + 1];
  // distinct counts other than one and two: small whole counts tallied by
  // index, anything else in a map, then merged in increasing order
  constexpr int kDirect = 1024;
  std::vector<double> direct(kDirect, 0.0);
  std::unordered_map<double, double> other;
  double sum = 0.0;
  uint32_t prev = 0;
  bool have_prev = false, all_positive = true;
  for (uint32_t e = e0; e < e1; ++e) {
    double v = csr.data[e];
    if (v > 0.0) {
      uint32_t c = csr.indices[e];
      // GeneData::new / PmlData::validate reject unsorted cells (ptmg.rs:51-67)
      if (have_prev && c <= prev)
        fail(NB_ERR_INVALID_ARGUMENT, "Cell indices must be strictly increasing.");
      prev = c;
      have_prev = true;
      sum += v;
      if (v == 1.0) ++out.n_one;
      else if (v == 2.0) ++out.n_two;
      else if (v < kDirect && v == std::floor(v)) direct[static_cast<int>(v)] += 1.0;
      else {
        other[v] += 1.0;
        if (!(v < 16777216.0 && v == std::floor(v))) out.small_whole = false;
      }
    } else {
      all_positive = false;
    }
  }
  if (all_positive && borrow) {
    out.cells = View<uint32_t>(csr.indices + e0, e1 - e0);
    out.counts = View<double>(csr.data + e0, e1 - e0);
  } else {  // the stored zeros left out
    out.own_cells_.reserve(e1 - e0);
    out.own_counts_.reserve(e1 - e0);
    for (uint32_t e = e0; e < e1; ++e) {
      if (csr.data[e] > 0.0) {
        out.own_cells_.push_back(csr.indices[e]);
        out.own_counts_.push_back(csr.data[e]);
      }
    }
    out.cells = out.own_cells_;
    out.counts = out.own_counts_;
  }
  out.mean_count = sum / static_cast<double>(csr.n_cells);
  std::vector<std::pair<double, double>> rest(other.begin(), other.end());
  std::sort(rest.begin(), rest.end());
  size_t r = 0;
  for (int v = 0; v < kDirect; ++v) {
    if (direct[v] == 0.0) continue;
    for (; r < rest.size() && rest[r].first < v; ++r) {
      out.big_values.push_back(rest[r].first);
      out.big_mult.push_back(rest[r].second);
    }
    out.big_values.push_back(static_cast<double>(v));
    out.big_mult.push_back(direct[v]);
  }
  for (; r < rest.size(); ++r) {
    out.big_values.push_back(rest[r].first);
    out.big_mult.push_back(rest[r].second);
  }
  return out;
}

}  // namespace nebula
