// Host-side types shared by the device driver and the CPU oracle: the
// per-run inputs every gene reads (nebula.rs:676-710 `Shared`), one gene's
// positive counts (ptmg.rs:1652-1664 `GeneCounts`), stage one's plan
// (nebula.rs:745-773 `GenePlan`), one gene's outcome (nebula.rs:713-726) and
// the error convention (src/errors.rs mapped to nb_status codes).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "nebula_cuda.h"

namespace nebula {

// An EdgeErrors value: the nb_status code and its message.
struct NbError {
  int32_t code;
  std::string message;
};
[[noreturn]] void fail(int32_t code, const std::string& message);

// NebulaParams (nebula.rs:207-258).
struct Params {
  double min0 = 1e-4, min1 = 1e-4, max0 = 10.0, max1 = 1000.0;
  int method = NB_METHOD_LN;
  double cutoff_cell = 20.0, kappa = 800.0, cpc = 0.005;
  uint64_t mincp = 5, min_subjects = 0;
  bool reml = false;
  double eps = 1e-6;
  static Params from(const nb_params* p);
  void validate() const;  // nebula.rs:266-289
};

// Everything the per-gene fit reads but never writes (nebula.rs:676-710).
struct Shared {
  std::vector<double> design;  // centred and scaled, row-major n_cells x n_coef
  std::vector<double> log_offset;
  std::vector<uint64_t> fid;   // subject boundaries, n_subjects + 1
  std::vector<double> sds;     // column standard deviations (centre_design)
  size_t n_cells = 0;
  int n_coef = 0;
  int n_subjects = 0;
  int intercept = 0;
  double log_mean_offset = 0.0;
  double cells_per_subject = 0.0;
  double cv2 = 0.0;
  std::vector<int> cell_columns;
  int method = NB_METHOD_LN;  // after the cells-per-subject override
  Params params;
};

// The gene-major count matrix as the caller handed it over.
struct CsrView {
  uint64_t n_genes, n_cells, nnz;
  const uint32_t* indptr;
  const uint32_t* indices;
  const double* data;
};

// Validation, offsets, centred design, subject totals and the expression
// filter of nebula_sparse_with (nebula.rs:512-657).
struct Prepared {
  Shared shared;
  CsrView counts{};
  std::vector<double> totals;  // gene-major n_genes x n_subjects (cumsum_y)
  std::vector<size_t> kept;    // genes that passed the filter
};
Prepared prepare(const nb_csr* counts, const uint64_t* subject_id, const double* design,
                 uint32_t n_coef, const double* offset, const nb_params* params);

// A read-only view of n contiguous values (the CUDA translation units that
// include this header compile as C++17, without std::span).
template <typename T>
struct View {
  const T* ptr = nullptr;
  size_t n = 0;
  View() = default;
  View(const T* p, size_t count) : ptr(p), n(count) {}
  View(const std::vector<T>& v) : ptr(v.data()), n(v.size()) {}  // NOLINT: views a vector in place
  const T* data() const { return ptr; }
  size_t size() const { return n; }
  bool empty() const { return n == 0; }
  const T* begin() const { return ptr; }
  const T* end() const { return ptr + n; }
  const T& operator[](size_t i) const { return ptr[i]; }
};

// One gene's positive counts (positive_indices, ptmg.rs:1681-1728). `cells`
// and `counts` view either the caller's CSR row itself (borrowed: every
// stored value of the row is positive) or the gene's own compacted copy; a
// move keeps the views valid, a copy is not allowed.
struct GeneCounts {
  View<uint32_t> cells;
  View<double> counts;
  double mean_count = 0.0;
  size_t n_one = 0, n_two = 0;
  // every count is a whole number below 2^24, so a float holds it exactly
  bool small_whole = true;
  // distinct counts other than one and two, increasing, with multiplicities:
  // the gamma-function terms take one lgamma per distinct value
  std::vector<double> big_values, big_mult;

  GeneCounts() = default;
  GeneCounts(GeneCounts&&) = default;
  GeneCounts& operator=(GeneCounts&&) = default;
  GeneCounts(const GeneCounts&) = delete;
  GeneCounts& operator=(const GeneCounts&) = delete;
  // Takes its own copy of n entries and views it.
  void own(const uint32_t* c, const double* y, size_t n) {
    own_cells_.assign(c, c + n);
    own_counts_.assign(y, y + n);
    cells = own_cells_;
    counts = own_counts_;
    small_whole = true;
    for (size_t i = 0; i < n; ++i)
      small_whole = small_whole && y[i] >= 0.0 && y[i] < 16777216.0 && y[i] == static_cast<double>(static_cast<int32_t>(y[i]));
  }

 private:
  friend GeneCounts positive_indices(const CsrView& csr, size_t gene, bool borrow);
  std::vector<uint32_t> own_cells_;
  std::vector<double> own_counts_;
};
// borrow: view the caller's row where every stored value is positive (the
// caller keeps `csr` alive while the result is used); otherwise copy.
GeneCounts positive_indices(const CsrView& csr, size_t gene, bool borrow = false);

// Stage one's decision for one gene (nebula.rs:745-773).
enum class Refit { None, Both, SubjectOnly };
struct GenePlan {
  int ord = 1;
  double sigma = 0.0, gamma = 0.0;
  int convergence = 1;
  std::vector<double> beta_start;
  Refit refit = Refit::Both;
};

// One gene's fit on the centred design scale (nebula.rs:713-726).
struct GeneOutcome {
  std::vector<double> beta, covariance, se;
  double subject = 0.0, cell = 0.0;
  int convergence = 1;
};

// The four scalars the profile objective reads off an inner fit
// (nebula.rs:1337-1346 `InnerFit`).
struct InnerFit {
  double log_likelihood, log_likelihood_prev, log_det, second_order;
};

// What a final (stage-three) inner fit hands finish_gene.
struct FinalFit {
  std::vector<double> beta, information;
  double log_likelihood = 0.0;
  int iterations = 0, backtracks = 0;
};

constexpr int kConvSuccess = 1;
constexpr int kConvCriticalPoint = -10;
constexpr int kConvMaxIter = -20;
constexpr int kConvSingular = -25;
constexpr int kConvNotFinite = -30;
constexpr int kConvStalled = -40;
constexpr int kConvOuterFailed = -50;
constexpr int kConvAtBound = -60;
constexpr int kPmlMaxIter = 50;       // pml.rs:52
constexpr int kPmlMaxBacktrack = 10;  // pml.rs:57

inline size_t packed_len(int n) { return static_cast<size_t>(n) * (n + 1) / 2; }

}  // namespace nebula
