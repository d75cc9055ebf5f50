// C-ABI over the reverse-communication stage-two search the device driver
// steps for every gene (the reference's StageTwoSearch, src/sc/nebula.rs:
// 1568-1951). The reference's own tests drive it the same way, with an
// objective that rejects chosen evaluations (nebula.rs:3515-3600): a raised
// Laplace order retried at order one, an order-one pass abandoned on a
// non-finite value, a roundoff-limited BOBYQA reported as failed.
#include <cmath>
#include <new>
#include <vector>

#include "../../../include/nebula_cuda.h"
#include "export.hpp"
#include "search.hpp"

struct nb_search {
  nebula::StageTwoSearch search;
  nb_search(const std::vector<double>& start, const std::vector<double>& lo, const std::vector<double>& hi, int ord,
            double radius_scale)
      : search(start, lo, hi, ord, radius_scale) {}
};

NB_API nb_search* nb_search_new(const double* start, const double* lower, const double* upper, uint32_t n,
                                uint32_t ord, double radius_scale) {
  if (!start || !lower || !upper || n < 1 || n > 2 || ord < 1 || ord > 3 || !(radius_scale > 0.0) ||
      !(radius_scale <= 1.0))
    return nullptr;
  for (uint32_t j = 0; j < n; ++j)
    if (!(std::isfinite(start[j]) && lower[j] < upper[j])) return nullptr;
  std::vector<double> s(start, start + n), lo(lower, lower + n), hi(upper, upper + n);
  try {
    return new nb_search(s, lo, hi, static_cast<int>(ord), radius_scale);
  } catch (...) {
    return nullptr;
  }
}

NB_API uint32_t nb_search_ask(const nb_search* h, double* points, uint32_t max_points) {
  if (!h) return 0;
  const auto& asked = h->search.ask();
  if (points) {
    size_t k = 0;
    for (size_t i = 0; i < asked.size() && i < max_points; ++i)
      for (double v : asked[i]) points[k++] = v;
  }
  return static_cast<uint32_t>(asked.size());
}

NB_API int32_t nb_search_tell(nb_search* h, const double* values, uint32_t n_values) {
  if (!h || !values) return NB_ERR_INVALID_ARGUMENT;
  if (n_values == 0 || n_values != h->search.ask().size()) return NB_ERR_LENGTH_MISMATCH;
  try {
    h->search.tell(std::vector<double>(values, values + n_values));
  } catch (...) {
    return NB_ERR_INVALID_ARGUMENT;
  }
  return NB_OK;
}

NB_API uint32_t nb_search_order(const nb_search* h) { return h ? static_cast<uint32_t>(h->search.order()) : 0; }

NB_API int32_t nb_search_result(const nb_search* h, double* x, int32_t* failed, uint32_t* evaluations) {
  if (!h) return -1;
  if (evaluations) *evaluations = static_cast<uint32_t>(h->search.evaluations());
  if (!h->search.done()) return -1;
  const auto r = h->search.result();
  if (!r) return 0;
  if (x)
    for (size_t j = 0; j < r->first.size(); ++j) x[j] = r->first[j];
  if (failed) *failed = r->second ? 1 : 0;
  return 1;
}

NB_API void nb_search_free(nb_search* h) { delete h; }
