// C-ABI over the reverse-communication BOBYQA (the reference exposes the same
// stepper publicly: src/numeric/bobyqa.rs:141 `BobyqaStepper`, :519 `ask`,
// :532 `tell`, :545 `result`).
#include <new>

#include "../../../include/nebula_cuda.h"
#include "bobyqa.hpp"
#include "export.hpp"

struct nb_bobyqa {
  nebula::Bobyqa search;
  nb_bobyqa(const double* x0, const double* lo, const double* hi, int n, double xtol, int maxeval,
            double radius_scale)
      : search(x0, lo, hi, n, xtol, maxeval, radius_scale) {}
};

NB_API nb_bobyqa* nb_bobyqa_new_scaled(const double* x0, const double* lower, const double* upper,
                                       uint32_t n, double xtol_rel, uint32_t maxeval, double radius_scale) {
  if (!x0 || !lower || !upper || n == 0 || !(radius_scale > 0.0)) return nullptr;
  auto* h = new (std::nothrow) nb_bobyqa(x0, lower, upper, static_cast<int>(n), xtol_rel,
                                         static_cast<int>(maxeval), radius_scale);
  if (h && !h->search.ok()) {
    delete h;
    return nullptr;
  }
  return h;
}

NB_API nb_bobyqa* nb_bobyqa_new(const double* x0, const double* lower, const double* upper,
                                uint32_t n, double xtol_rel, uint32_t maxeval) {
  return nb_bobyqa_new_scaled(x0, lower, upper, n, xtol_rel, maxeval, 1.0);
}

NB_API int32_t nb_bobyqa_ask(const nb_bobyqa* h, double* x) {
  if (!h) return 0;
  const double* p = h->search.ask();
  if (!p) return 0;
  for (int j = 0; j < h->search.n(); ++j) x[j] = p[j];
  return 1;
}

NB_API void nb_bobyqa_tell(nb_bobyqa* h, double value) {
  if (h) h->search.tell(value);
}

NB_API int32_t nb_bobyqa_result(const nb_bobyqa* h, double* x, double* f, uint32_t* evaluations) {
  if (!h) return 0;
  nebula::BobyqaResult r = h->search.result();
  if (x)
    for (int j = 0; j < h->search.n(); ++j) x[j] = r.x[j];
  if (f) *f = r.f;
  if (evaluations) *evaluations = static_cast<uint32_t>(r.evaluations);
  return static_cast<int32_t>(r.status);
}

NB_API void nb_bobyqa_free(nb_bobyqa* h) { delete h; }
