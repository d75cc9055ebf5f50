// ORACLE — test infrastructure only. FP64 CPU restatement of the warm-start
// network's forward pass, loss and gradient (layout, GELU and loss as
// csrc/host/mlp_layout.hpp states them), the reference the GPU kernels'
// gradients are checked against.
#include <cmath>
#include <cstdint>
#include <vector>

#include "mlp_layout.hpp"

#define ORACLE_API extern "C" __attribute__((visibility("default")))

namespace {

using namespace nebula::mlp;

double gelu(double x) { return 0.5 * x * (1.0 + std::erf(x / std::sqrt(2.0))); }
double gelu_grad(double x) {
  return 0.5 * (1.0 + std::erf(x / std::sqrt(2.0))) + x * std::exp(-0.5 * x * x) / std::sqrt(2.0 * M_PI);
}

struct Pass {
  double xn[kIn], a1[kHidden], h1[kHidden], a2[kHidden], h2[kHidden], y[kOut];
};

void forward(const float* w, const float* x, Pass* p) {
  for (int k = 0; k < kIn; ++k) p->xn[k] = (double(x[k]) - w[kInMean + k]) * w[kInScale + k];
  for (int i = 0; i < kHidden; ++i) {
    double a = w[kB1 + i];
    for (int k = 0; k < kIn; ++k) a += double(w[kW1 + i * kIn + k]) * p->xn[k];
    p->a1[i] = a;
    p->h1[i] = gelu(a);
  }
  for (int i = 0; i < kHidden; ++i) {
    double a = w[kB2 + i];
    for (int j = 0; j < kHidden; ++j) a += double(w[kW2 + i * kHidden + j]) * p->h1[j];
    p->a2[i] = a;
    p->h2[i] = gelu(a);
  }
  for (int o = 0; o < kOut; ++o) {
    double a = w[kB3 + o];
    for (int h = 0; h < kHidden; ++h) a += double(w[kW3 + o * kHidden + h]) * p->h2[h];
    p->y[o] = a;
  }
}

}  // namespace

// Inference, as nb_mlp_predict_cuda runs it: the weight matrices as BF16
// values (mlp_layout.hpp).
ORACLE_API void oracle_mlp_predict(const float* params, const float* features, uint64_t n, double* out) {
  float q[kParams];
  for (int i = 0; i < kParams; ++i) q[i] = is_weight(i) ? bf16_round(params[i]) : params[i];
  for (uint64_t s = 0; s < n; ++s) {
    Pass p;
    forward(q, features + s * kIn, &p);
    for (int o = 0; o < kOut; ++o) out[s * kOut + o] = p.y[o];
  }
}

// Mean loss over the n samples and its gradient (kParams values; the
// normalisation entries get zero).
ORACLE_API void oracle_mlp_loss_grad(const float* params, const float* features, const float* targets, uint64_t n,
                                     double* grad, double* loss) {
  for (int p = 0; p < kParams; ++p) grad[p] = 0.0;
  double total = 0.0;
  const double inv_n = 1.0 / static_cast<double>(n);
  for (uint64_t s = 0; s < n; ++s) {
    Pass p;
    forward(params, features + s * kIn, &p);
    double d3[kOut], d2[kHidden], d1[kHidden];
    for (int o = 0; o < kOut; ++o) {
      const double e = p.y[o] - targets[s * kOut + o];
      total += loss_weight(o) * e * e * 0.5;
      d3[o] = loss_weight(o) * e * inv_n;
    }
    for (int h = 0; h < kHidden; ++h) {
      double g = 0.0;
      for (int o = 0; o < kOut; ++o) g += double(params[kW3 + o * kHidden + h]) * d3[o];
      d2[h] = g * gelu_grad(p.a2[h]);
    }
    for (int i = 0; i < kHidden; ++i) {
      double g = 0.0;
      for (int h = 0; h < kHidden; ++h) g += double(params[kW2 + h * kHidden + i]) * d2[h];
      d1[i] = g * gelu_grad(p.a1[i]);
    }
    for (int i = 0; i < kHidden; ++i) {
      for (int k = 0; k < kIn; ++k) grad[kW1 + i * kIn + k] += d1[i] * p.xn[k];
      grad[kB1 + i] += d1[i];
      for (int j = 0; j < kHidden; ++j) grad[kW2 + i * kHidden + j] += d2[i] * p.h1[j];
      grad[kB2 + i] += d2[i];
    }
    for (int o = 0; o < kOut; ++o) {
      for (int h = 0; h < kHidden; ++h) grad[kW3 + o * kHidden + h] += d3[o] * p.h2[h];
      grad[kB3 + o] += d3[o];
    }
  }
  *loss = total * inv_n;
}
