// ln Gamma, digamma and trigamma for x > 0.
//
// The reference's ln_gamma delegates to statrs 0.18.0's Lanczos
// approximation (src/numeric/gamma.rs:213-216); here it is the C library's
// lgamma, accurate to an ulp or two. digamma and trigamma follow the
// reference's scheme (gamma.rs:229-327): unit-step upward recurrence to a
// threshold (20, and 21 for trigamma), then the asymptotic Bernoulli series
// (Abramowitz and Stegun 6.3.18 and 6.4.12).
#pragma once

#include <cmath>
#include <limits>

namespace nebula {

inline double ln_gamma(double x) { return std::lgamma(x); }

inline double digamma(double x) {
  if (!(x > 0.0) || !std::isfinite(x)) return std::numeric_limits<double>::quiet_NaN();
  double shifted = 0.0;
  while (x < 20.0) {
    shifted += 1.0 / x;
    x += 1.0;
  }
  // ln z - 1/(2z) - sum_k B_2k / (2k z^2k)
  const double z2 = 1.0 / (x * x);
  const double series =
      z2 * (1.0 / 12.0 -
            z2 * (1.0 / 120.0 -
                  z2 * (1.0 / 252.0 -
                        z2 * (1.0 / 240.0 - z2 * (1.0 / 132.0 - z2 * (691.0 / 32760.0 - z2 / 12.0))))));
  return std::log(x) - 0.5 / x - series - shifted;
}

inline double trigamma(double x) {
  if (!(x > 0.0) || !std::isfinite(x)) return std::numeric_limits<double>::quiet_NaN();
  double shifted = 0.0;
  while (x < 21.0) {
    shifted += 1.0 / (x * x);
    x += 1.0;
  }
  // 1/z + 1/(2 z^2) + sum_k B_2k / z^(2k+1)
  const double z = 1.0 / x, z2 = z * z;
  const double series =
      z2 * z * (1.0 / 6.0 -
                z2 * (1.0 / 30.0 -
                      z2 * (1.0 / 42.0 - z2 * (1.0 / 30.0 - z2 * (5.0 / 66.0 - z2 * (691.0 / 2730.0 - z2 * 7.0 / 6.0))))));
  return z + 0.5 * z2 + series + shifted;
}

}  // namespace nebula
