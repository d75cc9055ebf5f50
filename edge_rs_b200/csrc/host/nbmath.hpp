// exp and log for doubles, compiled identically for the host (g++) and the
// device (nvcc), so that the CUDA inner fit and its CPU oracle take
// bit-identical logarithms and exponentials and, with the same summation
// tree, produce bit-identical sweeps.
//
// exp: Cody and Waite's argument reduction x = k ln2 + r with ln2 split in a
// 32-bit head and a tail, |r| <= ln2 / 2, then the Taylor polynomial of
// degree 13 in Horner form (truncation below 5e-18 relative), and the scaling
// by 2^k built from the exponent bits in two factors so that results in the
// subnormal range round once.
//
// log: x = m 2^e with m in [sqrt(1/2), sqrt(2)), f = m - 1, s = f / (2 + f),
// ln m = 2 atanh(s) = 2s + 2s^3 (1/3 + s^2/5 + ... + s^20/23) with |s| <= 0.1716
// (truncation below 1e-18), and ln x = e ln2_hi + (e ln2_lo + ln m).
//
// Both are within about one ulp of the correctly rounded result (checked
// against the C library over the ranges the fits use) and handle 0, inf,
// NaN and subnormals.
//
// nb_exp_tab / nb_log_tab: the per-cell pair, by Tang's table-driven method
// (P. T. P. Tang, ACM TOMS 15(2) 1989 for exp, 16(4) 1990 for log), with the
// tables of nbmath_tables.inc (gen_nbmath_tables.py) passed by pointer so a
// kernel can serve them from shared memory. Fewer operations and a shorter
// dependency chain than the pair above, and no division:
//
// exp: n = rint(x 256/ln2), r = x - n ln2/256 (two-part constant, |r| <=
// ln2/512), exp(x) = 2^m 2^(j/256) (1 + q(r)) with n = 256 m + j, q the
// Taylor polynomial of exp(r) - 1 to degree 5 (truncation below 1e-20), the
// table value as hi + lo.
//
// log: x = 2^e m, m in [1, 2), j = round(256 (m - 1)) (j = 256 folds into
// e + 1, m / 2, j = 0), r = m inv_j - 1 exact in one FMA because inv_j has
// nine significant bits and |r| <= 2^-8, ln x = e ln2 + (-ln inv_j) +
// log1p(r), log1p's Taylor polynomial to degree 7 (truncation below 2^-59).
#pragma once

#include <cstdint>
#include <cstring>

#ifdef __CUDACC__
#define NB_HD __host__ __device__ __forceinline__
#else
#define NB_HD inline
#include <cmath>
#endif

namespace nebula {

NB_HD double nb_fma(double a, double b, double c) {
#ifdef __CUDA_ARCH__
  return __fma_rn(a, b, c);
#else
  return __builtin_fma(a, b, c);
#endif
}

NB_HD uint64_t nb_bits(double x) {
#ifdef __CUDA_ARCH__
  return static_cast<uint64_t>(__double_as_longlong(x));
#else
  uint64_t u;
  std::memcpy(&u, &x, 8);
  return u;
#endif
}

NB_HD double nb_from_bits(uint64_t u) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double(static_cast<long long>(u));
#else
  double x;
  std::memcpy(&x, &u, 8);
  return x;
#endif
}

NB_HD double nb_abs(double x) {
#ifdef __CUDA_ARCH__
  return fabs(x);
#else
  return std::fabs(x);
#endif
}

// 2^k for -1022 <= k <= 1023
NB_HD double nb_pow2(int k) { return nb_from_bits(static_cast<uint64_t>(k + 1023) << 52); }

// 1/x correctly rounded (the same double as 1.0 / x).
NB_HD double nb_recip(double x) {
#ifdef __CUDA_ARCH__
  return __drcp_rn(x);
#else
  return 1.0 / x;
#endif
}

NB_HD double nb_rint(double x) {
  // round to nearest (ties to even) for |x| < 2^51
  const double shifter = 6755399441055744.0;  // 1.5 * 2^52
  return (x + shifter) - shifter;
}

NB_HD double nb_exp(double x) {
  if (!(x == x)) return x;                      // NaN
  if (x > 709.782712893384) return 1.0 / 0.0;  // overflow
  if (x < -745.1332191019412) return 0.0;      // underflow
  const double log2e = 1.4426950408889634;
  const double ln2_hi = 6.93147180369123816490e-01;  // ln 2 in 32 bits
  const double ln2_lo = 1.90821492927058770002e-10;
  const double k = nb_rint(x * log2e);
  double r = nb_fma(-k, ln2_hi, x);
  r = nb_fma(-k, ln2_lo, r);
  // Taylor coefficients 1/n!, n = 13 .. 2
  double p = 1.6059043836821613e-10;
  p = nb_fma(p, r, 2.0876756987868100e-09);
  p = nb_fma(p, r, 2.5052108385441720e-08);
  p = nb_fma(p, r, 2.7557319223985893e-07);
  p = nb_fma(p, r, 2.7557319223985888e-06);
  p = nb_fma(p, r, 2.4801587301587302e-05);
  p = nb_fma(p, r, 1.9841269841269841e-04);
  p = nb_fma(p, r, 1.3888888888888889e-03);
  p = nb_fma(p, r, 8.3333333333333332e-03);
  p = nb_fma(p, r, 4.1666666666666664e-02);
  p = nb_fma(p, r, 1.6666666666666666e-01);
  p = nb_fma(p, r, 0.5);
  p = nb_fma(p, r, 1.0);
  const double er = nb_fma(p, r, 1.0);
  const int ki = static_cast<int>(k);
  if (ki >= -1021 && ki <= 1023) return er * nb_pow2(ki);
  // split the scale so that neither factor leaves the normal range
  const int k1 = ki / 2;
  return (er * nb_pow2(k1)) * nb_pow2(ki - k1);
}

NB_HD double nb_log(double x) {
  if (!(x == x)) return x;         // NaN
  if (x < 0.0) return 0.0 / 0.0;   // NaN
  if (x == 0.0) return -1.0 / 0.0;
  if (x == 1.0 / 0.0) return x;
  int e = 0;
  if (x < 2.2250738585072014e-308) {  // subnormal: scale into the normal range
    x *= 18014398509481984.0;         // 2^54
    e = -54;
  }
  uint64_t u = nb_bits(x);
  e += static_cast<int>((u >> 52) & 0x7ff) - 1023;
  double m = nb_from_bits((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);  // [1, 2)
  if (m > 1.4142135623730951) {
    m *= 0.5;
    e += 1;
  }
  const double f = m - 1.0;
  const double s = f / (2.0 + f);
  const double z = s * s;
  // 1/3 + z/5 + ... + z^10/23
  double q = 1.0 / 23.0;
  q = nb_fma(q, z, 1.0 / 21.0);
  q = nb_fma(q, z, 1.0 / 19.0);
  q = nb_fma(q, z, 1.0 / 17.0);
  q = nb_fma(q, z, 1.0 / 15.0);
  q = nb_fma(q, z, 1.0 / 13.0);
  q = nb_fma(q, z, 1.0 / 11.0);
  q = nb_fma(q, z, 1.0 / 9.0);
  q = nb_fma(q, z, 1.0 / 7.0);
  q = nb_fma(q, z, 1.0 / 5.0);
  q = nb_fma(q, z, 1.0 / 3.0);
  // ln m = 2s + 2 s z q, with f - s f kept exact-ish as 2s = f - s f
  const double two_s = f - s * f;
  const double lnm = nb_fma(2.0 * s * z, q, two_s);
  const double ln2_hi = 6.93147180369123816490e-01;
  const double ln2_lo = 1.90821492927058770002e-10;
  const double ed = static_cast<double>(e);
  return nb_fma(ed, ln2_hi, nb_fma(ed, ln2_lo, lnm));
}

// Tables of nb_exp_tab / nb_log_tab.
struct alignas(16) NbPair {
  double a, b;
};
struct NbTableData {
  NbPair exp2_frac[256];   // {hi, lo} of 2^(j/256)
  NbPair log_inv_hi[257];  // {inv_j, hi of -ln inv_j}
  double log_lo[257];      // lo of -ln inv_j
};
constexpr int kNbTableDoubles = static_cast<int>(sizeof(NbTableData) / sizeof(double));

// The host copy; device code reads a __device__ copy (nbmath_device.cuh)
// or a shared-memory copy of it.
inline constexpr NbTableData kNbTables = {
#include "nbmath_tables.inc"
};

NB_HD double nb_exp_tab(double x, const NbTableData* t) {
  const double inv_l = 0x1.71547652b82fep+8;    // 256 / ln 2
  const double l_hi = 0x1.62e42fef80000p-9;     // ln 2 / 256, 34 bits
  const double l_lo = 0x1.1cf79abc9e3b4p-44;
  if (nb_abs(x) < 707.0) {
    // The common range (NaN fails the test): the same steps as below with
    // the special cases left out. n = rint(x * inv_l), rounded once by the
    // fused shifter, is read from the shifter's low word instead of a
    // conversion, (n - n mod 256) / 256 is an arithmetic shift, and 2^m
    // stays normal (|m| <= 1020), so the scaling adds m to er's exponent
    // field (er is in [1/2, 2), the result normal: the same double as
    // er * 2^m).
    const double shifted = nb_fma(x, inv_l, 6755399441055744.0);  // 1.5 * 2^52
    const double n = shifted - 6755399441055744.0;
    double r = nb_fma(-n, l_hi, x);
    r = nb_fma(-n, l_lo, r);
    double p = nb_fma(r, 1.0 / 120.0, 1.0 / 24.0);
    p = nb_fma(p, r, 1.0 / 6.0);
    p = nb_fma(p, r, 0.5);
    const double q = nb_fma(r * r, p, r);
    const int ni = static_cast<int>(static_cast<uint32_t>(nb_bits(shifted)));
    const NbPair s = t->exp2_frac[ni & 255];
    const double er = s.a + nb_fma(s.a, q, s.b);
    return nb_from_bits(nb_bits(er) + (static_cast<uint64_t>(static_cast<int64_t>(ni >> 8)) << 52));
  }
  if (!(x == x)) return x;                      // NaN
  if (x > 709.782712893384) return 1.0 / 0.0;  // overflow
  if (x < -745.1332191019412) return 0.0;      // underflow
  const double n = nb_rint(x * inv_l);
  double r = nb_fma(-n, l_hi, x);
  r = nb_fma(-n, l_lo, r);
  double p = nb_fma(r, 1.0 / 120.0, 1.0 / 24.0);
  p = nb_fma(p, r, 1.0 / 6.0);
  p = nb_fma(p, r, 0.5);
  const double q = nb_fma(r * r, p, r);
  const int ni = static_cast<int>(n);
  const int j = ni & 255;
  const int m = (ni - j) / 256;
  const NbPair s = t->exp2_frac[j];
  const double er = s.a + nb_fma(s.a, q, s.b);
  if (m >= -1021 && m <= 1023) return er * nb_pow2(m);
  const int m1 = m / 2;
  return (er * nb_pow2(m1)) * nb_pow2(m - m1);
}

NB_HD double nb_log_tab(double x, const NbTableData* t) {
  const double ln2_hi = 0x1.62e42fee00000p-1;  // 32 bits: e ln2_hi is exact
  const double ln2_lo = 0x1.a39ef35793c76p-33;
  if (x >= 2.2250738585072014e-308 && x < 1.0 / 0.0) {
    // The common range (positive, normal, finite; NaN fails the test): the
    // same steps as below with the special cases left out, and e converted
    // to a double through the shifter.
    const uint64_t u = nb_bits(x);
    const int e = static_cast<int>(u >> 52) - 1023;
    const uint64_t f = u & 0x000fffffffffffffULL;
    const double m = nb_from_bits(f | 0x3ff0000000000000ULL);  // [1, 2)
    // j = 256 (m just below 2) has its own entry, inv = 1/2
    const int j = static_cast<int>((f + (1ULL << 43)) >> 44);
    const NbPair c = t->log_inv_hi[j];
    const double r = nb_fma(m, c.a, -1.0);
    double p = nb_fma(r, 1.0 / 7.0, -1.0 / 6.0);
    p = nb_fma(p, r, 0.2);
    p = nb_fma(p, r, -0.25);
    p = nb_fma(p, r, 1.0 / 3.0);
    p = nb_fma(p, r, -0.5);
    const double l1p = nb_fma(r * r, p, r);
    const double ed =
        nb_from_bits(0x4338000000000000ULL + static_cast<uint64_t>(static_cast<int64_t>(e))) - 6755399441055744.0;
    const double hi = nb_fma(ed, ln2_hi, c.b);
    const double lo = nb_fma(ed, ln2_lo, t->log_lo[j]);
    return hi + (lo + l1p);
  }
  if (!(x == x)) return x;         // NaN
  if (x < 0.0) return 0.0 / 0.0;   // NaN
  if (x == 0.0) return -1.0 / 0.0;
  if (x == 1.0 / 0.0) return x;
  int e = 0;
  if (x < 2.2250738585072014e-308) {  // subnormal: scale into the normal range
    x *= 18014398509481984.0;         // 2^54
    e = -54;
  }
  const uint64_t u = nb_bits(x);
  e += static_cast<int>((u >> 52) & 0x7ff) - 1023;
  const uint64_t f = u & 0x000fffffffffffffULL;
  const double m = nb_from_bits(f | 0x3ff0000000000000ULL);  // [1, 2)
  const int j = static_cast<int>((f + (1ULL << 43)) >> 44);  // 0 .. 256
  const NbPair c = t->log_inv_hi[j];
  const double r = nb_fma(m, c.a, -1.0);
  double p = nb_fma(r, 1.0 / 7.0, -1.0 / 6.0);
  p = nb_fma(p, r, 0.2);
  p = nb_fma(p, r, -0.25);
  p = nb_fma(p, r, 1.0 / 3.0);
  p = nb_fma(p, r, -0.5);
  const double l1p = nb_fma(r * r, p, r);
  const double ed = static_cast<double>(e);
  const double hi = nb_fma(ed, ln2_hi, c.b);
  const double lo = nb_fma(ed, ln2_lo, t->log_lo[j]);
  return hi + (lo + l1p);
}

}  // namespace nebula
