// BOBYQA as NLopt 2.7.1 runs it, restated as a coroutine. The arithmetic and
// the order of every operation follow Powell's code as NLopt translates it, so
// that a search fed the same values asks for the same points (the reference's
// restatement is src/numeric/bobyqa.rs; line citations below point there).
// Arrays keep Powell's one-based indexing so each block reads against the
// published Fortran.
#include "bobyqa.hpp"

#include <algorithm>
#include <cmath>
#include <limits>

namespace nebula {
namespace {

// TRSBOX: approximate minimiser of the quadratic model in the intersection of
// the trust region and the box (bobyqa.rs:2007-2423). Pointer arguments are
// zero-based views of the one-based arrays; xpt is column-major npt x n.
void trsbox(int n, int npt, const double* xpt, const double* xopt, const double* gopt,
            const double* hq, const double* pq, const double* sl, const double* su,
            double delta, double* xnew, double* d, double* gnew, double* xbdi, double* s,
            double* hs, double* hred, double* dsq, double* crvmin) {
  auto ix = [npt](int k, int j) { return (k - 1) + (j - 1) * npt; };
  long iterc = 0;
  int nact = 0;
  for (int i = 1; i <= n; ++i) {
    xbdi[i - 1] = 0.0;
    if (xopt[i - 1] <= sl[i - 1]) {
      if (gopt[i - 1] >= 0.0) xbdi[i - 1] = -1.0;
    } else if (xopt[i - 1] >= su[i - 1] && gopt[i - 1] <= 0.0) {
      xbdi[i - 1] = 1.0;
    }
    if (xbdi[i - 1] != 0.0) ++nact;
    d[i - 1] = 0.0;
    gnew[i - 1] = gopt[i - 1];
  }
  double delsq = delta * delta;
  double qred = 0.0;
  *crvmin = -1.0;
  double beta = 0.0, stepsq = 0.0, gredsq = 0.0, ggsav = 0.0, dredsq = 0.0, dredg = 0.0;
  double sredg = 0.0, angbd = 0.0, xsav = 0.0, shs = 0.0, sdec = 0.0;
  long itermax = 0, itcsav = 0;
  int iact = 0;

L20:
  beta = 0.0;
L30:
  stepsq = 0.0;
  for (int i = 1; i <= n; ++i) {
    if (xbdi[i - 1] != 0.0) {
      s[i - 1] = 0.0;
    } else if (beta == 0.0) {
      s[i - 1] = -gnew[i - 1];
    } else {
      s[i - 1] = beta * s[i - 1] - gnew[i - 1];
    }
    stepsq += s[i - 1] * s[i - 1];
  }
  if (stepsq == 0.0) goto L190;
  if (beta == 0.0) {
    gredsq = stepsq;
    itermax = iterc + n - nact;
  }
  if (gredsq * delsq <= qred * 1e-4 * qred) goto L190;
  goto L210;

L50: {
  double resid = delsq, ds = 0.0;
  shs = 0.0;
  for (int i = 1; i <= n; ++i) {
    if (xbdi[i - 1] == 0.0) {
      resid -= d[i - 1] * d[i - 1];
      ds += s[i - 1] * d[i - 1];
      shs += s[i - 1] * hs[i - 1];
    }
  }
  if (resid <= 0.0) goto L90;
  double temp = std::sqrt(stepsq * resid + ds * ds);
  double blen = ds < 0.0 ? (temp - ds) / stepsq : resid / (temp + ds);
  double stplen = blen;
  if (shs > 0.0) stplen = std::min(blen, gredsq / shs);
  iact = 0;
  for (int i = 1; i <= n; ++i) {
    if (s[i - 1] != 0.0) {
      double xsum = xopt[i - 1] + d[i - 1];
      double t = s[i - 1] > 0.0 ? (su[i - 1] - xsum) / s[i - 1] : (sl[i - 1] - xsum) / s[i - 1];
      if (t < stplen) {
        stplen = t;
        iact = i;
      }
    }
  }
  sdec = 0.0;
  if (stplen > 0.0) {
    ++iterc;
    double t = shs / stepsq;
    if (iact == 0 && t > 0.0) {
      *crvmin = std::min(*crvmin, t);
      if (*crvmin == -1.0) *crvmin = t;
    }
    ggsav = gredsq;
    gredsq = 0.0;
    for (int i = 1; i <= n; ++i) {
      gnew[i - 1] += stplen * hs[i - 1];
      if (xbdi[i - 1] == 0.0) gredsq += gnew[i - 1] * gnew[i - 1];
      d[i - 1] += stplen * s[i - 1];
    }
    sdec = std::max(stplen * (ggsav - 0.5 * stplen * shs), 0.0);
    qred += sdec;
  }
  if (iact > 0) {
    ++nact;
    xbdi[iact - 1] = 1.0;
    if (s[iact - 1] < 0.0) xbdi[iact - 1] = -1.0;
    delsq -= d[iact - 1] * d[iact - 1];
    if (delsq <= 0.0) goto L90;
    goto L20;
  }
  if (stplen < blen) {
    if (iterc == itermax) goto L190;
    if (sdec <= qred * 0.01) goto L190;
    beta = gredsq / ggsav;
    goto L30;
  }
}
L90:
  *crvmin = 0.0;
L100:
  if (nact + 1 >= n) goto L190;
  dredsq = 0.0;
  dredg = 0.0;
  gredsq = 0.0;
  for (int i = 1; i <= n; ++i) {
    if (xbdi[i - 1] == 0.0) {
      dredsq += d[i - 1] * d[i - 1];
      dredg += d[i - 1] * gnew[i - 1];
      gredsq += gnew[i - 1] * gnew[i - 1];
      s[i - 1] = d[i - 1];
    } else {
      s[i - 1] = 0.0;
    }
  }
  itcsav = iterc;
  goto L210;

L120: {
  ++iterc;
  double temp = gredsq * dredsq - dredg * dredg;
  if (temp <= qred * 1e-4 * qred) goto L190;
  temp = std::sqrt(temp);
  for (int i = 1; i <= n; ++i) {
    s[i - 1] = xbdi[i - 1] == 0.0 ? (dredg * d[i - 1] - dredsq * gnew[i - 1]) / temp : 0.0;
  }
  sredg = -temp;
  angbd = 1.0;
  iact = 0;
  for (int i = 1; i <= n; ++i) {
    if (xbdi[i - 1] == 0.0) {
      double tempa = xopt[i - 1] + d[i - 1] - sl[i - 1];
      double tempb = su[i - 1] - xopt[i - 1] - d[i - 1];
      if (tempa <= 0.0) {
        ++nact;
        xbdi[i - 1] = -1.0;
        goto L100;
      } else if (tempb <= 0.0) {
        ++nact;
        xbdi[i - 1] = 1.0;
        goto L100;
      }
      double ssq = d[i - 1] * d[i - 1] + s[i - 1] * s[i - 1];
      double a = xopt[i - 1] - sl[i - 1];
      double t = ssq - a * a;
      if (t > 0.0) {
        t = std::sqrt(t) - s[i - 1];
        if (angbd * t > tempa) {
          angbd = tempa / t;
          iact = i;
          xsav = -1.0;
        }
      }
      double b = su[i - 1] - xopt[i - 1];
      t = ssq - b * b;
      if (t > 0.0) {
        t = std::sqrt(t) + s[i - 1];
        if (angbd * t > tempb) {
          angbd = tempb / t;
          iact = i;
          xsav = 1.0;
        }
      }
    }
  }
  goto L210;
}

L150: {
  shs = 0.0;
  double dhs = 0.0, dhd = 0.0;
  for (int i = 1; i <= n; ++i) {
    if (xbdi[i - 1] == 0.0) {
      shs += s[i - 1] * hs[i - 1];
      dhs += d[i - 1] * hs[i - 1];
      dhd += d[i - 1] * hred[i - 1];
    }
  }
  double redmax = 0.0, redsav = 0.0, rdprev = 0.0, rdnext = 0.0;
  long isav = 0;
  long iu = static_cast<long>(angbd * 17.0 + 3.1);
  for (long i = 1; i <= iu; ++i) {
    double angt = angbd * static_cast<double>(i) / static_cast<double>(iu);
    double sth = (angt + angt) / (1.0 + angt * angt);
    double temp = shs + angt * (angt * dhd - dhs - dhs);
    double rednew = sth * (angt * dredg - sredg - 0.5 * sth * temp);
    if (rednew > redmax) {
      redmax = rednew;
      isav = i;
      rdprev = redsav;
    } else if (i == isav + 1) {
      rdnext = rednew;
    }
    redsav = rednew;
  }
  if (isav == 0) goto L190;
  double angt = 0.0;
  if (isav < iu) {
    double temp = (rdnext - rdprev) / (redmax + redmax - rdprev - rdnext);
    angt = angbd * (static_cast<double>(isav) + 0.5 * temp) / static_cast<double>(iu);
  }
  double cth = (1.0 - angt * angt) / (1.0 + angt * angt);
  double sth = (angt + angt) / (1.0 + angt * angt);
  double temp = shs + angt * (angt * dhd - dhs - dhs);
  sdec = sth * (angt * dredg - sredg - 0.5 * sth * temp);
  if (sdec <= 0.0) goto L190;
  dredg = 0.0;
  gredsq = 0.0;
  for (int i = 1; i <= n; ++i) {
    gnew[i - 1] = gnew[i - 1] + (cth - 1.0) * hred[i - 1] + sth * hs[i - 1];
    if (xbdi[i - 1] == 0.0) {
      d[i - 1] = cth * d[i - 1] + sth * s[i - 1];
      dredg += d[i - 1] * gnew[i - 1];
      gredsq += gnew[i - 1] * gnew[i - 1];
    }
    hred[i - 1] = cth * hred[i - 1] + sth * hs[i - 1];
  }
  qred += sdec;
  if (iact > 0 && isav == iu) {
    ++nact;
    xbdi[iact - 1] = xsav;
    goto L100;
  }
  if (sdec > qred * 0.01) goto L120;
}
L190:
  *dsq = 0.0;
  for (int i = 1; i <= n; ++i) {
    xnew[i - 1] = std::max(std::min(xopt[i - 1] + d[i - 1], su[i - 1]), sl[i - 1]);
    if (xbdi[i - 1] == -1.0) xnew[i - 1] = sl[i - 1];
    if (xbdi[i - 1] == 1.0) xnew[i - 1] = su[i - 1];
    d[i - 1] = xnew[i - 1] - xopt[i - 1];
    *dsq += d[i - 1] * d[i - 1];
  }
  return;

L210: {
  int ih = 0;
  for (int j = 1; j <= n; ++j) {
    hs[j - 1] = 0.0;
    for (int i = 1; i <= j; ++i) {
      ++ih;
      if (i < j) hs[j - 1] += hq[ih - 1] * s[i - 1];
      hs[i - 1] += hq[ih - 1] * s[j - 1];
    }
  }
  for (int k = 1; k <= npt; ++k) {
    if (pq[k - 1] != 0.0) {
      double temp = 0.0;
      for (int j = 1; j <= n; ++j) temp += xpt[ix(k, j)] * s[j - 1];
      temp *= pq[k - 1];
      for (int i = 1; i <= n; ++i) hs[i - 1] += temp * xpt[ix(k, i)];
    }
  }
  if (*crvmin != 0.0) goto L50;
  if (iterc > itcsav) goto L150;
  for (int i = 0; i < n; ++i) hred[i] = hs[i];
  goto L120;
}
}

// ALTMOV: two alternative positions for interpolation point knew, along a line
// through xopt and by a constrained Cauchy step (bobyqa.rs:2438-2710).
void altmov(int n, int npt, const double* xpt, const double* xopt, const double* bmat,
            const double* zmat, int ndim, const double* sl, const double* su, int kopt,
            int knew, double adelt, double* xnew, double* xalt, double* alpha,
            double* cauchy, double* glag, double* hcol, double* w) {
  auto ix = [npt](int k, int j) { return (k - 1) + (j - 1) * npt; };
  auto ib = [ndim](int k, int j) { return (k - 1) + (j - 1) * ndim; };
  auto iz = [npt](int k, int j) { return (k - 1) + (j - 1) * npt; };
  const double const_ = 1.0 + std::sqrt(2.0);

  for (int k = 1; k <= npt; ++k) hcol[k - 1] = 0.0;
  for (int j = 1; j <= npt - n - 1; ++j) {
    double temp = zmat[iz(knew, j)];
    for (int k = 1; k <= npt; ++k) hcol[k - 1] += temp * zmat[iz(k, j)];
  }
  *alpha = hcol[knew - 1];
  double ha = 0.5 * *alpha;
  for (int i = 1; i <= n; ++i) glag[i - 1] = bmat[ib(knew, i)];
  for (int k = 1; k <= npt; ++k) {
    double temp = 0.0;
    for (int j = 1; j <= n; ++j) temp += xpt[ix(k, j)] * xopt[j - 1];
    temp *= hcol[k - 1];
    for (int i = 1; i <= n; ++i) glag[i - 1] += temp * xpt[ix(k, i)];
  }

  double presav = 0.0, stpsav = 0.0;
  int ksav = 0;
  long ibdsav = 0;
  for (int k = 1; k <= npt; ++k) {
    if (k == kopt) continue;
    double dderiv = 0.0, distsq = 0.0;
    for (int i = 1; i <= n; ++i) {
      double temp = xpt[ix(k, i)] - xopt[i - 1];
      dderiv += glag[i - 1] * temp;
      distsq += temp * temp;
    }
    double subd = adelt / std::sqrt(distsq);
    double slbd = -subd;
    long ilbd = 0, iubd = 0;
    double sumin = std::min(1.0, subd);
    for (int i = 1; i <= n; ++i) {
      double temp = xpt[ix(k, i)] - xopt[i - 1];
      if (temp > 0.0) {
        if (slbd * temp < sl[i - 1] - xopt[i - 1]) {
          slbd = (sl[i - 1] - xopt[i - 1]) / temp;
          ilbd = -i;
        }
        if (subd * temp > su[i - 1] - xopt[i - 1]) {
          subd = std::max(sumin, (su[i - 1] - xopt[i - 1]) / temp);
          iubd = i;
        }
      } else if (temp < 0.0) {
        if (slbd * temp > su[i - 1] - xopt[i - 1]) {
          slbd = (su[i - 1] - xopt[i - 1]) / temp;
          ilbd = i;
        }
        if (subd * temp < sl[i - 1] - xopt[i - 1]) {
          subd = std::max(sumin, (sl[i - 1] - xopt[i - 1]) / temp);
          iubd = -i;
        }
      }
    }
    double step, vlag;
    long isbd;
    if (k == knew) {
      double diff = dderiv - 1.0;
      step = slbd;
      vlag = slbd * (dderiv - slbd * diff);
      isbd = ilbd;
      double temp = subd * (dderiv - subd * diff);
      if (std::fabs(temp) > std::fabs(vlag)) {
        step = subd;
        vlag = temp;
        isbd = iubd;
      }
      double tempd = 0.5 * dderiv;
      double tempa = tempd - diff * slbd;
      double tempb = tempd - diff * subd;
      if (tempa * tempb < 0.0) {
        temp = tempd * tempd / diff;
        if (std::fabs(temp) > std::fabs(vlag)) {
          step = tempd / diff;
          vlag = temp;
          isbd = 0;
        }
      }
    } else {
      step = slbd;
      vlag = slbd * (1.0 - slbd);
      isbd = ilbd;
      double temp = subd * (1.0 - subd);
      if (std::fabs(temp) > std::fabs(vlag)) {
        step = subd;
        vlag = temp;
        isbd = iubd;
      }
      if (subd > 0.5 && std::fabs(vlag) < 0.25) {
        step = 0.5;
        vlag = 0.25;
        isbd = 0;
      }
      vlag *= dderiv;
    }
    double temp = step * (1.0 - step) * distsq;
    double predsq = vlag * vlag * (vlag * vlag + ha * temp * temp);
    if (predsq > presav) {
      presav = predsq;
      ksav = k;
      stpsav = step;
      ibdsav = isbd;
    }
  }
  // With no line predicting a positive denominator Powell's code leaves ksav
  // at zero; stpsav is zero then, so any row gives xnew = xopt.
  ksav = std::max(ksav, 1);
  for (int i = 1; i <= n; ++i) {
    double temp = xopt[i - 1] + stpsav * (xpt[ix(ksav, i)] - xopt[i - 1]);
    xnew[i - 1] = std::max(sl[i - 1], std::min(su[i - 1], temp));
  }
  if (ibdsav < 0) xnew[-ibdsav - 1] = sl[-ibdsav - 1];
  if (ibdsav > 0) xnew[ibdsav - 1] = su[ibdsav - 1];

  double bigstp = adelt + adelt;
  int iflag = 0;
  double csave = 0.0;
  for (;;) {
    double wfixsq = 0.0, ggfree = 0.0;
    for (int i = 1; i <= n; ++i) {
      w[i - 1] = 0.0;
      double tempa = std::min(xopt[i - 1] - sl[i - 1], glag[i - 1]);
      double tempb = std::max(xopt[i - 1] - su[i - 1], glag[i - 1]);
      if (tempa > 0.0 || tempb < 0.0) {
        w[i - 1] = bigstp;
        ggfree += glag[i - 1] * glag[i - 1];
      }
    }
    if (ggfree == 0.0) {
      *cauchy = 0.0;
      return;
    }
    double step = 0.0;
    for (;;) {
      double temp = adelt * adelt - wfixsq;
      if (temp > 0.0) {
        double wsqsav = wfixsq;
        step = std::sqrt(temp / ggfree);
        ggfree = 0.0;
        for (int i = 1; i <= n; ++i) {
          if (w[i - 1] == bigstp) {
            double t = xopt[i - 1] - step * glag[i - 1];
            if (t <= sl[i - 1]) {
              w[i - 1] = sl[i - 1] - xopt[i - 1];
              wfixsq += w[i - 1] * w[i - 1];
            } else if (t >= su[i - 1]) {
              w[i - 1] = su[i - 1] - xopt[i - 1];
              wfixsq += w[i - 1] * w[i - 1];
            } else {
              ggfree += glag[i - 1] * glag[i - 1];
            }
          }
        }
        if (wfixsq > wsqsav && ggfree > 0.0) continue;
      }
      break;
    }
    double gw = 0.0;
    for (int i = 1; i <= n; ++i) {
      if (w[i - 1] == bigstp) {
        w[i - 1] = -step * glag[i - 1];
        xalt[i - 1] = std::max(sl[i - 1], std::min(su[i - 1], xopt[i - 1] + w[i - 1]));
      } else if (w[i - 1] == 0.0) {
        xalt[i - 1] = xopt[i - 1];
      } else if (glag[i - 1] > 0.0) {
        xalt[i - 1] = sl[i - 1];
      } else {
        xalt[i - 1] = su[i - 1];
      }
      gw += glag[i - 1] * w[i - 1];
    }
    double curv = 0.0;
    for (int k = 1; k <= npt; ++k) {
      double temp = 0.0;
      for (int j = 1; j <= n; ++j) temp += xpt[ix(k, j)] * w[j - 1];
      curv += hcol[k - 1] * temp * temp;
    }
    if (iflag == 1) curv = -curv;
    if (curv > -gw && curv < -const_ * gw) {
      double scale = -gw / curv;
      for (int i = 1; i <= n; ++i) {
        double temp = xopt[i - 1] + scale * w[i - 1];
        xalt[i - 1] = std::max(sl[i - 1], std::min(su[i - 1], temp));
      }
      double a = 0.5 * gw * scale;
      *cauchy = a * a;
    } else {
      double a = gw + 0.5 * curv;
      *cauchy = a * a;
    }
    if (iflag == 0) {
      for (int i = 1; i <= n; ++i) {
        glag[i - 1] = -glag[i - 1];
        w[n + i - 1] = xalt[i - 1];
      }
      csave = *cauchy;
      iflag = 1;
      continue;
    }
    if (csave > *cauchy) {
      for (int i = 1; i <= n; ++i) xalt[i - 1] = w[n + i - 1];
      *cauchy = csave;
    }
    return;
  }
}

// UPDATE: revises bmat and zmat when interpolation point knew moves
// (bobyqa.rs:2722-2788). vlag and w are zero-based views of length ndim.
void update(int n, int npt, double* bmat, double* zmat, int ndim, double* vlag, double beta,
            double denom, int knew, double* w) {
  auto ib = [ndim](int k, int j) { return (k - 1) + (j - 1) * ndim; };
  auto iz = [npt](int k, int j) { return (k - 1) + (j - 1) * npt; };
  const int nptm = npt - n - 1;
  double ztest = 0.0;
  for (int k = 1; k <= npt; ++k)
    for (int j = 1; j <= nptm; ++j) ztest = std::max(ztest, std::fabs(zmat[iz(k, j)]));
  ztest *= 1e-20;
  for (int j = 2; j <= nptm; ++j) {
    if (std::fabs(zmat[iz(knew, j)]) > ztest) {
      double a = zmat[iz(knew, 1)];
      double b = zmat[iz(knew, j)];
      double temp = std::sqrt(a * a + b * b);
      double tempa = a / temp;
      double tempb = b / temp;
      for (int i = 1; i <= npt; ++i) {
        double t = tempa * zmat[iz(i, 1)] + tempb * zmat[iz(i, j)];
        zmat[iz(i, j)] = tempa * zmat[iz(i, j)] - tempb * zmat[iz(i, 1)];
        zmat[iz(i, 1)] = t;
      }
    }
    zmat[iz(knew, j)] = 0.0;
  }
  for (int i = 1; i <= npt; ++i) w[i - 1] = zmat[iz(knew, 1)] * zmat[iz(i, 1)];
  double alpha = w[knew - 1];
  double tau = vlag[knew - 1];
  vlag[knew - 1] -= 1.0;
  double temp = std::sqrt(denom);
  double tempb = zmat[iz(knew, 1)] / temp;
  double tempa = tau / temp;
  for (int i = 1; i <= npt; ++i) zmat[iz(i, 1)] = tempa * zmat[iz(i, 1)] - tempb * vlag[i - 1];
  for (int j = 1; j <= n; ++j) {
    int jp = npt + j;
    w[jp - 1] = bmat[ib(knew, j)];
    double ta = (alpha * vlag[jp - 1] - tau * w[jp - 1]) / denom;
    double tb = (-beta * w[jp - 1] - tau * vlag[jp - 1]) / denom;
    for (int i = 1; i <= jp; ++i) {
      bmat[ib(i, j)] = bmat[ib(i, j)] + ta * vlag[i - 1] + tb * w[i - 1];
      if (i > npt) bmat[ib(jp, i - npt)] = bmat[ib(i, j)];
    }
  }
}

}  // namespace

// nlopt_set_default_initial_step, nlopt_compute_rescaling and bobyqa()'s
// adjustment of the start against the bounds (bobyqa.rs:318-511).
Bobyqa::Bobyqa(const double* x0, const double* lower, const double* upper, int n,
               double xtol_rel, int maxeval, double radius_scale)
    : n_(n), maxeval_(maxeval) {
  if (n <= 0) {
    ok_ = false;
    return;
  }
  std::vector<double> dx(n);
  const double inf = std::numeric_limits<double>::infinity();
  for (int i = 0; i < n; ++i) {
    double lb = lower[i], ub = upper[i], x = x0[i];
    double step = inf;
    if (std::isfinite(ub) && std::isfinite(lb) && (ub - lb) * 0.25 < step && ub > lb)
      step = (ub - lb) * 0.25;
    if (std::isfinite(ub) && ub - x < step && ub > x) step = (ub - x) * 0.75;
    if (std::isfinite(lb) && x - lb < step && x > lb) step = (x - lb) * 0.75;
    if (std::isinf(step)) {
      if (std::isfinite(ub) && std::fabs(ub - x) < std::fabs(step)) step = (ub - x) * 1.1;
      if (std::isfinite(lb) && std::fabs(x - lb) < std::fabs(step)) step = (x - lb) * 1.1;
    }
    if (std::isinf(step) || step == 0.0 || std::fpclassify(step) == FP_SUBNORMAL) step = x;
    if (std::isinf(step) || step == 0.0) step = 1.0;
    dx[i] = step;
  }
  s_.assign(n, 1.0);
  bool differ = false;
  for (int i = 1; i < n; ++i) differ = differ || dx[i] != dx[i - 1];
  if (n > 1 && differ)
    for (int i = 1; i < n; ++i) s_[i] = dx[i] / dx[0];
  for (double v : s_) {
    if (v == 0.0 || !std::isfinite(v)) {
      ok_ = false;
      return;
    }
  }
  x_.assign(n + 1, 0.0);
  xl_.assign(n + 1, 0.0);
  xu_.assign(n + 1, 0.0);
  for (int j = 1; j <= n; ++j) {
    x_[j] = x0[j - 1] / s_[j - 1];
    xl_[j] = lower[j - 1] / s_[j - 1];
    xu_[j] = upper[j - 1] / s_[j - 1];
    if (xl_[j] > xu_[j]) std::swap(xl_[j], xu_[j]);
  }
  rhobeg_ = std::fabs(dx[0] / s_[0]);
  rhoend_ = xtol_rel * rhobeg_;
  if (radius_scale < 1.0) rhobeg_ = std::max(rhobeg_ * radius_scale, 16.0 * rhoend_);
  npt_ = 2 * n + 1;
  ndim_ = npt_ + n;
  sl0_.assign(n + 1, 0.0);
  su0_.assign(n + 1, 0.0);
  for (int j = 1; j <= n; ++j) {
    double temp = xu_[j] - xl_[j];
    if (temp < rhobeg_ + rhobeg_) {
      ok_ = false;
      return;
    }
    sl0_[j] = xl_[j] - x_[j];
    su0_[j] = xu_[j] - x_[j];
    if (sl0_[j] >= -rhobeg_) {
      if (sl0_[j] >= 0.0) {
        x_[j] = xl_[j];
        sl0_[j] = 0.0;
        su0_[j] = temp;
      } else {
        x_[j] = xl_[j] + rhobeg_;
        sl0_[j] = -rhobeg_;
        su0_[j] = std::max(xu_[j] - x_[j], rhobeg_);
      }
    } else if (su0_[j] <= rhobeg_) {
      if (su0_[j] <= 0.0) {
        x_[j] = xu_[j];
        sl0_[j] = -temp;
        su0_[j] = 0.0;
      } else {
        x_[j] = xu_[j] - rhobeg_;
        sl0_[j] = std::min(xl_[j] - x_[j], -rhobeg_);
        su0_[j] = rhobeg_;
      }
    }
  }
  pending_.assign(n, 0.0);
  xbest_.assign(n + 1, 0.0);
  minf_ = inf;
  task_ = run();
}

Bobyqa::~Bobyqa() {
  if (task_.h) task_.h.destroy();
}

const double* Bobyqa::ask() const { return waiting_ ? pending_.data() : nullptr; }

bool Bobyqa::done() const { return !waiting_; }

void Bobyqa::tell(double value) {
  if (!waiting_) return;
  f_ = value;
  waiting_ = false;
  task_.h.resume();
}

BobyqaResult Bobyqa::result() const {
  BobyqaResult r;
  r.x.resize(n_);
  for (int j = 1; j <= n_; ++j) r.x[j - 1] = xbest_[j] * s_[j - 1];
  r.f = minf_;
  r.evaluations = nevals_;
  r.status = rc_;
  return r;
}

Bobyqa::Eval Bobyqa::request() {
  for (int j = 1; j <= n_; ++j) pending_[j - 1] = x_[j] * s_[j - 1];
  ++nevals_;
  waiting_ = true;
  return Eval{this};
}

// PRELIM, BOBYQB and RESCUE as one coroutine (bobyqa.rs:589-1986). Every
// local is declared before the first label so that the gotos cross no
// initialisation.
Bobyqa::Task Bobyqa::run() {
  const int n = n_, npt = npt_, ndim = ndim_, np = n + 1, nptm = npt - np, nh = n * np / 2;
  std::vector<double> xbase(n + 1, 0.0), xpt(npt * n, 0.0), fval(npt + 1, 0.0);
  std::vector<double> xopt(n + 1, 0.0), gopt(n + 1, 0.0), hq(nh + 1, 0.0), pq(npt + 1, 0.0);
  std::vector<double> bmat(ndim * n, 0.0), zmat(npt * nptm, 0.0), sl(sl0_), su(su0_);
  std::vector<double> xnew(n + 1, 0.0), xalt(n + 1, 0.0), d(n + 1, 0.0), vlag(ndim + 1, 0.0);
  std::vector<double> w(3 * ndim + n + npt + 1, 0.0);
  double f = 0.0;
  int kopt = 1, knew = 0, kbase = 1, nresc = 0, nfsav = 0;
  long ntrits = 0, itest = 0;
  double diffa = 0, diffb = 0, diffc = 0, rho = 0, delta = 0, xoptsq = 0, dsq = 0;
  double crvmin = 0, dnorm = 0, adelt = 0, distsq = 0, alpha = 0, cauchy = 0, beta = 0;
  double denom = 0, vquad = 0, ratio = 0, fopt = 0, fsave = 0;
  // prelim
  int nf = 0, nfm = 0, nfx = 0, ipt = 0, jpt = 0;
  double stepa = 0, stepb = 0, fbeg = 0;
  const double rhosq = rhobeg_ * rhobeg_, recip = 1.0 / rhosq;
  // rescue
  int kpt = 0, rip = 0, riq = 0, nrem = 0, kold = 0, rknew = 0;
  double rvquad = 0, fbase = 0, xp = 0, xq = 0, winc = 0, sfrac = 0, rbeta = 0, rdenom = 0;
  // rescue work-space locations inside w: ptsaux(r, j), ptsid(k), its own w(i)
  auto pa = [](int r, int j) { return 1 + (r - 1) + 2 * (j - 1); };
  auto pid = [n](int k) { return 2 * n + k; };
  auto rw = [ndim, n](int i) { return ndim + n + i; };
  auto pid_parts = [&](int k, int* ip, int* iq) {
    double v = w[pid(k)];
    long a = static_cast<long>(v);
    long b = static_cast<long>(static_cast<double>(np) * v - static_cast<double>(a) * np);
    *ip = static_cast<int>(std::max(a, 0L));
    *iq = static_cast<int>(std::max(b, 0L));
  };

  // ---------------- PRELIM (bobyqa.rs:589-800) ----------------
  for (int j = 1; j <= n; ++j) xbase[j] = x_[j];
PRELIM50:
  nfm = nf;
  nfx = nf - n;
  ++nf;
  if (nfm <= 2 * n) {
    if (nfm >= 1 && nfm <= n) {
      stepa = rhobeg_;
      if (su[nfm] == 0.0) stepa = -stepa;
      xpt[ix(nf, nfm)] = stepa;
    } else if (nfm > n) {
      stepa = xpt[ix(nf - n, nfx)];
      stepb = -rhobeg_;
      if (sl[nfx] == 0.0) stepb = std::min(2.0 * rhobeg_, su[nfx]);
      if (su[nfx] == 0.0) stepb = std::max(-2.0 * rhobeg_, sl[nfx]);
      xpt[ix(nf, nfx)] = stepb;
    }
  } else {
    int itemp = (nfm - np) / n;
    jpt = nfm - itemp * n - n;
    ipt = jpt + itemp;
    if (ipt > n) {
      itemp = jpt;
      jpt = ipt - n;
      ipt = itemp;
    }
    xpt[ix(nf, ipt)] = xpt[ix(ipt + 1, ipt)];
    xpt[ix(nf, jpt)] = xpt[ix(jpt + 1, jpt)];
  }
  for (int j = 1; j <= n; ++j) {
    double p = xpt[ix(nf, j)];
    x_[j] = std::min(std::max(xl_[j], xbase[j] + p), xu_[j]);
    if (p == sl[j]) x_[j] = xl_[j];
    if (p == su[j]) x_[j] = xu_[j];
  }
  f = co_await request();
  fval[nf] = f;
  if (nf == 1) {
    fbeg = f;
    kopt = 1;
  } else if (f < fval[kopt]) {
    kopt = nf;
  }
  if (nf <= 2 * n + 1) {
    if (nf >= 2 && nf <= n + 1) {
      gopt[nfm] = (f - fbeg) / stepa;
      if (npt < nf + n) {
        bmat[ib(1, nfm)] = -1.0 / stepa;
        bmat[ib(nf, nfm)] = 1.0 / stepa;
        bmat[ib(npt + nfm, nfm)] = -0.5 * rhosq;
      }
    } else if (nf >= n + 2) {
      int ih = nfx * (nfx + 1) / 2;
      double temp = (f - fbeg) / stepb;
      double diff = stepb - stepa;
      hq[ih] = 2.0 * (temp - gopt[nfx]) / diff;
      gopt[nfx] = (gopt[nfx] * stepb - temp * stepa) / diff;
      if (stepa * stepb < 0.0 && f < fval[nf - n]) {
        fval[nf] = fval[nf - n];
        fval[nf - n] = f;
        if (kopt == nf) kopt = nf - n;
        xpt[ix(nf - n, nfx)] = stepb;
        xpt[ix(nf, nfx)] = stepa;
      }
      bmat[ib(1, nfx)] = -(stepa + stepb) / (stepa * stepb);
      bmat[ib(nf, nfx)] = -0.5 / xpt[ix(nf - n, nfx)];
      bmat[ib(nf - n, nfx)] = -bmat[ib(1, nfx)] - bmat[ib(nf, nfx)];
      zmat[iz(1, nfx)] = std::sqrt(2.0) / (stepa * stepb);
      zmat[iz(nf, nfx)] = std::sqrt(0.5) / rhosq;
      zmat[iz(nf - n, nfx)] = -zmat[iz(1, nfx)] - zmat[iz(nf, nfx)];
    }
  } else {
    int ih = ipt * (ipt - 1) / 2 + jpt;
    zmat[iz(1, nfx)] = recip;
    zmat[iz(nf, nfx)] = recip;
    zmat[iz(ipt + 1, nfx)] = -recip;
    zmat[iz(jpt + 1, nfx)] = -recip;
    double temp = xpt[ix(nf, ipt)] * xpt[ix(nf, jpt)];
    hq[ih] = (fbeg - fval[ipt + 1] - fval[jpt + 1] + f) / temp;
  }
  if (stop_evals()) {
    rc_ = BobyqaStatus::MaxevalReached;
    goto AFTER_PRELIM;
  }
  if (nf < npt) goto PRELIM50;
AFTER_PRELIM:
  xoptsq = 0.0;
  for (int i = 1; i <= n; ++i) {
    xopt[i] = xpt[ix(kopt, i)];
    xoptsq += xopt[i] * xopt[i];
  }
  fsave = fval[1];
  if (rc_ != BobyqaStatus::Running) goto L720;

  // ---------------- BOBYQB (bobyqa.rs:807-1547) ----------------
  kbase = 1;
  rho = rhobeg_;
  delta = rho;
  nresc = nevals_;
  ntrits = 0;
  diffa = 0.0;
  diffb = 0.0;
  itest = 0;
  nfsav = nevals_;

L20:
  if (kopt != kbase) {
    int ih = 0;
    for (int j = 1; j <= n; ++j) {
      for (int i = 1; i <= j; ++i) {
        ++ih;
        if (i < j) gopt[j] += hq[ih] * xopt[i];
        gopt[i] += hq[ih] * xopt[j];
      }
    }
    if (nevals_ > npt) {
      for (int k = 1; k <= npt; ++k) {
        double temp = 0.0;
        for (int j = 1; j <= n; ++j) temp += xpt[ix(k, j)] * xopt[j];
        temp *= pq[k];
        for (int i = 1; i <= n; ++i) gopt[i] += temp * xpt[ix(k, i)];
      }
    }
  }

L60:
  trsbox(n, npt, xpt.data(), &xopt[1], &gopt[1], &hq[1], &pq[1], &sl[1], &su[1], delta,
         &xnew[1], &d[1], &w[1], &w[n + 1], &w[2 * n + 1], &w[3 * n + 1], &w[4 * n + 1], &dsq,
         &crvmin);
  dnorm = std::min(delta, std::sqrt(dsq));
  if (dnorm < 0.5 * rho) {
    ntrits = -1;
    distsq = (10.0 * rho) * (10.0 * rho);
    if (nevals_ <= nfsav + 2) goto L650;
    {
      double errbig = std::max(std::max(diffa, diffb), diffc);
      double frhosq = rho * 0.125 * rho;
      if (crvmin > 0.0 && errbig > frhosq * crvmin) goto L650;
      double bdtol = errbig / rho;
      for (int j = 1; j <= n; ++j) {
        double bdtest = bdtol;
        if (xnew[j] == sl[j]) bdtest = w[j];
        if (xnew[j] == su[j]) bdtest = -w[j];
        if (bdtest < bdtol) {
          double curv = hq[(j + j * j) / 2];
          for (int k = 1; k <= npt; ++k) {
            double v = xpt[ix(k, j)];
            curv += pq[k] * (v * v);
          }
          bdtest += 0.5 * curv * rho;
          if (bdtest < bdtol) goto L650;
        }
      }
    }
    goto L680;
  }
  ++ntrits;

L90:
  if (dsq <= xoptsq * 0.001) {
    double fracsq = xoptsq * 0.25;
    double sumpq = 0.0;
    for (int k = 1; k <= npt; ++k) {
      sumpq += pq[k];
      double sum = -0.5 * xoptsq;
      for (int i = 1; i <= n; ++i) sum += xpt[ix(k, i)] * xopt[i];
      w[npt + k] = sum;
      double temp = fracsq - 0.5 * sum;
      for (int i = 1; i <= n; ++i) {
        w[i] = bmat[ib(k, i)];
        vlag[i] = sum * xpt[ix(k, i)] + temp * xopt[i];
        int ip = npt + i;
        for (int j = 1; j <= i; ++j)
          bmat[ib(ip, j)] = bmat[ib(ip, j)] + w[i] * vlag[j] + vlag[i] * w[j];
      }
    }
    for (int jj = 1; jj <= nptm; ++jj) {
      double sumz = 0.0, sumw = 0.0;
      for (int k = 1; k <= npt; ++k) {
        sumz += zmat[iz(k, jj)];
        vlag[k] = w[npt + k] * zmat[iz(k, jj)];
        sumw += vlag[k];
      }
      for (int j = 1; j <= n; ++j) {
        double sum = (fracsq * sumz - 0.5 * sumw) * xopt[j];
        for (int k = 1; k <= npt; ++k) sum += vlag[k] * xpt[ix(k, j)];
        w[j] = sum;
        for (int k = 1; k <= npt; ++k) bmat[ib(k, j)] += sum * zmat[iz(k, jj)];
      }
      for (int i = 1; i <= n; ++i) {
        int ip = i + npt;
        double temp = w[i];
        for (int j = 1; j <= i; ++j) bmat[ib(ip, j)] += temp * w[j];
      }
    }
    int ih = 0;
    for (int j = 1; j <= n; ++j) {
      w[j] = -0.5 * sumpq * xopt[j];
      for (int k = 1; k <= npt; ++k) {
        w[j] += pq[k] * xpt[ix(k, j)];
        xpt[ix(k, j)] -= xopt[j];
      }
      for (int i = 1; i <= j; ++i) {
        ++ih;
        hq[ih] = hq[ih] + w[i] * xopt[j] + xopt[i] * w[j];
        bmat[ib(npt + i, j)] = bmat[ib(npt + j, i)];
      }
    }
    for (int i = 1; i <= n; ++i) {
      xbase[i] += xopt[i];
      xnew[i] -= xopt[i];
      sl[i] -= xopt[i];
      su[i] -= xopt[i];
      xopt[i] = 0.0;
    }
    xoptsq = 0.0;
  }
  if (ntrits == 0) goto L210;
  goto L230;

L190:
  // RESCUE (bobyqa.rs:1581-1986), entered with nfsav and kbase recorded.
  nfsav = nevals_;
  kbase = kopt;
  {
    sfrac = 0.5 / np;
    double sumpq = 0.0;
    winc = 0.0;
    for (int k = 1; k <= npt; ++k) {
      double dsqk = 0.0;
      for (int j = 1; j <= n; ++j) {
        xpt[ix(k, j)] -= xopt[j];
        dsqk += xpt[ix(k, j)] * xpt[ix(k, j)];
      }
      sumpq += pq[k];
      w[rw(ndim + k)] = dsqk;
      winc = std::max(winc, dsqk);
      for (int j = 1; j <= nptm; ++j) zmat[iz(k, j)] = 0.0;
    }
    int ih = 0;
    for (int j = 1; j <= n; ++j) {
      w[rw(j)] = 0.5 * sumpq * xopt[j];
      for (int k = 1; k <= npt; ++k) w[rw(j)] += pq[k] * xpt[ix(k, j)];
      for (int i = 1; i <= j; ++i) {
        ++ih;
        hq[ih] = hq[ih] + w[rw(i)] * xopt[j] + w[rw(j)] * xopt[i];
      }
    }
    for (int j = 1; j <= n; ++j) {
      xbase[j] += xopt[j];
      sl[j] -= xopt[j];
      su[j] -= xopt[j];
      xopt[j] = 0.0;
      w[pa(1, j)] = std::min(delta, su[j]);
      w[pa(2, j)] = std::max(-delta, sl[j]);
      if (w[pa(1, j)] + w[pa(2, j)] < 0.0) std::swap(w[pa(1, j)], w[pa(2, j)]);
      if (std::fabs(w[pa(2, j)]) < 0.5 * std::fabs(w[pa(1, j)])) w[pa(2, j)] = 0.5 * w[pa(1, j)];
      for (int i = 1; i <= ndim; ++i) bmat[ib(i, j)] = 0.0;
    }
    fbase = fval[kopt];
    w[pid(1)] = sfrac;
    for (int j = 1; j <= n; ++j) {
      int jp = j + 1, jpn = jp + n;
      w[pid(jp)] = j + sfrac;
      double a1 = w[pa(1, j)], a2 = w[pa(2, j)];
      if (jpn <= npt) {
        w[pid(jpn)] = static_cast<double>(j) / np + sfrac;
        double temp = 1.0 / (a1 - a2);
        bmat[ib(jp, j)] = -temp + 1.0 / a1;
        bmat[ib(jpn, j)] = temp + 1.0 / a2;
        bmat[ib(1, j)] = -bmat[ib(jp, j)] - bmat[ib(jpn, j)];
        zmat[iz(1, j)] = std::sqrt(2.0) / std::fabs(a1 * a2);
        zmat[iz(jp, j)] = zmat[iz(1, j)] * a2 * temp;
        zmat[iz(jpn, j)] = -zmat[iz(1, j)] * a1 * temp;
      } else {
        bmat[ib(1, j)] = -1.0 / a1;
        bmat[ib(jp, j)] = 1.0 / a1;
        bmat[ib(j + npt, j)] = -0.5 * (a1 * a1);
      }
    }
    if (npt >= n + np) {
      for (int k = 2 * np; k <= npt; ++k) {
        int iw = static_cast<int>((static_cast<double>(k - np) - 0.5) / n);
        int ip = k - np - iw * n;
        int iq = ip + iw;
        if (iq > n) iq -= n;
        w[pid(k)] = ip + static_cast<double>(iq) / np + sfrac;
        double temp = 1.0 / (w[pa(1, ip)] * w[pa(1, iq)]);
        zmat[iz(1, k - np)] = temp;
        zmat[iz(ip + 1, k - np)] = -temp;
        zmat[iz(iq + 1, k - np)] = -temp;
        zmat[iz(k, k - np)] = temp;
      }
    }
    nrem = npt;
    kold = 1;
    rknew = kopt;
    rbeta = 0.0;
    rdenom = 0.0;
  }
R80:
  for (int j = 1; j <= n; ++j) std::swap(bmat[ib(kold, j)], bmat[ib(rknew, j)]);
  for (int j = 1; j <= nptm; ++j) std::swap(zmat[iz(kold, j)], zmat[iz(rknew, j)]);
  w[pid(kold)] = w[pid(rknew)];
  w[pid(rknew)] = 0.0;
  w[rw(ndim + rknew)] = 0.0;
  --nrem;
  if (rknew != kopt) {
    std::swap(vlag[kold], vlag[rknew]);
    update(n, npt, bmat.data(), zmat.data(), ndim, &vlag[1], rbeta, rdenom, rknew, &w[rw(1)]);
    if (nrem == 0) goto RESCUE_END;
    for (int k = 1; k <= npt; ++k) w[rw(ndim + k)] = std::fabs(w[rw(ndim + k)]);
  }
R120: {
  double dsqmin = 0.0;
  for (int k = 1; k <= npt; ++k) {
    double v = w[rw(ndim + k)];
    if (v > 0.0 && (dsqmin == 0.0 || v < dsqmin)) {
      rknew = k;
      dsqmin = v;
    }
  }
  if (dsqmin == 0.0) goto R260_START;
  for (int j = 1; j <= n; ++j) w[rw(npt + j)] = xpt[ix(rknew, j)];
  for (int k = 1; k <= npt; ++k) {
    double sum = 0.0;
    if (k == kopt) {
    } else if (w[pid(k)] == 0.0) {
      for (int j = 1; j <= n; ++j) sum += w[rw(npt + j)] * xpt[ix(k, j)];
    } else {
      int ip, iq;
      pid_parts(k, &ip, &iq);
      if (ip > 0) sum = w[rw(npt + ip)] * w[pa(1, ip)];
      if (iq > 0) {
        int iw = ip == 0 ? 2 : 1;
        sum += w[rw(npt + iq)] * w[pa(iw, iq)];
      }
    }
    w[rw(k)] = 0.5 * sum * sum;
  }
  for (int k = 1; k <= npt; ++k) {
    double sum = 0.0;
    for (int j = 1; j <= n; ++j) sum += bmat[ib(k, j)] * w[rw(npt + j)];
    vlag[k] = sum;
  }
  rbeta = 0.0;
  for (int j = 1; j <= nptm; ++j) {
    double sum = 0.0;
    for (int k = 1; k <= npt; ++k) sum += zmat[iz(k, j)] * w[rw(k)];
    rbeta -= sum * sum;
    for (int k = 1; k <= npt; ++k) vlag[k] += sum * zmat[iz(k, j)];
  }
  double bsum = 0.0, dsqk = 0.0;
  for (int j = 1; j <= n; ++j) {
    double sum = 0.0;
    for (int k = 1; k <= npt; ++k) sum += bmat[ib(k, j)] * w[rw(k)];
    int jp = j + npt;
    bsum += sum * w[rw(jp)];
    for (int ip = npt + 1; ip <= ndim; ++ip) sum += bmat[ib(ip, j)] * w[rw(ip)];
    bsum += sum * w[rw(jp)];
    vlag[jp] = sum;
    double v = xpt[ix(rknew, j)];
    dsqk += v * v;
  }
  rbeta = 0.5 * dsqk * dsqk + rbeta - bsum;
  vlag[kopt] += 1.0;
  rdenom = 0.0;
  double vlmxsq = 0.0;
  for (int k = 1; k <= npt; ++k) {
    if (w[pid(k)] != 0.0) {
      double hdiag = 0.0;
      for (int j = 1; j <= nptm; ++j) hdiag += zmat[iz(k, j)] * zmat[iz(k, j)];
      double den = rbeta * hdiag + vlag[k] * vlag[k];
      if (den > rdenom) {
        kold = k;
        rdenom = den;
      }
    }
    vlmxsq = std::max(vlmxsq, vlag[k] * vlag[k]);
  }
  if (rdenom <= vlmxsq * 0.01) {
    w[rw(ndim + rknew)] = -w[rw(ndim + rknew)] - winc;
    goto R120;
  }
  goto R80;
}
R260_START:
  kpt = 0;
R260:
  ++kpt;
  if (kpt > npt) goto RESCUE_END;
  if (w[pid(kpt)] == 0.0) goto R260;
  if (stop_evals()) {
    rc_ = BobyqaStatus::MaxevalReached;
    goto RESCUE_END;
  }
  {
    int ih = 0;
    for (int j = 1; j <= n; ++j) {
      w[rw(j)] = xpt[ix(kpt, j)];
      xpt[ix(kpt, j)] = 0.0;
      double temp = pq[kpt] * w[rw(j)];
      for (int i = 1; i <= j; ++i) {
        ++ih;
        hq[ih] += temp * w[rw(i)];
      }
    }
    pq[kpt] = 0.0;
    pid_parts(kpt, &rip, &riq);
    if (rip > 0) {
      xp = w[pa(1, rip)];
      xpt[ix(kpt, rip)] = xp;
    }
    if (riq > 0) {
      xq = w[pa(1, riq)];
      if (rip == 0) xq = w[pa(2, riq)];
      xpt[ix(kpt, riq)] = xq;
    }
    double vq = fbase;
    int ihp = 0;
    if (rip > 0) {
      ihp = (rip + rip * rip) / 2;
      vq += xp * (gopt[rip] + 0.5 * xp * hq[ihp]);
    }
    if (riq > 0) {
      int ihq = (riq + riq * riq) / 2;
      vq += xq * (gopt[riq] + 0.5 * xq * hq[ihq]);
      if (rip > 0) {
        int iw = std::max(ihp, ihq) - std::abs(rip - riq);
        vq += xp * xq * hq[iw];
      }
    }
    for (int k = 1; k <= npt; ++k) {
      double temp = 0.0;
      if (rip > 0) temp += xp * xpt[ix(k, rip)];
      if (riq > 0) temp += xq * xpt[ix(k, riq)];
      vq += 0.5 * pq[k] * temp * temp;
    }
    rvquad = vq;
    for (int i = 1; i <= n; ++i) {
      double p = xpt[ix(kpt, i)];
      x_[i] = std::min(std::max(xl_[i], xbase[i] + p), xu_[i]);
      if (p == sl[i]) x_[i] = xl_[i];
      if (p == su[i]) x_[i] = xu_[i];
    }
  }
  f = co_await request();
  fval[kpt] = f;
  if (f < fval[kopt]) kopt = kpt;
  if (stop_evals()) {
    rc_ = BobyqaStatus::MaxevalReached;
    goto RESCUE_END;
  }
  {
    double diff = f - rvquad;
    for (int i = 1; i <= n; ++i) gopt[i] += diff * bmat[ib(kpt, i)];
    for (int k = 1; k <= npt; ++k) {
      double sum = 0.0;
      for (int j = 1; j <= nptm; ++j) sum += zmat[iz(k, j)] * zmat[iz(kpt, j)];
      double temp = diff * sum;
      if (w[pid(k)] == 0.0) {
        pq[k] += temp;
      } else {
        int ip, iq;
        pid_parts(k, &ip, &iq);
        int ihq = (iq * iq + iq) / 2;
        if (ip == 0) {
          double a = w[pa(2, iq)];
          hq[ihq] += temp * (a * a);
        } else {
          int ihp = (ip * ip + ip) / 2;
          double a = w[pa(1, ip)];
          hq[ihp] += temp * (a * a);
          if (iq > 0) {
            double b = w[pa(1, iq)];
            hq[ihq] += temp * (b * b);
            int iw = std::max(ihp, ihq) - std::abs(iq - ip);
            hq[iw] += temp * a * b;
          }
        }
      }
    }
    w[pid(kpt)] = 0.0;
  }
  goto R260;
RESCUE_END:
  // back in BOBYQB after the call to RESCUE (bobyqa.rs:1012-1033)
  xoptsq = 0.0;
  if (kopt != kbase) {
    for (int i = 1; i <= n; ++i) {
      xopt[i] = xpt[ix(kopt, i)];
      xoptsq += xopt[i] * xopt[i];
    }
  }
  if (rc_ != BobyqaStatus::Running) goto L720;
  nresc = nevals_;
  if (nfsav < nevals_) {
    nfsav = nevals_;
    goto L20;
  }
  if (ntrits > 0) goto L60;

L210:
  altmov(n, npt, xpt.data(), &xopt[1], bmat.data(), zmat.data(), ndim, &sl[1], &su[1], kopt,
         knew, adelt, &xnew[1], &xalt[1], &alpha, &cauchy, &w[1], &w[n + 1], &w[ndim + 1]);
  for (int i = 1; i <= n; ++i) d[i] = xnew[i] - xopt[i];

L230:
  for (int k = 1; k <= npt; ++k) {
    double suma = 0.0, sumb = 0.0, sum = 0.0;
    for (int j = 1; j <= n; ++j) {
      suma += xpt[ix(k, j)] * d[j];
      sumb += xpt[ix(k, j)] * xopt[j];
      sum += bmat[ib(k, j)] * d[j];
    }
    w[k] = suma * (0.5 * suma + sumb);
    vlag[k] = sum;
    w[npt + k] = suma;
  }
  beta = 0.0;
  for (int jj = 1; jj <= nptm; ++jj) {
    double sum = 0.0;
    for (int k = 1; k <= npt; ++k) sum += zmat[iz(k, jj)] * w[k];
    beta -= sum * sum;
    for (int k = 1; k <= npt; ++k) vlag[k] += sum * zmat[iz(k, jj)];
  }
  {
    dsq = 0.0;
    double bsum = 0.0, dx = 0.0;
    for (int j = 1; j <= n; ++j) {
      dsq += d[j] * d[j];
      double sum = 0.0;
      for (int k = 1; k <= npt; ++k) sum += w[k] * bmat[ib(k, j)];
      bsum += sum * d[j];
      int jp = npt + j;
      for (int i = 1; i <= n; ++i) sum += bmat[ib(jp, i)] * d[i];
      vlag[jp] = sum;
      bsum += sum * d[j];
      dx += d[j] * xopt[j];
    }
    beta = dx * dx + dsq * (xoptsq + dx + dx + 0.5 * dsq) + beta - bsum;
  }
  vlag[kopt] += 1.0;
  if (ntrits == 0) {
    double vk = vlag[knew];
    denom = vk * vk + alpha * beta;
    if (denom < cauchy && cauchy > 0.0) {
      for (int i = 1; i <= n; ++i) {
        xnew[i] = xalt[i];
        d[i] = xnew[i] - xopt[i];
      }
      cauchy = 0.0;
      goto L230;
    }
    if (denom <= 0.5 * (vk * vk)) {
      if (nevals_ > nresc) goto L190;
      rc_ = BobyqaStatus::RoundoffLimited;
      goto L720;
    }
  } else {
    double delsq = delta * delta, scaden = 0.0, biglsq = 0.0;
    knew = 0;
    for (int k = 1; k <= npt; ++k) {
      if (k == kopt) continue;
      double hdiag = 0.0;
      for (int jj = 1; jj <= nptm; ++jj) hdiag += zmat[iz(k, jj)] * zmat[iz(k, jj)];
      double den = beta * hdiag + vlag[k] * vlag[k];
      double dk = 0.0;
      for (int j = 1; j <= n; ++j) {
        double v = xpt[ix(k, j)] - xopt[j];
        dk += v * v;
      }
      double r = dk / delsq;
      double temp = std::max(1.0, r * r);
      if (temp * den > scaden) {
        scaden = temp * den;
        knew = k;
        denom = den;
      }
      biglsq = std::max(biglsq, temp * (vlag[k] * vlag[k]));
    }
    if (scaden <= 0.5 * biglsq) {
      if (nevals_ > nresc) goto L190;
      rc_ = BobyqaStatus::RoundoffLimited;
      goto L720;
    }
  }

L360:
  for (int i = 1; i <= n; ++i) {
    x_[i] = std::min(std::max(xl_[i], xbase[i] + xnew[i]), xu_[i]);
    if (xnew[i] == sl[i]) x_[i] = xl_[i];
    if (xnew[i] == su[i]) x_[i] = xu_[i];
  }
  if (stop_evals()) {
    rc_ = BobyqaStatus::MaxevalReached;
    goto L720;
  }
  f = co_await request();
  if (ntrits == -1) {
    fsave = f;
    rc_ = BobyqaStatus::XtolReached;
    if (fsave < fval[kopt]) {
      minf_ = f;
      xbest_ = x_;
      co_return;
    }
    goto L720;
  }
  {
    fopt = fval[kopt];
    vquad = 0.0;
    int ih = 0;
    for (int j = 1; j <= n; ++j) {
      vquad += d[j] * gopt[j];
      for (int i = 1; i <= j; ++i) {
        ++ih;
        double temp = d[i] * d[j];
        if (i == j) temp *= 0.5;
        vquad += hq[ih] * temp;
      }
    }
    for (int k = 1; k <= npt; ++k) {
      double v = w[npt + k];
      vquad += 0.5 * pq[k] * (v * v);
    }
    double diff = f - fopt - vquad;
    diffc = diffb;
    diffb = diffa;
    diffa = std::fabs(diff);
    if (dnorm > rho) nfsav = nevals_;
    if (ntrits > 0) {
      if (vquad >= 0.0) {
        rc_ = BobyqaStatus::RoundoffLimited;
        goto L720;
      }
      ratio = (f - fopt) / vquad;
      if (ratio <= 0.1) {
        delta = std::min(0.5 * delta, dnorm);
      } else if (ratio <= 0.7) {
        delta = std::max(0.5 * delta, dnorm);
      } else {
        delta = std::max(0.5 * delta, dnorm + dnorm);
      }
      if (delta <= rho * 1.5) delta = rho;
      if (f < fopt) {
        int ksav = knew;
        double densav = denom, delsq = delta * delta, scaden = 0.0, biglsq = 0.0;
        knew = 0;
        for (int k = 1; k <= npt; ++k) {
          double hdiag = 0.0;
          for (int jj = 1; jj <= nptm; ++jj) hdiag += zmat[iz(k, jj)] * zmat[iz(k, jj)];
          double den = beta * hdiag + vlag[k] * vlag[k];
          double dk = 0.0;
          for (int j = 1; j <= n; ++j) {
            double v = xpt[ix(k, j)] - xnew[j];
            dk += v * v;
          }
          double r = dk / delsq;
          double temp = std::max(1.0, r * r);
          if (temp * den > scaden) {
            scaden = temp * den;
            knew = k;
            denom = den;
          }
          biglsq = std::max(biglsq, temp * (vlag[k] * vlag[k]));
        }
        if (scaden <= 0.5 * biglsq) {
          knew = ksav;
          denom = densav;
        }
      }
    }
    update(n, npt, bmat.data(), zmat.data(), ndim, &vlag[1], beta, denom, knew, &w[1]);
    ih = 0;
    double pqold = pq[knew];
    pq[knew] = 0.0;
    for (int i = 1; i <= n; ++i) {
      double temp = pqold * xpt[ix(knew, i)];
      for (int j = 1; j <= i; ++j) {
        ++ih;
        hq[ih] += temp * xpt[ix(knew, j)];
      }
    }
    for (int jj = 1; jj <= nptm; ++jj) {
      double temp = diff * zmat[iz(knew, jj)];
      for (int k = 1; k <= npt; ++k) pq[k] += temp * zmat[iz(k, jj)];
    }
    fval[knew] = f;
    for (int i = 1; i <= n; ++i) {
      xpt[ix(knew, i)] = xnew[i];
      w[i] = bmat[ib(knew, i)];
    }
    for (int k = 1; k <= npt; ++k) {
      double suma = 0.0;
      for (int jj = 1; jj <= nptm; ++jj) suma += zmat[iz(knew, jj)] * zmat[iz(k, jj)];
      if (std::isinf(suma)) {
        rc_ = BobyqaStatus::RoundoffLimited;
        goto L720;
      }
      double sumb = 0.0;
      for (int j = 1; j <= n; ++j) sumb += xpt[ix(k, j)] * xopt[j];
      double temp = suma * sumb;
      for (int i = 1; i <= n; ++i) w[i] += temp * xpt[ix(k, i)];
    }
    for (int i = 1; i <= n; ++i) gopt[i] += diff * w[i];
    if (f < fopt) {
      kopt = knew;
      xoptsq = 0.0;
      ih = 0;
      for (int j = 1; j <= n; ++j) {
        xopt[j] = xnew[j];
        xoptsq += xopt[j] * xopt[j];
        for (int i = 1; i <= j; ++i) {
          ++ih;
          if (i < j) gopt[j] += hq[ih] * d[i];
          gopt[i] += hq[ih] * d[j];
        }
      }
      for (int k = 1; k <= npt; ++k) {
        double temp = 0.0;
        for (int j = 1; j <= n; ++j) temp += xpt[ix(k, j)] * d[j];
        temp *= pq[k];
        for (int i = 1; i <= n; ++i) gopt[i] += temp * xpt[ix(k, i)];
      }
    }
    if (ntrits > 0) {
      for (int k = 1; k <= npt; ++k) {
        vlag[k] = fval[k] - fval[kopt];
        w[k] = 0.0;
      }
      for (int j = 1; j <= nptm; ++j) {
        double sum = 0.0;
        for (int k = 1; k <= npt; ++k) sum += zmat[iz(k, j)] * vlag[k];
        for (int k = 1; k <= npt; ++k) w[k] += sum * zmat[iz(k, j)];
      }
      for (int k = 1; k <= npt; ++k) {
        double sum = 0.0;
        for (int j = 1; j <= n; ++j) sum += xpt[ix(k, j)] * xopt[j];
        w[k + npt] = w[k];
        w[k] *= sum;
      }
      double gqsq = 0.0, gisq = 0.0;
      for (int i = 1; i <= n; ++i) {
        double sum = 0.0;
        for (int k = 1; k <= npt; ++k) sum = sum + bmat[ib(k, i)] * vlag[k] + xpt[ix(k, i)] * w[k];
        if (xopt[i] == sl[i]) {
          double a = std::min(0.0, gopt[i]);
          gqsq += a * a;
          double b = std::min(0.0, sum);
          gisq += b * b;
        } else if (xopt[i] == su[i]) {
          double a = std::max(0.0, gopt[i]);
          gqsq += a * a;
          double b = std::max(0.0, sum);
          gisq += b * b;
        } else {
          gqsq += gopt[i] * gopt[i];
          gisq += sum * sum;
        }
        vlag[npt + i] = sum;
      }
      ++itest;
      if (gqsq < 10.0 * gisq) itest = 0;
      if (itest >= 3) {
        for (int i = 1; i <= std::max(npt, nh); ++i) {
          if (i <= n) gopt[i] = vlag[npt + i];
          if (i <= npt) pq[i] = w[npt + i];
          if (i <= nh) hq[i] = 0.0;
          itest = 0;
        }
      }
    }
    if (ntrits == 0) goto L60;
    if (f <= fopt + 0.1 * vquad) goto L60;
    double a = 2.0 * delta, b = 10.0 * rho;
    distsq = std::max(a * a, b * b);
  }

L650:
  knew = 0;
  for (int k = 1; k <= npt; ++k) {
    double sum = 0.0;
    for (int j = 1; j <= n; ++j) {
      double v = xpt[ix(k, j)] - xopt[j];
      sum += v * v;
    }
    if (sum > distsq) {
      knew = k;
      distsq = sum;
    }
  }
  if (knew > 0) {
    double dist = std::sqrt(distsq);
    if (ntrits == -1) {
      delta = std::min(0.1 * delta, 0.5 * dist);
      if (delta <= rho * 1.5) delta = rho;
    }
    ntrits = 0;
    adelt = std::max(std::min(0.1 * dist, delta), rho);
    dsq = adelt * adelt;
    goto L90;
  }
  if (ntrits == -1) goto L680;
  if (ratio > 0.0) goto L60;
  if (std::max(delta, dnorm) > rho) goto L60;

L680:
  if (rho > rhoend_) {
    delta = 0.5 * rho;
    ratio = rho / rhoend_;
    if (ratio <= 16.0) {
      rho = rhoend_;
    } else if (ratio <= 250.0) {
      rho = std::sqrt(ratio) * rhoend_;
    } else {
      rho *= 0.1;
    }
    delta = std::max(delta, rho);
    ntrits = 0;
    nfsav = nevals_;
    goto L60;
  }
  if (ntrits == -1) goto L360;

L720:
  for (int i = 1; i <= n; ++i) {
    x_[i] = std::min(std::max(xl_[i], xbase[i] + xopt[i]), xu_[i]);
    if (xopt[i] == sl[i]) x_[i] = xl_[i];
    if (xopt[i] == su[i]) x_[i] = xu_[i];
  }
  minf_ = fval[kopt];
  xbest_ = x_;
  if (rc_ == BobyqaStatus::Running) rc_ = BobyqaStatus::Success;
  (void)fsave;
  co_return;
}

}  // namespace nebula
