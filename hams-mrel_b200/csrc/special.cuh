// special.cuh -- FP64 device special functions of the free-surface Green functions.
//
// Same series and polynomial methods as HAMS-MREL's src/FinGrnExtSubs.f90
// (S. Zhang & J. Jin, "Computation of Special Functions", Wiley 1996):
// erf by its Taylor / asymptotic series (ERROR, :62), E1 by the rational fit
// (E1XA, :198), E_n by forward recurrence (ENXA, :135), Ei (EIX, :254),
// K0/K1 from the I0/I1 and K0 series or the large-argument expansions
// (IK01A, :538), J0/J1/Y0/Y1 from the 4/x polynomial fits (JY01B, :663).
// Thresholds written as single-precision literals in the reference are kept
// as the float value promoted to double (F4), so branch decisions agree.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "detmath.h"

#define HAMS_F4(x) ((double)(x##f))

namespace hams {

__device__ __forceinline__ double powi(double x, int n) {
  double r = 1.0, b = x;
  int e = n < 0 ? -n : n;
  while (e) {
    if (e & 1) r *= b;
    b *= b;
    e >>= 1;
  }
  return n < 0 ? 1.0 / r : r;
}

// erf(x), ERROR (FinGrnExtSubs.f90:62-96)
__device__ inline double erf_zj(double x) {
  const double eps = 1.0e-15, sqpi = 1.7724538509055159;  // sqrt(pi)
  double x2 = x * x;
  if (fabs(x) < 3.5) {
    double er = 1.0, r = 1.0;
    for (int k = 1; k <= 50; ++k) {
      r = r * x2 / (k + 0.5);
      er = er + r;
      if (fabs(r) <= fabs(er) * eps) break;
    }
    return 2.0 / sqpi * x * exp(-x2) * er;
  }
  double er = 1.0, r = 1.0;
  for (int k = 1; k <= 12; ++k) {
    r = -r * (k - 0.5) / x2;
    er = er + r;
  }
  double e = 1.0 - exp(-x2) / (fabs(x) * sqpi) * er;
  return x < 0.0 ? -e : e;
}

__device__ __forceinline__ double erfc_zj(double x) { return 1.0 - erf_zj(x); }
__device__ __forceinline__ double derfc_zj(double x) { return -2.0 / 1.7724538509055159 * exp(-(x * x)); }

// E1(x), E1XA (FinGrnExtSubs.f90:198-214)
__device__ inline double e1xa(double x) {
  if (x == 0.0) return 1.0e300;
  if (x <= 1.0)
    return -log(x) + ((((1.07857e-3 * x - 9.76004e-3) * x + 5.519968e-2) * x - 0.24991055) * x + 0.99999193) * x -
           0.57721566;
  double es1 = (((x + 8.5733287401) * x + 18.059016973) * x + 8.6347608925) * x + 0.2677737343;
  double es2 = (((x + 9.5733223454) * x + 25.6329561486) * x + 21.0996530827) * x + 3.9584969228;
  return exp(-x) / x * es1 / es2;
}

// E_n(x), ENXA (FinGrnExtSubs.f90:135-157)
__device__ inline double enxa(int n, double x) {
  double e1 = e1xa(x);
  if (n == 0) return exp(-x) / x;
  if (n == 1) return e1;
  double en = e1, ex = exp(-x);
  for (int k = 2; k <= n; ++k) {
    en = (ex - x * e1) / (k - 1.0);
    e1 = en;
  }
  return en;
}

// Ei(x), EIX (FinGrnExtSubs.f90:254-285)
__device__ inline double eix(double x) {
  if (x == 0.0) return -1.0e300;
  if (x <= 40.0) {
    double ei = 1.0, r = 1.0;
    for (int k = 1; k <= 100; ++k) {
      r = r * k * x / ((k + 1.0) * (k + 1.0));
      ei = ei + r;
      if (fabs(r / ei) <= 1.0e-15) break;
    }
    return 0.5772156649015328 + log(x) + x * ei;
  }
  double ei = 1.0, r = 1.0;
  for (int k = 1; k <= 20; ++k) {
    r = r * k / x;
    ei = ei + r;
  }
  return exp(x) / x * ei;
}

// fl(|num / den|) < 1e-15, the convergence test of the IK01A series, with
// the IEEE division taken only when the quotient lies within 1e-9 (relative)
// of the threshold.  Outside that band the product of |den| with the widened
// threshold, rounded once (relative error 2^-53), decides the same way the
// correctly rounded quotient would.  NaN, zero or extreme |den| fall back to
// the division.
__device__ __forceinline__ bool quot_below_1em15(double num, double den) {
  double an = fabs(num), ad = fabs(den);
  if (ad > 1e-280 && ad < 1e280) {
    if (an < (1.0e-15 * (1.0 - 1e-9)) * ad) return true;
    if (an > (1.0e-15 * (1.0 + 1e-9)) * ad) return false;
  }
  return fabs(num / den) < 1.0e-15;
}

// The same test for a positive partial sum den >= 1 and a positive term num
// (the I0 and I1 series): no range checks, and the common "not yet" outcome
// costs one product and one comparison.
__device__ __forceinline__ bool term_below_1em15(double num, double den) {
  if (num > (1.0e-15 * (1.0 + 1e-9)) * den) return false;
  if (num < (1.0e-15 * (1.0 - 1e-9)) * den) return true;
  return fabs(num / den) < 1.0e-15;
}

// 1.0 / k, k*k and k*(k+1) for k = 0..50 as doubles, rounded at compile time
// exactly as the run-time division and integer conversion.
struct SeriesConsts {
  double recip[51], kk[51], kk1[51];
  constexpr SeriesConsts() : recip{}, kk{}, kk1{} {
    for (int k = 1; k <= 50; ++k) {
      recip[k] = 1.0 / k;
      kk[k] = (double)(k * k);
      kk1[k] = (double)(k * (k + 1));
    }
  }
};
static __constant__ SeriesConsts c_series = SeriesConsts();

// K0(x), K1(x), IK01A (FinGrnExtSubs.f90:538-635).  K0/K1 feed the
// epsilon-accelerated series, whose result moves with the last bit of its
// inputs, so this routine uses the bit-reproducible exp/log of detmath.h and
// the operation order of the CPU checker; the kernels that call it for the
// EIGENE/PIDCOCK series are compiled without implicit fused multiply-adds.
// The reference compares the K0 series against a value it never initialised
// on the first pass; zero is used, which cannot stop the series early.
__device__ inline void ik01a(double x, double& bk0, double& bk1) {
  const double pi = 3.141592653589793, el = 0.5772156649015329;
  if (x == 0.0) {
    bk0 = 1.0e300;
    bk1 = 1.0e300;
    return;
  }
  double x2 = x * x, bi0, bi1, r;
  if (x <= 18.0) {
    bi0 = 1.0;
    r = 1.0;
    // r > 0 and bi0, bi1 >= 1 for x > 0 (a NaN x fails every comparison and
    // reaches the division, as in the reference)
    for (int k = 1; k <= 50; ++k) {
      r = 0.25 * r * x2 / c_series.kk[k];
      bi0 = bi0 + r;
      if (term_below_1em15(r, bi0)) break;
    }
    bi1 = 1.0;
    r = 1.0;
    for (int k = 1; k <= 50; ++k) {
      r = 0.25 * r * x2 / c_series.kk1[k];
      bi1 = bi1 + r;
      if (term_below_1em15(r, bi1)) break;
    }
    bi1 = 0.5 * x * bi1;
  } else {
    const double A[12] = {0.125, 7.03125e-2, 7.32421875e-2, 1.1215209960938e-1, 2.2710800170898e-1,
                          5.7250142097473e-1, 1.7277275025845, 6.0740420012735, 2.4380529699556e01,
                          1.1001714026925e02, 5.5133589612202e02, 3.0380905109224e03};
    const double B[12] = {-0.375, -1.171875e-1, -1.025390625e-1, -1.4419555664063e-1, -2.7757644653320e-1,
                          -6.7659258842468e-1, -1.9935317337513, -6.8839142681099, -2.7248827311269e01,
                          -1.2159789187654e02, -6.0384407670507e02, -3.3022722944809e03};
    int k0 = 12;
    if (x >= 35.0) k0 = 9;
    if (x >= 50.0) k0 = 7;
    double ca = dm_exp(x) / sqrt(2.0 * pi * x), xr = 1.0 / x;
    bi0 = 1.0;
    for (int k = 1; k <= k0; ++k) bi0 = bi0 + A[k - 1] * powi(xr, k);
    bi0 = ca * bi0;
    bi1 = 1.0;
    for (int k = 1; k <= k0; ++k) bi1 = bi1 + B[k - 1] * powi(xr, k);
    bi1 = ca * bi1;
  }
  if (x <= 9.0) {
    double ct = -(dm_log(x / 2.0) + el), w0 = 0.0, ww = 0.0;
    r = 1.0;
    bk0 = 0.0;
    for (int k = 1; k <= 50; ++k) {
      w0 = w0 + c_series.recip[k];
      r = 0.25 * r / c_series.kk[k] * x2;
      bk0 = bk0 + r * (w0 + ct);
      if (quot_below_1em15(bk0 - ww, bk0)) break;
      ww = bk0;
    }
    bk0 = bk0 + ct;
  } else {
    const double A1[8] = {0.125, 0.2109375, 1.0986328125, 1.1775970458984e01, 2.1461706161499e02,
                          5.9511522710323e03, 2.3347645606175e05, 1.2312234987631e07};
    double cb = 0.5 / x, xr2 = 1.0 / x2;
    bk0 = 1.0;
    for (int k = 1; k <= 8; ++k) bk0 = bk0 + A1[k - 1] * powi(xr2, k);
    bk0 = cb * bk0 / bi0;
  }
  bk1 = (1.0 / x - bi1 * bk0) / bi0;
}

// JY01B polynomial pieces (FinGrnExtSubs.f90:673-735); the 1.0766115157
// coefficient of Y0 is a single-precision literal in the reference (:683).
__device__ __forceinline__ double jy_j0s(double t2) {
  return ((((((-.5014415e-3 * t2 + .76771853e-2) * t2 - .0709253492) * t2 + .4443584263) * t2 - 1.7777560599) * t2 +
           3.9999973021) * t2 - 3.9999998721) * t2 + 1.0;
}
__device__ __forceinline__ double jy_j1s(double t, double t2) {
  return t * (((((((-.1289769e-3 * t2 + .22069155e-2) * t2 - .0236616773) * t2 + .1777582922) * t2 - .8888839649) *
                   t2 + 2.6666660544) * t2 - 3.9999999710) * t2 + 1.9999999998);
}
__device__ __forceinline__ double jy_y0s(double t2) {
  return (((((((-.567433e-4 * t2 + .859977e-3) * t2 - .94855882e-2) * t2 + .0772975809) * t2 - .4261737419) * t2 +
            1.4216421221) * t2 - 2.3498519931) * t2 + HAMS_F4(1.0766115157)) * t2 + .3674669052;
}
__device__ __forceinline__ double jy_y1s(double x, double t2) {
  return ((((((((.6535773e-3 * t2 - .0108175626) * t2 + .107657606) * t2 - .7268945577) * t2 + 3.1261399273) * t2 -
              7.3980241381) * t2 + 6.8529236342) * t2 + .3932562018) * t2 - .6366197726) / x;
}
__device__ __forceinline__ void jy_pq0(double t, double t2, double& p0, double& q0) {
  p0 = ((((-.9285e-5 * t2 + .43506e-4) * t2 - .122226e-3) * t2 + .434725e-3) * t2 - .4394275e-2) * t2 + .999999997;
  q0 = t * (((((.8099e-5 * t2 - .35614e-4) * t2 + .85844e-4) * t2 - .218024e-3) * t2 + .1144106e-2) * t2 - .031249995);
}
__device__ __forceinline__ void jy_pq1(double t, double t2, double& p1, double& q1) {
  p1 = ((((.10632e-4 * t2 - .50363e-4) * t2 + .145575e-3) * t2 - .559487e-3) * t2 + .7323931e-2) * t2 + 1.000000004;
  q1 = t * (((((-.9173e-5 * t2 + .40658e-4) * t2 - .99941e-4) * t2 + .266891e-3) * t2 - .1601836e-2) * t2 +
            .093749994);
}

// J0, J1, Y0, Y1 (JY01B, FinGrnExtSubs.f90:663-703)
__device__ inline void jy01b(double x, double& bj0, double& bj1, double& by0, double& by1) {
  const double pi = 3.141592653589793;
  if (x == 0.0) {
    bj0 = 1.0;
    bj1 = 0.0;
    by0 = -1.0e300;
    by1 = -1.0e300;
    return;
  }
  if (x <= 4.0) {
    double t = x / 4.0, t2 = t * t, lg = 2.0 / pi * log(x / 2.0);
    bj0 = jy_j0s(t2);
    bj1 = jy_j1s(t, t2);
    by0 = lg * bj0 + jy_y0s(t2);
    by1 = lg * bj1 + jy_y1s(x, t2);
    return;
  }
  double t = 4.0 / x, t2 = t * t, a0 = sqrt(2.0 / (pi * x)), p0, q0, p1, q1, s0, c0, s1, c1;
  jy_pq0(t, t2, p0, q0);
  jy_pq1(t, t2, p1, q1);
  sincos(x - .25 * pi, &s0, &c0);
  sincos(x - .75 * pi, &s1, &c1);
  bj0 = a0 * (p0 * c0 - q0 * s0);
  by0 = a0 * (p0 * s0 + q0 * c0);
  bj1 = a0 * (p1 * c1 - q1 * s1);
  by1 = a0 * (p1 * s1 + q1 * c1);
}

}  // namespace hams
