/*
 * detmath.h -- bit-reproducible, nearly correctly rounded exp, log, sin and
 * cos for host and device.
 *
 * The finite-depth Green function accelerates its eigenfunction series with
 * the Wynn epsilon algorithm, which extrapolates from differences of nearly
 * equal partial sums and stops on exact equalities.  One unit in the last
 * place of a sin/cos/exp/log result moves the extrapolated value by up to
 * 1e-3 for some panel pairs.  The series terms therefore use these functions:
 *   - every step is an IEEE add, multiply, divide or explicit fused
 *     multiply-add, so the CPU and the GPU produce the same bits;
 *   - the result is evaluated in double-double (error-free transforms built
 *     on fma) to about 100 bits and rounded once, so it is the correctly
 *     rounded value except when the exact result lies within ~2^-100 of a
 *     rounding boundary -- the same bits a correctly rounding math library
 *     (as the reference's compilers ship) returns.
 *
 * Methods (W.J. Cody & W. Waite, "Software Manual for the Elementary
 * Functions", 1980; T.J. Dekker 1971 for the double-double arithmetic):
 * additive range reduction by ln 2 or pi/2 split into short-mantissa parts,
 * Taylor polynomials on the reduced interval with the leading terms in
 * double-double; log uses 2 atanh(s), s = (m-1)/(m+1), m in [sqrt(1/2),
 * sqrt(2)).  Constants are ln 2, pi/2, 1/n! and 1/(2k+1) rounded from
 * 300-bit values.  Valid for |x| < 1e5 (sin/cos) and normal results (exp).
 */
#ifndef HAMS_DETMATH_H
#define HAMS_DETMATH_H

#include <math.h>

#if defined(__CUDACC__)
#define DM_FN __host__ __device__ __forceinline__
#else
#define DM_FN static inline
#endif

#define DM_LN2_HI 0.6931471806019545        /* ln 2: 32-bit head ...           */
#define DM_LN2_MID (-4.2009150726810846e-11) /* ... 53-bit middle ...            */
#define DM_LN2_LO (-1.3124698417785255e-27)  /* ... and tail                     */
#define DM_INV_LN2 1.4426950408889634
#define DM_PIO2_1 1.5707963267341256         /* pi/2: two 33-bit parts ...       */
#define DM_PIO2_2 6.077100506303966e-11
#define DM_PIO2_3 2.0222662487959506e-21     /* ... and a 53-bit tail            */
#define DM_TWO_OVER_PI 0.6366197723675814
#define DM_SQRT1_2 0.7071067811865476

typedef struct {
  double hi, lo;
} dm_dd;

DM_FN dm_dd dm_mk(double h, double l) {
  dm_dd r;
  r.hi = h;
  r.lo = l;
  return r;
}
/* a + b exactly, |a| >= |b| */
DM_FN dm_dd dm_fast2sum(double a, double b) {
  double s = a + b;
  return dm_mk(s, b - (s - a));
}
/* a + b exactly */
DM_FN dm_dd dm_2sum(double a, double b) {
  double s = a + b, bb = s - a;
  return dm_mk(s, (a - (s - bb)) + (b - bb));
}
/* a * b exactly */
DM_FN dm_dd dm_2prod(double a, double b) {
  double p = a * b;
  return dm_mk(p, fma(a, b, -p));
}
DM_FN dm_dd dm_ddmul(dm_dd a, dm_dd b) {
  dm_dd p = dm_2prod(a.hi, b.hi);
  double e = p.lo + (a.hi * b.lo + a.lo * b.hi);
  return dm_2sum(p.hi, e);
}
DM_FN dm_dd dm_ddadd(dm_dd a, dm_dd b) {
  dm_dd s = dm_2sum(a.hi, b.hi);
  double e = s.lo + (a.lo + b.lo);
  return dm_2sum(s.hi, e);
}

/* exp(x): x = k ln2 + r, |r| <= ln2/2; exp(r) by Taylor to r^17, terms up to
 * r^7 in double-double. */
DM_FN double dm_exp(double x) {
  if (x != x) return x;
  if (x > 709.78) return HUGE_VAL;
  if (x < -745.2) return 0.0;
  double k = floor(x * DM_INV_LN2 + 0.5);
  dm_dd r = dm_2sum(x - k * DM_LN2_HI, -(k * DM_LN2_MID));
  r.lo = r.lo - k * DM_LN2_LO;
  double t = 2.8114572543455206e-15; /* 1/17! */
  t = fma(t, r.hi, 4.779477332387385e-14);
  t = fma(t, r.hi, 7.647163731819816e-13);
  t = fma(t, r.hi, 1.1470745597729725e-11);
  t = fma(t, r.hi, 1.6059043836821613e-10);
  t = fma(t, r.hi, 2.08767569878681e-09);
  t = fma(t, r.hi, 2.505210838544172e-08);
  t = fma(t, r.hi, 2.755731922398589e-07);
  t = fma(t, r.hi, 2.7557319223985893e-06);
  t = fma(t, r.hi, 2.48015873015873e-05); /* 1/8! */
  dm_dd y = dm_mk(t, 0.0);
  y = dm_ddadd(dm_ddmul(y, r), dm_mk(0.0001984126984126984, 1.7209558293420705e-22));
  y = dm_ddadd(dm_ddmul(y, r), dm_mk(0.001388888888888889, -5.300543954373577e-20));
  y = dm_ddadd(dm_ddmul(y, r), dm_mk(0.008333333333333333, 1.1564823173178714e-19));
  y = dm_ddadd(dm_ddmul(y, r), dm_mk(0.041666666666666664, 2.3129646346357427e-18));
  y = dm_ddadd(dm_ddmul(y, r), dm_mk(0.16666666666666666, 9.25185853854297e-18));
  y = dm_ddadd(dm_ddmul(y, r), dm_mk(0.5, 0.0));
  y = dm_ddadd(dm_ddmul(y, r), dm_mk(1.0, 0.0));
  y = dm_ddadd(dm_ddmul(y, r), dm_mk(1.0, 0.0));
  return ldexp(y.hi, (int)k);
}

/* log(x), x > 0 finite: x = m 2^e, log m = 2 s (1 + s^2/3 + s^4/5 + ...),
 * s = (m-1)/(m+1) in double-double. */
DM_FN double dm_log(double x) {
  if (!(x > 0.0)) return x == 0.0 ? -HUGE_VAL : (x - x) / (x - x);
  if (x == HUGE_VAL) return x;
  int e;
  double m = frexp(x, &e); /* m in [0.5, 1) */
  if (m < DM_SQRT1_2) {
    m = m * 2.0;
    e = e - 1;
  }
  double num = m - 1.0; /* exact */
  dm_dd den = dm_2sum(m, 1.0);
  double sh = num / den.hi;
  double sl = (fma(-sh, den.hi, num) - sh * den.lo) / den.hi;
  dm_dd s = dm_2sum(sh, sl);
  dm_dd z = dm_ddmul(s, s);
  double q = 0.04; /* 1/25 */
  q = fma(q, z.hi, 0.043478260869565216);
  q = fma(q, z.hi, 0.047619047619047616);
  q = fma(q, z.hi, 0.05263157894736842);
  q = fma(q, z.hi, 0.058823529411764705);
  q = fma(q, z.hi, 0.06666666666666667);
  q = fma(q, z.hi, 0.07692307692307693);
  q = fma(q, z.hi, 0.09090909090909091);
  q = fma(q, z.hi, 0.1111111111111111); /* 1/9 */
  dm_dd y = dm_mk(q, 0.0);
  y = dm_ddadd(dm_ddmul(y, z), dm_mk(0.14285714285714285, 7.93016446160826e-18));
  y = dm_ddadd(dm_ddmul(y, z), dm_mk(0.2, -1.1102230246251566e-17));
  y = dm_ddadd(dm_ddmul(y, z), dm_mk(0.3333333333333333, 1.850371707708594e-17));
  y = dm_ddadd(dm_ddmul(y, z), dm_mk(1.0, 0.0));
  y = dm_ddmul(y, s);
  y = dm_mk(2.0 * y.hi, 2.0 * y.lo);
  double de = (double)e;
  dm_dd el = dm_2sum(de * DM_LN2_HI, de * DM_LN2_MID);
  el.lo = el.lo + de * DM_LN2_LO;
  return dm_ddadd(el, y).hi;
}

/* sin and cos of x: x = k pi/2 + r with r in double-double, |r| <= pi/4,
 * then the Taylor series of sin r and cos r with the leading terms in
 * double-double, and the quadrant of k. */
DM_FN void dm_sincos(double x, double* sp, double* cp) {
  double k = floor(x * DM_TWO_OVER_PI + 0.5);
  dm_dd r = dm_2sum(x - k * DM_PIO2_1, -(k * DM_PIO2_2));
  r = dm_2sum(r.hi, r.lo - k * DM_PIO2_3);
  dm_dd z = dm_ddmul(r, r);
  /* sin r = r * sum (-1)^j z^j / (2j+1)! */
  double t = -1.9572941063391263e-20; /* -1/21! */
  t = fma(t, z.hi, 8.22063524662433e-18);
  t = fma(t, z.hi, -2.8114572543455206e-15);
  t = fma(t, z.hi, 7.647163731819816e-13);
  t = fma(t, z.hi, -1.6059043836821613e-10);
  t = fma(t, z.hi, 2.505210838544172e-08);
  t = fma(t, z.hi, -2.7557319223985893e-06);
  t = fma(t, z.hi, 0.0001984126984126984); /* 1/7! with its sign: coefficient of z^3 is -1/7! */
  dm_dd ys = dm_mk(-t, 0.0);
  ys = dm_ddadd(dm_ddmul(ys, z), dm_mk(0.008333333333333333, 1.1564823173178714e-19));
  ys = dm_ddadd(dm_ddmul(ys, z), dm_mk(-0.16666666666666666, -9.25185853854297e-18));
  ys = dm_ddadd(dm_ddmul(ys, z), dm_mk(1.0, 0.0));
  ys = dm_ddmul(ys, r);
  /* cos r = sum (-1)^j z^j / (2j)! */
  double u = 8.896791392450574e-22; /* 1/22! */
  u = fma(u, z.hi, -4.110317623312165e-19);
  u = fma(u, z.hi, 1.5619206968586225e-16);
  u = fma(u, z.hi, -4.779477332387385e-14);
  u = fma(u, z.hi, 1.1470745597729725e-11);
  u = fma(u, z.hi, -2.08767569878681e-09);
  u = fma(u, z.hi, 2.755731922398589e-07);
  u = fma(u, z.hi, -2.48015873015873e-05);
  u = fma(u, z.hi, 0.001388888888888889); /* coefficient of z^3 is -1/6! */
  dm_dd yc = dm_mk(-u, 0.0);
  yc = dm_ddadd(dm_ddmul(yc, z), dm_mk(0.041666666666666664, 2.3129646346357427e-18));
  yc = dm_ddadd(dm_ddmul(yc, z), dm_mk(-0.5, 0.0));
  yc = dm_ddadd(dm_ddmul(yc, z), dm_mk(1.0, 0.0));
  double sr = ys.hi, cr = yc.hi;
  long long q = (long long)k & 3;
  if (q == 0) {
    *sp = sr;
    *cp = cr;
  } else if (q == 1) {
    *sp = cr;
    *cp = -sr;
  } else if (q == 2) {
    *sp = -sr;
    *cp = -cr;
  } else {
    *sp = -cr;
    *cp = sr;
  }
}

DM_FN double dm_sin(double x) {
  double s, c;
  dm_sincos(x, &s, &c);
  return s;
}

DM_FN double dm_cos(double x) {
  double s, c;
  dm_sincos(x, &s, &c);
  return c;
}

#endif
