/*
 * special.c -- special functions of the finite-depth Green function.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle_internal.h).
 *
 * Restates src/FinGrnExtSubs.f90 of HAMS-MREL: erf (ERROR), the exponential
 * integrals E_n, E_1, Ei (ENXA, E1XA, EIX), the Wynn-epsilon series limit
 * (Limes, T. Mishonov & E. Penev 2000), the modified Bessel functions K0/K1
 * (IK01A) and the Bessel functions J0/J1/Y0/Y1 (JY01B and its derived
 * variants).  The series/polynomial methods are the published ones of
 * S. Zhang & J. Jin, "Computation of Special Functions", Wiley 1996.
 */
#include "oracle_internal.h"
#include "detmath.h"

/* Fortran x**n for an integer exponent (binary powering). */
static double powi(double x, int n)
{
    double r = 1.0, b = x;
    int e = n < 0 ? -n : n;
    while (e) {
        if (e & 1) r *= b;
        b *= b;
        e >>= 1;
    }
    return n < 0 ? 1.0 / r : r;
}

/* ERROR, FinGrnExtSubs.f90:62-96 */
void orc_error(double x, double *err)
{
    const double eps = 1.0e-15, pi = 3.141592653589793;
    double x2 = x * x, er, r, c0;
    int k;
    if (fabs(x) < 3.5) {
        er = 1.0;
        r = 1.0;
        for (k = 1; k <= 50; ++k) {
            r = r * x2 / (k + 0.5);
            er = er + r;
            if (fabs(r) <= fabs(er) * eps) break;
        }
        c0 = 2.0 / sqrt(pi) * x * exp(-x2);
        *err = c0 * er;
    } else {
        er = 1.0;
        r = 1.0;
        for (k = 1; k <= 12; ++k) {
            r = -r * (k - 0.5) / x2;
            er = er + r;
        }
        c0 = exp(-x2) / (fabs(x) * sqrt(pi));
        *err = 1.0 - c0 * er;
        if (x < 0.0) *err = -*err;
    }
}

/* E1XA, FinGrnExtSubs.f90:198-214 */
void orc_e1xa(double x, double *e1)
{
    if (x == 0.0) {
        *e1 = 1.0e300;
    } else if (x <= 1.0) {
        *e1 = -log(x) +
              ((((1.07857e-3 * x - 9.76004e-3) * x + 5.519968e-2) * x - 0.24991055) * x +
               0.99999193) * x - 0.57721566;
    } else {
        double es1 = (((x + 8.5733287401) * x + 18.059016973) * x + 8.6347608925) * x + 0.2677737343;
        double es2 = (((x + 9.5733223454) * x + 25.6329561486) * x + 21.0996530827) * x + 3.9584969228;
        *e1 = exp(-x) / x * es1 / es2;
    }
}

/* ENXA, FinGrnExtSubs.f90:135-157 */
void orc_enxa(int n, double x, double *en)
{
    double e0 = exp(-x) / x, e1;
    int k;
    orc_e1xa(x, &e1);
    if (n == 0) {
        *en = e0;
    } else if (n == 1) {
        *en = e1;
    } else {
        for (k = 2; k <= n; ++k) {
            *en = (exp(-x) - x * e1) / (k - 1.0);
            e1 = *en;
        }
    }
}

/* EIX, FinGrnExtSubs.f90:254-285 */
void orc_eix(double x, double *ei)
{
    int k;
    double r;
    if (x == 0.0) {
        *ei = -1.0e300;
    } else if (x <= 40.0) {
        *ei = 1.0;
        r = 1.0;
        for (k = 1; k <= 100; ++k) {
            r = r * k * x / ((k + 1.0) * (k + 1.0));
            *ei = *ei + r;
            if (fabs(r / *ei) <= 1.0e-15) break;
        }
        *ei = 0.5772156649015328 + log(x) + x * *ei;
    } else {
        *ei = 1.0;
        r = 1.0;
        for (k = 1; k <= 20; ++k) {
            r = r * k / x;
            *ei = *ei + r;
        }
        *ei = exp(x) / x * *ei;
    }
}

/*
 * Limes, FinGrnExtSubs.f90:370-470: limit of a sequence of partial sums by
 * the epsilon algorithm.  s[0..n] is overwritten, exactly as the Fortran
 * INOUT argument.
 */
void orc_limes(int n, double *s, double *rlimes, int *ipade, int *kpade, double *err)
{
    double a[ORC_NK + 1];
    double amax = 0.0;
    int i, k;
    *rlimes = s[n];
    *err = fabs(s[n] - s[n - 1]);
    *ipade = n;
    *kpade = 0;
    for (i = 0; i <= n; ++i) a[i] = 0.0;
    k = 1;
    for (;;) {
        if (n - 2 * k + 1 < 0) break;
        for (i = 0; i <= n - 2 * k + 1; ++i) {
            if (s[i + 1] != s[i]) a[i] = a[i + 1] + 1.0 / (s[i + 1] - s[i]);
            else a[i] = a[i + 1];
        }
        if (n - 2 * k < 0) break;
        for (i = 0; i <= n - 2 * k; ++i) {
            if (a[i + 1] != a[i]) s[i] = s[i + 1] + 1.0 / (a[i + 1] - a[i]);
            else s[i] = s[i + 1];
            if (fabs(a[i]) > amax) {
                amax = fabs(a[i]);
                *rlimes = s[i];
                *kpade = k;
                *ipade = i + k;
                *err = 1.0 / amax;
                if (s[i + 1] == s[i]) return;
            }
        }
        k = k + 1;
    }
}

/*
 * IK01A, FinGrnExtSubs.f90:538-635: K0(x), K1(x) for x >= 0.  Its exp and
 * log are the bit-reproducible ones of detmath.h, shared with the GPU code:
 * K0/K1 feed the epsilon-accelerated series, which amplifies last-bit
 * differences of the math library.
 * The reference reads WW before assigning it on the first pass of the K0
 * series (FinGrnExtSubs.f90:608); it is taken as 0 here, which cannot stop
 * the series on its first term.
 */
void orc_ik01a(double x, double *bk0, double *bk1)
{
    static const double A[12] = {0.125, 7.03125e-2, 7.32421875e-2, 1.1215209960938e-1,
                                 2.2710800170898e-1, 5.7250142097473e-1, 1.7277275025845,
                                 6.0740420012735, 2.4380529699556e01, 1.1001714026925e02,
                                 5.5133589612202e02, 3.0380905109224e03};
    static const double B[12] = {-0.375, -1.171875e-1, -1.025390625e-1, -1.4419555664063e-1,
                                 -2.7757644653320e-1, -6.7659258842468e-1, -1.9935317337513,
                                 -6.8839142681099, -2.7248827311269e01, -1.2159789187654e02,
                                 -6.0384407670507e02, -3.3022722944809e03};
    static const double A1[8] = {0.125, 0.2109375, 1.0986328125, 1.1775970458984e01,
                                 2.1461706161499e02, 5.9511522710323e03, 2.3347645606175e05,
                                 1.2312234987631e07};
    const double pi = 3.141592653589793, el = 0.5772156649015329;
    double x2 = x * x, bi0, bi1, r, ca, xr, ct, w0, ww = 0.0, cb, xr2;
    int k, k0;
    if (x == 0.0) {
        *bk0 = 1.0e300;
        *bk1 = 1.0e300;
        return;
    } else if (x <= 18.0) {
        bi0 = 1.0;
        r = 1.0;
        for (k = 1; k <= 50; ++k) {
            r = 0.25 * r * x2 / (double)(k * k);
            bi0 = bi0 + r;
            if (fabs(r / bi0) < 1.0e-15) break;
        }
        bi1 = 1.0;
        r = 1.0;
        for (k = 1; k <= 50; ++k) {
            r = 0.25 * r * x2 / (double)(k * (k + 1));
            bi1 = bi1 + r;
            if (fabs(r / bi1) < 1.0e-15) break;
        }
        bi1 = 0.5 * x * bi1;
    } else {
        k0 = 12;
        if (x >= 35.0) k0 = 9;
        if (x >= 50.0) k0 = 7;
        ca = dm_exp(x) / sqrt(2.0 * pi * x);
        bi0 = 1.0;
        xr = 1.0 / x;
        for (k = 1; k <= k0; ++k) bi0 = bi0 + A[k - 1] * powi(xr, k);
        bi0 = ca * bi0;
        bi1 = 1.0;
        for (k = 1; k <= k0; ++k) bi1 = bi1 + B[k - 1] * powi(xr, k);
        bi1 = ca * bi1;
    }
    if (x <= 9.0) {
        ct = -(dm_log(x / 2.0) + el);
        *bk0 = 0.0;
        w0 = 0.0;
        r = 1.0;
        for (k = 1; k <= 50; ++k) {
            w0 = w0 + 1.0 / k;
            r = 0.25 * r / (double)(k * k) * x2;
            *bk0 = *bk0 + r * (w0 + ct);
            if (fabs((*bk0 - ww) / *bk0) < 1.0e-15) break;
            ww = *bk0;
        }
        *bk0 = *bk0 + ct;
    } else {
        cb = 0.5 / x;
        xr2 = 1.0 / x2;
        *bk0 = 1.0;
        for (k = 1; k <= 8; ++k) *bk0 = *bk0 + A1[k - 1] * powi(xr2, k);
        *bk0 = cb * *bk0 / bi0;
    }
    *bk1 = (1.0 / x - bi1 * *bk0) / bi0;
}

/* Polynomial pieces shared by JY01B and its derived variants,
 * FinGrnExtSubs.f90:673-735.  The Y0 coefficient 1.0766115157 carries no
 * D exponent in the reference (:683) and is therefore single precision. */
static double jy_j0_small(double t2)
{
    return ((((((-.5014415e-3 * t2 + .76771853e-2) * t2 - .0709253492) * t2 + .4443584263) * t2 -
              1.7777560599) * t2 + 3.9999973021) * t2 - 3.9999998721) * t2 + 1.0;
}
static double jy_j1_small(double t, double t2)
{
    return t * (((((((-.1289769e-3 * t2 + .22069155e-2) * t2 - .0236616773) * t2 + .1777582922) * t2 -
                   .8888839649) * t2 + 2.6666660544) * t2 - 3.9999999710) * t2 + 1.9999999998);
}
static double jy_y0_small(double t2)
{
    return (((((((-.567433e-4 * t2 + .859977e-3) * t2 - .94855882e-2) * t2 + .0772975809) * t2 -
               .4261737419) * t2 + 1.4216421221) * t2 - 2.3498519931) * t2 + F4(1.0766115157)) * t2 +
           .3674669052;
}
static double jy_y1_small(double x, double t2)
{
    return ((((((((.6535773e-3 * t2 - .0108175626) * t2 + .107657606) * t2 - .7268945577) * t2 +
                3.1261399273) * t2 - 7.3980241381) * t2 + 6.8529236342) * t2 + .3932562018) * t2 -
            .6366197726) / x;
}
static void jy_pq0(double t, double t2, double *p0, double *q0)
{
    *p0 = ((((-.9285e-5 * t2 + .43506e-4) * t2 - .122226e-3) * t2 + .434725e-3) * t2 - .4394275e-2) * t2 +
          .999999997;
    *q0 = t * (((((.8099e-5 * t2 - .35614e-4) * t2 + .85844e-4) * t2 - .218024e-3) * t2 + .1144106e-2) * t2 -
               .031249995);
}
static void jy_pq1(double t, double t2, double *p1, double *q1)
{
    *p1 = ((((.10632e-4 * t2 - .50363e-4) * t2 + .145575e-3) * t2 - .559487e-3) * t2 + .7323931e-2) * t2 +
          1.000000004;
    *q1 = t * (((((-.9173e-5 * t2 + .40658e-4) * t2 - .99941e-4) * t2 + .266891e-3) * t2 - .1601836e-2) * t2 +
               .093749994);
}

/* JY01B, FinGrnExtSubs.f90:663-703 */
void orc_jy01b(double x, double *bj0, double *bj1, double *by0, double *by1)
{
    const double pi = 3.141592653589793;
    if (x == 0.0) {
        *bj0 = 1.0;
        *bj1 = 0.0;
        *by0 = -1.0e300;
        *by1 = -1.0e300;
        return;
    } else if (x <= 4.0) {
        double t = x / 4.0, t2 = t * t;
        *bj0 = jy_j0_small(t2);
        *bj1 = jy_j1_small(t, t2);
        *by0 = jy_y0_small(t2);
        *by0 = 2.0 / pi * log(x / 2.0) * *bj0 + *by0;
        *by1 = jy_y1_small(x, t2);
        *by1 = 2.0 / pi * log(x / 2.0) * *bj1 + *by1;
    } else {
        double t = 4.0 / x, t2 = t * t, a0 = sqrt(2.0 / (pi * x)), p0, q0, p1, q1, ta0, ta1;
        jy_pq0(t, t2, &p0, &q0);
        ta0 = x - .25 * pi;
        *bj0 = a0 * (p0 * cos(ta0) - q0 * sin(ta0));
        *by0 = a0 * (p0 * sin(ta0) + q0 * cos(ta0));
        jy_pq1(t, t2, &p1, &q1);
        ta1 = x - .75 * pi;
        *bj1 = a0 * (p1 * cos(ta1) - q1 * sin(ta1));
        *by1 = a0 * (p1 * sin(ta1) + q1 * cos(ta1));
    }
}

/* JY01BJ, FinGrnExtSubs.f90:741-772 */
void orc_jy01bj(double x, double *bj0, double *bj1)
{
    const double pi = 3.141592653589793;
    if (x == 0.0) {
        *bj0 = 1.0;
        *bj1 = 0.0;
    } else if (x <= 4.0) {
        double t = x / 4.0, t2 = t * t;
        *bj0 = jy_j0_small(t2);
        *bj1 = jy_j1_small(t, t2);
    } else {
        double t = 4.0 / x, t2 = t * t, a0 = sqrt(2.0 / (pi * x)), p0, q0, p1, q1, ta0, ta1;
        jy_pq0(t, t2, &p0, &q0);
        ta0 = x - .25 * pi;
        *bj0 = a0 * (p0 * cos(ta0) - q0 * sin(ta0));
        jy_pq1(t, t2, &p1, &q1);
        ta1 = x - .75 * pi;
        *bj1 = a0 * (p1 * cos(ta1) - q1 * sin(ta1));
    }
}

/* JY01BY0, FinGrnExtSubs.f90:811-840 */
void orc_jy01by0(double x, double *by0)
{
    const double pi = 3.141592653589793;
    if (x == 0.0) {
        *by0 = -1.0e300;
    } else if (x <= 4.0) {
        double t = x / 4.0, t2 = t * t, bj0 = jy_j0_small(t2);
        *by0 = jy_y0_small(t2);
        *by0 = 2.0 / pi * log(x / 2.0) * bj0 + *by0;
    } else {
        double t = 4.0 / x, t2 = t * t, a0 = sqrt(2.0 / (pi * x)), p0, q0, ta0;
        jy_pq0(t, t2, &p0, &q0);
        ta0 = x - .25 * pi;
        *by0 = a0 * (p0 * sin(ta0) + q0 * cos(ta0));
    }
}

/* JY01BY1, FinGrnExtSubs.f90:875-903 */
void orc_jy01by1(double x, double *by1)
{
    const double pi = 3.141592653589793;
    if (x == 0.0) {
        *by1 = -1.0e300;
    } else if (x <= 4.0) {
        double t = x / 4.0, t2 = t * t, bj1 = jy_j1_small(t, t2);
        *by1 = jy_y1_small(x, t2);
        *by1 = 2.0 / pi * log(x / 2.0) * bj1 + *by1;
    } else {
        double t = 4.0 / x, t2 = t * t, a0 = sqrt(2.0 / (pi * x)), p1, q1, ta1;
        jy_pq1(t, t2, &p1, &q1);
        ta1 = x - .75 * pi;
        *by1 = a0 * (p1 * sin(ta1) + q1 * cos(ta1));
    }
}
