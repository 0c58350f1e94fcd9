/*
 * fingreen.c -- finite-depth free-surface Green function and derivatives.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle_internal.h).
 *
 * Restates src/FinGreen3D.f90 of HAMS-MREL (Y. Liu et al., "FinGreen3D",
 * Computer Physics Communications 2016): the region decomposition on R/h
 * into the LINTON (R/h < 0.0005), PIDCOCK (< 0.05), EIGENE (< 0.5) and EIGEN
 * branches, the Wynn-epsilon accelerated eigenfunction series, the image
 * sums of Pidcock, and Linton's Ewald-type representation with its adaptive
 * Gauss-Kronrod (7/15) quadratures.  Recursion is kept recursive here, in
 * the order of the reference (left half, then right half).
 * The sin/cos of the eigenfunction series terms (EIGEN, EIGENE, PIDCOCK) are
 * the bit-reproducible ones of detmath.h: the epsilon extrapolation of those
 * series turns one-ulp differences between math libraries into differences
 * of up to 1e-3 in single values, so the checker and the GPU code share one
 * implementation of them.
 */
#include "oracle_internal.h"
#include "detmath.h"

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

static const zdouble CI = I;

/* ---------------------------------------------------------------- */
/* EIGEN, FinGreen3D.f90:281-362 (R/h >= 0.5, at most 10 terms)      */
/* ---------------------------------------------------------------- */
static void eigen(double r, double zf, double zp, double wk, const double *wvn, int nk,
                  double h, zdouble grn[3])
{
    const double pi = 3.141592653589793;
    int i, nt = 10;
    double j0, j1, y0, y1, k0, k1, km, pm, rm[3];
    double zfh = zf + h, zph = zp + h, twokmh, kzf, kzp, ckzf, ckzp, skzf;
    double sr, sr1, dsrr, dsrz, dsr1r, dsr1z;
    zdouble nm0, p0, dp0;
    (void)nk;

    nm0 = h / 2.0 * (1.0 + sinh(2.0 * wk * h) / (2.0 * wk * h));
    p0 = pi / nm0 * cosh(wk * zfh) * cosh(wk * zph);
    dp0 = pi / nm0 * sinh(wk * zfh) * cosh(wk * zph);

    orc_jy01b(wk * r, &j0, &j1, &y0, &y1);
    grn[0] = p0 * (CI * j0 - y0);
    grn[1] = -wk * p0 * (CI * j1 - y1);
    grn[2] = wk * dp0 * (CI * j0 - y0);

    for (i = 2; i <= nt; ++i) {
        km = wvn[i - 1];
        twokmh = 2.0 * km * h;
        pm = 4.0 / (1.0 + dm_sin(twokmh) / twokmh) / h;
        orc_ik01a(km * r, &k0, &k1);
        kzf = km * zfh;
        kzp = km * zph;
        ckzf = dm_cos(kzf);
        ckzp = dm_cos(kzp);
        skzf = dm_sin(kzf);
        rm[0] = pm * k0 * ckzf * ckzp;
        rm[1] = -pm * km * k1 * ckzf * ckzp;
        rm[2] = -pm * km * k0 * skzf * ckzp;
        grn[0] += rm[0];
        grn[1] += rm[1];
        grn[2] += rm[2];
        if (fabs(rm[0]) < F4(1.E-6) && fabs(rm[1]) < F4(1.E-6) && fabs(rm[2]) < F4(1.E-6)) break;
    }

    sr = sqrt(r * r + (zf - zp) * (zf - zp));
    sr1 = sqrt(r * r + (zf + zp) * (zf + zp));
    dsrr = r / sr;
    dsrz = (zf - zp) / sr;
    dsr1r = r / sr1;
    dsr1z = (zf + zp) / sr1;
    grn[0] = grn[0] - (1.0 / sr + 1.0 / sr1);
    grn[1] = grn[1] + (dsrr / (sr * sr) + dsr1r / (sr1 * sr1));
    grn[2] = grn[2] + (dsrz / (sr * sr) + dsr1z / (sr1 * sr1));
}

/* ---------------------------------------------------------------- */
/* EIGENE, FinGreen3D.f90:413-506 (0.05 <= R/h < 0.5, epsilon algo) */
/* ---------------------------------------------------------------- */
static void eigene(double r, double zf, double zp, double wk, const double *wvn, int nk,
                   double h, zdouble grn[3])
{
    const double pi = 3.141592653589793;
    int i, nt, ip, kp;
    double j0, j1, y0, y1, k0, k1, km, pm, rm[3], rl[3], err, rhp;
    double g[ORC_NK], gr[ORC_NK], gz[ORC_NK];
    double zfh = zf + h, zph = zp + h, twokmh, kzf, kzp, ckzf, ckzp, skzf;
    double sr, sr1, dsrr, dsrz, dsr1r, dsr1z;
    zdouble nm0, p0, dp0;
    (void)nk;

    rhp = fabs(r / h);
    nt = (int)(F4(-88.89) * rhp + F4(54.45));

    nm0 = h / 2.0 * (1.0 + sinh(2.0 * wk * h) / (2.0 * wk * h));
    p0 = pi / nm0 * cosh(wk * zfh) * cosh(wk * zph);
    dp0 = pi / nm0 * sinh(wk * zfh) * cosh(wk * zph);

    orc_jy01b(wk * r, &j0, &j1, &y0, &y1);
    grn[0] = p0 * (CI * j0 - y0);
    grn[1] = -wk * p0 * (CI * j1 - y1);
    grn[2] = wk * dp0 * (CI * j0 - y0);

    g[0] = 0.0;
    gr[0] = 0.0;
    gz[0] = 0.0;
    for (i = 2; i <= nt; ++i) {
        km = wvn[i - 1];
        twokmh = 2.0 * km * h;
        pm = 4.0 / (1.0 + dm_sin(twokmh) / twokmh) / h;
        orc_ik01a(km * r, &k0, &k1);
        kzf = km * zfh;
        kzp = km * zph;
        ckzf = dm_cos(kzf);
        ckzp = dm_cos(kzp);
        skzf = dm_sin(kzf);
        rm[0] = pm * k0 * ckzf * ckzp;
        rm[1] = -pm * km * k1 * ckzf * ckzp;
        rm[2] = -pm * km * k0 * skzf * ckzp;
        g[i - 1] = g[i - 2] + rm[0];
        gr[i - 1] = gr[i - 2] + rm[1];
        gz[i - 1] = gz[i - 2] + rm[2];
    }
    orc_limes(nt - 1, g, &rl[0], &ip, &kp, &err);
    orc_limes(nt - 1, gr, &rl[1], &ip, &kp, &err);
    orc_limes(nt - 1, gz, &rl[2], &ip, &kp, &err);
    grn[0] += rl[0];
    grn[1] += rl[1];
    grn[2] += rl[2];

    sr = sqrt(r * r + (zf - zp) * (zf - zp));
    sr1 = sqrt(r * r + (zf + zp) * (zf + zp));
    dsrr = r / sr;
    dsrz = (zf - zp) / sr;
    dsr1r = r / sr1;
    dsr1z = (zf + zp) / sr1;
    grn[0] = grn[0] - (1.0 / sr + 1.0 / sr1);
    grn[1] = grn[1] + (dsrr / (sr * sr) + dsr1r / (sr1 * sr1));
    grn[2] = grn[2] + (dsrz / (sr * sr) + dsr1z / (sr1 * sr1));
}

/* ---------------------------------------------------------------- */
/* Pidcock image sums IMGS/DGSR/DGSZ, FinGreen3D.f90:908-1113       */
/* ---------------------------------------------------------------- */
/* AMN(0:4,0:4) in Fortran column order: AMN(m,n) = AMN_[m + 5 n]. */
static const double AMN_[25] = {
    0.0, -0.02525711, 0.00086546, -0.00004063, 0.00000193,
    0.05051418, -0.00692380, 0.00073292, -0.00006636, 0.00000398,
    0.00230838, -0.00097875, 0.00020597, -0.00003333, 0.00000524,
    0.00012934, -0.00010879, 0.00003965, -0.00000891, 0.0,
    0.00000913, -0.00001270, 0.00000466, 0.0, 0.0};
#define AMN(m, n) AMN_[(m) + 5 * (n)]

static double rs(double r, double z) { return sqrt(r * r + z * z); }

static double imgs(double r, double zf, double zp, double h)
{
    double t1 = r / h, t2 = (zf - zp) / h, t3 = (zf + zp + 2.0 * h) / h, sum1 = 0.0, sum2 = 0.0;
    int l, m, n;
    for (l = -1; l <= 1; ++l) sum1 = sum1 + 1.0 / rs(t1, t2 + 2.0 * l) + 1.0 / rs(t1, t3 + 2.0 * l);
    for (m = 0; m <= 4; ++m)
        for (n = 0; n <= 4; ++n)
            sum2 = sum2 + AMN(m, n) * pow(t1, 2.0 * m) * (pow(t2, 2.0 * n) + pow(t3, 2.0 * n));
    return (sum1 - 2.0 + sum2) / h;
}

static double dgsr(double r, double zf, double zp, double h)
{
    double t1 = r / h, t2 = (zf - zp) / h, t3 = (zf + zp + 2.0 * h) / h, sum1 = 0.0, sum2 = 0.0;
    int l, m, n;
    for (l = -1; l <= 1; ++l)
        sum1 = sum1 + t1 / powi(rs(t1, t2 + 2.0 * l), 3) + t1 / powi(rs(t1, t3 + 2.0 * l), 3);
    for (m = 1; m <= 4; ++m)
        for (n = 0; n <= 4; ++n)
            sum2 = sum2 + 2.0 * m * AMN(m, n) * pow(t1, 2.0 * m - 1.0) *
                              (pow(t2, 2.0 * n) + pow(t3, 2.0 * n));
    return (-sum1 + sum2) / (h * h);
}

static double dgsz(double r, double zf, double zp, double h)
{
    double t1 = r / h, t2 = (zf - zp) / h, t3 = (zf + zp + 2.0 * h) / h, sum1 = 0.0, sum2 = 0.0;
    int l, m, n;
    for (l = -1; l <= 1; ++l)
        sum1 = sum1 + (t2 + 2.0 * l) / powi(rs(t1, t2 + 2.0 * l), 3) +
               (t3 + 2.0 * l) / powi(rs(t1, t3 + 2.0 * l), 3);
    for (m = 0; m <= 4; ++m)
        for (n = 1; n <= 4; ++n)
            sum2 = sum2 + 2.0 * n * AMN(m, n) * pow(t1, 2.0 * m) *
                              (pow(t2, 2.0 * n - 1.0) + pow(t3, 2.0 * n - 1.0));
    return (-sum1 + sum2) / (h * h);
}

/* ---------------------------------------------------------------- */
/* PIDCOCK, FinGreen3D.f90:558-660 (0.0005 <= R/h < 0.05)            */
/* ---------------------------------------------------------------- */
static void pidcock(double r, double zf, double zp, double v, double wk, const double *wvn,
                    int nk, double h, zdouble grn[3])
{
    const double pi = 3.141592653589793, ga = 0.5772156649015328;
    int nt, i, ip, kp;
    double j0, j1, y0, y1, k0, k0t, k1, k1t, nm0, p0, dp0, x;
    double rm[3], sm[3], rl[3], err, rhp, um, umt, mp, ac, am, amt, dam, damt;
    double sr, sr1, dsrr, dsrz, dsr1r, dsr1z;
    double g[ORC_NK], gr[ORC_NK], gz[ORC_NK];
    (void)nk;

    nm0 = h / 2.0 * (1.0 + sinh(2.0 * wk * h) / (2.0 * wk * h));
    p0 = pi / nm0 * cosh(wk * (zf + h)) * cosh(wk * (zp + h));
    dp0 = wk * pi / nm0 * sinh(wk * (zf + h)) * cosh(wk * (zp + h));

    orc_jy01b(wk * r, &j0, &j1, &y0, &y1);
    grn[0] = p0 * (CI * j0 - y0) + 2.0 / h * (ga + log(r / 4.0 / h));
    grn[1] = -wk * p0 * (CI * j1 - y1) + 2.0 / (r * h);
    grn[2] = dp0 * (CI * j0 - y0);

    rhp = fabs(r / h);
    nt = (int)(F4(-1010.10) * rhp + F4(100.50));

    g[0] = 0.0;
    gr[0] = 0.0;
    gz[0] = 0.0;
    for (i = 2; i <= nt; ++i) {
        mp = (i - 1) * pi;
        umt = mp / h;
        um = wvn[i - 1];
        x = um * r;
        orc_ik01a(x, &k0, &k1);
        orc_ik01a(umt * r, &k0t, &k1t);
        ac = (um * um + v * v) / ((um * um + v * v) * h - v);
        am = ac * dm_cos(um * (zf + h)) * dm_cos(um * (zp + h));
        amt = dm_cos(umt * (zf + h)) * dm_cos(umt * (zp + h)) / h;
        dam = -um * ac * dm_sin(um * (zf + h)) * dm_cos(um * (zp + h));
        damt = -umt * dm_sin(umt * (zf + h)) * dm_cos(umt * (zp + h)) / h;
        rm[0] = am * k0 - amt * k0t;
        rm[1] = -um * am * k1 + umt * amt * k1t;
        rm[2] = dam * k0 - damt * k0t;
        g[i - 1] = g[i - 2] + rm[0];
        gr[i - 1] = gr[i - 2] + rm[1];
        gz[i - 1] = gz[i - 2] + rm[2];
    }
    orc_limes(nt - 1, g, &rl[0], &ip, &kp, &err);
    orc_limes(nt - 1, gr, &rl[1], &ip, &kp, &err);
    orc_limes(nt - 1, gz, &rl[2], &ip, &kp, &err);
    sm[0] = 4.0 * rl[0];
    sm[1] = 4.0 * rl[1];
    sm[2] = 4.0 * rl[2];
    grn[0] = grn[0] + sm[0] + imgs(r, zf, zp, h);
    grn[1] = grn[1] + sm[1] + dgsr(r, zf, zp, h);
    grn[2] = grn[2] + sm[2] + dgsz(r, zf, zp, h);

    sr = sqrt(r * r + (zf - zp) * (zf - zp));
    sr1 = sqrt(r * r + (zf + zp) * (zf + zp));
    dsrr = r / sr;
    dsrz = (zf - zp) / sr;
    dsr1r = r / sr1;
    dsr1z = (zf + zp) / sr1;
    grn[0] = grn[0] - (1.0 / sr + 1.0 / sr1);
    grn[1] = grn[1] + (dsrr / (sr * sr) + dsr1r / (sr1 * sr1));
    grn[2] = grn[2] + (dsrz / (sr * sr) + dsr1z / (sr1 * sr1));
}

/* ---------------------------------------------------------------- */
/* LINTON support: FinGreen3D.f90:1168-2748                          */
/* ---------------------------------------------------------------- */
static void chi(double zf, double zp, double h, double val[4])
{
    val[0] = -zp - zf;
    val[1] = 2.0 * h - zp + zf;
    val[2] = 2.0 * h + zp - zf;
    val[3] = 4.0 * h + zp + zf;
}
static const double DVAL[4] = {-1.0, 1.0, -1.0, 1.0}; /* DCHI, :2261 */

static void rchi(double r, double zf, double zp, double h, double ro[4], double dror[4], double droz[4])
{
    double val[4];
    int i;
    chi(zf, zp, h, val);
    for (i = 1; i <= 4; ++i) {
        ro[i - 1] = sqrt(r * r + val[i - 1] * val[i - 1]);
        dror[i - 1] = r / sqrt(r * r + val[i - 1] * val[i - 1]);
        droz[i - 1] = val[i - 1] * ((i & 1) ? -1.0 : 1.0) / sqrt(r * r + val[i - 1] * val[i - 1]);
    }
}

static zdouble nmf(double h, zdouble wvn) /* NM, :2280 */
{
    return h / 2.0 * (1.0 + csin(2.0 * wvn * h) / (2.0 * wvn * h));
}

static double derfcc(double x) /* DERFCC, :2295 */
{
    const double pi = 3.141592653589793;
    return -2.0 / sqrt(pi) * exp(-pow(x, 2.0));
}

static double erfcc(double x) /* ERFCC, :2313 */
{
    double err;
    orc_error(x, &err);
    return 1.0 - err;
}

static double f1(double r, double wvn, int no, double t) /* F1, :1882 */
{
    const double pi = 3.141592653589793;
    if (fabs(t) < 1.0e-8) return 0.0;
    if (no == 1) return exp(-(r * r) / 4.0 / t + wvn * wvn * t) / 4.0 / pi / t;
    return exp(-(r * r) / 4.0 / t - wvn * wvn * t) / 4.0 / pi / t;
}

static double f2(double r, double wvn, int no, double t) /* F2, :1957 */
{
    const double pi = 3.141592653589793;
    if (fabs(t) < 1.0e-8) return 0.0;
    if (no == 1) return -r * exp(-(r * r) / 4.0 / t + wvn * wvn * t) / 8.0 / pi / (t * t);
    return -r * exp(-(r * r) / 4.0 / t - wvn * wvn * t) / 8.0 / pi / (t * t);
}

static double g1(double v, double r, double zf, double zp, double h, double t) /* G1, :2033 */
{
    double sum = 0.0, val[4];
    int i;
    if (fabs(t) < 1.0e-8) return 0.0;
    chi(zf, zp, h, val);
    for (i = 0; i < 4; ++i) sum = sum + exp(-v * val[i]) * erfcc(val[i] / 2.0 / t - v * t);
    return exp(v * v * (t * t) - (r * r) / 4.0 / (t * t)) * sum / t;
}

static double g2(double v, double r, double zf, double zp, double h, double t) /* G2, :2106 */
{
    double sum = 0.0, val[4];
    int i;
    if (fabs(t) < 1.0e-8) return 0.0;
    chi(zf, zp, h, val);
    for (i = 0; i < 4; ++i) sum = sum + exp(-v * val[i]) * erfcc(val[i] / 2.0 / t - v * t);
    return r / 2.0 / (t * t * t) * exp(v * v * (t * t) - (r * r) / 4.0 / (t * t)) * sum;
}

static double g3(double v, double r, double zf, double zp, double h, double t) /* G3, :2180 */
{
    double sum = 0.0, val[4];
    int i;
    if (fabs(t) < 1.0e-8) return 0.0;
    chi(zf, zp, h, val);
    for (i = 0; i < 4; ++i)
        sum = sum - v * DVAL[i] * exp(-v * val[i]) * erfcc(val[i] / 2.0 / t - v * t) +
              exp(-v * val[i]) * derfcc(val[i] / 2.0 / t - v * t) * DVAL[i] / 2.0 / t;
    return exp(v * v * (t * t) - (r * r) / 4.0 / (t * t)) * sum / t;
}

static double funf(double v, double r, double zf, double zp, double h, double t, int tag)
{
    if (tag == 1) return g1(v, r, zf, zp, h, t);
    if (tag == 2) return g2(v, r, zf, zp, h, t);
    return g3(v, r, zf, zp, h, t);
}

static double fun(double r, double wvn, int no, double t, int tag)
{
    return tag == 1 ? f1(r, wvn, no, t) : f2(r, wvn, no, t);
}

/* Gauss-Kronrod 7/15 nodes and weights, FinGreen3D.f90:2395-2427 */
static const double XGQ[7] = {-0.949107912342759, -0.741531185599394, -0.405845151377397, 0.0,
                              0.405845151377397, 0.741531185599394, 0.949107912342759};
static const double WGQ[7] = {0.129484966168870, 0.279705391489277, 0.381830050505119,
                              0.417959183673469, 0.381830050505119, 0.279705391489277,
                              0.129484966168870};
static const double XKQ[15] = {-0.991455371120813, -0.949107912342759, -0.864864423359769,
                               -0.741531185599394, -0.586087235467691, -0.405845151377397,
                               -0.207784955007898, 0.0, 0.207784955007898, 0.405845151377397,
                               0.586087235467691, 0.741531185599394, 0.864864423359769,
                               0.949107912342759, 0.991455371120813};
static const double WKQ[15] = {0.022935322010529, 0.063092092629979, 0.104790010322250,
                               0.140653259715525, 0.169004726639267, 0.190350578064785,
                               0.204432940075298, 0.209482141084728, 0.204432940075298,
                               0.190350578064785, 0.169004726639267, 0.140653259715525,
                               0.104790010322250, 0.063092092629979, 0.022935322010529};

/* GK_INTEGF, :2387 */
static void gk_integf(double v, double r, double zf, double zp, double h, double a, double b,
                      double *gk, double *err, int tag)
{
    double stf[7], gi = 0.0;
    int i;
    for (i = 0; i < 7; ++i) {
        stf[i] = funf(v, r, zf, zp, h, 0.5 * (b + a + (b - a) * XGQ[i]), tag);
        gi = gi + WGQ[i] * (b - a) / 2.0 * stf[i];
    }
    *gk = 0.0;
    for (i = 1; i <= 15; ++i) {
        if (i % 2 == 0) *gk = *gk + WKQ[i - 1] * (b - a) / 2.0 * stf[i / 2 - 1];
        else *gk = *gk + WKQ[i - 1] * (b - a) / 2.0 * funf(v, r, zf, zp, h, 0.5 * (b + a + (b - a) * XKQ[i - 1]), tag);
    }
    *err = pow(200.0 * fabs(*gk - gi), 1.5);
}

/* AQUADF, :2515 */
static double aquadf(double v, double r, double zf, double zp, double h, double a, double b,
                     double eps, int tag)
{
    double gk, err;
    gk_integf(v, r, zf, zp, h, a, b, &gk, &err, tag);
    if (err > eps && fabs(a - b) > eps)
        return aquadf(v, r, zf, zp, h, a, (a + b) / 2.0, eps, tag) +
               aquadf(v, r, zf, zp, h, (a + b) / 2.0, b, eps, tag);
    return gk;
}

/* GK_INTEG, :2599 */
static void gk_integ(double r, double wvn, int no, double a, double b, double *gk, double *err, int tag)
{
    double stf[7], gi = 0.0;
    int i;
    for (i = 0; i < 7; ++i) {
        stf[i] = fun(r, wvn, no, 0.5 * (b + a + (b - a) * XGQ[i]), tag);
        gi = gi + WGQ[i] * (b - a) / 2.0 * stf[i];
    }
    *gk = 0.0;
    for (i = 1; i <= 15; ++i) {
        if (i % 2 == 0) *gk = *gk + WKQ[i - 1] * (b - a) / 2.0 * stf[i / 2 - 1];
        else *gk = *gk + WKQ[i - 1] * (b - a) / 2.0 * fun(r, wvn, no, 0.5 * (b + a + (b - a) * XKQ[i - 1]), tag);
    }
    *err = pow(200.0 * fabs(*gk - gi), 1.5);
}

/* AQUAD, :2728 */
static double aquad(double r, double wvn, int no, double a, double b, double eps, int tag)
{
    double gk, err;
    gk_integ(r, wvn, no, a, b, &gk, &err, tag);
    if (err > eps && fabs(a - b) > eps)
        return aquad(r, wvn, no, a, (a + b) / 2.0, eps, tag) + aquad(r, wvn, no, (a + b) / 2.0, b, eps, tag);
    return gk;
}

/* SA0, :1389 */
static double sa0(double r, double pa, double wk)
{
    const double ga = 0.5772156649015328, pi = 3.141592653589793, eps = F4(1.E-6);
    int n = 1, p;
    double s, rm = 100.0, en, psi, sgn = -1.0, facn = 1.0;
    s = -ga - 2.0 * log(wk * pa / 2.0);
    while (fabs(rm) > eps) {
        orc_enxa(n + 1, (r / pa) * (r / pa), &en);
        psi = 0.0;
        for (p = 1; p <= n; ++p) psi = psi + 1.0 / p;
        rm = sgn * pow(r / pa, 2.0 * n) / facn / n - pow(wk * pa / 2.0, 2.0 * n) / facn * en -
             2.0 * sgn / (facn * facn) * pow(wk * r / 2.0, 2.0 * n) * (log(wk * r / 2.0) + ga - psi);
        s = s + rm;
        n = n + 1;
        sgn = -sgn;
        facn = facn * n;
    }
    return s / 4.0 / pi;
}

/* DSA0, :1483 */
static double dsa0(double r, double pa, double wk)
{
    const double ga = 0.5772156649015328, pi = 3.141592653589793, eps = F4(1.E-6);
    int n = 1, p;
    double s = 0.0, rm = 100.0, en, psi, sgn = -1.0, facn = 1.0;
    while (fabs(rm) > eps) {
        orc_enxa(n, (r / pa) * (r / pa), &en);
        psi = 0.0;
        for (p = 1; p <= n; ++p) psi = psi + 1.0 / p;
        rm = 2.0 * sgn * pow(r / pa, 2.0 * n - 1.0) / facn / pa +
             pow(wk * pa / 2.0, 2.0 * n) / facn * en * 2.0 * r / (pa * pa) -
             2.0 * sgn * n * wk / (facn * facn) * pow(wk * r / 2.0, 2.0 * n - 1.0) * (log(wk * r / 2.0) + ga - psi) -
             2.0 * sgn / (facn * facn) * pow(wk * r / 2.0, 2.0 * n) / r;
        s = s + rm;
        n = n + 1;
        sgn = -sgn;
        facn = facn * n;
    }
    return s / 4.0 / pi;
}

/* SAM, :1575 */
static double sam(double r, double pa, double wvn)
{
    const double pi = 3.141592653589793, eps = F4(1.E-6);
    int n = 0;
    double s = 0.0, rm = 100.0, en, sgn = 1.0, facn = 1.0;
    while (fabs(rm) > eps) {
        orc_enxa(n + 1, (wvn * pa / 2.0) * (wvn * pa / 2.0), &en);
        rm = sgn * pow(r / pa, 2.0 * n) / facn * en;
        s = s + rm;
        n = n + 1;
        sgn = -sgn;
        facn = facn * n;
    }
    return s / 4.0 / pi;
}

/* DSAM, :1659 */
static double dsam(double r, double pa, double wvn)
{
    const double pi = 3.141592653589793, eps = F4(1.E-6);
    int n = 1;
    double s = 0.0, rm = 100.0, en, sgn = -1.0, facn = 1.0;
    while (fabs(rm) > eps) {
        orc_enxa(n + 1, (wvn * pa / 2.0) * (wvn * pa / 2.0), &en);
        rm = 2.0 * n * sgn * pow(r / pa, 2.0 * n - 1.0) / facn / pa * en;
        s = s + rm;
        n = n + 1;
        sgn = -sgn;
        facn = facn * n;
    }
    return s / 4.0 / pi;
}

/* COEF, :1168 */
static void coef(double r, double pa, double a, int m, const double *wvno, double wk, double *cof)
{
    const double pi = 3.141592653589793, eps = F4(1.E-6), step = 100.0;
    double dnt = pa * pa / 4.0, by0, p1, e1, ei;
    int i;
    if (fabs(r) < F4(1.E-6)) {
        orc_eix(wk * wk * dnt, &ei);
        cof[0] = -ei / 4.0 / pi;
    } else if (r / a <= 0.5) {
        cof[0] = sa0(r, pa, wk);
    } else {
        orc_jy01by0(wk * r, &by0);
        cof[0] = -by0 / 4.0 - aquad(r, wk, 1, 0.0, dnt, eps, 1);
    }
    for (i = 2; i <= m; ++i) {
        if (fabs(r) < F4(1.E-6)) {
            orc_e1xa(wvno[i - 1] * wvno[i - 1] * dnt, &e1);
            cof[i - 1] = e1 / 4.0 / pi;
        } else if (r / a <= 1.0) {
            cof[i - 1] = sam(r, pa, wvno[i - 1]);
        } else {
            p1 = dnt + step;
            while (fabs(f1(r, wvno[i - 1], i, p1)) > eps) p1 = p1 + step;
            cof[i - 1] = aquad(r, wvno[i - 1], i, dnt, p1, eps, 1);
        }
    }
}

/* DCOEF, :1281 */
static void dcoef(double r, double pa, double a, int m, const double *wvno, double wk, double *dcof)
{
    const double eps = F4(1.E-6), step = 100.0;
    double dnt = pa * pa / 4.0, by1, p1;
    int i;
    if (fabs(r) < F4(1.E-6)) {
        dcof[0] = 0.0;
    } else if (r / a <= 0.5) {
        dcof[0] = dsa0(r, pa, wk);
    } else {
        orc_jy01by1(wk * r, &by1);
        dcof[0] = wk * by1 / 4.0 - aquad(r, wk, 1, 0.0, dnt, eps, 2);
    }
    for (i = 2; i <= m; ++i) {
        if (fabs(r) < F4(1.E-6)) {
            dcof[i - 1] = 0.0;
        } else if (r / a <= 1.0) {
            dcof[i - 1] = dsam(r, pa, wvno[i - 1]);
        } else {
            p1 = dnt + step;
            while (fabs(f2(r, wvno[i - 1], i, p1)) > eps) p1 = p1 + step;
            dcof[i - 1] = aquad(r, wvno[i - 1], i, dnt, p1, eps, 2);
        }
    }
}

/* ---------------------------------------------------------------- */
/* LINTON, FinGreen3D.f90:712-861 (R/h < 0.0005)                     */
/* ---------------------------------------------------------------- */
static void linton(double r, double zf, double zp, double v, double wk, const double *wvno, int nk,
                   double h, zdouble grn[3])
{
    const double pi = 3.141592653589793, eps = F4(1.E-6);
    int nt, i;
    double pa, a, sr, sr1, sr2, dsrr, dsrz, dsr1r, dsr1z, dsr2r, dsr2z;
    double ro[4], dror[4], droz[4], errsum[3], bj0, bj1;
    double cof[ORC_NK], dcof[ORC_NK];
    zdouble km, rmv[3];
    (void)nk;

    if (v < 0.02) a = 3324.2 * powi(v, 3) - 258.89 * (v * v) + 8.3958 * v + 1.3208;
    else if (v < 0.1) a = -30.303 * powi(v, 3) - 2.8138 * (v * v) + 2.7740 * v + 0.05052;
    else if (v < 1.0) a = 1.5699 * powi(v, 3) - 2.5075 * (v * v) + 1.8316 * v + 0.1077;
    else a = -0.000069641 * powi(v, 3) - 0.0017082 * (v * v) + 0.45566 * v + 0.80551;
    a = fabs(a) / (wk * h);

    pa = a * h;
    sr = sqrt(r * r + (zf - zp) * (zf - zp));
    sr1 = sqrt(r * r + (2.0 * h + zf + zp) * (2.0 * h + zf + zp));
    sr2 = sqrt(r * r + (zf + zp) * (zf + zp));
    rchi(r, zf, zp, h, ro, dror, droz);
    dsrr = r / sr;
    dsrz = (zf - zp) / sr;
    dsr1r = r / sr1;
    dsr1z = (2.0 * h + zf + zp) / sr1;
    dsr2r = r / sr2;
    dsr2z = (zf + zp) / sr2;

    grn[0] = grn[1] = grn[2] = 0.0;
    nt = 20;
    coef(r, pa, a, nt, wvno, wk, cof);
    dcoef(r, pa, a, nt, wvno, wk, dcof);
    for (i = 1; i <= nt; ++i) {
        zdouble nmk, c1, c2;
        km = (i == 1) ? -CI * wk : (zdouble)wvno[i - 1];
        nmk = nmf(h, km);
        c1 = ccos(km * (zf + h));
        c2 = ccos(km * (zp + h));
        rmv[0] = -(cof[i - 1] / nmk * c1 * c2);
        rmv[1] = -(dcof[i - 1] / nmk * c1 * c2);
        rmv[2] = cof[i - 1] * km / nmk * csin(km * (zf + h)) * c2;
        grn[0] += rmv[0];
        grn[1] += rmv[1];
        grn[2] += rmv[2];
        if (i > 2 && cabs(rmv[0]) < eps && cabs(rmv[1]) < eps && cabs(rmv[2]) < eps) break;
    }

    errsum[0] = errsum[1] = errsum[2] = 0.0;
    for (i = 0; i < 4; ++i) {
        errsum[0] = errsum[0] + erfcc(ro[i] / pa) / (4.0 * pi * ro[i]);
        errsum[1] = errsum[1] + (derfcc(ro[i] / pa) / pa * dror[i] * ro[i] - dror[i] * erfcc(ro[i] / pa)) /
                                    (4.0 * pi * (ro[i] * ro[i]));
        errsum[2] = errsum[2] + (derfcc(ro[i] / pa) / pa * droz[i] * ro[i] - droz[i] * erfcc(ro[i] / pa)) /
                                    (4.0 * pi * (ro[i] * ro[i]));
    }
    if (fabs(sr) > F4(1.E-6)) {
        errsum[0] = errsum[0] + (erfcc(sr / pa) - 1.0) / (4.0 * pi * sr) + erfcc(sr1 / pa) / (4.0 * pi * sr1) -
                    1.0 / (4.0 * pi * sr2);
        errsum[1] = errsum[1] - (erfcc(sr / pa) - 1.0) / (4.0 * pi * (sr * sr)) * dsrr +
                    derfcc(sr / pa) / (4.0 * pi * sr * pa) * dsrr - erfcc(sr1 / pa) / (4.0 * pi * (sr1 * sr1)) * dsr1r +
                    derfcc(sr1 / pa) / (4.0 * pi * sr1 * pa) * dsr1r + dsr2r / (4.0 * pi * (sr2 * sr2));
        errsum[2] = errsum[2] - (erfcc(sr / pa) - 1.0) / (4.0 * pi * (sr * sr)) * dsrz +
                    derfcc(sr / pa) / (4.0 * pi * sr * pa) * dsrz - erfcc(sr1 / pa) / (4.0 * pi * (sr1 * sr1)) * dsr1z +
                    derfcc(sr1 / pa) / (4.0 * pi * sr1 * pa) * dsr1z + dsr2z / (4.0 * pi * (sr2 * sr2));
    } else {
        errsum[0] = errsum[0] + erfcc(sr1 / pa) / (4.0 * pi * sr1) - 1.0 / (4.0 * pi * sr2);
        errsum[1] = errsum[1] - erfcc(sr1 / pa) / (4.0 * pi * (sr1 * sr1)) * dsr1r +
                    derfcc(sr1 / pa) / (4.0 * pi * sr1 * pa) * dsr1r + dsr2r / (4.0 * pi * (sr2 * sr2));
        errsum[2] = errsum[2] - erfcc(sr1 / pa) / (4.0 * pi * (sr1 * sr1)) * dsr1z +
                    derfcc(sr1 / pa) / (4.0 * pi * sr1 * pa) * dsr1z + dsr2z / (4.0 * pi * (sr2 * sr2));
    }

    grn[0] = grn[0] - errsum[0] - v / 2.0 / pi * aquadf(v, r, zf, zp, h, 0.0, pa / 2.0, eps, 1);
    grn[1] = grn[1] - errsum[1] + v / 2.0 / pi * aquadf(v, r, zf, zp, h, 0.0, pa / 2.0, eps, 2);
    grn[2] = grn[2] - errsum[2] - v / 2.0 / pi * aquadf(v, r, zf, zp, h, 0.0, pa / 2.0, eps, 3);

    orc_jy01bj(wk * r, &bj0, &bj1);
    km = -CI * wk;
    {
        zdouble nmk = nmf(h, km);
        grn[0] = grn[0] - CI / 4.0 / nmk * bj0 * cosh(wk * (zf + h)) * cosh(wk * (zp + h));
        grn[1] = grn[1] + CI * wk / 4.0 / nmk * bj1 * cosh(wk * (zf + h)) * cosh(wk * (zp + h));
        grn[2] = grn[2] - CI * wk / 4.0 / nmk * bj0 * sinh(wk * (zf + h)) * cosh(wk * (zp + h));
    }
    grn[0] = -4.0 * pi * grn[0];
    grn[1] = -4.0 * pi * grn[1];
    grn[2] = -4.0 * pi * grn[2];
}

/* ---------------------------------------------------------------- */
/* Drivers                                                           */
/* ---------------------------------------------------------------- */
int orc_fin_branch(double rr, double h)
{
    double rhp = fabs(rr / h);
    if (rhp < 0.0005) return 0;
    if (rhp < 0.05) return 1;
    if (rhp < 0.5) return 2;
    return 3;
}

/* FINGREEN3D_R, FinGreen3D.f90:160-226 */
void orc_fingreen3d_r(double rr, double zf, double zp, double v, const double *wvn, int nk, double h,
                      zdouble grn[3], int tag)
{
    double r, r1, zpq = zf + zp, wk = wvn[0];
    zdouble fg[3];
    r = sqrt(rr * rr + (zp - zf) * (zp - zf));
    r1 = sqrt(rr * rr + zpq * zpq);
    switch (orc_fin_branch(rr, h)) {
    case 0: linton(rr, zf, zp, v, wk, wvn, nk, h, fg); break;
    case 1: pidcock(rr, zf, zp, v, wk, wvn, nk, h, fg); break;
    case 2: eigene(rr, zf, zp, wk, wvn, nk, h, fg); break;
    default: eigen(rr, zf, zp, wk, wvn, nk, h, fg); break;
    }
    grn[0] = fg[0];
    grn[1] = (rr != 0.0) ? fg[1] : 0.0;
    grn[2] = fg[2];
    if (tag == 2) {
        grn[0] = grn[0] + 1.0 / r1;
        grn[1] = grn[1] - rr / powi(r1, 3);
        grn[2] = grn[2] - zpq / powi(r1, 3);
    } else if (tag == 3) {
        grn[0] = grn[0] + (1.0 / r1 + 1.0 / r);
        grn[1] = grn[1] - (rr / powi(r1, 3) + rr / powi(r, 3));
        grn[2] = grn[2] - (zpq / powi(r1, 3) + (zf - zp) / powi(r, 3));
    }
}

/* FINGREEN3D, FinGreen3D.f90:81-155 */
void orc_fingreen3d(double xf, double xp, double yf, double yp, double zf, double zp, double v,
                    const double *wvn, int nk, double h, zdouble grn[4], int flag)
{
    double xpq = xf - xp, ypq = yf - yp, zpq = zf + zp;
    double rr = sqrt(xpq * xpq + ypq * ypq);
    double r = sqrt(rr * rr + (zp - zf) * (zp - zf));
    double r1 = sqrt(rr * rr + zpq * zpq);
    zdouble fg[3];
    int infinite = 0;
    grn[0] = grn[1] = grn[2] = grn[3] = 0.0;
    if (fabs(v) < F4(1.E-8)) {
        infinite = 0;
    } else if (fabs(v + 1.0) < F4(1.E-8)) {
        infinite = 1;
    } else {
        orc_fingreen3d_r(rr, zf, zp, v, wvn, nk, h, fg, flag);
        if (rr > F4(1.E-6)) {
            grn[1] = fg[1] * xpq / rr;
            grn[2] = fg[1] * ypq / rr;
        }
        grn[0] = fg[0];
        grn[3] = fg[2];
    }
    if (!infinite) {
        if (flag == 1) {
            grn[0] = grn[0] + 1.0 / r1;
            grn[1] = grn[1] - xpq / powi(r1, 3);
            grn[2] = grn[2] - ypq / powi(r1, 3);
            grn[3] = grn[3] - zpq / powi(r1, 3);
        } else {
            grn[0] = grn[0] + (1.0 / r1 + 1.0 / r);
            grn[1] = grn[1] - (xpq / powi(r1, 3) + xpq / powi(r, 3));
            grn[2] = grn[2] - (ypq / powi(r1, 3) + ypq / powi(r, 3));
            grn[3] = grn[3] - (zpq / powi(r1, 3) + (zf - zp) / powi(r, 3));
        }
    } else {
        if (flag == 1) {
            grn[0] = grn[0] - 1.0 / r1;
            grn[1] = grn[1] + xpq / powi(r1, 3);
            grn[2] = grn[2] + ypq / powi(r1, 3);
            grn[3] = grn[3] + zpq / powi(r1, 3);
        } else {
            grn[0] = grn[0] + (-1.0 / r1 + 1.0 / r);
            grn[1] = grn[1] + (xpq / powi(r1, 3) - xpq / powi(r, 3));
            grn[2] = grn[2] + (ypq / powi(r1, 3) - ypq / powi(r, 3));
            grn[3] = grn[3] + (zpq / powi(r1, 3) - (zf - zp) / powi(r, 3));
        }
    }
}
