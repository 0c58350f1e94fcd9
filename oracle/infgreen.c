/*
 * infgreen.c -- infinite-depth free-surface Green function.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle_internal.h).
 *
 * Restates src/InfGreen_Appr.f90 of HAMS-MREL: the global approximation of
 * the Havelock Green function by H. Wu, C. Zhang, Y. Zhu, W. Li, D. Wan,
 * F. Noblesse (2017) and its gradient by H. Liang, H. Wu, F. Noblesse (2018).
 * The reference keeps the intermediate quantities (dd, alpha, beta, sigma,
 * rho) in module variables that OpenMP threads share (InfGreen_Appr.f90:89-96);
 * they are locals here, which is what a race-free run of the reference
 * computes.
 */
#include "oracle_internal.h"

static const double PI = 3.141592653589793;
static const double GAMA = 0.5772156649; /* InfGreen_Appr.f90:86 */

typedef struct {
    double dd, alpha, beta, sigma, rho;
} gfpar;

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

/* GF_DivParameters, :209 */
static gfpar divpar(double hh, double vv)
{
    gfpar p;
    p.dd = sqrt(hh * hh + vv * vv);
    p.alpha = -vv / p.dd;
    p.beta = hh / p.dd;
    p.sigma = hh / (p.dd - vv);
    p.rho = p.dd / (1.0 + p.dd);
    return p;
}

/* Polynomials A(rho)..D(rho), dA..dC of Wu et al., :290-560 */
static double horner(const double *c, int deg, double t)
{
    double s = (c[deg - 1] + c[deg] * t) * t;
    int k;
    for (k = deg - 2; k >= 1; --k) s = (c[k] + s) * t;
    return c[0] + s;
}
static const double CA[10] = {+1.21, -13.328, +215.896, -1763.96, +8418.94, -24314.21, +42002.57, -41592.9, 21859.0, -4838.6};
static const double CB[10] = {+0.938, +5.373, -67.92, +796.534, -4780.77, +17137.74, -36618.81, +44894.06, -29030.24, +7671.22};
static const double CC[8] = {+1.268, -9.747, +209.653, -1397.89, +5155.67, -9844.35, +9136.4, -3272.62};
static const double CD[10] = {+0.632, -40.97, +667.16, -6072.07, +31127.39, -96293.05, +181856.75, -205690.43, +128170.2, -33744.6};
static const double CdA[10] = {+2.948, -24.53, +249.69, -754.85, -1187.71, +16370.75, -48811.41, +68220.87, -46688.0, +12622.25};
static const double CdB[10] = {+1.11, +2.894, -76.765, +1565.35, -11336.19, +44270.15, -97014.11, +118879.26, -76209.82, +19923.28};
static const double CdC[6] = {+14.19, -148.24, +847.8, -2318.58, +3168.35, -1590.27};

/* BesselJ0/J1/Y0/Y1, StruveH0/H1 polynomial approximations, :583-872 */
static double besj0(double xx)
{
    if (xx <= 3.0) {
        double yy = (xx / 3.0) * (xx / 3.0);
        return 0.999999999 + (-2.249999879 + (1.265623060 + (-0.316394552 + (0.044460948 + (-0.003954479 + 0.000212950 * yy) * yy) * yy) * yy) * yy) * yy;
    } else {
        double yy = 3.0 / xx, y2 = yy * yy;
        double f0 = 0.79788454 + (-0.00553897 + (0.00099336 + (-0.00044346 + (0.00020445 - 0.00004959 * y2) * y2) * y2) * y2) * y2;
        double th = xx - 0.25 * PI + (-0.04166592 + (0.00239399 + (-0.00073984 + (0.00031099 - 0.00007605 * y2) * y2) * y2) * y2) * yy;
        return f0 * cos(th) / sqrt(xx);
    }
}
static double besj1(double xx)
{
    if (xx <= 3.0) {
        double yy = xx / 3.0, y2 = yy * yy;
        double s = 0.5 + (-0.562499992 + (0.210937377 + (-0.039550040 + (0.004447331 + (-0.000330547 + 0.000015525 * y2) * y2) * y2) * y2) * y2) * y2;
        return s * xx;
    } else {
        double yy = 3.0 / xx, y2 = yy * yy;
        double f1 = 0.79788459 + (0.01662008 + (-0.00187002 + (0.00068519 + (-0.00029440 + 0.00006952 * y2) * y2) * y2) * y2) * y2;
        double th = xx - 0.75 * PI + (0.12499895 + (-0.00605240 + (0.00135825 + (-0.00049616 + 0.00011531 * y2) * y2) * y2) * y2) * yy;
        return f1 * cos(th) / sqrt(xx);
    }
}
static double besy0(double xx)
{
    if (xx <= 3.0) {
        double t = xx / 3.0;
        return (2.0 / PI) * log(xx / 2.0) * besj0(xx) + 0.367466907 + 0.605593797 * powi(t, 2) -
               0.743505078 * powi(t, 4) + 0.253005481 * powi(t, 6) - 0.042619616 * powi(t, 8) +
               0.004285691 * powi(t, 10) - 0.000250716 * powi(t, 12);
    } else {
        double u = 3.0 / xx;
        double f0 = 0.79788454 - 0.00553897 * powi(u, 2) + 0.00099336 * powi(u, 4) - 0.00044346 * powi(u, 6) +
                    0.00020445 * powi(u, 8) - 0.00004959 * powi(u, 10);
        double th = xx - 0.25 * PI - 0.04166592 * powi(u, 1) + 0.00239399 * powi(u, 3) - 0.00073984 * powi(u, 5) +
                    0.00031099 * powi(u, 7) - 0.00007605 * powi(u, 9);
        return f0 * sin(th) / sqrt(xx);
    }
}
static double besy1(double xx)
{
    if (xx <= 3.0) {
        double t = xx / 3.0;
        return (2.0 / PI) * (log(xx / 2.0) * besj1(xx) - 1.0 / xx) + 0.07373571 * powi(t, 1) +
               0.72276433 * powi(t, 3) - 0.43885620 * powi(t, 5) + 0.10418264 * powi(t, 7) -
               0.01340825 * powi(t, 9) + 0.00094249 * powi(t, 11);
    } else {
        double u = 3.0 / xx;
        double f1 = 0.79788459 + 0.01662008 * powi(u, 2) - 0.00187002 * powi(u, 4) + 0.00068519 * powi(u, 6) -
                    0.00029440 * powi(u, 8) + 0.00006952 * powi(u, 10);
        double th = xx - 3.0 * PI / 4.0 + 0.12499895 * powi(u, 1) - 0.00605240 * powi(u, 3) +
                    0.00135825 * powi(u, 5) - 0.00049616 * powi(u, 7) + 0.00011531 * powi(u, 9);
        return f1 * sin(th) / sqrt(xx);
    }
}
static double struveh0(double xx)
{
    if (xx <= 3.0) {
        double yy = (xx / 3.0) * (xx / 3.0);
        double s = 1.909859164 + (-1.909855001 + (0.687514637 + (-0.126164557 + (0.013828813 - 0.000876918 * yy) * yy) * yy) * yy) * yy;
        return s * (xx / 3.0);
    } else {
        double yy = (3.0 / xx) * (3.0 / xx);
        double c1 = 2.0 * (0.99999906 + (4.77228920 + (3.85542044 + 0.32303607 * yy) * yy) * yy);
        double c2 = PI * xx * (1.0 + (4.88331068 + (4.28957333 + 0.52120508 * yy) * yy) * yy);
        return c1 / c2 + besy0(xx);
    }
}
static double struveh1(double xx)
{
    if (xx <= 3.0) {
        double yy = (xx / 3.0) * (xx / 3.0);
        return (1.909859286 + (-1.145914713 + (0.294656958 + (-0.042070508 + (0.003785727 - 0.000207183 * yy) * yy) * yy) * yy) * yy) * yy;
    } else {
        double yy = (3.0 / xx) * (3.0 / xx);
        double c1 = 2.0 * (1.00000004 + (3.92205313 + (2.64893033 + 0.27450895 * yy) * yy) * yy);
        double c2 = PI * (1.0 + (3.81095112 + (2.26216956 + 0.10885141 * yy) * yy) * yy);
        return c1 / c2 + besy1(xx);
    }
}

/* GF_Func_L0 / Lp, :229-270 */
static double func_l0(const gfpar *p, double hh, double vv)
{
    double pp, rr, lp;
    (void)hh;
    pp = log(0.5 * (p->dd - vv)) + GAMA - 2.0 * p->dd * p->dd;
    pp = exp(vv) * pp;
    pp = pp + p->dd * p->dd - vv;
    rr = (1.0 - p->beta) * horner(CA, 9, p->rho);
    rr = rr - p->beta * horner(CB, 9, p->rho);
    rr = rr - p->alpha * horner(CC, 7, p->rho) / (1.0 + 6.0 * p->alpha * p->rho * (1.0 - p->rho));
    rr = rr + p->beta * (1.0 - p->beta) * horner(CD, 9, p->rho);
    lp = p->rho * powi(1.0 - p->rho, 3) * rr;
    return 2.0 * pp / (1.0 + powi(p->dd, 3)) + 2.0 * lp;
}

/* GF_Func_Ls / Lsp, :433-480 */
static double func_ls(const gfpar *p, double hh, double vv)
{
    double ps, qs, rr, lsp;
    ps = (p->beta + hh) / (p->dd - vv);
    ps = ps - 2.0 * p->beta + 2.0 * exp(vv) * p->dd - hh;
    qs = exp(-p->dd) * (1.0 - p->beta);
    qs = qs * (1.0 + p->dd / (1.0 + powi(p->dd, 3)));
    rr = p->beta * horner(CdA, 9, p->rho);
    rr = rr - (1.0 - p->alpha) * horner(CdB, 9, p->rho);
    rr = rr + p->beta * (1.0 - p->beta) * p->rho * (1.0 - 2.0 * p->rho) * horner(CdC, 5, p->rho);
    lsp = p->rho * powi(1.0 - p->rho, 3) * rr;
    return 2.0 * ps / (1.0 + powi(p->dd, 3)) - 4.0 * qs + 2.0 * lsp;
}

/* HavelockGF, :189-205 */
static void havelock(double hh, double vv, zdouble *gf, zdouble *gfh)
{
    gfpar p = divpar(hh, vv);
    zdouble w = 2.0 * PI * (struveh0(hh) - I * besj0(hh)) * exp(vv);
    zdouble wh = 2.0 * PI * (2.0 / PI - struveh1(hh) + I * besj1(hh)) * exp(vv);
    *gf = func_l0(&p, hh, vv) + w;
    *gfh = func_ls(&p, hh, vv) + wh;
}

/* INFGREEN3D, InfGreen_Appr.f90:104-186 */
void orc_infgreen3d(double xf, double xp, double yf, double yp, double zf, double zp, double v,
                    zdouble grn[4], int flag)
{
    double xpq = xf - xp, ypq = yf - yp, zpq = zp + zf;
    double rr = sqrt(xpq * xpq + ypq * ypq);
    double r = sqrt(rr * rr + (zp - zf) * (zp - zf));
    double r1 = sqrt(rr * rr + zpq * zpq);
    zdouble gf = 0.0, gfh = 0.0;
    grn[0] = grn[1] = grn[2] = grn[3] = 0.0;

    if (fabs(v) < F4(1.E-8)) {
        if (flag == 1) {
            grn[0] = grn[0] + 1.0 / r1;
            grn[1] = grn[1] - xpq / powi(r1, 3);
            grn[2] = grn[2] - ypq / powi(r1, 3);
            grn[3] = grn[3] - zpq / powi(r1, 3);
        } else {
            grn[0] = grn[0] + 1.0 / r1 + 1.0 / r;
            grn[1] = grn[1] - xpq / powi(r1, 3) - xpq / powi(r, 3);
            grn[2] = grn[2] - ypq / powi(r1, 3) - ypq / powi(r, 3);
            grn[3] = grn[3] - zpq / powi(r1, 3) - (zf - zp) / powi(r, 3);
        }
    } else if (fabs(v + 1.0) < F4(1.E-8)) {
        if (flag == 1) {
            grn[0] = grn[0] - 1.0 / r1;
            grn[1] = grn[1] + xpq / powi(r1, 3);
            grn[2] = grn[2] + ypq / powi(r1, 3);
            grn[3] = grn[3] + zpq / powi(r1, 3);
        } else {
            grn[0] = grn[0] - 1.0 / r1 + 1.0 / r;
            grn[1] = grn[1] + xpq / powi(r1, 3) - xpq / powi(r, 3);
            grn[2] = grn[2] + ypq / powi(r1, 3) - ypq / powi(r, 3);
            grn[3] = grn[3] + zpq / powi(r1, 3) - (zf - zp) / powi(r, 3);
        }
    } else {
        havelock(v * rr, v * zpq, &gf, &gfh);
        if (rr > F4(1.E-6)) {
            grn[1] = -(v * v) * gfh * xpq / rr;
            grn[2] = -(v * v) * gfh * ypq / rr;
        }
        grn[0] = -v * gf;
        grn[3] = -(v * v) * gf + 2.0 * v / r1;
        if (flag == 1) {
            grn[0] = grn[0] + 1.0 / r1;
            grn[1] = grn[1] - xpq / powi(r1, 3);
            grn[2] = grn[2] - ypq / powi(r1, 3);
            grn[3] = grn[3] - zpq / powi(r1, 3);
        } else {
            grn[0] = grn[0] + 1.0 / r1 + 1.0 / r;
            grn[1] = grn[1] - xpq / powi(r1, 3) - xpq / powi(r, 3);
            grn[2] = grn[2] - ypq / powi(r1, 3) - ypq / powi(r, 3);
            grn[3] = grn[3] - zpq / powi(r1, 3) - (zf - zp) / powi(r, 3);
        }
    }
}
