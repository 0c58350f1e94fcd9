// green.cuh -- FP64 device free-surface Green functions and their gradients.
//
// Finite depth: the region decomposition of FinGreen3D (Y. Liu et al., CPC
// 2016; HAMS-MREL src/FinGreen3D.f90:160-226) on R/h -- LINTON (< 0.0005),
// PIDCOCK (< 0.05), EIGENE (< 0.5), EIGEN -- with the same term counts,
// truncation thresholds and epsilon-algorithm extrapolation (Limes), so the
// values agree with the reference to rounding.  Recursive adaptive
// Gauss-Kronrod quadrature is run from an explicit per-thread stack, left
// half first, as the recursion visits it.
// Infinite depth: the Wu/Noblesse/Liang global approximation of the
// Havelock function (src/InfGreen_Appr.f90:104-872).
//
// The eigenfunction-series terms of EIGEN/EIGENE/PIDCOCK use the
// bit-reproducible sin/cos/exp/log of detmath.h in the operation order of the
// CPU checker: the epsilon extrapolation amplifies last-bit differences of a
// math library to up to 1e-3 in single values.
//
// Every routine returns the wave part of G with 1/r and 1/r1 removed, plus
// the point-source terms that FINGREEN3D / INFGREEN3D add back according to
// the near/far flag (FinGreen3D.f90:124-150, InfGreen_Appr.f90:130-183).
#pragma once
#include <cuComplex.h>
#include "special.cuh"

namespace hams {

struct cplx {
  double re, im;
};
__device__ __forceinline__ cplx cmk(double r, double i) { return cplx{r, i}; }
__device__ __forceinline__ cplx operator+(cplx a, cplx b) { return cplx{a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cplx operator-(cplx a, cplx b) { return cplx{a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ cplx operator*(cplx a, cplx b) {
  return cplx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ cplx operator*(double s, cplx a) { return cplx{s * a.re, s * a.im}; }
__device__ __forceinline__ cplx operator*(cplx a, double s) { return cplx{s * a.re, s * a.im}; }
__device__ __forceinline__ cplx cdiv(cplx a, cplx b) {
  // Smith's algorithm, as Fortran compilers divide complex numbers
  if (fabs(b.re) >= fabs(b.im)) {
    double r = b.im / b.re, d = b.re + b.im * r;
    return cplx{(a.re + a.im * r) / d, (a.im - a.re * r) / d};
  }
  double r = b.re / b.im, d = b.re * r + b.im;
  return cplx{(a.re * r + a.im) / d, (a.im * r - a.re) / d};
}
__device__ __forceinline__ double cabs_(cplx a) { return hypot(a.re, a.im); }
__device__ __forceinline__ cplx ccos_(cplx z) {
  double s, c;
  sincos(z.re, &s, &c);
  return cplx{c * cosh(z.im), -s * sinh(z.im)};
}
__device__ __forceinline__ cplx csin_(cplx z) {
  double s, c;
  sincos(z.re, &s, &c);
  return cplx{s * cosh(z.im), c * sinh(z.im)};
}

// Gradient set of one pair: value and d/dx, d/dy, d/dz at the source point.
struct grn4 {
  cplx g[4];
};

constexpr int kNK = 200;        // dispersion roots kept per frequency
constexpr int kMaxSeries = 100; // longest PIDCOCK series (NT <= 100)

// ---------------------------------------------------------------------------
// Wynn epsilon extrapolation of a sequence of partial sums s[0..n] (Limes,
// FinGrnExtSubs.f90:370-470); s is overwritten, as in the reference.
// ---------------------------------------------------------------------------
__device__ inline double limes(int n, double* s, double* a) {
  // Each column k of the reference's table is one pass over i.  Its two
  // loops (the odd column a, then the even column s with the running
  // maximum of |a|) are fused here: step i produces a(i+1) and then s(i)
  // from the same operands in the same order, so every entry and the
  // returned value are bit-identical; old s(i+1) and new a(i) are carried
  // in registers.  When the s loop of a column would be empty the a loop's
  // values are never read again, so that column is skipped.  Steps go in
  // pairs: the two new a entries depend on the previous column only, so
  // their reciprocals (and then the two s reciprocals) are independent and
  // overlap; the maximum test then runs in the reference's order, and an
  // early return discards the second step's stores, which nothing reads.
  double rl = s[n], amax = 0.0;
  for (int i = 0; i <= n; ++i) a[i] = 0.0;
  for (int k = 1;; ++k) {
    const int m = n - 2 * k;  // last i of the s loop
    if (m < 0) break;
    double s_i = s[0], s_i1 = s[1];
    double an_i = (s_i1 != s_i) ? a[1] + 1.0 / (s_i1 - s_i) : a[1];
    a[0] = an_i;
    int i = 0;
    for (; i < m; i += 2) {
      const double s_i2 = s[i + 2], a_i2 = a[i + 2], s_i3 = s[i + 3], a_i3 = a[i + 3];
      const double an_i1 = (s_i2 != s_i1) ? a_i2 + 1.0 / (s_i2 - s_i1) : a_i2;
      const double an_i2 = (s_i3 != s_i2) ? a_i3 + 1.0 / (s_i3 - s_i2) : a_i3;
      const double sn_i = (an_i1 != an_i) ? s_i1 + 1.0 / (an_i1 - an_i) : s_i1;
      const double sn_i1 = (an_i2 != an_i1) ? s_i2 + 1.0 / (an_i2 - an_i1) : s_i2;
      a[i + 1] = an_i1;
      a[i + 2] = an_i2;
      s[i] = sn_i;
      s[i + 1] = sn_i1;
      if (fabs(an_i) > amax) {
        amax = fabs(an_i);
        rl = sn_i;
        if (s_i1 == sn_i) return rl;
      }
      if (fabs(an_i1) > amax) {
        amax = fabs(an_i1);
        rl = sn_i1;
        if (s_i2 == sn_i1) return rl;
      }
      s_i1 = s_i3;
      an_i = an_i2;
    }
    if (i == m) {  // odd number of steps: the last one alone
      const double s_i2 = s[i + 2], a_i2 = a[i + 2];
      const double an_i1 = (s_i2 != s_i1) ? a_i2 + 1.0 / (s_i2 - s_i1) : a_i2;
      a[i + 1] = an_i1;
      const double sn_i = (an_i1 != an_i) ? s_i1 + 1.0 / (an_i1 - an_i) : s_i1;
      s[i] = sn_i;
      if (fabs(an_i) > amax) {
        amax = fabs(an_i);
        rl = sn_i;
        if (s_i1 == sn_i) return rl;
      }
    }
  }
  return rl;
}

// Rankine terms removed by every series branch (FinGreen3D.f90:349-359).
__device__ __forceinline__ void remove_rankine(double r, double zf, double zp, cplx g[3]) {
  double sr = sqrt(r * r + (zf - zp) * (zf - zp)), sr1 = sqrt(r * r + (zf + zp) * (zf + zp));
  g[0].re -= (1.0 / sr + 1.0 / sr1);
  g[1].re += (r / sr / (sr * sr) + r / sr1 / (sr1 * sr1));
  g[2].re += ((zf - zp) / sr / (sr * sr) + (zf + zp) / sr1 / (sr1 * sr1));
}

// Propagating-mode part shared by EIGEN/EIGENE/PIDCOCK (FinGreen3D.f90:311-322).
__device__ __forceinline__ void prop_mode(double r, double zfh, double zph, double wk, double h, cplx g[3]) {
  const double pi = 3.141592653589793;
  double nm0 = h / 2.0 * (1.0 + sinh(2.0 * wk * h) / (2.0 * wk * h));
  double czp = cosh(wk * zph);
  double p0 = pi / nm0 * cosh(wk * zfh) * czp;
  double dp0 = pi / nm0 * sinh(wk * zfh) * czp;
  double j0, j1, y0, y1;
  jy01b(wk * r, j0, j1, y0, y1);
  g[0] = cmk(-p0 * y0, p0 * j0);
  g[1] = cmk(wk * p0 * y1, -wk * p0 * j1);
  g[2] = cmk(-wk * dp0 * y0, wk * dp0 * j0);
}

// Per-mode factors of the eigenfunction series (mode number i >= 2, root
// wvn[i-1]): pm of EIGEN/EIGENE, ac of PIDCOCK, and the sin/cos of the
// vertical eigenfunctions at the source (zf + h) and field (zp + h) depths.
// Each depends on one mode and one panel only.  InlineModes evaluates them
// for one pair as FinGreen3D does; TableModes reads them from the
// per-frequency tables that k_mode_tables fills with the same expressions in
// the same rounding, so both give the same bits.
struct InlineModes {
  const double* __restrict__ wvn;
  double h, v, zfh, zph;
  __device__ __forceinline__ double umt(int i) const { return (i - 1) * 3.141592653589793 / h; }
  __device__ __forceinline__ double pm(int i) const {
    double km = wvn[i - 1], twokmh = 2.0 * km * h;
    return 4.0 / (1.0 + dm_sin(twokmh) / twokmh) / h;
  }
  __device__ __forceinline__ double ac(int i) const {
    double um = wvn[i - 1];
    return (um * um + v * v) / ((um * um + v * v) * h - v);
  }
  __device__ __forceinline__ void src(int i, double& s, double& c) const { dm_sincos(wvn[i - 1] * zfh, &s, &c); }
  __device__ __forceinline__ void srct(int i, double& s, double& c) const { dm_sincos(umt(i) * zfh, &s, &c); }
  __device__ __forceinline__ double fld(int i) const { return dm_cos(wvn[i - 1] * zph); }
  __device__ __forceinline__ double fldt(int i) const { return dm_cos(umt(i) * zph); }
};

constexpr int kModeMax = 100;  // mode numbers 0..99 (PIDCOCK uses up to 99)

// Per-frequency mode tables, laid out mode-major so that a warp of pairs with
// consecutive field points reads consecutive entries.
struct ModeTab {
  int n, tn;              // source panels, field points
  int nmode;              // modes 2..nmode-1 are filled
  const double* pm;       // (kModeMax)
  const double* ac;       // (kModeMax)
  const double2* src;     // (kModeMax, n): sin, cos of wvn[i-1] (zq + h)
  const double2* srct;    // (kModeMax, n): sin, cos of (i-1) pi/h (zq + h)
  const double* fld;      // (kModeMax, tn): cos of wvn[i-1] (zp + h)
  const double* fldt;     // (kModeMax, tn): cos of (i-1) pi/h (zp + h)
};

struct TableModes {
  const ModeTab& t;
  int j, f;  // source panel, field point
  __device__ __forceinline__ double pm(int i) const { return t.pm[i]; }
  __device__ __forceinline__ double ac(int i) const { return t.ac[i]; }
  __device__ __forceinline__ void src(int i, double& s, double& c) const {
    double2 q = t.src[(size_t)i * t.n + j];
    s = q.x;
    c = q.y;
  }
  __device__ __forceinline__ void srct(int i, double& s, double& c) const {
    double2 q = t.srct[(size_t)i * t.n + j];
    s = q.x;
    c = q.y;
  }
  __device__ __forceinline__ double fld(int i) const { return t.fld[(size_t)i * t.tn + f]; }
  __device__ __forceinline__ double fldt(int i) const { return t.fldt[(size_t)i * t.tn + f]; }
};

// EIGEN, FinGreen3D.f90:281-362 (R/h >= 0.5)
template <class MD>
__device__ inline void eigen(double r, double zf, double zp, double wk, const double* __restrict__ wvn, double h,
                             cplx g[3], const MD& md) {
  double zfh = zf + h, zph = zp + h;
  prop_mode(r, zfh, zph, wk, h, g);
  for (int i = 2; i <= 10; ++i) {
    double km = wvn[i - 1];
    double pm = md.pm(i);
    double k0, k1, skzf, ckzf;
    ik01a(km * r, k0, k1);
    md.src(i, skzf, ckzf);
    double ckzp = md.fld(i);
    double rm0 = pm * k0 * ckzf * ckzp, rm1 = -pm * km * k1 * ckzf * ckzp, rm2 = -pm * km * k0 * skzf * ckzp;
    g[0].re += rm0;
    g[1].re += rm1;
    g[2].re += rm2;
    if (fabs(rm0) < HAMS_F4(1.E-6) && fabs(rm1) < HAMS_F4(1.E-6) && fabs(rm2) < HAMS_F4(1.E-6)) break;
  }
  remove_rankine(r, zf, zp, g);
}

// Scratch for the epsilon tables of one thread: N >= the longest series.
template <int N>
struct SeriesScratchN {
  double s0[N], s1[N], s2[N], a[N];
};
constexpr int kEigenEMax = 50;   // EIGENE: NT = int(-88.89 R/h + 54.45) <= 50 for R/h >= 0.05
constexpr int kPidcockMax = 99;  // PIDCOCK: NT = int(-1010.10 R/h + 100.50) <= 99 for R/h >= 0.0005
using SeriesScratch = SeriesScratchN<kMaxSeries>;

// EIGENE, FinGreen3D.f90:413-506 (0.05 <= R/h < 0.5)
template <class MD, int N>
__device__ inline void eigene(double r, double zf, double zp, double wk, const double* __restrict__ wvn, double h,
                              cplx g[3], SeriesScratchN<N>& sc, const MD& md, int* overflow) {
  double rhp = fabs(r / h);
  int nt = (int)(HAMS_F4(-88.89) * rhp + HAMS_F4(54.45));
  if (nt > N) {  // outside the branch's range of R/h
    *overflow = 1;
    nt = N;
  }
  double zfh = zf + h, zph = zp + h;
  prop_mode(r, zfh, zph, wk, h, g);
  sc.s0[0] = sc.s1[0] = sc.s2[0] = 0.0;
  for (int i = 2; i <= nt; ++i) {
    double km = wvn[i - 1];
    double pm = md.pm(i);
    double k0, k1, skzf, ckzf;
    ik01a(km * r, k0, k1);
    md.src(i, skzf, ckzf);
    double ckzp = md.fld(i);
    sc.s0[i - 1] = sc.s0[i - 2] + pm * k0 * ckzf * ckzp;
    sc.s1[i - 1] = sc.s1[i - 2] + -pm * km * k1 * ckzf * ckzp;
    sc.s2[i - 1] = sc.s2[i - 2] + -pm * km * k0 * skzf * ckzp;
  }
  g[0].re += limes(nt - 1, sc.s0, sc.a);
  g[1].re += limes(nt - 1, sc.s1, sc.a);
  g[2].re += limes(nt - 1, sc.s2, sc.a);
  remove_rankine(r, zf, zp, g);
}

// Pidcock image sums IMGS/DGSR/DGSZ, FinGreen3D.f90:908-1113
static __constant__ double c_amn[25] = {
    0.0,        -0.02525711, 0.00086546,  -0.00004063, 0.00000193,  0.05051418,  -0.00692380,
    0.00073292, -0.00006636, 0.00000398,  0.00230838,  -0.00097875, 0.00020597,  -0.00003333,
    0.00000524, 0.00012934,  -0.00010879, 0.00003965,  -0.00000891, 0.0,         0.00000913,
    -0.00001270, 0.00000466, 0.0,         0.0};

__device__ inline void pidcock_images(double r, double zf, double zp, double h, double& gs, double& gr, double& gz) {
  double t1 = r / h, t2 = (zf - zp) / h, t3 = (zf + zp + 2.0 * h) / h;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int l = -1; l <= 1; ++l) {
    double a = t2 + 2.0 * l, b = t3 + 2.0 * l;
    double ra = sqrt(t1 * t1 + a * a), rb = sqrt(t1 * t1 + b * b);
    s0 += 1.0 / ra + 1.0 / rb;
    s1 += t1 / (ra * ra * ra) + t1 / (rb * rb * rb);
    s2 += a / (ra * ra * ra) + b / (rb * rb * rb);
  }
  // powers t^(2m), t^(2m-1) and t^(2n) as the reference's pow() calls
  double p1[5], p2[5], p3[5];
  for (int m = 0; m <= 4; ++m) {
    p1[m] = pow(t1, 2.0 * m);
    p2[m] = pow(t2, 2.0 * m);
    p3[m] = pow(t3, 2.0 * m);
  }
  double q0 = 0.0, q1 = 0.0, q2 = 0.0;
  for (int m = 0; m <= 4; ++m)
    for (int n = 0; n <= 4; ++n) {
      double amn = c_amn[m + 5 * n];
      q0 += amn * p1[m] * (p2[n] + p3[n]);
      if (m >= 1) q1 += 2.0 * m * amn * pow(t1, 2.0 * m - 1.0) * (p2[n] + p3[n]);
      if (n >= 1) q2 += 2.0 * n * amn * p1[m] * (pow(t2, 2.0 * n - 1.0) + pow(t3, 2.0 * n - 1.0));
    }
  gs = (s0 - 2.0 + q0) / h;
  gr = (-s1 + q1) / (h * h);
  gz = (-s2 + q2) / (h * h);
}

// Propagating mode and logarithmic terms of PIDCOCK, FinGreen3D.f90:581-591.
__device__ inline void pidcock_head(double r, double zfh, double zph, double wk, double h, cplx g[3]) {
  const double pi = 3.141592653589793, ga = 0.5772156649015328;
  double nm0 = h / 2.0 * (1.0 + sinh(2.0 * wk * h) / (2.0 * wk * h));
  double czp = cosh(wk * zph);
  double p0 = pi / nm0 * cosh(wk * zfh) * czp;
  double dp0 = wk * pi / nm0 * sinh(wk * zfh) * czp;
  double j0, j1, y0, y1;
  jy01b(wk * r, j0, j1, y0, y1);
  g[0] = cmk(-p0 * y0 + 2.0 / h * (ga + log(r / 4.0 / h)), p0 * j0);
  g[1] = cmk(wk * p0 * y1 + 2.0 / (r * h), -wk * p0 * j1);
  g[2] = cmk(-dp0 * y0, dp0 * j0);
}

// The epsilon-extrapolated mode-difference sums of PIDCOCK (FinGreen3D.f90:597-632)
template <class MD, int N>
__device__ inline void pidcock_sums(double r, double h, const double* __restrict__ wvn, SeriesScratchN<N>& sc,
                                    const MD& md, int* overflow, double l[3]) {
  const double pi = 3.141592653589793;
  double rhp = fabs(r / h);
  int nt = (int)(HAMS_F4(-1010.10) * rhp + HAMS_F4(100.50));
  if (nt > N) {  // outside the branch's range of R/h
    *overflow = 1;
    nt = N;
  }
  sc.s0[0] = sc.s1[0] = sc.s2[0] = 0.0;
  for (int i = 2; i <= nt; ++i) {
    double umt = (i - 1) * pi / h, um = wvn[i - 1];
    double k0, k1, k0t, k1t;
    ik01a(um * r, k0, k1);
    ik01a(umt * r, k0t, k1t);
    double ac = md.ac(i);
    double su, cu, sut, cut;
    md.src(i, su, cu);
    md.srct(i, sut, cut);
    double cup = md.fld(i), cutp = md.fldt(i);
    double am = ac * cu * cup, amt = cut * cutp / h;
    double dam = -um * ac * su * cup, damt = -umt * sut * cutp / h;
    sc.s0[i - 1] = sc.s0[i - 2] + (am * k0 - amt * k0t);
    sc.s1[i - 1] = sc.s1[i - 2] + (-um * am * k1 + umt * amt * k1t);
    sc.s2[i - 1] = sc.s2[i - 2] + (dam * k0 - damt * k0t);
  }
  l[0] = limes(nt - 1, sc.s0, sc.a);
  l[1] = limes(nt - 1, sc.s1, sc.a);
  l[2] = limes(nt - 1, sc.s2, sc.a);
}

// PIDCOCK's wave term from its three extrapolated sums: head + 4 l + images
// (FinGreen3D.f90:634-642), before the point-source terms are removed.
__device__ inline void pidcock_assemble(double r, double zf, double zp, double h, const double l[3], cplx g[3]) {
  double gs, gr, gz;
  pidcock_images(r, zf, zp, h, gs, gr, gz);
  g[0].re = g[0].re + 4.0 * l[0] + gs;
  g[1].re = g[1].re + 4.0 * l[1] + gr;
  g[2].re = g[2].re + 4.0 * l[2] + gz;
}

// PIDCOCK, FinGreen3D.f90:558-660 (0.0005 <= R/h < 0.05)
template <class MD, int N>
__device__ inline void pidcock(double r, double zf, double zp, double v, double wk, const double* __restrict__ wvn,
                               double h, cplx g[3], SeriesScratchN<N>& sc, const MD& md, int* overflow) {
  double zfh = zf + h, zph = zp + h;
  pidcock_head(r, zfh, zph, wk, h, g);
  double l[3];
  pidcock_sums(r, h, wvn, sc, md, overflow, l);
  pidcock_assemble(r, zf, zp, h, l, g);
  remove_rankine(r, zf, zp, g);
}

// ---------------------------------------------------------------------------
// LINTON (R/h < 0.0005), FinGreen3D.f90:712-861 and its support routines
// ---------------------------------------------------------------------------
static __constant__ double c_xgq[7] = {-0.949107912342759, -0.741531185599394, -0.405845151377397, 0.0,
                                0.405845151377397,  0.741531185599394,  0.949107912342759};
static __constant__ double c_wgq[7] = {0.129484966168870, 0.279705391489277, 0.381830050505119, 0.417959183673469,
                                0.381830050505119, 0.279705391489277, 0.129484966168870};
static __constant__ double c_xkq[15] = {-0.991455371120813, -0.949107912342759, -0.864864423359769, -0.741531185599394,
                                 -0.586087235467691, -0.405845151377397, -0.207784955007898, 0.0,
                                 0.207784955007898,  0.405845151377397,  0.586087235467691,  0.741531185599394,
                                 0.864864423359769,  0.949107912342759,  0.991455371120813};
static __constant__ double c_wkq[15] = {0.022935322010529, 0.063092092629979, 0.104790010322250, 0.140653259715525,
                                 0.169004726639267, 0.190350578064785, 0.204432940075298, 0.209482141084728,
                                 0.204432940075298, 0.190350578064785, 0.169004726639267, 0.140653259715525,
                                 0.104790010322250, 0.063092092629979, 0.022935322010529};

// Integrands F1/F2 (FinGreen3D.f90:1882-2020)
__device__ __forceinline__ double lin_f(int tag, double r, double wvn, int no, double t) {
  const double pi = 3.141592653589793;
  if (fabs(t) < 1.0e-8) return 0.0;
  double e = (no == 1) ? exp(-(r * r) / 4.0 / t + wvn * wvn * t) : exp(-(r * r) / 4.0 / t - wvn * wvn * t);
  return tag == 1 ? e / 4.0 / pi / t : -r * e / 8.0 / pi / (t * t);
}

// Integrands G1/G2/G3 (FinGreen3D.f90:2033-2214)
__device__ __forceinline__ double lin_g(int tag, double v, double r, double zf, double zp, double h, double t) {
  if (fabs(t) < 1.0e-8) return 0.0;
  const double val[4] = {-zp - zf, 2.0 * h - zp + zf, 2.0 * h + zp - zf, 4.0 * h + zp + zf};
  const double dval[4] = {-1.0, 1.0, -1.0, 1.0};
  double sum = 0.0;
  for (int i = 0; i < 4; ++i) {
    double ev = exp(-v * val[i]), arg = val[i] / 2.0 / t - v * t;
    if (tag == 3)
      sum = sum - v * dval[i] * ev * erfc_zj(arg) + ev * derfc_zj(arg) * dval[i] / 2.0 / t;
    else
      sum = sum + ev * erfc_zj(arg);
  }
  double e = exp(v * v * (t * t) - (r * r) / 4.0 / (t * t));
  if (tag == 2) return r / 2.0 / (t * t * t) * e * sum;
  return e * sum / t;
}

// 7/15-point Gauss-Kronrod on [a,b] (GK_INTEG / GK_INTEGF)
template <class F>
__device__ inline void gk15(const F& f, double a, double b, double& gk, double& err) {
  double stf[7], gi = 0.0, hw = (b - a) / 2.0;
  for (int i = 0; i < 7; ++i) {
    stf[i] = f(0.5 * (b + a + (b - a) * c_xgq[i]));
    gi = gi + c_wgq[i] * hw * stf[i];
  }
  gk = 0.0;
  for (int i = 1; i <= 15; ++i) {
    double fv = (i % 2 == 0) ? stf[i / 2 - 1] : f(0.5 * (b + a + (b - a) * c_xkq[i - 1]));
    gk = gk + c_wkq[i - 1] * hw * fv;
  }
  err = pow(200.0 * fabs(gk - gi), 1.5);
}

constexpr int kQuadStack = 64;

// Adaptive bisection of AQUAD / AQUADF (FinGreen3D.f90:2515, :2728), run
// depth-first from a bounded stack; *overflow is set if the stack is full.
template <class F>
__device__ inline double aquad(const F& f, double a, double b, double eps, int* overflow) {
  double sa[kQuadStack], sb[kQuadStack];
  int sp = 0;
  double sum = 0.0;
  sa[0] = a;
  sb[0] = b;
  sp = 1;
  while (sp > 0) {
    --sp;
    double x0 = sa[sp], x1 = sb[sp], gk, err;
    gk15(f, x0, x1, gk, err);
    if (err > eps && fabs(x0 - x1) > eps) {
      if (sp + 2 > kQuadStack) {
        *overflow = 1;
        sum += gk;
        continue;
      }
      double xm = (x0 + x1) / 2.0;
      sa[sp] = xm;  // right half below, left half on top
      sb[sp] = x1;
      sa[sp + 1] = x0;
      sb[sp + 1] = xm;
      sp += 2;
    } else {
      sum += gk;
    }
  }
  return sum;
}

// The quadrature of the LINTON branch, as a policy: one thread per pair
// (aquad), or one warp per pair (WarpQuad: the fifteen Kronrod nodes of an
// interval evaluated by fifteen lanes, every lane then forms the same 7- and
// 15-point sums in the reference's order, so the bisection decisions are the
// same on all lanes; the interval stack is in the warp's shared memory).
struct ThreadQuad {
  template <class F>
  __device__ double operator()(const F& f, double a, double b, double eps, int* overflow) const {
    return aquad(f, a, b, eps, overflow);
  }
};

struct WarpQuad {
  double* sa;  // kQuadStack interval bounds each, this warp's shared memory
  double* sb;
  int lane;
  template <class F>
  __device__ double operator()(const F& f, double a, double b, double eps, int* overflow) const {
    int sp = 1;
    double sum = 0.0;
    if (lane == 0) {
      sa[0] = a;
      sb[0] = b;
    }
    __syncwarp();
    while (sp > 0) {
      --sp;
      const double x0 = sa[sp], x1 = sb[sp], hw = (x1 - x0) / 2.0;
      double fv = 0.0;
      if (lane < 15) {  // Kronrod node lane + 1; the even ones are the Gauss nodes
        const int kk = lane + 1;
        const double c = (kk % 2 == 0) ? c_xgq[kk / 2 - 1] : c_xkq[kk - 1];
        fv = f(0.5 * (x1 + x0 + (x1 - x0) * c));
      }
      double v[15];
#pragma unroll
      for (int k = 0; k < 15; ++k) v[k] = __shfl_sync(0xffffffffu, fv, k);
      double gi = 0.0, gk = 0.0;
#pragma unroll
      for (int q = 0; q < 7; ++q) gi = gi + c_wgq[q] * hw * v[2 * q + 1];
#pragma unroll
      for (int kk = 1; kk <= 15; ++kk) gk = gk + c_wkq[kk - 1] * hw * v[kk - 1];
      const double err = pow(200.0 * fabs(gk - gi), 1.5);
      __syncwarp();  // every lane has read the interval before it is overwritten
      if (err > eps && fabs(x0 - x1) > eps) {
        if (sp + 2 > kQuadStack) {
          *overflow = 1;
          sum += gk;
          continue;
        }
        const double xm = (x0 + x1) / 2.0;
        if (lane == 0) {
          sa[sp] = xm;  // right half below, left half on top
          sb[sp] = x1;
          sa[sp + 1] = x0;
          sb[sp + 1] = xm;
        }
        sp += 2;
        __syncwarp();
      } else {
        sum += gk;
      }
    }
    return sum;
  }
};

// SA0/DSA0/SAM/DSAM series (FinGreen3D.f90:1389-1740)
__device__ inline double sa0(double r, double pa, double wk) {
  const double ga = 0.5772156649015328, pi = 3.141592653589793, eps = HAMS_F4(1.E-6);
  double s = -ga - 2.0 * log(wk * pa / 2.0), rm = 100.0, sgn = -1.0, facn = 1.0, psi = 0.0;
  for (int n = 1; fabs(rm) > eps && n < 400; ++n) {
    double en = enxa(n + 1, (r / pa) * (r / pa));
    psi = psi + 1.0 / n;
    rm = sgn * pow(r / pa, 2.0 * n) / facn / n - pow(wk * pa / 2.0, 2.0 * n) / facn * en -
         2.0 * sgn / (facn * facn) * pow(wk * r / 2.0, 2.0 * n) * (log(wk * r / 2.0) + ga - psi);
    s = s + rm;
    sgn = -sgn;
    facn = facn * (n + 1);
  }
  return s / 4.0 / pi;
}
__device__ inline double dsa0(double r, double pa, double wk) {
  const double ga = 0.5772156649015328, pi = 3.141592653589793, eps = HAMS_F4(1.E-6);
  double s = 0.0, rm = 100.0, sgn = -1.0, facn = 1.0, psi = 0.0;
  for (int n = 1; fabs(rm) > eps && n < 400; ++n) {
    double en = enxa(n, (r / pa) * (r / pa));
    psi = psi + 1.0 / n;
    rm = 2.0 * sgn * pow(r / pa, 2.0 * n - 1.0) / facn / pa + pow(wk * pa / 2.0, 2.0 * n) / facn * en * 2.0 * r / (pa * pa) -
         2.0 * sgn * n * wk / (facn * facn) * pow(wk * r / 2.0, 2.0 * n - 1.0) * (log(wk * r / 2.0) + ga - psi) -
         2.0 * sgn / (facn * facn) * pow(wk * r / 2.0, 2.0 * n) / r;
    s = s + rm;
    sgn = -sgn;
    facn = facn * (n + 1);
  }
  return s / 4.0 / pi;
}
__device__ inline double sam(double r, double pa, double wvn) {
  const double pi = 3.141592653589793, eps = HAMS_F4(1.E-6);
  double s = 0.0, rm = 100.0, sgn = 1.0, facn = 1.0, x = (wvn * pa / 2.0) * (wvn * pa / 2.0);
  for (int n = 0; fabs(rm) > eps && n < 400; ++n) {
    rm = sgn * pow(r / pa, 2.0 * n) / facn * enxa(n + 1, x);
    s = s + rm;
    sgn = -sgn;
    facn = facn * (n + 1);
  }
  return s / 4.0 / pi;
}
__device__ inline double dsam(double r, double pa, double wvn) {
  const double pi = 3.141592653589793, eps = HAMS_F4(1.E-6);
  double s = 0.0, rm = 100.0, sgn = -1.0, facn = 1.0, x = (wvn * pa / 2.0) * (wvn * pa / 2.0);
  for (int n = 1; fabs(rm) > eps && n < 400; ++n) {
    rm = 2.0 * n * sgn * pow(r / pa, 2.0 * n - 1.0) / facn / pa * enxa(n + 1, x);
    s = s + rm;
    sgn = -sgn;
    facn = facn * (n + 1);
  }
  return s / 4.0 / pi;
}

// COEF / DCOEF coefficient of eigenmode i (1-based), FinGreen3D.f90:1168-1388
template <class Q>
__device__ inline void lin_coef(int i, double r, double pa, double a, const double* __restrict__ wvn, double wk,
                                double& cof, double& dcof, int* overflow, const Q& quad) {
  const double pi = 3.141592653589793, eps = HAMS_F4(1.E-6), step = 100.0;
  double dnt = pa * pa / 4.0;
  if (i == 1) {
    if (fabs(r) < HAMS_F4(1.E-6)) {
      cof = -eix(wk * wk * dnt) / 4.0 / pi;
      dcof = 0.0;
    } else if (r / a <= 0.5) {
      cof = sa0(r, pa, wk);
      dcof = dsa0(r, pa, wk);
    } else {
      double j0, j1, y0, y1;
      jy01b(wk * r, j0, j1, y0, y1);
      cof = -y0 / 4.0 - quad([=](double t) { return lin_f(1, r, wk, 1, t); }, 0.0, dnt, eps, overflow);
      dcof = wk * y1 / 4.0 - quad([=](double t) { return lin_f(2, r, wk, 1, t); }, 0.0, dnt, eps, overflow);
    }
    return;
  }
  double km = wvn[i - 1];
  if (fabs(r) < HAMS_F4(1.E-6)) {
    cof = e1xa(km * km * dnt) / 4.0 / pi;
    dcof = 0.0;
  } else if (r / a <= 1.0) {
    cof = sam(r, pa, km);
    dcof = dsam(r, pa, km);
  } else {
    double p1 = dnt + step;
    for (int it = 0; fabs(lin_f(1, r, km, i, p1)) > eps && it < 100000; ++it) p1 = p1 + step;
    cof = quad([=](double t) { return lin_f(1, r, km, i, t); }, dnt, p1, eps, overflow);
    p1 = dnt + step;
    for (int it = 0; fabs(lin_f(2, r, km, i, p1)) > eps && it < 100000; ++it) p1 = p1 + step;
    dcof = quad([=](double t) { return lin_f(2, r, km, i, t); }, dnt, p1, eps, overflow);
  }
}

__device__ __forceinline__ cplx nm_mode(double h, cplx k) {  // NM, FinGreen3D.f90:2280
  cplx z = cmk(2.0 * k.re * h, 2.0 * k.im * h);
  cplx q = cdiv(csin_(z), z);
  return cmk(h / 2.0 * (1.0 + q.re), h / 2.0 * q.im);
}

template <class Q = ThreadQuad>
__device__ inline void linton(double r, double zf, double zp, double v, double wk, const double* __restrict__ wvn,
                              double h, cplx g[3], int* overflow, const Q& quad = Q{}) {
  const double pi = 3.141592653589793, eps = HAMS_F4(1.E-6);
  double a;
  if (v < 0.02) a = 3324.2 * (v * v * v) - 258.89 * (v * v) + 8.3958 * v + 1.3208;
  else if (v < 0.1) a = -30.303 * (v * v * v) - 2.8138 * (v * v) + 2.7740 * v + 0.05052;
  else if (v < 1.0) a = 1.5699 * (v * v * v) - 2.5075 * (v * v) + 1.8316 * v + 0.1077;
  else a = -0.000069641 * (v * v * v) - 0.0017082 * (v * v) + 0.45566 * v + 0.80551;
  a = fabs(a) / (wk * h);
  double pa = a * h;
  double sr = sqrt(r * r + (zf - zp) * (zf - zp));
  double sr1 = sqrt(r * r + (2.0 * h + zf + zp) * (2.0 * h + zf + zp));
  double sr2 = sqrt(r * r + (zf + zp) * (zf + zp));

  g[0] = g[1] = g[2] = cmk(0.0, 0.0);
  for (int i = 1; i <= 20; ++i) {
    double cof, dcof;
    lin_coef(i, r, pa, a, wvn, wk, cof, dcof, overflow, quad);
    cplx km = (i == 1) ? cmk(0.0, -wk) : cmk(wvn[i - 1], 0.0);
    cplx nmk = nm_mode(h, km);
    cplx c1 = ccos_(cmk(km.re * (zf + h), km.im * (zf + h)));
    cplx c2 = ccos_(cmk(km.re * (zp + h), km.im * (zp + h)));
    cplx s1 = csin_(cmk(km.re * (zf + h), km.im * (zf + h)));
    cplx cc = c1 * c2;
    cplx rm0 = -1.0 * (cdiv(cmk(cof, 0.0), nmk) * cc);
    cplx rm1 = -1.0 * (cdiv(cmk(dcof, 0.0), nmk) * cc);
    cplx rm2 = cdiv(cof * km, nmk) * s1 * c2;
    g[0] = g[0] + rm0;
    g[1] = g[1] + rm1;
    g[2] = g[2] + rm2;
    if (i > 2 && cabs_(rm0) < eps && cabs_(rm1) < eps && cabs_(rm2) < eps) break;
  }

  // Image sums with erfc damping (FinGreen3D.f90:801-832)
  const double val[4] = {-zp - zf, 2.0 * h - zp + zf, 2.0 * h + zp - zf, 4.0 * h + zp + zf};
  double es0 = 0.0, es1 = 0.0, es2 = 0.0;
  for (int i = 0; i < 4; ++i) {
    double ro = sqrt(r * r + val[i] * val[i]);
    double dror = r / ro, droz = val[i] * ((i & 1) ? 1.0 : -1.0) / ro;
    double ec = erfc_zj(ro / pa), dc = derfc_zj(ro / pa);
    es0 = es0 + ec / (4.0 * pi * ro);
    es1 = es1 + (dc / pa * dror * ro - dror * ec) / (4.0 * pi * (ro * ro));
    es2 = es2 + (dc / pa * droz * ro - droz * ec) / (4.0 * pi * (ro * ro));
  }
  double dsr1r = r / sr1, dsr1z = (2.0 * h + zf + zp) / sr1, dsr2r = r / sr2, dsr2z = (zf + zp) / sr2;
  double e1 = erfc_zj(sr1 / pa), d1 = derfc_zj(sr1 / pa);
  if (fabs(sr) > HAMS_F4(1.E-6)) {
    double dsrr = r / sr, dsrz = (zf - zp) / sr, e0 = erfc_zj(sr / pa), d0 = derfc_zj(sr / pa);
    es0 = es0 + (e0 - 1.0) / (4.0 * pi * sr) + e1 / (4.0 * pi * sr1) - 1.0 / (4.0 * pi * sr2);
    es1 = es1 - (e0 - 1.0) / (4.0 * pi * (sr * sr)) * dsrr + d0 / (4.0 * pi * sr * pa) * dsrr -
          e1 / (4.0 * pi * (sr1 * sr1)) * dsr1r + d1 / (4.0 * pi * sr1 * pa) * dsr1r + dsr2r / (4.0 * pi * (sr2 * sr2));
    es2 = es2 - (e0 - 1.0) / (4.0 * pi * (sr * sr)) * dsrz + d0 / (4.0 * pi * sr * pa) * dsrz -
          e1 / (4.0 * pi * (sr1 * sr1)) * dsr1z + d1 / (4.0 * pi * sr1 * pa) * dsr1z + dsr2z / (4.0 * pi * (sr2 * sr2));
  } else {
    es0 = es0 + e1 / (4.0 * pi * sr1) - 1.0 / (4.0 * pi * sr2);
    es1 = es1 - e1 / (4.0 * pi * (sr1 * sr1)) * dsr1r + d1 / (4.0 * pi * sr1 * pa) * dsr1r +
          dsr2r / (4.0 * pi * (sr2 * sr2));
    es2 = es2 - e1 / (4.0 * pi * (sr1 * sr1)) * dsr1z + d1 / (4.0 * pi * sr1 * pa) * dsr1z +
          dsr2z / (4.0 * pi * (sr2 * sr2));
  }
  double q1 = quad([=](double t) { return lin_g(1, v, r, zf, zp, h, t); }, 0.0, pa / 2.0, eps, overflow);
  double q2 = quad([=](double t) { return lin_g(2, v, r, zf, zp, h, t); }, 0.0, pa / 2.0, eps, overflow);
  double q3 = quad([=](double t) { return lin_g(3, v, r, zf, zp, h, t); }, 0.0, pa / 2.0, eps, overflow);
  g[0].re = g[0].re - es0 - v / 2.0 / pi * q1;
  g[1].re = g[1].re - es1 + v / 2.0 / pi * q2;
  g[2].re = g[2].re - es2 - v / 2.0 / pi * q3;

  // propagating mode written with J0 only (FinGreen3D.f90:845-852)
  double j0, j1, y0, y1;
  jy01b(wk * r, j0, j1, y0, y1);
  cplx nmk = nm_mode(h, cmk(0.0, -wk));
  double ch = cosh(wk * (zf + h)) * cosh(wk * (zp + h)), sh = sinh(wk * (zf + h)) * cosh(wk * (zp + h));
  cplx ci4 = cdiv(cmk(0.0, 0.25), nmk);
  g[0] = g[0] - ci4 * (j0 * ch);
  g[1] = g[1] + ci4 * (wk * j1 * ch);
  g[2] = g[2] - ci4 * (wk * j0 * sh);
  g[0] = -4.0 * pi * g[0];
  g[1] = -4.0 * pi * g[1];
  g[2] = -4.0 * pi * g[2];
}

// Branch of FINGREEN3D_R (FinGreen3D.f90:183-191)
enum FinBranch { kLinton = 0, kPidcock = 1, kEigenE = 2, kEigen = 3 };
__host__ __device__ __forceinline__ int fin_branch(double rr, double h) {
  double rhp = fabs(rr / h);
  if (rhp < 0.0005) return kLinton;
  if (rhp < 0.05) return kPidcock;
  if (rhp < 0.5) return kEigenE;
  return kEigen;
}

// Epsilon-table length of EIGENE / PIDCOCK for a pair (FinGreen3D.f90:434, :592).
__host__ __device__ __forceinline__ int fin_terms(double rr, double h) {
  double rhp = fabs(rr / h);
  int b = fin_branch(rr, h);
  if (b == kEigenE) return (int)(HAMS_F4(-88.89) * rhp + HAMS_F4(54.45));
  if (b == kPidcock) return (int)(HAMS_F4(-1010.10) * rhp + HAMS_F4(100.50));
  return b == kEigen ? 10 : 20;
}

// FINGREEN3D (FinGreen3D.f90:81-155) for one source (xq..) / field (xp..) pair
// of branch BR (compile-time, so each branch kernel carries only its own
// scratch SC, unused by LINTON and EIGEN).  v = omega^2/g, wk = wvn[0]; md
// supplies the per-mode factors (InlineModes or TableModes).
// Convenience form with inline mode factors.
template <int BR, class SC>
__device__ inline grn4 fingreen3d(double xq, double xp, double yq, double yp, double zq, double zp, double v,
                                  const double* __restrict__ wvn, double h, int flag, SC* sc, int* overflow);
__device__ inline grn4 finish_green(cplx fg[3], double xpq, double ypq, double zq, double zp, double rr, double r,
                                    double r1, int flag);
template <int BR, class MD, class SC>
__device__ inline grn4 fingreen3d(double xq, double xp, double yq, double yp, double zq, double zp, double v,
                                  const double* __restrict__ wvn, double h, int flag, SC* sc, int* overflow,
                                  const MD& md) {
  double xpq = xq - xp, ypq = yq - yp, zpq = zq + zp;
  double rr = sqrt(xpq * xpq + ypq * ypq);
  double r = sqrt(rr * rr + (zp - zq) * (zp - zq)), r1 = sqrt(rr * rr + zpq * zpq);
  cplx fg[3];
  double wk = wvn[0];
  if constexpr (BR == kLinton) linton(rr, zq, zp, v, wk, wvn, h, fg, overflow);
  else if constexpr (BR == kPidcock) pidcock(rr, zq, zp, v, wk, wvn, h, fg, *sc, md, overflow);
  else if constexpr (BR == kEigenE) eigene(rr, zq, zp, wk, wvn, h, fg, *sc, md, overflow);
  else eigen(rr, zq, zp, wk, wvn, h, fg, md);
  return finish_green(fg, xpq, ypq, zq, zp, rr, r, r1, flag);
}

// FINGREEN3D of the LINTON branch with the quadrature policy quad
// (WarpQuad: every lane of a warp calls it for the same pair).
template <class Q>
__device__ inline grn4 fingreen3d_linton(double xq, double xp, double yq, double yp, double zq, double zp, double v,
                                         const double* __restrict__ wvn, double h, int flag, int* overflow,
                                         const Q& quad) {
  double xpq = xq - xp, ypq = yq - yp, zpq = zq + zp;
  double rr = sqrt(xpq * xpq + ypq * ypq);
  double r = sqrt(rr * rr + (zp - zq) * (zp - zq)), r1 = sqrt(rr * rr + zpq * zpq);
  cplx fg[3];
  linton(rr, zq, zp, v, wvn[0], wvn, h, fg, overflow, quad);
  return finish_green(fg, xpq, ypq, zq, zp, rr, r, r1, flag);
}

// The tail of FINGREEN3D (FinGreen3D.f90:124-150): the wave part fg (G and
// its R and zq derivatives) projected on x and y, plus 1/r1 (and 1/r for far
// pairs) and their gradients.
__device__ inline grn4 finish_green(cplx fg[3], double xpq, double ypq, double zq, double zp, double rr, double r,
                                    double r1, int flag) {
  grn4 o;
  double zpq = zq + zp;
  if (rr == 0.0) fg[1] = cmk(0.0, 0.0);
  o.g[0] = fg[0];
  o.g[3] = fg[2];
  if (rr > HAMS_F4(1.E-6)) {
    o.g[1] = fg[1] * (xpq / rr);
    o.g[2] = fg[1] * (ypq / rr);
  } else {
    o.g[1] = o.g[2] = cmk(0.0, 0.0);
  }
  double ir1 = 1.0 / r1, ir13 = ir1 * ir1 * ir1;
  if (flag == 1) {
    o.g[0].re += ir1;
    o.g[1].re -= xpq * ir13;
    o.g[2].re -= ypq * ir13;
    o.g[3].re -= zpq * ir13;
  } else {
    double ir = 1.0 / r, ir3 = ir * ir * ir;
    o.g[0].re += (ir1 + ir);
    o.g[1].re -= (xpq * ir13 + xpq * ir3);
    o.g[2].re -= (ypq * ir13 + ypq * ir3);
    o.g[3].re -= (zpq * ir13 + (zq - zp) * ir3);
  }
  return o;
}

template <int BR, class SC>
__device__ inline grn4 fingreen3d(double xq, double xp, double yq, double yp, double zq, double zp, double v,
                                  const double* __restrict__ wvn, double h, int flag, SC* sc, int* overflow) {
  InlineModes md{wvn, h, v, zq + h, zp + h};
  return fingreen3d<BR>(xq, xp, yq, yp, zq, zp, v, wvn, h, flag, sc, overflow, md);
}

// Zero- and infinite-frequency limits of both Green functions
// (FinGreen3D.f90:124-150, InfGreen_Appr.f90:130-158): point-source terms only.
__device__ inline grn4 green_limit(bool infinite_freq, double xq, double xp, double yq, double yp, double zq, double zp,
                                   int flag) {
  double xpq = xq - xp, ypq = yq - yp, zpq = zq + zp;
  double rr = sqrt(xpq * xpq + ypq * ypq);
  double r = sqrt(rr * rr + (zp - zq) * (zp - zq)), r1 = sqrt(rr * rr + zpq * zpq);
  double s = infinite_freq ? -1.0 : 1.0, ir1 = 1.0 / r1, ir13 = ir1 * ir1 * ir1;
  grn4 o;
  for (int k = 0; k < 4; ++k) o.g[k] = cmk(0.0, 0.0);
  o.g[0].re = s * ir1;
  o.g[1].re = -s * xpq * ir13;
  o.g[2].re = -s * ypq * ir13;
  o.g[3].re = -s * zpq * ir13;
  if (flag != 1) {
    double ir = 1.0 / r, ir3 = ir * ir * ir;
    o.g[0].re += ir;
    o.g[1].re -= xpq * ir3;
    o.g[2].re -= ypq * ir3;
    o.g[3].re -= (zq - zp) * ir3;
  }
  return o;
}

// ---------------------------------------------------------------------------
// Infinite depth: Havelock function approximation (InfGreen_Appr.f90:189-872)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double hpoly(const double* c, int deg, double t) {
  double s = (c[deg - 1] + c[deg] * t) * t;
  for (int k = deg - 2; k >= 1; --k) s = (c[k] + s) * t;
  return c[0] + s;
}
static __constant__ double c_hA[10] = {+1.21, -13.328, +215.896, -1763.96, +8418.94, -24314.21, +42002.57, -41592.9, 21859.0, -4838.6};
static __constant__ double c_hB[10] = {+0.938, +5.373, -67.92, +796.534, -4780.77, +17137.74, -36618.81, +44894.06, -29030.24, +7671.22};
static __constant__ double c_hC[8] = {+1.268, -9.747, +209.653, -1397.89, +5155.67, -9844.35, +9136.4, -3272.62};
static __constant__ double c_hD[10] = {+0.632, -40.97, +667.16, -6072.07, +31127.39, -96293.05, +181856.75, -205690.43, +128170.2, -33744.6};
static __constant__ double c_hdA[10] = {+2.948, -24.53, +249.69, -754.85, -1187.71, +16370.75, -48811.41, +68220.87, -46688.0, +12622.25};
static __constant__ double c_hdB[10] = {+1.11, +2.894, -76.765, +1565.35, -11336.19, +44270.15, -97014.11, +118879.26, -76209.82, +19923.28};
static __constant__ double c_hdC[6] = {+14.19, -148.24, +847.8, -2318.58, +3168.35, -1590.27};

__device__ inline double hv_j0(double xx) {
  const double pi = 3.141592653589793;
  if (xx <= 3.0) {
    double yy = (xx / 3.0) * (xx / 3.0);
    return 0.999999999 + (-2.249999879 + (1.265623060 + (-0.316394552 + (0.044460948 + (-0.003954479 + 0.000212950 * yy) * yy) * yy) * yy) * yy) * yy;
  }
  double yy = 3.0 / xx, y2 = yy * yy;
  double f0 = 0.79788454 + (-0.00553897 + (0.00099336 + (-0.00044346 + (0.00020445 - 0.00004959 * y2) * y2) * y2) * y2) * y2;
  double th = xx - 0.25 * pi + (-0.04166592 + (0.00239399 + (-0.00073984 + (0.00031099 - 0.00007605 * y2) * y2) * y2) * y2) * yy;
  return f0 * cos(th) / sqrt(xx);
}
__device__ inline double hv_j1(double xx) {
  const double pi = 3.141592653589793;
  if (xx <= 3.0) {
    double yy = xx / 3.0, y2 = yy * yy;
    return (0.5 + (-0.562499992 + (0.210937377 + (-0.039550040 + (0.004447331 + (-0.000330547 + 0.000015525 * y2) * y2) * y2) * y2) * y2) * y2) * xx;
  }
  double yy = 3.0 / xx, y2 = yy * yy;
  double f1 = 0.79788459 + (0.01662008 + (-0.00187002 + (0.00068519 + (-0.00029440 + 0.00006952 * y2) * y2) * y2) * y2) * y2;
  double th = xx - 0.75 * pi + (0.12499895 + (-0.00605240 + (0.00135825 + (-0.00049616 + 0.00011531 * y2) * y2) * y2) * y2) * yy;
  return f1 * cos(th) / sqrt(xx);
}
__device__ inline double hv_y0(double xx) {
  const double pi = 3.141592653589793;
  if (xx <= 3.0) {
    double t = xx / 3.0, t2 = t * t;
    return (2.0 / pi) * log(xx / 2.0) * hv_j0(xx) + 0.367466907 + 0.605593797 * t2 - 0.743505078 * powi(t, 4) +
           0.253005481 * powi(t, 6) - 0.042619616 * powi(t, 8) + 0.004285691 * powi(t, 10) - 0.000250716 * powi(t, 12);
  }
  double u = 3.0 / xx;
  double f0 = 0.79788454 - 0.00553897 * powi(u, 2) + 0.00099336 * powi(u, 4) - 0.00044346 * powi(u, 6) +
              0.00020445 * powi(u, 8) - 0.00004959 * powi(u, 10);
  double th = xx - 0.25 * pi - 0.04166592 * u + 0.00239399 * powi(u, 3) - 0.00073984 * powi(u, 5) +
              0.00031099 * powi(u, 7) - 0.00007605 * powi(u, 9);
  return f0 * sin(th) / sqrt(xx);
}
__device__ inline double hv_y1(double xx) {
  const double pi = 3.141592653589793;
  if (xx <= 3.0) {
    double t = xx / 3.0;
    return (2.0 / pi) * (log(xx / 2.0) * hv_j1(xx) - 1.0 / xx) + 0.07373571 * t + 0.72276433 * powi(t, 3) -
           0.43885620 * powi(t, 5) + 0.10418264 * powi(t, 7) - 0.01340825 * powi(t, 9) + 0.00094249 * powi(t, 11);
  }
  double u = 3.0 / xx;
  double f1 = 0.79788459 + 0.01662008 * powi(u, 2) - 0.00187002 * powi(u, 4) + 0.00068519 * powi(u, 6) -
              0.00029440 * powi(u, 8) + 0.00006952 * powi(u, 10);
  double th = xx - 3.0 * pi / 4.0 + 0.12499895 * u - 0.00605240 * powi(u, 3) + 0.00135825 * powi(u, 5) -
              0.00049616 * powi(u, 7) + 0.00011531 * powi(u, 9);
  return f1 * sin(th) / sqrt(xx);
}
__device__ inline double hv_h0(double xx) {
  const double pi = 3.141592653589793;
  if (xx <= 3.0) {
    double yy = (xx / 3.0) * (xx / 3.0);
    return (1.909859164 + (-1.909855001 + (0.687514637 + (-0.126164557 + (0.013828813 - 0.000876918 * yy) * yy) * yy) * yy) * yy) * (xx / 3.0);
  }
  double yy = (3.0 / xx) * (3.0 / xx);
  double c1 = 2.0 * (0.99999906 + (4.77228920 + (3.85542044 + 0.32303607 * yy) * yy) * yy);
  double c2 = pi * xx * (1.0 + (4.88331068 + (4.28957333 + 0.52120508 * yy) * yy) * yy);
  return c1 / c2 + hv_y0(xx);
}
__device__ inline double hv_h1(double xx) {
  const double pi = 3.141592653589793;
  if (xx <= 3.0) {
    double yy = (xx / 3.0) * (xx / 3.0);
    return (1.909859286 + (-1.145914713 + (0.294656958 + (-0.042070508 + (0.003785727 - 0.000207183 * yy) * yy) * yy) * yy) * yy) * yy;
  }
  double yy = (3.0 / xx) * (3.0 / xx);
  double c1 = 2.0 * (1.00000004 + (3.92205313 + (2.64893033 + 0.27450895 * yy) * yy) * yy);
  double c2 = pi * (1.0 + (3.81095112 + (2.26216956 + 0.10885141 * yy) * yy) * yy);
  return c1 / c2 + hv_y1(xx);
}

// HavelockGF (InfGreen_Appr.f90:189-205): gf = L0 + W, gfh = Ls + Wh
__device__ inline void havelock(double hh, double vv, cplx& gf, cplx& gfh) {
  const double pi = 3.141592653589793, gama = 0.5772156649;
  double dd = sqrt(hh * hh + vv * vv), alpha = -vv / dd, beta = hh / dd, rho = dd / (1.0 + dd);
  double ev = exp(vv), dd3 = dd * dd * dd, omr3 = (1.0 - rho) * (1.0 - rho) * (1.0 - rho);
  double pp = (log(0.5 * (dd - vv)) + gama - 2.0 * dd * dd) * ev + dd * dd - vv;
  double rr = (1.0 - beta) * hpoly(c_hA, 9, rho) - beta * hpoly(c_hB, 9, rho) -
              alpha * hpoly(c_hC, 7, rho) / (1.0 + 6.0 * alpha * rho * (1.0 - rho)) +
              beta * (1.0 - beta) * hpoly(c_hD, 9, rho);
  double l0 = 2.0 * pp / (1.0 + dd3) + 2.0 * (rho * omr3 * rr);
  double ps = (beta + hh) / (dd - vv) - 2.0 * beta + 2.0 * ev * dd - hh;
  double qs = exp(-dd) * (1.0 - beta) * (1.0 + dd / (1.0 + dd3));
  double rs = beta * hpoly(c_hdA, 9, rho) - (1.0 - alpha) * hpoly(c_hdB, 9, rho) +
              beta * (1.0 - beta) * rho * (1.0 - 2.0 * rho) * hpoly(c_hdC, 5, rho);
  double ls = 2.0 * ps / (1.0 + dd3) - 4.0 * qs + 2.0 * (rho * omr3 * rs);
  double h0 = hv_h0(hh), j0 = hv_j0(hh), h1 = hv_h1(hh), j1 = hv_j1(hh);
  gf = cmk(l0 + 2.0 * pi * h0 * ev, -2.0 * pi * j0 * ev);
  gfh = cmk(ls + 2.0 * pi * (2.0 / pi - h1) * ev, 2.0 * pi * j1 * ev);
}

// INFGREEN3D (InfGreen_Appr.f90:104-186), regular frequency
__device__ inline grn4 infgreen3d(double xq, double xp, double yq, double yp, double zq, double zp, double v,
                                  int flag) {
  double xpq = xq - xp, ypq = yq - yp, zpq = zp + zq;
  double rr = sqrt(xpq * xpq + ypq * ypq);
  double r = sqrt(rr * rr + (zp - zq) * (zp - zq)), r1 = sqrt(rr * rr + zpq * zpq);
  cplx gf, gfh;
  havelock(v * rr, v * zpq, gf, gfh);
  grn4 o;
  double v2 = v * v;
  if (rr > HAMS_F4(1.E-6)) {
    o.g[1] = gfh * (-v2 * xpq / rr);
    o.g[2] = gfh * (-v2 * ypq / rr);
  } else {
    o.g[1] = o.g[2] = cmk(0.0, 0.0);
  }
  o.g[0] = gf * (-v);
  o.g[3] = cmk(-v2 * gf.re + 2.0 * v / r1, -v2 * gf.im);
  double ir1 = 1.0 / r1, ir13 = ir1 * ir1 * ir1;
  o.g[0].re += ir1;
  o.g[1].re -= xpq * ir13;
  o.g[2].re -= ypq * ir13;
  o.g[3].re -= zpq * ir13;
  if (flag != 1) {
    double ir = 1.0 / r, ir3 = ir * ir * ir;
    o.g[0].re += ir;
    o.g[1].re -= xpq * ir3;
    o.g[2].re -= ypq * ir3;
    o.g[3].re -= (zq - zp) * ir3;
  }
  return o;
}

}  // namespace hams
