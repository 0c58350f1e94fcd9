/*
 * bem.c -- per-frequency build-and-solve of the constant-panel BEM.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle_internal.h).
 *
 * Restates, for the oracle:
 *   DISPERSION            src/WavDynSubs.f90:40-127  (J.N. Newman 1990)
 *   CalWaveProperts       src/ImplementSubs.f90:40-151
 *   VINP / DINP           src/PatclVelct.f90:42-123
 *   geometry              src/NormalProcess.f90:46-441, ReadPanelMeshMulti.f90:122-200
 *   CALGREEN_MULTI[_IRR]  src/CalGreenFuncMulti.f90:112-318
 *   BODINT/RBC/DBC        src/BodyIntgrMulti.f90:48-173, BodyIntgr_irrMulti.f90:49-234
 *   ASSB_*_MULTI[_IRR]    src/AssbMatxMulti.f90:53-251, AssbMatx_irrMulti.f90:53-465
 *   *_SOLVER_MULTI        src/AssbMatxMulti.f90:257-383 (ZGETRF/ZGETRS semantics)
 *   RFORCE/EFORCE_MULTI   src/PotentWavForceMulti.f90:45-226
 * Pair tables are not stored: each field row evaluates its pairs and applies
 * them in the reference's accumulation order.
 */
#include <stdlib.h>
#include <string.h>
#include "hams_oracle.h"
#include "oracle_internal.h"
#ifdef _OPENMP
#include <omp.h>
#endif

static const double PI = 3.141592653589793;

/* Const_mod symmetry tables (WavDynMods.f90:149-159), Fortran (2,2) column order. */
static const double RXY_[4] = {1.0, 1.0, 1.0, -1.0};
static const double RX_[4] = {1.0, -1.0, 1.0, 1.0};
static const double RY_[4] = {1.0, 1.0, 1.0, -1.0};
static const double SX_[4] = {1.0, 1.0, 1.0, 1.0};
static const double SY_[4] = {1.0, -1.0, -1.0, 1.0};
#define T22(t, i, j) t[((i)-1) + 2 * ((j)-1)]

/* ------------------------------------------------------------------ */
/* Wave properties                                                     */
/* ------------------------------------------------------------------ */

/* DISPERSION, WavDynSubs.f90:40-127 (own g = 9.807, :58) */
void orc_dispersion(double *wvn, int nrt, double w, double h)
{
    const double g = 9.807, pi = 3.141592653589793;
    double x, y, t, u, trial, dnm, fun, dfun, d2fun, exx;
    int i;
    x = w * w * h / g;
    if (x > 0.0 && x <= 2.0) {
        y = sqrt(x) * (0.9994 + 0.1701 * x + F4(0.0305) * x * x);
    } else {
        t = x * exp(-2.0 * x);
        y = x + 2.0 * t - 6.0 * t * t;
    }
    if (fabs(y - x) < F4(1.E-10)) {
        wvn[0] = x / h;
    } else {
        exx = 1.0;
        while (exx > 1.0e-10) {
            trial = y;
            dnm = trial * trial - x * x;
            fun = log((trial + x) / (trial - x)) / 2.0 - trial;
            dfun = -x / dnm - 1.0;
            d2fun = 2.0 * x * trial / (dnm * dnm);
            y = trial - fun / dfun * (1.0 + (fun / dfun) * (d2fun / dfun) / 2.0);
            exx = fabs(y - trial);
        }
        wvn[0] = y / h;
    }
    u = 3.0 * x / (7.0 + 3.0 * x);
    t = 0.0159 + 0.1032 * u + 4.3152 * u * u - 2.8768 * u * u * u;
    for (i = 2; i <= nrt; ++i) {
        exx = 1.0;
        while (exx > 1.0e-10) {
            trial = t;
            y = (i - 1) * pi - trial;
            dnm = y * y + x * x;
            fun = atan2(x, y) - trial;
            dfun = x / dnm - 1.0;
            d2fun = 2.0 * x * trial / (dnm * dnm);
            t = trial - fun / dfun * (1.0 + (fun / dfun) * (d2fun / dfun) / 2.0);
            exx = fabs(t - trial);
        }
        y = (i - 1) * pi - t;
        wvn[i - 1] = y / h;
        t = t - pi * x / (x * x + pi * i * (pi * (i - 1) - t));
    }
}

void orc_dispersion_c(double *wvn, int32_t nrt, double w, double h) { orc_dispersion(wvn, nrt, w, h); }

/* CalWaveProperts, ImplementSubs.f90:40-151 */
void orc_wave_props(int32_t inft, double value, double h, double g, int32_t sybo_kk, orc_wave *o)
{
    memset(o, 0, sizeof(*o));
    if (sybo_kk == 1) {
        o->v = 0.0; o->wk = 0.0; o->w1 = 0.0; o->tp = -1.0; o->wl = -1.0;
        return;
    }
    if (sybo_kk == 2) {
        o->v = -1.0; o->wk = -1.0; o->w1 = -1.0; o->tp = 0.0; o->wl = 0.0;
        return;
    }
    if (inft == 1) {
        o->v = value;
        if (h <= 0.0) { o->wk = o->v; o->w1 = sqrt(g * o->v); }
        else { o->w1 = sqrt(g * o->v); orc_dispersion(o->wvn, ORC_NK, o->w1, h); o->wk = o->wvn[0]; }
        o->wl = 2.0 * PI / o->wk; o->tp = 2.0 * PI / o->w1;
    } else if (inft == 2) {
        o->wk = value;
        if (h <= 0.0) { o->v = o->wk; o->w1 = sqrt(g * o->v); }
        else { o->v = o->wk * tanh(o->wk * h); o->w1 = sqrt(g * o->v); orc_dispersion(o->wvn, ORC_NK, o->w1, h); }
        o->wl = 2.0 * PI / o->wk; o->tp = 2.0 * PI / o->w1;
    } else if (inft == 3) {
        o->w1 = value;
        o->v = o->w1 * o->w1 / g;
        if (h <= 0.0) o->wk = o->v;
        else { orc_dispersion(o->wvn, ORC_NK, o->w1, h); o->wk = o->wvn[0]; }
        o->wl = 2.0 * PI / o->wk; o->tp = 2.0 * PI / o->w1;
    } else if (inft == 4) {
        o->tp = value;
        o->w1 = 2.0 * PI / o->tp;
        o->v = o->w1 * o->w1 / g;
        if (h <= 0.0) o->wk = o->v;
        else { orc_dispersion(o->wvn, ORC_NK, o->w1, h); o->wk = o->wvn[0]; }
        o->wl = 2.0 * PI / o->wk;
    } else if (inft == 5) {
        o->wl = value;
        o->wk = 2.0 * PI / o->wl;
        if (h <= 0.0) { o->v = o->wk; o->w1 = sqrt(g * o->v); }
        else { o->v = o->wk * tanh(o->wk * h); o->w1 = sqrt(g * o->v); orc_dispersion(o->wvn, ORC_NK, o->w1, h); }
    }
}

/* ------------------------------------------------------------------ */
/* Incident wave                                                        */
/* ------------------------------------------------------------------ */
static void wave_w0k0(const orc_wave *w, double *w0, double *wk0)
{
    if (fabs(w->v) < F4(1.E-8)) { *w0 = F4(1.E-20); *wk0 = F4(1.E-20); }
    else if (fabs(w->v + 1.0) < F4(1.E-8)) { *w0 = F4(1.E+20); *wk0 = F4(1.E+20); }
    else { *w0 = w->w1; *wk0 = w->wk; }
}

/* VINP, PatclVelct.f90:42-77 */
static zdouble vinp(const orc_opts *o, const orc_wave *w, double x, double y, double z, double sita)
{
    double w0, wk0, wkx, dum;
    zdouble r;
    wave_w0k0(w, &w0, &wk0);
    wkx = wk0 * ((x - o->xw[0]) * cos(sita) + (y - o->xw[1]) * sin(sita));
    if (o->h < 0.0 || o->h > 500.0) {
        r = -I * o->amp * o->g / w0 * exp(wk0 * z) * cexp(I * wkx);
    } else {
        dum = -o->amp * w0 / (wk0 * sinh(wk0 * o->h));
        r = I * dum * cosh(wk0 * (z + o->h)) * cexp(I * wkx);
    }
    return r / I;
}

/* DINP, PatclVelct.f90:83-123 */
static void dinp(const orc_opts *o, const orc_wave *w, double x, double y, double z, double sita,
                 zdouble *dx, zdouble *dy, zdouble *dz)
{
    double w0, wk0, wkx, thkdh, thkdv;
    zdouble e;
    wave_w0k0(w, &w0, &wk0);
    wkx = wk0 * ((x - o->xw[0]) * cos(sita) + (y - o->xw[1]) * sin(sita));
    e = cexp(I * wkx);
    if (o->h < 0.0) {
        *dx = w0 * o->amp * exp(wk0 * z) * e * cos(sita);
        *dy = w0 * o->amp * exp(wk0 * z) * e * sin(sita);
        *dz = -I * w0 * o->amp * exp(wk0 * z) * e;
    } else {
        thkdh = cosh(wk0 * (z + o->h)) / sinh(wk0 * o->h);
        thkdv = sinh(wk0 * (z + o->h)) / sinh(wk0 * o->h);
        *dx = w0 * o->amp * thkdh * e * cos(sita);
        *dy = w0 * o->amp * thkdh * e * sin(sita);
        *dz = -I * w0 * o->amp * thkdv * e;
    }
    *dx = *dx / I;
    *dy = *dy / I;
    *dz = *dz / I;
}

/* ------------------------------------------------------------------ */
/* Geometry (CalNormalsMulti)                                          */
/* ------------------------------------------------------------------ */
static void tri_area(const double *p1, const double *p2, const double *p3, double *ds)
{ /* CalDeltaArea_Improved, NormalProcess.f90:373-396 */
    double v21[3], v13[3], v23[3], a, b, c, l1, l2, l3, l4;
    int k;
    for (k = 0; k < 3; ++k) { v21[k] = p1[k] - p2[k]; v23[k] = p3[k] - p2[k]; v13[k] = p3[k] - p1[k]; }
    a = sqrt(v21[0] * v21[0] + v21[1] * v21[1] + v21[2] * v21[2]);
    b = sqrt(v13[0] * v13[0] + v13[1] * v13[1] + v13[2] * v13[2]);
    c = sqrt(v23[0] * v23[0] + v23[1] * v23[1] + v23[2] * v23[2]);
    l1 = a + (b + c);
    l2 = c - (a - b);
    l3 = c + (a - b);
    l4 = a + (b - c);
    *ds = sqrt(l1 * l2 * l3 * l4) / 4.0;
}

static void prep_panels(const double *xyz, int ntnd, int nelem, const int32_t *ncn, const int32_t *ncon,
                        double *xyz_p, double *ds, double *pnsz, double *dxyz)
{
    int iel, j, k;
    for (iel = 0; iel < nelem; ++iel) {
        double p[4][3], s[3] = {0.0, 0.0, 0.0}, un[3], aun, ads;
        int nc = ncn[iel];
        for (j = 0; j < nc; ++j)
            for (k = 0; k < 3; ++k) p[j][k] = xyz[(ncon[iel + nelem * j] - 1) + ntnd * k];
        /* CalPanelCentre :134 */
        for (j = 0; j < nc; ++j)
            for (k = 0; k < 3; ++k) s[k] = s[k] + p[j][k];
        for (k = 0; k < 3; ++k) xyz_p[iel + nelem * k] = s[k] / nc;
        /* CalPanelArea :171 */
        tri_area(p[0], p[1], p[2], &ds[iel]);
        if (nc == 4) { tri_area(p[0], p[3], p[2], &ads); ds[iel] = ds[iel] + ads; }
        /* CalPanelChartLength :401 */
        {
            double m = 0.0, e;
            for (j = 0; j < nc; ++j) {
                int jn = (j + 1) % nc;
                e = sqrt((p[jn][0] - p[j][0]) * (p[jn][0] - p[j][0]) + (p[jn][1] - p[j][1]) * (p[jn][1] - p[j][1]) +
                         (p[jn][2] - p[j][2]) * (p[jn][2] - p[j][2]));
                if (j == 0 || e > m) m = e;
            }
            pnsz[iel] = m;
        }
        /* CalTransNormals :74 */
        if (nc == 3) {
            double v21[3], v23[3];
            for (k = 0; k < 3; ++k) { v21[k] = p[0][k] - p[1][k]; v23[k] = p[2][k] - p[1][k]; }
            un[0] = v21[1] * v23[2] - v21[2] * v23[1];
            un[1] = v21[2] * v23[0] - v21[0] * v23[2];
            un[2] = v21[0] * v23[1] - v21[1] * v23[0];
        } else {
            double v13[3], v24[3];
            for (k = 0; k < 3; ++k) { v13[k] = p[2][k] - p[0][k]; v24[k] = p[3][k] - p[1][k]; }
            un[0] = v24[1] * v13[2] - v24[2] * v13[1];
            un[1] = v24[2] * v13[0] - v24[0] * v13[2];
            un[2] = v24[0] * v13[1] - v24[1] * v13[0];
        }
        aun = sqrt(un[0] * un[0] + un[1] * un[1] + un[2] * un[2]);
        for (k = 0; k < 3; ++k) dxyz[iel + nelem * k] = un[k] / aun;
    }
}

static void rot_normals(const double *rg, int nelem, int i0, int i1, const double *xyz_p, double *dxyz)
{ /* CalRotNormals, NormalProcess.f90:46-62 */
    int iel;
    for (iel = i0; iel < i1; ++iel) {
        double x = xyz_p[iel], y = xyz_p[iel + nelem], z = xyz_p[iel + 2 * nelem];
        double n1 = dxyz[iel], n2 = dxyz[iel + nelem], n3 = dxyz[iel + 2 * nelem];
        dxyz[iel + 3 * nelem] = (y - rg[1]) * n3 - (z - rg[2]) * n2;
        dxyz[iel + 4 * nelem] = (z - rg[2]) * n1 - (x - rg[0]) * n3;
        dxyz[iel + 5 * nelem] = (x - rg[0]) * n2 - (y - rg[1]) * n1;
    }
}

void orc_geom_prepare(orc_geom *g, const double *xr)
{
    int b, i0 = 0;
    prep_panels(g->xyz, g->ntnd, g->nelem, g->ncn, g->ncon, g->xyz_p, g->ds, g->pnsz, g->dxyz);
    for (b = 0; b < g->nbody; ++b) {
        double rg[3] = {xr[b], xr[b + g->nbody], xr[b + 2 * g->nbody]};
        rot_normals(rg, g->nelem, i0, i0 + g->body_nelem[b], g->xyz_p, g->dxyz);
        i0 += g->body_nelem[b];
    }
    if (g->inelem > 0) {
        prep_panels(g->ixyz, g->intnd, g->inelem, g->incn, g->incon, g->ixyz_p, g->ids, g->ipnsz, g->idxyz);
        i0 = 0;
        for (b = 0; b < g->nbody; ++b) {
            double rg[3] = {xr[b], xr[b + g->nbody], xr[b + 2 * g->nbody]};
            rot_normals(rg, g->inelem, i0, i0 + g->body_inelem[b], g->ixyz_p, g->idxyz);
            i0 += g->body_inelem[b];
        }
    }
}

/* ------------------------------------------------------------------ */
/* Pair evaluation (CALGREEN_MULTI body)                                */
/* ------------------------------------------------------------------ */
static void field_point(const orc_geom *g, const double *p, int np, int iel, int is, double xf[3])
{
    if (g->isx == 1 && g->isy == 0) {
        xf[0] = T22(SY_, is, 1) * p[iel];
        xf[1] = T22(SX_, is, 1) * p[iel + np];
    } else {
        xf[0] = T22(SX_, is, 1) * p[iel];
        xf[1] = T22(SY_, is, 1) * p[iel + np];
    }
    xf[2] = p[iel + 2 * np];
}

static void rankine_pair(const orc_geom *g, int jel, const double xf[3], double *sij, double dij[3])
{
    int k, v, n = g->nelem;
    if (g->ncn[jel] == 3) {
        double q[3][3];
        for (v = 0; v < 3; ++v)
            for (k = 0; k < 3; ++k) q[v][k] = g->xyz[(g->ncon[jel + n * v] - 1) + g->ntnd * k];
        orc_sglint_tri(xf, q, sij, dij);
    } else {
        double q[4][3];
        for (v = 0; v < 4; ++v)
            for (k = 0; k < 3; ++k) q[v][k] = g->xyz[(g->ncon[jel + n * v] - 1) + g->ntnd * k];
        orc_sglint_quad(xf, q, sij, dij);
    }
}

/* One table entry: RKBN(4) and CGRN(4) of field point xf against source jel. */
static void pair_tables(const orc_geom *g, const orc_opts *o, const orc_wave *w, int jel, const double xf[3],
                        int flag, double rkn[4], zdouble grn[4])
{
    int n = g->nelem;
    double xq = g->xyz_p[jel], yq = g->xyz_p[jel + n], zq = g->xyz_p[jel + 2 * n], dij[3];
    rankine_pair(g, jel, xf, &rkn[0], dij);
    rkn[1] = dij[0];
    rkn[2] = dij[1];
    rkn[3] = dij[2];
    if (o->h < 0.0) orc_infgreen3d(xq, xf[0], yq, xf[1], zq, xf[2], w->v, grn, flag);
    else orc_fingreen3d(xq, xf[0], yq, xf[1], zq, xf[2], w->v, w->wvn, ORC_NK, o->h, grn, flag);
    if (o->grn_kind == 4) { /* REAL(4)/COMPLEX(4) table storage, WavDynMods.f90:204-223 */
        int k;
        for (k = 0; k < 4; ++k) {
            rkn[k] = (double)(float)rkn[k];
            grn[k] = (double)(float)creal(grn[k]) + I * (double)(float)cimag(grn[k]);
        }
    }
}

/* Per-source, per-image, per-system normal-derivative weight of DBC_MULTI_RIGHT. */
static zdouble dbc_weight(const orc_geom *g, const orc_opts *o, const orc_wave *w, int jel, int is, int ip,
                          double beta)
{
    int n = g->nelem;
    double xec[3] = {g->xyz_p[jel], g->xyz_p[jel + n], g->xyz_p[jel + 2 * n]}, xq, yq, zq;
    double e1 = g->dxyz[jel], e2 = g->dxyz[jel + n], e3 = g->dxyz[jel + 2 * n];
    zdouble dx, dy, dz;
    if (g->isx == 1 && g->isy == 0) {
        xq = T22(SY_, is, ip) * xec[0]; yq = T22(SX_, is, ip) * xec[1]; zq = xec[2];
        dinp(o, w, xq, yq, zq, beta, &dx, &dy, &dz);
        return T22(SY_, is, ip) * dx * e1 + T22(SX_, is, ip) * dy * e2 + dz * e3;
    }
    xq = T22(SX_, is, ip) * xec[0]; yq = T22(SY_, is, ip) * xec[1]; zq = xec[2];
    dinp(o, w, xq, yq, zq, beta, &dx, &dy, &dz);
    return T22(SX_, is, ip) * dx * e1 + T22(SY_, is, ip) * dy * e2 + dz * e3;
}

/* Mode weight of RBC_MULTI_RIGHT: TINRD(IS,MD,IP) += DUM * sign * DXYZ(JEL,MD). */
static double rbc_sign(const orc_geom *g, int is, int ip, int md)
{
    double sx = T22(SX_, is, ip), sy = T22(SY_, is, ip);
    if (g->isx == 1 && g->isy == 0) {
        switch (md) { case 1: return sy; case 2: return sx; case 3: return 1.0; case 4: return sx; case 5: return sy; default: return sy * sx; }
    }
    switch (md) { case 1: return sx; case 2: return sy; case 3: return 1.0; case 4: return sy; case 5: return sx; default: return sx * sy; }
}

/*
 * Fill one row of A (length n per system, column-major stride lda), of the
 * radiation RHS (6 nb columns per system) and diffraction RHS (per system,
 * per heading) for field point iel of the set (p, np): p = hull centres for
 * hull rows, lid centres for lid rows.  wdbc holds dbc_weight for all
 * (jel, is, ip, beta).
 */
static void assemble_row(const orc_geom *g, const orc_opts *o, const orc_wave *w, const double *p, int np, int iel,
                         int lid_row, int nbeta, const zdouble *wdbc, zdouble *arow, long lda, zdouble *brow,
                         long ldb, zdouble *drow, long ldd, double *rknbuf, zdouble *grnbuf)
{
    const int n = g->nelem, nsys = g->nsys, nb = g->nbody;
    int jel, is, ip, md, b, ib, j0;
    double dist, xi = p[iel], yi = p[iel + np], zi = p[iel + 2 * np];
    unsigned char *flags = (unsigned char *)malloc((size_t)n);

    /* CALGREEN_MULTI[_IRR] table entries for this row */
    for (jel = 0; jel < n; ++jel) {
        double xq = g->xyz_p[jel], yq = g->xyz_p[jel + n], zq = g->xyz_p[jel + 2 * n];
        dist = sqrt((xi - xq) * (xi - xq) + (yi - yq) * (yi - yq) + (zi - zq) * (zi - zq));
        flags[jel] = (dist <= 50.0 * g->pnsz[jel]) ? 1 : 0;
        for (is = 1; is <= nsys; ++is) {
            double xf[3];
            int tflag = flags[jel];
            field_point(g, p, np, iel, is, xf);
            if (lid_row) { /* CalGreenFuncMulti.f90:286-291 measures from the imaged point */
                double d2 = sqrt((xf[0] - xq) * (xf[0] - xq) + (xf[1] - yq) * (xf[1] - yq) + (xf[2] - zq) * (xf[2] - zq));
                tflag = (d2 <= 50.0 * g->pnsz[jel]) ? 1 : 0;
            }
            pair_tables(g, o, w, jel, xf, tflag, &rknbuf[4 * ((long)jel * nsys + is - 1)],
                        &grnbuf[4 * ((long)jel * nsys + is - 1)]);
        }
    }

    /* ASSB_LEFT: A(IEL,IEL) = 2 pi on hull rows (0 on lid rows), then pairs */
    for (ip = 1; ip <= nsys; ++ip)
        if (!lid_row) arow[(long)iel * lda + (long)(ip - 1) * lda * n] = 2.0 * PI;
    for (jel = 0; jel < n; ++jel) {
        double ear = g->ds[jel], e1 = g->dxyz[jel], e2 = g->dxyz[jel + n], e3 = g->dxyz[jel + 2 * n];
        for (is = 1; is <= nsys; ++is) {
            const double *rkn = &rknbuf[4 * ((long)jel * nsys + is - 1)];
            const zdouble *grn = &grnbuf[4 * ((long)jel * nsys + is - 1)];
            zdouble tindp;
            if (flags[jel]) tindp = (rkn[1] + grn[1] * ear) * e1 + (rkn[2] + grn[2] * ear) * e2 + (rkn[3] + grn[3] * ear) * e3;
            else tindp = (grn[1] * e1 + grn[2] * e2 + grn[3] * e3) * ear;
            for (ip = 1; ip <= nsys; ++ip) {
                zdouble *a = &arow[(long)jel * lda + (long)(ip - 1) * lda * n];
                *a = *a + T22(RXY_, is, ip) * tindp;
            }
        }
    }

    /* ASSB_RBC, per body: BTMP(MD,IP) over the body's source panels */
    j0 = 0;
    for (b = 0; b < nb; ++b) {
        zdouble btmp[6][2];
        memset(btmp, 0, sizeof(btmp));
        for (jel = j0; jel < j0 + g->body_nelem[b]; ++jel) {
            for (is = 1; is <= nsys; ++is) {
                const double *rkn = &rknbuf[4 * ((long)jel * nsys + is - 1)];
                const zdouble *grn = &grnbuf[4 * ((long)jel * nsys + is - 1)];
                zdouble dum = flags[jel] ? rkn[0] + grn[0] * g->ds[jel] : grn[0] * g->ds[jel];
                zdouble tinrd[6][2];
                memset(tinrd, 0, sizeof(tinrd));
                for (ip = 1; ip <= nsys; ++ip)
                    for (md = 1; md <= 6; ++md)
                        tinrd[md - 1][ip - 1] = tinrd[md - 1][ip - 1] + dum * rbc_sign(g, is, ip, md) * g->dxyz[jel + (long)n * (md - 1)];
                for (md = 0; md < 6; ++md)
                    for (ip = 0; ip < nsys; ++ip) btmp[md][ip] = btmp[md][ip] + tinrd[md][ip];
            }
        }
        for (md = 1; md <= 6; ++md)
            for (ip = 1; ip <= nsys; ++ip)
                for (is = 1; is <= nsys; ++is) {
                    zdouble *bb = &brow[(long)(6 * b + md - 1) * ldb + (long)(ip - 1) * ldb * 6 * nb];
                    *bb = *bb + T22(RXY_, ip, is) * btmp[md - 1][is - 1];
                }
        j0 += g->body_nelem[b];
    }

    /* ASSB_DBC, per heading */
    for (ib = 0; ib < nbeta; ++ib) {
        zdouble btmp[2] = {0.0, 0.0};
        for (jel = 0; jel < n; ++jel) {
            zdouble tinrd[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
            for (is = 1; is <= nsys; ++is) {
                const double *rkn = &rknbuf[4 * ((long)jel * nsys + is - 1)];
                const zdouble *grn = &grnbuf[4 * ((long)jel * nsys + is - 1)];
                zdouble d1 = flags[jel] ? rkn[0] + grn[0] * g->ds[jel] : grn[0] * g->ds[jel];
                for (ip = 1; ip <= nsys; ++ip) {
                    zdouble d2 = wdbc[(((long)ib * n + jel) * 2 + (is - 1)) * 2 + (ip - 1)];
                    tinrd[is - 1][ip - 1] = tinrd[is - 1][ip - 1] - d1 * d2;
                }
                for (ip = 0; ip < nsys; ++ip) btmp[ip] = btmp[ip] + tinrd[is - 1][ip];
            }
        }
        for (ip = 1; ip <= nsys; ++ip)
            for (is = 1; is <= nsys; ++is) {
                zdouble *dd = &drow[(long)(ip - 1) * ldd + (long)ib * ldd * nsys];
                *dd = *dd + T22(RXY_, ip, is) * btmp[is - 1];
            }
    }
    free(flags);
}

int32_t orc_assemble(const orc_geom *g, const orc_opts *o, const orc_wave *w, int32_t nbeta, const double *beta,
                     double *amat_d, double *brmat_d, double *bdmat_d)
{
    const int n = g->nelem, nsys = g->nsys, nb = g->nbody;
    const int nl = (o->irsp == 1) ? g->inelem : 0, tn = n + nl;
    zdouble *amat = (zdouble *)amat_d, *brmat = (zdouble *)brmat_d, *bdmat = (zdouble *)bdmat_d;
    zdouble *wdbc = (zdouble *)calloc((size_t)nbeta * n * 4, sizeof(zdouble));
    zdouble *afull = amat, *bfull = brmat, *dfull = bdmat;
    int ib, jel, is, ip, iel;
    int nthread = o->nthread > 0 ? o->nthread : 0;

    for (ib = 0; ib < nbeta; ++ib)
        for (jel = 0; jel < n; ++jel)
            for (is = 1; is <= nsys; ++is)
                for (ip = 1; ip <= nsys; ++ip)
                    wdbc[(((long)ib * n + jel) * 2 + (is - 1)) * 2 + (ip - 1)] = dbc_weight(g, o, w, jel, is, ip, beta[ib]);

    if (nl > 0) { /* extended (tn x n) system, normal equations afterwards */
        afull = (zdouble *)calloc((size_t)tn * n * nsys, sizeof(zdouble));
        bfull = (zdouble *)calloc((size_t)tn * 6 * nb * nsys, sizeof(zdouble));
        dfull = (zdouble *)calloc((size_t)tn * nsys * nbeta, sizeof(zdouble));
    } else {
        memset(amat, 0, sizeof(zdouble) * (size_t)n * n * nsys);
        memset(brmat, 0, sizeof(zdouble) * (size_t)n * 6 * nb * nsys);
        memset(bdmat, 0, sizeof(zdouble) * (size_t)n * nsys * nbeta);
    }

#pragma omp parallel num_threads(nthread > 0 ? nthread : omp_get_max_threads())
    {
        double *rknbuf = (double *)malloc(sizeof(double) * 4 * (size_t)n * nsys);
        zdouble *grnbuf = (zdouble *)malloc(sizeof(zdouble) * 4 * (size_t)n * nsys);
#pragma omp for schedule(dynamic, 16)
        for (iel = 0; iel < tn; ++iel) {
            int lid = iel >= n;
            const double *p = lid ? g->ixyz_p : g->xyz_p;
            int np = lid ? g->inelem : n, il = lid ? iel - n : iel;
            assemble_row(g, o, w, p, np, il, lid, nbeta, wdbc, afull + iel, tn, bfull + iel, tn, dfull + iel, tn,
                         rknbuf, grnbuf);
        }
        free(rknbuf);
        free(grnbuf);
    }

    if (nl > 0) { /* C = A^T A, D = A^T B (AssbMatx_irrMulti.f90:151-169, :300-315, :447-460) */
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthread > 0 ? nthread : omp_get_max_threads())
        for (ip = 0; ip < nsys; ++ip)
            for (iel = 0; iel < n; ++iel) {
                const zdouble *ai = afull + (long)ip * tn * n + (long)iel * tn;
                int j, k, md;
                for (j = 0; j < n; ++j) {
                    const zdouble *aj = afull + (long)ip * tn * n + (long)j * tn;
                    zdouble s = 0.0;
                    for (k = 0; k < tn; ++k) s = s + ai[k] * aj[k];
                    amat[(long)ip * n * n + (long)j * n + iel] = s;
                }
                for (md = 0; md < 6 * nb; ++md) {
                    const zdouble *bk = bfull + (long)ip * tn * 6 * nb + (long)md * tn;
                    zdouble s = 0.0;
                    for (k = 0; k < tn; ++k) s = s + bk[k] * ai[k];
                    brmat[(long)ip * n * 6 * nb + (long)md * n + iel] = s;
                }
                for (md = 0; md < nbeta; ++md) {
                    const zdouble *dk = dfull + ((long)md * nsys + ip) * tn;
                    zdouble s = 0.0;
                    for (k = 0; k < tn; ++k) s = s + dk[k] * ai[k];
                    bdmat[((long)md * nsys + ip) * n + iel] = s;
                }
            }
        free(afull);
        free(bfull);
        free(dfull);
    }
    free(wdbc);
    return 0;
}

/* Rows offset, offset+stride, ... of the hull system only (no lids, no
 * normal equations): the bounded sample the CPU-baseline timing uses.
 * Outputs have leading dimension nr = number of rows assembled (returned). */
int32_t orc_assemble_rows(const orc_geom *g, const orc_opts *o, const orc_wave *w, int32_t nbeta, const double *beta,
                          int32_t stride, int32_t offset, double *amat_d, double *brmat_d, double *bdmat_d)
{
    const int n = g->nelem, nsys = g->nsys, nb = g->nbody;
    int nr = 0, r;
    if (stride < 1 || offset < 0 || offset >= n) return 0;
    nr = (n - offset + stride - 1) / stride;
    zdouble *amat = (zdouble *)amat_d, *brmat = (zdouble *)brmat_d, *bdmat = (zdouble *)bdmat_d;
    zdouble *wdbc = (zdouble *)calloc((size_t)nbeta * n * 4, sizeof(zdouble));
    int ib, jel, is, ip;
    int nthread = o->nthread > 0 ? o->nthread : 0;
    for (ib = 0; ib < nbeta; ++ib)
        for (jel = 0; jel < n; ++jel)
            for (is = 1; is <= nsys; ++is)
                for (ip = 1; ip <= nsys; ++ip)
                    wdbc[(((long)ib * n + jel) * 2 + (is - 1)) * 2 + (ip - 1)] = dbc_weight(g, o, w, jel, is, ip, beta[ib]);
    memset(amat, 0, sizeof(zdouble) * (size_t)nr * n * nsys);
    memset(brmat, 0, sizeof(zdouble) * (size_t)nr * 6 * nb * nsys);
    memset(bdmat, 0, sizeof(zdouble) * (size_t)nr * nsys * nbeta);
#pragma omp parallel num_threads(nthread > 0 ? nthread : omp_get_max_threads())
    {
        double *rknbuf = (double *)malloc(sizeof(double) * 4 * (size_t)n * nsys);
        zdouble *grnbuf = (zdouble *)malloc(sizeof(zdouble) * 4 * (size_t)n * nsys);
#pragma omp for schedule(dynamic, 1)
        for (r = 0; r < nr; ++r)
            assemble_row(g, o, w, g->xyz_p, n, offset + r * stride, 0, nbeta, wdbc, amat + r, nr, brmat + r, nr,
                         bdmat + r, nr, rknbuf, grnbuf);
        free(rknbuf);
        free(grnbuf);
    }
    free(wdbc);
    return nr;
}

/* ------------------------------------------------------------------ */
/* Dense complex LU, ZGETRF/ZGETRS semantics                            */
/* ------------------------------------------------------------------ */
static inline double cabs1(zdouble z) { return fabs(creal(z)) + fabs(cimag(z)); }

int32_t orc_zgetrf(int32_t n, double *a_d, int32_t *ipiv, int32_t nthread)
{
    zdouble *a = (zdouble *)a_d;
    const int nb = 64;
    int k0, info = 0;
    int nth = nthread > 0 ? nthread : omp_get_max_threads();
    for (k0 = 0; k0 < n; k0 += nb) {
        int kb = (n - k0 < nb) ? n - k0 : nb, j, i, c;
        /* panel: columns k0..k0+kb-1 */
        for (j = k0; j < k0 + kb; ++j) {
            int p = j;
            double m = cabs1(a[(long)j * n + j]);
            for (i = j + 1; i < n; ++i)
                if (cabs1(a[(long)j * n + i]) > m) { m = cabs1(a[(long)j * n + i]); p = i; }
            ipiv[j] = p + 1;
            if (m == 0.0) { if (!info) info = j + 1; continue; }
            if (p != j)
                for (c = 0; c < n; ++c) {
                    zdouble t = a[(long)c * n + j];
                    a[(long)c * n + j] = a[(long)c * n + p];
                    a[(long)c * n + p] = t;
                }
            {
                zdouble r = 1.0 / a[(long)j * n + j];
                for (i = j + 1; i < n; ++i) a[(long)j * n + i] *= r;
            }
            for (c = j + 1; c < k0 + kb; ++c) {
                zdouble u = a[(long)c * n + j];
                for (i = j + 1; i < n; ++i) a[(long)c * n + i] -= a[(long)j * n + i] * u;
            }
        }
        /* U12 = L11^-1 A12 and A22 -= L21 U12, column by column */
#pragma omp parallel for schedule(dynamic, 4) num_threads(nth)
        for (c = k0 + kb; c < n; ++c) {
            zdouble *col = a + (long)c * n;
            int jj, ii;
            for (jj = k0; jj < k0 + kb; ++jj) {
                zdouble u = col[jj];
                const zdouble *l = a + (long)jj * n;
                for (ii = jj + 1; ii < k0 + kb; ++ii) col[ii] -= l[ii] * u;
            }
            for (jj = k0; jj < k0 + kb; ++jj) {
                zdouble u = col[jj];
                const zdouble *l = a + (long)jj * n;
                for (ii = k0 + kb; ii < n; ++ii) col[ii] -= l[ii] * u;
            }
        }
    }
    return info;
}

void orc_zgetrs(int32_t n, int32_t nrhs, const double *a_d, const int32_t *ipiv, double *b_d)
{
    const zdouble *a = (const zdouble *)a_d;
    zdouble *b = (zdouble *)b_d;
    int r;
#pragma omp parallel for schedule(static)
    for (r = 0; r < nrhs; ++r) {
        zdouble *x = b + (long)r * n;
        int i, j;
        for (i = 0; i < n; ++i) {
            int p = ipiv[i] - 1;
            if (p != i) { zdouble t = x[i]; x[i] = x[p]; x[p] = t; }
        }
        for (j = 0; j < n; ++j) {
            zdouble xj = x[j];
            const zdouble *l = a + (long)j * n;
            for (i = j + 1; i < n; ++i) x[i] -= l[i] * xj;
        }
        for (j = n - 1; j >= 0; --j) {
            const zdouble *u = a + (long)j * n;
            zdouble xj;
            x[j] = x[j] / u[j];
            xj = x[j];
            for (i = 0; i < j; ++i) x[i] -= u[i] * xj;
        }
    }
}

/* ------------------------------------------------------------------ */
/* Reductions                                                          */
/* ------------------------------------------------------------------ */
static double force_sign(const orc_geom *g, int ip, int k)
{ /* RX/RY pattern of RFORCE_MULTI / EFORCE_MULTI */
    const double *t = (g->isx == 1 && g->isy == 0) ? RX_ : RY_;
    switch (k) {
    case 1: return T22(t, ip, 1);
    case 2: return T22(t, ip, 2);
    case 3: return 1.0;
    case 4: return T22(t, ip, 2);
    case 5: return T22(t, ip, 1);
    default: return T22(t, ip, 1) * T22(t, ip, 2);
    }
}

void orc_forces(const orc_geom *g, const orc_opts *o, const orc_wave *w, int32_t nbeta, const double *beta,
                const double *xrad_d, const double *xdif_d, double *amas, double *bdmp, double *exfc_d)
{
    const int n = g->nelem, nsys = g->nsys, nb = g->nbody, ndof = 6 * nb;
    const zdouble *xrad = (const zdouble *)xrad_d, *xdif = (const zdouble *)xdif_d;
    zdouble *exfc = (zdouble *)exfc_d;
    zdouble *mx = (zdouble *)malloc(sizeof(zdouble) * (size_t)n * nsys);
    int bm, bn, md, k, iel, ip, is, ib, m0, mcount;

    /* RFORCE_MULTI for every (body M, body N) block, HAMS_Prog.f90:686-690 */
    m0 = 0;
    for (bm = 0; bm < nb; ++bm) {
        mcount = g->body_nelem[bm];
        for (bn = 0; bn < nb; ++bn) {
            double am[6][6], bd[6][6];
            memset(am, 0, sizeof(am));
            memset(bd, 0, sizeof(bd));
            for (md = 1; md <= 6; ++md) {
                /* MXPOT(IEL, 6(N-1)+MD, IP) = (1/NSYS) sum_IS X(IEL,MD,IS) RXY(IP,IS) */
                for (iel = m0; iel < m0 + mcount; ++iel)
                    for (ip = 1; ip <= nsys; ++ip) {
                        zdouble s = 0.0;
                        for (is = 1; is <= nsys; ++is)
                            s = s + xrad[(long)(is - 1) * n * ndof + (long)(6 * bn + md - 1) * n + iel] * T22(RXY_, ip, is);
                        mx[(long)(ip - 1) * n + iel] = s / nsys;
                    }
                for (iel = m0; iel < m0 + mcount; ++iel)
                    for (ip = 1; ip <= nsys; ++ip) {
                        zdouble p = mx[(long)(ip - 1) * n + iel];
                        zdouble rphi = I * o->rho * p * g->ds[iel];
                        zdouble iphi = I * o->rho * w->w1 * p * g->ds[iel];
                        for (k = 1; k <= 6; ++k) {
                            double sgn = force_sign(g, ip, k), nk = g->dxyz[iel + (long)n * (k - 1)];
                            if (k == 3) {
                                am[k - 1][md - 1] += cimag(rphi * nk);
                                bd[k - 1][md - 1] -= creal(iphi * nk);
                            } else {
                                am[k - 1][md - 1] += cimag(rphi * sgn * nk);
                                bd[k - 1][md - 1] -= creal(iphi * sgn * nk);
                            }
                        }
                    }
            }
            for (k = 0; k < 6; ++k)
                for (md = 0; md < 6; ++md) {
                    amas[(long)(6 * bn + md) * ndof + 6 * bm + k] = am[k][md];
                    bdmp[(long)(6 * bn + md) * ndof + 6 * bm + k] = bd[k][md];
                }
        }
        m0 += mcount;
    }

    /* EFORCE_MULTI per heading and body, HAMS_Prog.f90:706-722 */
    for (ib = 0; ib < nbeta; ++ib) {
        for (iel = 0; iel < n; ++iel)
            for (ip = 1; ip <= nsys; ++ip) {
                zdouble s = 0.0;
                for (is = 1; is <= nsys; ++is)
                    s = s + xdif[((long)ib * nsys + (is - 1)) * n + iel] * T22(RXY_, ip, is);
                mx[(long)(ip - 1) * n + iel] = s / nsys;
            }
        m0 = 0;
        for (bm = 0; bm < nb; ++bm) {
            zdouble force[6][2];
            memset(force, 0, sizeof(force));
            for (iel = m0; iel < m0 + g->body_nelem[bm]; ++iel)
                for (ip = 1; ip <= nsys; ++ip) {
                    const double *t = (g->isx == 1 && g->isy == 0) ? RX_ : RY_;
                    double xp = T22(t, ip, 1) * g->xyz_p[iel], yp = T22(t, ip, 2) * g->xyz_p[iel + n],
                           zp = g->xyz_p[iel + 2 * n];
                    zdouble phi;
                    if (o->isol == 1) phi = (mx[(long)(ip - 1) * n + iel] + vinp(o, w, xp, yp, zp, beta[ib])) * g->ds[iel];
                    else phi = mx[(long)(ip - 1) * n + iel] * g->ds[iel];
                    for (k = 1; k <= 6; ++k) {
                        double nk = g->dxyz[iel + (long)n * (k - 1)];
                        if (k == 3) force[k - 1][ip - 1] += phi * nk;
                        else force[k - 1][ip - 1] += phi * force_sign(g, ip, k) * nk;
                    }
                }
            for (k = 0; k < 6; ++k) {
                zdouble e = 0.0;
                for (ip = 0; ip < nsys; ++ip) e = e + force[k][ip];
                e = I * w->w1 * o->rho * e;
                exfc[(long)(6 * bm + k) * nbeta + ib] = e;
            }
            m0 += g->body_nelem[bm];
        }
    }
    free(mx);
}

/* ------------------------------------------------------------------ */
/* Whole frequency                                                      */
/* ------------------------------------------------------------------ */
int32_t orc_solve_frequency(const orc_geom *g, const orc_opts *o, const orc_wave *w, int32_t nbeta,
                            const double *beta, double *amas, double *bdmp, double *exfc)
{
    const int n = g->nelem, nsys = g->nsys, ndof = 6 * g->nbody;
    double *a = (double *)malloc(sizeof(double) * 2 * (size_t)n * n * nsys);
    double *b = (double *)malloc(sizeof(double) * 2 * (size_t)n * ndof * nsys);
    double *d = (double *)malloc(sizeof(double) * 2 * (size_t)n * nsys * (nbeta > 0 ? nbeta : 1));
    int32_t *ipiv = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
    int info = 0, ip, ib;
    orc_assemble(g, o, w, nbeta, beta, a, b, d);
    for (ip = 0; ip < nsys; ++ip) {
        double *aip = a + 2L * n * n * ip;
        int inf = orc_zgetrf(n, aip, ipiv, o->nthread);
        if (inf && !info) info = inf;
        orc_zgetrs(n, ndof, aip, ipiv, b + 2L * n * ndof * ip);
        for (ib = 0; ib < nbeta; ++ib) orc_zgetrs(n, 1, aip, ipiv, d + 2L * n * (ib * nsys + ip));
    }
    orc_forces(g, o, w, nbeta, beta, b, d, amas, bdmp, exfc);
    free(a);
    free(b);
    free(d);
    free(ipiv);
    return info;
}

/* ------------------------------------------------------------------ */
/* Single evaluations for the unit tests                               */
/* ------------------------------------------------------------------ */
void orc_fingreen3d_c(double xf, double xp, double yf, double yp, double zf, double zp, double v, const double *wvn,
                      int32_t nk, double h, double *grn, int32_t flag)
{
    orc_fingreen3d(xf, xp, yf, yp, zf, zp, v, wvn, nk, h, (zdouble *)grn, flag);
}
void orc_infgreen3d_c(double xf, double xp, double yf, double yp, double zf, double zp, double v, double *grn,
                      int32_t flag)
{
    orc_infgreen3d(xf, xp, yf, yp, zf, zp, v, (zdouble *)grn, flag);
}
int32_t orc_fin_branch_c(double rr, double h) { return orc_fin_branch(rr, h); }
void orc_sglint_c(const orc_geom *g, int32_t jel, const double *xf, double *out)
{
    rankine_pair(g, jel, xf, &out[0], &out[1]);
}
/* which: 0 erf, 1 E1, 2 Ei, 3 K0/K1, 4 J0/J1/Y0/Y1, 5..7 E_n (n=which-5) */
void orc_special_c(int32_t which, double x, double *out)
{
    switch (which) {
    case 0: orc_error(x, out); break;
    case 1: orc_e1xa(x, out); break;
    case 2: orc_eix(x, out); break;
    case 3: orc_ik01a(x, &out[0], &out[1]); break;
    case 4: orc_jy01b(x, &out[0], &out[1], &out[2], &out[3]); break;
    default: orc_enxa(which - 5, x, out); break;
    }
}
