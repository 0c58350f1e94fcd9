/*
 * io.c -- ControlFile.in / .pnl reader and HAMS-format writers of the oracle.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle_internal.h).
 *
 * Restates ReadControlFile (src/InputFiles.f90:46-224), the mesh readers
 * ReadBodyMesh[Multi]/ReadWTPLMesh[Multi] (src/ReadPanelMesh.f90:46-99,
 * src/ReadPanelMeshMulti.f90:46-111, including the LCS rotation and
 * translation on read), the generalized-mode normal override
 * (ReadPanelMeshMulti.f90:170-200) and the frequency loop of
 * src/HAMS_Prog.f90:613-733 with the OAMASS/ODAMPING/OEXFOR writers of
 * src/PotentWavForceMulti.f90 (formats 1000 and 1010).
 */
#include <ctype.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "hams_oracle.h"
#include "oracle_internal.h"

/* ---- line reader with Fortran record semantics ---- */
typedef struct {
    char **lines;
    int n, cur;
} reader;

static int rd_open(reader *r, const char *path)
{
    FILE *f = fopen(path, "r");
    char buf[4096];
    int cap = 256;
    r->n = 0;
    r->cur = 0;
    r->lines = NULL;
    if (!f) return -1;
    r->lines = (char **)malloc(sizeof(char *) * cap);
    while (fgets(buf, sizeof(buf), f)) {
        size_t l = strlen(buf);
        while (l && (buf[l - 1] == '\n' || buf[l - 1] == '\r')) buf[--l] = 0;
        if (r->n == cap) { cap *= 2; r->lines = (char **)realloc(r->lines, sizeof(char *) * cap); }
        r->lines[r->n++] = strdup(buf);
    }
    fclose(f);
    return 0;
}
static void rd_close(reader *r)
{
    int i;
    for (i = 0; i < r->n; ++i) free(r->lines[i]);
    free(r->lines);
}
static const char *rd_next(reader *r) { return r->cur < r->n ? r->lines[r->cur++] : NULL; }

/* Field [skip, skip+w) of a record, blank padded, blanks removed (BN). */
static void field(const char *line, int skip, int w, char *out)
{
    int len = (int)strlen(line), i, k = 0;
    for (i = skip; i < skip + w && i < len; ++i) {
        char c = line[i];
        if (c == '\t') c = ' ';
        if (c != ' ') out[k++] = c;
    }
    out[k] = 0;
}

/* Fortran F/E/D input editing with d implied decimals. */
static double fortran_real(const char *s, int d)
{
    char buf[128] = {0};
    int i, k = 0, has_point = 0;
    double v;
    if (!*s) return 0.0;
    for (i = 0; s[i] && k < 126; ++i) {
        char c = s[i];
        if (c == 'd' || c == 'D' || c == 'q' || c == 'Q') c = 'E';
        if (c == '.') has_point = 1;
        buf[k++] = c;
    }
    buf[k] = 0;
    /* an exponent written as a bare sign, e.g. 1.0+3 */
    for (i = 1; buf[i]; ++i)
        if ((buf[i] == '+' || buf[i] == '-') && isdigit((unsigned char)buf[i - 1])) {
            memmove(buf + i + 1, buf + i, strlen(buf + i) + 1);
            buf[i] = 'E';
            break;
        }
    v = strtod(buf, NULL);
    if (!has_point) {
        int e;
        for (e = 0; e < d; ++e) v /= 10.0;
    }
    return v;
}
static double read_f(reader *r, int skip, int w, int d)
{
    char f[256];
    const char *l = rd_next(r);
    field(l ? l : "", skip, w, f);
    return fortran_real(f, d);
}
static int read_i(reader *r, int skip, int w)
{
    char f[256];
    const char *l = rd_next(r);
    field(l ? l : "", skip, w, f);
    return (int)strtol(f, NULL, 10);
}

/* List-directed read of n reals spanning records. */
static int read_list(reader *r, int n, double *v)
{
    int got = 0;
    while (got < n) {
        const char *l = rd_next(r);
        char buf[4096], *tok, *save;
        if (!l) return -1;
        strncpy(buf, l, sizeof(buf) - 1);
        buf[sizeof(buf) - 1] = 0;
        for (tok = strtok_r(buf, " \t,", &save); tok && got < n; tok = strtok_r(NULL, " \t,", &save)) {
            char *p;
            for (p = tok; *p; ++p)
                if (*p == 'd' || *p == 'D') *p = 'E';
            v[got++] = strtod(tok, NULL);
        }
    }
    return 0;
}

/* ---- .pnl mesh ---- */
typedef struct {
    int nelem, ntnd, isx, isy;
    double *xyz; /* ntnd x 3, row-major */
    int *ncn, *ncon; /* ncon nelem x 4 row-major */
} mesh;

static int read_pnl(const char *path, mesh *m, int check_lid)
{
    reader r;
    double v[8];
    int i, j;
    if (rd_open(&r, path)) return -1;
    rd_next(&r); rd_next(&r); rd_next(&r);
    if (read_list(&r, 4, v)) { rd_close(&r); return -2; }
    m->nelem = (int)v[0];
    m->ntnd = (int)v[1];
    m->isx = (int)v[2];
    m->isy = (int)v[3];
    rd_next(&r); rd_next(&r);
    m->xyz = (double *)malloc(sizeof(double) * 3 * m->ntnd);
    m->ncn = (int *)malloc(sizeof(int) * m->nelem);
    m->ncon = (int *)calloc(4 * (size_t)m->nelem, sizeof(int));
    for (i = 0; i < m->ntnd; ++i) {
        if (read_list(&r, 4, v)) { rd_close(&r); return -3; }
        m->xyz[3 * i] = v[1];
        m->xyz[3 * i + 1] = v[2];
        m->xyz[3 * i + 2] = v[3];
        if (check_lid && fabs(v[3]) > F4(1.E-10)) { rd_close(&r); return -4; }
    }
    rd_next(&r); rd_next(&r); rd_next(&r);
    for (i = 0; i < m->nelem; ++i) {
        const char *l = rd_next(&r);
        char buf[1024], *tok, *save;
        int vals[6], k = 0;
        if (!l) { rd_close(&r); return -5; }
        strncpy(buf, l, sizeof(buf) - 1);
        buf[sizeof(buf) - 1] = 0;
        for (tok = strtok_r(buf, " \t,", &save); tok && k < 6; tok = strtok_r(NULL, " \t,", &save)) vals[k++] = atoi(tok);
        if (k < 2 || k < 2 + vals[1] || (vals[1] != 3 && vals[1] != 4)) { rd_close(&r); return -6; }
        m->ncn[i] = vals[1];
        for (j = 0; j < vals[1]; ++j) m->ncon[4 * i + j] = vals[2 + j];
    }
    rd_close(&r);
    return 0;
}
static void free_mesh(mesh *m)
{
    free(m->xyz);
    free(m->ncn);
    free(m->ncon);
}

/* ---- deck ---- */
int32_t orc_load_deck(const char *dir, orc_deck *d)
{
    char path[1024], bodycheck[256];
    reader r;
    int npet, ifs, i, b, nb, nl = 0;
    mesh *hm, *lm;
    orc_geom *g = &d->geom;

    memset(d, 0, sizeof(*d));
    snprintf(path, sizeof(path), "%s/ControlFile.in", dir);
    if (rd_open(&r, path)) return -1;
    rd_next(&r); rd_next(&r);
    d->opts.h = read_f(&r, 14, 30, 15);
    rd_next(&r); rd_next(&r);
    d->sybo = read_i(&r, 27, 16);
    d->inft = read_i(&r, 25, 16);
    d->ouft = read_i(&r, 25, 17);
    npet = read_i(&r, 26, 16);
    ifs = (d->sybo == 1) ? 2 : 0;
    if (npet > 0) {
        d->nper = ifs + npet;
        d->wvnb = (double *)calloc(d->nper, sizeof(double));
        read_list(&r, npet, d->wvnb + ifs);
    } else {
        double wk1, dwk;
        npet = -npet;
        d->nper = ifs + npet;
        d->wvnb = (double *)calloc(d->nper, sizeof(double));
        wk1 = read_f(&r, 27, 30, 15);
        dwk = read_f(&r, 19, 30, 15);
        for (i = ifs; i < d->nper; ++i) d->wvnb[i] = wk1 + (i - ifs) * dwk;
    }
    rd_next(&r); rd_next(&r);
    {
        const char *l = rd_next(&r);
        strncpy(bodycheck, l ? l : "", sizeof(bodycheck) - 1);
        bodycheck[sizeof(bodycheck) - 1] = 0;
    }
    nb = strstr(bodycheck, "multi") ? read_i(&r, 24, 16) : 1;
    if (nb < 1 || nb > ORC_MAXBODY) { rd_close(&r); return -2; }
    g->nbody = nb;
    d->lcs = (double *)calloc(4 * (size_t)nb, sizeof(double));
    if (nb > 1) {
        for (b = 0; b < nb; ++b) {
            const char *l = rd_next(&r);
            char f[64];
            int k;
            for (k = 0; k < 4; ++k) {
                field(l ? l : "", 26 + 12 * k, 12, f);
                d->lcs[b + nb * k] = fortran_real(f, 3);
            }
        }
        rd_next(&r); rd_next(&r); rd_next(&r);
    }
    d->nbeta = read_i(&r, 23, 16);
    if (d->nbeta > 0) {
        d->wvhd = (double *)calloc(d->nbeta, sizeof(double));
        read_list(&r, d->nbeta, d->wvhd);
    } else {
        double b1, db;
        d->nbeta = -d->nbeta;
        d->wvhd = (double *)calloc(d->nbeta, sizeof(double));
        b1 = read_f(&r, 20, 30, 15);
        db = read_f(&r, 17, 30, 15);
        for (i = 0; i < d->nbeta; ++i) d->wvhd[i] = b1 + i * db;
    }
    rd_next(&r); rd_next(&r);
    d->xr = (double *)calloc(3 * (size_t)nb, sizeof(double));
    for (b = 0; b < nb; ++b) {
        const char *l = rd_next(&r);
        char f[64];
        int k;
        for (k = 0; k < 3; ++k) {
            field(l ? l : "", 28 + 12 * k, 12, f);
            d->xr[b + nb * k] = fortran_real(f, 3);
        }
    }
    d->refl = read_f(&r, 26, 30, 15);
    d->opts.isol = read_i(&r, 26, 16);
    d->opts.irsp = read_i(&r, 23, 16);
    d->opts.nthread = read_i(&r, 23, 16);
    d->isolv = 1;
    {
        const char *l = r.cur < r.n ? r.lines[r.cur] : NULL;
        if (l && strstr(l, "Solver_type")) {
            char f[64];
            rd_next(&r);
            field(l, 26, 16, f);
            d->isolv = (int)strtol(f, NULL, 10);
            if (d->isolv < 1 || d->isolv > 2) d->isolv = 1;
        }
    }
    rd_close(&r);

    /* constants of Const_mod (WavDynMods.f90:146) and Initialisation (HydroStatic*.f90) */
    d->opts.rho = 1000.0;
    d->opts.g = 9.80665;
    d->opts.xw[0] = d->opts.xw[1] = 0.0;
    d->opts.amp = 1.0;
    d->opts.grn_kind = 8;

    /* meshes */
    hm = (mesh *)calloc(nb, sizeof(mesh));
    lm = (mesh *)calloc(nb, sizeof(mesh));
    g->nelem = g->ntnd = 0;
    g->body_nelem = (int32_t *)calloc(nb, sizeof(int32_t));
    g->body_inelem = (int32_t *)calloc(nb, sizeof(int32_t));
    for (b = 0; b < nb; ++b) {
        if (nb == 1) snprintf(path, sizeof(path), "%s/HullMesh.pnl", dir);
        else snprintf(path, sizeof(path), "%s/HullMesh_%d.pnl", dir, b + 1);
        if (read_pnl(path, &hm[b], 0)) return -3;
        g->isx = hm[b].isx;
        g->isy = hm[b].isy;
        g->body_nelem[b] = hm[b].nelem;
        g->nelem += hm[b].nelem;
        g->ntnd += hm[b].ntnd;
        if (d->opts.irsp) {
            if (nb == 1) snprintf(path, sizeof(path), "%s/WaterPlaneMesh.pnl", dir);
            else snprintf(path, sizeof(path), "%s/WaterPlaneMesh_%d.pnl", dir, b + 1);
            if (read_pnl(path, &lm[b], 1) == 0) {
                g->body_inelem[b] = lm[b].nelem;
                g->inelem += lm[b].nelem;
                g->intnd += lm[b].ntnd;
                nl = 1;
            } else if (nb == 1) {
                return -4;
            }
        }
    }
    if (g->isx == 1 && g->isy == 1) return -5;
    g->nsys = (g->isx == 0 && g->isy == 0) ? 1 : 2;
    (void)nl;

    {
        int n = g->nelem, nt = g->ntnd, ni = g->inelem, nti = g->intnd, off_e = 0, off_n = 0, ioff_e = 0, ioff_n = 0;
        g->xyz = (double *)calloc(3 * (size_t)nt, sizeof(double));
        g->ncn = (int32_t *)calloc(n, sizeof(int32_t));
        g->ncon = (int32_t *)calloc(4 * (size_t)n, sizeof(int32_t));
        g->xyz_p = (double *)calloc(3 * (size_t)n, sizeof(double));
        g->ds = (double *)calloc(n, sizeof(double));
        g->pnsz = (double *)calloc(n, sizeof(double));
        g->dxyz = (double *)calloc(6 * (size_t)n, sizeof(double));
        if (ni > 0) {
            g->ixyz = (double *)calloc(3 * (size_t)nti, sizeof(double));
            g->incn = (int32_t *)calloc(ni, sizeof(int32_t));
            g->incon = (int32_t *)calloc(4 * (size_t)ni, sizeof(int32_t));
            g->ixyz_p = (double *)calloc(3 * (size_t)ni, sizeof(double));
            g->ids = (double *)calloc(ni, sizeof(double));
            g->ipnsz = (double *)calloc(ni, sizeof(double));
            g->idxyz = (double *)calloc(6 * (size_t)ni, sizeof(double));
        }
        for (b = 0; b < nb; ++b) {
            double c = cos(d->lcs[b + 3 * nb]), s = sin(d->lcs[b + 3 * nb]);
            for (i = 0; i < hm[b].ntnd; ++i) {
                double x = hm[b].xyz[3 * i], y = hm[b].xyz[3 * i + 1];
                if (nb > 1) {
                    g->xyz[off_n + i] = 0.0 + d->lcs[b] + c * x - s * y;
                    g->xyz[off_n + i + nt] = 0.0 + d->lcs[b + nb] + s * x + c * y;
                } else {
                    g->xyz[off_n + i] = x;
                    g->xyz[off_n + i + nt] = y;
                }
                g->xyz[off_n + i + 2 * nt] = hm[b].xyz[3 * i + 2];
            }
            for (i = 0; i < hm[b].nelem; ++i) {
                int k;
                g->ncn[off_e + i] = hm[b].ncn[i];
                for (k = 0; k < 4; ++k)
                    g->ncon[off_e + i + (size_t)n * k] = hm[b].ncon[4 * i + k] ? hm[b].ncon[4 * i + k] + off_n : 0;
            }
            if (ni > 0 && g->body_inelem[b] > 0) {
                for (i = 0; i < lm[b].ntnd; ++i) {
                    double x = lm[b].xyz[3 * i], y = lm[b].xyz[3 * i + 1];
                    if (nb > 1) {
                        g->ixyz[ioff_n + i] = 0.0 + d->lcs[b] + c * x - s * y;
                        g->ixyz[ioff_n + i + nti] = 0.0 + d->lcs[b + nb] + s * x + c * y;
                    } else {
                        g->ixyz[ioff_n + i] = x;
                        g->ixyz[ioff_n + i + nti] = y;
                    }
                    g->ixyz[ioff_n + i + 2 * nti] = lm[b].xyz[3 * i + 2];
                }
                for (i = 0; i < lm[b].nelem; ++i) {
                    int k;
                    g->incn[ioff_e + i] = lm[b].ncn[i];
                    for (k = 0; k < 4; ++k)
                        g->incon[ioff_e + i + (size_t)ni * k] = lm[b].ncon[4 * i + k] ? lm[b].ncon[4 * i + k] + ioff_n : 0;
                }
                ioff_e += lm[b].nelem;
                ioff_n += lm[b].ntnd;
            }
            off_e += hm[b].nelem;
            off_n += hm[b].ntnd;
        }
    }
    for (b = 0; b < nb; ++b) {
        free_mesh(&hm[b]);
        if (lm[b].xyz) free_mesh(&lm[b]);
    }
    free(hm);
    free(lm);

    orc_geom_prepare(g, d->xr);

    /* generalized modes: gen_mod_{body}_{dof}.txt override dxyz */
    {
        int i0 = 0;
        for (b = 0; b < nb; ++b) {
            int dof;
            for (dof = 1; dof <= 6; ++dof) {
                FILE *f;
                if (nb == 1) snprintf(path, sizeof(path), "%s/gen_mod_1_%d.txt", dir, dof);
                else snprintf(path, sizeof(path), "%s/gen_mod_%d_%d.txt", dir, b + 1, dof);
                f = fopen(path, "r");
                if (!f) continue;
                for (i = 0; i < g->body_nelem[b]; ++i) {
                    int pid;
                    double val;
                    char line[512], *p;
                    if (!fgets(line, sizeof(line), f)) break;
                    for (p = line; *p; ++p)
                        if (*p == 'd' || *p == 'D') *p = 'E';
                    if (sscanf(line, "%d %lf", &pid, &val) != 2) break;
                    g->dxyz[i0 + pid - 1 + (size_t)g->nelem * (dof - 1)] = val;
                }
                fclose(f);
            }
            i0 += g->body_nelem[b];
        }
    }
    return 0;
}

void orc_free_deck(orc_deck *d)
{
    orc_geom *g = &d->geom;
    free(g->xyz); free(g->ncn); free(g->ncon); free(g->xyz_p); free(g->ds); free(g->pnsz); free(g->dxyz);
    free(g->body_nelem); free(g->body_inelem);
    free(g->ixyz); free(g->incn); free(g->incon); free(g->ixyz_p); free(g->ids); free(g->ipnsz); free(g->idxyz);
    free(d->wvnb); free(d->wvhd); free(d->xr); free(d->lcs);
    memset(d, 0, sizeof(*d));
}

/* Fortran Ew.d output (0.ddddE+xx form). */
static void fmt_e(char *out, int w, int dg, double v)
{
    char m[64], body[40];
    int e, k, neg = v < 0.0;
    if (v == 0.0) {
        char z[64];
        snprintf(z, sizeof(z), "0.%0*dE+00", dg, 0);
        snprintf(out, 64, "%*s", w, z);
        return;
    }
    if (isnan(v) || isinf(v)) { /* the Fortran runtime's spelling, right-aligned */
        snprintf(out, 64, "%*s", w, isnan(v) ? "NaN" : (v < 0.0 ? "-Infinity" : "Infinity"));
        return;
    }
    snprintf(m, sizeof(m), "%.*e", dg - 1, fabs(v));
    e = atoi(strchr(m, 'e') + 1) + 1;
    k = 0;
    body[k++] = '0';
    body[k++] = '.';
    body[k++] = m[0];
    {
        const char *p = m + 2;
        while (*p && *p != 'e') body[k++] = *p++;
    }
    body[k] = 0;
    {
        char full[56];
        if (e >= -99 && e <= 99) snprintf(full, sizeof(full), "%s%sE%c%02d", neg ? "-" : "", body, e < 0 ? '-' : '+', abs(e));
        else snprintf(full, sizeof(full), "%s%s%c%03d", neg ? "-" : "", body, e < 0 ? '-' : '+', abs(e));
        snprintf(out, 64, "%*s", w, full);
    }
}

int32_t orc_run_case(const char *inputdir, const char *outputdir, int32_t grn_kind, int32_t nthread)
{
    orc_deck d;
    int rc = orc_load_deck(inputdir, &d), kk, md, ib, b1, b2, nb;
    FILE *fam[6], *fdm[6], *fex[6];
    char path[1024], e[64];
    double *beta;
    if (rc) return rc;
    d.opts.grn_kind = grn_kind;
    if (nthread > 0) d.opts.nthread = nthread;
    nb = d.geom.nbody;
    for (md = 0; md < 6; ++md) {
        snprintf(path, sizeof(path), "%s/OAMASS%d.txt", outputdir, md + 1);
        fam[md] = fopen(path, "w");
        snprintf(path, sizeof(path), "%s/ODAMPING%d.txt", outputdir, md + 1);
        fdm[md] = fopen(path, "w");
        snprintf(path, sizeof(path), "%s/OEXFOR%d.txt", outputdir, md + 1);
        fex[md] = fopen(path, "w");
        if (!fam[md] || !fdm[md] || !fex[md]) return -10;
    }
    beta = (double *)malloc(sizeof(double) * d.nbeta);
    for (ib = 0; ib < d.nbeta; ++ib) beta[ib] = d.wvhd[ib] * ORC_PI / 180.0;
    for (kk = 0; kk < d.nper; ++kk) {
        orc_wave w;
        int ndof = 6 * nb;
        double *amas = (double *)calloc((size_t)ndof * ndof, sizeof(double));
        double *bdmp = (double *)calloc((size_t)ndof * ndof, sizeof(double));
        double *exfc = (double *)calloc(2 * (size_t)ndof * d.nbeta, sizeof(double));
        orc_wave_props(d.inft, d.wvnb[kk], d.opts.h, d.opts.g, d.sybo == 1 && kk < 2 ? kk + 1 : 0, &w);
        orc_solve_frequency(&d.geom, &d.opts, &w, d.nbeta, beta, amas, bdmp, exfc);
        /* RFORCE_MULTI writes, body pair (M,N) outer, row MD1 per file */
        for (b1 = 0; b1 < nb; ++b1)
            for (b2 = 0; b2 < nb; ++b2)
                for (md = 0; md < 6; ++md) {
                    int c;
                    fprintf(fam[md], "%7.3f %7.3f ", w.wk, w.w1);
                    fprintf(fdm[md], "%7.3f %7.3f ", w.wk, w.w1);
                    for (c = 0; c < 6; ++c) {
                        fmt_e(e, 14, 5, amas[(size_t)(6 * b2 + c) * ndof + 6 * b1 + md]);
                        fputs(e, fam[md]);
                        fmt_e(e, 14, 5, bdmp[(size_t)(6 * b2 + c) * ndof + 6 * b1 + md]);
                        fputs(e, fdm[md]);
                    }
                    fputc('\n', fam[md]);
                    fputc('\n', fdm[md]);
                }
        /* EFORCE_MULTI writes, heading outer, body inner */
        for (ib = 0; ib < d.nbeta; ++ib)
            for (b1 = 0; b1 < nb; ++b1)
                for (md = 0; md < 6; ++md) {
                    size_t idx = (size_t)(6 * b1 + md) * d.nbeta + ib;
                    fprintf(fex[md], "%7.3f %7.3f ", w.wk, w.w1);
                    fmt_e(e, 14, 6, exfc[2 * idx]);
                    fputs(e, fex[md]);
                    fmt_e(e, 14, 6, exfc[2 * idx + 1]);
                    fputs(e, fex[md]);
                    fputc('\n', fex[md]);
                }
        free(amas);
        free(bdmp);
        free(exfc);
    }
    for (md = 0; md < 6; ++md) {
        fclose(fam[md]);
        fclose(fdm[md]);
        fclose(fex[md]);
    }
    free(beta);
    orc_free_deck(&d);
    return 0;
}
