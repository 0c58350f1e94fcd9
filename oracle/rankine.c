/*
 * rankine.c -- analytic 1/r source integral over a flat panel.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle_internal.h).
 *
 * Restates SGLINTBD_TRI / SGLINTBD_QUAD of src/SingularIntgr.f90 (identical
 * arithmetic in src/SingularIntgrMulti.f90:44,252): J.N. Newman (1986),
 * "Distributions of sources and normal dipoles over a quadrilateral panel".
 * The triangle and quadrilateral forms keep the reference's opposite sign
 * conventions (SingularIntgr.f90:200-210 versus :430-440).
 */
#include "oracle_internal.h"

/* SGLINTBD_TRI, SingularIntgr.f90:44-245 (one triangle, IRR=1 path). */
void orc_sglint_tri(const double xf[3], const double xq[3][3], double *sij, double dij[3])
{
    double xv[3][3], p12[3], p13[3], po[3], po3[3], po1[3], po2[3], pof[3];
    double ui[3], uj[3], uk[3], ksi[4], eta[4];
    double alfa, x, y, z, st, sxt, syt, szt, n12, n3;
    int i, j;

    for (i = 0; i < 3; ++i)
        for (j = 0; j < 3; ++j) xv[i][j] = xq[i][j];
    *sij = 0.0;
    dij[0] = dij[1] = dij[2] = 0.0;

    for (j = 0; j < 3; ++j) {
        p12[j] = xv[1][j] - xv[0][j];
        p13[j] = xv[2][j] - xv[0][j];
    }
    alfa = (p12[0] * p13[0] + p12[1] * p13[1] + p12[2] * p13[2]) / (p12[0] * p12[0] + p12[1] * p12[1] + p12[2] * p12[2]);
    for (j = 0; j < 3; ++j) po[j] = xv[0][j] + alfa * p12[j];
    for (j = 0; j < 3; ++j) po3[j] = xv[2][j] - po[j];
    n12 = sqrt(p12[0] * p12[0] + p12[1] * p12[1] + p12[2] * p12[2]);
    n3 = sqrt(po3[0] * po3[0] + po3[1] * po3[1] + po3[2] * po3[2]);
    for (j = 0; j < 3; ++j) {
        ui[j] = p12[j] / n12;
        uj[j] = po3[j] / n3;
    }
    uk[0] = ui[1] * uj[2] - ui[2] * uj[1];
    uk[1] = ui[2] * uj[0] - ui[0] * uj[2];
    uk[2] = ui[0] * uj[1] - ui[1] * uj[0];
    for (j = 0; j < 3; ++j) pof[j] = xf[j] - po[j];
    x = ui[0] * pof[0] + ui[1] * pof[1] + ui[2] * pof[2];
    y = uj[0] * pof[0] + uj[1] * pof[1] + uj[2] * pof[2];
    z = uk[0] * pof[0] + uk[1] * pof[1] + uk[2] * pof[2];
    for (j = 0; j < 3; ++j) {
        po1[j] = xv[0][j] - po[j];
        po2[j] = xv[1][j] - po[j];
    }
    ksi[0] = -copysign(1.0, alfa) * sqrt(po1[0] * po1[0] + po1[1] * po1[1] + po1[2] * po1[2]);
    eta[0] = 0.0;
    ksi[1] = 0.0;
    eta[1] = sqrt(po3[0] * po3[0] + po3[1] * po3[1] + po3[2] * po3[2]);
    ksi[2] = sqrt(po2[0] * po2[0] + po2[1] * po2[1] + po2[2] * po2[2]);
    eta[2] = 0.0;
    ksi[3] = ksi[0];
    eta[3] = eta[0];

    st = sxt = syt = szt = 0.0;
    for (i = 0; i < 3; ++i) {
        double dksi = ksi[i + 1] - ksi[i], deta = eta[i + 1] - eta[i];
        double r1 = sqrt((ksi[i] - x) * (ksi[i] - x) + (eta[i] - y) * (eta[i] - y) + z * z);
        double r2 = sqrt((ksi[i + 1] - x) * (ksi[i + 1] - x) + (eta[i + 1] - y) * (eta[i + 1] - y) + z * z);
        double l = sqrt(dksi * dksi + deta * deta);
        double b1 = deta * ((ksi[i] - x) * (ksi[i] - x) + z * z) - dksi * (ksi[i] - x) * (eta[i] - y);
        double a1 = r1 * z * dksi;
        double b2 = deta * ((ksi[i + 1] - x) * (ksi[i + 1] - x) + z * z) - dksi * (ksi[i + 1] - x) * (eta[i + 1] - y);
        double a2 = r2 * z * dksi;
        if (!(fabs(z) < 1.0e-6)) szt = szt + atan2(b1 * a2 - b2 * a1, a1 * a2 + b1 * b2);
        if (fabs(r1 + r2 - l) < 1.0e-6) continue;
        {
            double lgrn = log((r1 + r2 + l) / (r1 + r2 - l));
            sxt = sxt - deta / l * lgrn;
            syt = syt + dksi / l * lgrn;
            st = st + (deta * (x - ksi[i]) - dksi * (y - eta[i])) / l * lgrn;
        }
    }
    st = st - z * szt;
    *sij = *sij + st;
    for (j = 0; j < 3; ++j) dij[j] = dij[j] + ui[j] * sxt + uj[j] * syt + uk[j] * szt;
}

/* SGLINTBD_QUAD, SingularIntgr.f90:252-445 (IRR=1 path). */
void orc_sglint_quad(const double xf[3], const double xq[4][3], double *sij, double dij[3])
{
    double pov[4][3], pon[4][3], po[3], pof[3], un[3], ui[3], uj[3], uk[3], ksi[5], eta[5];
    double x, y, z, st, sxt, syt, szt, nn;
    int i, j;

    *sij = 0.0;
    dij[0] = dij[1] = dij[2] = 0.0;
    for (j = 0; j < 3; ++j) po[j] = (xq[0][j] + xq[1][j] + xq[2][j] + xq[3][j]) / 4.0;
    for (j = 0; j < 3; ++j) {
        pov[0][j] = xq[0][j] - po[j];
        pov[1][j] = xq[1][j] - po[j];
    }
    un[0] = pov[0][1] * pov[1][2] - pov[0][2] * pov[1][1];
    un[1] = pov[0][2] * pov[1][0] - pov[0][0] * pov[1][2];
    un[2] = pov[0][0] * pov[1][1] - pov[0][1] * pov[1][0];
    nn = sqrt(pov[0][0] * pov[0][0] + pov[0][1] * pov[0][1] + pov[0][2] * pov[0][2]);
    for (j = 0; j < 3; ++j) ui[j] = pov[0][j] / nn;
    nn = sqrt(un[0] * un[0] + un[1] * un[1] + un[2] * un[2]);
    for (j = 0; j < 3; ++j) uk[j] = un[j] / nn;
    uj[0] = uk[1] * ui[2] - uk[2] * ui[1];
    uj[1] = uk[2] * ui[0] - uk[0] * ui[2];
    uj[2] = uk[0] * ui[1] - uk[1] * ui[0];
    for (j = 0; j < 3; ++j) pof[j] = xf[j] - po[j];
    x = ui[0] * pof[0] + ui[1] * pof[1] + ui[2] * pof[2];
    y = uj[0] * pof[0] + uj[1] * pof[1] + uj[2] * pof[2];
    z = uk[0] * pof[0] + uk[1] * pof[1] + uk[2] * pof[2];
    for (j = 0; j < 3; ++j) {
        pov[2][j] = xq[2][j] - po[j];
        pov[3][j] = xq[3][j] - po[j];
    }
    for (i = 0; i < 4; ++i) {
        double d = uk[0] * pov[i][0] + uk[1] * pov[i][1] + uk[2] * pov[i][2];
        for (j = 0; j < 3; ++j) pon[i][j] = pov[i][j] - d * uk[j];
    }
    for (i = 0; i < 4; ++i) {
        ksi[i] = ui[0] * pon[i][0] + ui[1] * pon[i][1] + ui[2] * pon[i][2];
        eta[i] = uj[0] * pon[i][0] + uj[1] * pon[i][1] + uj[2] * pon[i][2];
    }
    ksi[4] = ksi[0];
    eta[4] = eta[0];

    st = sxt = syt = szt = 0.0;
    for (i = 0; i < 4; ++i) {
        double dksi = ksi[i + 1] - ksi[i], deta = eta[i + 1] - eta[i];
        double r1 = sqrt((ksi[i] - x) * (ksi[i] - x) + (eta[i] - y) * (eta[i] - y) + z * z);
        double r2 = sqrt((ksi[i + 1] - x) * (ksi[i + 1] - x) + (eta[i + 1] - y) * (eta[i + 1] - y) + z * z);
        double l = sqrt(dksi * dksi + deta * deta);
        double b1, a1, b2, a2;
        if (fabs(l) < 1.0e-8) continue; /* overlapping vertices, :416 */
        b1 = deta * ((ksi[i] - x) * (ksi[i] - x) + z * z) - dksi * (ksi[i] - x) * (eta[i] - y);
        a1 = r1 * z * dksi;
        b2 = deta * ((ksi[i + 1] - x) * (ksi[i + 1] - x) + z * z) - dksi * (ksi[i + 1] - x) * (eta[i + 1] - y);
        a2 = r2 * z * dksi;
        if (!(fabs(z) < 1.0e-6)) szt = szt + atan2(b1 * a2 - b2 * a1, a1 * a2 + b1 * b2);
        if (fabs(r1 + r2 - l) < 1.0e-6) continue;
        {
            double lgrn = log((r1 + r2 + l) / (r1 + r2 - l));
            sxt = sxt - deta / l * lgrn;
            syt = syt + dksi / l * lgrn;
            st = st - (deta * (x - ksi[i]) - dksi * (y - eta[i])) / l * lgrn;
        }
    }
    st = st + z * szt;
    *sij = *sij + st;
    for (j = 0; j < 3; ++j) dij[j] = -(dij[j] + ui[j] * sxt + uj[j] * syt + uk[j] * szt);
}
