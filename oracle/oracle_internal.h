/*
 * oracle_internal.h -- internal declarations of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle is a plain-C, FP64, thread-safe
 * restatement of HAMS-MREL's per-frequency build-and-solve path.  It exists
 * to check the CUDA product path and to time a CPU baseline; the product
 * library never links, loads or calls it.
 *
 * Every function cites the reference routine (path:line inside the
 * HAMS-MREL project) whose arithmetic it restates.  Fortran single-precision
 * literals (a constant written without a D exponent) are reproduced with F4()
 * so that thresholds and polynomial coefficients round exactly as in the
 * reference build.
 */
#ifndef HAMS_ORACLE_INTERNAL_H
#define HAMS_ORACLE_INTERNAL_H

#include <complex.h>
#include <math.h>
#include <stdint.h>

typedef double complex zdouble;

/* A Fortran REAL*4 literal promoted to REAL*8. */
#define F4(x) ((double)(x##f))

#define ORC_PI 3.141592653589793
#define ORC_NK 200

/* ---- special functions: src/FinGrnExtSubs.f90 ---- */
void orc_error(double x, double *err);                 /* ERROR  :62  */
void orc_enxa(int n, double x, double *en);            /* ENXA   :135 */
void orc_e1xa(double x, double *e1);                   /* E1XA   :198 */
void orc_eix(double x, double *ei);                    /* EIX    :254 */
void orc_limes(int n, double *s, double *rlimes, int *ipade, int *kpade,
               double *err);                           /* Limes  :370 */
void orc_ik01a(double x, double *bk0, double *bk1);    /* IK01A  :538 */
void orc_jy01b(double x, double *bj0, double *bj1, double *by0,
               double *by1);                           /* JY01B  :663 */
void orc_jy01bj(double x, double *bj0, double *bj1);   /* JY01BJ :741 */
void orc_jy01by0(double x, double *by0);               /* JY01BY0:811 */
void orc_jy01by1(double x, double *by1);               /* JY01BY1:875 */

/* ---- Green functions ---- */
void orc_fingreen3d(double xf, double xp, double yf, double yp, double zf,
                    double zp, double v, const double *wvn, int nk, double h,
                    zdouble grn[4], int flag);     /* FinGreen3D.f90:81 */
void orc_fingreen3d_r(double rr, double zf, double zp, double v,
                      const double *wvn, int nk, double h, zdouble grn[3],
                      int tag);                    /* FinGreen3D.f90:160 */
void orc_infgreen3d(double xf, double xp, double yf, double yp, double zf,
                    double zp, double v, zdouble grn[4],
                    int flag);                     /* InfGreen_Appr.f90:104 */

/* Branch of FINGREEN3D_R taken for a horizontal distance rr and depth h
 * (FinGreen3D.f90:183-191): 0 LINTON, 1 PIDCOCK, 2 EIGENE, 3 EIGEN. */
int orc_fin_branch(double rr, double h);

/* ---- Rankine panel integrals: src/SingularIntgr.f90 ---- */
void orc_sglint_tri(const double xf[3], const double xq[3][3], double *sij,
                    double dij[3]);                /* :44  */
void orc_sglint_quad(const double xf[3], const double xq[4][3], double *sij,
                     double dij[3]);               /* :252 */

/* ---- wave properties: src/WavDynSubs.f90, src/ImplementSubs.f90 ---- */
void orc_dispersion(double *wvn, int nrt, double w, double h);

#endif
