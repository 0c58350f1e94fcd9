/*
 * hams_oracle.h -- public interface of the CPU oracle (loaded by the tests
 * and by the CPU-baseline leg of bench.py through ctypes).
 *
 * TEST INFRASTRUCTURE ONLY.  The oracle restates HAMS-MREL's per-frequency
 * build-and-solve in plain C and FP64.  It is the checker of the CUDA path
 * and the timed CPU baseline; no product code links or calls it.
 *
 * Array conventions follow the reference's Fortran module arrays: column-major,
 * mesh connectivity 1-based, complex values as interleaved (re, im) doubles.
 */
#ifndef HAMS_ORACLE_H
#define HAMS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAXBODY 512

/* Panel geometry after BuildCombinedArrays (CalGreenFuncMulti.f90:53). */
typedef struct orc_geom {
    int32_t nelem;        /* hull panels, all bodies */
    int32_t ntnd;         /* hull nodes, all bodies */
    int32_t nbody;
    int32_t isx, isy;     /* symmetry flags of the .pnl header */
    int32_t nsys;         /* 1, or 2 with one plane of symmetry */
    double *xyz;          /* (ntnd,3)  global node coordinates          */
    int32_t *ncn;         /* (nelem)   3 or 4 vertices                   */
    int32_t *ncon;        /* (nelem,4) node ids, 1-based                 */
    double *xyz_p;        /* (nelem,3) panel centres                     */
    double *ds;           /* (nelem)   panel areas                       */
    double *pnsz;         /* (nelem)   longest panel edge                */
    double *dxyz;         /* (nelem,6) generalized normals n, r x n      */
    int32_t *body_nelem;  /* (nbody)   panels per body                   */
    /* interior water-plane (lid) panels, used when irsp = 1 */
    int32_t inelem, intnd;
    double *ixyz;         /* (intnd,3)  */
    int32_t *incn;        /* (inelem)   */
    int32_t *incon;       /* (inelem,4) */
    double *ixyz_p;       /* (inelem,3) */
    double *ids;          /* (inelem)   */
    double *ipnsz;        /* (inelem)   */
    double *idxyz;        /* (inelem,6) */
    int32_t *body_inelem; /* (nbody)    */
} orc_geom;

typedef struct orc_opts {
    double h;        /* water depth, < 0 for infinite depth           */
    double rho, g;   /* density and gravity of the force / wave terms  */
    double xw[2];    /* incident-wave reference point                  */
    double amp;      /* wave amplitude                                 */
    int32_t isol;    /* 1 total potential, 2 scattered                 */
    int32_t irsp;    /* 1 = irregular-frequency removal with lids      */
    int32_t grn_kind;/* 8 = FP64 tables, 4 = tables rounded to FP32    */
    int32_t nthread; /* OpenMP threads (0 = runtime default)           */
} orc_opts;

typedef struct orc_wave {
    double v;        /* omega^2 / g (0 and -1 are the SYBO limits)   */
    double wk;       /* wave number                                  */
    double w1;       /* angular frequency                            */
    double tp;       /* period                                       */
    double wl;       /* wave length                                  */
    double wvn[200]; /* dispersion roots (finite depth)              */
} orc_wave;

/* CalWaveProperts (ImplementSubs.f90:40) for one input value of type inft
 * (1 deep-water wave number, 2 wave number, 3 frequency, 4 period, 5 wave
 * length); sybo_kk = 1 or 2 selects the zero / infinite frequency limits. */
void orc_wave_props(int32_t inft, double value, double h, double g, int32_t sybo_kk, orc_wave *out);
void orc_dispersion_c(double *wvn, int32_t nrt, double w, double h);

/* CalNormalsMulti geometry (ReadPanelMeshMulti.f90:122): fills xyz_p, ds,
 * pnsz, dxyz of the hull (and lid) panels from the nodes; xr is (nbody,3). */
void orc_geom_prepare(orc_geom *g, const double *xr);

/* Single evaluations, for unit parity. grn is 4 complex (8 doubles). */
void orc_fingreen3d_c(double xf, double xp, double yf, double yp, double zf, double zp, double v,
                      const double *wvn, int32_t nk, double h, double *grn, int32_t flag);
void orc_infgreen3d_c(double xf, double xp, double yf, double yp, double zf, double zp, double v,
                      double *grn, int32_t flag);
int32_t orc_fin_branch_c(double rr, double h);
/* Rankine integral of panel jel (0-based) at field point xf: out = S, D(3). */
void orc_sglint_c(const orc_geom *g, int32_t jel, const double *xf, double *out);
void orc_special_c(int32_t which, double x, double *out);

/* Assembly (CALGREEN_MULTI + ASSB_LEFT/RBC/DBC_MULTI), no factorisation.
 *   amat  (n,n,nsys) complex   -- unfactored influence matrix
 *   brmat (n,6*nbody,nsys)     -- radiation right-hand sides
 *   bdmat (n,nsys,nbeta)       -- diffraction right-hand sides
 * With irsp = 1 the lid rows are built and the normal equations C = A^T A,
 * D = A^T B of AssbMatx_irrMulti.f90 replace amat/brmat/bdmat (all n x ...).
 * Returns 0. */
int32_t orc_assemble(const orc_geom *g, const orc_opts *o, const orc_wave *w, int32_t nbeta,
                     const double *beta, double *amat, double *brmat, double *bdmat);

/* Hull rows offset, offset+stride, ... only (no lids): a bounded sample of
 * orc_assemble for CPU timing. Leading dimension = returned row count. */
int32_t orc_assemble_rows(const orc_geom *g, const orc_opts *o, const orc_wave *w, int32_t nbeta,
                          const double *beta, int32_t stride, int32_t offset, double *amat,
                          double *brmat, double *bdmat);
/* Partial-pivot complex LU (ZGETRF semantics, 1-based ipiv) and solve. */
int32_t orc_zgetrf(int32_t n, double *a, int32_t *ipiv, int32_t nthread);
void orc_zgetrs(int32_t n, int32_t nrhs, const double *a, const int32_t *ipiv, double *b);

/* Reductions RFORCE_MULTI / EFORCE_MULTI (PotentWavForceMulti.f90).
 *   xrad (n,6*nbody,nsys): solved radiation systems before symmetry recombination
 *   xdif (n,nsys,nbeta)  : solved diffraction systems
 *   amas, bdmp (6nb,6nb) ; exfc (nbeta,6nb) complex */
void orc_forces(const orc_geom *g, const orc_opts *o, const orc_wave *w, int32_t nbeta,
                const double *beta, const double *xrad, const double *xdif, double *amas,
                double *bdmp, double *exfc);

/* Whole frequency: assemble, LU, solve, reductions. Returns the ZGETRF info. */
int32_t orc_solve_frequency(const orc_geom *g, const orc_opts *o, const orc_wave *w, int32_t nbeta,
                            const double *beta, double *amas, double *bdmp, double *exfc);

/* Whole deck: ControlFile.in + .pnl in, HAMS-format OAMASS/ODAMPING/OEXFOR
 * files out (HAMS_Prog.f90 multi-body loop). Returns 0 on success. */
int32_t orc_run_case(const char *inputdir, const char *outputdir, int32_t grn_kind, int32_t nthread);

/* Deck loader used by orc_run_case, exposed for the tests. */
typedef struct orc_deck {
    orc_opts opts;
    orc_geom geom;
    int32_t sybo, inft, ouft, nper, nbeta;
    double *wvnb;   /* (nper) input frequency values */
    double *wvhd;   /* (nbeta) headings, degrees     */
    double *xr;     /* (nbody,3) rotation centres    */
    double *lcs;    /* (nbody,4)                     */
    double refl;
    int32_t isolv;
} orc_deck;
int32_t orc_load_deck(const char *inputdir, orc_deck *d);
void orc_free_deck(orc_deck *d);

#ifdef __cplusplus
}
#endif
#endif
