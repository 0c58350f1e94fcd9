/*
 * hams_gpu.h -- C ABI of the B200 per-frequency BEM build-and-solve.
 *
 * Drop-in for the frequency-loop body of HAMS-MREL (src/HAMS_Prog.f90): the
 * host (the reference's Fortran driver through iso_c_binding, the C++ driver
 * hams_b200_run, or Python through ctypes) keeps reading ControlFile.in and
 * the .pnl meshes and writing the HAMS/WAMIT files; everything from the
 * Green-function tables to the force reductions runs on the GPU behind
 * these calls.
 *
 * Conventions
 *   - every call returns an int status: 0 ok; > 0 the 1-based index of a
 *     zero pivot in the LU factorisation (LAPACK INFO style); < 0 an error
 *     code below; hams_last_error() gives the message of the calling thread;
 *   - arrays are host memory laid out as the reference's Fortran arrays:
 *     column-major, mesh connectivity 1-based, complex values as
 *     interleaved (re, im) doubles;
 *   - a context owns one CUDA stream and its device buffers; use one context
 *     per host thread.
 */
#ifndef HAMS_GPU_H
#define HAMS_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HAMS_NK 200 /* dispersion roots per frequency, WavDynMods.f90:59 (NK) */

enum {
  HAMS_OK = 0,
  HAMS_ERR_ARG = -1,         /* invalid argument                      */
  HAMS_ERR_CUDA = -2,        /* CUDA runtime / library failure         */
  HAMS_ERR_UNSUPPORTED = -3, /* option not built (see message)         */
  HAMS_ERR_NOMEM = -4,       /* device or host allocation failed       */
  HAMS_ERR_NUMERIC = -5      /* non-finite result or refinement stalled*/
};

/* Complex64 factorisation of the mixed form.  BLOCK: 64-row blocks pivoted
 * inside each diagonal block, the complex products as real GEMMs on the
 * tensor cores with FP32 accumulation -- inputs rounded to TF32
 * (BLOCK_TF32, the default) or FP32 emulated on BF16 tensor cores
 * (BLOCK_EMU, needs the cuBLAS 12.9 emulation; with an older cuBLAS loaded
 * in the process it runs as BLOCK_TF32); the library's partially pivoted LU
 * (LIBRARY) is also the fallback when the refinement of a block
 * factorisation does not converge. */
enum { HAMS_LU_BLOCK_TF32 = 0, HAMS_LU_BLOCK_EMU = 1, HAMS_LU_LIBRARY = 2 };

/* Linear solver (ControlFile Solver_type, InputFiles.f90:177-191).  GMRES
 * (IterativeSolvers.f90:324-484): restarted, right-preconditioned -- by the
 * LU factors of each body's diagonal block with two or more bodies
 * (:176-253), by the diagonal with one body (:154-174) -- every right-hand
 * side from zero, all right-hand sides advanced together (one matrix product
 * per iteration); FP64 in every precision form.  A solve that misses the
 * tolerance keeps its last iterate and says so in hams_last_note, as the
 * reference warns and goes on (:475-480).  Without lids its products use the
 * H-matrix of the influence matrix (HMatrix.f90: cluster tree of the panel
 * centres, ACA-compressed admissible blocks), as the reference's do; with
 * lids (IRSP = 1) it iterates on the normal equations with dense products
 * (AssbMatx_irr.f90:494-498). */
enum { HAMS_SOLVER_LU = 1, HAMS_SOLVER_GMRES = 2 };

/* Numerical form of a solve. */
enum {
  HAMS_PREC_FP64 = 0,  /* plain FP64 drop-in: FP64 assembly, FP64 LU           */
  HAMS_PREC_MIXED = 1  /* FP64 assembly, complex64 LU + FP64 iterative refinement */
};

/*
 * Panel geometry after CalNormals[Multi] and BuildCombinedArrays
 * (ReadPanelMeshMulti.f90:122, CalGreenFuncMulti.f90:53): the module arrays
 * XYZ_GLOBAL_MULTI_COMB, NCN/NCON_MULTI_COMB, XYZ_GLOBAL_MULTI_COMB_P,
 * DS/PNSZ/DXYZ_MULTI_COMB and the interior water-plane centres iXYZ_..._P.
 */
typedef struct hams_geom {
  int32_t nelem;               /* hull panels of all bodies (N)                  */
  int32_t ntnd;                /* hull nodes                                      */
  int32_t nbody;               /* bodies                                          */
  int32_t isx, isy;            /* symmetry flags of the .pnl header: 0 0, or one
                                  of them 1 for a half mesh (x >= 0 mirrored in
                                  x = 0, or y >= 0 in y = 0; reference points on
                                  the plane), unfolded into the full bodies    */
  const double *xyz;           /* (ntnd,3)  node coordinates                      */
  const int32_t *ncn;          /* (nelem)   vertices per panel, 3 or 4            */
  const int32_t *ncon;         /* (nelem,4) vertex node ids, 1-based              */
  const double *xyz_p;         /* (nelem,3) panel centres                         */
  const double *ds;            /* (nelem)   panel areas                           */
  const double *pnsz;          /* (nelem)   longest panel edge                    */
  const double *dxyz;          /* (nelem,6) generalized normals n and r x n       */
  const int32_t *body_nelem;   /* (nbody)   panels of each body, in order         */
  int32_t inelem;              /* interior water-plane panels (0: none)           */
  const double *ixyz_p;        /* (inelem,3) water-plane panel centres            */
} hams_geom;

typedef struct hams_opts {
  double depth;     /* H: water depth, < 0 for infinite depth                    */
  double rho, g;    /* density and gravity of the force and incident-wave terms  */
  double xw[2];     /* incident-wave reference point (XW)                        */
  double amp;       /* wave amplitude (AMP)                                      */
  int32_t isol;     /* 1 total potential, 2 scattered (ISOL)                     */
  int32_t irsp;     /* 1: remove irregular frequencies with water-plane lids     */
  int32_t precision;/* HAMS_PREC_FP64 or HAMS_PREC_MIXED                         */
  int32_t device;   /* CUDA device ordinal                                       */
  double refine_tol;/* mixed: relative residual target of the refinement (<=0: 1e-12) */
  int32_t refine_max;/* mixed: refinement sweeps (<=0: 30)                       */
  int32_t lu_kind;  /* mixed: HAMS_LU_BLOCK_TF32 (0), HAMS_LU_BLOCK_EMU, HAMS_LU_LIBRARY */
  int32_t batch_lanes;/* hams_solve_batch: frequencies in flight (<=0: 8)          */
  int32_t solver;   /* HAMS_SOLVER_LU (0 or 1) or HAMS_SOLVER_GMRES (2), ISOLV     */
  int32_t gmres_restart;/* GMRES restart length (<=0: 25, IterativeSolvers.f90:56) */
  int32_t gmres_maxit;  /* GMRES iterations over all restarts (<=0: 100, :58)    */
  double gmres_tol; /* GMRES relative residual target (<=0: 1e-4, :57)          */
  double aca_tol;   /* GMRES: ACA tolerance of the H-matrix blocks (<=0: 1e-4,
                       HMatrix.f90:60)                                          */
  int32_t gmres_dense;/* GMRES: 0 products with the H-matrix (the reference's
                       choice without lids, AssbMatx[Multi].f90:284-288), 1 with
                       the dense matrix; with lids always dense (:494-498)      */
  int32_t body_blocks;/* 1: compute the wave Green function of each distinct
                       (field body, source body) block once and copy it to
                       the blocks of identical body pairs (hams_body_blocks);
                       without lids only.  0: every pair (the reference)     */
  int32_t lu_graph; /* mixed, HAMS_LU_BLOCK_TF32: 1 records the block LU's
                       factorisation and triangular solves as CUDA graphs
                       (once per frequency lane and right-hand-side count) and
                       replays them -- a lower latency for one frequency at a
                       time; with several frequencies in flight the replays
                       overlap less than direct launches, so batches leave it
                       at 0 (launched directly)                             */
  int32_t reserved;
} hams_opts;

/* One frequency after CalWaveProperts (ImplementSubs.f90:40): V = w^2/g
 * (0 and -1 for the zero / infinite frequency limits), wave number, angular
 * frequency and the dispersion roots WVN (finite depth only). */
typedef struct hams_wave {
  double v, wk, w1, tp, wl;
  double wvn[HAMS_NK];
} hams_wave;

typedef struct hams_ctx hams_ctx;

/* Replaces CalWaveProperts + DISPERSION (ImplementSubs.f90:40,
 * WavDynSubs.f90:40).  inft: 1 deep-water wave number, 2 wave number,
 * 3 angular frequency, 4 period, 5 wave length; sybo_kk = 1 / 2 selects the
 * zero / infinite frequency limit (SYBO = 1 decks), 0 a regular frequency. */
int hams_wave_properties(int32_t inft, double value, double depth, double g, int32_t sybo_kk, hams_wave *out);

/* Panel centres, areas, longest edges and generalized normals (n, r x n
 * about each body's reference point xr (nbody,3)) from the nodes: CalNormals
 * / CalNormalsMulti (ReadPanelMesh.f90:110, ReadPanelMeshMulti.f90:122) with
 * the routines of NormalProcess.f90.  Host-only; outputs as in hams_geom. */
int hams_prepare_geometry(int32_t ntnd, const double *xyz, int32_t nelem, const int32_t *ncn, const int32_t *ncon,
                          int32_t nbody, const int32_t *body_nelem, const double *xr, double *xyz_p, double *ds,
                          double *pnsz, double *dxyz);

/* Blocks of identical body pairs (hams_opts.body_blocks).  Body b is a
 * translate of an earlier body t when they have the same panels in the same
 * order and every vertex, centre, area, longest edge and unit normal of b is
 * t's moved by one horizontal offset (within tol times the mesh size; tol <= 0:
 * 1e-9).  The (field b1, source b2) block then equals the first block
 * (c1, c2), in column-major order of k = b1 + nbody b2, whose bodies are
 * translates of the same bodies with the same horizontal offset of c2 from
 * c1: rep[k] receives that block's k (rep (nbody, nbody); rep[k] = k for a
 * block computed in full).  Geometries with water-plane lids (inelem > 0)
 * keep every block.  Host-only.  Returns the number of distinct blocks, or
 * -1 on a null argument. */
int hams_body_blocks(const hams_geom *geo, double tol, int32_t *rep);

/* Uploads the geometry, evaluates the frequency-independent Rankine panel
 * integrals (SGLINTBD_*, SingularIntgr.f90:44,252) for every field/source
 * pair and sorts the pairs by Green-function branch.  Replaces the setup of
 * HAMS_Prog.f90:423-570 on the device side. */
int hams_ctx_create(const hams_geom *geom, const hams_opts *opts, hams_ctx **out);
/* Destroys a context and its batch lanes.  Their device buffers, streams and
 * cuBLAS/cuSOLVER handles are kept by the library (per device, at most a
 * third of the device's memory and 32 handle sets) for the contexts created
 * after it, so that a sequence of contexts allocates and creates handles
 * once; hams_release_cached returns them. */
void hams_ctx_destroy(hams_ctx *ctx);
/* Frees the device memory and destroys the streams and handles that destroyed
 * contexts left to the library (no counterpart in the reference).  Call it
 * with no context in use on the device whose memory is wanted elsewhere. */
void hams_release_cached(void);

/*
 * One frequency, all headings: the body of HAMS_Prog.f90:615-723 --
 * CALGREEN_MULTI, ASSB_LEFT/RBC/DBC_MULTI, RADIATION/DIFFRACTION_SOLVER_MULTI,
 * RFORCE_MULTI and EFORCE_MULTI (and their _IRR forms when opts.irsp = 1).
 *   beta_rad (nbeta)      headings in radians
 *   amas, bdmp (6nb,6nb)  AMAS/BDMP_MULTI_COMB(KK,:,:): added mass, damping
 *   exfc (nbeta,6nb)      EXFC_MULTI_COMB(KK,:,:): complex excitation
 * Any output pointer may be NULL.
 */
int hams_solve_frequency(hams_ctx *ctx, const hams_wave *wave, int32_t nbeta, const double *beta_rad, double *amas,
                         double *bdmp, double *exfc);

/* nfreq frequencies, results stacked along a leading frequency index:
 * amas/bdmp (nfreq,6nb,6nb), exfc (nfreq,nbeta,6nb), column-major as
 * AMAS_MULTI_COMB / EXFC_MULTI_COMB.  opts.batch_lanes frequencies are in
 * flight at once, each on its own stream and host thread with its own
 * per-frequency buffers (about 1.3 GB per lane at 5,400 panels), sharing the
 * context's geometry; lanes are created on first use and kept.  Returns the
 * first error, or the singular-pivot index of the first frequency with one. */
int hams_solve_batch(hams_ctx *ctx, int32_t nfreq, const hams_wave *waves, int32_t nbeta, const double *beta_rad,
                     double *amas, double *bdmp, double *exfc);

/* The assembled systems of one frequency, before factorisation, for checks:
 *   amat (n,n)        A of ASSB_LEFT_MULTI (or C = A^T A with lids)
 *   brmat (n,6nb)     radiation right-hand sides (or A^T B)
 *   bdmat (n,nbeta)   diffraction right-hand sides (or A^T B)
 * Any output pointer may be NULL.  A context made from a half mesh
 * (ISX or ISY = 1) holds the unfolded mesh and returns HAMS_ERR_UNSUPPORTED. */
int hams_assemble(hams_ctx *ctx, const hams_wave *wave, int32_t nbeta, const double *beta_rad, double *amat,
                  double *brmat, double *bdmat);

/* Batch evaluation of FINGREEN3D (depth > 0) or INFGREEN3D (depth < 0) for
 * npts source/field pairs: pts (npts,6) = (xq, yq, zq, xp, yp, zp) per row,
 * flag (npts) the near/far flag, grn (npts,4) complex output (G, dG/dx,
 * dG/dy, dG/dz at the source).  Runs on the context's device. */
int hams_eval_green(hams_ctx *ctx, const hams_wave *wave, int32_t npts, const double *pts, const int32_t *flag,
                    double *grn);

/* hams_eval_green without any device allocation (no counterpart in the
 * reference).  For callers that cannot allocate device memory: a host loop
 * that evaluates Green functions while solves run on other streams of the
 * same device (cudaFree inside hams_eval_green synchronizes the whole device
 * and stalls them), or a process whose device memory is fully committed to
 * the per-frequency systems.  The staging lives in one fixed reservation per
 * device of HAMS_EVAL_STATIC_MAX_POINTS points (about 464 KiB of device
 * memory); larger npts is rejected with HAMS_ERR_ARG.  The first call on a
 * device looks the reservation up (cudaGetSymbolAddress) and caches it; make
 * that first call before any stream capture on the device.  Calls on one
 * device share the reservation: each call waits for its own stream before it
 * returns, so calls one after another are safe, but calls that overlap in
 * time on one device (from several host threads) race and must be
 * serialised by the caller.  The call reads the context's geometry only (the
 * wave numbers are staged in the reservation too), but it enqueues on the
 * context's stream and counts its launch there: pass a context that is not
 * solving during the call (solves may run on other contexts of the device).
 * Same arguments and results as hams_eval_green. */
#define HAMS_EVAL_STATIC_MAX_POINTS 4096
int hams_eval_green_static(hams_ctx *ctx, const hams_wave *wave, int32_t npts, const double *pts,
                           const int32_t *flag, double *grn);

/*
 * MLP surrogate of the finite-depth evanescent Green function (no
 * counterpart in the reference; the reference always sums the series of
 * FinGreen3D.f90:281-506).  Inputs per panel pair: X = R/h, the source and
 * field depths above the bottom (zq+h)/h, (zp+h)/h, and K = k0 h tanh(k0 h);
 * outputs the evanescent part of the wave term (without the propagating mode
 * and with 1/r, 1/r1 removed) and its R and zq derivatives, in depth units,
 * scaled by X, X^2, X^2.  Domain X in [0.05, 3], depths in [0.5, 1],
 * K in [0.04, 40]; 4 SiLU hidden layers of width 128.
 */
typedef struct hams_sg_train {
  int32_t n_train, n_test; /* samples generated from the series (training, held out) */
  int32_t batch, steps;    /* minibatch size, Adam steps                              */
  int32_t nslice;          /* K values sampled (log-spaced over the domain)           */
  int32_t reserved0;
  uint64_t seed;
  double lr;               /* peak learning rate (warm-up, then cosine decay)         */
  double reserved[4];
} hams_sg_train;

/* Number of floats in a parameter vector. */
int32_t hams_surrogate_param_count(void);
/* n training samples from the series: raw (n,7) = X, Zq, Zp, K, t0, t1, t2. */
int hams_surrogate_samples(int32_t device, int32_t n, uint64_t seed, int32_t nslice, double *raw);
/* Generates samples and trains on the GPU; params receives the network,
 * stats (9): held-out RMS error / RMS of t0..t2, max error / max |t| of
 * t0..t2, final training loss, training and sampling time (ms). */
int hams_surrogate_train(int32_t device, const hams_sg_train *cfg, float *params, double *stats);
/* Reference FP32 evaluation: x (n,4) = X, Zq, Zp, K -> t (n,3). */
int hams_surrogate_eval(int32_t device, const float *params, int32_t n, const double *x, double *t);
/* Mean squared error of normalised outputs and its gradient for inputs
 * feats (4,n) (features in [-1,1]) and normalised targets targ (3,n). */
int hams_surrogate_grad(int32_t device, const float *params, int32_t n, const float *feats, const float *targ,
                        double *loss, float *grad);

/* Switches the surrogate on for the far pairs of ctx (params: a trained
 * vector, nparams = hams_surrogate_param_count()) or off (params NULL).  A
 * pair is far when its centre distance exceeds far_factor times the source
 * panel's longest edge, it lies in the network's domain, and it falls in the
 * EIGENE or EIGEN branch; frequencies with K outside the domain keep the
 * series for all pairs.  Finite depth only. */
int hams_ctx_set_surrogate(hams_ctx *ctx, const float *params, int32_t nparams, double far_factor);

/* Frequencies the surrogate serves: those with K = k0 h tanh(k0 h) in
 * [kmin, kmax] (inside the network's domain, 0.04 to 40, the default);
 * other frequencies keep the series for all pairs.  Where the outputs are
 * small differences of large terms (damping as w -> 0, excitation of deep
 * bodies at short waves, the bands around irregular frequencies) the
 * surrogate's error is amplified, and this range keeps those frequencies
 * on the series. */
int hams_ctx_set_surrogate_range(hams_ctx *ctx, double kmin, double kmax);

/* The series judges the surrogate, frequency by frequency (no counterpart in
 * the reference, which has no surrogate).  With tol > 0, every frequency the
 * network serves (mixed precision, LU solver, no lids) is checked after its
 * solve: the series re-evaluates a sample of about 16,000 far pairs, giving
 * the network's RMS relative error per cell of its input domain (R/h x
 * source depth x field depth); that error, taken coherent (every far-pair
 * entry of A and S replaced by its cell's error times the entry), is carried to
 * first order through the factorisation already made and the force
 * reductions, giving the estimated error of added mass, damping and
 * excitation.  When the largest (times a safety factor calibrated on the
 * 5,400-panel array) exceeds tol, the series takes the frequency back: its
 * far pairs are evaluated again with the series and the solution is refined
 * (FP64 residuals) from the network's, with the network's factors as the
 * preconditioner -- no second factorisation; should that refinement stall,
 * the series' matrix is factored.  hams_last_note says which ("refined to
 * the series" or "re-solved with the series") and hams_last_timings reports
 * the estimates.  The probe goes through the same system, so it is amplified
 * where the system amplifies: the long-wave damping (a small imaginary part
 * of large potentials) and the bands around irregular frequencies, which
 * the hand-picked K range of hams_ctx_set_surrogate_range otherwise keeps on
 * the series.  tol = 0 (the default) switches the judgement off. */
int hams_ctx_set_surrogate_tolerance(hams_ctx *ctx, double tol);

/* Timing of the last solve in milliseconds: [0] Green/assembly kernels,
 * [1] right-hand sides, [2] factorisation + solves, [3] reductions,
 * [4] whole call, [5..8] Green kernels of the LINTON, PIDCOCK, EIGENE and
 * EIGEN branches (finite depth), [9] LU factorisation, [10] refinement
 * sweeps (mixed form) or GMRES iterations, [11..14] pairs in each branch, [15] the mixed
 * form's factorisation (HAMS_LU_*; -1 for FP64), [16] the surrogate kernel
 * (or the series standing in for it), [17] pairs the surrogate evaluated,
 * [18] the mixed form's largest residual reduction factor over one refinement
 * sweep (about the condition number times the factorisation's error),
 * [19] pairs copied from identical body blocks (hams_opts.body_blocks),
 * and, for a frequency the surrogate solved with a tolerance set
 * (hams_ctx_set_surrogate_tolerance): [20] the network's sampled relative
 * error on the far-pair entries of A, [21] of S, [22..24] the estimated
 * relative error of added mass, damping and excitation, [25] the estimate
 * the decision uses, [26] 1 if the series took the frequency back,
 * [27] the pairs sampled.  n is the capacity of ms (28 fills all). Returns the number
 * written. */
int hams_last_timings(hams_ctx *ctx, double *ms, int32_t n);

/* Field points (ControlFile Number_of_field_points, InputFiles.f90:193-203):
 * every later solve of ctx also evaluates the potentials at these nfp points
 * xfp (nfp,3) from the solved panel potentials (CalPotentialMulti,
 * PressureElevationMulti.f90:55-272): the influence of every hull panel at
 * each point (Rankine integral at the point, SGLINTBD_MULTI_QUAD2/TRI2, plus
 * the wave Green function), divided by 2 pi for a point on a hull panel and
 * 4 pi in the fluid.  nfp = 0 switches them off. */
int hams_ctx_set_field_points(hams_ctx *ctx, int32_t nfp, const double *xfp);

/* The field-point potentials of frequency k of the last hams_solve_batch
 * (k = 0 after hams_solve_frequency): pot (nfp, 6nb + 2 nbeta) complex,
 * column-major -- the radiation potential of each body mode (unit velocity,
 * columns 6b+m), the diffraction potential of each heading (scattered plus
 * incident for ISOL = 1, as CalPotentialMulti adds VINP), then the incident
 * potential alone of each heading (CalPotentialIncMulti, :277-300).
 * Pressure is i w rho times a potential, elevation i w / g times it (rho and
 * 1 at the zero and infinite frequency limits), CalPressureMulti /
 * CalElevationMulti :305-348. */
int hams_field_potentials(hams_ctx *ctx, int32_t k, double *pot);

/* What the last solve of ctx decided on its own, e.g. the reason it fell back
 * from the block LU to the library LU, or a GMRES solve that missed its
 * tolerance; after hams_solve_batch each frequency's note, prefixed by its
 * index.  Empty when nothing. */
const char *hams_last_note(hams_ctx *ctx);

/* Kernels of this library launched since the context was created (library
 * calls into cuBLAS / cuSOLVER / CUB are counted by hams_library_call_count). */
int64_t hams_launch_count(hams_ctx *ctx);
int64_t hams_library_call_count(hams_ctx *ctx);

/* Device-time marks on the context's stream: hams_mark records event `slot`
 * (0..7); hams_mark_elapsed waits for mark b and returns the milliseconds
 * between marks a and b. */
int hams_mark(hams_ctx *ctx, int32_t slot);
int hams_mark_elapsed(hams_ctx *ctx, int32_t a, int32_t b, double *ms);

/* FP64 fused multiply-add throughput of the device in TFLOP/s (2 flops per
 * FMA), measured with independent dependency chains on every SM: the
 * denominator of the Green-function kernels' roofline. */
int hams_measure_fp64_peak(int32_t device, double *tflops);

/* Diagnostic (no counterpart in the reference): the mixed form's
 * tensor-core GEMM (tcgen05.mma kind::tf32, FP32 accumulation) on host
 * arrays, for tests: C = alpha A B + beta C with A m x k row-major (lda, a
 * multiple of 4), B k x n column-major (ldb, a multiple of 4), C m x n
 * column-major, or row-major with c_rowmajor (ldc); variant 0, 1, 2 the tile
 * of 128 x 64, 128 x 128 or 128 x 256 columns of C per CTA, -1 the
 * autotuner's pick. */
int hams_diag_gemm_tf32(int32_t device, int32_t m, int32_t n, int32_t k, float alpha, const float *a, int32_t lda,
                        const float *b, int32_t ldb, float beta, float *c, int32_t ldc, int32_t c_rowmajor,
                        int32_t variant);

/* Diagnostic (no counterpart in the reference): mean device time in ms of
 * that GEMM (variant 0-2, or -1 for the autotuner's pick) on device-resident
 * operands of shape m x n x k, over reps launches after one untimed. */
int hams_diag_gemm_tf32_time(int32_t device, int32_t variant, int32_t m, int32_t n, int32_t k, int32_t reps,
                             double *ms);

/* Message of the last failing call on this thread ("" if none). */
const char *hams_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
