// green_series.cu -- the epsilon-accelerated finite-depth Green kernels.
//
// EIGENE and PIDCOCK (FinGreen3D.f90:413-660) sum up to 100 eigenfunction
// terms and extrapolate them with the Wynn epsilon algorithm (Limes), which
// divides by differences of nearly equal partial sums and stops on exact
// equalities.  This file is compiled with --fmad=false so that every product
// and sum of those series is rounded exactly as in the CPU checker; the
// transcendental functions inside them come from detmath.h.  The remaining
// kernels (hams_gpu.cu) keep fused multiply-adds.
#include "kernels.cuh"
#include "rankine.cuh"

// 128 threads and at most 64 registers per thread (8 blocks per SM): the
// series are latency-bound, and the extra resident warps outweigh the few
// spills (measured on the 5,400-panel array: EIGENE 54 ms at 116 registers,
// 38 ms at 64).
template <int BR, int N>
__global__ void __launch_bounds__(128, 8) k_green_series(DevGeom g, WaveDev w, const double* __restrict__ wvn,
                                                      hams::ModeTab mt, const uint32_t* __restrict__ pairs,
                                                      long long count, const double* __restrict__ rs,
                                                      const double* __restrict__ rd, double2* __restrict__ A,
                                                      double2* __restrict__ S, int* ovf) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  size_t p = pairs[t];
  int i = (int)(p % (size_t)g.tn), j = (int)(p / (size_t)g.tn);
  int flag = near_flag(g, i, j);
  double xp = g.fxyz[i], yp = g.fxyz[i + g.tn], zp = g.fxyz[i + 2 * g.tn];
  double xq = g.xq[j], yq = g.xq[j + g.n], zq = g.xq[j + 2 * g.n];
  grn4 G;
  if (w.limit) {
    G = hams::green_limit(w.limit == 2, xq, xp, yq, yp, zq, zp, flag);
  } else {
    hams::SeriesScratchN<N> sc;
    hams::TableModes md{mt, j, i};
    int o = 0;
    G = hams::fingreen3d<BR>(xq, xp, yq, yp, zq, zp, w.v, wvn, w.h, flag, &sc, &o, md);
    if (o) atomicOr(ovf, 1);
  }
  store_pair(g, p, i, j, G, rs, rd, A, S);
}

void launch_green_series(int br, unsigned blocks, cudaStream_t st, DevGeom g, WaveDev w, const double* wvn,
                         const hams::ModeTab& mt, const uint32_t* pairs, long long count, const double* rs,
                         const double* rd, double2* A, double2* S, int* ovf) {
  if (br == hams::kPidcock)
    k_green_series<hams::kPidcock, hams::kPidcockMax>
        <<<blocks, 128, 0, st>>>(g, w, wvn, mt, pairs, count, rs, rd, A, S, ovf);
  else
    k_green_series<hams::kEigenE, hams::kEigenEMax>
        <<<blocks, 128, 0, st>>>(g, w, wvn, mt, pairs, count, rs, rd, A, S, ovf);
}

// Per-frequency mode tables (ModeTab) for modes 2..nmode-1: one thread per
// (mode, panel) entry, the expressions of InlineModes (green.cuh), compiled
// here without fused multiply-adds like the series that read them.  Slot 1
// holds the propagating mode's factors for the surrogate kernel: pm[1] =
// pi / NM0, src = (sinh, cosh) of k0 (zq + h), fld = cosh of k0 (zp + h).
__global__ void k_mode_tables(DevGeom g, WaveDev w, const double* __restrict__ wvn, int nmode, double* pm, double* ac,
                              double2* src, double2* srct, double* fld, double* fldt) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  int i = blockIdx.y + 1;  // mode number (1: propagating-mode factors)
  if (i >= nmode) return;
  const double h = w.h;
  if (i == 1) {
    const double wk = w.wk;
    if (k < g.n) {
      double zfh = g.xq[k + 2 * g.n] + h;
      src[g.n + k] = make_double2(sinh(wk * zfh), cosh(wk * zfh));
    }
    if (k < g.tn) fld[g.tn + k] = cosh(wk * (g.fxyz[k + 2 * g.tn] + h));
    if (k == 0) pm[1] = 3.141592653589793 / (h / 2.0 * (1.0 + sinh(2.0 * wk * h) / (2.0 * wk * h)));
    return;
  }
  if (k < g.n) {
    hams::InlineModes md{wvn, h, w.v, g.xq[k + 2 * g.n] + h, 0.0};
    double s, c;
    md.src(i, s, c);
    src[(size_t)i * g.n + k] = make_double2(s, c);
    md.srct(i, s, c);
    srct[(size_t)i * g.n + k] = make_double2(s, c);
  }
  if (k < g.tn) {
    hams::InlineModes md{wvn, h, w.v, 0.0, g.fxyz[k + 2 * g.tn] + h};
    fld[(size_t)i * g.tn + k] = md.fld(i);
    fldt[(size_t)i * g.tn + k] = md.fldt(i);
  }
  if (k == 0) {
    hams::InlineModes md{wvn, h, w.v, 0.0, 0.0};
    pm[i] = md.pm(i);
    ac[i] = md.ac(i);
  }
}

void launch_mode_tables(cudaStream_t st, DevGeom g, WaveDev w, const double* wvn, int nmode, double* pm, double* ac,
                        double2* src, double2* srct, double* fld, double* fldt) {
  dim3 grid((g.tn + 127) / 128, nmode - 1);
  k_mode_tables<<<grid, 128, 0, st>>>(g, w, wvn, nmode, pm, ac, src, srct, fld, fldt);
}

// Batch Green evaluation of hams_eval_green: any branch, one pair per thread.
__global__ void k_eval_green(int npts, const double* __restrict__ pts, const int* __restrict__ flag, WaveDev w,
                             const double* __restrict__ wvn, double2* __restrict__ out, int* ovf) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts) return;
  double xq = pts[t], yq = pts[t + npts], zq = pts[t + 2 * (size_t)npts];
  double xp = pts[t + 3 * (size_t)npts], yp = pts[t + 4 * (size_t)npts], zp = pts[t + 5 * (size_t)npts];
  grn4 G;
  if (w.limit) {
    G = hams::green_limit(w.limit == 2, xq, xp, yq, yp, zq, zp, flag[t]);
  } else if (w.h < 0.0) {
    G = hams::infgreen3d(xq, xp, yq, yp, zq, zp, w.v, flag[t]);
  } else {
    int o = 0;
    double rr = sqrt((xq - xp) * (xq - xp) + (yq - yp) * (yq - yp));
    switch (hams::fin_branch(rr, w.h)) {
      case hams::kLinton: G = hams::fingreen3d<hams::kLinton>(xq, xp, yq, yp, zq, zp, w.v, wvn, w.h, flag[t], (void*)nullptr, &o); break;
      case hams::kPidcock: {
        hams::SeriesScratchN<hams::kPidcockMax> sc;
        G = hams::fingreen3d<hams::kPidcock>(xq, xp, yq, yp, zq, zp, w.v, wvn, w.h, flag[t], &sc, &o);
        break;
      }
      case hams::kEigenE: {
        hams::SeriesScratchN<hams::kEigenEMax> sc;
        G = hams::fingreen3d<hams::kEigenE>(xq, xp, yq, yp, zq, zp, w.v, wvn, w.h, flag[t], &sc, &o);
        break;
      }
      default: G = hams::fingreen3d<hams::kEigen>(xq, xp, yq, yp, zq, zp, w.v, wvn, w.h, flag[t], (void*)nullptr, &o); break;
    }
    if (o) atomicOr(ovf, 1);
  }
  for (int k = 0; k < 4; ++k) out[t + (size_t)k * npts] = make_double2(G.g[k].re, G.g[k].im);
}


// Source (S) and normal-dipole (D) influence of every hull panel J at field
// point f, the terms CalPotentialMulti sums (PressureElevationMulti.f90:81-137):
// S = FLAG*SIJ + G ds, D = (FLAG*DIJ + grad G ds) . n_J, with the Rankine
// integrals at the field point (SGLINTBD_MULTI_QUAD2/TRI2,
// SingularIntgrMulti.f90:454-776) and FLAG = (distance <= 50 PNSZ_J).
__global__ void k_field_pairs(DevGeom g, WaveDev w, const double* __restrict__ wvn, int nfp,
                              const double* __restrict__ xfp, double2* __restrict__ Sf, double2* __restrict__ Df,
                              int* ovf) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (f >= nfp) return;
  const double xp = xfp[f], yp = xfp[f + nfp], zp = xfp[f + 2 * (size_t)nfp];
  const double xq = g.xq[j], yq = g.xq[j + g.n], zq = g.xq[j + 2 * g.n];
  const double dist = sqrt((xp - xq) * (xp - xq) + (yp - yq) * (yp - yq) + (zp - zq) * (zp - zq));
  const int flag = dist <= 50.0 * g.pnsz[j] ? 1 : 0;
  const double xf[3] = {xp, yp, zp};
  hams::rk4 r;
  if (g.ncn[j] == 3) {
    double q[3][3];
    for (int v = 0; v < 3; ++v)
      for (int c = 0; c < 3; ++c) q[v][c] = g.vtx[(size_t)j * 12 + v * 3 + c];
    r = hams::sglint_tri(xf, q);
  } else {
    double q[4][3];
    for (int v = 0; v < 4; ++v)
      for (int c = 0; c < 3; ++c) q[v][c] = g.vtx[(size_t)j * 12 + v * 3 + c];
    r = hams::sglint_quad(xf, q);
  }
  grn4 G;
  if (w.limit) {
    G = hams::green_limit(w.limit == 2, xq, xp, yq, yp, zq, zp, flag);
  } else if (w.h < 0.0) {
    G = hams::infgreen3d(xq, xp, yq, yp, zq, zp, w.v, flag);
  } else {
    int o = 0;
    const double rr = sqrt((xq - xp) * (xq - xp) + (yq - yp) * (yq - yp));
    switch (hams::fin_branch(rr, w.h)) {
      case hams::kLinton: G = hams::fingreen3d<hams::kLinton>(xq, xp, yq, yp, zq, zp, w.v, wvn, w.h, flag, (void*)nullptr, &o); break;
      case hams::kPidcock: {
        hams::SeriesScratchN<hams::kPidcockMax> sc;
        G = hams::fingreen3d<hams::kPidcock>(xq, xp, yq, yp, zq, zp, w.v, wvn, w.h, flag, &sc, &o);
        break;
      }
      case hams::kEigenE: {
        hams::SeriesScratchN<hams::kEigenEMax> sc;
        G = hams::fingreen3d<hams::kEigenE>(xq, xp, yq, yp, zq, zp, w.v, wvn, w.h, flag, &sc, &o);
        break;
      }
      default: G = hams::fingreen3d<hams::kEigen>(xq, xp, yq, yp, zq, zp, w.v, wvn, w.h, flag, (void*)nullptr, &o); break;
    }
    if (o) atomicOr(ovf, 1);
  }
  const double ds = g.ds[j], n1 = g.nrm[j], n2 = g.nrm[j + g.n], n3 = g.nrm[j + 2 * g.n];
  double sre = G.g[0].re * ds, sim = G.g[0].im * ds;
  double dre = (G.g[1].re * n1 + G.g[2].re * n2 + G.g[3].re * n3) * ds;
  double dim = (G.g[1].im * n1 + G.g[2].im * n2 + G.g[3].im * n3) * ds;
  if (flag) {
    sre = r.s + G.g[0].re * ds;
    dre = (r.dx + G.g[1].re * ds) * n1 + (r.dy + G.g[2].re * ds) * n2 + (r.dz + G.g[3].re * ds) * n3;
  }
  Sf[f + (size_t)nfp * j] = make_double2(sre, sim);
  Df[f + (size_t)nfp * j] = make_double2(dre, dim);
}

void launch_field_pairs(cudaStream_t st, DevGeom g, WaveDev w, const double* wvn, int nfp, const double* xfp,
                        double2* Sf, double2* Df, int* ovf) {
  k_field_pairs<<<dim3((nfp + 127) / 128, g.n), 128, 0, st>>>(g, w, wvn, nfp, xfp, Sf, Df, ovf);
}

void launch_eval_green(unsigned blocks, cudaStream_t st, int npts, const double* pts, const int* flag, WaveDev w,
                       const double* wvn, double2* out, int* ovf) {
  k_eval_green<<<blocks, 128, 0, st>>>(npts, pts, flag, w, wvn, out, ovf);
}
