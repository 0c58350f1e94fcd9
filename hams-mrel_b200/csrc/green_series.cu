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


void launch_eval_green(unsigned blocks, cudaStream_t st, int npts, const double* pts, const int* flag, WaveDev w,
                       const double* wvn, double2* out, int* ovf) {
  k_eval_green<<<blocks, 128, 0, st>>>(npts, pts, flag, w, wvn, out, ovf);
}
