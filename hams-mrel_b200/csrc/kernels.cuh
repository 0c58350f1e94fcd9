// kernels.cuh -- definitions shared by the assembly kernels of hams_gpu.cu
// and the epsilon-series kernels of green_series.cu.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "green.cuh"

using hams::cplx;
using hams::grn4;

// geometry as the kernels see it
struct DevGeom {
  int n, tn, nb;
  const double* xq;    // source centres (n,3)
  const double* fxyz;  // field points (tn,3): hull centres then lid centres
  const double* ds;    // (n)
  const double* pnsz;  // (n)
  const double* nrm;   // (n,6)
  const double* vtx;   // (n,4,3): vertices of each source panel (v = 0..3)
  const int* ncn;      // (n)
  const int* body;     // (n) body of each source panel
  const int* bstart;   // (nb+1)
};

struct WaveDev {
  double v, wk, w1, h;
  int limit;  // 0 regular, 1 zero frequency, 2 infinite frequency
};

__device__ __forceinline__ int near_flag(const DevGeom& g, int i, int j) {
  double dx = g.fxyz[i] - g.xq[j], dy = g.fxyz[i + g.tn] - g.xq[j + g.n], dz = g.fxyz[i + 2 * g.tn] - g.xq[j + 2 * g.n];
  return sqrt(dx * dx + dy * dy + dz * dz) <= 50.0 * g.pnsz[j] ? 1 : 0;
}

// A(I,J) (double layer, with 2 pi on the hull diagonal) and S(I,J) (single
// layer) of one pair from its Green-function set, as BODINT_MULTI_LEFT and
// RBC/DBC_MULTI_RIGHT combine them (BodyIntgrMulti.f90:48-173).
// The same from the pair's source-panel area ds, normal n1..n3 and Rankine
// terms rsp, rdp already in registers.
__device__ __forceinline__ void store_pair_v(size_t p, int i, int j, const grn4& G, double ds, double n1, double n2,
                                             double n3, double rsp, double rdp, double2* __restrict__ A,
                                             double2* __restrict__ S) {
  double are = rdp + ds * (G.g[1].re * n1 + G.g[2].re * n2 + G.g[3].re * n3);
  double aim = ds * (G.g[1].im * n1 + G.g[2].im * n2 + G.g[3].im * n3);
  if (i == j) are += 2.0 * 3.141592653589793;  // A(I,I) = 2 pi on hull rows (AssbMatxMulti.f90:75)
  A[p] = make_double2(are, aim);
  S[p] = make_double2(rsp + G.g[0].re * ds, G.g[0].im * ds);
}

__device__ __forceinline__ void store_pair(const DevGeom& g, size_t p, int i, int j, const grn4& G,
                                           const double* __restrict__ rs, const double* __restrict__ rd,
                                           double2* __restrict__ A, double2* __restrict__ S) {
  store_pair_v(p, i, j, G, g.ds[j], g.nrm[j], g.nrm[j + g.n], g.nrm[j + 2 * g.n], rs[p], rd[p], A, S);
}


// Launchers of the kernels compiled without implicit fused multiply-adds
// (green_series.cu): the EIGENE (br = 2) and PIDCOCK (br = 1) branches, whose
// epsilon-extrapolated series must see the same operation sequence as the
// CPU checker, the per-frequency mode tables they read, and the batch
// evaluator.
void launch_green_series(int br, unsigned blocks, cudaStream_t st, DevGeom g, WaveDev w, const double* wvn,
                         const hams::ModeTab& mt, const uint32_t* pairs, long long count, const double* rs,
                         const double* rd, double2* A, double2* S, int* ovf);
void launch_mode_tables(cudaStream_t st, DevGeom g, WaveDev w, const double* wvn, int nmode, double* pm, double* ac,
                        double2* src, double2* srct, double* fld, double* fldt);
void launch_eval_green(unsigned blocks, cudaStream_t st, int npts, const double* pts, const int* flag, WaveDev w,
                       const double* wvn, double2* out, int* ovf);
// Influence of every hull panel at nfp field points xfp (nfp,3): Sf, Df (nfp x n).
void launch_field_pairs(cudaStream_t st, DevGeom g, WaveDev w, const double* wvn, int nfp, const double* xfp,
                        double2* Sf, double2* Df, int* ovf);
