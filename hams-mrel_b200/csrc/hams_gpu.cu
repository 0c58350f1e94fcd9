// hams_gpu.cu -- B200 per-frequency BEM build-and-solve behind the C ABI of
// include/hams_gpu.h.
//
// Device pipeline of one frequency (N hull panels, NL lid panels, TN = N+NL
// field points, NB bodies, NBETA headings):
//   1. green kernels  -- per Green-function branch, over the branch's sorted
//      pair list: FINGREEN3D / INFGREEN3D for the pair, fused with the
//      BODINT_MULTI_LEFT / RBC algebra, writes A(I,J) (double layer) and
//      S(I,J) (single layer) in FP64 complex, column-major TN x N.
//   2. rhs kernels    -- B_rad(I,6b+m) = sum_{J in b} S(I,J) n_m(J) and
//      B_dif(I,beta) = -sum_J S(I,J) (grad phi_I . n)(J), chunked over J with
//      a fixed-order final sum (deterministic).
//   3. lid rows       -- C = A^T A, D = A^T B (plain transpose, as
//      AssbMatx_irrMulti.f90:151-169,300-315,447-460) with cuBLAS ZGEMM.
//   4. solve          -- FP64: cuSOLVER ZGETRF/ZGETRS.  Mixed: complex64
//      CGETRF of a rounded copy, then FP64 iterative refinement with the
//      FP64 matrix kept in HBM (residual r = b - A x by ZGEMM, correction by
//      CGETRS, update in FP64).
//   5. force kernels  -- RFORCE_MULTI / EFORCE_MULTI reductions.
// Frequency-independent work (Rankine panel integrals, branch sort of the
// pairs) happens once in hams_ctx_create.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <complex>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include "../../include/hams_gpu.h"
#include "green.cuh"
#include "rankine.cuh"

using hams::cplx;
using hams::grn4;

// ---------------------------------------------------------------------------
// error reporting
// ---------------------------------------------------------------------------
static thread_local std::string g_err;

static int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CU(call)                                                                                \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) return fail(HAMS_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call, \
                                       cudaGetErrorString(e_));                                 \
  } while (0)
#define CUB_(call)                                                                                       \
  do {                                                                                                   \
    cublasStatus_t e_ = (call);                                                                          \
    if (e_ != CUBLAS_STATUS_SUCCESS) return fail(HAMS_ERR_CUDA, "%s:%d %s: cublas status %d", __FILE__, \
                                                 __LINE__, #call, (int)e_);                              \
  } while (0)
#define CUS(call)                                                                                          \
  do {                                                                                                     \
    cusolverStatus_t e_ = (call);                                                                          \
    if (e_ != CUSOLVER_STATUS_SUCCESS) return fail(HAMS_ERR_CUDA, "%s:%d %s: cusolver status %d", __FILE__, \
                                                   __LINE__, #call, (int)e_);                              \
  } while (0)
#define TRY(call)           \
  do {                      \
    int rc_ = (call);       \
    if (rc_ < 0) return rc_; \
  } while (0)

#include "kernels.cuh"
#include "lu_mixed.h"
#include "gemm_tf32.h"
#include "green_sg.h"
#include "hmatrix.h"
#include "surrogate.h"

// ---------------------------------------------------------------------------
// setup kernels
// ---------------------------------------------------------------------------
// Rankine integrals of every (field, source) pair: rs = FLAG * SIJ,
// rd = FLAG * DIJ . n_J (the only Rankine quantities the assembly uses).
__global__ void k_rankine(DevGeom g, double* __restrict__ rs, double* __restrict__ rd) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y;
  if (i >= g.tn) return;
  size_t p = (size_t)i + (size_t)j * g.tn;
  if (!near_flag(g, i, j)) {
    rs[p] = 0.0;
    rd[p] = 0.0;
    return;
  }
  double xf[3] = {g.fxyz[i], g.fxyz[i + g.tn], g.fxyz[i + 2 * g.tn]};
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
  rs[p] = r.s;
  rd[p] = r.dx * g.nrm[j] + r.dy * g.nrm[j + g.n] + r.dz * g.nrm[j + 2 * g.n];
}

// Sort key of a pair: branch << 8 | series length.  With the surrogate on,
// EIGENE / EIGEN pairs farther apart than far x the source panel's size and
// inside the network's domain go to bins 4 (EIGENE) and 5 (EIGEN).  Pairs of
// a body block copied from an identical one (copied[field body + nb x source
// body], hams_opts.body_blocks) go to bin 6, which no Green kernel reads.
__global__ void k_pair_keys(DevGeom g, double h, int sg_on, double far, const unsigned char* __restrict__ copied,
                            uint32_t* __restrict__ keys, uint32_t* __restrict__ idx) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y;
  if (i >= g.tn) return;
  size_t p = (size_t)i + (size_t)j * g.tn;
  double dx = g.xq[j] - g.fxyz[i], dy = g.xq[j + g.n] - g.fxyz[i + g.tn];
  double rr = sqrt(dx * dx + dy * dy);
  int b = hams::fin_branch(rr, h);
  int nt = hams::fin_terms(rr, h);
  if (sg_on && (b == hams::kEigenE || b == hams::kEigen)) {
    double zq = g.xq[j + 2 * g.n], zp = g.fxyz[i + 2 * g.tn], dz = zq - zp;
    bool far_pair = sqrt(dx * dx + dy * dy + dz * dz) > far * g.pnsz[j];
    if (far_pair && sg::in_domain(rr / h, (zq + h) / h, (zp + h) / h, sg::kKmin)) b = b == hams::kEigenE ? 4 : 5;
  }
  if (copied && i < g.n && copied[g.body[i] + g.nb * g.body[j]]) b = 6;
  keys[p] = (uint32_t)(b << 8) | (uint32_t)(nt & 0xff);
  idx[p] = (uint32_t)p;
}

// First index of each bin b = 0..nbins in the sorted keys (key >> 8 is the bin).
__global__ void k_bin_offsets(const uint32_t* __restrict__ keys, long long np, int nbins, long long* off) {
  const int b = threadIdx.x;
  if (b > nbins) return;
  const uint32_t v = (uint32_t)b << 8;
  long long lo = 0, hi = np;
  while (lo < hi) {
    const long long mid = lo + (hi - lo) / 2;
    if (keys[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  off[b] = lo;
}

// ---------------------------------------------------------------------------
// per-frequency assembly: Green function fused with the pair algebra
// ---------------------------------------------------------------------------
// LINTON (BR = 0) and EIGEN (BR = 3) pairs; the epsilon-series branches are
// in green_series.cu.
// EIGEN runs at 8 blocks per SM like the series kernels; LINTON's adaptive
// quadrature keeps its registers.
// ---------------------------------------------------------------------------
// the series' judgement of the surrogate
// ---------------------------------------------------------------------------
// dst[k] = src[k * stride], k < count
__global__ void k_stride_pick(const uint32_t* __restrict__ src, long long count, long long stride,
                              uint32_t* __restrict__ dst) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < count) dst[k] = src[k * stride];
}

// the A and S entries of the listed pairs: out[k] = A[p_k], out[ns + k] = S[p_k]
__global__ void k_gather_pairs(const uint32_t* __restrict__ list, int ns, const double2* __restrict__ A,
                               const double2* __restrict__ S, double2* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ns) return;
  out[k] = A[list[k]];
  out[ns + k] = S[list[k]];
}

// out = {sum |A1 - A2|^2, sum (Re A2)^2, sum |S1 - S2|^2, sum (Re S2)^2} over the samples (one CTA)
__global__ void __launch_bounds__(1024) k_sample_err(const double2* __restrict__ g1, const double2* __restrict__ g2,
                                                     int ns, double* __restrict__ out) {
  __shared__ double red[4][32];
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  for (int k = threadIdx.x; k < ns; k += blockDim.x) {
    const double2 a1 = g1[k], a2 = g2[k], s1 = g1[ns + k], s2 = g2[ns + k];
    v[0] += (a1.x - a2.x) * (a1.x - a2.x) + (a1.y - a2.y) * (a1.y - a2.y);
    v[1] += a2.x * a2.x;
    v[2] += (s1.x - s2.x) * (s1.x - s2.x) + (s1.y - s2.y) * (s1.y - s2.y);
    v[3] += s2.x * s2.x;
  }
  for (int q = 0; q < 4; ++q) {
    for (int o = 16; o; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = v[q];
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    for (int q = 0; q < 4; ++q) {
      double x = threadIdx.x < (blockDim.x >> 5) ? red[q][threadIdx.x] : 0.0;
      for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if (threadIdx.x == 0) out[q] = x;
    }
  }
}

// The network's error is modelled per cell of its input domain: R/h (log,
// kJX cells) x source depth x field depth ((z + h)/h, kJZ cells each).
constexpr int kJX = 24, kJZ = 3, kJCells = kJX * kJZ * kJZ;

__device__ __forceinline__ int judge_cell(double X, double Zq, double Zp) {
  const int cx = min(kJX - 1, max(0, (int)(kJX * log(X / sg::kXmin) / log(sg::kXmax / sg::kXmin))));
  const int cq = min(kJZ - 1, max(0, (int)(kJZ * (Zq - sg::kZmin) / (sg::kZmax - sg::kZmin))));
  const int cp = min(kJZ - 1, max(0, (int)(kJZ * (Zp - sg::kZmin) / (sg::kZmax - sg::kZmin))));
  return cx + kJX * (cq + kJZ * cp);
}

__device__ __forceinline__ int pair_cell(const DevGeom& g, double h, size_t p) {
  const int i = (int)(p % (size_t)g.tn), j = (int)(p / (size_t)g.tn);
  const double dx = g.xq[j] - g.fxyz[i], dy = g.xq[j + g.n] - g.fxyz[i + g.tn];
  return judge_cell(sqrt(dx * dx + dy * dy) / h, (g.xq[j + 2 * g.n] + h) / h, (g.fxyz[i + 2 * g.tn] + h) / h);
}

// Per cell, the sampled sums acc[4c..4c+3] += {(network - series)^2,
// (Re series)^2} of the A entries, then of the S entries (acc zeroed by the
// caller): the cell's RMS relative error of the network is the square root
// of their ratio.
__global__ void k_judge_fit(DevGeom g, double h, const uint32_t* __restrict__ list, int ns,
                            const double2* __restrict__ g1, const double2* __restrict__ g2, double* __restrict__ acc) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ns) return;
  const int c = pair_cell(g, h, list[k]);
  const double2 a1 = g1[k], a2 = g2[k], s1 = g1[ns + k], s2 = g2[ns + k];
  atomicAdd(acc + 4 * c, (a1.x - a2.x) * (a1.x - a2.x) + (a1.y - a2.y) * (a1.y - a2.y));
  atomicAdd(acc + 4 * c + 1, a2.x * a2.x);
  atomicAdd(acc + 4 * c + 2, (s1.x - s2.x) * (s1.x - s2.x) + (s1.y - s2.y) * (s1.y - s2.y));
  atomicAdd(acc + 4 * c + 3, s2.x * s2.x);
}

// The judgement's cell map: for every pair (i, j) (entry i + j tn) the cell
// of the network's input domain when the network evaluates the pair (the
// criterion of k_pair_keys' bins 4 and 5, copied body blocks included), else
// kNoCell.  Frequency-independent: built once with the surrogate.
constexpr unsigned char kNoCell = 255;
static_assert(kJCells < kNoCell, "cell index must fit below kNoCell");
__global__ void k_probe_map(DevGeom g, double h, double far, unsigned char* __restrict__ map) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (i >= g.tn) return;
  const double dx = g.xq[j] - g.fxyz[i], dy = g.xq[j + g.n] - g.fxyz[i + g.tn];
  const double rr = sqrt(dx * dx + dy * dy);
  const int b = hams::fin_branch(rr, h);
  unsigned char cell = kNoCell;
  if (b == hams::kEigenE || b == hams::kEigen) {
    const double zq = g.xq[j + 2 * g.n], zp = g.fxyz[i + 2 * g.tn], dz = zq - zp;
    if (sqrt(dx * dx + dy * dy + dz * dz) > far * g.pnsz[j] &&
        sg::in_domain(rr / h, (zq + h) / h, (zp + h) / h, sg::kKmin))
      cell = (unsigned char)judge_cell(rr / h, (zq + h) / h, (zp + h) / h);
  }
  map[(size_t)i + (size_t)j * g.tn] = cell;
}

// The probe scales of this frequency: per cell the network's RMS relative
// error on A (scale[2c]) and S (scale[2c + 1]) from the sampled sums acc.
// The error probe of an entry is its cell's scale times the entry's real
// part -- the network's error with its cell's size and the same sign
// everywhere, the coherent case; 0 for the pairs the network leaves alone.
__global__ void k_probe_scales(const double* __restrict__ acc, double* __restrict__ scale) {
  for (int c = threadIdx.x; c < kJCells; c += blockDim.x) {
    scale[2 * c] = acc[4 * c + 1] > 0.0 ? sqrt(acc[4 * c] / acc[4 * c + 1]) : 0.0;
    scale[2 * c + 1] = acc[4 * c + 3] > 0.0 ? sqrt(acc[4 * c + 2] / acc[4 * c + 3]) : 0.0;
  }
}

// B (tn x nrhs, ld tn) -= PA X with PA the error probe of A and X (n x nrhs,
// ld n, complex64), the probe never stored; FP32 products and sums (the
// result is an error estimate).  A block: 32 rows x 64 right-hand sides, j
// in tiles of 32 through double-buffered shared memory, the next tile's
// values loaded into registers while the current one is applied; each of
// the 256 threads owns 2 rows x 4 right-hand sides.  Grid: ceil(tn / 32).
constexpr int kPrRows = 32, kPrCols = 64, kPrJ = 32, kPrXLd = kPrCols + 2, kPrThreads = 256;
__global__ void __launch_bounds__(kPrThreads) k_probe_apply(DevGeom g, const unsigned char* __restrict__ map,
                                                            const double* __restrict__ scale,
                                                            const double2* __restrict__ A,
                                                            const float2* __restrict__ X, int nrhs,
                                                            double2* __restrict__ B) {
  __shared__ __align__(16) float sP[2][kPrJ][kPrRows];
  __shared__ __align__(16) float2 sX[2][kPrJ][kPrXLd];
  __shared__ float sScale[kJCells];
  const int t = threadIdx.x, i0 = blockIdx.x * kPrRows, rg = t & 15, cg = t >> 4;
  for (int c = t; c < kJCells; c += kPrThreads) sScale[c] = (float)scale[2 * c];
  __syncthreads();
  constexpr int kLP = kPrJ * kPrRows / kPrThreads, kLX = kPrJ * kPrCols / kPrThreads;  // loads per thread
  const int il = t & 31, jq = t >> 5;  // loader roles: row il of the P tile; X tile row il, columns jq + 8 q
  for (int k0 = 0; k0 < nrhs; k0 += kPrCols) {
    float2 a[2][4];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int q = 0; q < 4; ++q) a[r][q] = make_float2(0.0f, 0.0f);
    float pv[kLP];
    float2 xv[kLX];
    auto load = [&](int j0) {
      const int i = i0 + il;
#pragma unroll
      for (int q = 0; q < kLP; ++q) {
        const int j = j0 + jq + 8 * q;
        float v = 0.0f;
        if (i < g.tn && j < g.n) {
          const size_t p = (size_t)i + (size_t)j * g.tn;
          const unsigned char cell = map[p];
          if (cell != kNoCell) v = sScale[cell] * (float)A[p].x;
        }
        pv[q] = v;
      }
      const int j = j0 + il;
#pragma unroll
      for (int q = 0; q < kLX; ++q) {
        const int k = k0 + jq + 8 * q;
        xv[q] = (j < g.n && k < nrhs) ? X[(size_t)j + (size_t)k * g.n] : make_float2(0.0f, 0.0f);
      }
    };
    auto store = [&](int buf) {
#pragma unroll
      for (int q = 0; q < kLP; ++q) sP[buf][jq + 8 * q][il] = pv[q];
#pragma unroll
      for (int q = 0; q < kLX; ++q) sX[buf][il][jq + 8 * q] = xv[q];
    };
    load(0);
    store(0);
    __syncthreads();
    int buf = 0;
    for (int j0 = 0; j0 < g.n; j0 += kPrJ) {
      const bool more = j0 + kPrJ < g.n;
      if (more) load(j0 + kPrJ);  // in flight while the current tile is applied
#pragma unroll 8
      for (int jl = 0; jl < kPrJ; ++jl) {
        const float2 p = *reinterpret_cast<const float2*>(&sP[buf][jl][2 * rg]);
        const float4 x01 = *reinterpret_cast<const float4*>(&sX[buf][jl][4 * cg]);
        const float4 x23 = *reinterpret_cast<const float4*>(&sX[buf][jl][4 * cg + 2]);
        const float2 x[4] = {make_float2(x01.x, x01.y), make_float2(x01.z, x01.w), make_float2(x23.x, x23.y),
                             make_float2(x23.z, x23.w)};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          a[0][q].x = fmaf(p.x, x[q].x, a[0][q].x);
          a[0][q].y = fmaf(p.x, x[q].y, a[0][q].y);
          a[1][q].x = fmaf(p.y, x[q].x, a[1][q].x);
          a[1][q].y = fmaf(p.y, x[q].y, a[1][q].y);
        }
      }
      if (more) store(buf ^ 1);  // the other buffer: its last readers passed the barrier below
      __syncthreads();
      buf ^= 1;
    }
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int i = i0 + 2 * rg + r;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int k = k0 + 4 * cg + q;
        if (i < g.tn && k < nrhs) {
          double2* o = B + (size_t)i + (size_t)k * g.tn;
          *o = make_double2(o->x - (double)a[r][q].x, o->y - (double)a[r][q].y);
        }
      }
    }
    __syncthreads();  // the buffers are reloaded for the next chunk of right-hand sides
  }
}

template <int BR>
__global__ void __launch_bounds__(128, BR == hams::kEigen ? 8 : 1) k_green_fin(DevGeom g, WaveDev w, const double* __restrict__ wvn,
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
    int o = 0;
    hams::TableModes md{mt, j, i};
    G = hams::fingreen3d<BR>(xq, xp, yq, yp, zq, zp, w.v, wvn, w.h, flag, (void*)nullptr, &o, md);
    if (o) atomicOr(ovf, 1);
  }
  store_pair(g, p, i, j, G, rs, rd, A, S);
}

// The LINTON branch with one warp per pair: the pair's adaptive
// Gauss-Kronrod integrals spread their nodes over the warp's lanes
// (hams::WarpQuad); lane 0 stores the pair.  The branch has few pairs (the
// panels of one vertical column of a body), each a long chain of FP64
// quadrature, so a thread per pair leaves most of the GPU idle.  128 threads
// per CTA, 4 pairs.
constexpr int kLintonWarps = 4;
// Below this many LINTON pairs per SM the warp-per-pair kernel runs (on the
// 5,400-panel 3 x 3 array: 4,200 pairs with body blocks 1.5 ms against 6.5 ms
// for a thread per pair at 0.2 rad/s; all 37,800 pairs 9.2 ms against 3.7 ms,
// mean over frequencies).
constexpr int kLintonWarpPairsPerSm = 64;
__global__ void __launch_bounds__(32 * kLintonWarps) k_green_linton(DevGeom g, WaveDev w, const double* __restrict__ wvn,
                                                                  const uint32_t* __restrict__ pairs, long long count,
                                                                  const double* __restrict__ rs,
                                                                  const double* __restrict__ rd,
                                                                  double2* __restrict__ A, double2* __restrict__ S,
                                                                  int* ovf) {
  __shared__ double stack[kLintonWarps][2][hams::kQuadStack];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const long long t = (long long)blockIdx.x * kLintonWarps + wl;
  if (t >= count) return;  // the whole warp
  size_t p = pairs[t];
  int i = (int)(p % (size_t)g.tn), j = (int)(p / (size_t)g.tn);
  int flag = near_flag(g, i, j);
  double xp = g.fxyz[i], yp = g.fxyz[i + g.tn], zp = g.fxyz[i + 2 * g.tn];
  double xq = g.xq[j], yq = g.xq[j + g.n], zq = g.xq[j + 2 * g.n];
  grn4 G;
  if (w.limit) {
    G = hams::green_limit(w.limit == 2, xq, xp, yq, yp, zq, zp, flag);
  } else {
    int o = 0;
    const hams::WarpQuad quad{stack[wl][0], stack[wl][1], lane};
    G = hams::fingreen3d_linton(xq, xp, yq, yp, zq, zp, w.v, wvn, w.h, flag, &o, quad);
    if (o && lane == 0) atomicOr(ovf, 1);
  }
  if (lane == 0) store_pair(g, p, i, j, G, rs, rd, A, S);
}

__global__ void __launch_bounds__(128) k_green_inf(DevGeom g, WaveDev w, const unsigned char* __restrict__ copied,
                                                   const double* __restrict__ rs, const double* __restrict__ rd,
                                                   double2* __restrict__ A, double2* __restrict__ S) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int j = blockIdx.y;
  if (i >= g.tn) return;
  if (copied && i < g.n && copied[g.body[i] + g.nb * g.body[j]]) return;  // filled by k_copy_blocks
  size_t p = (size_t)i + (size_t)j * g.tn;
  int flag = near_flag(g, i, j);
  double xp = g.fxyz[i], yp = g.fxyz[i + g.tn], zp = g.fxyz[i + 2 * g.tn];
  double xq = g.xq[j], yq = g.xq[j + g.n], zq = g.xq[j + 2 * g.n];
  grn4 G = w.limit ? hams::green_limit(w.limit == 2, xq, xp, yq, yp, zq, zp, flag)
                   : hams::infgreen3d(xq, xp, yq, yp, zq, zp, w.v, flag);
  store_pair(g, p, i, j, G, rs, rd, A, S);
}

// Body blocks of identical body pairs (hams_opts.body_blocks): blk holds 6
// ints per block -- destination first row and column, source first row and
// column, rows, columns -- and block z copies its A and S entries, one
// source column per blockIdx.y, after the Green kernels have filled the
// source block.
__global__ void __launch_bounds__(256) k_copy_blocks(const int* __restrict__ blk, int tn, double2* __restrict__ A,
                                                     double2* __restrict__ S) {
  const int* b = blk + 6 * blockIdx.z;
  const int nj = b[5], ni = b[4];
  for (int j = blockIdx.y; j < nj; j += gridDim.y) {
    const size_t d0 = (size_t)b[0] + (size_t)(b[1] + j) * tn, s0 = (size_t)b[2] + (size_t)(b[3] + j) * tn;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ni; i += gridDim.x * blockDim.x) {
      A[d0 + i] = A[s0 + i];
      S[d0 + i] = S[s0 + i];
    }
  }
}

// ---------------------------------------------------------------------------
// incident wave (PatclVelct.f90:42-123)
// ---------------------------------------------------------------------------
struct IncWave {
  double w0, wk0, h, amp, g, xw0, xw1;
};

__host__ __device__ inline IncWave inc_params(const WaveDev& w, double amp, double g, double xw0, double xw1) {
  IncWave o;
  if (fabs(w.v) < HAMS_F4(1.E-8)) {
    o.w0 = HAMS_F4(1.E-20);
    o.wk0 = HAMS_F4(1.E-20);
  } else if (fabs(w.v + 1.0) < HAMS_F4(1.E-8)) {
    o.w0 = HAMS_F4(1.E+20);
    o.wk0 = HAMS_F4(1.E+20);
  } else {
    o.w0 = w.w1;
    o.wk0 = w.wk;
  }
  o.h = w.h;
  o.amp = amp;
  o.g = g;
  o.xw0 = xw0;
  o.xw1 = xw1;
  return o;
}

// grad(phi_I) . n at (x,y,z) for heading beta (DINP, PatclVelct.f90:83)
__device__ __forceinline__ cplx dinp_n(const IncWave& q, double x, double y, double z, double beta, double n1,
                                        double n2, double n3) {
  double sb, cb, s, c;
  sincos(beta, &sb, &cb);
  double wkx = q.wk0 * ((x - q.xw0) * cb + (y - q.xw1) * sb);
  sincos(wkx, &s, &c);
  double fh, fv;
  if (q.h < 0.0) {
    fh = fv = exp(q.wk0 * z);
  } else {
    double sh = sinh(q.wk0 * q.h);
    fh = cosh(q.wk0 * (z + q.h)) / sh;
    fv = sinh(q.wk0 * (z + q.h)) / sh;
  }
  // DPOX/CI = -i * w0 amp fh e^{i wkx} cos(beta); DPOZ/CI = -w0 amp fv e^{i wkx}
  double a = q.w0 * q.amp;
  cplx e = hams::cmk(c, s);
  cplx dx = hams::cmk(e.im, -e.re) * (a * fh * cb);
  cplx dy = hams::cmk(e.im, -e.re) * (a * fh * sb);
  cplx dz = e * (-a * fv);
  return dx * n1 + dy * n2 + dz * n3;
}

// phi_I at (x,y,z) (VINP, PatclVelct.f90:42)
__device__ __forceinline__ cplx vinp(const IncWave& q, double x, double y, double z, double beta) {
  double sb, cb, s, c;
  sincos(beta, &sb, &cb);
  double wkx = q.wk0 * ((x - q.xw0) * cb + (y - q.xw1) * sb);
  sincos(wkx, &s, &c);
  cplx e = hams::cmk(c, s);
  if (q.h < 0.0 || q.h > 500.0) {
    // (-i amp g / w0 e^{k z} e^{i wkx}) / i
    return e * (-q.amp * q.g / q.w0 * exp(q.wk0 * z));
  }
  double dum = -q.amp * q.w0 / (q.wk0 * sinh(q.wk0 * q.h));
  return e * (dum * cosh(q.wk0 * (z + q.h)));
}

// Boundary values of the field-point potentials (CalPotentialMulti,
// PressureElevationMulti.f90:161-230): column 6b+m the generalized normal m
// on the panels of body b (FACTOR_NORMAL), column 6nb+k minus the incident
// normal velocity of heading k.
__global__ void k_field_bc(DevGeom g, int nbeta, const double2* __restrict__ wd, double2* __restrict__ bc) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, col = blockIdx.y;
  if (j >= g.n) return;
  double2 v = make_double2(0.0, 0.0);
  if (col < 6 * g.nb) {
    if (g.body[j] == col / 6) v.x = g.nrm[j + (size_t)(col % 6) * g.n];
  } else {
    const double2 q = wd[j + (size_t)(col - 6 * g.nb) * g.n];
    v = make_double2(-q.x, -q.y);
  }
  bc[j + (size_t)g.n * col] = v;
}

// out (nfp, ncol + nbeta): the summed potentials over 2 pi or 4 pi, the
// incident potential added to the diffraction columns of the total-potential
// solution (PressureElevationMulti.f90:253-266), then the incident potential
// alone per heading (CalPotentialIncMulti, :277-300).
__global__ void k_field_finish(int nfp, int ncol, int nrad, int nbeta, const double* __restrict__ xfp,
                               const double* __restrict__ sld, IncWave q, const double* __restrict__ beta, int add_inc,
                               const double2* __restrict__ pot, double2* __restrict__ out) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x, col = blockIdx.y;
  if (f >= nfp) return;
  cplx inc = hams::cmk(0.0, 0.0);
  const int k = col < ncol ? col - nrad : col - ncol;
  if (add_inc && (col >= ncol || col >= nrad)) inc = vinp(q, xfp[f], xfp[f + nfp], xfp[f + 2 * (size_t)nfp], beta[k]);
  double2 v;
  if (col < ncol) {
    const double2 p = pot[f + (size_t)nfp * col];
    v = make_double2(p.x / sld[f], p.y / sld[f]);
    if (col >= nrad) v = make_double2(v.x + inc.re, v.y + inc.im);
  } else {
    v = make_double2(inc.re, inc.im);
  }
  out[f + (size_t)nfp * col] = v;
}

// w(J,beta) = grad(phi_I)(x_J) . n_J for every source panel and heading
__global__ void k_dbc_weights(DevGeom g, WaveDev w, IncWave q, const double* __restrict__ beta, int nbeta,
                              double2* __restrict__ wd) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  int b = blockIdx.y;
  if (j >= g.n || b >= nbeta) return;
  cplx r = dinp_n(q, g.xq[j], g.xq[j + g.n], g.xq[j + 2 * g.n], beta[b], g.nrm[j], g.nrm[j + g.n],
                  g.nrm[j + 2 * g.n]);
  wd[j + (size_t)b * g.n] = make_double2(r.re, r.im);
}

// ---------------------------------------------------------------------------
// right-hand sides: chunked reductions over source panels
// ---------------------------------------------------------------------------
constexpr int kChunk = 256;  // source panels per chunk (chunks never straddle bodies)

// part(c, I, k): k < 6 radiation mode k of the chunk's body, k >= 6 heading k-6.
// With PROBE the entries of S are replaced by their error probe (the scale
// of their cell, map and k_probe_scales, times Re S): the right-hand sides of
// the probe.
template <bool PROBE>
__global__ void __launch_bounds__(128) k_rhs_partial(DevGeom g, const double2* __restrict__ S,
                                                     const int2* __restrict__ chunks, const double2* __restrict__ wd,
                                                     int nbeta, double2* __restrict__ part,
                                                     const unsigned char* __restrict__ map = nullptr,
                                                     const double* __restrict__ scale = nullptr) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int c = blockIdx.y;
  if (i >= g.tn) return;
  int j0 = chunks[c].x, j1 = chunks[c].y;
  int nk = 6 + nbeta;
  double2* out = part + ((size_t)c * g.tn + i) * nk;
  // one pass over the chunk's entries of S for the radiation sums and the
  // first 8 headings (each sum in the order of j, as before), one more per
  // further 8 headings
  double rr[6] = {0, 0, 0, 0, 0, 0}, ri[6] = {0, 0, 0, 0, 0, 0};
  for (int b0 = 0; b0 == 0 || b0 < nbeta; b0 += 8) {
    double dr[8] = {0, 0, 0, 0, 0, 0, 0, 0}, di[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int nbb = max(0, min(8, nbeta - b0));
    for (int j = j0; j < j1; ++j) {
      double2 s = S[(size_t)i + (size_t)j * g.tn];
      if (PROBE) {
        const unsigned char cell = map[(size_t)i + (size_t)j * g.tn];
        s = make_double2(cell != kNoCell ? scale[2 * cell + 1] * s.x : 0.0, 0.0);
      }
      if (b0 == 0) {
#pragma unroll
        for (int m = 0; m < 6; ++m) {
          double nm = g.nrm[j + (size_t)m * g.n];
          rr[m] += s.x * nm;
          ri[m] += s.y * nm;
        }
      }
#pragma unroll
      for (int b = 0; b < 8; ++b)
        if (b < nbb) {
          double2 wv = wd[j + (size_t)(b0 + b) * g.n];
          dr[b] -= s.x * wv.x - s.y * wv.y;
          di[b] -= s.x * wv.y + s.y * wv.x;
        }
    }
    if (b0 == 0)
      for (int m = 0; m < 6; ++m) out[m] = make_double2(rr[m], ri[m]);
    for (int b = 0; b < nbb; ++b) out[6 + b0 + b] = make_double2(dr[b], di[b]);
  }
}

// B (tn, 6nb + nbeta): radiation columns of body b, then diffraction columns.
__global__ void k_rhs_final(int tn, int nb, int nchunks, const int* __restrict__ chunk_body,
                            const double2* __restrict__ part, int nbeta, double2* __restrict__ B) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= tn) return;
  int nk = 6 + nbeta, ldb = tn;
  for (int b = 0; b < nb; ++b)
    for (int m = 0; m < 6; ++m) B[i + (size_t)(6 * b + m) * ldb] = make_double2(0.0, 0.0);
  for (int c = 0; c < nchunks; ++c) {
    const double2* p = part + ((size_t)c * tn + i) * nk;
    int b = chunk_body[c];
    for (int m = 0; m < 6; ++m) {
      double2 v = B[i + (size_t)(6 * b + m) * ldb];
      B[i + (size_t)(6 * b + m) * ldb] = make_double2(v.x + p[m].x, v.y + p[m].y);
    }
  }
  for (int k = 0; k < nbeta; ++k) {
    double sr = 0.0, si = 0.0;
    for (int c = 0; c < nchunks; ++c) {
      const double2* p = part + ((size_t)c * tn + i) * nk;
      sr += p[6 + k].x;
      si += p[6 + k].y;
    }
    B[i + (size_t)(6 * nb + k) * ldb] = make_double2(sr, si);
  }
}

// ---------------------------------------------------------------------------
// reductions (RFORCE_MULTI / EFORCE_MULTI)
// ---------------------------------------------------------------------------
// One block per (body bm, mode k, solution column col).
//   col < 6nb : amas(6bm+k, col) = rho sum DS n_k Re X ; bdmp = rho w1 sum DS n_k Im X
//   col >= 6nb: exfc(beta, 6bm+k) = i w1 rho sum (X + phi_I) DS n_k
__global__ void k_forces(DevGeom g, WaveDev w, IncWave q, const double* __restrict__ beta, int nbeta, int isol,
                         double rho, const double2* __restrict__ X, int ldx, double* __restrict__ amas,
                         double* __restrict__ bdmp, double2* __restrict__ exfc) {
  int bm = blockIdx.x, k = blockIdx.y, col = blockIdx.z;
  int ndof = 6 * g.nb;
  int i0 = g.bstart[bm], i1 = g.bstart[bm + 1];
  double sr = 0.0, si = 0.0;
  for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
    double2 x = X[i + (size_t)col * ldx];
    if (col >= ndof && isol == 1) {
      cplx f = vinp(q, g.xq[i], g.xq[i + g.n], g.xq[i + 2 * g.n], beta[col - ndof]);
      x.x += f.re;
      x.y += f.im;
    }
    double wgt = g.ds[i] * g.nrm[i + (size_t)k * g.n];
    sr += x.x * wgt;
    si += x.y * wgt;
  }
  __shared__ double shr[256], shi[256];
  shr[threadIdx.x] = sr;
  shi[threadIdx.x] = si;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      shr[threadIdx.x] += shr[threadIdx.x + s];
      shi[threadIdx.x] += shi[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  sr = shr[0];
  si = shi[0];
  if (col < ndof) {
    amas[(6 * bm + k) + (size_t)col * ndof] = rho * sr;
    bdmp[(6 * bm + k) + (size_t)col * ndof] = rho * w.w1 * si;
  } else {
    // i * w1 * rho * (sr + i si)
    exfc[(col - ndof) + (size_t)(6 * bm + k) * nbeta] = make_double2(-w.w1 * rho * si, w.w1 * rho * sr);
  }
}

// ---------------------------------------------------------------------------
// mixed precision helpers
// ---------------------------------------------------------------------------
__global__ void k_z2c(const double2* __restrict__ a, float2* __restrict__ b, size_t n) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (; t < n; t += (size_t)gridDim.x * blockDim.x) b[t] = make_float2((float)a[t].x, (float)a[t].y);
}
// b (ld ldb) <- the n x n complex128 matrix a (ld n) rounded to complex64
__global__ void k_z2c_ld(const double2* __restrict__ a, float2* __restrict__ b, int n, int ldb) {
  const size_t tot = (size_t)n * n;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (size_t)gridDim.x * blockDim.x)
    b[(t / n) * ldb + t % n] = make_float2((float)a[t].x, (float)a[t].y);
}
__global__ void k_c2z_add(const float2* __restrict__ a, double2* __restrict__ b, size_t n) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (; t < n; t += (size_t)gridDim.x * blockDim.x) b[t] = make_double2(b[t].x + (double)a[t].x, b[t].y + (double)a[t].y);
}
__global__ void k_c2z(const float2* __restrict__ a, double2* __restrict__ b, size_t n) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (; t < n; t += (size_t)gridDim.x * blockDim.x) b[t] = make_double2((double)a[t].x, (double)a[t].y);
}
// per-column max |r| / max |b| ratios -> out[col]
// d[i] = M[i, i], or 1 where |M[i, i]| < 1e-30 (IterativeSolvers.f90:166-171)
__global__ void k_jacobi_setup(const double2* __restrict__ M, int n, double2* __restrict__ d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double2 v = M[i + (size_t)i * n];
  d[i] = hypot(v.x, v.y) < 1e-30 ? make_double2(1.0, 0.0) : v;
}

// Z[i + n c] /= d[i]
__global__ void k_jacobi_apply(const double2* __restrict__ d, int n, int ncol, double2* __restrict__ Z) {
  size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)n * ncol) return;
  const double2 a = d[e % n], z = Z[e];
  const double den = a.x * a.x + a.y * a.y;
  Z[e] = make_double2((z.x * a.x + z.y * a.y) / den, (z.y * a.x - z.x * a.y) / den);
}

// out[c] = 2-norm of column c of W (n x ncol, ld n)
__global__ void k_colnorm2(const double2* __restrict__ W, int n, double* __restrict__ out) {
  const int col = blockIdx.x;
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double2 v = W[i + (size_t)col * n];
    s += v.x * v.x + v.y * v.y;
  }
  __shared__ double sh[256];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[col] = sqrt(sh[0]);
}

// dst[i + dstride c] = W[i + n c] / nrm[c], zero where nrm[c] <= 1e-30
// (IterativeSolvers.f90:412-416)
__global__ void k_normalize_into(const double2* __restrict__ W, int n, int ncol, const double* __restrict__ nrm,
                                 double2* __restrict__ dst, size_t dstride) {
  size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)n * ncol) return;
  const int c = (int)(e / n), i = (int)(e % n);
  const double s = nrm[c] > 1e-30 ? 1.0 / nrm[c] : 0.0;
  const double2 v = W[e];
  dst[i + dstride * c] = make_double2(v.x * s, v.y * s);
}

__global__ void k_colnorm_ratio(const double2* __restrict__ r, const double2* __restrict__ b, int n, int ld,
                                double* __restrict__ out) {
  int col = blockIdx.x;
  double mr = 0.0, mb = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double2 x = r[i + (size_t)col * ld], y = b[i + (size_t)col * ld];
    mr = fmax(mr, fabs(x.x) + fabs(x.y));
    mb = fmax(mb, fabs(y.x) + fabs(y.y));
  }
  __shared__ double s1[256], s2[256];
  s1[threadIdx.x] = mr;
  s2[threadIdx.x] = mb;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      s1[threadIdx.x] = fmax(s1[threadIdx.x], s1[threadIdx.x + s]);
      s2[threadIdx.x] = fmax(s2[threadIdx.x], s2[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) out[col] = s2[0] > 0.0 ? s1[0] / s2[0] : s1[0];
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
constexpr int kBins = 7;

// The device memory of contexts and lanes comes from a process-wide cache
// per device: a buffer a context frees (its stream synchronised) is kept and
// handed to the next allocation of a size it fits (at most twice that size),
// so that contexts created one after another -- a sweep of decks, the
// heterogeneous cases, a context rebuilt for new options -- take neither
// cudaMalloc nor cudaFree (which waits for the whole device) again.  The
// cache holds at most a third of the device's memory; an allocation that
// fails releases the device's cached buffers and tries once more.
namespace devcache {
struct Dev {
  std::multimap<size_t, void*> free;  // bytes -> block
  size_t cached = 0, cap = 0;
};
std::mutex mu;
std::map<int, Dev> devs;

inline size_t round_bytes(size_t b) { return b < (1u << 20) ? (b + 255) / 256 * 256 : (b + (2u << 20) - 1) / (2u << 20) * (2u << 20); }

void* take(size_t bytes) {
  int dev = 0;
  cudaGetDevice(&dev);
  const size_t want = round_bytes(bytes);
  {
    std::lock_guard<std::mutex> lock(mu);
    Dev& d = devs[dev];
    auto it = d.free.lower_bound(want);
    if (it != d.free.end() && it->first <= 2 * want) {
      void* p = it->second;
      d.cached -= it->first;
      d.free.erase(it);
      return p;
    }
  }
  void* p = nullptr;
  if (cudaMalloc(&p, want) == cudaSuccess) return p;
  cudaGetLastError();
  {  // out of memory: give the cached blocks back and try once more
    std::lock_guard<std::mutex> lock(mu);
    Dev& d = devs[dev];
    for (auto& f : d.free) cudaFree(f.second);
    d.free.clear();
    d.cached = 0;
  }
  p = nullptr;
  if (cudaMalloc(&p, want) == cudaSuccess) return p;
  cudaGetLastError();
  return nullptr;
}

// The block p (of `bytes`, as requested from take) back to the cache; the
// caller guarantees that no work in flight still uses it.
void give(void* p, size_t bytes) {
  if (!p) return;
  int dev = 0;
  cudaGetDevice(&dev);
  const size_t have = round_bytes(bytes);
  std::lock_guard<std::mutex> lock(mu);
  Dev& d = devs[dev];
  if (d.cap == 0) {
    size_t fr = 0, tot = 0;
    d.cap = cudaMemGetInfo(&fr, &tot) == cudaSuccess ? tot / 3 : (size_t)8 << 30;
  }
  if (d.cached + have > d.cap) {
    cudaFree(p);
    return;
  }
  d.free.emplace(have, p);
  d.cached += have;
}
}  // namespace devcache

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  bool own = true;  // false: a view of another context's buffer
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  int alloc(size_t count) {
    if (count <= n && p) return 0;
    // the old block may still be in use by queued work: wait, as cudaFree did
    if (p && own) cudaDeviceSynchronize();
    release(true);
    if (count == 0) return 0;
    p = static_cast<T*>(devcache::take(count * sizeof(T)));
    if (!p) return fail(HAMS_ERR_NOMEM, "cudaMalloc of %zu bytes failed", count * sizeof(T));
    n = count;
    return 0;
  }
  void view(const DBuf& o) {
    release(true);
    p = o.p;
    n = o.n;
    own = false;
  }
  // idle: nothing queued uses the buffer any more (the owner's stream is
  // synchronised); otherwise the device is synchronised first
  void release(bool idle = false) {
    if (p && own) {
      if (!idle) cudaDeviceSynchronize();
      devcache::give(p, n * sizeof(T));
    }
    p = nullptr;
    n = 0;
    own = true;
  }
};

// A recorded launch sequence of the block LU (opts.lu_graph): the graph of
// one call of the factorisation or of a solve, valid while the pointers it
// was recorded with stay the same.
struct LuGraph {
  cudaGraphExec_t exec = nullptr;
  const void* key[4] = {};  // the buffers the recording used
  int nrhs = 0;
  long long launches = 0;
};

struct hams_ctx {
  int dev = 0;
  cudaStream_t st = nullptr;
  cublasHandle_t blas = nullptr;
  cusolverDnHandle_t solver = nullptr;
  hams_opts opts{};
  int n = 0, nl = 0, tn = 0, nb = 0;
  std::vector<int> body_nelem;
  std::vector<double> xyz_p;  // hull panel centres (n x 3), host copy for the H-matrix cluster tree
  std::vector<double> vtx_h, pnsz_h, nrm_h;  // host copies for the field points' on-body test
  std::vector<int> ncn_h;
  // field points (hams_ctx_set_field_points): coordinates, 2 pi / 4 pi per
  // point, and the potentials of the last solve (host) or of each frequency
  // of the last batch
  int nfp = 0;
  DBuf<double> fp_x, fp_sld;
  DBuf<double2> fp_S, fp_D, fp_bc, fp_pot, fp_out;
  std::vector<double> fp_last;
  std::vector<std::vector<double>> fp_batch;
  bool hm_ready = false;      // GMRES: cluster tree uploaded to hm
  hmat::Dev hm;
  DBuf<double2> hxp, hyp, hw;  // H-matrix product work arrays
  // geometry
  DBuf<double> xq, fxyz, ds, pnsz, nrm, vtx;
  DBuf<int> ncn, body, bstart;
  DevGeom g{};
  // frequency-independent pair data
  DBuf<double> rs, rd;
  DBuf<uint32_t> pairs;
  // start offsets into pairs of bins 0-3 (branches LINTON, PIDCOCK, EIGENE,
  // EIGEN), 4-5 (surrogate pairs of EIGENE, EIGEN), 6 (pairs of copied body
  // blocks); bin_off[7] = total
  long long bin_off[kBins + 1] = {};
  // identical body blocks (hams_opts.body_blocks): per (field, source) body
  // pair 1 when copied, and the copies (6 ints each, k_copy_blocks)
  DBuf<unsigned char> blk_copied;
  DBuf<int> blk_list;
  int nblk = 0, blk_rows = 0, blk_cols = 0;
  long long blk_pairs = 0;
  // chunks of source panels for the RHS reduction
  std::vector<int2> chunks_h;
  DBuf<int2> chunks;
  DBuf<int> chunk_body;
  // per-frequency buffers
  DBuf<double2> A, S, B, part, wd, C, D, X, R;
  DBuf<float2> Af, Xf, luw;
  DBuf<double2> gv, gw, gz, gy, gpre;  // GMRES: Krylov basis, work, preconditioned, coefficients, body blocks
  DBuf<double> gnrm;
  DBuf<int> gpiv;
  DBuf<int> perm;
  int lu_used = -1;  // mixed form: factorisation used by the last solve (HAMS_LU_*)
  DBuf<double> wvn, beta, outbuf, colratio;
  DBuf<double> mt_pm, mt_ac, mt_fld, mt_fldt;  // per-frequency mode tables (finite depth)
  DBuf<double2> mt_src, mt_srct;
  hams::ModeTab mt{};
  DBuf<int> ipiv, info, ovf;
  DBuf<char> work;
  DBuf<char> work32;
  // timing: ev[0..5] stage marks, evb[0..4] branch marks, evf after the factorisation
  cudaEvent_t ev[6] = {};
  cudaEvent_t evb[6] = {};
  cudaEvent_t evf = nullptr;
  cudaEvent_t evc = nullptr;  // start of the last solve_one
  static constexpr int kTimings = 28;
  double last_ms[kTimings] = {};
  std::atomic<long long> launches{0};   // kernels of this library
  std::atomic<long long> lib_calls{0};  // cuBLAS / cuSOLVER / CUB calls
  cudaEvent_t marks[8] = {};
  int refine_sweeps = 0;
  double ir_rate = 0.0;  // largest residual reduction factor of one refinement sweep
  // batch lanes: contexts that share this one's geometry and pair data (views)
  // and own their stream, handles and per-frequency buffers
  std::vector<hams_ctx*> lanes;
  bool is_lane = false;
  // MLP surrogate of far-field pairs (hams_ctx_set_surrogate)
  int sg_on = 0;
  double sg_far = 3.0;
  double sg_kmin = sg::kKmin, sg_kmax = sg::kKmax;  // frequencies (K = k0 h tanh k0 h) given to the surrogate
  DBuf<uint16_t> sg_wh;
  DBuf<float> sg_w0, sg_bias;
  SgDev sgd{};
  int sms = 148;
  int sg_used = 0;  // the last solve evaluated its far pairs with the surrogate
  // the series' judgement of the surrogate (hams_ctx_set_surrogate_tolerance):
  // sampled far pairs evaluated both ways, the outputs' sensitivity probe
  double sg_tol = 0.0;
  DBuf<uint32_t> sg_samp;  // sampled surrogate pairs: sg_ns4 of bin 4, then sg_ns5 of bin 5
  int sg_ns4 = 0, sg_ns5 = 0;
  DBuf<double2> sg_g1, sg_g2;  // the sampled A and S entries from the network, then from the series
  DBuf<unsigned char> sg_map;  // the judgement's cell of every pair the network evaluates (k_probe_map)
  DBuf<double> sg_scale;       // this frequency's probe scale per cell (k_probe_scales)
  // the block LU's recorded graphs (opts.lu_graph): the factorisation, the solve per right-hand-side count
  LuGraph lu_factor_graph;
  std::map<int, LuGraph> lu_solve_graph;
  // the judgement's probe in the first refinement sweep: pending (requested
  // for this solve), folded (done: dX in jdX), its right-hand sides jB
  bool judge_pending = false, judge_folded = false;
  int judge_nbeta = 0;
  DBuf<double2> jB;
  DBuf<float2> jdX;
  DBuf<double> sg_red, sg_cells, outbuf2;
  double sg_judge[8] = {};  // e_A, e_S, kappa_A, kappa_B, kappa_X, estimate, taken back by the series, samples
  std::string note;  // what the last solve changed on its own (fallbacks), or empty
  bool unfolded = false;  // built from a half mesh (ISX or ISY = 1), see unfold_symmetry
};

static int launch_check(hams_ctx* c, int count = 1) {
  c->launches += count;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(HAMS_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
  return 0;
}

extern "C" int hams_wave_properties(int32_t inft, double value, double depth, double g, int32_t sybo_kk,
                                    hams_wave* o);

extern "C" const char* hams_last_error(void) { return g_err.c_str(); }

// error reporting for the other translation units of the library
int hams_set_error(int code, const char* msg) { return fail(code, "%s", msg); }

static bool handles_to_pool(hams_ctx* c);
static void release_handle_pool();

extern "C" void hams_release_cached(void) {
  int cur = 0;
  cudaGetDevice(&cur);
  {
    std::lock_guard<std::mutex> lock(devcache::mu);
    for (auto& d : devcache::devs) {
      cudaSetDevice(d.first);
      for (auto& f : d.second.free) cudaFree(f.second);
      d.second.free.clear();
      d.second.cached = 0;
    }
  }
  release_handle_pool();
  cudaSetDevice(cur);
}

extern "C" void hams_ctx_destroy(hams_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->dev);
  for (hams_ctx* l : c->lanes) hams_ctx_destroy(l);
  c->lanes.clear();
  if (c->st) cudaStreamSynchronize(c->st);
  if (c->lu_factor_graph.exec) cudaGraphExecDestroy(c->lu_factor_graph.exec);
  for (auto& g : c->lu_solve_graph)
    if (g.second.exec) cudaGraphExecDestroy(g.second.exec);
  // the context's stream is idle: its buffers go back to the cache without a device-wide wait
  auto rel = [](auto&... b) { (b.release(true), ...); };
  rel(c->fp_x, c->fp_sld, c->fp_S, c->fp_D, c->fp_bc, c->fp_pot, c->fp_out, c->hxp, c->hyp, c->hw);
  rel(c->xq, c->fxyz, c->ds, c->pnsz, c->nrm, c->vtx, c->ncn, c->body, c->bstart, c->rs, c->rd, c->pairs);
  rel(c->blk_copied, c->blk_list, c->chunks, c->chunk_body, c->A, c->S, c->B, c->part, c->wd, c->C, c->D, c->X, c->R);
  rel(c->Af, c->Xf, c->luw, c->gv, c->gw, c->gz, c->gy, c->gpre, c->gnrm, c->gpiv, c->perm);
  rel(c->wvn, c->beta, c->outbuf, c->colratio, c->mt_pm, c->mt_ac, c->mt_fld, c->mt_fldt, c->mt_src, c->mt_srct);
  rel(c->ipiv, c->info, c->ovf, c->work, c->work32, c->sg_wh, c->sg_w0, c->sg_bias, c->sg_samp, c->sg_g1, c->sg_g2);
  rel(c->sg_map, c->sg_scale, c->jB, c->jdX, c->sg_red, c->sg_cells, c->outbuf2);
  hmat::free_dev(c->hm);
  if (!handles_to_pool(c)) {
    for (auto& e : c->ev)
      if (e) cudaEventDestroy(e);
    for (auto& e : c->evb)
      if (e) cudaEventDestroy(e);
    for (auto& e : c->marks)
      if (e) cudaEventDestroy(e);
    if (c->evf) cudaEventDestroy(c->evf);
    if (c->evc) cudaEventDestroy(c->evc);
    if (c->solver) cusolverDnDestroy(c->solver);
    if (c->blas) cublasDestroy(c->blas);
    if (c->st) cudaStreamDestroy(c->st);
  }
  delete c;
}

static int ctx_frequency_buffers(hams_ctx* c);

// Sorted pair list and bin offsets (finite depth); rebuilt when the surrogate
// is switched on or off.
static int build_pairs(hams_ctx* c) {
  const int n = c->n, tn = c->tn;
  size_t np = (size_t)tn * n;
  if (np > 0xffffffffull) return fail(HAMS_ERR_UNSUPPORTED, "%zu pairs exceed the 32-bit pair index", np);
  DBuf<uint32_t> keys, keys2, idx;
  TRY(keys.alloc(np)); TRY(keys2.alloc(np)); TRY(idx.alloc(np)); TRY(c->pairs.alloc(np));
  dim3 grid2((tn + 127) / 128, n);
  k_pair_keys<<<grid2, 128, 0, c->st>>>(c->g, c->opts.depth, c->sg_on, c->sg_far, c->nblk ? c->blk_copied.p : nullptr,
                                         keys.p, idx.p);
  TRY(launch_check(c));
  size_t tmp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys.p, keys2.p, idx.p, c->pairs.p, np, 0, 11, c->st);
  DBuf<char> tbuf;
  TRY(tbuf.alloc(tmp));
  CU(cub::DeviceRadixSort::SortPairs(tbuf.p, tmp, keys.p, keys2.p, idx.p, c->pairs.p, np, 0, 11, c->st));
  c->lib_calls += 1;
  // bin boundaries: first index of each bin in the sorted keys, found on the
  // device (a binary search per bin) so that only kBins + 1 numbers come back
  DBuf<long long> offs;
  TRY(offs.alloc(kBins + 1));
  k_bin_offsets<<<1, 32, 0, c->st>>>(keys2.p, (long long)np, kBins, offs.p);
  TRY(launch_check(c));
  CU(cudaMemcpyAsync(c->bin_off, offs.p, (kBins + 1) * sizeof(long long), cudaMemcpyDeviceToHost, c->st));
  CU(cudaStreamSynchronize(c->st));
  return 0;
}

static int ctx_setup(hams_ctx* c, const hams_geom* geo) {
  const int n = c->n, tn = c->tn, nb = c->nb;
  // host staging: source centres, normals, vertices, field points
  std::vector<double> xq(3 * (size_t)n), fx(3 * (size_t)tn), vtx(12 * (size_t)n, 0.0);
  std::vector<int> body(n), bst(nb + 1, 0);
  for (int k = 0; k < 3; ++k)
    for (int i = 0; i < n; ++i) {
      xq[i + (size_t)k * n] = geo->xyz_p[i + (size_t)k * n];
      fx[i + (size_t)k * tn] = geo->xyz_p[i + (size_t)k * n];
    }
  for (int k = 0; k < 3; ++k)
    for (int i = 0; i < c->nl; ++i) fx[n + i + (size_t)k * tn] = geo->ixyz_p[i + (size_t)k * c->nl];
  for (int j = 0; j < n; ++j) {
    int nc = geo->ncn[j];
    if (nc != 3 && nc != 4) return fail(HAMS_ERR_ARG, "panel %d has %d vertices (3 or 4 expected)", j + 1, nc);
    for (int v = 0; v < nc; ++v) {
      int id = geo->ncon[j + (size_t)v * n];
      if (id < 1 || id > geo->ntnd) return fail(HAMS_ERR_ARG, "panel %d vertex %d: node id %d out of range", j + 1, v + 1, id);
      for (int k = 0; k < 3; ++k) vtx[(size_t)j * 12 + v * 3 + k] = geo->xyz[(id - 1) + (size_t)k * geo->ntnd];
    }
  }
  int off = 0;
  for (int b = 0; b < nb; ++b) {
    bst[b] = off;
    for (int i = 0; i < geo->body_nelem[b]; ++i) body[off + i] = b;
    off += geo->body_nelem[b];
  }
  bst[nb] = off;
  if (off != n) return fail(HAMS_ERR_ARG, "body_nelem sums to %d, nelem is %d", off, n);
  TRY(c->xq.alloc(3 * (size_t)n)); TRY(c->fxyz.alloc(3 * (size_t)tn)); TRY(c->ds.alloc(n)); TRY(c->pnsz.alloc(n));
  TRY(c->nrm.alloc(6 * (size_t)n)); TRY(c->vtx.alloc(12 * (size_t)n)); TRY(c->ncn.alloc(n)); TRY(c->body.alloc(n));
  TRY(c->bstart.alloc(nb + 1));
  c->vtx_h = vtx;
  c->ncn_h.assign(geo->ncn, geo->ncn + n);
  c->pnsz_h.assign(geo->pnsz, geo->pnsz + n);
  c->nrm_h.assign(geo->dxyz, geo->dxyz + 6 * (size_t)n);
  CU(cudaMemcpyAsync(c->xq.p, xq.data(), 3 * (size_t)n * 8, cudaMemcpyHostToDevice, c->st));
  CU(cudaMemcpyAsync(c->fxyz.p, fx.data(), 3 * (size_t)tn * 8, cudaMemcpyHostToDevice, c->st));
  CU(cudaMemcpyAsync(c->ds.p, geo->ds, (size_t)n * 8, cudaMemcpyHostToDevice, c->st));
  CU(cudaMemcpyAsync(c->pnsz.p, geo->pnsz, (size_t)n * 8, cudaMemcpyHostToDevice, c->st));
  CU(cudaMemcpyAsync(c->nrm.p, geo->dxyz, 6 * (size_t)n * 8, cudaMemcpyHostToDevice, c->st));
  CU(cudaMemcpyAsync(c->vtx.p, vtx.data(), 12 * (size_t)n * 8, cudaMemcpyHostToDevice, c->st));
  CU(cudaMemcpyAsync(c->ncn.p, geo->ncn, (size_t)n * 4, cudaMemcpyHostToDevice, c->st));
  CU(cudaMemcpyAsync(c->body.p, body.data(), (size_t)n * 4, cudaMemcpyHostToDevice, c->st));
  CU(cudaMemcpyAsync(c->bstart.p, bst.data(), (size_t)(nb + 1) * 4, cudaMemcpyHostToDevice, c->st));
  c->g = DevGeom{n, tn, nb, c->xq.p, c->fxyz.p, c->ds.p, c->pnsz.p, c->nrm.p, c->vtx.p, c->ncn.p, c->body.p, c->bstart.p};

  // Rankine tables
  size_t np = (size_t)tn * n;
  TRY(c->rs.alloc(np));
  TRY(c->rd.alloc(np));
  dim3 grid2((tn + 127) / 128, n);
  k_rankine<<<grid2, 128, 0, c->st>>>(c->g, c->rs.p, c->rd.p);
  TRY(launch_check(c));

  // identical body blocks: which (field, source) body blocks are copies
  c->nblk = 0;
  c->blk_pairs = 0;
  if (c->opts.body_blocks && nb > 1 && c->nl == 0) {
    std::vector<int32_t> rep((size_t)nb * nb);
    if (hams_body_blocks(geo, 1e-9, rep.data()) < 0) return fail(HAMS_ERR_ARG, "body blocks: bad geometry");
    std::vector<unsigned char> copied((size_t)nb * nb, 0);
    std::vector<int> lst;
    for (int k = 0; k < nb * nb; ++k) {
      if (rep[k] == k) continue;
      const int b1 = k % nb, b2 = k / nb, c1 = rep[k] % nb, c2 = rep[k] / nb;
      copied[k] = 1;
      const int ni = bst[b1 + 1] - bst[b1], nj = bst[b2 + 1] - bst[b2];
      lst.insert(lst.end(), {bst[b1], bst[b2], bst[c1], bst[c2], ni, nj});
      c->blk_rows = std::max(c->blk_rows, ni);
      c->blk_cols = std::max(c->blk_cols, nj);
      c->blk_pairs += (long long)ni * nj;
      ++c->nblk;
    }
    if (c->nblk > 65535) {  // one grid z index per copy: keep every block instead
      c->nblk = 0;
      c->blk_pairs = 0;
    }
    if (c->nblk) {
      TRY(c->blk_copied.alloc(copied.size()));
      TRY(c->blk_list.alloc(lst.size()));
      CU(cudaMemcpyAsync(c->blk_copied.p, copied.data(), copied.size(), cudaMemcpyHostToDevice, c->st));
      CU(cudaMemcpyAsync(c->blk_list.p, lst.data(), lst.size() * 4, cudaMemcpyHostToDevice, c->st));
      CU(cudaStreamSynchronize(c->st));
    }
  }

  // branch-sorted pair list (finite depth)
  if (c->opts.depth >= 0.0) TRY(build_pairs(c));

  // chunks of source panels for the RHS reduction
  c->chunks_h.clear();
  std::vector<int> cb;
  for (int b = 0; b < nb; ++b)
    for (int j = bst[b]; j < bst[b + 1]; j += kChunk) {
      c->chunks_h.push_back(make_int2(j, std::min(j + kChunk, bst[b + 1])));
      cb.push_back(b);
    }
  TRY(c->chunks.alloc(c->chunks_h.size()));
  TRY(c->chunk_body.alloc(cb.size()));
  CU(cudaMemcpyAsync(c->chunks.p, c->chunks_h.data(), c->chunks_h.size() * sizeof(int2), cudaMemcpyHostToDevice, c->st));
  CU(cudaMemcpyAsync(c->chunk_body.p, cb.data(), cb.size() * sizeof(int), cudaMemcpyHostToDevice, c->st));

  TRY(ctx_frequency_buffers(c));
  CU(cudaStreamSynchronize(c->st));
  return 0;
}

// Buffers of one frequency in flight: mode tables, A and S, roots, flags.
static int ctx_frequency_buffers(hams_ctx* c) {
  const int n = c->n, tn = c->tn;
  size_t np = (size_t)tn * n;
  if (c->opts.depth >= 0.0) {
    const size_t km = hams::kModeMax;
    TRY(c->mt_pm.alloc(km)); TRY(c->mt_ac.alloc(km));
    TRY(c->mt_src.alloc(km * n)); TRY(c->mt_srct.alloc(km * n));
    TRY(c->mt_fld.alloc(km * tn)); TRY(c->mt_fldt.alloc(km * tn));
    // modes needed by the longest series present: PIDCOCK 99, EIGENE 50, EIGEN 10
    int nmode = 11;
    if (c->bin_off[3] > c->bin_off[2] || c->bin_off[5] > c->bin_off[4]) nmode = hams::kEigenEMax + 1;
    if (c->bin_off[2] > c->bin_off[1]) nmode = hams::kPidcockMax + 1;
    c->mt = hams::ModeTab{n, tn, nmode, c->mt_pm.p, c->mt_ac.p, c->mt_src.p, c->mt_srct.p, c->mt_fld.p, c->mt_fldt.p};
  }
  TRY(c->A.alloc(np));
  TRY(c->S.alloc(np));
  TRY(c->wvn.alloc(HAMS_NK));
  TRY(c->ovf.alloc(1));
  TRY(c->ipiv.alloc(n));
  TRY(c->info.alloc(2));  // the solver's info word and the tensor-core kernels' error word
  return 0;
}

// Streams, library handles and events of destroyed contexts and lanes, per
// device, for the next ones (cuBLAS and cuSOLVER handles are slow to create;
// the library leaves their settings at the defaults except the stream, which
// stays bound to the handle's own stream).
struct HandleSet {
  cudaStream_t st;
  cublasHandle_t blas;
  cusolverDnHandle_t solver;
  cudaEvent_t ev[6], evb[6], marks[8], evf, evc;
};
static std::mutex g_hpool_mu;
static std::map<int, std::vector<HandleSet>> g_hpool;
constexpr size_t kHandlePoolMax = 32;  // per device

static bool handles_from_pool(hams_ctx* c) {
  std::lock_guard<std::mutex> lock(g_hpool_mu);
  auto& v = g_hpool[c->dev];
  if (v.empty()) return false;
  const HandleSet h = v.back();
  v.pop_back();
  c->st = h.st;
  c->blas = h.blas;
  c->solver = h.solver;
  for (int k = 0; k < 6; ++k) c->ev[k] = h.ev[k], c->evb[k] = h.evb[k];
  for (int k = 0; k < 8; ++k) c->marks[k] = h.marks[k];
  c->evf = h.evf;
  c->evc = h.evc;
  return true;
}

// The handles of c (its stream synchronised) back to the pool; false if the
// pool is full (the caller destroys them).
static bool handles_to_pool(hams_ctx* c) {
  if (!c->st || !c->blas || !c->solver || !c->evf || !c->evc) return false;
  for (int k = 0; k < 6; ++k)
    if (!c->ev[k] || !c->evb[k]) return false;
  for (int k = 0; k < 8; ++k)
    if (!c->marks[k]) return false;
  std::lock_guard<std::mutex> lock(g_hpool_mu);
  auto& v = g_hpool[c->dev];
  if (v.size() >= kHandlePoolMax) return false;
  HandleSet h;
  h.st = c->st;
  h.blas = c->blas;
  h.solver = c->solver;
  for (int k = 0; k < 6; ++k) h.ev[k] = c->ev[k], h.evb[k] = c->evb[k];
  for (int k = 0; k < 8; ++k) h.marks[k] = c->marks[k];
  h.evf = c->evf;
  h.evc = c->evc;
  v.push_back(h);
  return true;
}

static void release_handle_pool() {
  std::lock_guard<std::mutex> lock(g_hpool_mu);
  for (auto& d : g_hpool) {
    cudaSetDevice(d.first);
    for (auto& h : d.second) {
      for (auto e : h.ev) cudaEventDestroy(e);
      for (auto e : h.evb) cudaEventDestroy(e);
      for (auto e : h.marks) cudaEventDestroy(e);
      cudaEventDestroy(h.evf);
      cudaEventDestroy(h.evc);
      cusolverDnDestroy(h.solver);
      cublasDestroy(h.blas);
      cudaStreamDestroy(h.st);
    }
    d.second.clear();
  }
}

// Stream, library handles and events of a context, on its device.
static int ctx_handles(hams_ctx* c) {
  if (cudaSetDevice(c->dev) != cudaSuccess) return fail(HAMS_ERR_CUDA, "cudaSetDevice(%d) failed", c->dev);
  if (handles_from_pool(c)) {
    cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->dev);
    return 0;
  }
  if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess)
    return fail(HAMS_ERR_CUDA, "stream creation failed");
  if (cublasCreate(&c->blas) != CUBLAS_STATUS_SUCCESS) return fail(HAMS_ERR_CUDA, "cublasCreate failed");
  if (cusolverDnCreate(&c->solver) != CUSOLVER_STATUS_SUCCESS) return fail(HAMS_ERR_CUDA, "cusolverDnCreate failed");
  cublasSetStream(c->blas, c->st);
  cusolverDnSetStream(c->solver, c->st);
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->dev);
  for (auto& e : c->ev) CU(cudaEventCreate(&e));
  for (auto& e : c->evb) CU(cudaEventCreate(&e));
  for (auto& e : c->marks) CU(cudaEventCreate(&e));
  CU(cudaEventCreate(&c->evf));
  CU(cudaEventCreate(&c->evc));
  return 0;
}

// A batch lane of c: its own stream, handles and per-frequency buffers; the
// geometry, Rankine terms and pair lists are views of c's.
static int make_lane(hams_ctx* c, hams_ctx** out) {
  hams_ctx* l = new hams_ctx();
  l->is_lane = true;
  l->opts = c->opts;
  l->dev = c->dev;
  l->n = c->n;
  l->nl = c->nl;
  l->tn = c->tn;
  l->nb = c->nb;
  l->body_nelem = c->body_nelem;
  l->xyz_p = c->xyz_p;
  l->nfp = c->nfp;
  if (c->nfp > 0) {
    l->fp_x.view(c->fp_x);
    l->fp_sld.view(c->fp_sld);
  }
  int rc = ctx_handles(l);
  if (!rc) {
    l->xq.view(c->xq); l->fxyz.view(c->fxyz); l->ds.view(c->ds); l->pnsz.view(c->pnsz); l->nrm.view(c->nrm);
    l->vtx.view(c->vtx); l->ncn.view(c->ncn); l->body.view(c->body); l->bstart.view(c->bstart);
    l->rs.view(c->rs); l->rd.view(c->rd); l->pairs.view(c->pairs); l->chunks.view(c->chunks);
    l->chunk_body.view(c->chunk_body);
    l->blk_copied.view(c->blk_copied); l->blk_list.view(c->blk_list);
    l->nblk = c->nblk; l->blk_rows = c->blk_rows; l->blk_cols = c->blk_cols; l->blk_pairs = c->blk_pairs;
    l->g = c->g;
    for (int b = 0; b <= kBins; ++b) l->bin_off[b] = c->bin_off[b];
    l->sg_on = c->sg_on;
    l->sg_far = c->sg_far;
    l->sg_kmin = c->sg_kmin;
    l->sg_kmax = c->sg_kmax;
    l->sgd = c->sgd;
    l->sg_tol = c->sg_tol;
    l->sg_samp.view(c->sg_samp);
    l->sg_map.view(c->sg_map);
    l->sg_ns4 = c->sg_ns4;
    l->sg_ns5 = c->sg_ns5;
    l->sms = c->sms;
    l->chunks_h = c->chunks_h;
    rc = ctx_frequency_buffers(l);
  }
  if (rc < 0) {
    std::string keep = g_err;
    hams_ctx_destroy(l);
    g_err = keep;
    return rc;
  }
  *out = l;
  return 0;
}

// Geometric symmetry (ISX = 1: the mesh holds the half x >= 0 of every body,
// mirrored in the plane x = 0; ISY = 1: the half y >= 0, mirrored in y = 0).
// The reference solves the symmetric and antisymmetric systems of the half
// mesh (NSYS = 2: field points imaged with the SX/SY signs, A, B and D
// combined with RXY, HAMS_Prog.f90 and CalGreenFuncMulti.f90).  Both
// systems together are the full body's system in another basis, so here the
// half mesh is unfolded into the full one: each body's panels followed by
// their mirror images (nodes appended after the originals, vertex order
// reversed so the normals stay outward), the mirrored centres, areas and
// sizes, n' = M n and (r x n)' = -M (r x n) for the mirror M, which holds
// for reference points on the symmetry plane (the plane the reference's
// sign tables assume).  Water-plane panel centres are mirrored the same way
// and appended.  The forces are then those of the full bodies, as the
// reference reports them.
struct Unfolded {
  std::vector<double> xyz, xyz_p, ds, pnsz, dxyz, ixyz_p;
  std::vector<int32_t> ncn, ncon, body_nelem;
  hams_geom g{};
};

static void unfold_symmetry(const hams_geom* geo, Unfolded& u) {
  const int n = geo->nelem, nt = geo->ntnd, nb = geo->nbody, n2 = 2 * n, nt2 = 2 * nt;
  const int ax = geo->isx ? 0 : 1;  // the coordinate the mirror negates
  u.xyz.resize((size_t)3 * nt2);
  for (int k = 0; k < 3; ++k)
    for (int i = 0; i < nt; ++i) {
      const double v = geo->xyz[i + (size_t)k * nt];
      u.xyz[i + (size_t)k * nt2] = v;
      u.xyz[nt + i + (size_t)k * nt2] = k == ax ? -v : v;
    }
  u.ncn.resize(n2);
  u.ncon.assign((size_t)4 * n2, 0);
  u.xyz_p.resize((size_t)3 * n2);
  u.ds.resize(n2);
  u.pnsz.resize(n2);
  u.dxyz.resize((size_t)6 * n2);
  u.body_nelem.resize(nb);
  // sign of each dxyz column under the mirror: n' = M n, (r x n)' = -M (r x n)
  double sgn[6];
  for (int k = 0; k < 3; ++k) {
    sgn[k] = k == ax ? -1.0 : 1.0;
    sgn[3 + k] = k == ax ? 1.0 : -1.0;
  }
  int src = 0, dst = 0;
  for (int b = 0; b < nb; ++b) {
    const int m = geo->body_nelem[b];
    for (int half = 0; half < 2; ++half)
      for (int q = 0; q < m; ++q, ++dst) {
        const int i = src + q, nc = geo->ncn[i];
        u.ncn[dst] = nc;
        for (int v = 0; v < nc; ++v) {
          // mirrored panels: vertices 0, nc-1, ..., 1 of the mirrored nodes
          const int sv = half == 0 ? v : (v == 0 ? 0 : nc - v);
          const int id = geo->ncon[i + (size_t)sv * n];
          u.ncon[dst + (size_t)v * n2] = half == 0 ? id : id + nt;
        }
        for (int k = 0; k < 3; ++k) {
          const double v = geo->xyz_p[i + (size_t)k * n];
          u.xyz_p[dst + (size_t)k * n2] = half == 1 && k == ax ? -v : v;
        }
        u.ds[dst] = geo->ds[i];
        u.pnsz[dst] = geo->pnsz[i];
        for (int k = 0; k < 6; ++k) u.dxyz[dst + (size_t)k * n2] = (half == 1 ? sgn[k] : 1.0) * geo->dxyz[i + (size_t)k * n];
      }
    u.body_nelem[b] = 2 * m;
    src += m;
  }
  u.g = *geo;
  u.g.isx = u.g.isy = 0;
  u.g.nelem = n2;
  u.g.ntnd = nt2;
  u.g.xyz = u.xyz.data();
  u.g.ncn = u.ncn.data();
  u.g.ncon = u.ncon.data();
  u.g.xyz_p = u.xyz_p.data();
  u.g.ds = u.ds.data();
  u.g.pnsz = u.pnsz.data();
  u.g.dxyz = u.dxyz.data();
  u.g.body_nelem = u.body_nelem.data();
  if (geo->inelem > 0 && geo->ixyz_p) {
    const int nl = geo->inelem, nl2 = 2 * nl;
    u.ixyz_p.resize((size_t)3 * nl2);
    for (int k = 0; k < 3; ++k)
      for (int i = 0; i < nl; ++i) {
        const double v = geo->ixyz_p[i + (size_t)k * nl];
        u.ixyz_p[i + (size_t)k * nl2] = v;
        u.ixyz_p[nl + i + (size_t)k * nl2] = k == ax ? -v : v;
      }
    u.g.inelem = nl2;
    u.g.ixyz_p = u.ixyz_p.data();
  }
}

extern "C" int hams_ctx_create(const hams_geom* geo, const hams_opts* opts, hams_ctx** out) {
  g_err.clear();
  if (!geo || !opts || !out) return fail(HAMS_ERR_ARG, "null argument");
  *out = nullptr;
  if (geo->nelem <= 0 || geo->nbody <= 0 || !geo->xyz || !geo->ncn || !geo->ncon || !geo->xyz_p || !geo->ds ||
      !geo->pnsz || !geo->dxyz || !geo->body_nelem)
    return fail(HAMS_ERR_ARG, "incomplete geometry");
  if (geo->isx < 0 || geo->isx > 1 || geo->isy < 0 || geo->isy > 1)
    return fail(HAMS_ERR_ARG, "ISX/ISY must be 0 or 1");
  if (geo->isx && geo->isy) return fail(HAMS_ERR_UNSUPPORTED, "ISX = ISY = 1 (two symmetry planes) is not supported");
  Unfolded unf;
  if (geo->isx || geo->isy) {
    for (int i = 0; i < geo->nelem; ++i)
      if (geo->ncn[i] != 3 && geo->ncn[i] != 4)
        return fail(HAMS_ERR_ARG, "panel %d has %d vertices (3 or 4 expected)", i + 1, geo->ncn[i]);
    if (2.0 * geo->nelem * 2.0 * geo->nelem > 4294967295.0) return fail(HAMS_ERR_UNSUPPORTED, "unfolded mesh too large");
    unfold_symmetry(geo, unf);
    geo = &unf.g;
  }
  if (opts->irsp == 1 && (geo->inelem <= 0 || !geo->ixyz_p)) return fail(HAMS_ERR_ARG, "irsp=1 needs water-plane panels");
  if (opts->precision != HAMS_PREC_FP64 && opts->precision != HAMS_PREC_MIXED)
    return fail(HAMS_ERR_ARG, "unknown precision %d", opts->precision);
  if (opts->solver < 0 || opts->solver > HAMS_SOLVER_GMRES) return fail(HAMS_ERR_ARG, "unknown solver %d", opts->solver);
  hams_ctx* c = new hams_ctx();
  c->unfolded = geo == &unf.g;
  c->opts = *opts;
  c->dev = opts->device;
  c->n = geo->nelem;
  c->nl = opts->irsp == 1 ? geo->inelem : 0;
  c->tn = c->n + c->nl;
  c->nb = geo->nbody;
  c->body_nelem.assign(geo->body_nelem, geo->body_nelem + geo->nbody);
  c->xyz_p.assign(geo->xyz_p, geo->xyz_p + (size_t)3 * geo->nelem);
  int rc = ctx_handles(c);
  if (!rc) rc = ctx_setup(c, geo);
  if (!rc && c->opts.precision == HAMS_PREC_MIXED && c->opts.solver != HAMS_SOLVER_GMRES &&
      c->opts.lu_kind == HAMS_LU_BLOCK_TF32) {
    // tile variants of the block LU's GEMMs for this order (classes measured
    // once per device and process)
    std::vector<int> shapes;
    mixed_lu_gemm_shapes(c->n, shapes);
    if (gemm_tf32_autotune(c->st, (int)shapes.size() / 3, shapes.data()))
      rc = fail(HAMS_ERR_CUDA, "GEMM autotuner failed: %s", cudaGetErrorString(cudaGetLastError()));
  }
  if (rc < 0) {
    std::string keep = g_err;
    hams_ctx_destroy(c);
    g_err = keep;
    return rc;
  }
  *out = c;
  return 0;
}

static WaveDev wave_dev(const hams_ctx* c, const hams_wave* w) {
  WaveDev d;
  d.v = w->v;
  d.wk = w->wk;
  d.w1 = w->w1;
  d.h = c->opts.depth;
  d.limit = 0;
  if (fabs(w->v) < HAMS_F4(1.E-8)) d.limit = 1;
  else if (fabs(w->v + 1.0) < HAMS_F4(1.E-8)) d.limit = 2;
  return d;
}

// Assemble A (tn x n) and the right-hand sides B (tn x (6nb+nbeta)) on the
// device; force_series keeps the series for the far pairs of a surrogate
// context (the re-solve of a frequency the series judged).
// The far pairs (bins 4 and 5 of k_pair_keys) from the series: EIGENE and
// EIGEN, as their own bins would (FinGreen3D.f90:413-660).
static int far_series(hams_ctx* c, const WaveDev& wd) {
  const long long ce = c->bin_off[5] - c->bin_off[4], cg = c->bin_off[6] - c->bin_off[5];
  if (ce > 0)
    launch_green_series(hams::kEigenE, (unsigned)((ce + 127) / 128), c->st, c->g, wd, c->wvn.p, c->mt,
                        c->pairs.p + c->bin_off[4], ce, c->rs.p, c->rd.p, c->A.p, c->S.p, c->ovf.p);
  if (cg > 0)
    k_green_fin<3><<<(unsigned)((cg + 127) / 128), 128, 0, c->st>>>(c->g, wd, c->wvn.p, c->mt,
                                                                    c->pairs.p + c->bin_off[5], cg, c->rs.p, c->rd.p,
                                                                    c->A.p, c->S.p, c->ovf.p);
  return launch_check(c, (ce > 0) + (cg > 0));
}

// The copies of the identical body blocks, then the right-hand sides B from S
// and this frequency's diffraction weights (already in wd).
static int copy_blocks_and_rhs(hams_ctx* c, int nbeta) {
  const int tn = c->tn, nb = c->nb;
  if (c->nblk) {
    dim3 grid((unsigned)std::min((c->blk_rows + 255) / 256, 4), (unsigned)std::min(c->blk_cols, 1024),
              (unsigned)c->nblk);
    k_copy_blocks<<<grid, 256, 0, c->st>>>(c->blk_list.p, c->tn, c->A.p, c->S.p);
    TRY(launch_check(c));
  }
  const int nch = (int)c->chunks_h.size();
  k_rhs_partial<false><<<dim3((tn + 127) / 128, nch), 128, 0, c->st>>>(c->g, c->S.p, c->chunks.p, c->wd.p, nbeta, c->part.p);
  k_rhs_final<<<(tn + 127) / 128, 128, 0, c->st>>>(tn, nb, nch, c->chunk_body.p, c->part.p, nbeta, c->B.p);
  return launch_check(c, 2);
}

static int assemble_dev(hams_ctx* c, const hams_wave* w, int nbeta, bool force_series = false) {
  const int n = c->n, tn = c->tn, nb = c->nb, nrhs = 6 * nb + nbeta;
  WaveDev wd = wave_dev(c, w);
  if (c->opts.depth >= 0.0 && !wd.limit) CU(cudaMemcpyAsync(c->wvn.p, w->wvn, HAMS_NK * 8, cudaMemcpyHostToDevice, c->st));
  CU(cudaMemsetAsync(c->ovf.p, 0, sizeof(int), c->st));
  CU(cudaEventRecord(c->ev[0], c->st));
  if (c->opts.depth < 0.0) {
    dim3 grid((tn + 127) / 128, n);
    k_green_inf<<<grid, 128, 0, c->st>>>(c->g, wd, c->nblk ? c->blk_copied.p : nullptr, c->rs.p, c->rd.p, c->A.p,
                                         c->S.p);
    TRY(launch_check(c));
  } else {
    if (!wd.limit) {
      launch_mode_tables(c->st, c->g, wd, c->wvn.p, c->mt.nmode, c->mt_pm.p, c->mt_ac.p, c->mt_src.p, c->mt_srct.p,
                         c->mt_fld.p, c->mt_fldt.p);
      TRY(launch_check(c));
    }
    for (int br = 0; br < 4; ++br) {
      long long cnt = c->bin_off[br + 1] - c->bin_off[br];
      CU(cudaEventRecord(c->evb[br], c->st));
      if (cnt <= 0) continue;
      const uint32_t* lst = c->pairs.p + c->bin_off[br];
      unsigned blocks = (unsigned)((cnt + 127) / 128);
      switch (br) {
        case 0:
          // few pairs (body blocks): a warp per pair for latency; many: a thread per pair, whose
          // one wave over the GPU costs less than the warps' redundant lanes
          if (cnt < (long long)c->sms * kLintonWarpPairsPerSm)
            k_green_linton<<<(unsigned)((cnt + kLintonWarps - 1) / kLintonWarps), 32 * kLintonWarps, 0, c->st>>>(
                c->g, wd, c->wvn.p, lst, cnt, c->rs.p, c->rd.p, c->A.p, c->S.p, c->ovf.p);
          else
            k_green_fin<0><<<blocks, 128, 0, c->st>>>(c->g, wd, c->wvn.p, c->mt, lst, cnt, c->rs.p, c->rd.p, c->A.p,
                                                      c->S.p, c->ovf.p);
          break;
        case 1:
        case 2: launch_green_series(br, blocks, c->st, c->g, wd, c->wvn.p, c->mt, lst, cnt, c->rs.p, c->rd.p, c->A.p, c->S.p, c->ovf.p); break;
        default: k_green_fin<3><<<blocks, 128, 0, c->st>>>(c->g, wd, c->wvn.p, c->mt, lst, cnt, c->rs.p, c->rd.p, c->A.p, c->S.p, c->ovf.p); break;
      }
      TRY(launch_check(c));
    }
    CU(cudaEventRecord(c->evb[4], c->st));
    // far pairs: the surrogate, or the series when this frequency is outside its domain
    const long long cs = c->bin_off[6] - c->bin_off[4];
    const double hh = c->opts.depth, K = wd.wk * hh * tanh(wd.wk * hh);
    if (cs > 0) {
      if (!force_series && !wd.limit && K >= c->sg_kmin && K <= c->sg_kmax) {
        if (launch_green_sg(c->st, c->sms, c->g, wd, c->sgd, c->mt, K, c->pairs.p + c->bin_off[4], cs, c->rs.p,
                            c->rd.p, c->A.p, c->S.p, c->ovf.p))
          return fail(HAMS_ERR_CUDA, "surrogate kernel launch failed");
        c->launches += 1;
        c->sg_used = 1;
        const int ns = c->sg_ns4 + c->sg_ns5;
        if (c->sg_tol > 0.0 && ns > 0) {
          // the sampled far pairs: the network's entries, then the series' over them (the entries of A
          // and S at the samples end up from the series)
          TRY(c->sg_g1.alloc(2 * (size_t)ns));
          TRY(c->sg_g2.alloc(2 * (size_t)ns));
          TRY(c->sg_red.alloc(4));
          const unsigned gb = (unsigned)((ns + 255) / 256);
          k_gather_pairs<<<gb, 256, 0, c->st>>>(c->sg_samp.p, ns, c->A.p, c->S.p, c->sg_g1.p);
          TRY(launch_check(c));
          if (c->sg_ns4 > 0)
            launch_green_series(hams::kEigenE, (unsigned)((c->sg_ns4 + 127) / 128), c->st, c->g, wd, c->wvn.p, c->mt,
                                c->sg_samp.p, c->sg_ns4, c->rs.p, c->rd.p, c->A.p, c->S.p, c->ovf.p);
          if (c->sg_ns5 > 0)
            k_green_fin<3><<<(unsigned)((c->sg_ns5 + 127) / 128), 128, 0, c->st>>>(
                c->g, wd, c->wvn.p, c->mt, c->sg_samp.p + c->sg_ns4, c->sg_ns5, c->rs.p, c->rd.p, c->A.p, c->S.p,
                c->ovf.p);
          TRY(launch_check(c, (c->sg_ns4 > 0) + (c->sg_ns5 > 0)));
          k_gather_pairs<<<gb, 256, 0, c->st>>>(c->sg_samp.p, ns, c->A.p, c->S.p, c->sg_g2.p);
          k_sample_err<<<1, 1024, 0, c->st>>>(c->sg_g1.p, c->sg_g2.p, ns, c->sg_red.p);
          TRY(c->sg_cells.alloc(4 * kJCells));
          CU(cudaMemsetAsync(c->sg_cells.p, 0, 4 * kJCells * sizeof(double), c->st));
          k_judge_fit<<<gb, 256, 0, c->st>>>(c->g, hh, c->sg_samp.p, ns, c->sg_g1.p, c->sg_g2.p, c->sg_cells.p);
          TRY(launch_check(c, 3));
        }
      } else {
        TRY(far_series(c, wd));
        c->sg_used = 0;
      }
    }
    CU(cudaEventRecord(c->evb[5], c->st));
  }
  if (c->nblk) {
    dim3 grid((unsigned)std::min((c->blk_rows + 255) / 256, 4), (unsigned)std::min(c->blk_cols, 1024),
              (unsigned)c->nblk);
    k_copy_blocks<<<grid, 256, 0, c->st>>>(c->blk_list.p, c->tn, c->A.p, c->S.p);
    TRY(launch_check(c));
  }
  CU(cudaEventRecord(c->ev[1], c->st));
  // right-hand sides
  int nch = (int)c->chunks_h.size();
  TRY(c->wd.alloc((size_t)n * std::max(nbeta, 1)));
  TRY(c->part.alloc((size_t)nch * tn * (6 + nbeta)));
  TRY(c->B.alloc((size_t)tn * nrhs));
  if (nbeta > 0) {
    IncWave q = inc_params(wd, c->opts.amp, c->opts.g, c->opts.xw[0], c->opts.xw[1]);
    k_dbc_weights<<<dim3((n + 127) / 128, nbeta), 128, 0, c->st>>>(c->g, wd, q, c->beta.p, nbeta, c->wd.p);
    TRY(launch_check(c));
  }
  k_rhs_partial<false><<<dim3((tn + 127) / 128, nch), 128, 0, c->st>>>(c->g, c->S.p, c->chunks.p, c->wd.p, nbeta, c->part.p);
  TRY(launch_check(c));
  k_rhs_final<<<(tn + 127) / 128, 128, 0, c->st>>>(tn, nb, nch, c->chunk_body.p, c->part.p, nbeta, c->B.p);
  TRY(launch_check(c));
  CU(cudaEventRecord(c->ev[2], c->st));
  return 0;
}

// Xf (n x nrhs) <- (L U)^-1 Xf with the factors the last mixed solve left in Af.
// Runs body (the launches of one factorisation or solve on c->st) as a CUDA
// graph: recorded on first use (or when the buffers moved), replayed after.
// A recording the runtime refuses turns the option off for the context and
// runs body directly.
template <class F>
static int lu_graph_run(hams_ctx* c, LuGraph& gr, const void* k0, const void* k1, const void* k2, const void* k3,
                        int nrhs, long long* launches, F&& body) {
  const void* key[4] = {k0, k1, k2, k3};
  bool same = gr.exec && gr.nrhs == nrhs;
  for (int q = 0; q < 4 && same; ++q) same = gr.key[q] == key[q];
  if (!same) {
    if (gr.exec) cudaGraphExecDestroy(gr.exec);
    gr.exec = nullptr;
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGetLastError();
      c->opts.lu_graph = 0;
      return body(launches);
    }
    long long la = 0;
    const int rc = body(&la);
    const cudaError_t e = cudaStreamEndCapture(c->st, &g);
    if (rc || e != cudaSuccess || !g || cudaGraphInstantiate(&gr.exec, g, 0) != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      gr.exec = nullptr;
      c->opts.lu_graph = 0;  // run directly from now on
      c->note += (c->note.empty() ? "" : "; ") + std::string("block LU graph not recorded: launched directly");
      g_err.clear();
      return body(launches);
    }
    cudaGraphDestroy(g);
    for (int q = 0; q < 4; ++q) gr.key[q] = key[q];
    gr.nrhs = nrhs;
    gr.launches = la;
  }
  if (cudaGraphLaunch(gr.exec, c->st) != cudaSuccess) return fail(HAMS_ERR_CUDA, "block LU graph launch failed");
  *launches += gr.launches;
  return 0;
}

static int mixed_apply(hams_ctx* c, int nrhs) {
  const int n = c->n, lda = mixed_lu_ld(n);
  if (c->lu_used == HAMS_LU_LIBRARY) {
    CUS(cusolverDnCgetrs(c->solver, CUBLAS_OP_N, n, nrhs, (cuComplex*)c->Af.p, lda, c->ipiv.p, (cuComplex*)c->Xf.p, n,
                         c->info.p));
    c->lib_calls += 1;
    return 0;
  }
  long long la = 0, lb = 0;
  const bool own = c->lu_used == HAMS_LU_BLOCK_TF32;
  auto body = [&](long long* l) {
    return mixed_lu_solve(c->st, c->blas, own, CUBLAS_COMPUTE_32F_EMULATED_16BFX9, n, lda, nrhs, c->Af.p, c->perm.p,
                          c->Xf.p, c->luw.p, c->info.p + 1, l, &lb);
  };
  int rc;
  if (own && c->opts.lu_graph == 1) {
    LuGraph& gr = c->lu_solve_graph[nrhs];
    rc = lu_graph_run(c, gr, c->Af.p, c->perm.p, c->Xf.p, c->luw.p, nrhs, &la, body);
  } else {
    rc = body(&la);
  }
  c->launches += la;
  c->lib_calls += lb;
  if (rc) return fail(HAMS_ERR_CUDA, "block LU solve failed (%d)", rc);
  return 0;
}

// The surrogate judgement's probe right-hand sides at the solution X:
// out (n x nrhs) = dB - dA X, xs a complex64 scratch of n x nrhs.
static int judge_rhs(hams_ctx* c, int nbeta, const double2* X, double2* out, float2* xs);

// FP64 iterative refinement of X (n x nrhs) for M X = rhs (ld ldr = n) with
// the complex64 factors in Af: R = rhs - M X, X += (L U)^-1 R until the
// residual of every column is below refine_tol of that column's scale.  X
// may come from another matrix close to M (the correction then carries the
// difference as well).  Returns HAMS_ERR_NUMERIC when the refinement stalls.
static int mixed_refine(hams_ctx* c, const double2* M, const double2* rhs, int ldr, int nrhs) {
  const int n = c->n;
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), mone = make_cuDoubleComplex(-1.0, 0.0);
  const size_t nx = (size_t)n * nrhs;
  const bool block = c->lu_used != HAMS_LU_LIBRARY;
  const double tol = c->opts.refine_tol > 0.0 ? c->opts.refine_tol : 1e-12;
  const int maxit = c->opts.refine_max > 0 ? c->opts.refine_max : 30;
  std::vector<double> ratio(nrhs);
  double prev = 1e300;
  c->refine_sweeps = 0;
  c->ir_rate = 0.0;
  for (int it = 0;; ++it) {
    // R = rhs - M_fp64 X   (M still holds the FP64 matrix)
    CU(cudaMemcpy2DAsync(c->R.p, (size_t)n * 16, rhs, (size_t)ldr * 16, (size_t)n * 16, nrhs, cudaMemcpyDeviceToDevice, c->st));
    CUB_(cublasZgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, n, nrhs, n, &mone, (const cuDoubleComplex*)M, n,
                     (cuDoubleComplex*)c->X.p, n, &one, (cuDoubleComplex*)c->R.p, n));
    c->lib_calls += 1;
    k_colnorm_ratio<<<nrhs, 256, 0, c->st>>>(c->R.p, rhs, n, n, c->colratio.p);  // ldr == n here
    TRY(launch_check(c));
    // the relative residual is checked against the rhs column scale
    CU(cudaMemcpyAsync(ratio.data(), c->colratio.p, nrhs * 8, cudaMemcpyDeviceToHost, c->st));
    int werr = 0;
    if (block) CU(cudaMemcpyAsync(&werr, c->info.p + 1, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CU(cudaStreamSynchronize(c->st));
    if (werr) return fail(HAMS_ERR_CUDA, "block LU solve: a tensor-core GEMM gave up waiting on its pipeline (%d)", werr);
    double worst = 0.0;
    for (double r : ratio) worst = std::max(worst, r);
    c->refine_sweeps = it;
    if (it > 0 && prev > 0.0) c->ir_rate = std::max(c->ir_rate, worst / prev);
    if (!(worst == worst)) return fail(HAMS_ERR_NUMERIC, "non-finite residual in iterative refinement");
    if (worst <= tol) break;
    if (it >= maxit) return fail(HAMS_ERR_NUMERIC, "iterative refinement: %.3e after %d sweeps", worst, it);
    if (it > 4 && worst > 0.5 * prev) return fail(HAMS_ERR_NUMERIC, "iterative refinement stalled at %.3e", worst);
    prev = worst;
    // the surrogate judgement's probe rides on the first sweep: its right-hand
    // sides dB - dA X (at this X, to first order the same estimate) go through
    // the same solve as the residual
    const bool fold = c->judge_pending;
    if (fold) {
      TRY(c->jdX.alloc(nx));
      TRY(c->jB.alloc(nx));
      TRY(judge_rhs(c, c->judge_nbeta, c->X.p, c->jB.p, c->jdX.p));
    }
    k_z2c<<<592, 256, 0, c->st>>>(c->R.p, c->Xf.p, nx);
    if (fold) k_z2c<<<592, 256, 0, c->st>>>(c->jB.p, c->Xf.p + nx, nx);
    TRY(launch_check(c, fold ? 2 : 1));
    TRY(mixed_apply(c, fold ? 2 * nrhs : nrhs));
    k_c2z_add<<<592, 256, 0, c->st>>>(c->Xf.p, c->X.p, nx);
    TRY(launch_check(c));
    if (fold) {
      CU(cudaMemcpyAsync(c->jdX.p, c->Xf.p + nx, nx * sizeof(float2), cudaMemcpyDeviceToDevice, c->st));
      c->judge_pending = false;
      c->judge_folded = true;
    }
  }
  return 0;
}

// Mixed form: X (n x nrhs, FP64) from the FP64 matrix M (n x n) and the
// right-hand sides rhs (ld ldr = n): complex64 factorisation of M (block LU
// of lu_mixed.cu, or the library's Cgetrf), then FP64 iterative refinement
// R = rhs - M X, X += LU^-1 R until the residual of every column is below
// refine_tol of that column's scale.  Returns HAMS_ERR_NUMERIC when the
// factorisation breaks down or the refinement stalls.
static int mixed_solve(hams_ctx* c, double2* M, const double2* rhs, int ldr, int nrhs, int kind, int* info_host) {
  const int n = c->n, lda = mixed_lu_ld(n);
  const size_t nx = (size_t)n * nrhs;
  TRY(c->Af.alloc((size_t)lda * n));
  TRY(c->Xf.alloc(c->judge_pending ? 2 * nx : nx));  // room for the judgement's probe in the first sweep
  TRY(c->R.alloc(nx));
  TRY(c->colratio.alloc(nrhs));
  CU(cudaMemcpy2DAsync(c->X.p, (size_t)n * 16, rhs, (size_t)ldr * 16, (size_t)n * 16, nrhs, cudaMemcpyDeviceToDevice, c->st));
  k_z2c_ld<<<1184, 256, 0, c->st>>>(M, c->Af.p, n, lda);
  TRY(launch_check(c));
  const bool block = kind != HAMS_LU_LIBRARY;
  c->lu_used = kind;
  if (block) {
    TRY(c->luw.alloc(mixed_lu_workspace_elems(n, c->judge_pending ? 2 * nrhs : nrhs)));
    TRY(c->perm.alloc(n));
    long long la = 0, lb = 0;
    // TF32: the library's tcgen05 GEMM; the FP32 emulation on BF16 tensor cores is cuBLAS's
    const bool own = kind == HAMS_LU_BLOCK_TF32;
    auto body = [&](long long* l) {
      return mixed_lu_factor(c->st, c->blas, own, CUBLAS_COMPUTE_32F_EMULATED_16BFX9, n, lda, c->Af.p, c->perm.p,
                             c->luw.p, c->info.p, l, &lb);
    };
    int rc = (own && c->opts.lu_graph == 1)
                 ? lu_graph_run(c, c->lu_factor_graph, c->Af.p, c->perm.p, c->luw.p, c->info.p, 0, &la, body)
                 : body(&la);
    c->launches += la;
    c->lib_calls += lb;
    if (rc == 1) return fail(HAMS_ERR_NUMERIC, "block LU: CUDA failed");
    if (rc) return fail(HAMS_ERR_NUMERIC, "block LU: cuBLAS status %d in GEMM %d of block %d", rc % 100, rc % 1000 / 100,
                        rc / 1000);
    int word[2] = {0, 0};
    CU(cudaMemcpyAsync(word, c->info.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CU(cudaStreamSynchronize(c->st));
    if (word[1]) return fail(HAMS_ERR_CUDA, "block LU: a tensor-core GEMM gave up waiting on its pipeline (%d)", word[1]);
    if (word[0] <= n) return fail(HAMS_ERR_NUMERIC, "block LU: zero pivot in column %d", word[0]);
    *info_host = 0;
  } else {
    int lw = 0;
    CUS(cusolverDnCgetrf_bufferSize(c->solver, n, n, (cuComplex*)c->Af.p, lda, &lw));
    TRY(c->work32.alloc((size_t)lw * sizeof(cuComplex)));
    CUS(cusolverDnCgetrf(c->solver, n, n, (cuComplex*)c->Af.p, lda, (cuComplex*)c->work32.p, c->ipiv.p, c->info.p));
    c->lib_calls += 1;
    CU(cudaMemcpyAsync(info_host, c->info.p, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  }
  CU(cudaEventRecord(c->evf, c->st));
  k_z2c<<<592, 256, 0, c->st>>>(c->X.p, c->Xf.p, nx);
  TRY(launch_check(c));
  TRY(mixed_apply(c, nrhs));
  k_c2z<<<592, 256, 0, c->st>>>(c->Xf.p, c->X.p, nx);
  TRY(launch_check(c));
  return mixed_refine(c, M, rhs, ldr, nrhs);
}

// GMRES (IterativeSolvers.f90:324-484, ZGMRES_SOLVE): X (n x nrhs) from the
// FP64 matrix M and the right-hand sides rhs, every column from zero,
// restarted every m steps, right-preconditioned by the LU factors of each
// body's diagonal block (:176-253) or, with one body, by the diagonal
// (:154-174).  All columns advance together: one ZGEMM per step, classical
// Gram-Schmidt applied twice as strided-batched GEMVs (the reference's
// modified Gram-Schmidt one vector at a time, :399-406), the small
// Hessenberg least-squares problems (Givens rotations) on the host.  A column
// that misses the tolerance after gmres_maxit steps keeps its last iterate
// and the solve's note says so (:475-480).  Without lids the products (Krylov
// steps and restart residuals) use the H-matrix of M (HMatrix.f90, as
// AssbMatx[Multi].f90:284-288 do); the preconditioner is built from M itself.
static int gmres_solve(hams_ctx* c, double2* M, const double2* rhs, int nrhs) {
  const int n = c->n, nb = c->nb;
  const int m = c->opts.gmres_restart > 0 ? c->opts.gmres_restart : 25;
  const int maxit = c->opts.gmres_maxit > 0 ? c->opts.gmres_maxit : 100;
  const double tol = c->opts.gmres_tol > 0.0 ? c->opts.gmres_tol : 1e-4;
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0),
                        mone = make_cuDoubleComplex(-1.0, 0.0);
  const size_t vs = (size_t)n * (m + 1);  // basis stride of one column
  TRY(c->gv.alloc(vs * nrhs));
  TRY(c->gw.alloc((size_t)n * nrhs));
  TRY(c->gz.alloc((size_t)n * nrhs));
  TRY(c->gy.alloc((size_t)(m + 1) * nrhs));
  TRY(c->gnrm.alloc(nrhs));
  const bool use_h = c->nl == 0 && c->opts.gmres_dense == 0;
  if (use_h) {
    if (!c->hm_ready) {
      hmat::Tree t;
      hmat::build_tree(c->xyz_p.data(), n, t);
      if (hmat::upload(t, c->hm)) return fail(HAMS_ERR_NOMEM, "H-matrix: device allocation failed");
      c->hm_ready = true;
    }
    const double aca = c->opts.aca_tol > 0.0 ? c->opts.aca_tol : hmat::kAcaTol;
    if (hmat::compress(c->st, M, aca, c->hm)) return fail(HAMS_ERR_CUDA, "H-matrix: ACA launch failed");
    c->launches += 1 + (c->hm.nlow > 0);
    std::vector<int> hr(c->hm.nlow);
    std::vector<long long> hoff;
    if (c->hm.nlow > 0) CU(cudaMemcpyAsync(hr.data(), c->hm.rank, sizeof(int) * hr.size(), cudaMemcpyDeviceToHost, c->st));
    CU(cudaStreamSynchronize(c->st));
    const long long wsize = hmat::product_offsets(c->st, hr, nrhs, c->hm, hoff);
    TRY(c->hw.alloc((size_t)wsize));
    TRY(c->hxp.alloc((size_t)n * nrhs));
    TRY(c->hyp.alloc((size_t)n * nrhs));
    CU(cudaStreamSynchronize(c->st));  // hoff is read by the copy above
  }
  // Y (n x nrhs) = M X, with the H-matrix or the dense matrix
  auto product = [&](const double2* Xin, double2* Y) -> int {
    if (use_h) {
      long long la = 0;
      if (hmat::matvec(c->st, c->hm, Xin, Y, nrhs, c->hxp.p, c->hyp.p, c->hw.p, &la))
        return fail(HAMS_ERR_CUDA, "H-matrix product launch failed");
      c->launches += la;
      return 0;
    }
    CUB_(cublasZgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, n, nrhs, n, &one, (cuDoubleComplex*)M, n,
                     (const cuDoubleComplex*)Xin, n, &zero, (cuDoubleComplex*)Y, n));
    c->lib_calls += 1;
    return 0;
  };
  // preconditioner: LU of each body's diagonal block, packed one after
  // another, or the diagonal of M with one body
  std::vector<size_t> boff(nb + 1, 0);
  std::vector<int> bst(nb + 1, 0);
  for (int b = 0; b < nb; ++b) {
    bst[b + 1] = bst[b] + c->body_nelem[b];
    boff[b + 1] = boff[b] + (size_t)c->body_nelem[b] * c->body_nelem[b];
  }
  TRY(c->gpiv.alloc(n));
  if (nb == 1) {
    TRY(c->gpre.alloc(n));
    k_jacobi_setup<<<(n + 255) / 256, 256, 0, c->st>>>(M, n, c->gpre.p);
    TRY(launch_check(c));
  } else {
    TRY(c->gpre.alloc(boff[nb]));
    int lwmax = 0;
    for (int b = 0; b < nb; ++b) {
      const int nn = c->body_nelem[b];
      CU(cudaMemcpy2DAsync(c->gpre.p + boff[b], (size_t)nn * 16, M + bst[b] + (size_t)bst[b] * n, (size_t)n * 16,
                           (size_t)nn * 16, nn, cudaMemcpyDeviceToDevice, c->st));
      int lw = 0;
      CUS(cusolverDnZgetrf_bufferSize(c->solver, nn, nn, (cuDoubleComplex*)(c->gpre.p + boff[b]), nn, &lw));
      lwmax = std::max(lwmax, lw);
    }
    TRY(c->work.alloc((size_t)lwmax * sizeof(cuDoubleComplex)));
    for (int b = 0; b < nb; ++b) {
      const int nn = c->body_nelem[b];
      CUS(cusolverDnZgetrf(c->solver, nn, nn, (cuDoubleComplex*)(c->gpre.p + boff[b]), nn,
                           (cuDoubleComplex*)c->work.p, c->gpiv.p + bst[b], c->info.p));
    }
    c->lib_calls += 2 * nb;
  }
  CU(cudaEventRecord(c->evf, c->st));
  auto precond = [&](double2* Z) -> int {  // Z (n x nrhs) <- P^-1 Z
    if (nb == 1) {
      k_jacobi_apply<<<(unsigned)(((size_t)n * nrhs + 255) / 256), 256, 0, c->st>>>(c->gpre.p, n, nrhs, Z);
      return launch_check(c);
    }
    for (int b = 0; b < nb; ++b) {
      const int nn = c->body_nelem[b];
      CUS(cusolverDnZgetrs(c->solver, CUBLAS_OP_N, nn, nrhs, (cuDoubleComplex*)(c->gpre.p + boff[b]), nn,
                           c->gpiv.p + bst[b], (cuDoubleComplex*)(Z + bst[b]), n, c->info.p));
    }
    c->lib_calls += nb;
    return 0;
  };
  // right-hand-side norms
  k_colnorm2<<<nrhs, 256, 0, c->st>>>(rhs, n, c->gnrm.p);
  TRY(launch_check(c));
  std::vector<double> bnorm(nrhs), nr(nrhs);
  CU(cudaMemcpyAsync(bnorm.data(), c->gnrm.p, nrhs * 8, cudaMemcpyDeviceToHost, c->st));
  CU(cudaMemsetAsync(c->X.p, 0, (size_t)n * nrhs * 16, c->st));
  CU(cudaMemcpyAsync(c->gw.p, rhs, (size_t)n * nrhs * 16, cudaMemcpyDeviceToDevice, c->st));  // R = B - A 0
  CU(cudaStreamSynchronize(c->st));
  typedef std::complex<double> zc;
  std::vector<zc> H((size_t)(m + 1) * m * nrhs), g((size_t)(m + 1) * nrhs), sn((size_t)m * nrhs);
  std::vector<double> cr((size_t)m * nrhs), beta(nrhs);
  std::vector<zc> hcol((size_t)(m + 1) * nrhs), y((size_t)(m + 1) * nrhs);
  int iters = 0;
  bool done = false;
  while (!done) {
    // V_0 = R / |R|
    k_colnorm2<<<nrhs, 256, 0, c->st>>>(c->gw.p, n, c->gnrm.p);
    k_normalize_into<<<(unsigned)(((size_t)n * nrhs + 255) / 256), 256, 0, c->st>>>(c->gw.p, n, nrhs, c->gnrm.p,
                                                                                    c->gv.p, vs);
    TRY(launch_check(c, 2));
    CU(cudaMemcpyAsync(beta.data(), c->gnrm.p, nrhs * 8, cudaMemcpyDeviceToHost, c->st));
    CU(cudaStreamSynchronize(c->st));
    bool all = true;
    for (int r = 0; r < nrhs; ++r) {
      g[(size_t)r * (m + 1)] = beta[r];
      for (int i = 1; i <= m; ++i) g[(size_t)r * (m + 1) + i] = 0.0;
      if (beta[r] > tol * bnorm[r]) all = false;
    }
    if (all) break;
    int k = 0;  // Arnoldi steps done in this cycle
    for (int j = 0; j < m && iters < maxit; ++j, ++k, ++iters) {
      // W = A M^-1 V_j
      CU(cudaMemcpy2DAsync(c->gz.p, (size_t)n * 16, c->gv.p + (size_t)j * n, vs * 16, (size_t)n * 16, nrhs,
                           cudaMemcpyDeviceToDevice, c->st));
      TRY(precond(c->gz.p));
      TRY(product(c->gz.p, c->gw.p));
      for (size_t e = 0; e < hcol.size(); ++e) hcol[e] = 0.0;
      for (int pass = 0; pass < 2; ++pass) {  // classical Gram-Schmidt, twice
        CUB_(cublasZgemvStridedBatched(c->blas, CUBLAS_OP_C, n, j + 1, &one, (cuDoubleComplex*)c->gv.p, n, (long long)vs,
                                       (cuDoubleComplex*)c->gw.p, 1, n, &zero, (cuDoubleComplex*)c->gy.p, 1, m + 1,
                                       nrhs));
        CUB_(cublasZgemvStridedBatched(c->blas, CUBLAS_OP_N, n, j + 1, &mone, (cuDoubleComplex*)c->gv.p, n, (long long)vs,
                                       (cuDoubleComplex*)c->gy.p, 1, m + 1, &one, (cuDoubleComplex*)c->gw.p, 1, n,
                                       nrhs));
        c->lib_calls += 2;
        CU(cudaMemcpyAsync(y.data(), c->gy.p, (size_t)(m + 1) * nrhs * 16, cudaMemcpyDeviceToHost, c->st));
        CU(cudaStreamSynchronize(c->st));
        for (int r = 0; r < nrhs; ++r)
          for (int i = 0; i <= j; ++i) hcol[(size_t)r * (m + 1) + i] += y[(size_t)r * (m + 1) + i];
      }
      k_colnorm2<<<nrhs, 256, 0, c->st>>>(c->gw.p, n, c->gnrm.p);
      k_normalize_into<<<(unsigned)(((size_t)n * nrhs + 255) / 256), 256, 0, c->st>>>(
          c->gw.p, n, nrhs, c->gnrm.p, c->gv.p + (size_t)(j + 1) * n, vs);
      TRY(launch_check(c, 2));
      CU(cudaMemcpyAsync(nr.data(), c->gnrm.p, nrhs * 8, cudaMemcpyDeviceToHost, c->st));
      CU(cudaStreamSynchronize(c->st));
      all = true;
      for (int r = 0; r < nrhs; ++r) {
        zc* h = &hcol[(size_t)r * (m + 1)];
        h[j + 1] = nr[r];
        for (int i = 0; i < j; ++i) {  // earlier rotations
          const size_t q = (size_t)r * m + i;
          zc a = h[i], b = h[i + 1];
          h[i] = cr[q] * a + sn[q] * b;
          h[i + 1] = -std::conj(sn[q]) * a + cr[q] * b;
        }
        // complex Givens rotation: cr real, [cr sn; -conj(sn) cr] (h_j, h_j+1) = (rho, 0)
        const double aa = std::abs(h[j]), bb = std::abs(h[j + 1]), rho = std::hypot(aa, bb);
        const size_t q = (size_t)r * m + j;
        if (bb < 1e-30) {
          cr[q] = 1.0;
          sn[q] = 0.0;
        } else if (aa < 1e-30) {
          cr[q] = 0.0;
          sn[q] = std::conj(h[j + 1]) / bb;
        } else {
          cr[q] = aa / rho;
          sn[q] = (h[j] / aa) * std::conj(h[j + 1]) / rho;
        }
        const zc gj = g[(size_t)r * (m + 1) + j];
        g[(size_t)r * (m + 1) + j] = cr[q] * gj;
        g[(size_t)r * (m + 1) + j + 1] = -std::conj(sn[q]) * gj;
        h[j] = cr[q] * h[j] + sn[q] * h[j + 1];
        h[j + 1] = 0.0;
        for (int i = 0; i <= j; ++i) H[((size_t)r * m + j) * (m + 1) + i] = h[i];
        if (std::abs(g[(size_t)r * (m + 1) + j + 1]) > tol * bnorm[r]) all = false;
      }
      if (all) {
        ++k;
        ++iters;
        break;
      }
    }
    if (k == 0) return fail(HAMS_ERR_NUMERIC, "GMRES: no progress");
    // y = R^-1 g per column, X += M^-1 (V y)
    for (int r = 0; r < nrhs; ++r) {
      zc* yr = &y[(size_t)r * (m + 1)];
      for (int i = k - 1; i >= 0; --i) {
        zc s = g[(size_t)r * (m + 1) + i];
        for (int l = i + 1; l < k; ++l) s -= H[((size_t)r * m + l) * (m + 1) + i] * yr[l];
        const zc d = H[((size_t)r * m + i) * (m + 1) + i];
        yr[i] = std::abs(d) < 1e-30 ? 0.0 : s / d;
      }
      for (int i = k; i <= m; ++i) yr[i] = 0.0;
    }
    CU(cudaMemcpyAsync(c->gy.p, y.data(), (size_t)(m + 1) * nrhs * 16, cudaMemcpyHostToDevice, c->st));
    CUB_(cublasZgemvStridedBatched(c->blas, CUBLAS_OP_N, n, k, &one, (cuDoubleComplex*)c->gv.p, n, (long long)vs,
                                   (cuDoubleComplex*)c->gy.p, 1, m + 1, &zero, (cuDoubleComplex*)c->gz.p, 1, n, nrhs));
    c->lib_calls += 1;
    TRY(precond(c->gz.p));
    CUB_(cublasZaxpy(c->blas, n * nrhs, &one, (cuDoubleComplex*)c->gz.p, 1, (cuDoubleComplex*)c->X.p, 1));
    // true residual R = B - A X for the next cycle and the stop test
    TRY(product(c->X.p, c->gz.p));
    CU(cudaMemcpyAsync(c->gw.p, rhs, (size_t)n * nrhs * 16, cudaMemcpyDeviceToDevice, c->st));
    CUB_(cublasZaxpy(c->blas, n * nrhs, &mone, (cuDoubleComplex*)c->gz.p, 1, (cuDoubleComplex*)c->gw.p, 1));
    c->lib_calls += 3;
    if (iters >= maxit) {
      k_colnorm2<<<nrhs, 256, 0, c->st>>>(c->gw.p, n, c->gnrm.p);
      TRY(launch_check(c));
      CU(cudaMemcpyAsync(nr.data(), c->gnrm.p, nrhs * 8, cudaMemcpyDeviceToHost, c->st));
      CU(cudaStreamSynchronize(c->st));
      double worst = 0.0;
      for (int r = 0; r < nrhs; ++r) worst = std::max(worst, bnorm[r] > 0 ? nr[r] / bnorm[r] : nr[r]);
      if (worst > tol) {
        char buf[128];
        std::snprintf(buf, sizeof buf, "GMRES: relative residual %.3e after %d steps (tolerance %.1e)", worst, iters,
                      tol);
        c->note += (c->note.empty() ? "" : "; ") + std::string(buf);
      }
      done = true;
    }
  }
  c->refine_sweeps = iters;
  return 0;
}

// Solve on the device: X (n x nrhs) from A, B (or normal equations with lids).
static int solve_dev(hams_ctx* c, int nrhs, int* info_host) {
  const int n = c->n, tn = c->tn;
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
  double2* M = c->A.p;  // matrix to factor
  double2* rhs = c->B.p;
  int ldr = tn;
  if (c->nl > 0) {
    TRY(c->C.alloc((size_t)n * n));
    TRY(c->D.alloc((size_t)n * nrhs));
    CUB_(cublasZgemm(c->blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, tn, &one, (cuDoubleComplex*)c->A.p, tn,
                     (cuDoubleComplex*)c->A.p, tn, &zero, (cuDoubleComplex*)c->C.p, n));
    CUB_(cublasZgemm(c->blas, CUBLAS_OP_T, CUBLAS_OP_N, n, nrhs, tn, &one, (cuDoubleComplex*)c->A.p, tn,
                     (cuDoubleComplex*)c->B.p, tn, &zero, (cuDoubleComplex*)c->D.p, n));
    c->lib_calls += 2;
    M = c->C.p;
    rhs = c->D.p;
    ldr = n;
  }
  TRY(c->X.alloc((size_t)n * nrhs));
  CU(cudaMemcpy2DAsync(c->X.p, (size_t)n * 16, rhs, (size_t)ldr * 16, (size_t)n * 16, nrhs, cudaMemcpyDeviceToDevice, c->st));
  *info_host = 0;
  c->note.clear();
  // with lids GMRES iterates on the normal equations, as the reference does
  // (AssbMatx_irr.f90:494-498)
  if (c->opts.solver == HAMS_SOLVER_GMRES) return gmres_solve(c, M, rhs, nrhs);
  if (c->opts.precision == HAMS_PREC_FP64) {
    int lw = 0;
    CUS(cusolverDnZgetrf_bufferSize(c->solver, n, n, (cuDoubleComplex*)M, n, &lw));
    TRY(c->work.alloc((size_t)lw * sizeof(cuDoubleComplex)));
    // M is overwritten by its factors
    CUS(cusolverDnZgetrf(c->solver, n, n, (cuDoubleComplex*)M, n, (cuDoubleComplex*)c->work.p, c->ipiv.p, c->info.p));
    CU(cudaEventRecord(c->evf, c->st));
    CUS(cusolverDnZgetrs(c->solver, CUBLAS_OP_N, n, nrhs, (cuDoubleComplex*)M, n, c->ipiv.p, (cuDoubleComplex*)c->X.p, n, c->info.p));
    c->lib_calls += 2;
    CU(cudaMemcpyAsync(info_host, c->info.p, sizeof(int), cudaMemcpyDeviceToHost, c->st));
    return 0;
  }
  // mixed: complex64 LU of a rounded copy + FP64 iterative refinement; the
  // block LU falls back to the library's partially pivoted LU when its
  // refinement does not converge
  int kind = c->opts.lu_kind;
  if (kind == HAMS_LU_BLOCK_EMU) {
    int ver = 0;
    if (cublasGetVersion(c->blas, &ver) != CUBLAS_STATUS_SUCCESS || ver < 120900) {
      kind = HAMS_LU_BLOCK_TF32;  // FP32 emulation on BF16 tensor cores arrived with cuBLAS 12.9
      c->note = "cuBLAS " + std::to_string(ver) + " has no BF16x9 emulation: block LU on TF32";
    }
  }
  if (kind == HAMS_LU_BLOCK_EMU || kind == HAMS_LU_BLOCK_TF32) {
    int rc = mixed_solve(c, M, rhs, ldr, nrhs, kind, info_host);
    if (rc == 0) return 0;
    if (rc != HAMS_ERR_NUMERIC) return rc;
    c->note += (c->note.empty() ? "" : "; ") + std::string("block LU replaced by the library LU: ") + g_err;
    g_err.clear();
    // a probe the block LU's sweep carried is redone with the library's factors
    c->judge_pending = c->judge_pending || c->judge_folded;
    c->judge_folded = false;
  }
  return mixed_solve(c, M, rhs, ldr, nrhs, HAMS_LU_LIBRARY, info_host);
}

static int forces_dev(hams_ctx* c, const hams_wave* w, int nbeta) {
  const int nb = c->nb, ndof = 6 * nb, nrhs = ndof + nbeta;
  WaveDev wd = wave_dev(c, w);
  IncWave q = inc_params(wd, c->opts.amp, c->opts.g, c->opts.xw[0], c->opts.xw[1]);
  size_t tot = 2 * (size_t)ndof * ndof + 2 * (size_t)ndof * std::max(nbeta, 1);
  TRY(c->outbuf.alloc(tot));
  double* amas = c->outbuf.p;
  double* bdmp = amas + (size_t)ndof * ndof;
  double2* exfc = (double2*)(bdmp + (size_t)ndof * ndof);
  k_forces<<<dim3(nb, 6, nrhs), 256, 0, c->st>>>(c->g, wd, q, c->beta.p, nbeta, c->opts.isol, c->opts.rho, c->X.p,
                                                 c->n, amas, bdmp, exfc);
  return launch_check(c);
}

// Potentials at the field points from the solved panel potentials X
// (CalPotentialMulti, PressureElevationMulti.f90:55-272): the influence of
// every panel at every point (k_field_pairs), then
// POT = (S_f BC - D_f X) / (2 pi or 4 pi) as two complex GEMMs, the incident
// potential added for the total-potential solution; copied to fp_last.
static int field_dev(hams_ctx* c, const hams_wave* w, int nbeta) {
  const int n = c->n, nfp = c->nfp, nrad = 6 * c->nb, ncol = nrad + nbeta;
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0),
                        mone = make_cuDoubleComplex(-1.0, 0.0);
  WaveDev wd = wave_dev(c, w);
  TRY(c->fp_S.alloc((size_t)nfp * n));
  TRY(c->fp_D.alloc((size_t)nfp * n));
  TRY(c->fp_bc.alloc((size_t)n * ncol));
  TRY(c->fp_pot.alloc((size_t)nfp * ncol));
  TRY(c->fp_out.alloc((size_t)nfp * (ncol + nbeta)));
  launch_field_pairs(c->st, c->g, wd, c->wvn.p, nfp, c->fp_x.p, c->fp_S.p, c->fp_D.p, c->ovf.p);
  k_field_bc<<<dim3((n + 127) / 128, ncol), 128, 0, c->st>>>(c->g, nbeta, c->wd.p, c->fp_bc.p);
  TRY(launch_check(c, 2));
  CUB_(cublasZgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, nfp, ncol, n, &one, (cuDoubleComplex*)c->fp_S.p, nfp,
                   (cuDoubleComplex*)c->fp_bc.p, n, &zero, (cuDoubleComplex*)c->fp_pot.p, nfp));
  CUB_(cublasZgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, nfp, ncol, n, &mone, (cuDoubleComplex*)c->fp_D.p, nfp,
                   (cuDoubleComplex*)c->X.p, n, &one, (cuDoubleComplex*)c->fp_pot.p, nfp));
  c->lib_calls += 2;
  IncWave q = inc_params(wd, c->opts.amp, c->opts.g, c->opts.xw[0], c->opts.xw[1]);
  const int add_inc = c->opts.isol == 1 && !wd.limit;
  k_field_finish<<<dim3((nfp + 127) / 128, ncol + nbeta), 128, 0, c->st>>>(nfp, ncol, nrad, nbeta, c->fp_x.p,
                                                                            c->fp_sld.p, q, c->beta.p, add_inc,
                                                                            c->fp_pot.p, c->fp_out.p);
  TRY(launch_check(c));
  c->fp_last.resize(2 * (size_t)nfp * (ncol + nbeta));
  CU(cudaMemcpyAsync(c->fp_last.data(), c->fp_out.p, c->fp_last.size() * 8, cudaMemcpyDeviceToHost, c->st));
  return 0;
}

// Safety factor of the judgement: the largest ratio of a frequency's true
// error (against the plain series) to its estimate, observed on the
// 5,400-panel 3 x 3 array of cylinders (h = 50 m) over 0.2-2.5 rad/s, rounded up.
constexpr double kJudgeSafety = 1.0;

// The series' judgement of a frequency solved with the surrogate: an estimate
// of the surrogate's relative error in added mass, damping and excitation.
//   e      the network's relative error on the far-pair entries of A and S,
//          from the pairs sampled during the assembly (k_sample_err);
//   the error model: per cell of the network's input domain (R/h x source
//          depth x field depth), the RMS of (network - series) relative to
//          the series' real parts over the samples of that cell (k_judge_fit);
//   the probe: every far-pair entry of A and S replaced by its cell's
//          error taken coherent, r Re(entry) (k_probe_scales), the first-order change
//          of the solution, dX = (L U)^-1 (dB - dA X), carried through the
//          force reductions: the estimated change of each output, relative
//          to the output.
// The estimate is kJudgeSafety times the largest of the three.  A, S and X
// are kept, B is overwritten.  Requires the mixed solve's factors.
static int judge_rhs(hams_ctx* c, int nbeta, const double2* X, double2* out, float2* xs) {
  const int n = c->n, tn = c->tn, nb = c->nb, nrhs = 6 * nb + nbeta;
  if (!c->sg_map.p) return fail(HAMS_ERR_ARG, "surrogate judgement without its cell map");
  TRY(c->sg_scale.alloc(2 * kJCells));
  k_probe_scales<<<1, 256, 0, c->st>>>(c->sg_cells.p, c->sg_scale.p);
  // dB: the right-hand sides of the probe of S (this frequency's diffraction weights are still in wd)
  const int nch = (int)c->chunks_h.size();
  k_rhs_partial<true><<<dim3((tn + 127) / 128, nch), 128, 0, c->st>>>(c->g, c->S.p, c->chunks.p, c->wd.p, nbeta,
                                                                      c->part.p, c->sg_map.p, c->sg_scale.p);
  k_rhs_final<<<(tn + 127) / 128, 128, 0, c->st>>>(tn, nb, nch, c->chunk_body.p, c->part.p, nbeta, out);
  // out = dB - dA X, X rounded to complex64 in xs
  const size_t nx = (size_t)n * nrhs;
  k_z2c<<<592, 256, 0, c->st>>>(X, xs, nx);
  k_probe_apply<<<(tn + kPrRows - 1) / kPrRows, kPrThreads, 0, c->st>>>(c->g, c->sg_map.p, c->sg_scale.p, c->A.p, xs,
                                                                         nrhs, out);
  return launch_check(c, 5);
}

// The estimate from dX (complex64, n x nrhs): the forces of X + dX against
// those of X (outbuf), relative per output.
static int judge_finish(hams_ctx* c, const hams_wave* w, int nbeta, const float2* dX) {
  const int n = c->n, nb = c->nb, ndof = 6 * nb, nrhs = ndof + nbeta;
  const double eps = 1.0;  // the probe is the modelled error itself
  WaveDev wd = wave_dev(c, w);
  const size_t nx = (size_t)n * nrhs;
  TRY(c->R.alloc(nx));
  CU(cudaMemcpyAsync(c->R.p, c->X.p, nx * 16, cudaMemcpyDeviceToDevice, c->st));
  k_c2z_add<<<592, 256, 0, c->st>>>(dX, c->R.p, nx);
  TRY(launch_check(c));
  const size_t tot = 2 * (size_t)ndof * ndof + 2 * (size_t)ndof * std::max(nbeta, 1);
  TRY(c->outbuf2.alloc(tot));
  IncWave q = inc_params(wd, c->opts.amp, c->opts.g, c->opts.xw[0], c->opts.xw[1]);
  double* a2 = c->outbuf2.p;
  k_forces<<<dim3(nb, 6, nrhs), 256, 0, c->st>>>(c->g, wd, q, c->beta.p, nbeta, c->opts.isol, c->opts.rho, c->R.p,
                                                 c->n, a2, a2 + (size_t)ndof * ndof,
                                                 (double2*)(a2 + 2 * (size_t)ndof * ndof));
  TRY(launch_check(c));
  std::vector<double> o1(tot), o2(tot);
  double red[4] = {0.0, 0.0, 0.0, 0.0};
  CU(cudaMemcpyAsync(o1.data(), c->outbuf.p, tot * 8, cudaMemcpyDeviceToHost, c->st));
  CU(cudaMemcpyAsync(o2.data(), c->outbuf2.p, tot * 8, cudaMemcpyDeviceToHost, c->st));
  CU(cudaMemcpyAsync(red, c->sg_red.p, 4 * 8, cudaMemcpyDeviceToHost, c->st));
  CU(cudaStreamSynchronize(c->st));
  auto kappa = [&](size_t off, size_t cnt) {
    double d = 0.0, r = 0.0;
    for (size_t e = off; e < off + cnt; ++e) {
      d += (o2[e] - o1[e]) * (o2[e] - o1[e]);
      r += o1[e] * o1[e];
    }
    return r > 0.0 ? std::sqrt(d / r) / eps : 0.0;
  };
  const size_t na = (size_t)ndof * ndof;
  double* j = c->sg_judge;  // e_A, e_S (sampled), the estimated error of A, B, X, the estimate
  j[0] = red[1] > 0.0 ? std::sqrt(red[0] / red[1]) : 0.0;
  j[1] = red[3] > 0.0 ? std::sqrt(red[2] / red[3]) : 0.0;
  j[2] = kappa(0, na);
  j[3] = kappa(na, na);
  j[4] = nbeta > 0 ? kappa(2 * na, 2 * (size_t)ndof * nbeta) : 0.0;
  j[5] = kJudgeSafety * std::max(j[2], std::max(j[3], j[4]));
  j[7] = (double)(c->sg_ns4 + c->sg_ns5);
  return 0;
}

// The judgement after the solve.  When the mixed solve's first refinement
// sweep already carried the probe (mixed_refine, judge_pending), dX is in
// jdX; otherwise (no sweep was needed) the probe gets its own solve.
static int surrogate_judge(hams_ctx* c, const hams_wave* w, int nbeta) {
  if (c->judge_folded) return judge_finish(c, w, nbeta, c->jdX.p);
  const int n = c->n, nrhs = 6 * c->nb + nbeta;
  const size_t nx = (size_t)n * nrhs;
  TRY(c->R.alloc(nx));
  TRY(judge_rhs(c, nbeta, c->X.p, c->B.p, reinterpret_cast<float2*>(c->R.p)));
  k_z2c<<<592, 256, 0, c->st>>>(c->B.p, c->Xf.p, nx);  // tn == n: B is n x nrhs, contiguous
  TRY(launch_check(c));
  TRY(mixed_apply(c, nrhs));
  return judge_finish(c, w, nbeta, c->Xf.p);
}

// A frequency the judgement gave to the series, without a new factorisation:
// the far pairs again from the series (the near pairs of A and S are the
// series' already), the block copies and right-hand sides again, then FP64
// refinement from the network's solution with the network's factors -- the
// network's matrix is within its error of the series' one, so the factors
// are as good a preconditioner for it as for their own.  HAMS_ERR_NUMERIC
// when the refinement stalls (the caller then factors the series' matrix).
static int series_refine(hams_ctx* c, const hams_wave* w, int nbeta) {
  const int nrhs = 6 * c->nb + nbeta;
  TRY(far_series(c, wave_dev(c, w)));
  TRY(copy_blocks_and_rhs(c, nbeta));
  return mixed_refine(c, c->A.p, c->B.p, c->tn, nrhs);
}

static int solve_one(hams_ctx* c, const hams_wave* w, int nbeta, const double* beta, double* amas, double* bdmp,
                     double* exfc) {
  const int ndof = 6 * c->nb;
  if (nbeta < 0) return fail(HAMS_ERR_ARG, "nbeta < 0");
  TRY(c->beta.alloc(std::max(nbeta, 1)));
  if (nbeta > 0) CU(cudaMemcpyAsync(c->beta.p, beta, (size_t)nbeta * 8, cudaMemcpyHostToDevice, c->st));
  CU(cudaEventRecord(c->evc, c->st));
  for (double& v : c->sg_judge) v = 0.0;
  TRY(assemble_dev(c, w, nbeta));
  const bool judged = c->sg_used && c->sg_tol > 0.0 && c->sg_ns4 + c->sg_ns5 > 0 &&
                      c->opts.precision == HAMS_PREC_MIXED && c->opts.solver != HAMS_SOLVER_GMRES && c->nl == 0;
  c->judge_pending = judged;
  c->judge_folded = false;
  c->judge_nbeta = nbeta;
  int info = 0;
  const int src = solve_dev(c, ndof + nbeta, &info);
  c->judge_pending = false;
  TRY(src);
  CU(cudaEventRecord(c->ev[3], c->st));
  TRY(forces_dev(c, w, nbeta));
  if (judged) {
    TRY(surrogate_judge(c, w, nbeta));
    c->judge_folded = false;
    if (c->sg_judge[5] > c->sg_tol) {  // the series takes this frequency
      const std::string keep = c->note;
      const char* how = "refined to the series";
      int rc = series_refine(c, w, nbeta);
      if (rc == HAMS_ERR_NUMERIC) {  // the refinement stalled: factor the series' matrix
        g_err.clear();
        how = "re-solved with the series";
        TRY(assemble_dev(c, w, nbeta, true));
        TRY(solve_dev(c, ndof + nbeta, &info));
      } else if (rc) {
        return rc;
      }
      CU(cudaEventRecord(c->ev[3], c->st));
      TRY(forces_dev(c, w, nbeta));
      c->sg_judge[6] = 1.0;
      char buf[160];
      std::snprintf(buf, sizeof buf, "surrogate estimate %.2e > %.2e: %s", c->sg_judge[5], c->sg_tol, how);
      c->note = keep.empty() ? std::string(buf) : keep + "; " + buf;
    }
  }
  if (c->nfp > 0) TRY(field_dev(c, w, nbeta));
  CU(cudaEventRecord(c->ev[4], c->st));
  double* o = c->outbuf.p;
  if (amas) CU(cudaMemcpyAsync(amas, o, (size_t)ndof * ndof * 8, cudaMemcpyDeviceToHost, c->st));
  if (bdmp) CU(cudaMemcpyAsync(bdmp, o + (size_t)ndof * ndof, (size_t)ndof * ndof * 8, cudaMemcpyDeviceToHost, c->st));
  if (exfc && nbeta > 0)
    CU(cudaMemcpyAsync(exfc, o + 2 * (size_t)ndof * ndof, (size_t)ndof * nbeta * 16, cudaMemcpyDeviceToHost, c->st));
  int ovf = 0;
  CU(cudaMemcpyAsync(&ovf, c->ovf.p, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CU(cudaEventRecord(c->ev[5], c->st));
  CU(cudaStreamSynchronize(c->st));
  float ms;
  cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]); c->last_ms[0] = ms;
  cudaEventElapsedTime(&ms, c->ev[1], c->ev[2]); c->last_ms[1] = ms;
  cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]); c->last_ms[2] = ms;
  cudaEventElapsedTime(&ms, c->ev[3], c->ev[4]); c->last_ms[3] = ms;
  cudaEventElapsedTime(&ms, c->evc, c->ev[5]); c->last_ms[4] = ms;
  for (int b = 0; b < 4; ++b) {
    c->last_ms[5 + b] = 0.0;
    c->last_ms[11 + b] = (double)(c->bin_off[b + 1] - c->bin_off[b]);
    if (c->opts.depth >= 0.0 && cudaEventElapsedTime(&ms, c->evb[b], c->evb[b + 1]) == cudaSuccess) c->last_ms[5 + b] = ms;
  }
  if (cudaEventElapsedTime(&ms, c->ev[2], c->evf) == cudaSuccess) c->last_ms[9] = ms;
  c->last_ms[10] = (c->opts.precision == HAMS_PREC_MIXED || c->opts.solver == HAMS_SOLVER_GMRES)
                       ? (double)c->refine_sweeps : 0.0;
  c->last_ms[15] = c->opts.precision == HAMS_PREC_MIXED ? (double)c->lu_used : -1.0;
  c->last_ms[16] = 0.0;
  if (c->opts.depth >= 0.0 && cudaEventElapsedTime(&ms, c->evb[4], c->evb[5]) == cudaSuccess) c->last_ms[16] = ms;
  c->last_ms[17] = c->sg_used ? (double)(c->bin_off[6] - c->bin_off[4]) : 0.0;
  c->last_ms[18] = c->opts.precision == HAMS_PREC_MIXED ? c->ir_rate : 0.0;
  c->last_ms[19] = (double)c->blk_pairs;
  for (int k = 0; k < 8; ++k) c->last_ms[20 + k] = c->sg_judge[k];
  if (ovf & 2) return fail(HAMS_ERR_CUDA, "surrogate kernel: a tensor-core completion wait gave up");
  if (ovf) return fail(HAMS_ERR_NUMERIC, "adaptive quadrature stack overflow in the LINTON branch");
  if (info > 0) return info;  // singular pivot, LAPACK style
  return 0;
}

extern "C" int hams_solve_frequency(hams_ctx* c, const hams_wave* w, int32_t nbeta, const double* beta, double* amas,
                                    double* bdmp, double* exfc) {
  if (c) c->fp_batch.clear();
  g_err.clear();
  if (!c || !w || (nbeta > 0 && !beta)) return fail(HAMS_ERR_ARG, "null argument");
  if (cudaSetDevice(c->dev) != cudaSuccess) return fail(HAMS_ERR_CUDA, "cudaSetDevice failed");
  return solve_one(c, w, nbeta, beta, amas, bdmp, exfc);
}

// Frequencies in flight at once in hams_solve_batch when opts.batch_lanes is 0.
constexpr int kDefaultLanes = 8;

extern "C" int hams_solve_batch(hams_ctx* c, int32_t nfreq, const hams_wave* waves, int32_t nbeta, const double* beta,
                                double* amas, double* bdmp, double* exfc) {
  g_err.clear();
  if (!c || !waves || nfreq < 0 || (nbeta > 0 && !beta)) return fail(HAMS_ERR_ARG, "null argument");
  if (cudaSetDevice(c->dev) != cudaSuccess) return fail(HAMS_ERR_CUDA, "cudaSetDevice failed");
  if (nfreq == 0) return 0;
  const int ndof = 6 * c->nb;
  int L = c->opts.batch_lanes > 0 ? c->opts.batch_lanes : kDefaultLanes;
  L = std::max(1, std::min(L, nfreq));
  while ((int)c->lanes.size() < L - 1) {
    hams_ctx* l = nullptr;
    TRY(make_lane(c, &l));
    c->lanes.push_back(l);
  }
  std::vector<hams_ctx*> lane{c};
  for (int t = 0; t + 1 < L; ++t) lane.push_back(c->lanes[t]);
  std::vector<int> rc_of(nfreq, 0), lane_rc(L, 0);
  std::vector<std::string> lane_err(L), note_of(nfreq);
  c->fp_batch.assign(c->nfp > 0 ? nfreq : 0, std::vector<double>());
  // each lane takes the next unsolved frequency when it is free (frequencies
  // cost unevenly: out-of-range ones keep the series), on its own stream and
  // host thread; every result lands at its frequency's index
  std::atomic<int> next{0};
  auto run = [&](int t) {
    if (cudaSetDevice(c->dev) != cudaSuccess) {
      lane_rc[t] = HAMS_ERR_CUDA;
      lane_err[t] = "cudaSetDevice failed";
      return;
    }
    std::vector<double> a((size_t)ndof * ndof), b((size_t)ndof * ndof), x(2 * (size_t)ndof * std::max(nbeta, 1));
    for (int k = next.fetch_add(1); k < nfreq; k = next.fetch_add(1)) {
      int rc = solve_one(lane[t], &waves[k], nbeta, beta, a.data(), b.data(), x.data());
      if (rc < 0) {
        lane_rc[t] = rc;
        lane_err[t] = g_err;
        return;
      }
      rc_of[k] = rc;
      note_of[k] = lane[t]->note;
      if (c->nfp > 0) c->fp_batch[k] = lane[t]->fp_last;
      // scatter into (nfreq, ...) column-major arrays with the frequency index leading
      for (size_t e = 0; e < (size_t)ndof * ndof; ++e) {
        if (amas) amas[k + e * nfreq] = a[e];
        if (bdmp) bdmp[k + e * nfreq] = b[e];
      }
      if (exfc)
        for (size_t e = 0; e < (size_t)ndof * nbeta; ++e) {
          exfc[2 * (k + e * nfreq)] = x[2 * e];
          exfc[2 * (k + e * nfreq) + 1] = x[2 * e + 1];
        }
    }
  };
  std::vector<std::thread> th;
  for (int t = 1; t < L; ++t) th.emplace_back(run, t);
  run(0);
  for (auto& x : th) x.join();
  c->note.clear();  // the batch's note: each frequency's own, in order
  for (int k = 0; k < nfreq; ++k)
    if (!note_of[k].empty()) c->note += (c->note.empty() ? "" : "; ") + ("frequency " + std::to_string(k) + ": ") + note_of[k];
  for (int t = 0; t < L; ++t)
    if (lane_rc[t] < 0) {
      g_err = lane_err[t];
      return lane_rc[t];
    }
  for (int k = 0; k < nfreq; ++k)
    if (rc_of[k] > 0) return rc_of[k];  // singular pivot of the first such frequency
  return 0;
}

extern "C" int hams_assemble(hams_ctx* c, const hams_wave* w, int32_t nbeta, const double* beta, double* amat,
                             double* brmat, double* bdmat) {
  g_err.clear();
  if (!c || !w || (nbeta > 0 && !beta)) return fail(HAMS_ERR_ARG, "null argument");
  if (c->unfolded)
    return fail(HAMS_ERR_UNSUPPORTED, "hams_assemble: the context holds the unfolded mesh of a half-mesh deck");
  if (cudaSetDevice(c->dev) != cudaSuccess) return fail(HAMS_ERR_CUDA, "cudaSetDevice failed");
  const int n = c->n, tn = c->tn, ndof = 6 * c->nb, nrhs = ndof + nbeta;
  TRY(c->beta.alloc(std::max(nbeta, 1)));
  if (nbeta > 0) CU(cudaMemcpyAsync(c->beta.p, beta, (size_t)nbeta * 8, cudaMemcpyHostToDevice, c->st));
  TRY(assemble_dev(c, w, nbeta));
  const double2 *M = c->A.p, *R = c->B.p;
  int ldm = tn;
  if (c->nl > 0) {
    const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
    TRY(c->C.alloc((size_t)n * n));
    TRY(c->D.alloc((size_t)n * nrhs));
    CUB_(cublasZgemm(c->blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, tn, &one, (cuDoubleComplex*)c->A.p, tn,
                     (cuDoubleComplex*)c->A.p, tn, &zero, (cuDoubleComplex*)c->C.p, n));
    CUB_(cublasZgemm(c->blas, CUBLAS_OP_T, CUBLAS_OP_N, n, nrhs, tn, &one, (cuDoubleComplex*)c->A.p, tn,
                     (cuDoubleComplex*)c->B.p, tn, &zero, (cuDoubleComplex*)c->D.p, n));
    M = c->C.p;
    R = c->D.p;
    ldm = n;
  }
  if (amat) CU(cudaMemcpy2DAsync(amat, (size_t)n * 16, M, (size_t)ldm * 16, (size_t)n * 16, n, cudaMemcpyDeviceToHost, c->st));
  if (brmat)
    CU(cudaMemcpy2DAsync(brmat, (size_t)n * 16, R, (size_t)ldm * 16, (size_t)n * 16, ndof, cudaMemcpyDeviceToHost, c->st));
  if (bdmat && nbeta > 0)
    CU(cudaMemcpy2DAsync(bdmat, (size_t)n * 16, R + (size_t)ndof * ldm, (size_t)ldm * 16, (size_t)n * 16, nbeta,
                         cudaMemcpyDeviceToHost, c->st));
  CU(cudaStreamSynchronize(c->st));
  return 0;
}

extern "C" int hams_eval_green(hams_ctx* c, const hams_wave* w, int32_t npts, const double* pts, const int32_t* flag,
                               double* grn) {
  g_err.clear();
  if (!c || !w || npts < 0 || (npts > 0 && (!pts || !flag || !grn))) return fail(HAMS_ERR_ARG, "null argument");
  if (npts == 0) return 0;
  if (cudaSetDevice(c->dev) != cudaSuccess) return fail(HAMS_ERR_CUDA, "cudaSetDevice failed");
  DBuf<double> dp;
  DBuf<int> df;
  DBuf<double2> dout;
  TRY(dp.alloc(6 * (size_t)npts));
  TRY(df.alloc(npts));
  TRY(dout.alloc(4 * (size_t)npts));
  CU(cudaMemcpyAsync(dp.p, pts, 6 * (size_t)npts * 8, cudaMemcpyHostToDevice, c->st));
  CU(cudaMemcpyAsync(df.p, flag, (size_t)npts * 4, cudaMemcpyHostToDevice, c->st));
  WaveDev wd = wave_dev(c, w);
  if (c->opts.depth >= 0.0 && !wd.limit) CU(cudaMemcpyAsync(c->wvn.p, w->wvn, HAMS_NK * 8, cudaMemcpyHostToDevice, c->st));
  CU(cudaMemsetAsync(c->ovf.p, 0, sizeof(int), c->st));
  launch_eval_green((npts + 127) / 128, c->st, npts, dp.p, df.p, wd, c->wvn.p, dout.p, c->ovf.p);
  TRY(launch_check(c));
  CU(cudaMemcpyAsync(grn, dout.p, 4 * (size_t)npts * 16, cudaMemcpyDeviceToHost, c->st));
  int ovf = 0;
  CU(cudaMemcpyAsync(&ovf, c->ovf.p, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CU(cudaStreamSynchronize(c->st));
  dp.release();
  df.release();
  dout.release();
  if (ovf) return fail(HAMS_ERR_NUMERIC, "adaptive quadrature stack overflow in the LINTON branch");
  return 0;
}

// ---------------------------------------------------------------------------
// hams_eval_green_static: hams_eval_green without device allocation.  Its
// staging lives in one fixed reservation per device: the results (4 complex
// per point), the points (6 doubles), the flags, the overflow word and the
// frequency's wave numbers (so that the call touches none of the context's
// per-frequency buffers, which a solve on another stream may be using).
// ---------------------------------------------------------------------------
constexpr size_t kStaticPts = HAMS_EVAL_STATIC_MAX_POINTS;
constexpr size_t kStaticOutOff = 0;                                   // double2 (4 * kStaticPts)
constexpr size_t kStaticPtsOff = kStaticOutOff + 4 * kStaticPts * 16;  // double (6 * kStaticPts)
constexpr size_t kStaticFlagOff = kStaticPtsOff + 6 * kStaticPts * 8;  // int (kStaticPts)
constexpr size_t kStaticOvfOff = kStaticFlagOff + kStaticPts * 4;      // int
constexpr size_t kStaticWvnOff = (kStaticOvfOff + 4 + 7) / 8 * 8;      // double (HAMS_NK)
constexpr size_t kStaticBytes = (kStaticWvnOff + HAMS_NK * 8 + 255) / 256 * 256;
static __device__ __align__(256) unsigned char g_eval_static[kStaticBytes];

constexpr int kStaticMaxDevices = 64;
static std::mutex g_static_mu;
static unsigned char* g_static_addr[kStaticMaxDevices] = {};

// Address of the reservation on device `dev` (which must be current): looked
// up with cudaGetSymbolAddress on the first call for that device, then cached.
static int static_scratch(int dev, unsigned char** out) {
  if (dev < 0 || dev >= kStaticMaxDevices) return fail(HAMS_ERR_UNSUPPORTED, "device ordinal %d >= %d", dev, kStaticMaxDevices);
  std::lock_guard<std::mutex> lock(g_static_mu);
  if (!g_static_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_eval_static);
    if (e != cudaSuccess || !p) return fail(HAMS_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    g_static_addr[dev] = (unsigned char*)p;
  }
  *out = g_static_addr[dev];
  return 0;
}

extern "C" int hams_eval_green_static(hams_ctx* c, const hams_wave* w, int32_t npts, const double* pts,
                                      const int32_t* flag, double* grn) {
  g_err.clear();
  if (!c || !w || npts < 0 || (npts > 0 && (!pts || !flag || !grn))) return fail(HAMS_ERR_ARG, "null argument");
  if (npts > HAMS_EVAL_STATIC_MAX_POINTS)
    return fail(HAMS_ERR_ARG, "npts %d exceeds the static reservation of %d points", npts, HAMS_EVAL_STATIC_MAX_POINTS);
  if (npts == 0) return 0;
  if (cudaSetDevice(c->dev) != cudaSuccess) return fail(HAMS_ERR_CUDA, "cudaSetDevice failed");
  unsigned char* base = nullptr;
  TRY(static_scratch(c->dev, &base));
  double2* dout = (double2*)(base + kStaticOutOff);
  double* dp = (double*)(base + kStaticPtsOff);
  int* df = (int*)(base + kStaticFlagOff);
  int* dovf = (int*)(base + kStaticOvfOff);
  double* dwvn = (double*)(base + kStaticWvnOff);
  CU(cudaMemcpyAsync(dp, pts, 6 * (size_t)npts * 8, cudaMemcpyHostToDevice, c->st));
  CU(cudaMemcpyAsync(df, flag, (size_t)npts * 4, cudaMemcpyHostToDevice, c->st));
  WaveDev wd = wave_dev(c, w);
  if (c->opts.depth >= 0.0 && !wd.limit) CU(cudaMemcpyAsync(dwvn, w->wvn, HAMS_NK * 8, cudaMemcpyHostToDevice, c->st));
  CU(cudaMemsetAsync(dovf, 0, sizeof(int), c->st));  // the overflow word must start at zero
  launch_eval_green((npts + 127) / 128, c->st, npts, dp, df, wd, dwvn, dout, dovf);
  TRY(launch_check(c));
  CU(cudaMemcpyAsync(grn, dout, 4 * (size_t)npts * 16, cudaMemcpyDeviceToHost, c->st));
  int ovf = 0;
  CU(cudaMemcpyAsync(&ovf, dovf, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CU(cudaStreamSynchronize(c->st));
  if (ovf) return fail(HAMS_ERR_NUMERIC, "adaptive quadrature stack overflow in the LINTON branch");
  return 0;
}

extern "C" int hams_ctx_set_surrogate_range(hams_ctx* c, double kmin, double kmax) {
  g_err.clear();
  if (!c || c->is_lane) return fail(HAMS_ERR_ARG, "null context");
  if (!(kmin >= sg::kKmin && kmax <= sg::kKmax && kmin <= kmax))
    return fail(HAMS_ERR_ARG, "K range [%g, %g] is not inside the network's domain [%g, %g]", kmin, kmax, sg::kKmin,
                sg::kKmax);
  if (cudaSetDevice(c->dev) != cudaSuccess) return fail(HAMS_ERR_CUDA, "cudaSetDevice failed");
  for (hams_ctx* l : c->lanes) CU(cudaStreamSynchronize(l->st));
  CU(cudaStreamSynchronize(c->st));
  c->sg_kmin = kmin;
  c->sg_kmax = kmax;
  for (hams_ctx* l : c->lanes) {
    l->sg_kmin = kmin;
    l->sg_kmax = kmax;
  }
  return 0;
}

extern "C" int hams_ctx_set_surrogate_tolerance(hams_ctx* c, double tol) {
  g_err.clear();
  if (!c || c->is_lane) return fail(HAMS_ERR_ARG, "null context");
  if (!(tol >= 0.0)) return fail(HAMS_ERR_ARG, "tolerance must be >= 0");
  if (cudaSetDevice(c->dev) != cudaSuccess) return fail(HAMS_ERR_CUDA, "cudaSetDevice failed");
  for (hams_ctx* l : c->lanes) CU(cudaStreamSynchronize(l->st));
  CU(cudaStreamSynchronize(c->st));
  c->sg_tol = tol;
  for (hams_ctx* l : c->lanes) l->sg_tol = tol;
  return 0;
}

// The pairs the judgement samples: every stride-th pair of the surrogate's
// bins (sorted by series length, so the sample spans every length), about
// kJudgeSamples in all.
constexpr long long kJudgeSamples = 16384;
static int build_judge_samples(hams_ctx* c) {
  c->sg_ns4 = c->sg_ns5 = 0;
  const long long c4 = c->bin_off[5] - c->bin_off[4], c5 = c->bin_off[6] - c->bin_off[5];
  if (!c->sg_on || c4 + c5 <= 0) return 0;
  const long long stride = std::max(1LL, (c4 + c5) / kJudgeSamples);
  const long long n4 = (c4 + stride - 1) / stride, n5 = (c5 + stride - 1) / stride;
  TRY(c->sg_samp.alloc((size_t)std::max(n4 + n5, 1LL)));
  if (n4 > 0) k_stride_pick<<<(unsigned)((n4 + 255) / 256), 256, 0, c->st>>>(c->pairs.p + c->bin_off[4], n4, stride, c->sg_samp.p);
  if (n5 > 0)
    k_stride_pick<<<(unsigned)((n5 + 255) / 256), 256, 0, c->st>>>(c->pairs.p + c->bin_off[5], n5, stride,
                                                                 c->sg_samp.p + n4);
  TRY(launch_check(c, (n4 > 0) + (n5 > 0)));
  c->sg_ns4 = (int)n4;
  c->sg_ns5 = (int)n5;
  return 0;
}

extern "C" int hams_ctx_set_surrogate(hams_ctx* c, const float* params, int32_t nparams, double far_factor) {
  g_err.clear();
  if (!c || c->is_lane) return fail(HAMS_ERR_ARG, "null context");
  if (params && nparams != sg::kParams)
    return fail(HAMS_ERR_ARG, "surrogate parameter vector has %d floats, %d expected", nparams, sg::kParams);
  if (params && !(far_factor > 0.0)) return fail(HAMS_ERR_ARG, "far_factor must be positive");
  if (c->opts.depth < 0.0 && params) return fail(HAMS_ERR_UNSUPPORTED, "the surrogate covers finite depth only");
  if (cudaSetDevice(c->dev) != cudaSuccess) return fail(HAMS_ERR_CUDA, "cudaSetDevice failed");
  for (hams_ctx* l : c->lanes) CU(cudaStreamSynchronize(l->st));
  CU(cudaStreamSynchronize(c->st));
  if (params) {
    std::vector<__half> wh;
    std::vector<float> w0, bias;
    pack_surrogate(params, wh, w0, bias);
    TRY(c->sg_wh.alloc(wh.size()));
    TRY(c->sg_w0.alloc(w0.size()));
    TRY(c->sg_bias.alloc(bias.size()));
    CU(cudaMemcpy(c->sg_wh.p, wh.data(), wh.size() * 2, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(c->sg_w0.p, w0.data(), w0.size() * 4, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(c->sg_bias.p, bias.data(), bias.size() * 4, cudaMemcpyHostToDevice));
    c->sgd.wh = reinterpret_cast<const __half*>(c->sg_wh.p);
    c->sgd.w0 = c->sg_w0.p;
    c->sgd.bias = c->sg_bias.p;
    for (int k = 0; k < sg::kOut; ++k) {
      c->sgd.mean[k] = params[sg::kNormOff + k];
      c->sgd.scale[k] = params[sg::kNormOff + sg::kOut + k];
    }
    c->sg_on = 1;
    c->sg_far = far_factor;
  } else {
    c->sg_on = 0;
  }
  TRY(build_pairs(c));
  TRY(build_judge_samples(c));
  if (c->sg_on) {
    TRY(c->sg_map.alloc((size_t)c->tn * c->n));
    k_probe_map<<<dim3((c->tn + 127) / 128, c->n), 128, 0, c->st>>>(c->g, c->opts.depth, c->sg_far, c->sg_map.p);
    TRY(launch_check(c));
  }
  int nmode = c->mt.nmode;
  if (c->bin_off[3] > c->bin_off[2] || c->bin_off[5] > c->bin_off[4]) nmode = std::max(nmode, hams::kEigenEMax + 1);
  c->mt.nmode = nmode;
  for (hams_ctx* l : c->lanes) {
    for (int b = 0; b <= kBins; ++b) l->bin_off[b] = c->bin_off[b];
    l->pairs.view(c->pairs);
    l->sg_on = c->sg_on;
    l->sg_far = c->sg_far;
    l->sg_kmin = c->sg_kmin;
    l->sg_kmax = c->sg_kmax;
    l->sgd = c->sgd;
    l->sg_samp.view(c->sg_samp);
    l->sg_map.view(c->sg_map);
    l->sg_ns4 = c->sg_ns4;
    l->sg_ns5 = c->sg_ns5;
    l->mt.nmode = nmode;
  }
  return 0;
}

extern "C" int hams_last_timings(hams_ctx* c, double* ms, int32_t n) {
  if (!c || !ms) return 0;
  int k = std::min<int>(n, hams_ctx::kTimings);
  for (int i = 0; i < k; ++i) ms[i] = c->last_ms[i];
  return k;
}

extern "C" const char* hams_last_note(hams_ctx* c) { return c ? c->note.c_str() : ""; }

extern "C" int hams_ctx_set_field_points(hams_ctx* c, int32_t nfp, const double* xfp) {
  g_err.clear();
  if (!c || c->is_lane) return fail(HAMS_ERR_ARG, "null context");
  if (nfp < 0 || (nfp > 0 && !xfp)) return fail(HAMS_ERR_ARG, "bad field points");
  if (cudaSetDevice(c->dev) != cudaSuccess) return fail(HAMS_ERR_CUDA, "cudaSetDevice failed");
  for (hams_ctx* l : c->lanes) CU(cudaStreamSynchronize(l->st));
  CU(cudaStreamSynchronize(c->st));
  c->nfp = nfp;
  c->fp_last.clear();
  c->fp_batch.clear();
  if (nfp > 0) {
    // 2 pi for a point on a hull panel (in its plane and inside its edges),
    // 4 pi in the fluid (PressureElevationMulti.f90:203-252)
    const int n = c->n;
    std::vector<double> sld(nfp);
    for (int f = 0; f < nfp; ++f) {
      const double x[3] = {xfp[f], xfp[f + nfp], xfp[f + 2 * (size_t)nfp]};
      bool onbody = false;
      for (int j = 0; j < n && !onbody; ++j) {
        const double* e = &c->nrm_h[j];
        const double en[3] = {e[0], e[(size_t)n], e[2 * (size_t)n]};
        const double tolp = std::max(1e-6, 1e-3 * c->pnsz_h[j]), tola = 1e-3 * c->pnsz_h[j] * c->pnsz_h[j];
        const double* v0 = &c->vtx_h[(size_t)j * 12];
        const double dpln = (x[0] - v0[0]) * en[0] + (x[1] - v0[1]) * en[1] + (x[2] - v0[2]) * en[2];
        if (std::fabs(dpln) > tolp) continue;
        double smin = 1e30, smax = -1e30;
        const int nv = c->ncn_h[j];
        for (int k = 0; k < nv; ++k) {
          const double* a = &c->vtx_h[(size_t)j * 12 + 3 * k];
          const double* b = &c->vtx_h[(size_t)j * 12 + 3 * ((k + 1) % nv)];
          const double ev[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
          const double wv[3] = {x[0] - a[0], x[1] - a[1], x[2] - a[2]};
          const double sv = (ev[1] * wv[2] - ev[2] * wv[1]) * en[0] + (ev[2] * wv[0] - ev[0] * wv[2]) * en[1] +
                            (ev[0] * wv[1] - ev[1] * wv[0]) * en[2];
          smin = std::min(smin, sv);
          smax = std::max(smax, sv);
        }
        if (smin >= -tola || smax <= tola) onbody = true;
      }
      sld[f] = (onbody ? 2.0 : 4.0) * 3.141592653589793;
    }
    TRY(c->fp_x.alloc(3 * (size_t)nfp));
    TRY(c->fp_sld.alloc(nfp));
    CU(cudaMemcpy(c->fp_x.p, xfp, 3 * (size_t)nfp * 8, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(c->fp_sld.p, sld.data(), (size_t)nfp * 8, cudaMemcpyHostToDevice));
  }
  for (hams_ctx* l : c->lanes) {
    l->nfp = nfp;
    l->fp_last.clear();
    if (nfp > 0) {
      l->fp_x.view(c->fp_x);
      l->fp_sld.view(c->fp_sld);
    }
  }
  return 0;
}

extern "C" int hams_field_potentials(hams_ctx* c, int32_t k, double* pot) {
  g_err.clear();
  if (!c || !pot) return fail(HAMS_ERR_ARG, "null argument");
  const std::vector<double>* src = nullptr;
  if (!c->fp_batch.empty()) {
    if (k < 0 || k >= (int)c->fp_batch.size()) return fail(HAMS_ERR_ARG, "frequency %d not in the last batch", k);
    src = &c->fp_batch[k];
  } else {
    if (k != 0) return fail(HAMS_ERR_ARG, "frequency %d: the last solve was a single frequency", k);
    src = &c->fp_last;
  }
  if (src->empty()) return fail(HAMS_ERR_ARG, "no field potentials (no field points, or no solve since they were set)");
  std::memcpy(pot, src->data(), src->size() * 8);
  return 0;
}

extern "C" int64_t hams_launch_count(hams_ctx* c) {
  if (!c) return 0;
  long long t = c->launches.load();
  for (hams_ctx* l : c->lanes) t += l->launches.load();
  return (int64_t)t;
}

extern "C" int64_t hams_library_call_count(hams_ctx* c) {
  if (!c) return 0;
  long long t = c->lib_calls.load();
  for (hams_ctx* l : c->lanes) t += l->lib_calls.load();
  return (int64_t)t;
}

extern "C" int hams_mark(hams_ctx* c, int32_t slot) {
  if (!c || slot < 0 || slot >= 8) return fail(HAMS_ERR_ARG, "bad mark slot");
  CU(cudaEventRecord(c->marks[slot], c->st));
  return 0;
}

extern "C" int hams_mark_elapsed(hams_ctx* c, int32_t a, int32_t b, double* ms) {
  if (!c || !ms || a < 0 || a >= 8 || b < 0 || b >= 8) return fail(HAMS_ERR_ARG, "bad mark slot");
  CU(cudaEventSynchronize(c->marks[b]));
  float f = 0.0f;
  CU(cudaEventElapsedTime(&f, c->marks[a], c->marks[b]));
  *ms = f;
  return 0;
}

// Dependent-chain FP64 FMA throughput: each thread runs 8 independent chains.
__global__ void k_fp64_peak(double* out, int iters) {
  double a0 = threadIdx.x * 1e-9, a1 = a0 + 1e-9, a2 = a0 + 2e-9, a3 = a0 + 3e-9;
  double a4 = a0 + 4e-9, a5 = a0 + 5e-9, a6 = a0 + 6e-9, a7 = a0 + 7e-9;
  const double m = 0.999999999, c = 1e-12;
  for (int i = 0; i < iters; ++i) {
    a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
    a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
  }
  double s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == 12345.0) out[0] = s;  // keeps the chains live
}

extern "C" int hams_measure_fp64_peak(int32_t device, double* tflops) {
  g_err.clear();
  if (!tflops) return fail(HAMS_ERR_ARG, "null argument");
  CU(cudaSetDevice(device));
  int sms = 0;
  CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  DBuf<double> out;
  TRY(out.alloc(1));
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  const int iters = 1 << 16, threads = 256, blocks = sms * 8;
  k_fp64_peak<<<blocks, threads>>>(out.p, 1024);  // warm-up
  CU(cudaEventRecord(e0));
  k_fp64_peak<<<blocks, threads>>>(out.p, iters);
  CU(cudaEventRecord(e1));
  CU(cudaEventSynchronize(e1));
  float ms = 0.0f;
  CU(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *tflops = 2.0 * 8.0 * iters * (double)threads * blocks / (ms * 1e-3) / 1e12;
  return 0;
}

// ---------------------------------------------------------------------------
// Diagnostic: the block LU's tensor-core GEMM on host arrays
// ---------------------------------------------------------------------------
extern "C" int hams_diag_gemm_tf32(int32_t device, int32_t m, int32_t n, int32_t k, float alpha, const float* a,
                                   int32_t lda, const float* b, int32_t ldb, float beta, float* c, int32_t ldc,
                                   int32_t c_rowmajor, int32_t variant) {
  g_err.clear();
  if (m < 1 || n < 1 || k < 1 || !a || !b || !c || lda < k || ldb < k || (lda & 3) || (ldb & 3) ||
      ldc < (c_rowmajor ? n : m) || variant < -1 || variant > 2)
    return fail(HAMS_ERR_ARG, "bad GEMM arguments");
  if (cudaSetDevice(device) != cudaSuccess) return fail(HAMS_ERR_CUDA, "cudaSetDevice(%d) failed", device);
  const size_t na = (size_t)m * lda, nb = (size_t)n * ldb, nc = c_rowmajor ? (size_t)m * ldc : (size_t)n * ldc;
  DBuf<float> da, db, dc;
  DBuf<int> derr;
  TRY(da.alloc(na));
  TRY(db.alloc(nb));
  TRY(dc.alloc(nc));
  TRY(derr.alloc(1));
  CU(cudaMemcpy(da.p, a, na * 4, cudaMemcpyHostToDevice));
  CU(cudaMemcpy(db.p, b, nb * 4, cudaMemcpyHostToDevice));
  CU(cudaMemcpy(dc.p, c, nc * 4, cudaMemcpyHostToDevice));
  CU(cudaMemset(derr.p, 0, sizeof(int)));
  const int v = variant >= 0 ? variant : gemm_tf32_pick(m, n, k);
  if (gemm_tf32_variant(0, v, m, n, k, alpha, da.p, lda, db.p, ldb, beta, dc.p, ldc, c_rowmajor != 0, derr.p))
    return fail(HAMS_ERR_CUDA, "gemm_tf32 launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  int err = 0;
  CU(cudaMemcpy(&err, derr.p, sizeof(int), cudaMemcpyDeviceToHost));
  CU(cudaMemcpy(c, dc.p, nc * 4, cudaMemcpyDeviceToHost));
  if (err) return fail(HAMS_ERR_CUDA, "gemm_tf32: a pipeline wait gave up (%d)", err);
  return 0;
}

// Diagnostic: device time of the block LU's GEMM (variant as above) on
// device-resident operands of the given shape, mean of reps launches after
// one untimed launch.
extern "C" int hams_diag_gemm_tf32_time(int32_t device, int32_t variant, int32_t m, int32_t n, int32_t k,
                                        int32_t reps, double* ms) {
  g_err.clear();
  if (m < 1 || n < 1 || k < 1 || reps < 1 || !ms || variant < -1 || variant > 2)
    return fail(HAMS_ERR_ARG, "bad GEMM arguments");
  if (cudaSetDevice(device) != cudaSuccess) return fail(HAMS_ERR_CUDA, "cudaSetDevice(%d) failed", device);
  const int ld = (k + 3) / 4 * 4;
  DBuf<float> da, db, dc;
  DBuf<int> derr;
  TRY(da.alloc((size_t)m * ld));
  TRY(db.alloc((size_t)n * ld));
  TRY(dc.alloc((size_t)m * n));
  TRY(derr.alloc(1));
  CU(cudaMemset(da.p, 0, (size_t)m * ld * 4));
  CU(cudaMemset(db.p, 0, (size_t)n * ld * 4));
  CU(cudaMemset(dc.p, 0, (size_t)m * n * 4));
  CU(cudaMemset(derr.p, 0, sizeof(int)));
  const int v = variant >= 0 ? variant : gemm_tf32_pick(m, n, k);
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  int rc = gemm_tf32_variant(0, v, m, n, k, -1.0f, da.p, ld, db.p, ld, 1.0f, dc.p, m, false, derr.p);
  cudaEventRecord(e0, 0);
  for (int r = 0; r < reps && !rc; ++r)
    rc = gemm_tf32_variant(0, v, m, n, k, -1.0f, da.p, ld, db.p, ld, 1.0f, dc.p, m, false, derr.p);
  cudaEventRecord(e1, 0);
  cudaEventSynchronize(e1);
  float t = 0.0f;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int err = 0;
  CU(cudaMemcpy(&err, derr.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (rc || err) return fail(HAMS_ERR_CUDA, "gemm_tf32 failed (%d, %d)", rc, err);
  *ms = t / reps;
  return 0;
}
