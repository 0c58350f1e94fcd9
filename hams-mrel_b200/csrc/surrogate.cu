// surrogate.cu -- training and reference evaluation of the MLP surrogate of
// the finite-depth evanescent Green function (shape and scaling: surrogate.h).
//
// Samples come from the library's own FINGREEN3D series (EIGENE / EIGEN
// branches, green.cuh) at random (R/h, depths, K): K runs over a table of
// nslice values whose dispersion roots come from DISPERSION
// (WavDynSubs.f90:40-127, host_wave.cpp).  Training is plain minibatch Adam
// on the mean squared error of the normalised outputs, with hand-written
// FP32 kernels: a tiled GEMM for the forward pass and both backward
// products, the bias + SiLU epilogue and its derivative, the bias-gradient
// row sums and the Adam update.  The assembly uses the trained parameters in
// a tensor-core inference kernel (hams_gpu.cu); the FP32 forward pass here is
// the reference the tests and the training statistics use.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <random>
#include <string>
#include <vector>

#include "../../include/hams_gpu.h"
#include "host_wave.h"
#include "kernels.cuh"
#include "surrogate.h"

int hams_set_error(int code, const char* msg);  // hams_gpu.cu

namespace {

constexpr int kTab = 64;  // dispersion roots kept per K slice (EIGENE uses <= 50)

#define SG_CU(x)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (x);                                                                 \
    if (e_ != cudaSuccess) return hams_set_error(HAMS_ERR_CUDA, cudaGetErrorString(e_)); \
  } while (0)

template <class T>
struct Buf {
  T* p = nullptr;
  Buf() = default;
  Buf(const Buf&) = delete;
  ~Buf() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(size_t n) { return cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)); }
};

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double unif(unsigned long long& s) {
  s = mix64(s);
  return (double)(s >> 11) * (1.0 / 9007199254740992.0);
}

// One sample per thread: inputs (X, Zq, Zp, K) and targets (t0, t1, t2) in raw
// (n x 7, column-major), the FINGREEN3D series evaluated with h = 1.
__global__ void k_sg_samples(int n, unsigned long long seed, int nslice, const double* __restrict__ Ks,
                             const double* __restrict__ wvn_tab, double* raw, int* ovf) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned long long s = seed ^ (0x632be59bd9b4e019ull * (unsigned long long)(i + 1));
  const double X = sg::kXmin * exp(unif(s) * log(sg::kXmax / sg::kXmin));
  const double Zq = sg::kZmin + unif(s) * (sg::kZmax - sg::kZmin);
  const double Zp = sg::kZmin + unif(s) * (sg::kZmax - sg::kZmin);
  const int sl = min(nslice - 1, (int)(unif(s) * nslice));
  const double K = Ks[sl];
  const double* wvn = wvn_tab + (size_t)sl * kTab;
  const double zq = Zq - 1.0, zp = Zp - 1.0, wk = wvn[0];
  hams::InlineModes md{wvn, 1.0, K, Zq, Zp};
  hams::cplx fg[3], pr[3];
  int o = 0;
  if (hams::fin_branch(X, 1.0) == hams::kEigenE) {
    hams::SeriesScratchN<hams::kEigenEMax> sc;
    hams::eigene(X, zq, zp, wk, wvn, 1.0, fg, sc, md, &o);
  } else {
    hams::eigen(X, zq, zp, wk, wvn, 1.0, fg, md);
  }
  hams::prop_mode(X, Zq, Zp, wk, 1.0, pr);
  if (o) atomicOr(ovf, 1);
  raw[i] = X;
  raw[i + (size_t)n] = Zq;
  raw[i + 2 * (size_t)n] = Zp;
  raw[i + 3 * (size_t)n] = K;
  double rk[3];
  sg::rankine_parts(X, zq, zp, rk);
  raw[i + 4 * (size_t)n] = X * (fg[0].re - pr[0].re - rk[0]);
  raw[i + 5 * (size_t)n] = X * X * (fg[1].re - pr[1].re - rk[1]);
  raw[i + 6 * (size_t)n] = X * X * (fg[2].re - pr[2].re - rk[2]);
}

// network inputs (4 x n) and normalised targets (3 x n) from raw samples
__global__ void k_sg_prepare(int n, const double* __restrict__ raw, const double* __restrict__ norm, float* feats,
                             float* targ) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float f[sg::kIn];
  sg::features(raw[i], raw[i + (size_t)n], raw[i + 2 * (size_t)n], raw[i + 3 * (size_t)n], f);
  for (int k = 0; k < sg::kIn; ++k) feats[k + sg::kIn * (size_t)i] = f[k];
  if (targ)
    for (int k = 0; k < sg::kOut; ++k)
      targ[k + sg::kOut * (size_t)i] = (float)((raw[i + (4 + k) * (size_t)n] - norm[k]) / norm[sg::kOut + k]);
}

// C (M x N, ldc) = alpha op(A) op(B) + beta C, column-major, FP32.  With
// gridDim.z > 1 each z slice sums kchunk of the K range and adds alpha times
// its part to C atomically (C zeroed by the caller, beta unused).
template <bool TA, bool TB>
__global__ void __launch_bounds__(256) k_sgemm(int M, int N, int K, float alpha, const float* __restrict__ A, int lda,
                                               const float* __restrict__ B, int ldb, float beta, float* C, int ldc,
                                               int kchunk) {
  __shared__ float As[16][65];
  __shared__ float Bs[16][65];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int m0 = blockIdx.x * 64, n0 = blockIdx.y * 64;
  float acc[4][4];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
  const int kb = blockIdx.z * kchunk, ke = min(K, kb + kchunk);
  for (int k0 = kb; k0 < ke; k0 += 16) {
    for (int e = threadIdx.x; e < 1024; e += 256) {
      int mm, kk;
      if (!TA) { mm = e % 64; kk = e / 64; } else { kk = e % 16; mm = e / 16; }
      int m = m0 + mm, k = k0 + kk;
      float v = 0.0f;
      if (m < M && k < ke) v = TA ? A[k + (size_t)lda * m] : A[m + (size_t)lda * k];
      As[kk][mm] = v;
    }
    for (int e = threadIdx.x; e < 1024; e += 256) {
      int kk, nn;
      if (!TB) { kk = e % 16; nn = e / 16; } else { nn = e % 64; kk = e / 64; }
      int k = k0 + kk, c = n0 + nn;
      float v = 0.0f;
      if (k < ke && c < N) v = TB ? B[c + (size_t)ldb * k] : B[k + (size_t)ldb * c];
      Bs[kk][nn] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      float a[4], b[4];
      for (int i = 0; i < 4; ++i) a[i] = As[kk][tx + 16 * i];
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][ty + 16 * j];
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      int m = m0 + tx + 16 * i, c = n0 + ty + 16 * j;
      if (m < M && c < N) {
        float* p = C + m + (size_t)ldc * c;
        if (gridDim.z > 1) atomicAdd(p, alpha * acc[i][j]);
        else *p = alpha * acc[i][j] + (beta != 0.0f ? beta * *p : 0.0f);
      }
    }
}

__device__ __forceinline__ float sigm(float z) { return 1.0f / (1.0f + expf(-z)); }

// Z (rows x n) += b; H = silu(Z) (act) or Z
__global__ void k_bias_act(int rows, int n, float* Z, const float* __restrict__ b, float* H, int act) {
  size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)rows * n) return;
  int r = (int)(e % rows);
  float z = Z[e] + b[r];
  Z[e] = z;
  H[e] = act ? z * sigm(z) : z;
}

// dZ = dH * silu'(Z)
__global__ void k_silu_back(size_t cnt, const float* __restrict__ dH, const float* __restrict__ Z, float* dZ) {
  size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= cnt) return;
  float z = Z[e], s = sigm(z);
  dZ[e] = dH[e] * s * (1.0f + z * (1.0f - s));
}

// dY = 2 (Y - T) / (rows n); loss += sum (Y - T)^2 / (rows n)
__global__ void k_mse(size_t cnt, const float* __restrict__ Y, const float* __restrict__ T, float* dY, double* loss) {
  size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  float d = 0.0f;
  if (e < cnt) {
    d = Y[e] - T[e];
    dY[e] = 2.0f * d / (float)cnt;
  }
  float s = d * d;
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0 && s != 0.0f) atomicAdd(loss, (double)s / (double)cnt);
}

// db[r] = sum_c dZ[r + rows c]
__global__ void k_rowsum(int rows, int n, const float* __restrict__ dZ, float* db) {
  int r = blockIdx.x;
  float s = 0.0f;
  for (int c = threadIdx.x; c < n; c += blockDim.x) s += dZ[r + (size_t)rows * c];
  __shared__ float sh[256];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k; k >>= 1) {
    if (threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[r] = sh[0];
}

__global__ void k_adam(int n, float* p, const float* __restrict__ g, float* m, float* v, float lr, float b1, float b2,
                       float c1, float c2) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float gi = g[i];
  float mi = b1 * m[i] + (1.0f - b1) * gi, vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
}

inline unsigned nb(size_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// Split K when the output has few tiles (the weight gradients, K = batch).
template <bool TA, bool TB>
void gemm(cudaStream_t st, int M, int N, int K, float alpha, const float* A, int lda, const float* B, int ldb,
          float beta, float* C, int ldc) {
  const int tiles = ((M + 63) / 64) * ((N + 63) / 64);
  int splits = 1, chunk = K;
  if (tiles < 64 && K >= 1024) {
    splits = std::min((K + 511) / 512, 256);
    chunk = ((K + splits - 1) / splits + 15) / 16 * 16;
    splits = (K + chunk - 1) / chunk;
    if (ldc == M) cudaMemsetAsync(C, 0, (size_t)M * N * sizeof(float), st);
    else
      for (int c = 0; c < N; ++c) cudaMemsetAsync(C + (size_t)ldc * c, 0, (size_t)M * sizeof(float), st);
  }
  k_sgemm<TA, TB><<<dim3((M + 63) / 64, (N + 63) / 64, splits), 256, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C,
                                                                             ldc, chunk);
}

// Activations of one batch: Z_l, H_l (layer_out(l) x n) and their gradients.
struct Net {
  int cap = 0;
  Buf<float> Z[sg::kLayers], H[sg::kLayers], dH, dZ, dZ2;
  cudaError_t alloc(int n) {
    cap = n;
    cudaError_t e = cudaSuccess;
    for (int l = 0; l < sg::kLayers && e == cudaSuccess; ++l) {
      e = Z[l].alloc((size_t)sg::layer_out(l) * n);
      if (e == cudaSuccess) e = H[l].alloc((size_t)sg::layer_out(l) * n);
    }
    if (e == cudaSuccess) e = dH.alloc((size_t)sg::kWidth * n);
    if (e == cudaSuccess) e = dZ.alloc((size_t)sg::kWidth * n);
    if (e == cudaSuccess) e = dZ2.alloc((size_t)sg::kWidth * n);
    return e;
  }
  // outputs (normalised) in H[kLayers - 1]
  void forward(cudaStream_t st, const float* P, const float* X, int n) {
    const float* in = X;
    for (int l = 0; l < sg::kLayers; ++l) {
      const int fi = sg::layer_in(l), fo = sg::layer_out(l);
      gemm<false, false>(st, fo, n, fi, 1.0f, P + sg::w_off(l), fo, in, fi, 0.0f, Z[l].p, fo);
      k_bias_act<<<nb((size_t)fo * n), 256, 0, st>>>(fo, n, Z[l].p, P + sg::b_off(l), H[l].p, l < sg::kLayers - 1);
      in = H[l].p;
    }
  }
  // gradient G of the mean squared error against T (normalised targets)
  void backward(cudaStream_t st, const float* P, const float* X, const float* T, int n, float* G, double* loss) {
    const int L = sg::kLayers;
    float* dcur = dZ.p;  // dZ of the current layer
    k_mse<<<nb((size_t)sg::kOut * n), 256, 0, st>>>((size_t)sg::kOut * n, H[L - 1].p, T, dcur, loss);
    for (int l = L - 1; l >= 0; --l) {
      const int fi = sg::layer_in(l), fo = sg::layer_out(l);
      const float* hin = l ? H[l - 1].p : X;
      gemm<false, true>(st, fo, fi, n, 1.0f, dcur, fo, hin, fi, 0.0f, G + sg::w_off(l), fo);  // dW = dZ H^T
      k_rowsum<<<fo, 256, 0, st>>>(fo, n, dcur, G + sg::b_off(l));
      if (l == 0) break;
      gemm<true, false>(st, fi, n, fo, 1.0f, P + sg::w_off(l), fo, dcur, fo, 0.0f, dH.p, fi);  // dH = W^T dZ
      float* dnext = (dcur == dZ.p) ? dZ2.p : dZ.p;
      k_silu_back<<<nb((size_t)fi * n), 256, 0, st>>>((size_t)fi * n, dH.p, Z[l - 1].p, dnext);
      dcur = dnext;
    }
  }
};

struct Dev {
  int dev;
  bool ok;
  explicit Dev(int d) : dev(d), ok(cudaSetDevice(d) == cudaSuccess) {}
};

// K slices log-spaced over the domain and their dispersion roots (h = 1):
// DISPERSION's x = w^2 h / 9.807 is the slice's K.
void k_slices(int nslice, std::vector<double>& Ks, std::vector<double>& tab) {
  Ks.resize(nslice);
  tab.assign((size_t)nslice * kTab, 0.0);
  std::vector<double> w(HAMS_NK);
  for (int s = 0; s < nslice; ++s) {
    double K = sg::kKmin * std::exp((s + 0.5) / nslice * std::log(sg::kKmax / sg::kKmin));
    hams_dispersion(w.data(), kTab, std::sqrt(K * 9.807), 1.0);
    // the network's K is k0 h tanh(k0 h), the same as x up to the root's rounding
    Ks[s] = w[0] * std::tanh(w[0]);
    for (int k = 0; k < kTab; ++k) tab[(size_t)s * kTab + k] = w[k];
  }
}

int make_samples(int n, unsigned long long seed, int nslice, double* d_raw) {
  std::vector<double> Ks, tab;
  k_slices(nslice, Ks, tab);
  Buf<double> dK, dT;
  Buf<int> dovf;
  SG_CU(dK.alloc(Ks.size()));
  SG_CU(dT.alloc(tab.size()));
  SG_CU(dovf.alloc(1));
  SG_CU(cudaMemcpy(dK.p, Ks.data(), Ks.size() * 8, cudaMemcpyHostToDevice));
  SG_CU(cudaMemcpy(dT.p, tab.data(), tab.size() * 8, cudaMemcpyHostToDevice));
  SG_CU(cudaMemset(dovf.p, 0, 4));
  k_sg_samples<<<nb(n, 128), 128>>>(n, seed, nslice, dK.p, dT.p, d_raw, dovf.p);
  SG_CU(cudaGetLastError());
  int ovf = 0;
  SG_CU(cudaMemcpy(&ovf, dovf.p, 4, cudaMemcpyDeviceToHost));
  if (ovf) return hams_set_error(HAMS_ERR_NUMERIC, "surrogate samples: series longer than its table");
  return 0;
}

}  // namespace

extern "C" int32_t hams_surrogate_param_count(void) { return sg::kParams; }

extern "C" int hams_surrogate_samples(int32_t device, int32_t n, uint64_t seed, int32_t nslice, double* raw) {
  if (n <= 0 || nslice <= 0 || !raw) return hams_set_error(HAMS_ERR_ARG, "bad surrogate sample request");
  Dev d(device);
  if (!d.ok) return hams_set_error(HAMS_ERR_CUDA, "cudaSetDevice failed");
  Buf<double> draw;
  SG_CU(draw.alloc((size_t)7 * n));
  int rc = make_samples(n, seed, nslice, draw.p);
  if (rc) return rc;
  SG_CU(cudaMemcpy(raw, draw.p, (size_t)7 * n * 8, cudaMemcpyDeviceToHost));
  return 0;
}

extern "C" int hams_surrogate_eval(int32_t device, const float* params, int32_t n, const double* x, double* t) {
  if (!params || n <= 0 || !x || !t) return hams_set_error(HAMS_ERR_ARG, "bad surrogate evaluation request");
  Dev d(device);
  if (!d.ok) return hams_set_error(HAMS_ERR_CUDA, "cudaSetDevice failed");
  std::vector<double> raw((size_t)7 * n, 0.0);
  std::copy(x, x + (size_t)4 * n, raw.begin());
  Buf<double> draw, dnorm;
  Buf<float> dP, dF;
  SG_CU(draw.alloc(raw.size()));
  SG_CU(dnorm.alloc(2 * sg::kOut));
  SG_CU(dP.alloc(sg::kParams));
  SG_CU(dF.alloc((size_t)sg::kIn * n));
  std::vector<double> norm(2 * sg::kOut);
  for (int k = 0; k < 2 * sg::kOut; ++k) norm[k] = params[sg::kNormOff + k];
  SG_CU(cudaMemcpy(draw.p, raw.data(), raw.size() * 8, cudaMemcpyHostToDevice));
  SG_CU(cudaMemcpy(dnorm.p, norm.data(), norm.size() * 8, cudaMemcpyHostToDevice));
  SG_CU(cudaMemcpy(dP.p, params, sg::kParams * 4, cudaMemcpyHostToDevice));
  k_sg_prepare<<<nb(n), 256>>>(n, draw.p, dnorm.p, dF.p, nullptr);
  Net net;
  SG_CU(net.alloc(n));
  net.forward(0, dP.p, dF.p, n);
  SG_CU(cudaGetLastError());
  std::vector<float> y((size_t)sg::kOut * n);
  SG_CU(cudaMemcpy(y.data(), net.H[sg::kLayers - 1].p, y.size() * 4, cudaMemcpyDeviceToHost));
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < sg::kOut; ++k)
      t[i + (size_t)k * n] = norm[k] + norm[sg::kOut + k] * (double)y[k + (size_t)sg::kOut * i];
  return 0;
}

extern "C" int hams_surrogate_grad(int32_t device, const float* params, int32_t n, const float* feats,
                                   const float* targ, double* loss, float* grad) {
  if (!params || n <= 0 || !feats || !targ || !loss || !grad)
    return hams_set_error(HAMS_ERR_ARG, "bad surrogate gradient request");
  Dev d(device);
  if (!d.ok) return hams_set_error(HAMS_ERR_CUDA, "cudaSetDevice failed");
  Buf<float> dP, dF, dT, dG;
  Buf<double> dl;
  SG_CU(dP.alloc(sg::kParams));
  SG_CU(dF.alloc((size_t)sg::kIn * n));
  SG_CU(dT.alloc((size_t)sg::kOut * n));
  SG_CU(dG.alloc(sg::kParams));
  SG_CU(dl.alloc(1));
  SG_CU(cudaMemcpy(dP.p, params, sg::kParams * 4, cudaMemcpyHostToDevice));
  SG_CU(cudaMemcpy(dF.p, feats, (size_t)sg::kIn * n * 4, cudaMemcpyHostToDevice));
  SG_CU(cudaMemcpy(dT.p, targ, (size_t)sg::kOut * n * 4, cudaMemcpyHostToDevice));
  SG_CU(cudaMemset(dG.p, 0, sg::kParams * 4));
  SG_CU(cudaMemset(dl.p, 0, 8));
  Net net;
  SG_CU(net.alloc(n));
  net.forward(0, dP.p, dF.p, n);
  net.backward(0, dP.p, dF.p, dT.p, n, dG.p, dl.p);
  SG_CU(cudaGetLastError());
  SG_CU(cudaMemcpy(grad, dG.p, sg::kParams * 4, cudaMemcpyDeviceToHost));
  SG_CU(cudaMemcpy(loss, dl.p, 8, cudaMemcpyDeviceToHost));
  return 0;
}

extern "C" int hams_surrogate_train(int32_t device, const hams_sg_train* cfg, float* params, double* stats) {
  if (!cfg || !params || cfg->n_train <= 0 || cfg->n_test <= 0 || cfg->batch <= 0 || cfg->steps <= 0 ||
      cfg->nslice <= 0 || cfg->batch > cfg->n_train)
    return hams_set_error(HAMS_ERR_ARG, "bad surrogate training configuration");
  Dev d(device);
  if (!d.ok) return hams_set_error(HAMS_ERR_CUDA, "cudaSetDevice failed");
  auto t0 = std::chrono::steady_clock::now();
  const int ntr = cfg->n_train, nte = cfg->n_test, B = cfg->batch, ntot = ntr + nte;
  Buf<double> draw, dnorm;
  SG_CU(draw.alloc((size_t)7 * ntot));
  int rc = make_samples(ntot, cfg->seed, cfg->nslice, draw.p);
  if (rc) return rc;
  // output normalisation from the training samples
  std::vector<double> raw((size_t)7 * ntot);
  SG_CU(cudaMemcpy(raw.data(), draw.p, raw.size() * 8, cudaMemcpyDeviceToHost));
  auto t1 = std::chrono::steady_clock::now();
  std::vector<double> norm(2 * sg::kOut);
  for (int k = 0; k < sg::kOut; ++k) {
    double s = 0.0, s2 = 0.0;
    for (int i = 0; i < ntr; ++i) {
      double v = raw[i + (size_t)(4 + k) * ntot];
      s += v;
      s2 += v * v;
    }
    double mean = s / ntr, var = std::max(s2 / ntr - mean * mean, 1e-30);
    norm[k] = (double)(float)mean;  // stored with the parameters as floats
    norm[sg::kOut + k] = (double)(float)std::sqrt(var);
  }
  SG_CU(dnorm.alloc(norm.size()));
  SG_CU(cudaMemcpy(dnorm.p, norm.data(), norm.size() * 8, cudaMemcpyHostToDevice));
  Buf<float> dF, dT;
  SG_CU(dF.alloc((size_t)sg::kIn * ntot));
  SG_CU(dT.alloc((size_t)sg::kOut * ntot));
  k_sg_prepare<<<nb(ntot), 256>>>(ntot, draw.p, dnorm.p, dF.p, dT.p);
  // initial parameters: uniform(+-sqrt(6 / (fan_in + fan_out))), zero biases
  std::vector<float> P(sg::kParams, 0.0f);
  std::mt19937_64 gen(cfg->seed ^ 0x5bd1e995ull);
  for (int l = 0; l < sg::kLayers; ++l) {
    const int fi = sg::layer_in(l), fo = sg::layer_out(l);
    std::uniform_real_distribution<float> u(-std::sqrt(6.0f / (fi + fo)), std::sqrt(6.0f / (fi + fo)));
    for (int e = 0; e < fi * fo; ++e) P[sg::w_off(l) + e] = u(gen);
  }
  for (int k = 0; k < 2 * sg::kOut; ++k) P[sg::kNormOff + k] = (float)norm[k];
  Buf<float> dP, dG, dm, dv;
  Buf<double> dl;
  SG_CU(dP.alloc(sg::kParams));
  SG_CU(dG.alloc(sg::kParams));
  SG_CU(dm.alloc(sg::kParams));
  SG_CU(dv.alloc(sg::kParams));
  SG_CU(dl.alloc(1));
  SG_CU(cudaMemcpy(dP.p, P.data(), sg::kParams * 4, cudaMemcpyHostToDevice));
  SG_CU(cudaMemset(dm.p, 0, sg::kParams * 4));
  SG_CU(cudaMemset(dv.p, 0, sg::kParams * 4));
  SG_CU(cudaMemset(dl.p, 0, 8));
  Net net;
  SG_CU(net.alloc(std::max(B, nte)));
  const int nw = sg::kNormOff;  // trained parameters (the normalisation stays fixed)
  const int nbatch = ntr / B, warm = std::min(500, cfg->steps / 10 + 1);
  const float b1 = 0.9f, b2 = 0.999f;
  double last = 0.0;
  for (int it = 0; it < cfg->steps; ++it) {
    const int bi = it % nbatch, ep = it / nbatch;
    const size_t off = ((size_t)bi * B + (size_t)ep * 977 * 13) % (size_t)(ntr - B + 1);
    const float* X = dF.p + off * sg::kIn;
    const float* T = dT.p + off * sg::kOut;
    net.forward(0, dP.p, X, B);
    net.backward(0, dP.p, X, T, B, dG.p, dl.p);
    double frac = (double)it / cfg->steps;
    double lr = cfg->lr * (it < warm ? (it + 1.0) / warm : 0.5 * (1.0 + std::cos(3.141592653589793 * frac)) * 0.999 + 0.001);
    float c1 = 1.0f - std::pow(b1, (float)(it + 1)), c2 = 1.0f - std::pow(b2, (float)(it + 1));
    k_adam<<<nb(nw), 256>>>(nw, dP.p, dG.p, dm.p, dv.p, (float)lr, b1, b2, c1, c2);
    if ((it + 1) % 1000 == 0 || it + 1 == cfg->steps) {
      double l = 0.0;
      SG_CU(cudaMemcpy(&l, dl.p, 8, cudaMemcpyDeviceToHost));
      SG_CU(cudaMemset(dl.p, 0, 8));
      last = l / ((it % 1000) + 1);
    }
  }
  SG_CU(cudaGetLastError());
  SG_CU(cudaMemcpy(params, dP.p, sg::kParams * 4, cudaMemcpyDeviceToHost));
  auto t2 = std::chrono::steady_clock::now();
  // held-out error of the trained network, in target units
  net.forward(0, dP.p, dF.p + (size_t)ntr * sg::kIn, nte);
  std::vector<float> y((size_t)sg::kOut * nte);
  SG_CU(cudaMemcpy(y.data(), net.H[sg::kLayers - 1].p, y.size() * 4, cudaMemcpyDeviceToHost));
  if (stats) {
    for (int k = 0; k < sg::kOut; ++k) {
      double se = 0.0, st = 0.0, me = 0.0, mt = 0.0;
      for (int i = 0; i < nte; ++i) {
        double tv = raw[ntr + i + (size_t)(4 + k) * ntot];
        double pv = norm[k] + norm[sg::kOut + k] * (double)y[k + (size_t)sg::kOut * i];
        se += (pv - tv) * (pv - tv);
        st += tv * tv;
        me = std::max(me, std::fabs(pv - tv));
        mt = std::max(mt, std::fabs(tv));
      }
      stats[k] = std::sqrt(se / st);
      stats[3 + k] = me / mt;
    }
    stats[6] = last;
    stats[7] = std::chrono::duration<double, std::milli>(t2 - t1).count();
    stats[8] = std::chrono::duration<double, std::milli>(t1 - t0).count();
  }
  return 0;
}
