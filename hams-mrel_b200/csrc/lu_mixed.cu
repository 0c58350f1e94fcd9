// lu_mixed.cu -- complex64 LU of the influence matrix for the mixed form.
//
// The mixed form factors a complex64 copy of A and recovers FP64 accuracy
// by iterative refinement against the FP64 matrix (hams_gpu.cu: mixed_solve),
// which replaces ZGETRF/ZGETRS of RADIATION_SOLVER_MULTI /
// DIFFRACTION_SOLVER_MULTI (AssbMatxMulti.f90:112,279,346) there.  The
// factorisation only has to be a good preconditioner, so it is organised for
// the tensor cores instead of following LAPACK's pivot order:
//
//   for each panel of kPB = 4 diagonal blocks (256 columns):
//     for each diagonal block k (kNB = 64 rows) of the panel:
//       k_diag_lu    one CTA factors A_kk = P_k^T L_kk U_kk in shared memory
//                    with partial pivoting inside the block, and forms
//                    L_kk^-1 and U_kk^-1;
//       k_apply_perm applies P_k to the rest of block row k;
//       GEMM         L_ik = A_ik U_kk^-1 below the block, U_kj = L_kk^-1 A_kj
//                    and A_ij -= L_ik U_kj for the panel's columns only;
//     GEMM           the panel's U rows for the columns right of it, by
//                    block forward substitution with the L_kk^-1;
//     GEMM           A_tt -= L_t,panel U_panel,t, one rank-256 trailing
//                    update per panel (the trailing matrix is read and
//                    written once per 256 columns instead of once per 64).
//
// The complex products run as real GEMMs on the real expansions of the
// complex matrices (cuBLAS, tensor cores, FP32 accumulation; inputs rounded
// to TF32, or FP32 emulated on BF16 tensor cores).  Pivoting is local to
// each diagonal block (P is block diagonal); the FP64 refinement checks the
// result, and the caller falls back to a partially pivoted LU if the
// refinement does not converge.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "lu_mixed.h"

namespace {

constexpr int kNB = 64;
constexpr int kPB = 4;   // diagonal blocks per panel: the trailing update runs once per kPB kNB columns
constexpr int kLd = kNB + 1;  // padded shared-memory leading dimension

// Real expansion of complex matrices.  A complex p x q matrix X becomes the
// real 2p x 2q matrix X^ with the 2 x 2 block [[xr, -xi], [xi, xr]] in place
// of each entry; a complex q x r matrix B stored interleaved (column-major
// float2) is, viewed as floats, the real 2q x r matrix with rows re, im.
// Then (X B) viewed as floats = X^ B_real and (X Y)^ = X^ Y^, so every
// complex product of the factorisation is one real GEMM on tensor cores.
__device__ __forceinline__ void put_expanded(float* E, int lde, int i, int k, float2 x) {
  E[(size_t)(2 * k) * lde + 2 * i] = x.x;
  E[(size_t)(2 * k) * lde + 2 * i + 1] = x.y;
  E[(size_t)(2 * k + 1) * lde + 2 * i] = -x.y;
  E[(size_t)(2 * k + 1) * lde + 2 * i + 1] = x.x;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ float2 cmac(float2 s, float2 a, float2 b) {
  return make_float2(s.x + a.x * b.x - a.y * b.y, s.y + a.x * b.y + a.y * b.x);
}

// Inverse of the unit lower (lower) or the upper triangle of T (kNB x kNB,
// ld kLd) into X: the 8 x 8 diagonal blocks by substitution, then three
// doubling levels X21 = -X22 (L21 X11) (lower) or X12 = -X11 (U12 X22)
// (upper), each product spread over the block's 256 threads; W holds the
// inner products of one level (at most 32 columns).
__device__ void tri_inverse(const float2* T, float2* X, float2* W, bool lower) {
  const int tid = threadIdx.x;
  for (int e = tid; e < kNB * kNB; e += 256) X[(e / kNB) * kLd + e % kNB] = make_float2(0.0f, 0.0f);
  __syncthreads();
  if (tid < kNB) {
    const int c = tid, b0 = c & ~7;
    if (lower) {
      X[c * kLd + c] = make_float2(1.0f, 0.0f);
      for (int i = c + 1; i < b0 + 8; ++i) {
        float2 acc = make_float2(0.0f, 0.0f);
        for (int k = c; k < i; ++k) acc = cmac(acc, T[k * kLd + i], X[c * kLd + k]);
        X[c * kLd + i] = make_float2(-acc.x, -acc.y);
      }
    } else {
      for (int i = c; i >= b0; --i) {
        float2 acc = make_float2(i == c ? 1.0f : 0.0f, 0.0f);
        for (int k = i + 1; k <= c; ++k) {
          float2 t = cmac(make_float2(0.0f, 0.0f), T[k * kLd + i], X[c * kLd + k]);
          acc.x -= t.x;
          acc.y -= t.y;
        }
        const float2 d = T[i * kLd + i];
        const float dd = d.x * d.x + d.y * d.y;
        X[c * kLd + i] = dd > 0.0f ? make_float2((acc.x * d.x + acc.y * d.y) / dd, (acc.y * d.x - acc.x * d.y) / dd)
                                   : make_float2(0.0f, 0.0f);
      }
    }
  }
  __syncthreads();
  for (int sz = 8; sz < kNB; sz *= 2) {
    const int tot = (kNB / (2 * sz)) * sz * sz;
    for (int e = tid; e < tot; e += 256) {
      const int q = e / (sz * sz), rem = e % (sz * sz), c = rem / sz, i = rem % sz, b0 = 2 * sz * q;
      float2 acc = make_float2(0.0f, 0.0f);
      if (lower)  // W = L21 X11
        for (int k = c; k < sz; ++k) acc = cmac(acc, T[(b0 + k) * kLd + b0 + sz + i], X[(b0 + c) * kLd + b0 + k]);
      else  // W = U12 X22
        for (int k = 0; k <= c; ++k) acc = cmac(acc, T[(b0 + sz + k) * kLd + b0 + i], X[(b0 + sz + c) * kLd + b0 + sz + k]);
      W[(q * sz + c) * kLd + i] = acc;
    }
    __syncthreads();
    for (int e = tid; e < tot; e += 256) {
      const int q = e / (sz * sz), rem = e % (sz * sz), c = rem / sz, i = rem % sz, b0 = 2 * sz * q;
      float2 acc = make_float2(0.0f, 0.0f);
      if (lower) {  // X21 = -X22 W
        for (int k = 0; k <= i; ++k) acc = cmac(acc, X[(b0 + sz + k) * kLd + b0 + sz + i], W[(q * sz + c) * kLd + k]);
        X[(b0 + c) * kLd + b0 + sz + i] = make_float2(-acc.x, -acc.y);
      } else {  // X12 = -X11 W
        for (int k = i; k < sz; ++k) acc = cmac(acc, X[(b0 + k) * kLd + b0 + i], W[(q * sz + c) * kLd + k]);
        X[(b0 + sz + c) * kLd + b0 + i] = make_float2(-acc.x, -acc.y);
      }
    }
    __syncthreads();
  }
}

// One CTA of 256 threads: LU with partial pivoting of the nbk x nbk
// diagonal block at (k0, k0), written back in place (unit L below, U on and
// above the diagonal); the block's row permutation as global source rows in
// perm; the expansions of L^-1 and U^-1 (2nbk x 2nbk, ld 2 kNB) in invL,
// invU.  info gets 1 + the first global column whose pivot is zero.  A
// partial last block is padded with the identity to kNB.
__global__ void __launch_bounds__(256) k_diag_lu(float2* A, int lda, int k0, int nbk, int* perm, float* invL,
                                                 float* invU, int* info) {
  extern __shared__ float2 sm[];
  float2* T = sm;                  // [col * kLd + row]
  float2* X = sm + kNB * kLd;      // L^-1
  float2* Y = sm + 2 * kNB * kLd;  // U^-1
  float2* W = sm + 3 * kNB * kLd;  // inversion scratch (32 columns)
  __shared__ int piv[kNB];
  __shared__ int prm[kNB];
  const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
  for (int e = tid; e < kNB * kNB; e += 256) {
    int r = e % kNB, c = e / kNB;
    T[c * kLd + r] = (r < nbk && c < nbk) ? A[(size_t)(k0 + c) * lda + k0 + r]
                                          : make_float2(r == c ? 1.0f : 0.0f, 0.0f);
  }
  __syncthreads();
  for (int j = 0; j < nbk; ++j) {
    if (tid < 32) {
      float best = -1.0f;
      int bi = j;
      for (int r = j + tid; r < nbk; r += 32) {
        float2 v = T[j * kLd + r];
        float a = fabsf(v.x) + fabsf(v.y);
        if (a > best) {
          best = a;
          bi = r;
        }
      }
      for (int o = 16; o; o >>= 1) {
        float ob = __shfl_xor_sync(0xffffffffu, best, o);
        int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      if (tid == 0) {
        piv[j] = bi;
        if (!(best > 0.0f)) atomicMin(info, k0 + j + 1);
      }
    }
    __syncthreads();
    // row swap j <-> p and the multipliers of column j in one pass, from the
    // values before the swap: thread t swaps column t (t != j) and scales
    // row t of column j (t > j, t != p); thread j handles rows j and p of
    // column j
    {
      const int p = piv[j];
      const float2 d = T[j * kLd + p];  // the pivot
      const float dd = d.x * d.x + d.y * d.y;
      const float2 rcp = dd > 0.0f ? make_float2(d.x / dd, -d.y / dd) : make_float2(0.0f, 0.0f);
      if (tid < nbk) {
        if (tid != j) {
          if (p != j) {
            float2 t = T[tid * kLd + j];
            T[tid * kLd + j] = T[tid * kLd + p];
            T[tid * kLd + p] = t;
          }
          if (tid > j && tid != p && dd > 0.0f) T[j * kLd + tid] = cmul(T[j * kLd + tid], rcp);
        } else {
          const float2 old = T[j * kLd + j];
          T[j * kLd + j] = d;
          if (p != j) T[j * kLd + p] = dd > 0.0f ? cmul(old, rcp) : old;
        }
      }
    }
    __syncthreads();
    // rank-1 update: tx walks rows (consecutive in shared memory), ty columns
    for (int c = j + 1 + ty; c < nbk; c += 16) {
      float2 u = T[c * kLd + j];
      for (int r = j + 1 + tx; r < nbk; r += 16) {
        float2 l = T[j * kLd + r], t = T[c * kLd + r];
        T[c * kLd + r] = make_float2(t.x - (l.x * u.x - l.y * u.y), t.y - (l.x * u.y + l.y * u.x));
      }
    }
    __syncthreads();
  }
  if (tid == 0) {  // the block permutation: the same swaps applied to row indices
    for (int i = 0; i < nbk; ++i) prm[i] = i;
    for (int j = 0; j < nbk; ++j) {
      int t = prm[j];
      prm[j] = prm[piv[j]];
      prm[piv[j]] = t;
    }
  }
  tri_inverse(T, X, W, true);
  tri_inverse(T, Y, W, false);
  for (int e = tid; e < nbk * nbk; e += 256) {
    int r = e % nbk, c = e / nbk;
    A[(size_t)(k0 + c) * lda + k0 + r] = T[c * kLd + r];
    put_expanded(invL, 2 * kNB, r, c, X[c * kLd + r]);
    put_expanded(invU, 2 * kNB, r, c, Y[c * kLd + r]);
  }
  for (int i = tid; i < nbk; i += 256) perm[k0 + i] = k0 + prm[i];
}

// E (2w x 2nbk, ld 2w) <- expansion of the w x nbk column panel at (k1, k0).
__global__ void k_expand_panel(const float2* __restrict__ A, int lda, int k1, int k0, int w, int nbk, float* E) {
  size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)w * nbk) return;
  int i = (int)(e % w), k = (int)(e / w);
  put_expanded(E, 2 * w, i, k, A[(size_t)(k0 + k) * lda + k1 + i]);
}

// Rows k0..k0+nbk-1 of every column outside the diagonal block take the
// block's permutation: row k0+i receives old row perm[k0+i].
__global__ void k_apply_perm(float2* A, int lda, int n, int k0, int nbk, const int* __restrict__ perm) {
  __shared__ float2 tile[kNB][33];
  const int c0 = blockIdx.x * 32, tx = threadIdx.x % 32, ty = threadIdx.x / 32;  // 256 threads: 8 x 32
  const int c = c0 + tx;
  const bool live = c < n && (c < k0 || c >= k0 + nbk);
  for (int i = ty; i < nbk; i += 8)
    if (live) tile[i][tx] = A[(size_t)c * lda + perm[k0 + i]];
  __syncthreads();
  for (int i = ty; i < nbk; i += 8)
    if (live) A[(size_t)c * lda + k0 + i] = tile[i][tx];
}

// X (n x nrhs, ld n) <- rows gathered by perm.
__global__ void k_gather_rows(const float2* __restrict__ src, float2* __restrict__ dst, int n, int nrhs,
                              const int* __restrict__ perm) {
  size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)n * nrhs) return;
  int r = (int)(e % n);
  size_t c = e / n;
  dst[e] = src[c * n + perm[r]];
}

cublasStatus_t sgemm(cublasHandle_t h, cublasComputeType_t ct, int m, int n, int k, float alpha, const float* A,
                     int lda, const float* B, int ldb, float beta, float* C, int ldc) {
  return cublasGemmEx(h, CUBLAS_OP_N, CUBLAS_OP_N, m, n, k, &alpha, A, CUDA_R_32F, lda, B, CUDA_R_32F, ldb, &beta, C,
                      CUDA_R_32F, ldc, ct, CUBLAS_GEMM_DEFAULT);
}

}  // namespace

// Workspace (floats): U rows W1 (2kNB x n), expanded L column of a block and
// its source (2 x 2n x 2kNB), the expanded inverses of a panel's diagonal
// blocks (2 x kPB x 2kNB x 2kNB), the expanded L rows of a block left of it
// in its panel (2kNB x 2kNB (kPB - 1)) and the expanded L columns of a whole
// panel (2n x 2kNB kPB).
size_t mixed_lu_workspace_elems(int n) {
  const size_t K2 = 2 * kNB;
  return (K2 * n + 2 * (2 * (size_t)n * K2) + 2 * kPB * K2 * K2 + K2 * K2 * (kPB - 1) + 2 * (size_t)n * K2 * kPB) / 2 +
         1;
}

int mixed_lu_factor(cudaStream_t st, cublasHandle_t blas, cublasComputeType_t ct, int n, float2* A, int* perm,
                    float2* work, int* dinfo, long long* launches, long long* lib_calls) {
  const int smem = (3 * kNB + 32) * kLd * (int)sizeof(float2);
  if (cudaFuncSetAttribute(k_diag_lu, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) return 1;
  const int K2 = 2 * kNB, PW = kPB * kNB;
  float* W1 = (float*)work;                     // U rows, real 2nbk x w (ld 2kNB)
  float* Ehat = W1 + (size_t)K2 * n;            // expanded A_ik, 2w x 2nbk (ld 2w)
  float* Lhat = Ehat + (size_t)2 * n * K2;      // expanded L_ik, 2w x 2nbk (ld 2w)
  float* invL = Lhat + (size_t)2 * n * K2;      // kPB x (2nbk x 2nbk, ld 2kNB)
  float* invU = invL + (size_t)kPB * K2 * K2;
  float* E2 = invU + (size_t)kPB * K2 * K2;     // expanded L rows left of a block, 2nbk x 2(k0 - p0) (ld 2nbk)
  float* Ebig = E2 + (size_t)K2 * K2 * (kPB - 1);  // expanded L columns of a panel, 2wt x 2(p1 - p0) (ld 2wt)
  if (cudaMemsetAsync(dinfo, 0x7f, sizeof(int), st) != cudaSuccess) return 1;  // large positive: no zero pivot
  if (cudaMemsetAsync(invL, 0, 2 * (size_t)kPB * K2 * K2 * sizeof(float), st) != cudaSuccess) return 1;
  float* Ar = (float*)A;  // A viewed as floats: 2n x n, ld 2n
  const size_t ldr = 2 * (size_t)n;
  cublasStatus_t bs;
  for (int p0 = 0, pb = 0; p0 < n; p0 += PW, ++pb) {
    const int p1 = std::min(n, p0 + PW);
    // the panel's column blocks, updates confined to the panel's columns
    for (int s = 0, k0 = p0; k0 < p1; ++s, k0 += kNB) {
      const int b = pb * kPB + s, nbk = std::min(kNB, n - k0), k1 = k0 + nbk, wr = n - k1, wp = p1 - k1,
                k2 = 2 * nbk;
      float* iL = invL + (size_t)s * K2 * K2;
      float* iU = invU + (size_t)s * K2 * K2;
      k_diag_lu<<<1, 256, smem, st>>>(A, n, k0, nbk, perm, iL, iU, dinfo);
      k_apply_perm<<<(n + 31) / 32, 256, 0, st>>>(A, n, n, k0, nbk, perm);
      *launches += 2;
      if (cudaGetLastError() != cudaSuccess) return 1;
      if (wr <= 0) break;
      k_expand_panel<<<(unsigned)(((size_t)wr * nbk + 255) / 256), 256, 0, st>>>(A, n, k1, k0, wr, nbk, Ehat);
      *launches += 1;
      if (cudaGetLastError() != cudaSuccess) return 1;
      // L_ik^ = A_ik^ U_kk^-1^
      if ((bs = sgemm(blas, ct, 2 * wr, k2, k2, 1.0f, Ehat, 2 * wr, iU, K2, 0.0f, Lhat, 2 * wr)) != CUBLAS_STATUS_SUCCESS)
        return 200 + 1000 * b + (int)bs;
      *lib_calls += 1;
      if (wp > 0) {
        float* Akj = Ar + (size_t)k1 * ldr + 2 * k0;  // real 2nbk x wp, ld 2n
        float* Aij = Ar + (size_t)k1 * ldr + 2 * k1;  // real 2wr x wp, ld 2n
        // U_kj = L_kk^-1 A_kj and A_ij -= L_ik U_kj inside the panel
        if ((bs = sgemm(blas, ct, k2, wp, k2, 1.0f, iL, K2, Akj, (int)ldr, 0.0f, W1, K2)) != CUBLAS_STATUS_SUCCESS)
          return 100 + 1000 * b + (int)bs;
        if ((bs = sgemm(blas, ct, 2 * wr, wp, k2, -1.0f, Lhat, 2 * wr, W1, K2, 1.0f, Aij, (int)ldr)) !=
            CUBLAS_STATUS_SUCCESS)
          return 300 + 1000 * b + (int)bs;
        *lib_calls += 2;
        if (cudaMemcpy2DAsync(Akj, ldr * 4, W1, (size_t)K2 * 4, (size_t)k2 * 4, wp, cudaMemcpyDeviceToDevice, st) !=
            cudaSuccess)
          return 1;
      }
      // L_ik = the even columns of L_ik^
      if (cudaMemcpy2DAsync(A + (size_t)k0 * n + k1, (size_t)n * 8, Lhat, (size_t)2 * (2 * wr) * 4, (size_t)2 * wr * 4,
                            nbk, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return 1;
    }
    const int wt = n - p1;
    if (wt <= 0) break;
    // U rows of the panel for the columns right of it: block forward
    // substitution with the panel's unit lower diagonal blocks
    float* Upt = Ar + (size_t)p1 * ldr + 2 * p0;  // real 2(p1 - p0) x wt, ld 2n
    for (int s = 0, k0 = p0; k0 < p1; ++s, k0 += kNB) {
      const int b = pb * kPB + s, nbk = std::min(kNB, p1 - k0), k2 = 2 * nbk;
      float* Akt = Ar + (size_t)p1 * ldr + 2 * k0;  // real 2nbk x wt, ld 2n
      if (s > 0) {
        const int wl = k0 - p0;  // A_kt -= L_k,[p0,k0) U_[p0,k0),t
        k_expand_panel<<<(unsigned)(((size_t)nbk * wl + 255) / 256), 256, 0, st>>>(A, n, k0, p0, nbk, wl, E2);
        *launches += 1;
        if (cudaGetLastError() != cudaSuccess) return 1;
        if ((bs = sgemm(blas, ct, k2, wt, 2 * wl, -1.0f, E2, k2, Upt, (int)ldr, 1.0f, Akt, (int)ldr)) !=
            CUBLAS_STATUS_SUCCESS)
          return 400 + 1000 * b + (int)bs;
        *lib_calls += 1;
      }
      if ((bs = sgemm(blas, ct, k2, wt, k2, 1.0f, invL + (size_t)s * K2 * K2, K2, Akt, (int)ldr, 0.0f, W1, K2)) !=
          CUBLAS_STATUS_SUCCESS)
        return 500 + 1000 * b + (int)bs;
      *lib_calls += 1;
      if (cudaMemcpy2DAsync(Akt, ldr * 4, W1, (size_t)K2 * 4, (size_t)k2 * 4, wt, cudaMemcpyDeviceToDevice, st) !=
          cudaSuccess)
        return 1;
    }
    // the trailing update of the whole panel at once: A_tt -= L_t,panel U_panel,t
    const int pw = p1 - p0;
    k_expand_panel<<<(unsigned)(((size_t)wt * pw + 255) / 256), 256, 0, st>>>(A, n, p1, p0, wt, pw, Ebig);
    *launches += 1;
    if (cudaGetLastError() != cudaSuccess) return 1;
    float* Att = Ar + (size_t)p1 * ldr + 2 * p1;  // real 2wt x wt, ld 2n
    if ((bs = sgemm(blas, ct, 2 * wt, wt, 2 * pw, -1.0f, Ebig, 2 * wt, Upt, (int)ldr, 1.0f, Att, (int)ldr)) !=
        CUBLAS_STATUS_SUCCESS)
      return 600 + 1000 * pb * kPB + (int)bs;
    *lib_calls += 1;
  }
  return 0;
}

int mixed_lu_solve(cudaStream_t st, cublasHandle_t blas, int n, int nrhs, const float2* A, const int* perm, float2* X,
                   float2* tmp, long long* launches, long long* lib_calls) {
  size_t tot = (size_t)n * nrhs;
  k_gather_rows<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(X, tmp, n, nrhs, perm);
  *launches += 1;
  if (cudaGetLastError() != cudaSuccess) return 1;
  const cuComplex one = make_cuComplex(1.0f, 0.0f);
  if (cublasCtrsm(blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_UNIT, n, nrhs, &one,
                  (const cuComplex*)A, n, (cuComplex*)tmp, n) != CUBLAS_STATUS_SUCCESS)
    return 2;
  if (cublasCtrsm(blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, n, nrhs, &one,
                  (const cuComplex*)A, n, (cuComplex*)tmp, n) != CUBLAS_STATUS_SUCCESS)
    return 2;
  *lib_calls += 2;
  if (cudaMemcpyAsync(X, tmp, tot * sizeof(float2), cudaMemcpyDeviceToDevice, st) != cudaSuccess) return 1;
  return 0;
}
