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
//       k_perm_expand applies P_k to the rest of block row k and expands the
//                    block column below for the GEMMs;
//       GEMM         L_ik = A_ik U_kk^-1 below the block, U_kj = L_kk^-1 A_kj
//                    and A_ij -= L_ik U_kj for the panel's columns only;
//     GEMM           the panel's U rows for the columns right of it, by
//                    block forward substitution with the L_kk^-1;
//     GEMM           A_tt -= L_t,panel U_panel,t, one rank-256 trailing
//                    update per panel (the trailing matrix is read and
//                    written once per 256 columns instead of once per 64).
//
// The complex products run as real GEMMs on the real expansions of the
// complex matrices, on the library's tcgen05 kernel (gemm_tf32.cu: TF32
// operands, FP32 accumulation in tensor memory), or on cuBLAS when the
// caller asks for its FP32 emulation on BF16 tensor cores.  Every left
// operand is laid out K-major (expanded panels written row-major by
// k_expand_rm, L_kk^-1 row-major) and every right operand is a column-major
// slice of the matrix itself, so no operand is transposed in memory.
// Pivoting is local to each diagonal block (P is block diagonal); the FP64
// refinement checks the result, and the caller falls back to a partially
// pivoted LU if the refinement does not converge.
//
// The solve (ZGETRS's part) is GEMMs as well.  The factorisation ends with
// k_panel_inverse, which forms the inverse of every panel's 256 x 256
// diagonal block of L and of U from the inverses of its four 64 x 64 blocks
// (one CTA per panel and triangle, written expanded and row-major).  Each
// triangle is then one pass over the panels: X_p = T_pp^-1 Y_p (one GEMM),
// and the rest of the right-hand sides take T's panel column times X_p (the
// column expanded by k_expand_rm, one GEMM) -- two GEMMs per panel on the
// full GPU, no waits between CTAs.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "gemm_tf32.h"
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

// The same expansion stored row-major (E[row * lde + col]): the K-major
// layout of a left operand of the tensor-core GEMM.
__device__ __forceinline__ void put_expanded_rm(float* E, int lde, int i, int k, float2 x) {
  *reinterpret_cast<float2*>(E + (size_t)(2 * i) * lde + 2 * k) = make_float2(x.x, -x.y);
  *reinterpret_cast<float2*>(E + (size_t)(2 * i + 1) * lde + 2 * k) = make_float2(x.y, x.x);
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ float2 cmac(float2 s, float2 a, float2 b) {
  return make_float2(s.x + a.x * b.x - a.y * b.y, s.y + a.x * b.y + a.y * b.x);
}

// Barrier of one 128-thread half of the block (named barrier bar, 1 or 2).
__device__ __forceinline__ void group_sync(int bar) { asm volatile("bar.sync %0, 128;" ::"r"(bar) : "memory"); }

// Inverse of the unit lower (lower) or the upper triangle of T (kNB x kNB,
// ld kLd) into X: the 8 x 8 diagonal blocks by substitution, then three
// doubling levels X21 = -X22 (L21 X11) (lower) or X12 = -X11 (U12 X22)
// (upper), each product spread over 128 threads (tid 0..127 of one half of
// the block, synchronised by the named barrier bar, so that the two halves
// form the two inverses at once); W holds the inner products of one level
// (at most 32 columns).
__device__ void tri_inverse(const float2* T, float2* X, float2* W, bool lower, int tid, int bar) {
  for (int e = tid; e < kNB * kNB; e += 128) X[(e / kNB) * kLd + e % kNB] = make_float2(0.0f, 0.0f);
  group_sync(bar);
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
  group_sync(bar);
  for (int sz = 8; sz < kNB; sz *= 2) {
    const int tot = (kNB / (2 * sz)) * sz * sz;
    for (int e = tid; e < tot; e += 128) {
      const int q = e / (sz * sz), rem = e % (sz * sz), c = rem / sz, i = rem % sz, b0 = 2 * sz * q;
      float2 acc = make_float2(0.0f, 0.0f);
      if (lower)  // W = L21 X11
        for (int k = c; k < sz; ++k) acc = cmac(acc, T[(b0 + k) * kLd + b0 + sz + i], X[(b0 + c) * kLd + b0 + k]);
      else  // W = U12 X22
        for (int k = 0; k <= c; ++k) acc = cmac(acc, T[(b0 + sz + k) * kLd + b0 + i], X[(b0 + sz + c) * kLd + b0 + sz + k]);
      W[(q * sz + c) * kLd + i] = acc;
    }
    group_sync(bar);
    for (int e = tid; e < tot; e += 128) {
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
    group_sync(bar);
  }
}

// One CTA of 256 threads: LU with partial pivoting of the nbk x nbk
// diagonal block at (k0, k0), written back in place (unit L below, U on and
// above the diagonal); the block's row permutation as global source rows in
// perm; the expansions of L^-1 (row-major) and U^-1 (column-major), 2nbk x
// 2nbk with ld 2 kNB, in invL, invU -- the K-major layouts of a left and a
// right GEMM operand; and the complex kNB x kNB inverses (column-major, the
// identity-padded block for a partial last block) in invLc, invUc for the
// triangular solves.  info gets 1 + the first global column whose pivot is
// zero.  A partial last block is padded with the identity to kNB.
__global__ void __launch_bounds__(256) k_diag_lu(float2* A, int lda, int k0, int nbk, int* perm, float* invL,
                                                 float* invU, float2* invLc, float2* invUc, int* info) {
  extern __shared__ float2 sm[];
  float2* T = sm;                  // [col * kLd + row]
  float2* X = sm + kNB * kLd;      // L^-1
  float2* Y = sm + 2 * kNB * kLd;  // U^-1
  float2* W = sm + 3 * kNB * kLd;  // inversion scratch (32 columns for each inverse)
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
  __syncthreads();  // the factors and prm are complete
  if (tid < 128)
    tri_inverse(T, X, W, true, tid, 1);
  else
    tri_inverse(T, Y, W + 32 * kLd, false, tid - 128, 2);
  __syncthreads();
  for (int e = tid; e < nbk * nbk; e += 256) {
    int r = e % nbk, c = e / nbk;
    A[(size_t)(k0 + c) * lda + k0 + r] = T[c * kLd + r];
    put_expanded_rm(invL, 2 * kNB, r, c, X[c * kLd + r]);
    put_expanded(invU, 2 * kNB, r, c, Y[c * kLd + r]);
  }
  for (int e = tid; e < kNB * kNB; e += 256) {
    int r = e % kNB, c = e / kNB;
    invLc[e] = X[c * kLd + r];
    invUc[e] = Y[c * kLd + r];
  }
  for (int i = tid; i < nbk; i += 256) perm[k0 + i] = k0 + prm[i];
}


// E (2w x 2kc, row-major, ld lde) <- the real expansion of the complex w x kc
// block of A at (r0, c0): a 32 x 32 tile through shared memory, so that the
// column-major reads of A and the row-major writes of E are both coalesced.
__global__ void __launch_bounds__(256) k_expand_rm(const float2* __restrict__ A, int lda, int r0, int c0, int w,
                                                   int kc, float* __restrict__ E, int lde) {
  __shared__ float2 tile[32][33];
  const int i0 = blockIdx.x * 32, k0 = blockIdx.y * 32, tx = threadIdx.x % 32, ty = threadIdx.x / 32;
  for (int c = ty; c < 32; c += 8)
    if (i0 + tx < w && k0 + c < kc) tile[c][tx] = A[(size_t)(c0 + k0 + c) * lda + r0 + i0 + tx];
  __syncthreads();
  for (int r = ty; r < 32; r += 8)
    if (i0 + r < w && k0 + tx < kc) put_expanded_rm(E, lde, i0 + r, k0 + tx, tile[tx][r]);
}

// The complex L_ik (wr x nbk) into A at (k1, k0) from the row-major
// expansion Lhat (2wr x 2nbk, ld ldl): entry (i, c) is (Lhat[2i][2c],
// Lhat[2i+1][2c]).
__global__ void __launch_bounds__(256) k_extract_l(const float* __restrict__ Lhat, int ldl, int wr, int nbk,
                                                   float2* __restrict__ A, int lda, int k1, int k0) {
  __shared__ float2 tile[32][33];
  const int i0 = blockIdx.x * 32, c0 = blockIdx.y * 32, tx = threadIdx.x % 32, ty = threadIdx.x / 32;
  for (int r = ty; r < 32; r += 8)
    if (i0 + r < wr && c0 + tx < nbk)
      tile[r][tx] = make_float2(Lhat[(size_t)(2 * (i0 + r)) * ldl + 2 * (c0 + tx)],
                                Lhat[(size_t)(2 * (i0 + r) + 1) * ldl + 2 * (c0 + tx)]);
  __syncthreads();
  for (int c = ty; c < 32; c += 8)
    if (i0 + tx < wr && c0 + c < nbk) A[(size_t)(k0 + c0 + c) * lda + k1 + i0 + tx] = tile[tx][c];
}

// Two independent steps after a diagonal block, in one launch of 256-thread
// blocks.  The first pblocks blocks: rows k0..k0+nbk-1 of every column
// outside the diagonal block take the block's permutation (row k0+i receives
// old row perm[k0+i]).  The others: Ehat (2wr x 2nbk, row-major, ld lde) <-
// the real expansion of the block column below the diagonal block (rows
// k0+nbk.., columns k0..k0+nbk-1), as k_expand_rm.  The permutation writes
// only rows of the diagonal block outside its columns, the expansion reads
// only its columns below it.
__global__ void __launch_bounds__(256) k_perm_expand(float2* A, int lda, int n, int k0, int nbk,
                                                     const int* __restrict__ perm, int pblocks, int wr,
                                                     float* __restrict__ E, int lde) {
  __shared__ float2 tile[kNB][33];
  const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;  // 8 x 32
  if ((int)blockIdx.x < pblocks) {
    const int c = blockIdx.x * 32 + tx;
    const bool live = c < n && (c < k0 || c >= k0 + nbk);
    for (int i = ty; i < nbk; i += 8)
      if (live) tile[i][tx] = A[(size_t)c * lda + perm[k0 + i]];
    __syncthreads();
    for (int i = ty; i < nbk; i += 8)
      if (live) A[(size_t)c * lda + k0 + i] = tile[i][tx];
    return;
  }
  const int b = blockIdx.x - pblocks, nbx = (wr + 31) / 32, r0 = k0 + nbk;
  const int i0 = (b % nbx) * 32, q0 = (b / nbx) * 32;
  for (int c = ty; c < 32; c += 8)
    if (i0 + tx < wr && q0 + c < nbk) tile[c][tx] = A[(size_t)(k0 + q0 + c) * lda + r0 + i0 + tx];
  __syncthreads();
  for (int r = ty; r < 32; r += 8)
    if (i0 + r < wr && q0 + tx < nbk) put_expanded_rm(E, lde, i0 + r, q0 + tx, tile[tx][r]);
}

// ---------------------------------------------------------------------------
// Panel inverses and the GEMM triangular solves
// ---------------------------------------------------------------------------
constexpr int kTLd = kNB + 4;  // column stride of a shared 64 x 64 block (float2; 16-byte aligned columns)
constexpr int kPW = kPB * kNB;  // panel width (columns)
constexpr int kPLd = 2 * kPW;   // leading dimension of an expanded panel inverse (floats)
constexpr int kInvSmem = 6 * kNB * kTLd * (int)sizeof(float2);

__device__ __forceinline__ void cmac_add(float2& s, float2 a, float2 b) {
  s.x += a.x * b.x - a.y * b.y;
  s.y += a.x * b.y + a.y * b.x;
}

// dst (64 x 64, column-major, ld kTLd) <- the rows x cols block at src (ld
// lds, column-major), zero outside it.
__device__ __forceinline__ void load_block(float2* dst, const float2* __restrict__ src, size_t lds, int rows,
                                           int cols) {
  for (int e = threadIdx.x; e < kNB * kNB; e += 256) {
    const int r = e % kNB, c = e / kNB;
    dst[c * kTLd + r] = (r < rows && c < cols) ? src[(size_t)c * lds + r] : make_float2(0.0f, 0.0f);
  }
}

// acc (this thread's 4 rows x 4 columns of a 64 x 64 product) += X Y, X and
// Y column-major in shared memory (ld kTLd).
__device__ __forceinline__ void block_mac(float2 (&acc)[4][4], const float2* X, const float2* Y, int r0, int c0) {
#pragma unroll 4
  for (int k = 0; k < kNB; ++k) {
    const float4 t01 = *reinterpret_cast<const float4*>(X + k * kTLd + r0);
    const float4 t23 = *reinterpret_cast<const float4*>(X + k * kTLd + r0 + 2);
    const float2 t[4] = {make_float2(t01.x, t01.y), make_float2(t01.z, t01.w), make_float2(t23.x, t23.y),
                         make_float2(t23.z, t23.w)};
    float2 y[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) y[u] = Y[(c0 + u) * kTLd + k];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int u = 0; u < 4; ++u) cmac_add(acc[i][u], t[i], y[u]);
  }
}

// The inverses of the diagonal blocks of the panels (kPW columns), from the
// inverses of their kNB diagonal blocks: blockIdx.x the panel, blockIdx.y 0
// the unit lower L_pp (block (i, j), i > j: -L_ii^-1 sum_{k=j..i-1} L_ik
// Z_kj), 1 the upper U_pp (block (i, j), i < j: -U_ii^-1 sum_{k=i+1..j}
// U_ik Z_kj), column by column of blocks.  Each is written expanded and
// row-major (kPLd x kPLd, zero outside the panel's width): the left operand
// of the solve's diagonal GEMM.  256 threads, kInvSmem bytes of shared memory.
__global__ void __launch_bounds__(256, 1) k_panel_inverse(const float2* __restrict__ A, int lda, int n,
                                                          const float2* __restrict__ invLc,
                                                          const float2* __restrict__ invUc, float* __restrict__ invLp,
                                                          float* __restrict__ invUp) {
  extern __shared__ __align__(16) float2 sm[];
  float2* Z[kPB];
  for (int b = 0; b < kPB; ++b) Z[b] = sm + b * kNB * kTLd;
  float2* sB = sm + kPB * kNB * kTLd;  // the current block of A, then the sum
  float2* sI = sB + kNB * kTLd;         // the current diagonal-block inverse
  const int p = blockIdx.x, tid = threadIdx.x, r0 = (tid % 16) * 4, c0 = (tid / 16) * 4;
  const bool lower = blockIdx.y == 0;
  const int p0 = p * kPW, pw = min(kPW, n - p0), nbk = (pw + kNB - 1) / kNB;
  const float2* invc = lower ? invLc : invUc;
  float* out = (lower ? invLp : invUp) + (size_t)p * kPLd * kPLd;
  for (int e = tid; e < kPLd * kPLd / 4; e += 256) reinterpret_cast<float4*>(out)[e] = make_float4(0.f, 0.f, 0.f, 0.f);
  auto width = [&](int b) { return min(kNB, pw - b * kNB); };
  auto write_block = [&](const float2* zb, int bi, int bj) {
    for (int e = tid; e < kNB * kNB; e += 256) {
      const int r = e % kNB, c = e / kNB;
      if (r < width(bi) && c < width(bj)) put_expanded_rm(out, kPLd, bi * kNB + r, bj * kNB + c, zb[c * kTLd + r]);
    }
  };
  __syncthreads();  // the zero fill before the blocks' writes
  for (int j = 0; j < nbk; ++j) {
    const int bj = p * kPB + j;
    load_block(Z[j], invc + (size_t)bj * kNB * kNB, kNB, width(j), width(j));
    __syncthreads();
    write_block(Z[j], j, j);
    for (int s = 1; s <= (lower ? nbk - 1 - j : j); ++s) {
      const int i = lower ? j + s : j - s;  // the block row to form
      float2 acc[4][4];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int u = 0; u < 4; ++u) acc[a][u] = make_float2(0.0f, 0.0f);
      const int ka = lower ? j : i + 1, kb = lower ? i - 1 : j;
      for (int k = ka; k <= kb; ++k) {
        __syncthreads();  // sB is free
        load_block(sB, A + (size_t)(p0 + k * kNB) * lda + p0 + i * kNB, lda, width(i), width(k));
        __syncthreads();
        block_mac(acc, sB, Z[k], r0, c0);
      }
      __syncthreads();
      for (int a = 0; a < 4; ++a)
        for (int u = 0; u < 4; ++u) sB[(c0 + u) * kTLd + r0 + a] = acc[a][u];
      load_block(sI, invc + (size_t)(p * kPB + i) * kNB * kNB, kNB, width(i), width(i));
      __syncthreads();
      float2 z[4][4];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int u = 0; u < 4; ++u) z[a][u] = make_float2(0.0f, 0.0f);
      block_mac(z, sI, sB, r0, c0);
      for (int a = 0; a < 4; ++a)
        for (int u = 0; u < 4; ++u) Z[i][(c0 + u) * kTLd + r0 + a] = make_float2(-z[a][u].x, -z[a][u].y);
      __syncthreads();
      write_block(Z[i], i, j);
    }
    __syncthreads();
  }
}

// Y (n x nrhs, ld ldy) <- rows perm of B (n x nrhs, ld n); rows n..ldy-1 zero.
__global__ void k_gather_rows(const float2* __restrict__ B, int n, int nrhs, const int* __restrict__ perm,
                              float2* __restrict__ Y, int ldy) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x, q = blockIdx.y;
  if (r >= ldy || q >= nrhs) return;
  Y[(size_t)q * ldy + r] = r < n ? B[(size_t)q * n + (perm ? perm[r] : r)] : make_float2(0.0f, 0.0f);
}

// X (n x nrhs, ld n) <- the first n rows of Y (ld ldy).
__global__ void k_copy_rows(const float2* __restrict__ Y, int ldy, int n, int nrhs, float2* __restrict__ X) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x, q = blockIdx.y;
  if (r >= n || q >= nrhs) return;
  X[(size_t)q * n + r] = Y[(size_t)q * ldy + r];
}

// ---------------------------------------------------------------------------
// GEMM dispatch: C = alpha A B + beta C, A K-major (row-major m x k), B
// K-major (column-major k x n), C column-major or row-major.
// ---------------------------------------------------------------------------
struct Gemm {
  bool own;
  cublasHandle_t blas;
  cublasComputeType_t ct;
  cudaStream_t st;
  int* err;
  long long* launches;
  long long* lib_calls;
};

// 0, 1 on a launch error, or 10 + cuBLAS status
int gemm(const Gemm& g, int m, int n, int k, float alpha, const float* A, int lda, const float* B, int ldb, float beta,
         float* C, int ldc, bool c_rowmajor) {
  if (m <= 0 || n <= 0 || k <= 0) return 0;
  if (g.own) {
    *g.launches += 1;
    return gemm_tf32(g.st, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, c_rowmajor, g.err);
  }
  *g.lib_calls += 1;
  cublasStatus_t s;
  if (!c_rowmajor)  // A row-major m x k is the column-major k x m matrix: op T
    s = cublasGemmEx(g.blas, CUBLAS_OP_T, CUBLAS_OP_N, m, n, k, &alpha, A, CUDA_R_32F, lda, B, CUDA_R_32F, ldb, &beta,
                     C, CUDA_R_32F, ldc, g.ct, CUBLAS_GEMM_DEFAULT);
  else  // C^T = B^T A^T, column-major n x m
    s = cublasGemmEx(g.blas, CUBLAS_OP_T, CUBLAS_OP_N, n, m, k, &alpha, B, CUDA_R_32F, ldb, A, CUDA_R_32F, lda, &beta,
                     C, CUDA_R_32F, ldc, g.ct, CUBLAS_GEMM_DEFAULT);
  return s == CUBLAS_STATUS_SUCCESS ? 0 : 10 + (int)s;
}

// X (m x n, column-major, ld ldx, m <= 128) <- T X with T (m x m, row-major,
// ld ldt).  The library's kernel runs it in place: C is one 128-row tile, so
// each CTA reads its own columns of X whole (TMA) before its epilogue writes
// them, and no two CTAs share a column.  cuBLAS gives no such guarantee, so
// there the product goes through W (m x n, ld m) and is copied back.
int gemm_rows_inplace(const Gemm& g, int m, int n, const float* T, int ldt, float* X, int ldx, float* W) {
  if (g.own) return gemm(g, m, n, m, 1.0f, T, ldt, X, ldx, 0.0f, X, ldx, false);
  int rc = gemm(g, m, n, m, 1.0f, T, ldt, X, ldx, 0.0f, W, m, false);
  if (rc) return rc;
  return cudaMemcpy2DAsync(X, (size_t)ldx * 4, W, (size_t)m * 4, (size_t)m * 4, n, cudaMemcpyDeviceToDevice, g.st) ==
                 cudaSuccess
             ? 0
             : 1;
}

// Workspace offsets (floats, each a multiple of 4): W1 (2kNB x n,
// column-major), Ehat and Lhat (2n x 2kNB, row-major), the expanded inverses
// of a panel's diagonal blocks (kPB each, L^-1 row-major, U^-1
// column-major), E2 (2kNB x 2kNB (kPB - 1), row-major), Ebig (2n x 2kNB kPB,
// row-major), the complex inverses of every diagonal block (kNB x kNB each, L
// then U), the expanded inverses of every panel's diagonal block (kPLd x
// kPLd each, L then U), then the solve's two right-hand-side arrays (n
// rounded up to even x nrhs, complex).
struct Layout {
  size_t W1, Ehat, Lhat, invL, invU, E2, Ebig, invLc, invUc, invLp, invUp, Y, Z, total;
  int nl;
  Layout(int n, int nrhs) {
    const size_t K2 = 2 * kNB, nblk = (size_t)(n + kNB - 1) / kNB, np = (size_t)(n + kPW - 1) / kPW;
    nl = n + (n & 1);
    W1 = 0;
    Ehat = W1 + K2 * n;
    Lhat = Ehat + 2 * (size_t)n * K2;
    invL = Lhat + 2 * (size_t)n * K2;
    invU = invL + kPB * K2 * K2;
    E2 = invU + kPB * K2 * K2;
    Ebig = E2 + K2 * K2 * (kPB - 1);
    invLc = Ebig + 2 * (size_t)n * K2 * kPB;  // complex from here on; offsets stay in floats
    invUc = invLc + 2 * nblk * kNB * kNB;
    invLp = invUc + 2 * nblk * kNB * kNB;
    invUp = invLp + np * kPLd * kPLd;
    Y = invUp + np * kPLd * kPLd;
    Z = Y + 2 * (size_t)nl * std::max(nrhs, 1);
    total = Z + 2 * (size_t)nl * std::max(nrhs, 1);
  }
};

}  // namespace

size_t mixed_lu_workspace_elems(int n, int nrhs) { return Layout(n, nrhs).total / 2 + 1; }

int mixed_lu_factor(cudaStream_t st, cublasHandle_t blas, bool own_gemm, cublasComputeType_t ct, int n, int lda,
                    float2* A, int* perm, float2* work, int* dinfo, long long* launches, long long* lib_calls) {
  const int smem = (3 * kNB + 64) * kLd * (int)sizeof(float2);  // T, L^-1, U^-1, two 32-column scratches
  if (cudaFuncSetAttribute(k_diag_lu, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) return 1;
  if (lda < n || (lda & 1)) return 1;
  const int K2 = 2 * kNB, PW = kPB * kNB;
  const Layout L(n, 0);
  float* ws = (float*)work;
  float* W1 = ws + L.W1;      // U rows, real 2nbk x w (column-major, ld 2kNB)
  float* Ehat = ws + L.Ehat;  // expanded A_ik, 2wr x 2nbk (row-major, ld 2kNB)
  float* Lhat = ws + L.Lhat;  // expanded L_ik, 2wr x 2nbk (row-major, ld 2kNB)
  float* invL = ws + L.invL;  // kPB x (2kNB x 2kNB), row-major
  float* invU = ws + L.invU;  // kPB x (2kNB x 2kNB), column-major
  float* E2 = ws + L.E2;      // expanded L rows left of a block in its panel, 2nbk x 2(k0 - p0) (row-major)
  float* Ebig = ws + L.Ebig;  // expanded L columns of a panel, 2wt x 2(p1 - p0) (row-major)
  float2* invLc = (float2*)(ws + L.invLc);
  float2* invUc = (float2*)(ws + L.invUc);
  if (cudaMemsetAsync(dinfo, 0x7f, sizeof(int), st) != cudaSuccess) return 1;  // large positive: no zero pivot
  if (cudaMemsetAsync(dinfo + 1, 0, sizeof(int), st) != cudaSuccess) return 1;
  Gemm g{own_gemm, blas, ct, st, dinfo + 1, launches, lib_calls};
  float* Ar = (float*)A;  // A viewed as floats: 2 lda x n, column-major
  const int ldr = 2 * lda;
  auto expand = [&](int r0, int c0, int w, int kc, float* E, int lde) {
    dim3 grid((unsigned)((w + 31) / 32), (unsigned)((kc + 31) / 32));
    k_expand_rm<<<grid, 256, 0, st>>>(A, lda, r0, c0, w, kc, E, lde);
    *launches += 1;
    return cudaGetLastError() == cudaSuccess;
  };
  auto code = [](int rc, int g, int b) { return rc == 1 ? 1 : 100 * g + 1000 * b + rc - 10; };
  int rc;
  for (int p0 = 0, pb = 0; p0 < n; p0 += PW, ++pb) {
    const int p1 = std::min(n, p0 + PW);
    // the panel's column blocks, updates confined to the panel's columns
    for (int s = 0, k0 = p0; k0 < p1; ++s, k0 += kNB) {
      const int b = pb * kPB + s, nbk = std::min(kNB, n - k0), k1 = k0 + nbk, wr = n - k1, wp = p1 - k1,
                k2 = 2 * nbk;
      float* iL = invL + (size_t)s * K2 * K2;
      float* iU = invU + (size_t)s * K2 * K2;
      k_diag_lu<<<1, 256, smem, st>>>(A, lda, k0, nbk, perm, iL, iU, invLc + (size_t)b * kNB * kNB,
                                      invUc + (size_t)b * kNB * kNB, dinfo);
      {  // the block's permutation and the expansion of its column below, one launch
        const int pb = (n + 31) / 32, nex = wr > 0 ? ((wr + 31) / 32) * ((nbk + 31) / 32) : 0;
        k_perm_expand<<<pb + nex, 256, 0, st>>>(A, lda, n, k0, nbk, perm, pb, wr, Ehat, K2);
      }
      *launches += 2;
      if (cudaGetLastError() != cudaSuccess) return 1;
      if (wr <= 0) break;
      // L_ik^ = A_ik^ U_kk^-1^ (row-major: the left operand of the update below)
      if ((rc = gemm(g, 2 * wr, k2, k2, 1.0f, Ehat, K2, iU, K2, 0.0f, Lhat, K2, true))) return code(rc, 2, b);
      if (wp > 0) {
        float* Akj = Ar + (size_t)k1 * ldr + 2 * k0;  // real 2nbk x wp, ld 2 lda
        float* Aij = Ar + (size_t)k1 * ldr + 2 * k1;  // real 2wr x wp, ld 2 lda
        // U_kj = L_kk^-1 A_kj and A_ij -= L_ik U_kj inside the panel
        if ((rc = gemm_rows_inplace(g, k2, wp, iL, K2, Akj, ldr, W1))) return code(rc, 1, b);
        if ((rc = gemm(g, 2 * wr, wp, k2, -1.0f, Lhat, K2, Akj, ldr, 1.0f, Aij, ldr, false))) return code(rc, 3, b);
      }
      {  // L_ik into A
        dim3 grid((unsigned)((wr + 31) / 32), (unsigned)((nbk + 31) / 32));
        k_extract_l<<<grid, 256, 0, st>>>(Lhat, K2, wr, nbk, A, lda, k1, k0);
        *launches += 1;
        if (cudaGetLastError() != cudaSuccess) return 1;
      }
    }
    const int wt = n - p1;
    if (wt <= 0) break;
    // U rows of the panel for the columns right of it: block forward
    // substitution with the panel's unit lower diagonal blocks
    float* Upt = Ar + (size_t)p1 * ldr + 2 * p0;  // real 2(p1 - p0) x wt, ld 2 lda
    for (int s = 0, k0 = p0; k0 < p1; ++s, k0 += kNB) {
      const int b = pb * kPB + s, nbk = std::min(kNB, p1 - k0), k2 = 2 * nbk;
      float* Akt = Ar + (size_t)p1 * ldr + 2 * k0;  // real 2nbk x wt, ld 2 lda
      if (s > 0) {
        const int wl = k0 - p0;  // A_kt -= L_k,[p0,k0) U_[p0,k0),t
        if (!expand(k0, p0, nbk, wl, E2, 2 * wl)) return 1;
        if ((rc = gemm(g, k2, wt, 2 * wl, -1.0f, E2, 2 * wl, Upt, ldr, 1.0f, Akt, ldr, false))) return code(rc, 4, b);
      }
      if ((rc = gemm_rows_inplace(g, k2, wt, invL + (size_t)s * K2 * K2, K2, Akt, ldr, W1))) return code(rc, 5, b);
    }
    // the trailing update of the whole panel at once: A_tt -= L_t,panel U_panel,t
    const int pw = p1 - p0;
    if (!expand(p1, p0, wt, pw, Ebig, 2 * pw)) return 1;
    float* Att = Ar + (size_t)p1 * ldr + 2 * p1;  // real 2wt x wt, ld 2 lda
    if ((rc = gemm(g, 2 * wt, wt, 2 * pw, -1.0f, Ebig, 2 * pw, Upt, ldr, 1.0f, Att, ldr, false)))
      return code(rc, 6, pb * kPB);
  }
  // the panels' diagonal-block inverses for the solves
  if (cudaFuncSetAttribute(k_panel_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, kInvSmem) != cudaSuccess)
    return 1;
  const int np = (n + kPW - 1) / kPW;
  k_panel_inverse<<<dim3((unsigned)np, 2), 256, kInvSmem, st>>>(A, lda, n, invLc, invUc, ws + L.invLp, ws + L.invUp);
  *launches += 1;
  if (cudaGetLastError() != cudaSuccess) return 1;
  return 0;
}

void mixed_lu_gemm_shapes(int n, std::vector<int>& shapes) {
  const int PW = kPB * kNB;
  auto add = [&](int m, int nn, int k) {
    if (m > 0 && nn > 0 && k > 0) shapes.insert(shapes.end(), {m, nn, k});
  };
  for (int p0 = 0; p0 < n; p0 += PW) {
    const int p1 = std::min(n, p0 + PW), wt = n - p1;
    for (int k0 = p0; k0 < p1; k0 += kNB) {
      const int nbk = std::min(kNB, n - k0), k1 = k0 + nbk, wr = n - k1, wp = p1 - k1, k2 = 2 * nbk;
      add(2 * wr, k2, k2);
      add(k2, wp, k2);
      add(2 * wr, wp, k2);
      if (k0 > p0) add(k2, wt, 2 * (k0 - p0));
      add(k2, wt, k2);
    }
    add(2 * wt, wt, 2 * (p1 - p0));
  }
}

int mixed_lu_solve(cudaStream_t st, cublasHandle_t blas, bool own_gemm, cublasComputeType_t ct, int n, int lda,
                   int nrhs, const float2* A, const int* perm, float2* X, float2* work, int* dflag,
                   long long* launches, long long* lib_calls) {
  if (nrhs <= 0) return 0;
  const Layout L(n, nrhs);
  float* ws = (float*)work;
  const int nl = L.nl, ldy = 2 * nl, np = (n + kPW - 1) / kPW;
  float2* Y = (float2*)(ws + L.Y);  // Y, then Z: n rounded up to even x nrhs, complex
  float* Yr = ws + L.Y;  // the real views: 2 nl x nrhs, column-major
  float* Zr = ws + L.Z;
  float* Ebig = ws + L.Ebig;
  Gemm g{own_gemm, blas, ct, st, dflag, launches, lib_calls};
  auto expand = [&](int r0, int c0, int w, int kc, int lde) {
    dim3 grid((unsigned)((w + 31) / 32), (unsigned)((kc + 31) / 32));
    k_expand_rm<<<grid, 256, 0, st>>>(A, lda, r0, c0, w, kc, Ebig, lde);
    *launches += 1;
    return cudaGetLastError() == cudaSuccess;
  };
  const dim3 rows((unsigned)((nl + 255) / 256), (unsigned)nrhs);
  k_gather_rows<<<rows, 256, 0, st>>>(X, n, nrhs, perm, Y, nl);  // Y = P X
  *launches += 1;
  if (cudaGetLastError() != cudaSuccess) return 1;
  int rc;
  // forward, Z = L^-1 Y: per panel Z_p = L_pp^-1 Y_p, then Y below -= L_(below, p) Z_p
  for (int p = 0; p < np; ++p) {
    const int p0 = p * kPW, p1 = std::min(n, p0 + kPW), pw = p1 - p0, lde = (2 * pw + 3) / 4 * 4;
    if ((rc = gemm(g, 2 * pw, nrhs, 2 * pw, 1.0f, ws + L.invLp + (size_t)p * kPLd * kPLd, kPLd, Yr + 2 * p0, ldy,
                   0.0f, Zr + 2 * p0, ldy, false)))
      return 10 + rc;
    if (p1 < n) {
      if (!expand(p1, p0, n - p1, pw, lde)) return 1;
      if ((rc = gemm(g, 2 * (n - p1), nrhs, 2 * pw, -1.0f, Ebig, lde, Zr + 2 * p0, ldy, 1.0f, Yr + 2 * p1, ldy,
                     false)))
        return 10 + rc;
    }
  }
  // backward, Y = U^-1 Z: per panel from the last, Y_p = U_pp^-1 Z_p, then Z above -= U_(above, p) Y_p
  for (int p = np - 1; p >= 0; --p) {
    const int p0 = p * kPW, p1 = std::min(n, p0 + kPW), pw = p1 - p0, lde = (2 * pw + 3) / 4 * 4;
    if ((rc = gemm(g, 2 * pw, nrhs, 2 * pw, 1.0f, ws + L.invUp + (size_t)p * kPLd * kPLd, kPLd, Zr + 2 * p0, ldy,
                   0.0f, Yr + 2 * p0, ldy, false)))
      return 10 + rc;
    if (p0 > 0) {
      if (!expand(0, p0, p0, pw, lde)) return 1;
      if ((rc = gemm(g, 2 * p0, nrhs, 2 * pw, -1.0f, Ebig, lde, Yr + 2 * p0, ldy, 1.0f, Zr, ldy, false)))
        return 10 + rc;
    }
  }
  k_copy_rows<<<dim3((unsigned)((n + 255) / 256), (unsigned)nrhs), 256, 0, st>>>(Y, nl, n, nrhs, X);
  *launches += 1;
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
