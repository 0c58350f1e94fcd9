// lu_mixed.h -- complex64 block LU for the mixed form (lu_mixed.cu).
#pragma once
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <vector>

// Elements (float2) of the workspace mixed_lu_factor / mixed_lu_solve need
// for order n and nrhs right-hand sides.
size_t mixed_lu_workspace_elems(int n, int nrhs);

// Leading dimension (complex elements) of the matrix the block LU works on:
// n rounded up to even, so that every column of the float view starts on a
// 16-byte boundary (the tensor-memory-accelerator copies need it).
inline int mixed_lu_ld(int n) { return n + (n & 1); }

// In-place factorisation P A = L U of the n x n complex64 matrix A (leading
// dimension lda = mixed_lu_ld(n)), P block diagonal (pivoting inside each
// 64-row diagonal block); perm (n) receives the permutation as source rows,
// dinfo[0] 1 + the first column with a zero pivot (or a large value if
// none), dinfo[1] the tensor-core kernels' error word (nonzero if a pipeline
// wait gave up).  With own_gemm the products run on the library's tcgen05
// kernel (TF32 operands, FP32 accumulation); otherwise on cuBLAS with
// compute type ct.  Returns 0, 1 on a CUDA or launch error, or 100 g + 1000 b
// + status for a cuBLAS error of GEMM g at block b.
int mixed_lu_factor(cudaStream_t st, cublasHandle_t blas, bool own_gemm, cublasComputeType_t ct, int n, int lda,
                    float2* A, int* perm, float2* work, int* dinfo, long long* launches, long long* lib_calls);

// X (n x nrhs, ld n) <- (P^T L U)^-1 X with the factors of mixed_lu_factor:
// per 256-column panel one GEMM with the panel's diagonal-block inverse
// (formed by the factorisation) and one with the panel's column of L (or U)
// for the rest, on the same GEMM as the factorisation (own_gemm: the
// library's tcgen05 kernel; otherwise cuBLAS with compute type ct).
// dflag: the tensor-core kernels' error word (nonzero if a pipeline wait gave
// up).  Returns 0, 1 on a CUDA or launch error, or 10 + a GEMM's status.
int mixed_lu_solve(cudaStream_t st, cublasHandle_t blas, bool own_gemm, cublasComputeType_t ct, int n, int lda,
                   int nrhs, const float2* A, const int* perm, float2* X, float2* work, int* dflag,
                   long long* launches, long long* lib_calls);

// The (m, n, k) shapes of the real GEMMs mixed_lu_factor runs for order n,
// three ints each (the input of the GEMM autotuner).
void mixed_lu_gemm_shapes(int n, std::vector<int>& shapes);
