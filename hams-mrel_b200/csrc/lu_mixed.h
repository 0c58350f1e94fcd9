// lu_mixed.h -- complex64 block LU for the mixed form (lu_mixed.cu).
#pragma once
#include <cublas_v2.h>
#include <cuda_runtime.h>

// Elements (float2) of the workspace mixed_lu_factor needs for order n.
size_t mixed_lu_workspace_elems(int n);

// In-place factorisation P A = L U of the n x n complex64 matrix A (ld n),
// P block diagonal (pivoting inside each 64-row diagonal block); perm (n)
// receives the permutation as source rows, dinfo 1 + the first column with
// a zero pivot (or a large value if none).  GEMMs run on cuBLAS with compute
// type ct.  Returns 0, 1 on a CUDA error, or 100 g + 1000 b + status for a
// cuBLAS error of GEMM g (1-3) at block b.
int mixed_lu_factor(cudaStream_t st, cublasHandle_t blas, cublasComputeType_t ct, int n, float2* A, int* perm,
                    float2* work, int* dinfo, long long* launches, long long* lib_calls);

// X (n x nrhs, ld n) <- (P^T L U)^-1 X using the factors of mixed_lu_factor;
// tmp holds n x nrhs elements.
int mixed_lu_solve(cudaStream_t st, cublasHandle_t blas, int n, int nrhs, const float2* A, const int* perm, float2* X,
                   float2* tmp, long long* launches, long long* lib_calls);
