// gemm_tf32.h -- real GEMM on the fifth-generation tensor cores (tcgen05.mma
// kind::tf32, FP32 accumulation in tensor memory), the product kernel of the
// complex64 block LU of the mixed form (lu_mixed.cu).
#pragma once
#include <cuda_runtime.h>

// C = alpha * A B + beta * C with
//   A  m x k, K-major: element (i, l) at A[i * lda + l]
//   B  k x n, K-major: element (l, j) at B[j * ldb + l]   (column-major B)
//   C  m x n, column-major (element (i, j) at C[j * ldc + i]), or, with
//      c_rowmajor, row-major (C[i * ldc + j]).
// A and B are read as TF32 (the low 13 mantissa bits ignored), products are
// accumulated in FP32.  A, B 16-byte aligned, lda and ldb multiples of 4.
// err: device word that receives bit 0 if a pipeline wait gave up (the
// kernel then stops and returns; the caller turns it into an error).
// Returns 0, or 1 on a launch or tensor-map error.
int gemm_tf32(cudaStream_t st, int m, int n, int k, float alpha, const float* A, int lda, const float* B, int ldb,
              float beta, float* C, int ldc, bool c_rowmajor, int* err);
