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

// The same product with an explicit tile variant: 0 = 128 x 64, 1 = 128 x 128,
// 2 = 128 x 256 (rows x columns of C per CTA).  Every variant sums each
// element over the K panels in the same order.
int gemm_tf32_variant(cudaStream_t st, int variant, int m, int n, int k, float alpha, const float* A, int lda,
                      const float* B, int ldb, float beta, float* C, int ldc, bool c_rowmajor, int* err);

// The autotuner.  gemm_tf32 takes the variant measured fastest for the shape
// class of (m, n, k) on this device (M by powers of two of 128-row tiles, N of
// 64-column tiles, K by 128), or a size heuristic for a class not measured.
// gemm_tf32_autotune measures the classes of the nshape shapes (m, n, k) not
// measured yet, each on scratch operands of its largest shape (the variants
// in turn for six rounds on stream st, each launch timed alone, the first
// round a warm-up), and records the variant with the fastest launch.
// Returns 0 or 1.
int gemm_tf32_pick(int m, int n, int k);
int gemm_tf32_autotune(cudaStream_t st, int nshape, const int* shapes);
int gemm_tf32_tuned_count();
