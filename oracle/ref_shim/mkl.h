/* Minimal column-major CBLAS subset standing in for MKL when the reference
 * PB-SAM sources are compiled as a test oracle.  Own code: plain GEMM/GEMV
 * semantics (y = alpha*A*x + beta*y, C = alpha*A*B + beta*C), summing over k
 * in ascending order.  Only the NoTrans/ColMajor forms the reference calls
 * (src/lautil.cpp:42-72) are provided. */
#ifndef PBSAM_ORACLE_MKL_SHIM_H
#define PBSAM_ORACLE_MKL_SHIM_H

typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;

static inline void cblas_dgemv(const CBLAS_ORDER, const CBLAS_TRANSPOSE, const int M, const int N,
                               const double alpha, const double *A, const int lda,
                               const double *X, const int incX, const double beta,
                               double *Y, const int incY)
{
  for (int i = 0; i < M; i++) {
    double s = 0.0;
    for (int k = 0; k < N; k++) s += A[(long)k * lda + i] * X[(long)k * incX];
    Y[(long)i * incY] = alpha * s + (beta == 0.0 ? 0.0 : beta * Y[(long)i * incY]);
  }
}

static inline void cblas_dgemm(const CBLAS_ORDER, const CBLAS_TRANSPOSE, const CBLAS_TRANSPOSE,
                               const int M, const int N, const int K, const double alpha,
                               const double *A, const int lda, const double *B, const int ldb,
                               const double beta, double *C, const int ldc)
{
  for (int j = 0; j < N; j++)
    for (int i = 0; i < M; i++) {
      double s = 0.0;
      for (int k = 0; k < K; k++) s += A[(long)k * lda + i] * B[(long)j * ldb + k];
      C[(long)j * ldc + i] = alpha * s + (beta == 0.0 ? 0.0 : beta * C[(long)j * ldc + i]);
    }
}

#endif
