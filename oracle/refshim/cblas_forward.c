/*
 * Forwards cblas_dgemm to the OpenBLAS build that ships inside the image's
 * scipy wheel (exported there as scipy_cblas_dgemm, OpenBLAS 0.3.30, LP64).
 * Used only by the oracle build of the reference solver (oracle/_ref); the
 * reference's makefile selects a system CBLAS instead (makefile:20-40).
 * Test infrastructure: never linked into the product library.
 */
#include "cblas.h"

void scipy_cblas_dgemm(int order, int transA, int transB, int M, int N, int K,
                       double alpha, const double *A, int lda, const double *B,
                       int ldb, double beta, double *C, int ldc);

void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE transA,
                 enum CBLAS_TRANSPOSE transB, int M, int N, int K, double alpha,
                 const double *A, int lda, const double *B, int ldb, double beta,
                 double *C, int ldc) {
  scipy_cblas_dgemm((int)order, (int)transA, (int)transB, M, N, K, alpha, A, lda,
                    B, ldb, beta, C, ldc);
}

void scipy_openblas_set_num_threads(int n);

/* Pins the BLAS to n threads (the reference's timed runs use 1 BLAS thread and
 * OpenMP across elements, makefile:47-48 with -D_OMP). */
void fr_refshim_blas_threads(int n) { scipy_openblas_set_num_threads(n); }
