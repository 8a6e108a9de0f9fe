/*
 * Minimal CBLAS declaration used only to compile the reference solver's own
 * sources into the oracle build (oracle/_ref).  The reference calls exactly one
 * BLAS routine, a row-major double GEMM (reference: src/solver.cpp:556-572 and
 * every other operator application), so this header declares only that.
 * Test infrastructure: never linked into the product library.
 */
#ifndef FR_ORACLE_REFSHIM_CBLAS_H
#define FR_ORACLE_REFSHIM_CBLAS_H
#ifdef __cplusplus
extern "C" {
#endif
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
typedef enum CBLAS_ORDER CBLAS_LAYOUT;
void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE transA,
                 enum CBLAS_TRANSPOSE transB, int M, int N, int K, double alpha,
                 const double *A, int lda, const double *B, int ldb, double beta,
                 double *C, int ldc);
#ifdef __cplusplus
}
#endif
#endif
