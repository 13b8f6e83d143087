/* CBLAS declarations for the oracle's reference build (OpenBLAS provides the
 * symbols).  Only what the reference's CPU path calls.  With
 * VMPI_SCIPY_OPENBLAS the names map to the scipy_-prefixed exports of the
 * OpenBLAS build that ships inside the scipy wheel. */
#ifndef VMPI_CBLAS_H
#define VMPI_CBLAS_H
#ifdef VMPI_SCIPY_OPENBLAS
#define cblas_dgemm scipy_cblas_dgemm
#define openblas_set_num_threads scipy_openblas_set_num_threads
#endif
typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef CBLAS_LAYOUT CBLAS_ORDER;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;
void cblas_dgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, const int m,
                 const int n, const int k, const double alpha, const double *A, const int lda,
                 const double *B, const int ldb, const double beta, double *C, const int ldc);
void openblas_set_num_threads(int n);
#endif
