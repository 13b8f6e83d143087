/* Serialises the reference's cuBLAS wrappers across vmpi rank threads (TEST AND
 * COMPARISON INFRASTRUCTURE ONLY).
 *
 * src/cuda_proxy.cu:151-174 keeps one static cuBLAS handle per process, which
 * is right for one MPI rank per process but not for ranks that are threads of
 * one process: cuBLAS handles must not be used by two threads at once.  The
 * build compiles cuda_proxy.cu with each handle-using wrapper renamed to
 * vgpu_raw_<name>; the reference's C files keep calling <name>, which lands
 * here, takes one process-wide lock and calls the original.  Each original
 * synchronises its stream before returning (cuda_proxy.cu:222-229), so the
 * lock spans exactly one library call and its completion. */
#include <pthread.h>
#include <stdint.h>
#include "cuda_proxy.h"

#define RAW(f) vgpu_raw_##f

void RAW(cuda_cublas_dcopy)(const int n, const double *x, const int incx, double *y, const int incy);
void RAW(cuda_cublas_dscal)(const int n, const double alpha, double *x, const int incx);
double RAW(cuda_cublas_ddot)(const int n, const double *x, const int incx, const double *y,
                             const int incy);
void RAW(cuda_cublas_dgemm)(cublas_enum_t transA, cublas_enum_t transB, const int m, const int n,
                            const int k, const double alpha, const double *A, const int ldA,
                            const double *B, const int ldB, const double beta, double *C,
                            const int ldC);
void RAW(cuda_cublas_dgeam)(cublas_enum_t transA, cublas_enum_t transB, const int m, const int n,
                            const double alpha, const double *A, const int ldA, const double beta,
                            const double *B, const int ldB, double *C, const int ldC);
void RAW(cuda_cublas_dtrsm)(cublas_enum_t side, cublas_enum_t uplo, cublas_enum_t trans,
                            cublas_enum_t diag, const int m, const int n, const double alpha,
                            const double *A, const int ldA, double *B, const int ldB);
int RAW(cuda_cusolver_dpotrf)(const char uplo, const int n, double *A, const int ldA);
int RAW(cuda_cusolver_dsyevd)(const char jobz, const char uplo, const int n, double *A,
                              const int ldA, double *W);

static pthread_mutex_t lib_lock = PTHREAD_MUTEX_INITIALIZER;

#define LOCKED(stmt) do { pthread_mutex_lock(&lib_lock); stmt; pthread_mutex_unlock(&lib_lock); } while (0)

void cuda_cublas_dcopy(const int n, const double *x, const int incx, double *y, const int incy)
{
    LOCKED(RAW(cuda_cublas_dcopy)(n, x, incx, y, incy));
}

void cuda_cublas_dscal(const int n, const double alpha, double *x, const int incx)
{
    LOCKED(RAW(cuda_cublas_dscal)(n, alpha, x, incx));
}

double cuda_cublas_ddot(const int n, const double *x, const int incx, const double *y, const int incy)
{
    double r;
    LOCKED(r = RAW(cuda_cublas_ddot)(n, x, incx, y, incy));
    return r;
}

void cuda_cublas_dgemm(cublas_enum_t transA, cublas_enum_t transB, const int m, const int n,
                       const int k, const double alpha, const double *A, const int ldA,
                       const double *B, const int ldB, const double beta, double *C, const int ldC)
{
    LOCKED(RAW(cuda_cublas_dgemm)(transA, transB, m, n, k, alpha, A, ldA, B, ldB, beta, C, ldC));
}

void cuda_cublas_dgeam(cublas_enum_t transA, cublas_enum_t transB, const int m, const int n,
                       const double alpha, const double *A, const int ldA, const double beta,
                       const double *B, const int ldB, double *C, const int ldC)
{
    LOCKED(RAW(cuda_cublas_dgeam)(transA, transB, m, n, alpha, A, ldA, beta, B, ldB, C, ldC));
}

void cuda_cublas_dtrsm(cublas_enum_t side, cublas_enum_t uplo, cublas_enum_t trans,
                       cublas_enum_t diag, const int m, const int n, const double alpha,
                       const double *A, const int ldA, double *B, const int ldB)
{
    LOCKED(RAW(cuda_cublas_dtrsm)(side, uplo, trans, diag, m, n, alpha, A, ldA, B, ldB));
}

int cuda_cusolver_dpotrf(const char uplo, const int n, double *A, const int ldA)
{
    int r;
    LOCKED(r = RAW(cuda_cusolver_dpotrf)(uplo, n, A, ldA));
    return r;
}

int cuda_cusolver_dsyevd(const char jobz, const char uplo, const int n, double *A, const int ldA,
                         double *W)
{
    int r;
    LOCKED(r = RAW(cuda_cusolver_dsyevd)(jobz, uplo, n, A, ldA, W));
    return r;
}
