/* CholeskyQR of a tall-skinny B through the ca3dmm engine on one B200: the
 * caller flow of the reference's examples/example_CholeskyQR.c:52-193 with the
 * engines folded onto virtual ranks:
 *   S = B^T B               (ca3dmm_engine_init_BTB + exec)
 *   R^-1 = inv(chol(S))     (host, upper triangular, like the reference's rank 0)
 *   Q = B R^-1              (ca3dmm_engine_init, m = nrow, n = k = ncol)
 *   S1 = Q^T Q, max |S1 - I| (the reference's orthogonality check)
 *
 *   example_cholesky_qr nrow ncol [gemm_mode 0|1] [slices] [p] [cond_exp]
 *
 * B(i, j) = u(i, j) * 10^(cond_exp * (j / (ncol - 1) - 1/2)) with u uniform in
 * [0, 1) from a seeded hash; cond_exp = 0 is the reference's uniform fill. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <cuda_runtime_api.h>
#include "ca3dmm.h"
#include "cuda_proxy.h"

static double uniform(uint64_t i, uint64_t j)
{
    uint64_t z = 0x9E3779B97F4A7C15ull * (i + 1) ^ (j + 0x632BE59BD9B4E019ull) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double) (z >> 11) * (1.0 / 9007199254740992.0);
}

/* S = R^T R, R upper triangular, in place (column-major, lower part zeroed). */
static int cholesky_upper(double *S, int n)
{
    for (int j = 0; j < n; j++) {
        double d = S[j + (size_t) j * n];
        for (int k = 0; k < j; k++) d -= S[k + (size_t) j * n] * S[k + (size_t) j * n];
        if (!(d > 0.0)) return j + 1;
        const double r = sqrt(d);
        S[j + (size_t) j * n] = r;
        for (int i = j + 1; i < n; i++) {
            double s = S[j + (size_t) i * n];
            for (int k = 0; k < j; k++) s -= S[k + (size_t) j * n] * S[k + (size_t) i * n];
            S[j + (size_t) i * n] = s / r;
        }
    }
    for (int j = 0; j < n; j++)
        for (int i = j + 1; i < n; i++) S[i + (size_t) j * n] = 0.0;
    return 0;
}

/* In-place inverse of an upper triangular R (column-major). */
static void invert_upper(double *R, int n)
{
    for (int j = 0; j < n; j++) {
        R[j + (size_t) j * n] = 1.0 / R[j + (size_t) j * n];
        const double rjj = R[j + (size_t) j * n];
        for (int i = 0; i < j; i++) {          /* column j above the diagonal */
            double s = 0.0;
            for (int k = i; k < j; k++) s += R[i + (size_t) k * n] * R[k + (size_t) j * n];
            R[i + (size_t) j * n] = -s * rjj;
        }
    }
}

#define CK(x)                                                                           \
    do {                                                                                \
        cudaError_t e_ = (x);                                                           \
        if (e_ != cudaSuccess) {                                                        \
            fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, \
                    __LINE__);                                                          \
            return 2;                                                                   \
        }                                                                               \
    } while (0)

int main(int argc, char **argv)
{
    const int nrow = argc > 1 ? atoi(argv[1]) : 100000;
    const int ncol = argc > 2 ? atoi(argv[2]) : 500;
    const int mode = argc > 3 ? atoi(argv[3]) : CA3DMM_GEMM_PLAIN;
    const int slices = argc > 4 ? atoi(argv[4]) : 7;
    const int p = argc > 5 ? atoi(argv[5]) : 32;
    const double cond_exp = argc > 6 ? atof(argv[6]) : 0.0;
    if (nrow < 1 || ncol < 1 || nrow < ncol || p < 1) {
        fprintf(stderr, "usage: %s nrow ncol [gemm_mode] [slices] [p] [cond_exp]\n", argv[0]);
        return 1;
    }
    printf("Random matrix B size %d * %d, gemm mode %d (%d slices), %d virtual ranks\n", nrow,
           ncol, mode, slices, p);
    const size_t nb = (size_t) nrow * ncol, ns = (size_t) ncol * ncol;
    double *hB = (double *) malloc(sizeof(double) * nb), *hS = (double *) malloc(sizeof(double) * ns);
    for (int j = 0; j < ncol; j++) {
        const double sc = pow(10.0, cond_exp * ((ncol > 1 ? (double) j / (ncol - 1) : 0.0) - 0.5));
        for (int i = 0; i < nrow; i++) hB[i + (size_t) j * nrow] = uniform(i, j) * sc;
    }
    double *dB, *dS, *dR, *dQ;
    CK(cudaMalloc((void **) &dB, sizeof(double) * nb));
    CK(cudaMalloc((void **) &dQ, sizeof(double) * nb));
    CK(cudaMalloc((void **) &dS, sizeof(double) * ns));
    CK(cudaMalloc((void **) &dR, sizeof(double) * ns));
    CK(cudaMemcpy(dB, hB, sizeof(double) * nb, cudaMemcpyHostToDevice));

    MPI_Comm comm;
    select_cuda_device_by_mpi_local_rank();   /* as examples/example_CholeskyQR.c does */
    if (ca3dmm_vcomm_create(p, &comm)) return 1;
    /* S = B^T B */
    ca3dmm_engine_p ce_S;
    ca3dmm_engine_init_BTB(ncol, nrow, 0, nrow, 0, ncol, 0, ncol, 0, ncol, NULL, comm,
                           DEV_TYPE_CUDA, &ce_S, NULL);
    if (!ce_S) return 1;
    if (ca3dmm_engine_set_gemm_mode(ce_S, mode, slices)) return 1;
    printf("CA3DMM process grid for B^T B : %d * %d * %d\n", ce_S->mp, ce_S->np, ce_S->kp);
    cudaEvent_t ev[4];
    for (int i = 0; i < 4; i++) CK(cudaEventCreate(&ev[i]));
    ca3dmm_engine_exec(ce_S, NULL, 0, dB, nrow, dS, ncol);     /* warm-up: plan upload */
    CK(cudaEventRecord(ev[0], 0));
    ca3dmm_engine_exec(ce_S, NULL, 0, dB, nrow, dS, ncol);
    CK(cudaEventRecord(ev[1], 0));
    if (ca3dmm_engine_last_error(ce_S)) return 1;
    /* R^-1 = inv(chol(S)) on the host */
    CK(cudaMemcpy(hS, dS, sizeof(double) * ns, cudaMemcpyDeviceToHost));
    const int info = cholesky_upper(hS, ncol);
    if (info) {
        printf("Cholesky factorization of B^T B failed at column %d\n", info);
        return 3;
    }
    invert_upper(hS, ncol);
    CK(cudaMemcpy(dR, hS, sizeof(double) * ns, cudaMemcpyHostToDevice));
    /* Q = B R^-1 */
    ca3dmm_engine_p ce_Q;
    ca3dmm_engine_init(nrow, ncol, ncol, 0, 0, 0, nrow, 0, ncol, 0, ncol, 0, ncol, 0, nrow, 0, ncol,
                       NULL, comm, DEV_TYPE_CUDA, &ce_Q, NULL);
    if (!ce_Q) return 1;
    if (ca3dmm_engine_set_gemm_mode(ce_Q, mode, slices)) return 1;
    ca3dmm_engine_exec(ce_Q, dB, nrow, dR, ncol, dQ, nrow);     /* warm-up */
    CK(cudaEventRecord(ev[2], 0));
    ca3dmm_engine_exec(ce_Q, dB, nrow, dR, ncol, dQ, nrow);
    CK(cudaEventRecord(ev[3], 0));
    if (ca3dmm_engine_last_error(ce_Q)) return 1;
    /* S1 = Q^T Q and the orthogonality error */
    ca3dmm_engine_exec(ce_S, NULL, 0, dQ, nrow, dS, ncol);
    if (ca3dmm_engine_last_error(ce_S)) return 1;
    CK(cudaMemcpy(hS, dS, sizeof(double) * ns, cudaMemcpyDeviceToHost));
    double err = 0.0;
    for (int j = 0; j < ncol; j++)
        for (int i = 0; i < ncol; i++) {
            const double v = fabs(hS[i + (size_t) j * ncol] - (i == j ? 1.0 : 0.0));
            err = v > err ? v : err;
        }
    float t_s = 0, t_q = 0;
    CK(cudaEventElapsedTime(&t_s, ev[0], ev[1]));
    CK(cudaEventElapsedTime(&t_q, ev[2], ev[3]));
    printf("B^T B  : %.3f ms, %.2f TFLOP/s\n", t_s, 2.0 * ncol * ncol * (double) nrow / (t_s * 1e9));
    printf("B R^-1 : %.3f ms, %.2f TFLOP/s\n", t_q, 2.0 * ncol * ncol * (double) nrow / (t_q * 1e9));
    printf("CA3DMM CholeskyQR max error : %e\n", err);
    ca3dmm_engine_free(&ce_Q);
    ca3dmm_engine_free(&ce_S);
    ca3dmm_vcomm_free(&comm);
    cudaFree(dB); cudaFree(dQ); cudaFree(dS); cudaFree(dR);
    free(hB); free(hS);
    return 0;
}
