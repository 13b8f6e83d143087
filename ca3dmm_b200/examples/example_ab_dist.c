/* C = op(A) * op(B) on p ranks of the multi-GPU engine (include/ca3dmm_dist.h):
 * the reference's examples/example_AB.c:17-316 as run under mpirun -np p, with
 * the ranks as threads of this process.  Same command line, same deterministic
 * fill, same 1D column blocks of A, B and C per rank (example_AB.c:85-98), same
 * output lines, and the same validation rule (an entry is an error when its
 * relative difference from the closed form of the fill exceeds 1e-12).
 *
 *   [CA3DMM_DIST_RANKS=p] [CA3DMM_DIST_TRANSPORT=threads|nccl]
 *   example_ab_dist m n k transA transB check_correct n_test dev_type [mp np kp]
 *
 * p defaults to mp * np * kp when a grid is given, else 2.  The threads
 * transport exchanges through host memory and runs every rank on the current
 * GPU; nccl puts rank r on GPU r (it needs p GPUs).  The GEMM mode comes from
 * CA3DMM_GEMM_MODE (0 plain FP64, 1 INT8 slices, 2 modular). */
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <cuda_runtime_api.h>
#include "ca3dmm.h"
#include "ca3dmm_dist.h"

typedef struct {
    int rank, p, use_nccl;
    int m, n, k, ta, tb, chk, n_test, gemm_mode, slices;
    const int *grid;
    ca3dmm_transport_t *tr;
    const unsigned char *nccl_id;
    /* results */
    int rc, errors, info[10];
    double *ms;        /* [4][n_test] per exec: operand exchange, GEMM, C exchange, total */
} rank_arg_t;

static int get_int_param(int argc, char **argv, int argi, int default_val, int min_val, int max_val)
{
    int res = default_val;
    if (argc >= argi + 1) {
        res = atoi(argv[argi]);
        if (res < min_val || res > max_val) res = default_val;
    }
    return res;
}

static void *rank_main(void *arg_)
{
    rank_arg_t *a = (rank_arg_t *) arg_;
    const int r = a->rank, p = a->p;
    ca3dmm_transport_t ncc, *tr = a->tr + r;
    if (a->use_nccl) {
        if (cudaSetDevice(r) != cudaSuccess ||
            ca3dmm_transport_nccl_create(p, r, a->nccl_id, &ncc) != 0) {
            a->rc = 1;
            return NULL;
        }
        tr = &ncc;
    }
    const int A_nrow = a->ta ? a->k : a->m, A_ncol = a->ta ? a->m : a->k;
    const int B_nrow = a->tb ? a->n : a->k, B_ncol = a->tb ? a->k : a->n;
    const int C_nrow = a->m, C_ncol = a->n;
    int A_scol, A_ncl, B_scol, B_ncl, C_scol, C_ncl;
    calc_block_spos_size(A_ncol, p, r, &A_scol, &A_ncl);
    calc_block_spos_size(B_ncol, p, r, &B_scol, &B_ncl);
    calc_block_spos_size(C_ncol, p, r, &C_scol, &C_ncl);
    const size_t A_sz = (size_t) A_nrow * A_ncl, B_sz = (size_t) B_nrow * B_ncl,
                 C_sz = (size_t) C_nrow * C_ncl;
    double *A_h = (double *) malloc(sizeof(double) * (A_sz + 1));
    double *B_h = (double *) malloc(sizeof(double) * (B_sz + 1));
    double *C_h = (double *) malloc(sizeof(double) * (C_sz + 1));
    double *A_d = NULL, *B_d = NULL, *C_d = NULL;
    if (!A_h || !B_h || !C_h || cudaMalloc((void **) &A_d, sizeof(double) * (A_sz + 1)) ||
        cudaMalloc((void **) &B_d, sizeof(double) * (B_sz + 1)) ||
        cudaMalloc((void **) &C_d, sizeof(double) * (C_sz + 1))) {
        a->rc = 1;
        return NULL;
    }
    for (int j = 0; j < A_ncl; j++)
        for (int i = 0; i < A_nrow; i++)
            A_h[i + (size_t) j * A_nrow] = 0.19 * (double) i + 0.24 * (double) (j + A_scol);
    for (int j = 0; j < B_ncl; j++)
        for (int i = 0; i < B_nrow; i++)
            B_h[i + (size_t) j * B_nrow] = 0.11 * (double) i + 0.12 * (double) (j + B_scol);
    cudaMemcpy(A_d, A_h, sizeof(double) * A_sz, cudaMemcpyHostToDevice);
    cudaMemcpy(B_d, B_h, sizeof(double) * B_sz, cudaMemcpyHostToDevice);
    ca3dmm_dist_engine_p e = NULL;
    a->rc = ca3dmm_dist_engine_init(a->m, a->n, a->k, a->ta, a->tb, 0, 0, A_nrow, A_scol, A_ncl, 0,
                                    B_nrow, B_scol, B_ncl, 0, C_nrow, C_scol, C_ncl, a->grid, tr,
                                    a->gemm_mode, a->slices, &e);
    if (!a->rc) {
        ca3dmm_dist_engine_info(e, a->info);
        a->rc = ca3dmm_dist_engine_exec(e, A_d, A_nrow, B_d, B_nrow, C_d, C_nrow);   /* warm-up */
    }
    double prev[4] = {0, 0, 0, 0};
    if (!a->rc) ca3dmm_dist_engine_stats(e, prev);
    for (int t = 0; t < a->n_test && !a->rc; t++) {
        a->rc = ca3dmm_dist_engine_exec(e, A_d, A_nrow, B_d, B_nrow, C_d, C_nrow);
        double now[4];
        ca3dmm_dist_engine_stats(e, now);
        for (int q = 0; q < 4; q++) {
            a->ms[q * a->n_test + t] = now[q] - prev[q];
            prev[q] = now[q];
        }
    }
    if (!a->rc && a->chk) {
        cudaMemcpy(C_h, C_d, sizeof(double) * C_sz, cudaMemcpyDeviceToHost);
        const double a1 = a->ta ? 0.24 : 0.19, a2 = a->ta ? 0.19 : 0.24;
        const double b1 = a->tb ? 0.12 : 0.11, b2 = a->tb ? 0.11 : 0.12;
        const double kk = (double) a->k, S1 = kk * (kk - 1.0) / 2.0;
        const double S2 = (kk - 1.0) * kk * (2.0 * kk - 1.0) / 6.0;
        for (int j = 0; j < C_ncl; j++)
            for (int i = 0; i < C_nrow; i++) {
                const double jj = (double) (j + C_scol);
                const double c = a1 * b1 * i * S1 + a1 * b2 * (double) i * jj * kk + a2 * b1 * S2 +
                                 a2 * b2 * jj * S1;
                if (fabs((C_h[i + (size_t) j * C_nrow] - c) / c) > 1e-12) a->errors++;
            }
    }
    if (e) ca3dmm_dist_engine_free(&e);
    if (a->use_nccl) ca3dmm_transport_nccl_free(&ncc);
    cudaFree(A_d);
    cudaFree(B_d);
    cudaFree(C_d);
    free(A_h);
    free(B_h);
    free(C_h);
    return NULL;
}

int main(int argc, char **argv)
{
    if ((argc == 2) && ((strcmp(argv[1], "--help") == 0) || (strcmp(argv[1], "-h") == 0))) {
        printf("Usage: %s m n k transA(0 or 1) transB(0 or 1) check_correct(0 or 1) n_test dev_type"
               " [mp np kp]\n", argv[0]);
        return 0;
    }
    int m = get_int_param(argc, argv, 1, 4096, 1, 8388608);
    int n = get_int_param(argc, argv, 2, 4096, 1, 8388608);
    int k = get_int_param(argc, argv, 3, 4096, 1, 8388608);
    int ta = get_int_param(argc, argv, 4, 0, 0, 1);
    int tb = get_int_param(argc, argv, 5, 0, 0, 1);
    int chk = get_int_param(argc, argv, 6, 1, 0, 1);
    int n_test = get_int_param(argc, argv, 7, 10, 1, 100);
    int dev_type = get_int_param(argc, argv, 8, DEV_TYPE_CUDA, DEV_TYPE_CUDA, DEV_TYPE_CUDA_MPI_DIRECT);
    int grid[3] = {0, 0, 0}, *proc_grid = NULL;
    if (argc >= 12) {
        grid[0] = atoi(argv[9]);
        grid[1] = atoi(argv[10]);
        grid[2] = atoi(argv[11]);
        proc_grid = grid;
    }
    const char *pv = getenv("CA3DMM_DIST_RANKS");
    int p = pv ? atoi(pv) : (proc_grid ? grid[0] * grid[1] * grid[2] : 2);
    if (p < 1 || p > 1024) {
        fprintf(stderr, "invalid number of ranks %d\n", p);
        return 1;
    }
    const char *tv = getenv("CA3DMM_DIST_TRANSPORT");
    const int use_nccl = tv && strcmp(tv, "nccl") == 0;
    const char *gv = getenv("CA3DMM_GEMM_MODE");
    const int gemm_mode = gv ? atoi(gv) : 0;
    printf("Test problem size m * n * k : %d * %d * %d\n", m, n, k);
    printf("Transpose A / B             : %d / %d\n", ta, tb);
    printf("Number of tests             : %d\n", n_test);
    printf("Check result correctness    : %d\n", chk);
    printf("Device type                 : %d\n", dev_type);
    printf("\n");
    fflush(stdout);

    unsigned char id[128];
    ca3dmm_transport_t *tr = (ca3dmm_transport_t *) calloc((size_t) p, sizeof(ca3dmm_transport_t));
    rank_arg_t *args = (rank_arg_t *) calloc((size_t) p, sizeof(rank_arg_t));
    pthread_t *th = (pthread_t *) calloc((size_t) p, sizeof(pthread_t));
    if (!tr || !args || !th) return 1;
    if (use_nccl) {
        int ndev = 0;
        cudaGetDeviceCount(&ndev);
        if (ndev < p || ca3dmm_nccl_unique_id(id) != 0) {
            fprintf(stderr, "the nccl transport needs %d GPUs (found %d)\n", p, ndev);
            return 1;
        }
    } else if (ca3dmm_transport_threads_create(p, tr) != 0) {
        return 1;
    }
    for (int r = 0; r < p; r++) {
        rank_arg_t *a = &args[r];
        a->rank = r; a->p = p; a->use_nccl = use_nccl;
        a->m = m; a->n = n; a->k = k; a->ta = ta; a->tb = tb; a->chk = chk; a->n_test = n_test;
        a->gemm_mode = gemm_mode; a->slices = gemm_mode == 1 ? 7 : 0;
        a->grid = proc_grid; a->tr = tr; a->nccl_id = id;
        a->ms = (double *) calloc(4 * (size_t) n_test, sizeof(double));
        pthread_create(&th[r], NULL, rank_main, a);
    }
    int rc = 0, errors = 0;
    for (int r = 0; r < p; r++) {
        pthread_join(th[r], NULL);
        rc |= args[r].rc;
        errors += args[r].errors;
    }
    if (!use_nccl) ca3dmm_transport_threads_free(tr);
    if (rc) {
        fprintf(stderr, "a rank failed (error %d)\n", rc);
        return 1;
    }
    const int *g = args[0].info;
    const int mb = (m + g[0] - 1) / g[0], nb = (n + g[1] - 1) / g[1], kb = (k + g[2] - 1) / g[2];
    double min_comm_vol = (double) m * (double) n * (double) k / (double) p;
    min_comm_vol = 3.0 * pow(min_comm_vol, 2.0 / 3.0) * (double) p;
    double curr_comm_vol = ((double) mb * nb + (double) mb * kb + (double) nb * kb) * (double) p;
    printf("CA3DMM partition info:\n");
    printf("Process grid mp * np * kp  : %d * %d * %d\n", g[0], g[1], g[2]);
    printf("Work cuboid  mb * nb * kb  : %d * %d * %d\n", mb, nb, kb);
    printf("Process utilization        : %.2f %% \n", 100.0 * (1.0 - (double) g[3] / (double) p));
    printf("Comm. volume / lower bound : %.2f\n", curr_comm_vol / min_comm_vol);
    printf("\n");
    /* per exec, the slowest rank's time of each phase */
    const char *names[6] = {"\nA, B, C redist   : ", "\nA / B allgather  : ",
                            "\n2D Cannon        : ", "\nC reduce-scatter : ",
                            "\nmatmul only      : ", "\ntotal execution  : "};
    const int src[6] = {0, -1, 1, 2, -2, 3};
    for (int row = 0; row < 6; row++) {
        printf("%s", names[row]);
        for (int t = 0; t < n_test; t++) {
            double v = 0.0;
            for (int r = 0; r < p; r++) {
                const double *ms = args[r].ms;
                double x = src[row] >= 0 ? ms[src[row] * n_test + t]
                           : src[row] == -2 ? ms[1 * n_test + t] + ms[2 * n_test + t] : 0.0;
                if (x > v) v = x;
            }
            printf("%.0lf ", v);
        }
    }
    printf("\n\n");
    if (chk) printf("CA3DMM output : %d error(s)\n", errors);
    for (int r = 0; r < p; r++) free(args[r].ms);
    free(args);
    free(tr);
    free(th);
    return errors ? 1 : 0;
}
