/* C = op(A) * op(B) through the ca3dmm engine on one B200: the driver of the
 * reference's examples/example_AB.c:17-316 on the folded engine, with the
 * same command line, the same deterministic fill and the same output lines,
 * so that scripts written for the reference's output parse this one.
 *
 *   [CA3DMM_VRANKS=p] example_ab m n k transA transB check_correct n_test dev_type [mp np kp]
 *
 * The reference's rank count comes from mpirun -np p; here the number of
 * virtual ranks comes from CA3DMM_VRANKS (default: mp * np * kp when a grid is
 * given, else 1).  dev_type is 1 (DEV_TYPE_CUDA) or 2 (DEV_TYPE_CUDA_MPI_DIRECT):
 * this engine has no host path.  The 1D column layout of the reference's ranks
 * concatenates to the whole matrix, which is what the folded call is given.
 * The check compares every C entry with the closed form of the fill
 *   op(A)(i, l) = a1 i + a2 l,  op(B)(l, j) = b1 l + b2 j,
 *   C(i, j) = a1 b1 i S1 + a1 b2 i j k + a2 b1 S2 + a2 b2 j S1,
 *   S1 = sum_l l, S2 = sum_l l^2 (l < k),
 * in place of the reference's cblas_dgemm, with the same rule: an entry is an
 * error when its relative difference exceeds 1e-12.  The GEMM mode comes from
 * CA3DMM_GEMM_MODE (0 plain FP64, 1 INT8 slices, 2 modular). */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <cuda_runtime_api.h>
#include "ca3dmm.h"
#include "cuda_proxy.h"

static int get_int_param(int argc, char **argv, int argi, int default_val, int min_val,
                         int max_val)
{
    int res = default_val;
    if (argc >= argi + 1) {
        res = atoi(argv[argi]);
        if (res < min_val || res > max_val) res = default_val;
    }
    return res;
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
    int trans_A = get_int_param(argc, argv, 4, 0, 0, 1);
    int trans_B = get_int_param(argc, argv, 5, 0, 0, 1);
    int chk_res = get_int_param(argc, argv, 6, 1, 0, 1);
    int n_test = get_int_param(argc, argv, 7, 10, 1, 100);
    dev_type_t dev_type = get_int_param(argc, argv, 8, DEV_TYPE_CUDA, DEV_TYPE_CUDA,
                                        DEV_TYPE_CUDA_MPI_DIRECT);
    int grid[3] = {0, 0, 0}, *proc_grid = NULL;
    if (argc >= 12) {
        grid[0] = atoi(argv[9]);
        grid[1] = atoi(argv[10]);
        grid[2] = atoi(argv[11]);
        proc_grid = grid;
    }
    /* one process per GPU under an MPI launcher: this process' GPU, as the
     * reference's drivers choose it (examples/example_AB.c:43-46) */
    select_cuda_device_by_mpi_local_rank();
    const char *pv = getenv("CA3DMM_VRANKS");
    int n_proc = pv ? atoi(pv) : (proc_grid ? grid[0] * grid[1] * grid[2] : 1);
    if (n_proc < 1) n_proc = 1;
    MPI_Comm comm = NULL;
    if (ca3dmm_vcomm_create(n_proc, &comm) != 0) {
        fprintf(stderr, "invalid number of virtual ranks %d\n", n_proc);
        return 1;
    }

    printf("Test problem size m * n * k : %d * %d * %d\n", m, n, k);
    printf("Transpose A / B             : %d / %d\n", trans_A, trans_B);
    printf("Number of tests             : %d\n", n_test);
    printf("Check result correctness    : %d\n", chk_res);
    printf("Device type                 : %d\n", dev_type);
    printf("\n");
    fflush(stdout);

    const int A_nrow = trans_A ? k : m, A_ncol = trans_A ? m : k;
    const int B_nrow = trans_B ? n : k, B_ncol = trans_B ? k : n;
    const int C_nrow = m, C_ncol = n;
    const size_t A_msize = sizeof(double) * (size_t) A_nrow * (size_t) A_ncol;
    const size_t B_msize = sizeof(double) * (size_t) B_nrow * (size_t) B_ncol;
    const size_t C_msize = sizeof(double) * (size_t) C_nrow * (size_t) C_ncol;
    double *A_h = (double *) malloc(A_msize), *B_h = (double *) malloc(B_msize);
    double *C_h = (double *) malloc(C_msize);
    double *A_d = (double *) dev_type_malloc(A_msize, dev_type);
    double *B_d = (double *) dev_type_malloc(B_msize, dev_type);
    double *C_d = (double *) dev_type_malloc(C_msize, dev_type);
    if (!A_h || !B_h || !C_h || !A_d || !B_d || !C_d) {
        fprintf(stderr, "allocation failed\n");
        return 1;
    }
    for (int j = 0; j < A_ncol; j++)
        for (int i = 0; i < A_nrow; i++)
            A_h[i + (size_t) j * A_nrow] = 0.19 * (double) i + 0.24 * (double) j;
    for (int j = 0; j < B_ncol; j++)
        for (int i = 0; i < B_nrow; i++)
            B_h[i + (size_t) j * B_nrow] = 0.11 * (double) i + 0.12 * (double) j;
    dev_type_memcpy(A_d, A_h, A_msize, dev_type, DEV_TYPE_HOST);
    dev_type_memcpy(B_d, B_h, B_msize, dev_type, DEV_TYPE_HOST);

    /* the whole matrices as the source blocks, the whole C as the output */
    ca3dmm_engine_p ce = NULL;
    size_t ce_workbuf_bytes = 0;
    ca3dmm_engine_init(m, n, k, trans_A, trans_B, 0, A_nrow, 0, A_ncol, 0, B_nrow, 0, B_ncol, 0,
                       C_nrow, 0, C_ncol, proc_grid, comm, dev_type, &ce, &ce_workbuf_bytes);
    void *workbuf_h = NULL, *workbuf_d = NULL;
    MALLOC_ATTACH_WORKBUF(ca3dmm_engine_attach_workbuf, ca3dmm_engine_free, ce, dev_type,
                          ce_workbuf_bytes, workbuf_h, workbuf_d);
    if (ce == NULL) {
        fprintf(stderr, "ca3dmm_engine_init failed\n");
        return 1;
    }
    {
        int mb = (m + ce->mp - 1) / ce->mp;
        int nb = (n + ce->np - 1) / ce->np;
        int kb = (k + ce->kp - 1) / ce->kp;
        double min_comm_vol = (double) m * (double) n * (double) k / (double) n_proc;
        min_comm_vol = 3.0 * pow(min_comm_vol, 2.0 / 3.0) * (double) n_proc;
        double curr_comm_vol = (double) mb * nb + (double) mb * kb + (double) nb * kb;
        curr_comm_vol *= (double) n_proc;
        printf("CA3DMM partition info:\n");
        printf("Process grid mp * np * kp  : %d * %d * %d\n", ce->mp, ce->np, ce->kp);
        printf("Work cuboid  mb * nb * kb  : %d * %d * %d\n", mb, nb, kb);
        printf("Process utilization        : %.2f %% \n",
               100.0 * (1.0 - (double) ce->rp / (double) n_proc));
        printf("Comm. volume / lower bound : %.2f\n", curr_comm_vol / min_comm_vol);
        printf("Rank 0 work buffer size    : %.2f MBytes\n", (double) ce_workbuf_bytes / 1048576.0);
        printf("\n");
        fflush(stdout);
    }

    /* warm-up, then n_test timed execs with the phase times of each */
    ca3dmm_engine_exec(ce, A_d, A_nrow, B_d, B_nrow, C_d, C_nrow);
    ca3dmm_engine_reset_stat(ce);
    double *mss = (double *) calloc(6 * (size_t) n_test, sizeof(double));
    double *redist_mss = mss, *agvAB_mss = mss + n_test, *cannon_mss = mss + 2 * n_test;
    double *reduce_mss = mss + 3 * n_test, *matmul_mss = mss + 4 * n_test, *exec_mss = mss + 5 * n_test;
    double redist_ms = 0.0, agvAB_ms = 0.0, cannon_ms = 0.0, reduce_ms = 0.0, exec_ms = 0.0;
    for (int i = 0; i < n_test; i++) {
        ca3dmm_engine_exec(ce, A_d, A_nrow, B_d, B_nrow, C_d, C_nrow);
        redist_mss[i] = ce->redist_ms - redist_ms;
        agvAB_mss[i] = ce->agvAB_ms - agvAB_ms;
        cannon_mss[i] = ce->cannon_ms - cannon_ms;
        reduce_mss[i] = ce->reduce_ms - reduce_ms;
        exec_mss[i] = ce->exec_ms - exec_ms;
        matmul_mss[i] = agvAB_mss[i] + cannon_mss[i] + reduce_mss[i];
        redist_ms = ce->redist_ms;
        agvAB_ms = ce->agvAB_ms;
        cannon_ms = ce->cannon_ms;
        reduce_ms = ce->reduce_ms;
        exec_ms = ce->exec_ms;
    }
    const char *names[6] = {"\nA, B, C redist   : ", "\nA / B allgather  : ",
                            "\n2D Cannon        : ", "\nC reduce-scatter : ",
                            "\nmatmul only      : ", "\ntotal execution  : "};
    for (int r = 0; r < 6; r++) {
        printf("%s", names[r]);
        for (int i = 0; i < n_test; i++) printf("%.0lf ", mss[r * n_test + i]);
    }
    printf("\n\n");
    ca3dmm_engine_print_stat(ce);
    free(mss);
    int rc = ca3dmm_engine_last_error(ce) ? 1 : 0;

    if (chk_res) {
        dev_type_memcpy(C_h, C_d, C_msize, DEV_TYPE_HOST, dev_type);
        const double a1 = trans_A ? 0.24 : 0.19, a2 = trans_A ? 0.19 : 0.24;
        const double b1 = trans_B ? 0.12 : 0.11, b2 = trans_B ? 0.11 : 0.12;
        const double kk = (double) k, S1 = kk * (kk - 1.0) / 2.0;
        const double S2 = (kk - 1.0) * kk * (2.0 * kk - 1.0) / 6.0;
        int errors = 0;
        for (int j = 0; j < C_ncol; j++)
            for (int i = 0; i < C_nrow; i++) {
                const double c = a1 * b1 * i * S1 + a1 * b2 * (double) i * (double) j * kk +
                                 a2 * b1 * S2 + a2 * b2 * j * S1;
                const double relerr = fabs((C_h[i + (size_t) j * C_nrow] - c) / c);
                if (relerr > 1e-12) errors++;
            }
        printf("CA3DMM output : %d error(s)\n", errors);
        if (errors) rc = 1;
    }
    free(A_h);
    free(B_h);
    free(C_h);
    dev_type_free(A_d, dev_type);
    dev_type_free(B_d, dev_type);
    dev_type_free(C_d, dev_type);
    ca3dmm_engine_free(&ce);
    dev_type_free(workbuf_d, dev_type);
    ca3dmm_vcomm_free(&comm);
    return rc;
}
