/* C = B^T B through the ca3dmm engine on one B200: the driver of the
 * reference's examples/example_BTB.c:17-184 on the folded engine, with the
 * same command line, fill and output lines.
 *
 *   [CA3DMM_VRANKS=p] example_btb m k check_correct n_test dev_type
 *
 * B is k x m with B(i, j) = 0.11 i + 0.12 j; the virtual rank count comes from
 * CA3DMM_VRANKS (default 1) in place of mpirun -np.  The check compares every
 * entry of C with the closed form
 *   C(i, j) = sum_l (0.11 l + 0.12 i)(0.11 l + 0.12 j)
 *           = 0.0121 S2 + 0.0132 (i + j) S1 + 0.0144 i j k,
 * S1 = sum_l l, S2 = sum_l l^2 (l < k), and counts relative differences above
 * 1e-12, as the reference does against cblas_dgemm. */
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
        printf("Usage: %s m k check_correct(0 or 1) n_test dev_type\n", argv[0]);
        return 0;
    }
    int m = get_int_param(argc, argv, 1, 4096, 1, 8388608);
    int n = m;
    int k = get_int_param(argc, argv, 2, 4096, 1, 8388608);
    int chk_res = get_int_param(argc, argv, 3, 1, 0, 1);
    int n_test = get_int_param(argc, argv, 4, 10, 1, 100);
    dev_type_t dev_type = get_int_param(argc, argv, 5, DEV_TYPE_CUDA, DEV_TYPE_CUDA,
                                        DEV_TYPE_CUDA_MPI_DIRECT);
    /* one process per GPU under an MPI launcher: this process' GPU, as the
     * reference's drivers choose it (examples/example_AB.c:43-46) */
    select_cuda_device_by_mpi_local_rank();
    const char *pv = getenv("CA3DMM_VRANKS");
    int n_proc = pv ? atoi(pv) : 1;
    if (n_proc < 1) n_proc = 1;
    MPI_Comm comm = NULL;
    if (ca3dmm_vcomm_create(n_proc, &comm) != 0) {
        fprintf(stderr, "invalid number of virtual ranks %d\n", n_proc);
        return 1;
    }

    printf("Test problem size m * n * k : %d * %d * %d\n", m, n, k);
    printf("Number of tests             : %d\n", n_test);
    printf("Check result correctness    : %d\n", chk_res);
    printf("Device type                 : %d\n", dev_type);
    printf("\n");
    fflush(stdout);

    const int B_nrow = k, B_ncol = n, C_nrow = n, C_ncol = n;
    const size_t B_msize = sizeof(double) * (size_t) B_nrow * (size_t) B_ncol;
    const size_t C_msize = sizeof(double) * (size_t) C_nrow * (size_t) C_ncol;
    double *B_h = (double *) malloc(B_msize), *C_h = (double *) malloc(C_msize);
    double *B_d = (double *) dev_type_malloc(B_msize, dev_type);
    double *C_d = (double *) dev_type_malloc(C_msize, dev_type);
    if (!B_h || !C_h || !B_d || !C_d) {
        fprintf(stderr, "allocation failed\n");
        return 1;
    }
    for (int j = 0; j < B_ncol; j++)
        for (int i = 0; i < B_nrow; i++)
            B_h[i + (size_t) j * B_nrow] = 0.11 * (double) i + 0.12 * (double) j;
    dev_type_memcpy(B_d, B_h, B_msize, dev_type, DEV_TYPE_HOST);

    ca3dmm_engine_p ce = NULL;
    size_t ce_workbuf_bytes = 0;
    ca3dmm_engine_init_BTB(n, k, 0, B_nrow, 0, B_ncol, 0, C_nrow, 0, C_ncol, NULL, comm, dev_type,
                           &ce, &ce_workbuf_bytes);
    void *workbuf_h = NULL, *workbuf_d = NULL;
    MALLOC_ATTACH_WORKBUF(ca3dmm_engine_attach_workbuf, ca3dmm_engine_free, ce, dev_type,
                          ce_workbuf_bytes, workbuf_h, workbuf_d);
    if (ce == NULL) {
        fprintf(stderr, "ca3dmm_engine_init_BTB failed\n");
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
        printf("\n");
        fflush(stdout);
    }

    ca3dmm_engine_exec(ce, NULL, 0, B_d, B_nrow, C_d, C_nrow);
    ca3dmm_engine_reset_stat(ce);
    for (int itest = 0; itest < n_test; itest++)
        ca3dmm_engine_exec(ce, NULL, 0, B_d, B_nrow, C_d, C_nrow);
    ca3dmm_engine_print_stat(ce);
    int rc = ca3dmm_engine_last_error(ce) ? 1 : 0;

    if (chk_res) {
        dev_type_memcpy(C_h, C_d, C_msize, DEV_TYPE_HOST, dev_type);
        const double kk = (double) k, S1 = kk * (kk - 1.0) / 2.0;
        const double S2 = (kk - 1.0) * kk * (2.0 * kk - 1.0) / 6.0;
        int errors = 0;
        for (int j = 0; j < C_ncol; j++)
            for (int i = 0; i < C_nrow; i++) {
                const double c = 0.11 * 0.11 * S2 + 0.11 * 0.12 * ((double) i + (double) j) * S1 +
                                 0.12 * 0.12 * (double) i * (double) j * kk;
                const double relerr = fabs((C_h[i + (size_t) j * C_nrow] - c) / c);
                if (relerr > 1e-12) errors++;
            }
        printf("CA3DMM output : %d error(s)\n", errors);
        if (errors) rc = 1;
    }
    free(B_h);
    free(C_h);
    dev_type_free(B_d, dev_type);
    dev_type_free(C_d, dev_type);
    ca3dmm_engine_free(&ce);
    dev_type_free(workbuf_d, dev_type);
    ca3dmm_vcomm_free(&comm);
    return rc;
}
