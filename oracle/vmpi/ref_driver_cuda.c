/* Driver of the reference's own GPU path under vmpi (TEST AND COMPARISON
 * INFRASTRUCTURE ONLY; context figures, never the product).
 *
 * Runs the unmodified reference (src/ca3dmm.c and friends compiled with
 * USE_CUDA, src/cuda_proxy.cu rebuilt for sm_100a) with DEV_TYPE_CUDA exactly
 * as examples/example_AB.c:100-190 drives it: p rank threads on one GPU, 1D
 * column partition of A, B and C, device input blocks filled through pinned
 * host mirrors, a caller-allocated work buffer (MALLOC_ATTACH_WORKBUF), one
 * warm-up exec, reset, ntest timed execs between barriers.  Every rank's
 * cuBLAS calls are serialised by ref_cuda_serial.c, since the reference keeps
 * one static cuBLAS handle per process (src/cuda_proxy.cu:151-174) and its
 * ranks are threads here. */
#include <stdlib.h>
#include <string.h>
#include <omp.h>
#include "mpi.h"
#include "cblas.h"
#include "ca3dmm.h"
#include "dev_type.h"

typedef struct {
    int m, n, k, ta, tb, btb, ntest;
    const int *grid;
    const double *A, *B;
    double *C;
    double *times;     /* [ntest][2]: exec ms, matmul-only ms (rank 0) */
    int *grid_out;
    int fail;
} cjob_t;

static double *to_device(const double *src, size_t count)
{
    size_t bytes = sizeof(double) * (count > 0 ? count : 1);
    double *h = (double *) dev_type_malloc(bytes, DEV_TYPE_HOST);
    double *d = (double *) dev_type_malloc(bytes, DEV_TYPE_CUDA);
    if (count > 0) memcpy(h, src, sizeof(double) * count);
    dev_type_memcpy(d, h, bytes, DEV_TYPE_CUDA, DEV_TYPE_HOST);
    dev_type_free(h, DEV_TYPE_HOST);
    return d;
}

static void rank_main_cuda(int rank, void *arg)
{
    cjob_t *j = (cjob_t *) arg;
    omp_set_num_threads(1);
    int p;
    MPI_Comm_size(MPI_COMM_WORLD, &p);
    const int a_nrow = j->ta ? j->k : j->m, a_ncol = j->ta ? j->m : j->k;
    const int b_nrow = j->btb ? j->k : (j->tb ? j->n : j->k);
    const int b_ncol = j->btb ? j->n : (j->tb ? j->k : j->n);
    const int c_nrow = j->btb ? j->n : j->m, c_ncol = j->n;
    int as, an, bs, bn, cs, cn;
    calc_block_spos_size(a_ncol, p, rank, &as, &an);
    calc_block_spos_size(b_ncol, p, rank, &bs, &bn);
    calc_block_spos_size(c_ncol, p, rank, &cs, &cn);
    double *A_d = NULL;
    double *B_d = to_device(j->B + (size_t) bs * b_nrow, (size_t) b_nrow * bn);
    if (!j->btb) A_d = to_device(j->A + (size_t) as * a_nrow, (size_t) a_nrow * an);
    size_t c_count = (size_t) c_nrow * cn;
    double *C_d = (double *) dev_type_malloc(sizeof(double) * (c_count > 0 ? c_count : 1),
                                             DEV_TYPE_CUDA);
    ca3dmm_engine_p ce = NULL;
    size_t wb = 0;
    if (j->btb)
        ca3dmm_engine_init_BTB(j->n, j->k, 0, b_nrow, bs, bn, 0, c_nrow, cs, cn, j->grid,
                               MPI_COMM_WORLD, DEV_TYPE_CUDA, &ce, &wb);
    else
        ca3dmm_engine_init(j->m, j->n, j->k, j->ta, j->tb, 0, a_nrow, as, an, 0, b_nrow, bs, bn,
                           0, c_nrow, cs, cn, j->grid, MPI_COMM_WORLD, DEV_TYPE_CUDA, &ce, &wb);
    void *wh = NULL, *wd = NULL;
    if (ce) MALLOC_ATTACH_WORKBUF(ca3dmm_engine_attach_workbuf, ca3dmm_engine_free, ce,
                                  DEV_TYPE_CUDA, wb, wh, wd);
    if (!ce) {
        j->fail = 1;
    } else {
        if (rank == 0) {
            j->grid_out[0] = ce->mp; j->grid_out[1] = ce->np; j->grid_out[2] = ce->kp;
            j->grid_out[3] = ce->rp;
        }
        ca3dmm_engine_exec(ce, A_d, a_nrow, B_d, b_nrow, C_d, c_nrow);      /* warm-up */
        ca3dmm_engine_reset_stat(ce);
        double agv = 0, can = 0, red = 0, ex = 0;
        for (int t = 0; t < j->ntest; t++) {
            MPI_Barrier(MPI_COMM_WORLD);
            ca3dmm_engine_exec(ce, A_d, a_nrow, B_d, b_nrow, C_d, c_nrow);
            if (rank == 0 && j->times) {
                j->times[2 * t] = ce->exec_ms - ex;
                j->times[2 * t + 1] = (ce->agvAB_ms - agv) + (ce->cannon_ms - can) +
                                      (ce->reduce_ms - red);
            }
            agv = ce->agvAB_ms; can = ce->cannon_ms; red = ce->reduce_ms; ex = ce->exec_ms;
        }
        if (c_count > 0) {
            double *h = (double *) dev_type_malloc(sizeof(double) * c_count, DEV_TYPE_HOST);
            dev_type_memcpy(h, C_d, sizeof(double) * c_count, DEV_TYPE_HOST, DEV_TYPE_CUDA);
            memcpy(j->C + (size_t) cs * c_nrow, h, sizeof(double) * c_count);
            dev_type_free(h, DEV_TYPE_HOST);
        }
        ca3dmm_engine_free(&ce);
    }
    dev_type_free(wh, DEV_TYPE_HOST);
    dev_type_free(wd, DEV_TYPE_CUDA);
    dev_type_free(A_d, DEV_TYPE_CUDA);
    dev_type_free(B_d, DEV_TYPE_CUDA);
    dev_type_free(C_d, DEV_TYPE_CUDA);
}

/* C = op(A) op(B) (btb = 0) or B^T B (btb = 1, A ignored) through the
 * reference's GPU path on p rank threads sharing one GPU.  A, B and C are
 * whole column-major host matrices.  Returns 0, or nonzero when a rank failed
 * or a wait timed out. */
int ref_ca3dmm_cuda(int p, int m, int n, int k, int ta, int tb, int btb, const int *grid,
                    const double *A, const double *B, double *C, int ntest, double *times,
                    int *grid_out, double timeout_s)
{
    openblas_set_num_threads(1);
    cjob_t j;
    memset(&j, 0, sizeof(j));
    j.m = m; j.n = n; j.k = k; j.ta = ta; j.tb = tb; j.btb = btb; j.ntest = ntest;
    j.grid = grid; j.A = A; j.B = B; j.C = C; j.times = times; j.grid_out = grid_out;
    int rc = vmpi_run(p, rank_main_cuda, &j, timeout_s);
    return rc || j.fail;
}
