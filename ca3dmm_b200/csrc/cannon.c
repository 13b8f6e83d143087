/* 2D Cannon engine folded onto one GPU (src/cannon.c:16-720).
 *
 * The np_dim x np_dim virtual ranks of the communicator hold the m x n x k
 * product between them; with every block in one HBM the initial skew and the
 * ring shifts are an indexing choice, so the np_dim shift-and-multiply steps
 * of every rank run as one grouped FP64 DMMA launch over the whole product
 * (C := alpha A B + beta C, src/cannon.c:406: beta on the first step only).
 * The caller's A / B are read in place when the TMA rules allow it (16-byte
 * aligned base, even leading dimension); otherwise they are first packed into
 * the engine's work buffer. */
#include <math.h>
#include <string.h>
#include <cuda_runtime_api.h>
#include "ca3dmm_util.h"
#include "ca3dmm_kernels.h"
#include "cannon.h"
#include "partition.h"

typedef struct {
    size_t off_plan, off_pack, off_A, off_B, total;
    void *stage;
    int *status_h;
    cudaEvent_t ev[2];
} cplan_t;

void cannon_engine_init(const int m, const int n, const int k, MPI_Comm comm, dev_type_t dev_type,
                        cannon_engine_p *engine_, size_t *workbuf_bytes)
{
    if (engine_ == NULL) return;
    *engine_ = NULL;
    if (is_dev_type_valid(dev_type) == 0) {
        ERROR_PRINTF("Invalid device type %d\n", dev_type);
        return;
    }
    int n_proc = ca3dmm_vcomm_size(comm);
    int np_dim = (int) sqrt((double) n_proc);
    if (n_proc < 1 || np_dim * np_dim != n_proc) {
        ERROR_PRINTF("Communicator size %d is not a square number\n", n_proc);
        return;
    }
    if (m < 0 || n < 0 || k < 0) {
        ERROR_PRINTF("Invalid matrix size m, n, k = %d, %d, %d\n", m, n, k);
        return;
    }
    double t0 = ca3dmm_wtime_sec();
    cannon_engine_p e = (cannon_engine_p) calloc(1, sizeof(cannon_engine_s));
    cplan_t *cp = (cplan_t *) calloc(1, sizeof(cplan_t));
    if (!e || !cp) { free(e); free(cp); return; }
    e->m = m; e->n = n; e->k = k;
    e->my_rank = 0; e->rank_row = 0; e->rank_col = 0;
    e->np_dim = np_dim;
    e->comm = comm;
    e->dev_type = dev_type;
    calc_block_spos_size(m, np_dim, 0, &e->A_srow, &e->A_nrow);
    calc_block_spos_size(k, np_dim, 0, &e->A_scol, &e->A_ncol);
    calc_block_spos_size(k, np_dim, 0, &e->B_srow, &e->B_nrow);
    calc_block_spos_size(n, np_dim, 0, &e->B_scol, &e->B_ncol);
    calc_block_spos_size(m, np_dim, 0, &e->C_srow, &e->C_nrow);
    calc_block_spos_size(n, np_dim, 0, &e->C_scol, &e->C_ncol);
    e->max_A_blk_size = (m / np_dim + 1) * (k / np_dim + 1);
    e->max_B_blk_size = (k / np_dim + 1) * (n / np_dim + 1);
    e->max_C_blk_size = (m / np_dim + 1) * (n / np_dim + 1);
    /* gemm_cycle as the reference computes it (src/cannon.c:86-99); the
     * folded engine always runs one GEMM over the whole k, so it is reported
     * only. */
    int min_k_blk_size;
    GET_ENV_INT_VAR(min_k_blk_size, "CANNON_MIN_KBLK_SIZE", "min_k_blk_size", 160, 16, 8192);
    e->gemm_cycle = 1;
    if (e->A_ncol > 0 && e->A_ncol < min_k_blk_size) {
        e->gemm_cycle = (min_k_blk_size + e->A_ncol - 1) / e->A_ncol;
        if (e->gemm_cycle > np_dim) e->gemm_cycle = np_dim;
    }
    e->m_displs = (int *) malloc(sizeof(int) * (np_dim + 1));
    e->n_displs = (int *) malloc(sizeof(int) * (np_dim + 1));
    e->k_displs = (int *) malloc(sizeof(int) * (np_dim + 1));
    int dummy;
    for (int i = 0; i <= np_dim; i++) {
        calc_block_spos_size(m, np_dim, i, e->m_displs + i, &dummy);
        calc_block_spos_size(n, np_dim, i, e->n_displs + i, &dummy);
        calc_block_spos_size(k, np_dim, i, e->k_displs + i, &dummy);
    }
    size_t off = 0;
    cp->off_plan = off; off += 256 + (ca3dmm_dgemm_plan_bytes(1) + 255) / 256 * 256;
    cp->off_pack = off; off += 256;
    cp->off_A = off; off += ((size_t) ca3dmm_round_up(m > 0 ? m : 1, 2) * (size_t) k * 8 + 255) / 256 * 256;
    cp->off_B = off; off += ((size_t) ca3dmm_round_up(k > 0 ? k : 1, 2) * (size_t) n * 8 + 255) / 256 * 256;
    cp->total = off;
    e->workbuf_bytes = off;
    e->impl = cp;
    if (cudaMallocHost(&cp->stage, 256 + ca3dmm_dgemm_plan_bytes(1) + 256) != cudaSuccess ||
        cudaMallocHost((void **) &cp->status_h, 64) != cudaSuccess) {
        cannon_engine_free(&e);
        return;
    }
    cudaEventCreate(&cp->ev[0]);
    cudaEventCreate(&cp->ev[1]);
    if (workbuf_bytes != NULL) {
        e->alloc_workbuf = 0;
        *workbuf_bytes = cp->total;
    } else {
        e->alloc_workbuf = 1;
        void *wh = NULL, *wd = NULL;
        MALLOC_ATTACH_WORKBUF(cannon_engine_attach_workbuf, cannon_engine_free, e, dev_type,
                              cp->total, wh, wd);
        if (e == NULL) return;
    }
    e->init_ms = 1000.0 * (ca3dmm_wtime_sec() - t0);
    *engine_ = e;
}

void cannon_engine_attach_workbuf(cannon_engine_p e, void *workbuf_h, void *workbuf_d)
{
    if (e == NULL) return;
    cplan_t *cp = (cplan_t *) e->impl;
    e->workbuf_h = workbuf_h;
    e->workbuf_d = workbuf_d;
    if (workbuf_d) {
        e->A_recv_d = (char *) workbuf_d + cp->off_A;
        e->B_recv_d = (char *) workbuf_d + cp->off_B;
    }
}

void cannon_engine_free(cannon_engine_p *engine_)
{
    if (engine_ == NULL || *engine_ == NULL) return;
    cannon_engine_p e = *engine_;
    cplan_t *cp = (cplan_t *) e->impl;
    if (e->alloc_workbuf && e->workbuf_d) dev_type_free(e->workbuf_d, DEV_TYPE_CUDA);
    free(e->m_displs);
    free(e->n_displs);
    free(e->k_displs);
    if (cp) {
        if (cp->stage) cudaFreeHost(cp->stage);
        if (cp->status_h) cudaFreeHost(cp->status_h);
        cudaEventDestroy(cp->ev[0]);
        cudaEventDestroy(cp->ev[1]);
        free(cp);
    }
    free(e);
    *engine_ = NULL;
}

static int tma_ok(const void *p, long long ld) { return ((uintptr_t) p % 16 == 0) && (ld % 2 == 0); }

static int cannon_exec_device(cannon_engine_p e, double alpha, double beta, const double *A,
                              const double *B, double *C)
{
    cplan_t *cp = (cplan_t *) e->impl;
    char *w = (char *) e->workbuf_d;
    if (!w) return CA3DMM_EINVAL;
    const int m = e->m, n = e->n, k = e->k;
    long long lda = m, ldb = k;
    char *h = (char *) cp->stage;
    /* pack misaligned operands into the work buffer (descriptor slots at off_pack) */
    const double *Ause = A, *Buse = B;
    if (!tma_ok(A, lda) && m > 0 && k > 0) {
        ca3dmm_pack_desc_t d;
        memset(&d, 0, sizeof(d));
        d.rows = m; d.cols = k; d.lds = lda; d.ldd = ca3dmm_round_up(m, 2);
        Ause = (const double *) e->A_recv_d;
        lda = d.ldd;
        int tiles = ca3dmm_pack_tiles(&d, 1);
        CA3DMM_CUDA_TRY(cudaMemcpy(w + cp->off_pack, &d, sizeof(d), cudaMemcpyHostToDevice));
        int rc = ca3dmm_pack_launch(A, (double *) e->A_recv_d,
                                    (const ca3dmm_pack_desc_t *) (w + cp->off_pack), 1, tiles, 0);
        if (rc) return rc;
    }
    if (!tma_ok(B, ldb) && k > 0 && n > 0) {
        ca3dmm_pack_desc_t d;
        memset(&d, 0, sizeof(d));
        d.rows = k; d.cols = n; d.lds = ldb; d.ldd = ca3dmm_round_up(k, 2);
        Buse = (const double *) e->B_recv_d;
        ldb = d.ldd;
        int tiles = ca3dmm_pack_tiles(&d, 1);
        CA3DMM_CUDA_TRY(cudaMemcpy(w + cp->off_pack + 64, &d, sizeof(d), cudaMemcpyHostToDevice));
        int rc = ca3dmm_pack_launch(B, (double *) e->B_recv_d,
                                    (const ca3dmm_pack_desc_t *) (w + cp->off_pack + 64), 1, tiles,
                                    0);
        if (rc) return rc;
    }
    ca3dmm_dgemm_desc_t g;
    memset(&g, 0, sizeof(g));
    g.A = Ause; g.lda = lda; g.B = Buse; g.ldb = ldb; g.C = C; g.ldc = m;
    g.m = m; g.n = n; g.k = k; g.alpha = alpha; g.beta = beta;
    int tiles = 0;
    int rc = ca3dmm_dgemm_plan_encode(&g, 1, h + 256, &tiles);
    if (rc) return rc;
    memset(h, 0, 256);
    CA3DMM_CUDA_TRY(cudaMemcpy(w + cp->off_plan, h, 256 + ca3dmm_dgemm_plan_bytes(1), cudaMemcpyHostToDevice));
    cudaEventRecord(cp->ev[0], 0);
    rc = ca3dmm_dgemm_launch(w + cp->off_plan + 256, 1, tiles, 0, (int *) (w + cp->off_plan), 5.0, 0);
    if (rc) return rc;
    cudaEventRecord(cp->ev[1], 0);
    CA3DMM_CUDA_TRY(cudaMemcpy(cp->status_h, w + cp->off_plan, sizeof(int), cudaMemcpyDeviceToHost));
    if (cp->status_h[0]) return CA3DMM_ETIMEOUT;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, cp->ev[0], cp->ev[1]);
    e->gemm_ms += ms;
    return CA3DMM_OK;
}

void cannon_engine_exec(cannon_engine_p e, const double alpha, const double beta, double *A_blk,
                        double *B_blk, double *C_blk)
{
    if (e == NULL) {
        ERROR_PRINTF("cannon_engine not initialized\n");
        return;
    }
    if (e->m == 0 || e->n == 0) return;
    double t0 = ca3dmm_wtime_sec();
    int rc = cannon_exec_device(e, alpha, beta, A_blk, B_blk, C_blk);
    e->last_error = rc;
    if (rc) {
        ERROR_PRINTF("cannon_engine_exec failed (error %d)\n", rc);
        return;
    }
    e->exec_ms += 1000.0 * (ca3dmm_wtime_sec() - t0);
    e->n_exec++;
}

void cannon_engine_reset_stat(cannon_engine_p e)
{
    if (e == NULL) return;
    e->shift0_ms = 0.0;
    e->lshift_ms = 0.0;
    e->gemm_ms = 0.0;
    e->hd_trans_ms = 0.0;
    e->exec_ms = 0.0;
    e->n_exec = 0;
}

void cannon_engine_print_stat(cannon_engine_p e)
{
    if (e == NULL) return;
    if (e->n_exec == 0) {
        WARNING_PRINTF("No cannon_engine statistic data to print\n");
        return;
    }
    double gf = (double) e->C_nrow * (double) e->C_ncol * (double) e->k;
    gf = gf * 2.0 * (double) e->n_exec / e->exec_ms * 1e3 / 1e9;
    printf("--------------- 2D Cannon algorithm engine ---------------\n");
    printf("* Initialization : %.2f ms\n", e->init_ms);
    printf("* Number of executions  : %d\n", e->n_exec);
    printf("* Execution time (avg)  : %.2f ms\n", e->exec_ms / e->n_exec);
    printf("  * Initial shift       : %.2f ms\n", e->shift0_ms / e->n_exec);
    printf("  * Loop shift wait     : %.2f ms\n", e->lshift_ms / e->n_exec);
    printf("  * Local DGEMM         : %.2f ms\n", e->gemm_ms / e->n_exec);
    printf("* Per-rank performance  : %.2f GFlops\n", gf);
    printf("----------------------------------------------------------\n");
}
