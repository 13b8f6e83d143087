/* Driver of the reference's own CPU path under vmpi (TEST INFRASTRUCTURE ONLY).
 *
 * Runs the unmodified reference (src/ca3dmm.c and friends, DEV_TYPE_HOST,
 * OpenBLAS) exactly as examples/example_AB.c and example_BTB.c drive it: p
 * rank threads, 1D column partition of A, B and C (example_AB.c:85-98), one
 * warm-up exec, reset, ntest timed execs (example_AB.c:168-190).  The caller
 * passes the whole A and B; each rank copies its columns and returns its C
 * columns, and every rank's engine fields in the 34-int geometry layout of
 * the oracle (orc_rank_geometry). */
#include <stdlib.h>
#include <string.h>
#include <omp.h>
#include "mpi.h"
#include "cblas.h"
#include "ca3dmm.h"
#include "mat_redist.h"

typedef struct {
    int m, n, k, ta, tb, btb, ntest;
    const int *grid;
    const double *A, *B;
    double *C;
    double *times;     /* [ntest][2]: exec ms, matmul-only ms (rank 0) */
    int *geom;         /* [p][34] */
    int *grid_out;     /* mp, np, kp, rp */
    int fail;
} job_t;

static void fields(ca3dmm_engine_p e, int *g)
{
    memset(g, 0, 34 * sizeof(int));
    g[0] = e->is_active;
    if (!e->is_active) return;
    g[1] = e->rank_m; g[2] = e->rank_n; g[3] = e->rank_k;
    g[4] = e->task_m_num; g[5] = e->task_m_id; g[6] = e->task_n_num; g[7] = e->task_n_id;
    g[8] = e->task_k_num; g[9] = e->task_k_id;
    g[10] = e->A_2dmm_srow; g[11] = e->A_2dmm_scol; g[12] = e->A_2dmm_nrow; g[13] = e->A_2dmm_ncol;
    g[14] = e->B_2dmm_srow; g[15] = e->B_2dmm_scol; g[16] = e->B_2dmm_nrow; g[17] = e->B_2dmm_ncol;
    g[18] = e->C_2dmm_srow; g[19] = e->C_2dmm_scol; g[20] = e->C_2dmm_nrow; g[21] = e->C_2dmm_ncol;
    g[22] = e->C_out_srow; g[23] = e->C_out_scol; g[24] = e->C_out_nrow; g[25] = e->C_out_ncol;
    g[26] = e->A_rd_srow; g[27] = e->A_rd_scol; g[28] = e->A_rd_nrow; g[29] = e->A_rd_ncol;
    g[30] = e->B_rd_srow; g[31] = e->B_rd_scol; g[32] = e->B_rd_nrow; g[33] = e->B_rd_ncol;
}

static void rank_main(int rank, void *arg)
{
    job_t *j = (job_t *) arg;
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
    double *A = NULL, *B = (double *) malloc(sizeof(double) * (size_t) b_nrow * (bn > 0 ? bn : 1));
    double *C = (double *) malloc(sizeof(double) * (size_t) c_nrow * (cn > 0 ? cn : 1));
    memcpy(B, j->B + (size_t) bs * b_nrow, sizeof(double) * (size_t) b_nrow * bn);
    if (!j->btb) {
        A = (double *) malloc(sizeof(double) * (size_t) a_nrow * (an > 0 ? an : 1));
        memcpy(A, j->A + (size_t) as * a_nrow, sizeof(double) * (size_t) a_nrow * an);
    }
    ca3dmm_engine_p ce = NULL;
    size_t wb = 0;
    if (j->btb)
        ca3dmm_engine_init_BTB(j->n, j->k, 0, b_nrow, bs, bn, 0, c_nrow, cs, cn, j->grid,
                               MPI_COMM_WORLD, DEV_TYPE_HOST, &ce, &wb);
    else
        ca3dmm_engine_init(j->m, j->n, j->k, j->ta, j->tb, 0, a_nrow, as, an, 0, b_nrow, bs, bn, 0,
                           c_nrow, cs, cn, j->grid, MPI_COMM_WORLD, DEV_TYPE_HOST, &ce, &wb);
    if (!ce) { j->fail = 1; free(A); free(B); free(C); return; }
    void *wh = malloc(wb > 0 ? wb : 8);
    ca3dmm_engine_attach_workbuf(ce, wh, NULL);
    fields(ce, j->geom + (size_t) rank * 34);
    if (rank == 0) {
        j->grid_out[0] = ce->mp; j->grid_out[1] = ce->np; j->grid_out[2] = ce->kp;
        j->grid_out[3] = ce->rp;
    }
    ca3dmm_engine_exec(ce, A, a_nrow, B, b_nrow, C, c_nrow);     /* warm-up */
    ca3dmm_engine_reset_stat(ce);
    double agv = 0, can = 0, red = 0, ex = 0;
    for (int t = 0; t < j->ntest; t++) {
        MPI_Barrier(MPI_COMM_WORLD);
        ca3dmm_engine_exec(ce, A, a_nrow, B, b_nrow, C, c_nrow);
        if (rank == 0 && j->times) {
            j->times[2 * t] = ce->exec_ms - ex;
            j->times[2 * t + 1] = (ce->agvAB_ms - agv) + (ce->cannon_ms - can) + (ce->reduce_ms - red);
        }
        agv = ce->agvAB_ms; can = ce->cannon_ms; red = ce->reduce_ms; ex = ce->exec_ms;
    }
    memcpy(j->C + (size_t) cs * c_nrow, C, sizeof(double) * (size_t) c_nrow * cn);
    ca3dmm_engine_free(&ce);
    free(wh); free(A); free(B); free(C);
}

/* C = op(A) op(B) (btb = 0) or B^T B (btb = 1, A ignored) on p rank threads.
 * Returns 0, or nonzero when a rank failed or a wait timed out. */
int ref_ca3dmm(int p, int m, int n, int k, int ta, int tb, int btb, const int *grid,
               const double *A, const double *B, double *C, int ntest, double *times, int *geom,
               int *grid_out, double timeout_s)
{
    openblas_set_num_threads(1);
    job_t j;
    memset(&j, 0, sizeof(j));
    j.m = m; j.n = n; j.k = k; j.ta = ta; j.tb = tb; j.btb = btb; j.ntest = ntest;
    j.grid = grid; j.A = A; j.B = B; j.C = C; j.times = times; j.geom = geom;
    j.grid_out = grid_out;
    int rc = vmpi_run(p, rank_main, &j, timeout_s);
    return rc || j.fail;
}

/* Fault injection for the harness tests: rank `dead` returns at once, the
 * others run one ca3dmm_engine_init; vmpi must report the failure by
 * timeout instead of hanging. */
typedef struct { int dead, m; } fault_t;

static void fault_main(int rank, void *arg)
{
    fault_t *f = (fault_t *) arg;
    if (rank == f->dead) return;
    omp_set_num_threads(1);
    int p;
    MPI_Comm_size(MPI_COMM_WORLD, &p);
    int s, z;
    calc_block_spos_size(f->m, p, rank, &s, &z);
    ca3dmm_engine_p ce = NULL;
    size_t wb;
    ca3dmm_engine_init(f->m, f->m, f->m, 0, 0, 0, f->m, s, z, 0, f->m, s, z, -1, -1, -1, -1, NULL,
                       MPI_COMM_WORLD, DEV_TYPE_HOST, &ce, &wb);
    /* the partial engine is leaked on purpose: its peer is gone */
}

int ref_fault_run(int p, int dead_rank, int m, double timeout_s)
{
    fault_t f = {dead_rank, m};
    return vmpi_run(p, fault_main, &f, timeout_s);
}

/* The reference's mat_redist (src/mat_redist.c) on p rank threads: rank r owns
 * source rectangle src_rects[4r..] and requires req_rects[4r..] (row-major
 * view, {srow, scol, nrow, ncol}) of a row-major matrix G (ldg columns).  Each
 * rank fills its source block from G, runs mat_redist_engine_init/exec with
 * DEV_TYPE_HOST, and writes its required block to out at out_offs[r] (row-major,
 * ld = its ncol).  Returns 0, or nonzero when a rank failed or timed out. */
typedef struct {
    const int *src, *req;
    const double *G;
    int ldg;
    double *out;
    const long long *offs;
    int fail;
} redist_t;

static void redist_main(int rank, void *arg)
{
    redist_t *j = (redist_t *) arg;
    omp_set_num_threads(1);
    const int *s = j->src + 4 * rank, *r = j->req + 4 * rank;
    double *sb = (double *) malloc(sizeof(double) * ((size_t) s[2] * s[3] + 1));
    double *db = (double *) calloc((size_t) r[2] * r[3] + 1, sizeof(double));
    for (int i = 0; i < s[2]; i++)
        for (int c = 0; c < s[3]; c++)
            sb[(size_t) i * s[3] + c] = j->G[(size_t) (s[0] + i) * j->ldg + s[1] + c];
    mat_redist_engine_p e = NULL;
    mat_redist_engine_init(s[0], s[1], s[2], s[3], r[0], r[1], r[2], r[3], MPI_COMM_WORLD,
                           MPI_DOUBLE, sizeof(double), DEV_TYPE_HOST, &e, NULL);
    if (e == NULL) {
        j->fail = 1;
    } else {
        mat_redist_engine_exec(e, sb, s[3] > 0 ? s[3] : 1, db, r[3] > 0 ? r[3] : 1);
        memcpy(j->out + j->offs[rank], db, sizeof(double) * (size_t) r[2] * r[3]);
        mat_redist_engine_free(&e);
    }
    free(sb);
    free(db);
}

int ref_redist(int p, const int *src_rects, const int *req_rects, const double *G, int ldg,
               double *out, const long long *out_offs, double timeout_s)
{
    redist_t j = {src_rects, req_rects, G, ldg, out, out_offs, 0};
    int rc = vmpi_run(p, redist_main, &j, timeout_s);
    return rc || j.fail;
}
