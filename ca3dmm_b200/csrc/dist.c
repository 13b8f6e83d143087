/* CA3DMM over several GPUs from C (include/ca3dmm_dist.h): every rank's grid
 * geometry from the folded engine's arithmetic (ca3dmm_engine_vrank_info,
 * src/ca3dmm.c:23-722), the operand and C exchange plans, and an exec of
 * batched rectangle copies (mat_redist_layouts), the transport's all-to-all,
 * the single-GPU engine for the local GEMM and the slab-ordered sum. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <cuda_runtime_api.h>
#include "ca3dmm_util.h"
#include "ca3dmm_kernels.h"
#include "ca3dmm.h"
#include "ca3dmm_dist.h"

enum { MAT_A = 0, MAT_B = 1 };

typedef struct {
    int r0, nr, c0, nc;         /* srow, nrow, scol, ncol (column-major) */
} rect_t;

typedef struct {
    int mat;
    rect_t x;
    long long off;              /* element offset in the exchange buffer */
    int slab;                   /* C pieces: the sender's slab */
} piece_t;

struct ca3dmm_dist_engine {
    ca3dmm_transport_t tr;
    int W, me, btb, m, n, k, ta, tb, mode, slices;
    int mp, np, kp, rp;
    rect_t *srcA, *srcB, *dstC, *cblk;
    int *active, *slab, *k0, *kz;
    int nuniq;                  /* this rank's distinct panels (1 or 2) */
    int umat[2];
    rect_t urect[2];
    int panel_of[2];            /* index into the distinct panels of op(A) / op(B) */
    piece_t *send, *recv, *csend, *crecv;
    int nsend, nrecv, ncsend, ncrecv;
    long long *scnt, *sdsp, *rcnt, *rdsp, *cscnt, *csdsp, *crcnt, *crdsp;
    long long stot, rtot, cstot, crtot;
    /* device side, made at the first exec */
    int ready;
    mat_redist_layouts_p pack_ab, unpack_ab, pack_c, unpack_c;
    int nmy;                    /* my source blocks in pack_ab (A then B) */
    int mymat[2];
    ca3dmm_engine_p local;
    MPI_Comm local_comm;
    double *d_send, *d_recv, *d_panel[2], *d_cbuf, *d_csend, *d_crecv, *d_layers;
    double *h_send, *h_recv;    /* host staging (transports without device buffers) */
    int whole;                  /* one rank holding everything on a 1 x 1 x 1 grid */
    double st[4];
    int n_exec;
};

static rect_t mk(int r0, int nr, int c0, int nc)
{
    rect_t r = {r0, nr, c0, nc};
    return r;
}

static long long area(rect_t r) { return (long long) r.nr * (long long) r.nc; }

static int inter(rect_t a, rect_t b, rect_t *o)
{
    const int r0 = a.r0 > b.r0 ? a.r0 : b.r0, r1 = (a.r0 + a.nr < b.r0 + b.nr) ? a.r0 + a.nr : b.r0 + b.nr;
    const int c0 = a.c0 > b.c0 ? a.c0 : b.c0, c1 = (a.c0 + a.nc < b.c0 + b.nc) ? a.c0 + a.nc : b.c0 + b.nc;
    if (r1 <= r0 || c1 <= c0) return 0;
    *o = mk(r0, r1 - r0, c0, c1 - c0);
    return 1;
}

static int same(rect_t a, rect_t b)
{
    return a.r0 == b.r0 && a.nr == b.nr && a.c0 == b.c0 && a.nc == b.nc;
}

static rect_t src_of(const struct ca3dmm_dist_engine *e, int mat, int r)
{
    return (mat == MAT_B || e->btb) ? e->srcB[r] : e->srcA[r];
}

/* rank r's op(A) and op(B) panels in the stored matrices' coordinates */
static void panels_of(const struct ca3dmm_dist_engine *e, int r, int mat[2], rect_t rc[2])
{
    if (!e->active[r]) {
        mat[0] = MAT_A; mat[1] = MAT_B;
        rc[0] = rc[1] = mk(0, 0, 0, 0);
        return;
    }
    const rect_t c = e->cblk[r];
    const int k0 = e->k0[r], kz = e->kz[r];
    if (e->btb) {              /* op(A) = B^T: rows k, columns = C rows */
        mat[0] = mat[1] = MAT_B;
        rc[0] = mk(k0, kz, c.r0, c.nr);
        rc[1] = mk(k0, kz, c.c0, c.nc);
        return;
    }
    mat[0] = MAT_A;
    mat[1] = MAT_B;
    rc[0] = e->ta ? mk(k0, kz, c.r0, c.nr) : mk(c.r0, c.nr, k0, kz);
    rc[1] = e->tb ? mk(c.c0, c.nc, k0, kz) : mk(k0, kz, c.c0, c.nc);
}

static int uniq_of(const struct ca3dmm_dist_engine *e, int r, int mat[2], rect_t rc[2])
{
    int pm[2];
    rect_t pr[2];
    panels_of(e, r, pm, pr);
    mat[0] = pm[0];
    rc[0] = pr[0];
    if (pm[1] == pm[0] && same(pr[1], pr[0])) return 1;
    mat[1] = pm[1];
    rc[1] = pr[1];
    return 2;
}

/* stacking offset (columns) of a matrix in the batched copies, so that pieces
 * of A and B never meet: B after the stored A's columns */
static int moff(const struct ca3dmm_dist_engine *e, int mat)
{
    if (mat == MAT_A || e->btb) return 0;
    return e->ta ? e->m : e->k;
}

/* a column-major rectangle at stacking offset `off` as the row-major
 * rectangle {srow, scol, nrow, ncol} of the transposed matrix */
static void rm(rect_t r, int off, int *out)
{
    out[0] = r.c0 + off;
    out[1] = r.r0;
    out[2] = r.nc;
    out[3] = r.nr;
}

static void *xcalloc(size_t n, size_t s) { return calloc(n ? n : 1, s); }

static int plan_operands(struct ca3dmm_dist_engine *e)
{
    const int W = e->W, me = e->me;
    e->send = (piece_t *) xcalloc((size_t) 2 * W, sizeof(piece_t));
    e->recv = (piece_t *) xcalloc((size_t) 2 * W, sizeof(piece_t));
    e->scnt = (long long *) xcalloc(W, sizeof(long long));
    e->sdsp = (long long *) xcalloc(W, sizeof(long long));
    e->rcnt = (long long *) xcalloc(W, sizeof(long long));
    e->rdsp = (long long *) xcalloc(W, sizeof(long long));
    if (!e->send || !e->recv || !e->scnt || !e->sdsp || !e->rcnt || !e->rdsp) return CA3DMM_ENOMEM;
    long long tot = 0;
    for (int d = 0; d < W; d++) {
        int um[2];
        rect_t ur[2];
        const int nu = uniq_of(e, d, um, ur);
        e->sdsp[d] = tot;
        for (int u = 0; u < nu; u++) {
            rect_t x;
            if (!inter(src_of(e, um[u], me), ur[u], &x)) continue;
            piece_t p = {um[u], x, tot, 0};
            e->send[e->nsend++] = p;
            tot += area(x);
        }
        e->scnt[d] = tot - e->sdsp[d];
    }
    e->stot = tot;
    e->nuniq = uniq_of(e, me, e->umat, e->urect);
    tot = 0;
    for (int q = 0; q < W; q++) {
        e->rdsp[q] = tot;
        for (int u = 0; u < e->nuniq; u++) {
            rect_t x;
            if (!inter(src_of(e, e->umat[u], q), e->urect[u], &x)) continue;
            piece_t p = {e->umat[u], x, tot, 0};
            e->recv[e->nrecv++] = p;
            tot += area(x);
        }
        e->rcnt[q] = tot - e->rdsp[q];
    }
    e->rtot = tot;
    int pm[2];
    rect_t pr[2];
    panels_of(e, me, pm, pr);
    for (int i = 0; i < 2; i++)
        e->panel_of[i] = (e->nuniq == 2 && (pm[i] != e->umat[0] || !same(pr[i], e->urect[0]))) ? 1 : 0;
    return CA3DMM_OK;
}

static int plan_c(struct ca3dmm_dist_engine *e)
{
    const int W = e->W, me = e->me;
    e->csend = (piece_t *) xcalloc(W, sizeof(piece_t));
    e->crecv = (piece_t *) xcalloc(W, sizeof(piece_t));
    e->cscnt = (long long *) xcalloc(W, sizeof(long long));
    e->csdsp = (long long *) xcalloc(W, sizeof(long long));
    e->crcnt = (long long *) xcalloc(W, sizeof(long long));
    e->crdsp = (long long *) xcalloc(W, sizeof(long long));
    if (!e->csend || !e->crecv || !e->cscnt || !e->csdsp || !e->crcnt || !e->crdsp)
        return CA3DMM_ENOMEM;
    long long tot = 0;
    for (int d = 0; d < W; d++) {
        rect_t x;
        e->csdsp[d] = tot;
        if (e->active[me] && inter(e->cblk[me], e->dstC[d], &x)) {
            piece_t p = {0, x, tot, 0};
            e->csend[e->ncsend++] = p;
            tot += area(x);
        }
        e->cscnt[d] = tot - e->csdsp[d];
    }
    e->cstot = tot;
    tot = 0;
    for (int q = 0; q < W; q++) {
        rect_t x;
        e->crdsp[q] = tot;
        if (e->active[q] && inter(e->cblk[q], e->dstC[me], &x)) {
            piece_t p = {0, x, tot, e->slab[q]};
            e->crecv[e->ncrecv++] = p;
            tot += area(x);
        }
        e->crcnt[q] = tot - e->crdsp[q];
    }
    e->crtot = tot;
    return CA3DMM_OK;
}

int ca3dmm_dist_engine_init(int m, int n, int k, int trans_A, int trans_B, int btb,
                            int src_A_srow, int src_A_nrow, int src_A_scol, int src_A_ncol,
                            int src_B_srow, int src_B_nrow, int src_B_scol, int src_B_ncol,
                            int dst_C_srow, int dst_C_nrow, int dst_C_scol, int dst_C_ncol,
                            const int *proc_grid, const ca3dmm_transport_t *tr, int gemm_mode,
                            int slices, ca3dmm_dist_engine_p *out)
{
    if (!out || !tr || tr->size < 1 || tr->rank < 0 || tr->rank >= tr->size || !tr->allgather_ll ||
        !tr->alltoallv_d)
        return CA3DMM_EINVAL;
    *out = NULL;
    struct ca3dmm_dist_engine *e = (struct ca3dmm_dist_engine *) calloc(1, sizeof(*e));
    if (!e) return CA3DMM_ENOMEM;
    e->tr = *tr;
    const int W = tr->size;
    e->W = W;
    e->me = tr->rank;
    e->btb = btb ? 1 : 0;
    e->m = btb ? n : m;
    e->n = n;
    e->k = k;
    e->ta = btb ? 1 : (trans_A ? 1 : 0);
    e->tb = btb ? 0 : (trans_B ? 1 : 0);
    e->mode = gemm_mode;
    e->slices = slices;
    /* every rank's rectangles and arguments: each rank checks all of them, so
     * an inconsistent call fails on every rank before any exchange */
    enum { NV = 23 };
    long long mine[NV] = {btb ? 0 : src_A_srow, btb ? 0 : src_A_nrow, btb ? 0 : src_A_scol,
                          btb ? 0 : src_A_ncol, src_B_srow, src_B_nrow, src_B_scol, src_B_ncol,
                          dst_C_srow, dst_C_nrow, dst_C_scol, dst_C_ncol, m, n, k, e->ta, e->tb,
                          e->btb, gemm_mode, slices, proc_grid ? proc_grid[0] : -1,
                          proc_grid ? proc_grid[1] : -1, proc_grid ? proc_grid[2] : -1};
    long long *all = (long long *) xcalloc((size_t) W * NV, sizeof(long long));
    e->srcA = (rect_t *) xcalloc(W, sizeof(rect_t));
    e->srcB = (rect_t *) xcalloc(W, sizeof(rect_t));
    e->dstC = (rect_t *) xcalloc(W, sizeof(rect_t));
    e->cblk = (rect_t *) xcalloc(W, sizeof(rect_t));
    e->active = (int *) xcalloc(W, sizeof(int));
    e->slab = (int *) xcalloc(W, sizeof(int));
    e->k0 = (int *) xcalloc(W, sizeof(int));
    e->kz = (int *) xcalloc(W, sizeof(int));
    int rc = (!all || !e->srcA || !e->srcB || !e->dstC || !e->cblk || !e->active || !e->slab ||
              !e->k0 || !e->kz) ? CA3DMM_ENOMEM : CA3DMM_OK;
    if (!rc && tr->allgather_ll(tr->ctx, mine, NV, all)) rc = CA3DMM_ECUDA;
    for (int r = 0; r < W && !rc; r++) {
        const long long *a = all + (size_t) r * NV;
        for (int i = 12; i < NV; i++)
            if (a[i] != all[i]) {
                if (e->me == 0) ERROR_PRINTF("ranks disagree on m, n, k, transposes, mode or grid\n");
                rc = CA3DMM_EINVAL;
                break;
            }
        e->srcA[r] = mk((int) a[0], (int) a[1], (int) a[2], (int) a[3]);
        e->srcB[r] = mk((int) a[4], (int) a[5], (int) a[6], (int) a[7]);
        e->dstC[r] = mk((int) a[8], (int) a[9], (int) a[10], (int) a[11]);
    }
    free(all);
    if (!rc && (m < 1 || n < 1 || k < 1 || gemm_mode < 0 || gemm_mode > 2)) rc = CA3DMM_EINVAL;
    /* rectangles inside their matrices */
    const int a_r = e->ta ? k : m, a_c = e->ta ? m : k;
    const int b_r = btb ? k : (e->tb ? n : k), b_c = btb ? n : (e->tb ? k : n);
    for (int r = 0; r < W && !rc; r++) {
        const rect_t *chk[3] = {&e->srcA[r], &e->srcB[r], &e->dstC[r]};
        const int rows[3] = {a_r, b_r, e->m}, cols[3] = {a_c, b_c, e->n};
        for (int t = btb ? 1 : 0; t < 3; t++) {
            const rect_t x = *chk[t];
            if (x.r0 < 0 || x.nr < 0 || x.c0 < 0 || x.nc < 0 || x.r0 + x.nr > rows[t] ||
                x.c0 + x.nc > cols[t]) {
                if (e->me == 0)
                    ERROR_PRINTF("rank %d's %s rectangle (%d, %d, %d, %d) is outside the %d x %d "
                                 "matrix\n", r, t == 0 ? "src_A" : t == 1 ? "src_B" : "dst_C",
                                 x.r0, x.nr, x.c0, x.nc, rows[t], cols[t]);
                rc = CA3DMM_EINVAL;
            }
        }
    }
    /* the reference's grid and every rank's cuboid: the folded engine's
     * arithmetic for p = W (no CUDA call) */
    if (!rc) {
        MPI_Comm vc = NULL;
        ca3dmm_engine_p geo = NULL;
        size_t wb = 0;
        if (ca3dmm_vcomm_create(W, &vc)) rc = CA3DMM_EINVAL;
        if (!rc && btb)
            ca3dmm_engine_init_BTB(n, k, 0, k, 0, n, 0, n, 0, n, proc_grid, vc, DEV_TYPE_CUDA, &geo,
                                   &wb);
        else if (!rc)
            ca3dmm_engine_init(m, n, k, e->ta, e->tb, 0, a_r, 0, a_c, 0, b_r, 0, b_c, 0, m, 0, n,
                               proc_grid, vc, DEV_TYPE_CUDA, &geo, &wb);
        if (!rc && !geo) rc = CA3DMM_EINVAL;
        if (!rc) {
            e->mp = geo->mp; e->np = geo->np; e->kp = geo->kp; e->rp = geo->rp;
            for (int r = 0; r < W; r++) {
                int g[34];
                ca3dmm_engine_vrank_info(geo, r, g);
                e->active[r] = g[0];
                e->slab[r] = g[0] ? g[9] : -1;
                e->cblk[r] = g[0] ? mk(g[18], g[20], g[19], g[21]) : mk(0, 0, 0, 0);
                if (g[0]) calc_block_spos_size(k, e->kp, g[9], &e->k0[r], &e->kz[r]);
            }
        }
        if (geo) ca3dmm_engine_free(&geo);
        if (vc) ca3dmm_vcomm_free(&vc);
    }
    /* the active ranks of each slab tile C; every panel is covered */
    if (!rc) {
        long long *cover = (long long *) xcalloc(e->kp, sizeof(long long));
        for (int r = 0; r < W && cover; r++)
            if (e->active[r]) cover[e->slab[r]] += area(e->cblk[r]);
        for (int s = 0; s < e->kp && cover && !rc; s++)
            if (cover[s] != (long long) e->m * e->n) rc = CA3DMM_EINVAL;
        free(cover);
        for (int r = 0; r < W && !rc; r++) {
            int um[2];
            rect_t ur[2];
            const int nu = uniq_of(e, r, um, ur);
            for (int u = 0; u < nu && !rc; u++) {
                long long got = 0;
                for (int q = 0; q < W; q++) {
                    rect_t x;
                    if (inter(src_of(e, um[u], q), ur[u], &x)) got += area(x);
                }
                if (got < area(ur[u])) {
                    if (e->me == 0)
                        ERROR_PRINTF("the source blocks do not cover rank %d's %s panel\n", r,
                                     um[u] == MAT_A ? "A" : "B");
                    rc = CA3DMM_EINVAL;
                }
            }
        }
    }
    if (!rc) rc = plan_operands(e);
    if (!rc) rc = plan_c(e);
    if (!rc && W == 1 && e->kp == 1) {
        const int full_a = btb || (e->srcA[0].r0 == 0 && e->srcA[0].nr == a_r && e->srcA[0].c0 == 0 &&
                                   e->srcA[0].nc == a_c);
        const int full_b = e->srcB[0].r0 == 0 && e->srcB[0].nr == b_r && e->srcB[0].c0 == 0 &&
                           e->srcB[0].nc == b_c;
        const int full_c = e->dstC[0].r0 == 0 && e->dstC[0].nr == e->m && e->dstC[0].c0 == 0 &&
                           e->dstC[0].nc == e->n;
        e->whole = full_a && full_b && full_c;
    }
    if (rc) {
        ca3dmm_dist_engine_free(&e);
        return rc;
    }
    *out = e;
    return CA3DMM_OK;
}

/* device side: buffers, batched copies and the local engine */
static int prepare(struct ca3dmm_dist_engine *e)
{
    if (e->ready) return CA3DMM_OK;
    const int me = e->me;
    int rc = CA3DMM_OK;
    const rect_t c = e->cblk[me];
    /* idempotent: a retry after a failed attempt reuses what was made */
    if (!e->local && e->active[me] && c.nr > 0 && c.nc > 0 && e->kz[me] > 0) {
        int pm[2];
        rect_t pr[2];
        panels_of(e, me, pm, pr);
        if (!e->local_comm && ca3dmm_vcomm_create(1, &e->local_comm)) return CA3DMM_EINVAL;
        const int ar = pr[0].nr, ac = pr[0].nc, br = pr[1].nr, bc = pr[1].nc;
        ca3dmm_engine_init(c.nr, c.nc, e->kz[me], e->ta, e->tb, 0, ar, 0, ac, 0, br, 0, bc, 0, c.nr,
                           0, c.nc, NULL, e->local_comm, DEV_TYPE_CUDA, &e->local, NULL);
        if (!e->local) return CA3DMM_EINVAL;
        if (e->mode != CA3DMM_GEMM_PLAIN &&
            (rc = ca3dmm_engine_set_gemm_mode(e->local, e->mode, e->slices)) != 0)
            return rc;
    }
    if (e->whole) {
        e->ready = 1;
        return CA3DMM_OK;
    }
#define DALLOC(p, n)                                                                        \
    do {                                                                                    \
        if (!(p) && cudaMalloc((void **) &(p), sizeof(double) * (size_t) ((n) > 0 ? (n) : 1)) != \
                        cudaSuccess) {                                                      \
            (p) = NULL;                                                                     \
            return CA3DMM_ENOMEM;                                                           \
        }                                                                                   \
    } while (0)
    DALLOC(e->d_send, e->stot);
    DALLOC(e->d_recv, e->rtot);
    for (int u = 0; u < e->nuniq; u++) DALLOC(e->d_panel[u], area(e->urect[u]));
    DALLOC(e->d_cbuf, e->active[me] ? area(c) : 0);
    DALLOC(e->d_csend, e->cstot);
    DALLOC(e->d_crecv, e->crtot);
    DALLOC(e->d_layers, (long long) e->kp * area(e->dstC[me]));
#undef DALLOC
    if (!e->tr.device_buffers && !e->h_send) {
        size_t hb = sizeof(double) * (size_t) (1 + (e->stot > e->cstot ? e->stot : e->cstot));
        size_t rb = sizeof(double) * (size_t) (1 + (e->rtot > e->crtot ? e->rtot : e->crtot));
        if (cudaMallocHost((void **) &e->h_send, hb) != cudaSuccess ||
            cudaMallocHost((void **) &e->h_recv, rb) != cudaSuccess)
            return CA3DMM_ENOMEM;
    }
    /* operands: my blocks -> send pieces; received pieces -> my panels */
    const int nmats = e->btb ? 1 : 2;
    /* rectangle lists of the four batched copies, in turn: my blocks (<= 2) /
     * send pieces, received pieces / my panels (<= 2), my C block (1) / C
     * send pieces */
    const size_t nrect = (size_t) 2 + (size_t) e->nsend + (size_t) e->nrecv + (size_t) e->ncsend;
    int *sr = (int *) xcalloc(4 * nrect, sizeof(int));
    int *dr = (int *) xcalloc(4 * nrect, sizeof(int));
    if (!sr || !dr) { free(sr); free(dr); return CA3DMM_ENOMEM; }
    e->nmy = 0;
    for (int t = 0; t < nmats; t++) {
        const int mat = e->btb ? MAT_B : t;
        const rect_t s = src_of(e, mat, me);
        if (area(s) > 0) {
            rm(s, moff(e, mat), sr + 4 * e->nmy);
            e->mymat[e->nmy++] = mat;
        }
    }
    for (int i = 0; i < e->nsend; i++) rm(e->send[i].x, moff(e, e->send[i].mat), dr + 4 * i);
    if (e->nmy > 0 && e->nsend > 0 && !e->pack_ab)
        rc = mat_redist_layouts_init(e->nmy, sr, e->nsend, dr, &e->pack_ab);
    for (int i = 0; !rc && i < e->nrecv; i++) rm(e->recv[i].x, moff(e, e->recv[i].mat), sr + 4 * i);
    for (int u = 0; !rc && u < e->nuniq; u++) rm(e->urect[u], moff(e, e->umat[u]), dr + 4 * u);
    if (!rc && e->nrecv > 0 && e->nuniq > 0 && area(e->urect[0]) > 0 && !e->unpack_ab)
        rc = mat_redist_layouts_init(e->nrecv, sr, e->nuniq, dr, &e->unpack_ab);
    /* C: my C_2dmm block -> send pieces; received pieces -> slab layers of dst_C */
    const rect_t d = e->dstC[me];
    const int layers = e->kp > 1 ? e->kp : 1;
    if (!rc && e->active[me] && area(c) > 0 && e->ncsend > 0 && !e->pack_c) {
        rm(c, 0, sr);
        for (int i = 0; i < e->ncsend; i++) rm(e->csend[i].x, 0, dr + 4 * i);
        rc = mat_redist_layouts_init(1, sr, e->ncsend, dr, &e->pack_c);
    }
    if (!rc && area(d) > 0 && e->ncrecv > 0 && !e->unpack_c) {
        int *s2 = (int *) xcalloc(4 * (size_t) e->ncrecv, sizeof(int));
        int *d2 = (int *) xcalloc(4 * (size_t) layers, sizeof(int));
        if (!s2 || !d2) rc = CA3DMM_ENOMEM;
        for (int i = 0; !rc && i < e->ncrecv; i++)
            rm(e->crecv[i].x, (e->kp > 1 ? e->crecv[i].slab : 0) * e->n, s2 + 4 * i);
        for (int j = 0; !rc && j < layers; j++) rm(d, j * e->n, d2 + 4 * j);
        if (!rc) rc = mat_redist_layouts_init(e->ncrecv, s2, layers, d2, &e->unpack_c);
        free(s2);
        free(d2);
    }
    free(sr);
    free(dr);
    if (!rc) e->ready = 1;
    return rc;
}

static int exchange(struct ca3dmm_dist_engine *e, const double *d_send, long long stot,
                    const long long *scnt, const long long *sdsp, double *d_recv, long long rtot,
                    const long long *rcnt, const long long *rdsp)
{
    if (e->tr.device_buffers) {
        if (e->tr.alltoallv_d(e->tr.ctx, d_send, scnt, sdsp, d_recv, rcnt, rdsp, NULL))
            return CA3DMM_ECUDA;
        CA3DMM_CUDA_TRY(cudaDeviceSynchronize());
        return CA3DMM_OK;
    }
    if (stot > 0)
        CA3DMM_CUDA_TRY(cudaMemcpy(e->h_send, d_send, sizeof(double) * (size_t) stot,
                                   cudaMemcpyDeviceToHost));
    if (e->tr.alltoallv_d(e->tr.ctx, e->h_send, scnt, sdsp, e->h_recv, rcnt, rdsp, NULL))
        return CA3DMM_ECUDA;
    if (rtot > 0)
        CA3DMM_CUDA_TRY(cudaMemcpy(d_recv, e->h_recv, sizeof(double) * (size_t) rtot,
                                   cudaMemcpyHostToDevice));
    return CA3DMM_OK;
}

int ca3dmm_dist_engine_exec(ca3dmm_dist_engine_p e, const double *A, int ldA, const double *B,
                            int ldB, double *C, int ldC)
{
    if (!e) return CA3DMM_EINVAL;
    const int me = e->me;
    int rc = prepare(e);
    if (rc) return rc;
    const double t0 = ca3dmm_wtime_sec();
    if (e->whole) {
        if (e->btb) { A = B; ldA = ldB; }
        ca3dmm_engine_exec(e->local, A, ldA, B, ldB, C, ldC);
        rc = ca3dmm_engine_last_error(e->local);
        const double dt = 1e3 * (ca3dmm_wtime_sec() - t0);
        e->st[1] += dt;
        e->st[3] += dt;
        e->n_exec++;
        return rc;
    }
    /* 1. operands */
    if (e->pack_ab) {
        const void *sb[2];
        int sl[2];
        for (int i = 0; i < e->nmy; i++) {
            const int mat = e->mymat[i];
            sb[i] = (mat == MAT_A) ? (const void *) A : (const void *) B;
            sl[i] = (mat == MAT_A) ? ldA : ldB;
        }
        void **db = (void **) xcalloc(e->nsend, sizeof(void *));
        int *dl = (int *) xcalloc(e->nsend, sizeof(int));
        if (!db || !dl) { free(db); free(dl); return CA3DMM_ENOMEM; }
        for (int i = 0; i < e->nsend; i++) {
            db[i] = e->d_send + e->send[i].off;
            dl[i] = e->send[i].x.nr > 0 ? e->send[i].x.nr : 1;
        }
        rc = mat_redist_layouts_exec(e->pack_ab, sb, sl, db, dl, NULL);
        free(db);
        free(dl);
        if (rc) return rc;
    }
    rc = exchange(e, e->d_send, e->stot, e->scnt, e->sdsp, e->d_recv, e->rtot, e->rcnt, e->rdsp);
    if (rc) return rc;
    if (e->unpack_ab) {
        const void **sb = (const void **) xcalloc(e->nrecv, sizeof(void *));
        int *sl = (int *) xcalloc(e->nrecv, sizeof(int));
        if (!sb || !sl) { free(sb); free(sl); return CA3DMM_ENOMEM; }
        for (int i = 0; i < e->nrecv; i++) {
            sb[i] = e->d_recv + e->recv[i].off;
            sl[i] = e->recv[i].x.nr > 0 ? e->recv[i].x.nr : 1;
        }
        void *db[2];
        int dl[2];
        for (int u = 0; u < e->nuniq; u++) {
            db[u] = e->d_panel[u];
            dl[u] = e->urect[u].nr > 0 ? e->urect[u].nr : 1;
        }
        rc = mat_redist_layouts_exec(e->unpack_ab, sb, sl, db, dl, NULL);
        free(sb);
        free(sl);
        if (rc) return rc;
    }
    CA3DMM_CUDA_TRY(cudaDeviceSynchronize());
    const double t1 = ca3dmm_wtime_sec();
    /* 2. the local GEMM */
    const rect_t c = e->cblk[me];
    if (e->local) {
        int pm[2];
        rect_t pr[2];
        panels_of(e, me, pm, pr);
        ca3dmm_engine_exec(e->local, e->d_panel[e->panel_of[0]], pr[0].nr > 0 ? pr[0].nr : 1,
                           e->d_panel[e->panel_of[1]], pr[1].nr > 0 ? pr[1].nr : 1, e->d_cbuf,
                           c.nr > 0 ? c.nr : 1);
        rc = ca3dmm_engine_last_error(e->local);
        if (rc) return rc;
    } else if (e->active[me] && area(c) > 0) {
        CA3DMM_CUDA_TRY(cudaMemset(e->d_cbuf, 0, sizeof(double) * (size_t) area(c)));   /* kz = 0 */
    }
    CA3DMM_CUDA_TRY(cudaDeviceSynchronize());
    const double t2 = ca3dmm_wtime_sec();
    /* 3. C pieces to their owners, slab layers summed in slab order */
    if (e->pack_c) {
        const void *sb[1] = {e->d_cbuf};
        int sl[1] = {c.nr > 0 ? c.nr : 1};
        void **db = (void **) xcalloc(e->ncsend, sizeof(void *));
        int *dl = (int *) xcalloc(e->ncsend, sizeof(int));
        if (!db || !dl) { free(db); free(dl); return CA3DMM_ENOMEM; }
        for (int i = 0; i < e->ncsend; i++) {
            db[i] = e->d_csend + e->csend[i].off;
            dl[i] = e->csend[i].x.nr > 0 ? e->csend[i].x.nr : 1;
        }
        rc = mat_redist_layouts_exec(e->pack_c, sb, sl, db, dl, NULL);
        free(db);
        free(dl);
        if (rc) return rc;
    }
    rc = exchange(e, e->d_csend, e->cstot, e->cscnt, e->csdsp, e->d_crecv, e->crtot, e->crcnt,
                  e->crdsp);
    if (rc) return rc;
    const rect_t d = e->dstC[me];
    if (area(d) > 0 && e->unpack_c) {
        const long long z = area(d);
        const int layers = e->kp > 1 ? e->kp : 1;
        const void **sb = (const void **) xcalloc(e->ncrecv, sizeof(void *));
        int *sl = (int *) xcalloc(e->ncrecv, sizeof(int));
        void **db = (void **) xcalloc(layers, sizeof(void *));
        int *dl = (int *) xcalloc(layers, sizeof(int));
        if (!sb || !sl || !db || !dl) rc = CA3DMM_ENOMEM;
        for (int i = 0; !rc && i < e->ncrecv; i++) {
            sb[i] = e->d_crecv + e->crecv[i].off;
            sl[i] = e->crecv[i].x.nr > 0 ? e->crecv[i].x.nr : 1;
        }
        for (int j = 0; !rc && j < layers; j++) {
            db[j] = e->kp > 1 ? (void *) (e->d_layers + (size_t) j * z) : (void *) C;
            dl[j] = e->kp > 1 ? d.nr : ldC;
        }
        if (!rc) rc = mat_redist_layouts_exec(e->unpack_c, sb, sl, db, dl, NULL);
        if (!rc && e->kp > 1)
            rc = ca3dmm_reduce_slabs_launch(e->d_layers, z, d.nr, e->kp, d.nr, d.nc, C, ldC, NULL);
        free(sb); free(sl); free(db); free(dl);
        if (rc) return rc;
    }
    CA3DMM_CUDA_TRY(cudaDeviceSynchronize());
    const double t3 = ca3dmm_wtime_sec();
    e->st[0] += 1e3 * (t1 - t0);
    e->st[1] += 1e3 * (t2 - t1);
    e->st[2] += 1e3 * (t3 - t2);
    e->st[3] += 1e3 * (t3 - t0);
    e->n_exec++;
    return CA3DMM_OK;
}

int ca3dmm_dist_engine_info(ca3dmm_dist_engine_p e, int out[10])
{
    if (!e || !out) return CA3DMM_EINVAL;
    const rect_t c = e->cblk[e->me];
    const int v[10] = {e->mp, e->np, e->kp, e->rp, e->active[e->me], e->slab[e->me],
                       c.r0, c.nr, c.c0, c.nc};
    memcpy(out, v, sizeof(v));
    return CA3DMM_OK;
}

int ca3dmm_dist_engine_counts(ca3dmm_dist_engine_p e, long long *send_ab, long long *recv_ab,
                              long long *send_c, long long *recv_c)
{
    if (!e) return CA3DMM_EINVAL;
    for (int r = 0; r < e->W; r++) {
        if (send_ab) send_ab[r] = e->scnt[r];
        if (recv_ab) recv_ab[r] = e->rcnt[r];
        if (send_c) send_c[r] = e->cscnt[r];
        if (recv_c) recv_c[r] = e->crcnt[r];
    }
    return CA3DMM_OK;
}

int ca3dmm_dist_engine_stats(ca3dmm_dist_engine_p e, double out[4])
{
    if (!e) return -1;
    if (out) memcpy(out, e->st, sizeof(e->st));
    return e->n_exec;
}

void ca3dmm_dist_engine_free(ca3dmm_dist_engine_p *pe)
{
    if (!pe || !*pe) return;
    struct ca3dmm_dist_engine *e = *pe;
    if (e->pack_ab) mat_redist_layouts_free(&e->pack_ab);
    if (e->unpack_ab) mat_redist_layouts_free(&e->unpack_ab);
    if (e->pack_c) mat_redist_layouts_free(&e->pack_c);
    if (e->unpack_c) mat_redist_layouts_free(&e->unpack_c);
    if (e->local) ca3dmm_engine_free(&e->local);
    if (e->local_comm) ca3dmm_vcomm_free(&e->local_comm);
    double *dev[] = {e->d_send, e->d_recv, e->d_panel[0], e->d_panel[1], e->d_cbuf, e->d_csend,
                     e->d_crecv, e->d_layers};
    for (size_t i = 0; i < sizeof(dev) / sizeof(dev[0]); i++)
        if (dev[i]) cudaFree(dev[i]);
    if (e->h_send) cudaFreeHost(e->h_send);
    if (e->h_recv) cudaFreeHost(e->h_recv);
    free(e->srcA); free(e->srcB); free(e->dstC); free(e->cblk);
    free(e->active); free(e->slab); free(e->k0); free(e->kz);
    free(e->send); free(e->recv); free(e->csend); free(e->crecv);
    free(e->scnt); free(e->sdsp); free(e->rcnt); free(e->rdsp);
    free(e->cscnt); free(e->csdsp); free(e->crcnt); free(e->crdsp);
    free(e);
    *pe = NULL;
}
