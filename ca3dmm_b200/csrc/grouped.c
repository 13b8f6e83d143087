/* Batched independent FP64 GEMMs: one pack launch per operand side and one
 * persistent grouped GEMM launch (plain FP64 DMMA, or split precision by INT8
 * slices or by the modular scheme) for the whole batch.  See
 * include/ca3dmm_grouped.h. */
#include <stdint.h>
#include <string.h>
#include <cuda_runtime_api.h>
#include "ca3dmm_util.h"
#include "ca3dmm_kernels.h"
#include "ca3dmm_ozaki.h"
#include "ca3dmm_crt.h"
#include "ca3dmm_grouped.h"

#define GALIGN 256

struct ca3dmm_grouped {
    int nprob, mode, slices;
    int *m, *n, *k, *ta, *tb;
    int *order;                   /* launch order of the problems: longest k first */
    int a_kmajor;                 /* plain mode: A layout of the launch (the majority's) */
    long long *lda_p, *ldb_p;     /* leading dimensions of the packed copies */
    size_t *offA, *offB;          /* byte offsets of the packed copies */
    /* work buffer layout */
    size_t off_status, off_packA, off_packB, off_gemm, off_ozplan, off_crtplan, off_A, off_B,
        off_oz, total;
    size_t oz_bytes, crt_bytes, stage_bytes;
    void *workbuf_d;
    int alloc_workbuf;
    void *stage;                  /* pinned host staging of the plan */
    int *status_h;
    cudaEvent_t ev[2];
    int events_ok;
    void *stream;
    int sync;
    /* cache of the last exec's arguments */
    int plan_valid;
    const double **cA, **cB;
    double **cC;
    int *cldA, *cldB, *cldC;
    int tiles_A, tiles_B, gemm_tiles;
    ca3dmm_dgemm_desc_t *gd;
    ca3dmm_oz_blk_t *ob;
    ca3dmm_oz_src_t *os;
    ca3dmm_oz_group_t *og;
    ca3dmm_oz_plan_t oz;
    ca3dmm_crt_group_t *cg;       /* modular mode: one group per problem, in launch order */
    ca3dmm_crt_plan_t crt;
    double last_ms;
};

static size_t galign(size_t x) { return (x + GALIGN - 1) / GALIGN * GALIGN; }

/* The persistent GEMM kernels hand out tiles round-robin in launch order, and
 * a tile's time grows with its problem's k.  Ordering the problems by k,
 * longest first, makes each round of tiles nearly uniform, so no SM is left
 * with a long tile while the others idle (longest-processing-time first). */
static int by_key(const void *a, const void *b)
{
    const unsigned long long x = *(const unsigned long long *) a, y = *(const unsigned long long *) b;
    return x < y ? -1 : (x > y);
}

/* order[] = problem indices by k descending, ties in index order */
static int order_by_k(int nprob, const int *k, int *order)
{
    unsigned long long *key = (unsigned long long *) malloc(sizeof(unsigned long long) * nprob);
    if (!key) return CA3DMM_ENOMEM;
    for (int i = 0; i < nprob; i++)
        key[i] = ((unsigned long long) (0x7fffffff - k[i]) << 32) | (unsigned) i;
    qsort(key, (size_t) nprob, sizeof(*key), by_key);
    for (int i = 0; i < nprob; i++) order[i] = (int) (key[i] & 0xffffffffu);
    free(key);
    return CA3DMM_OK;
}

void ca3dmm_grouped_free(ca3dmm_grouped_p *gp)
{
    if (!gp || !*gp) return;
    ca3dmm_grouped_p g = *gp;
    free(g->m); free(g->n); free(g->k); free(g->ta); free(g->tb); free(g->order);
    free(g->lda_p); free(g->ldb_p); free(g->offA); free(g->offB);
    free(g->cA); free(g->cB); free(g->cC); free(g->cldA); free(g->cldB); free(g->cldC);
    free(g->gd); free(g->ob); free(g->os); free(g->og); free(g->cg);
    if (g->stage) cudaFreeHost(g->stage);
    if (g->status_h) cudaFreeHost(g->status_h);
    if (g->events_ok) { cudaEventDestroy(g->ev[0]); cudaEventDestroy(g->ev[1]); }
    if (g->alloc_workbuf && g->workbuf_d) cudaFree(g->workbuf_d);
    free(g);
    *gp = NULL;
}

int ca3dmm_grouped_init(int nprob, const int *m, const int *n, const int *k, const int *trans_A,
                        const int *trans_B, int gemm_mode, int slices, ca3dmm_grouped_p *gp,
                        size_t *workbuf_bytes)
{
    if (!gp) return CA3DMM_EINVAL;
    *gp = NULL;
    if (nprob < 1 || nprob > 32768 || !m || !n || !k) return CA3DMM_EINVAL;
    if (gemm_mode < 0 || gemm_mode > 2) return CA3DMM_EINVAL;
    if (gemm_mode == 1 && (slices < 2 || slices > 8)) return CA3DMM_EINVAL;
    int kmax = 0;
    for (int i = 0; i < nprob; i++) {
        if (m[i] < 1 || n[i] < 1 || k[i] < 1) {
            ERROR_PRINTF("grouped GEMM %d: invalid size %d x %d x %d\n", i, m[i], n[i], k[i]);
            return CA3DMM_EINVAL;
        }
        if (k[i] > kmax) kmax = k[i];
    }
    if (gemm_mode == 2) {
        /* moduli: the given count (8..18), or the fewest that give 51-bit
         * integers for the deepest product; every k within the exact range */
        if (kmax > CA3DMM_CRT_MAX_K) return CA3DMM_EINVAL;
        if (slices == 0) {
            slices = CA3DMM_CRT_MAX_MODULI;
            for (int nm = 8; nm <= CA3DMM_CRT_MAX_MODULI; nm++)
                if (ca3dmm_crt_bits(nm, kmax) >= 51) { slices = nm; break; }
        }
        if (slices < 8 || slices > CA3DMM_CRT_MAX_MODULI || ca3dmm_crt_bits(slices, kmax) < 2)
            return CA3DMM_EINVAL;
    }
    ca3dmm_grouped_p g = (ca3dmm_grouped_p) calloc(1, sizeof(*g));
    if (!g) return CA3DMM_ENOMEM;
    g->nprob = nprob;
    g->mode = gemm_mode;
    g->slices = slices;
    g->sync = 1;
    size_t ni = sizeof(int) * nprob;
    g->m = malloc(ni); g->n = malloc(ni); g->k = malloc(ni); g->ta = malloc(ni); g->tb = malloc(ni);
    g->order = malloc(ni);
    g->lda_p = malloc(sizeof(long long) * nprob); g->ldb_p = malloc(sizeof(long long) * nprob);
    g->offA = malloc(sizeof(size_t) * nprob); g->offB = malloc(sizeof(size_t) * nprob);
    g->cA = calloc(nprob, sizeof(void *)); g->cB = calloc(nprob, sizeof(void *));
    g->cC = calloc(nprob, sizeof(void *));
    g->cldA = calloc(nprob, sizeof(int)); g->cldB = calloc(nprob, sizeof(int));
    g->cldC = calloc(nprob, sizeof(int));
    g->gd = calloc(nprob, sizeof(ca3dmm_dgemm_desc_t));
    g->ob = calloc(2 * (size_t) nprob, sizeof(ca3dmm_oz_blk_t));
    g->os = calloc(2 * (size_t) nprob, sizeof(ca3dmm_oz_src_t));
    g->og = calloc(nprob, sizeof(ca3dmm_oz_group_t));
    g->cg = calloc(nprob, sizeof(ca3dmm_crt_group_t));
    if (!g->m || !g->n || !g->k || !g->ta || !g->tb || !g->order || !g->lda_p || !g->ldb_p || !g->offA ||
        !g->offB || !g->cA || !g->cB || !g->cC || !g->cldA || !g->cldB || !g->cldC || !g->gd ||
        !g->ob || !g->os || !g->og || !g->cg) {
        ca3dmm_grouped_free(&g);
        return CA3DMM_ENOMEM;
    }
    for (int i = 0; i < nprob; i++) {
        g->m[i] = m[i]; g->n[i] = n[i]; g->k[i] = k[i];
        g->ta[i] = trans_A ? (trans_A[i] != 0) : 0;
        g->tb[i] = trans_B ? (trans_B[i] != 0) : 0;
    }
    if (order_by_k(nprob, g->k, g->order)) {
        ca3dmm_grouped_free(&g);
        return CA3DMM_ENOMEM;
    }
    size_t off = 0;
    g->off_status = off; off = galign(off + 64);
    g->off_packA = off; off = galign(off + sizeof(ca3dmm_pack_desc_t) * nprob);
    g->off_packB = off; off = galign(off + sizeof(ca3dmm_pack_desc_t) * nprob);
    g->off_gemm = off; off = galign(off + ca3dmm_dgemm_plan_bytes(nprob));
    g->off_ozplan = off; off = galign(off + ca3dmm_oz_plan_bytes(nprob));
    g->off_crtplan = off; off = galign(off + ca3dmm_crt_plan_bytes(2 * nprob, nprob));
    g->stage_bytes = off;
    g->off_A = off;
    if (gemm_mode == 0) {
        /* One A layout per DMMA launch: K-major when most A bytes are
         * transposed (those are then read in place), else M-major. */
        double bytes_t = 0.0, bytes_n = 0.0;
        for (int i = 0; i < nprob; i++) *(g->ta[i] ? &bytes_t : &bytes_n) += (double) m[i] * k[i];
        g->a_kmajor = bytes_t > bytes_n;
        for (int i = 0; i < nprob; i++) {
            g->lda_p[i] = ca3dmm_round_up(g->a_kmajor ? k[i] : m[i], 2);
            g->offA[i] = off;
            off = galign(off + sizeof(double) * (size_t) g->lda_p[i] *
                                   (size_t) (g->a_kmajor ? m[i] : k[i]));
        }
        g->off_B = off;
        for (int i = 0; i < nprob; i++) {
            g->ldb_p[i] = ca3dmm_round_up(k[i], 2);
            g->offB[i] = off;
            off = galign(off + sizeof(double) * (size_t) g->ldb_p[i] * (size_t) n[i]);
        }
    }
    g->off_oz = off;
    if (gemm_mode == 1) {
        g->oz_bytes = ca3dmm_oz_work_bytes(nprob, m, k, nprob, k, n, slices);
        off = galign(off + g->oz_bytes);
    }
    if (gemm_mode == 2) {
        g->crt_bytes = ca3dmm_crt_work_bytes(nprob, m, k, nprob, k, n, nprob, m, n, slices);
        off = galign(off + g->crt_bytes);
    }
    g->total = off;
    if (workbuf_bytes) {
        *workbuf_bytes = g->total;
    } else {
        void *w = NULL;
        if (cudaMalloc(&w, g->total) != cudaSuccess) {
            ca3dmm_grouped_free(&g);
            return CA3DMM_ENOMEM;
        }
        g->alloc_workbuf = 1;
        int rc = ca3dmm_grouped_attach_workbuf(g, w);
        if (rc) {
            ca3dmm_grouped_free(&g);
            return rc;
        }
    }
    *gp = g;
    return CA3DMM_OK;
}

int ca3dmm_grouped_attach_workbuf(ca3dmm_grouped_p g, void *workbuf_d)
{
    if (!g || !workbuf_d || ((uintptr_t) workbuf_d & 255)) return CA3DMM_EINVAL;
    g->workbuf_d = workbuf_d;
    if (!g->stage) {
        CA3DMM_CUDA_TRY(cudaMallocHost(&g->stage, g->stage_bytes));
        CA3DMM_CUDA_TRY(cudaMallocHost((void **) &g->status_h, 64));
        memset(g->status_h, 0, 64);
        g->events_ok = cudaEventCreate(&g->ev[0]) == cudaSuccess &&
                       cudaEventCreate(&g->ev[1]) == cudaSuccess;
    }
    g->plan_valid = 0;
    return CA3DMM_OK;
}

void ca3dmm_grouped_set_stream(ca3dmm_grouped_p g, void *stream, int sync)
{
    if (!g) return;
    g->stream = stream;
    g->sync = sync ? 1 : 0;
}

double ca3dmm_grouped_last_ms(ca3dmm_grouped_p g) { return g ? g->last_ms : 0.0; }

static int same_args(ca3dmm_grouped_p g, const double *const *A, const int *ldA,
                     const double *const *B, const int *ldB, double *const *C, const int *ldC)
{
    if (!g->plan_valid) return 0;
    for (int i = 0; i < g->nprob; i++)
        if (g->cA[i] != A[i] || g->cB[i] != B[i] || g->cC[i] != C[i] || g->cldA[i] != ldA[i] ||
            g->cldB[i] != ldB[i] || g->cldC[i] != ldC[i])
            return 0;
    return 1;
}

static int build_plan(ca3dmm_grouped_p g, const double *const *A, const int *ldA,
                      const double *const *B, const int *ldB, double *const *C, const int *ldC,
                      cudaStream_t st)
{
    char *w = (char *) g->workbuf_d, *h = (char *) g->stage;
    const int np = g->nprob;
    memset(h, 0, 64);
    if (g->mode == 0) {
        ca3dmm_pack_desc_t *pa = (ca3dmm_pack_desc_t *) (h + g->off_packA);
        ca3dmm_pack_desc_t *pb = (ca3dmm_pack_desc_t *) (h + g->off_packB);
        /* An operand in the launch's layout with an even leading dimension and a
         * 16-byte aligned start is read in place; the others are packed (A into
         * the launch's layout, B K-major). */
        const int ak = g->a_kmajor;
        for (int i = 0; i < np; i++) {
            /* sources by absolute address (NULL base), packed copies relative to w */
            const int a_direct = g->ta[i] == ak && !(ldA[i] & 1) && !((uintptr_t) A[i] & 15);
            const int b_direct = !g->tb[i] && !(ldB[i] & 1) && !((uintptr_t) B[i] & 15);
            memset(&pa[i], 0, sizeof(pa[i]));
            if (!a_direct) {
                /* K-major copy of op(A) = the k x m matrix op(A)^T */
                pa[i].rows = ak ? g->k[i] : g->m[i];
                pa[i].cols = ak ? g->m[i] : g->k[i];
                pa[i].trans = ak ? !g->ta[i] : g->ta[i];
                pa[i].lds = ldA[i];
                pa[i].src_off = (long long) ((uintptr_t) A[i] / sizeof(double));
                pa[i].dst_off = (long long) (g->offA[i] / sizeof(double));
                pa[i].ldd = g->lda_p[i];
            }
            memset(&pb[i], 0, sizeof(pb[i]));
            if (!b_direct) {
                pb[i].rows = g->k[i]; pb[i].cols = g->n[i]; pb[i].trans = g->tb[i];
                pb[i].lds = ldB[i];
                pb[i].src_off = (long long) ((uintptr_t) B[i] / sizeof(double));
                pb[i].dst_off = (long long) (g->offB[i] / sizeof(double));
                pb[i].ldd = g->ldb_p[i];
            }
        }
        for (int j = 0; j < np; j++) {
            const int i = g->order[j];
            ca3dmm_dgemm_desc_t *q = &g->gd[j];
            if (pa[i].rows) { q->A = (const double *) (w + g->offA[i]); q->lda = g->lda_p[i]; }
            else { q->A = A[i]; q->lda = ldA[i]; }
            if (pb[i].rows) { q->B = (const double *) (w + g->offB[i]); q->ldb = g->ldb_p[i]; }
            else { q->B = B[i]; q->ldb = ldB[i]; }
            q->C = C[i]; q->ldc = ldC[i];
            q->m = g->m[i]; q->n = g->n[i]; q->k = g->k[i];
            q->alpha = 1.0; q->beta = 0.0;
            q->a_kmajor = ak;
        }
        g->tiles_A = ca3dmm_pack_tiles(pa, np);
        g->tiles_B = ca3dmm_pack_tiles(pb, np);
        int rc = ca3dmm_dgemm_plan_encode(g->gd, np, h + g->off_gemm, &g->gemm_tiles);
        if (rc) return rc;
    } else {
        /* split precision: operand blocks read where they lie (absolute bases) */
        for (int i = 0; i < np; i++) {
            g->ob[i].r0 = 0; g->ob[i].c0 = 0; g->ob[i].rows = g->m[i]; g->ob[i].cols = g->k[i];
            g->ob[i].alias = -1;
            g->os[i].base = A[i]; g->os[i].ld = ldA[i]; g->os[i].trans = g->ta[i];
            g->ob[np + i].r0 = 0; g->ob[np + i].c0 = 0;
            g->ob[np + i].rows = g->k[i]; g->ob[np + i].cols = g->n[i];
            g->ob[np + i].alias = -1;
            g->os[np + i].base = B[i]; g->os[np + i].ld = ldB[i]; g->os[np + i].trans = g->tb[i];
        }
        int rc;
        if (g->mode == 2) {
            for (int j = 0; j < np; j++) {
                const int i = g->order[j];
                g->cg[j].a_blk = i; g->cg[j].b_blk = i;
                g->cg[j].C = C[i]; g->cg[j].ldc = ldC[i];
                g->cg[j].m = g->m[i]; g->cg[j].n = g->n[i]; g->cg[j].k = g->k[i];
                g->cg[j].band = 0;
            }
            rc = ca3dmm_crt_plan_encode(&g->crt, g->slices, np, g->ob, g->os, np, g->ob + np,
                                        g->os + np, np, g->cg, w + g->off_oz, g->crt_bytes,
                                        h + g->off_crtplan, w + g->off_crtplan);
        } else {
            for (int j = 0; j < np; j++) {
                const int i = g->order[j];
                g->og[j].a_blk = i; g->og[j].b_blk = i;
                g->og[j].row0 = 0; g->og[j].col0 = 0;
                g->og[j].C = C[i]; g->og[j].ldc = ldC[i];
                g->og[j].m = g->m[i]; g->og[j].n = g->n[i]; g->og[j].k = g->k[i];
            }
            rc = ca3dmm_oz_plan_encode(&g->oz, g->slices, np, g->ob, g->os, np, g->ob + np,
                                       g->os + np, np, g->og, 0, NULL, w + g->off_oz, g->oz_bytes,
                                       h + g->off_ozplan, w + g->off_ozplan);
        }
        if (rc) return rc;
    }
    CA3DMM_CUDA_TRY(cudaMemcpyAsync(w, h, g->stage_bytes, cudaMemcpyHostToDevice, st));
    for (int i = 0; i < np; i++) {
        g->cA[i] = A[i]; g->cB[i] = B[i]; g->cC[i] = C[i];
        g->cldA[i] = ldA[i]; g->cldB[i] = ldB[i]; g->cldC[i] = ldC[i];
    }
    g->plan_valid = 1;
    return CA3DMM_OK;
}

int ca3dmm_grouped_exec(ca3dmm_grouped_p g, const double *const *A, const int *ldA,
                        const double *const *B, const int *ldB, double *const *C, const int *ldC)
{
    if (!g || !g->workbuf_d || !A || !B || !C || !ldA || !ldB || !ldC) return CA3DMM_EINVAL;
    for (int i = 0; i < g->nprob; i++) {
        const int ar = g->ta[i] ? g->k[i] : g->m[i], br = g->tb[i] ? g->n[i] : g->k[i];
        if (!A[i] || !B[i] || !C[i] || ldA[i] < ar || ldB[i] < br || ldC[i] < g->m[i] ||
            ((uintptr_t) A[i] & 7) || ((uintptr_t) B[i] & 7) || ((uintptr_t) C[i] & 7)) {
            ERROR_PRINTF("grouped GEMM %d: invalid pointer or leading dimension\n", i);
            return CA3DMM_EINVAL;
        }
    }
    cudaStream_t st = (cudaStream_t) g->stream;
    char *w = (char *) g->workbuf_d;
    int rc;
    if (!same_args(g, A, ldA, B, ldB, C, ldC)) {
        rc = build_plan(g, A, ldA, B, ldB, C, ldC, st);
        if (rc) return rc;
    } else {
        CA3DMM_CUDA_TRY(cudaMemsetAsync(w + g->off_status, 0, 64, st));
    }
    int timing = g->sync && g->events_ok;
    if (timing) cudaEventRecord(g->ev[0], st);
    int *status = (int *) (w + g->off_status);
    if (g->mode == 0) {
        rc = ca3dmm_pack_launch(NULL, (double *) w, (const ca3dmm_pack_desc_t *) (w + g->off_packA),
                                g->nprob, g->tiles_A, st);
        if (rc) return rc;
        rc = ca3dmm_pack_launch(NULL, (double *) w, (const ca3dmm_pack_desc_t *) (w + g->off_packB),
                                g->nprob, g->tiles_B, st);
        if (rc) return rc;
        rc = ca3dmm_dgemm_launch(w + g->off_gemm, g->nprob, g->gemm_tiles, g->a_kmajor, status,
                                 5.0, st);
        if (rc) return rc;
    } else if (g->mode == 2) {
        rc = ca3dmm_crt_run_pack(&g->crt, NULL, NULL, st);
        if (!rc) rc = ca3dmm_crt_run_gemm(&g->crt, NULL, status, 5.0, st);
        if (!rc) rc = ca3dmm_crt_run_reconstruct(&g->crt, 0, g->nprob, 0, 0x7fffffff, st);
        if (!rc) rc = ca3dmm_crt_run_nonfinite(&g->crt, 0, g->nprob, 0, 0x7fffffff, NULL, NULL, st);
        if (rc) return rc;
    } else {
        rc = ca3dmm_oz_run_pack(&g->oz, NULL, NULL, st);
        if (rc) return rc;
        rc = ca3dmm_oz_run_gemm(&g->oz, status, 5.0, st);
        if (rc) return rc;
        rc = ca3dmm_oz_run_nonfinite(&g->oz, NULL, NULL, NULL, st);
        if (rc) return rc;
    }
    if (timing) cudaEventRecord(g->ev[1], st);
    if (g->sync) {
        CA3DMM_CUDA_TRY(cudaMemcpyAsync(g->status_h, status, sizeof(int), cudaMemcpyDeviceToHost, st));
        CA3DMM_CUDA_TRY(cudaStreamSynchronize(st));
        if (g->status_h[0]) {
            ERROR_PRINTF("grouped GEMM: device status %d (a bounded wait ran out)\n", g->status_h[0]);
            return CA3DMM_ETIMEOUT;
        }
        if (timing) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, g->ev[0], g->ev[1]);
            g->last_ms = ms;
        }
    }
    return CA3DMM_OK;
}
