/* Block redistribution folded onto one GPU (src/mat_redist.c:44-419).
 *
 * With one source block per call, the rectangle intersections of
 * src/mat_redist.c:9-41 leave a single piece (req inside src) and the
 * pack -> Neighbor_alltoallv -> unpack pipeline becomes one device block
 * copy.  Row-major view as in the reference: a row-major nrow x ncol block is
 * the column-major ncol x nrow block the pack kernel copies. */
#include <string.h>
#include <cuda_runtime_api.h>
#include "ca3dmm_util.h"
#include "ca3dmm_kernels.h"
#include "mat_redist.h"

void mat_redist_engine_init(const int src_srow, const int src_scol, const int src_nrow,
                            const int src_ncol, const int req_srow, const int req_scol,
                            const int req_nrow, const int req_ncol, MPI_Comm comm,
                            MPI_Datatype dtype, const size_t dt_size, dev_type_t dev_type,
                            mat_redist_engine_p *engine_, size_t *workbuf_bytes)
{
    if (engine_ == NULL) return;
    *engine_ = NULL;
    if (is_dev_type_valid(dev_type) == 0) {
        ERROR_PRINTF("Invalid device type %d\n", dev_type);
        return;
    }
    if (dt_size != 8) {
        ERROR_PRINTF("Unsupported element size %zu (8-byte elements only)\n", dt_size);
        return;
    }
    if (req_nrow > 0 && req_ncol > 0 &&
        (req_srow < src_srow || req_scol < src_scol || req_srow + req_nrow > src_srow + src_nrow ||
         req_scol + req_ncol > src_scol + src_ncol)) {
        ERROR_PRINTF("Folded call: the required block must lie inside the source block\n");
        return;
    }
    mat_redist_engine_p e = (mat_redist_engine_p) calloc(1, sizeof(mat_redist_engine_s));
    if (!e) return;
    e->graph_comm = comm;
    e->dtype = dtype;
    e->dt_size = dt_size;
    e->nproc = ca3dmm_vcomm_size(comm);
    e->rank = 0;
    e->src_srow = src_srow; e->src_scol = src_scol; e->src_nrow = src_nrow; e->src_ncol = src_ncol;
    e->req_srow = req_srow; e->req_scol = req_scol; e->req_nrow = req_nrow; e->req_ncol = req_ncol;
    e->dev_type = dev_type;
    int nonempty = req_nrow > 0 && req_ncol > 0;
    e->n_proc_send = e->n_proc_recv = nonempty;
    e->send_cnt = e->recv_cnt = nonempty ? req_nrow * req_ncol : 0;
    e->send_ranks = (int *) calloc(1, sizeof(int));
    e->recv_ranks = (int *) calloc(1, sizeof(int));
    e->send_sizes = (int *) calloc(1, sizeof(int));
    e->recv_sizes = (int *) calloc(1, sizeof(int));
    e->send_displs = (int *) calloc(2, sizeof(int));
    e->recv_displs = (int *) calloc(2, sizeof(int));
    e->sblk_sizes = (int *) calloc(4, sizeof(int));
    e->rblk_sizes = (int *) calloc(4, sizeof(int));
    if (nonempty) {
        e->send_sizes[0] = e->recv_sizes[0] = e->send_cnt;
        e->send_displs[1] = e->recv_displs[1] = e->send_cnt;
        int blk[4] = {req_srow, req_scol, req_nrow, req_ncol};
        memcpy(e->sblk_sizes, blk, sizeof(blk));
        memcpy(e->rblk_sizes, blk, sizeof(blk));
    }
    size_t bytes = 256;
    if (workbuf_bytes != NULL) {
        e->alloc_workbuf = 0;
        *workbuf_bytes = bytes;
    } else {
        e->alloc_workbuf = 1;
        void *wh = NULL, *wd = NULL;
        MALLOC_ATTACH_WORKBUF(mat_redist_engine_attach_workbuf, mat_redist_engine_free, e, dev_type,
                              bytes, wh, wd);
        if (e == NULL) return;
    }
    *engine_ = e;
}

void mat_redist_engine_attach_workbuf(mat_redist_engine_p e, void *workbuf_h, void *workbuf_d)
{
    if (e == NULL) return;
    e->workbuf_h = workbuf_h;
    e->workbuf_d = workbuf_d;
}

void mat_redist_engine_free(mat_redist_engine_p *engine_)
{
    if (engine_ == NULL || *engine_ == NULL) return;
    mat_redist_engine_p e = *engine_;
    free(e->send_ranks); free(e->recv_ranks); free(e->send_sizes); free(e->recv_sizes);
    free(e->send_displs); free(e->recv_displs); free(e->sblk_sizes); free(e->rblk_sizes);
    if (e->alloc_workbuf && e->workbuf_d) dev_type_free(e->workbuf_d, DEV_TYPE_CUDA);
    free(e);
    *engine_ = NULL;
}

void mat_redist_engine_exec(mat_redist_engine_p e, const void *src_blk, const int src_ld,
                            void *dst_blk, const int dst_ld)
{
    if (e == NULL) {
        ERROR_PRINTF("mat_redist_engine not initialized\n");
        return;
    }
    e->last_error = CA3DMM_OK;
    if (e->req_nrow <= 0 || e->req_ncol <= 0) return;
    if (!e->workbuf_d || src_ld < e->src_ncol || dst_ld < e->req_ncol) {
        ERROR_PRINTF("mat_redist_engine_exec: invalid work buffer or leading dimension\n");
        e->last_error = CA3DMM_EINVAL;
        return;
    }
    ca3dmm_pack_desc_t d;
    memset(&d, 0, sizeof(d));
    d.rows = e->req_ncol;
    d.cols = e->req_nrow;
    d.lds = src_ld;
    d.ldd = dst_ld;
    d.src_off = (long long) (e->req_srow - e->src_srow) * src_ld + (e->req_scol - e->src_scol);
    int tiles = ca3dmm_pack_tiles(&d, 1);
    if (cudaMemcpy(e->workbuf_d, &d, sizeof(d), cudaMemcpyHostToDevice) != cudaSuccess) {
        e->last_error = CA3DMM_ECUDA;
        return;
    }
    int rc = ca3dmm_pack_launch((const double *) src_blk, (double *) dst_blk,
                                (const ca3dmm_pack_desc_t *) e->workbuf_d, 1, tiles, 0);
    if (rc == CA3DMM_OK && cudaDeviceSynchronize() != cudaSuccess) rc = CA3DMM_ECUDA;
    e->last_error = rc;
    if (rc) ERROR_PRINTF("mat_redist_engine_exec failed (error %d)\n", rc);
}

/* ---- arbitrary layouts --------------------------------------------------- */

/* One non-empty intersection of source block i and required block j, in the
 * global row-major coordinates of src/mat_redist.c:9-41. */
typedef struct {
    int src, dst;
    int srow, scol, nrow, ncol;
} piece_t;

struct mat_redist_layouts {
    int nsrc, nreq, npiece;
    int *src_rects, *req_rects;
    piece_t *pieces;
    ca3dmm_pack_desc_t *desc_h;   /* pinned staging of the descriptors */
    ca3dmm_pack_desc_t *desc_d;
};

int mat_redist_layouts_init(int nsrc, const int *src_rects, int nreq, const int *req_rects,
                            mat_redist_layouts_p *out)
{
    if (!out) return CA3DMM_EINVAL;
    *out = NULL;
    if (nsrc < 1 || nreq < 1 || !src_rects || !req_rects) return CA3DMM_EINVAL;
    for (int i = 0; i < nsrc + nreq; i++) {
        const int *r = i < nsrc ? src_rects + 4 * i : req_rects + 4 * (i - nsrc);
        if (r[0] < 0 || r[1] < 0 || r[2] < 0 || r[3] < 0) return CA3DMM_EINVAL;
    }
    mat_redist_layouts_p L = (mat_redist_layouts_p) calloc(1, sizeof(*L));
    if (!L) return CA3DMM_ENOMEM;
    L->nsrc = nsrc;
    L->nreq = nreq;
    L->src_rects = (int *) malloc(sizeof(int) * 4 * (size_t) nsrc);
    L->req_rects = (int *) malloc(sizeof(int) * 4 * (size_t) nreq);
    L->pieces = (piece_t *) malloc(sizeof(piece_t) * (size_t) nsrc * (size_t) nreq);
    if (!L->src_rects || !L->req_rects || !L->pieces) {
        mat_redist_layouts_free(&L);
        return CA3DMM_ENOMEM;
    }
    memcpy(L->src_rects, src_rects, sizeof(int) * 4 * (size_t) nsrc);
    memcpy(L->req_rects, req_rects, sizeof(int) * 4 * (size_t) nreq);
    for (int j = 0; j < nreq; j++)
        for (int i = 0; i < nsrc; i++) {
            const int *s = src_rects + 4 * i, *r = req_rects + 4 * j;
            const int r0 = s[0] > r[0] ? s[0] : r[0], c0 = s[1] > r[1] ? s[1] : r[1];
            const int r1 = s[0] + s[2] < r[0] + r[2] ? s[0] + s[2] : r[0] + r[2];
            const int c1 = s[1] + s[3] < r[1] + r[3] ? s[1] + s[3] : r[1] + r[3];
            if (r1 <= r0 || c1 <= c0) continue;
            piece_t *p = &L->pieces[L->npiece++];
            p->src = i; p->dst = j;
            p->srow = r0; p->scol = c0; p->nrow = r1 - r0; p->ncol = c1 - c0;
        }
    if (L->npiece > 0) {
        const size_t bytes = sizeof(ca3dmm_pack_desc_t) * (size_t) L->npiece;
        if (cudaMallocHost((void **) &L->desc_h, bytes) != cudaSuccess) L->desc_h = NULL;
        if (cudaMalloc((void **) &L->desc_d, bytes) != cudaSuccess) L->desc_d = NULL;
        if (!L->desc_h || !L->desc_d) {
            mat_redist_layouts_free(&L);
            return CA3DMM_ENOMEM;
        }
    }
    *out = L;
    return CA3DMM_OK;
}

int mat_redist_layouts_pieces(mat_redist_layouts_p L) { return L ? L->npiece : 0; }

int mat_redist_layouts_exec(mat_redist_layouts_p L, const void *const *src_blks,
                            const int *src_lds, void *const *dst_blks, const int *dst_lds,
                            void *stream)
{
    if (!L || !src_blks || !src_lds || !dst_blks || !dst_lds) return CA3DMM_EINVAL;
    for (int i = 0; i < L->nsrc; i++)
        if (src_lds[i] < L->src_rects[4 * i + 3] || ((uintptr_t) src_blks[i] & 7)) return CA3DMM_EINVAL;
    for (int j = 0; j < L->nreq; j++)
        if (dst_lds[j] < L->req_rects[4 * j + 3] || ((uintptr_t) dst_blks[j] & 7)) return CA3DMM_EINVAL;
    if (L->npiece == 0) return CA3DMM_OK;
    cudaStream_t st = (cudaStream_t) stream;
    /* the staging is rewritten below: the previous exec's upload must be done */
    CA3DMM_CUDA_TRY(cudaStreamSynchronize(st));
    for (int k = 0; k < L->npiece; k++) {
        const piece_t *p = &L->pieces[k];
        const int *s = L->src_rects + 4 * p->src, *r = L->req_rects + 4 * p->dst;
        ca3dmm_pack_desc_t *d = &L->desc_h[k];
        memset(d, 0, sizeof(*d));
        /* a row-major nrow x ncol piece is the column-major ncol x nrow block the
         * pack kernel copies; absolute addresses in units of 8 bytes (NULL bases) */
        d->rows = p->ncol;
        d->cols = p->nrow;
        d->lds = src_lds[p->src];
        d->ldd = dst_lds[p->dst];
        d->src_off = (long long) ((uintptr_t) src_blks[p->src] / 8) +
                     (long long) (p->srow - s[0]) * src_lds[p->src] + (p->scol - s[1]);
        d->dst_off = (long long) ((uintptr_t) dst_blks[p->dst] / 8) +
                     (long long) (p->srow - r[0]) * dst_lds[p->dst] + (p->scol - r[1]);
    }
    const int tiles = ca3dmm_pack_tiles(L->desc_h, L->npiece);
    CA3DMM_CUDA_TRY(cudaMemcpyAsync(L->desc_d, L->desc_h, sizeof(ca3dmm_pack_desc_t) * L->npiece,
                                    cudaMemcpyHostToDevice, st));
    int rc = ca3dmm_pack_launch(NULL, NULL, L->desc_d, L->npiece, tiles, st);
    if (rc) return rc;
    if (!stream) CA3DMM_CUDA_TRY(cudaStreamSynchronize(st));
    return CA3DMM_OK;
}

void mat_redist_layouts_free(mat_redist_layouts_p *Lp)
{
    if (!Lp || !*Lp) return;
    mat_redist_layouts_p L = *Lp;
    free(L->src_rects);
    free(L->req_rects);
    free(L->pieces);
    if (L->desc_h) cudaFreeHost(L->desc_h);
    if (L->desc_d) cudaFree(L->desc_d);
    free(L);
    *Lp = NULL;
}
