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
