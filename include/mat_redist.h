/* Matrix block redistribution: same struct fields, names and signatures as
 * src/mat_redist.h:7-100 (row-major view, as in the reference).
 *
 * Folded onto one GPU: the caller holds the whole source block, so the
 * alltoallv of the reference becomes one batched device pack of the required
 * rectangle (the intersection lists of src/mat_redist.c:44-236 collapse to
 * the single source rectangle).  dt_size 8 (MPI_DOUBLE) is supported. */
#ifndef CA3DMM_MAT_REDIST_H
#define CA3DMM_MAT_REDIST_H

#include "ca3dmm_vmpi.h"
#include "dev_type.h"

struct mat_redist_engine {
    MPI_Comm graph_comm;    /* Virtual communicator */
    MPI_Datatype dtype;     /* Matrix element data type (MPI_DOUBLE) */
    size_t dt_size;         /* Element size in bytes (8) */
    int nproc;              /* Number of virtual ranks in comm */
    int rank;               /* 0 */
    int src_srow;           /* The starting row of the source matrix block */
    int src_scol;           /* The starting column of the source matrix block */
    int src_nrow;           /* Number of rows of the source matrix block */
    int src_ncol;           /* Number of columns of the source matrix block */
    int req_srow;           /* The starting row required */
    int req_scol;           /* The starting column required */
    int req_nrow;           /* Number of rows required */
    int req_ncol;           /* Number of columns required */
    int n_proc_send;        /* 1 if the required block is non-empty, else 0 */
    int n_proc_recv;        /* 1 if the required block is non-empty, else 0 */
    int send_cnt;           /* Number of elements moved */
    int recv_cnt;           /* Number of elements moved */
    int alloc_workbuf;      /* If work_buf is allocated by mat_redist_engine */
    int *send_ranks;        /* Size n_proc_send: {0} */
    int *send_sizes;        /* Size n_proc_send */
    int *send_displs;       /* Size n_proc_send+1 */
    int *sblk_sizes;        /* Size n_proc_send*4: srow, scol, nrow, ncol */
    int *recv_ranks;        /* Size n_proc_recv: {0} */
    int *recv_sizes;        /* Size n_proc_recv */
    int *recv_displs;       /* Size n_proc_recv+1 */
    int *rblk_sizes;        /* Size n_proc_recv*4 */
    int *send_info0;        /* unused */
    int *recv_info0;        /* unused */
    void *sendbuf_h;        /* unused */
    void *recvbuf_h;        /* unused */
    void *sendbuf_d;        /* unused */
    void *recvbuf_d;        /* unused */
    void *workbuf_h;        /* unused */
    void *workbuf_d;        /* device work buffer: one pack descriptor */
    double hd_trans_ms;     /* Host-device transfer: 0 */
    dev_type_t dev_type;    /* Data resident device type */
    /* ---- appended by this build ---- */
    int last_error;
};
typedef struct mat_redist_engine mat_redist_engine_s;
typedef struct mat_redist_engine *mat_redist_engine_p;

#ifdef __cplusplus
extern "C" {
#endif

/* src/mat_redist.h:69-74 */
void mat_redist_engine_init(const int src_srow, const int src_scol, const int src_nrow,
                            const int src_ncol, const int req_srow, const int req_scol,
                            const int req_nrow, const int req_ncol, MPI_Comm comm,
                            MPI_Datatype dtype, const size_t dt_size, dev_type_t dev_type,
                            mat_redist_engine_p *engine_, size_t *workbuf_bytes);
/* src/mat_redist.h:84 */
void mat_redist_engine_attach_workbuf(mat_redist_engine_p engine, void *workbuf_h, void *workbuf_d);
/* src/mat_redist.h:87 */
void mat_redist_engine_free(mat_redist_engine_p *engine_);
/* src/mat_redist.h:96-100: copy the required block (row-major, ld dst_ld)
 * out of the source block (row-major, ld src_ld); device pointers. */
void mat_redist_engine_exec(mat_redist_engine_p engine, const void *src_blk, const int src_ld,
                            void *dst_blk, const int dst_ld);

/* ---- arbitrary layouts (appended by this build) ----------------------------
 * The reference redistributes between two distributed layouts with every rank
 * calling mat_redist_engine_init/exec on its own source rectangle and the
 * rectangle it requires (src/mat_redist.c:44-419: intersections of each
 * rank's source block with every rank's required block, packed, exchanged by
 * Neighbor_alltoallv, unpacked).  Folded onto one GPU: the caller gives all
 * nsrc source rectangles and all nreq required rectangles at once (row-major
 * view as in the reference; rect k = {srow, scol, nrow, ncol} at 4k), and exec
 * copies, for every pair (i, j), the intersection of source block i and
 * required block j from src_blks[i] (row-major, ld src_lds[i]) into
 * dst_blks[j] (ld dst_lds[j]) in one batched device launch.  Required
 * elements that no source block holds are left untouched; source blocks
 * should not overlap (an element held twice is copied from either).
 * 8-byte elements; device pointers.  exec on stream NULL is synchronous,
 * otherwise enqueued on the given cudaStream_t. */
typedef struct mat_redist_layouts *mat_redist_layouts_p;
int mat_redist_layouts_init(int nsrc, const int *src_rects, int nreq, const int *req_rects,
                            mat_redist_layouts_p *layouts);
int mat_redist_layouts_pieces(mat_redist_layouts_p layouts);   /* non-empty intersections */
int mat_redist_layouts_exec(mat_redist_layouts_p layouts, const void *const *src_blks,
                            const int *src_lds, void *const *dst_blks, const int *dst_lds,
                            void *stream);
void mat_redist_layouts_free(mat_redist_layouts_p *layouts);

#ifdef __cplusplus
}
#endif
#endif
