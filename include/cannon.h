/* 2D Cannon engine: same struct fields, names and signatures as
 * src/cannon.h:7-109.  Folded onto one GPU: the np_dim x np_dim virtual ranks
 * of the communicator all live in one call, the ring shifts are indexing, and
 * the np_dim local DGEMMs collapse into one grouped FP64 DMMA launch over the
 * whole m x n x k product.  Public fields describe virtual rank 0, as the
 * reference's rank 0 sees them. */
#ifndef CA3DMM_CANNON_H
#define CA3DMM_CANNON_H

#include "ca3dmm_vmpi.h"
#include "dev_type.h"

struct cannon_engine {
    int m, n, k;               /* Size of A (m * k), B (k * n), C (m * n) matrices */
    int my_rank;               /* Rank of this process in the target communicator (0) */
    int rank_row;              /* Row rank of virtual rank 0 in the 2D grid */
    int rank_col;              /* Column rank of virtual rank 0 in the 2D grid */
    int np_dim;                /* Number of virtual ranks on each dimension */
    int A_srow, A_scol;        /* 1st row & col of A block of virtual rank 0 */
    int B_srow, B_scol;        /* 1st row & col of B block of virtual rank 0 */
    int C_srow, C_scol;        /* 1st row & col of C block of virtual rank 0 */
    int A_nrow, A_ncol;        /* Rows & cols of A block of virtual rank 0 */
    int B_nrow, B_ncol;        /* Rows & cols of B block of virtual rank 0 */
    int C_nrow, C_ncol;        /* Rows & cols of C block of virtual rank 0 */
    int gemm_cycle;            /* Shift steps per local GEMM (reference rule, reported only) */
    int max_A_blk_size;        /* (m/np_dim+1) * (k/np_dim+1) */
    int max_B_blk_size;        /* (k/np_dim+1) * (n/np_dim+1) */
    int max_C_blk_size;        /* (m/np_dim+1) * (n/np_dim+1) */
    int alloc_workbuf;         /* If work_buf is allocated by cannon_engine */
    int *m_displs;             /* Size np_dim+1, partitioning displacements on m */
    int *n_displs;             /* Size np_dim+1, partitioning displacements on n */
    int *k_displs;             /* Size np_dim+1, partitioning displacements on k */
    void *A_recv_h;            /* unused (no host staging) */
    void *A_stack_h;           /* unused */
    void *B_recv_h;            /* unused */
    void *B_stack_h;           /* unused */
    void *A_recv_d;            /* device: aligned copy of A when the caller's A is not TMA-aligned */
    void *A_stack_d;           /* unused */
    void *B_recv_d;            /* device: aligned copy of B when the caller's B is not TMA-aligned */
    void *B_stack_d;           /* unused */
    void *workbuf_h;           /* host work buffer (unused, may be NULL) */
    void *workbuf_d;           /* device work buffer */
    void *A_gemm_h;            /* unused */
    void *B_gemm_h;            /* unused */
    dev_type_t dev_type;       /* Data resident device type */
    MPI_Comm comm;             /* Virtual communicator (np_dim^2 ranks) */

    /* Statistic data */
    double init_ms;            /* Time (ms) used in initialization */
    double shift0_ms;          /* Initial shift: 0 (indexing only) */
    double lshift_ms;          /* Loop shift: 0 (indexing only) */
    double gemm_ms;            /* Device time (ms) of the local DGEMM launches */
    double exec_ms;            /* Time (ms) of the whole Cannon execution */
    double hd_trans_ms;        /* Host-device transfer: 0 (device-resident) */
    int n_exec;                /* Number of Cannon executions */

    /* ---- appended by this build ---- */
    size_t workbuf_bytes;      /* device work buffer size */
    void *impl;                /* opaque device plan */
    int last_error;            /* 0 or the first CA3DMM_E* error of the last call */
};
typedef struct cannon_engine cannon_engine_s;
typedef struct cannon_engine *cannon_engine_p;

#ifdef __cplusplus
extern "C" {
#endif

/* src/cannon.h:69-72 */
void cannon_engine_init(const int m, const int n, const int k, MPI_Comm comm, dev_type_t dev_type,
                        cannon_engine_p *engine_, size_t *workbuf_bytes);
/* src/cannon.h:83 */
void cannon_engine_attach_workbuf(cannon_engine_p engine, void *workbuf_h, void *workbuf_d);
/* src/cannon.h:86 */
void cannon_engine_free(cannon_engine_p *engine_);
/* src/cannon.h:100-103.  Folded: A_blk is the whole m x k A (ld m), B_blk the
 * whole k x n B (ld k), C_blk the whole m x n C (ld m), all device memory.
 * C := alpha * A * B + beta * C.  A_blk and B_blk are not modified. */
void cannon_engine_exec(cannon_engine_p engine, const double alpha, const double beta,
                        double *A_blk, double *B_blk, double *C_blk);
/* src/cannon.h:106 */
void cannon_engine_reset_stat(cannon_engine_p engine);
/* src/cannon.h:109 (src/cannon.c:699-720 format) */
void cannon_engine_print_stat(cannon_engine_p engine);

#ifdef __cplusplus
}
#endif
#endif
