/* CA3DMM engine: C := op(A) * op(B) on one B200.
 *
 * Same struct fields (names, order), entry points, argument meaning and error
 * behaviour as src/ca3dmm.h:10-200, folded onto one GPU: the communicator
 * holds p virtual ranks (ca3dmm_vcomm_create), the library's own
 * mp x np x kp grid (src/partition.c) decides the work cuboids, and one host
 * call executes every virtual rank's share:
 *   pack/transpose kernels  <- mat_redist + cublasDgeam + allgather,
 *   one grouped FP64 DMMA   <- the per-rank Cannon cublasDgemm steps,
 *   FP64 slab reduction     <- the kp reduce-scatter,
 *   optional split-precision (Ozaki INT8 on tcgen05) in place of the DMMA GEMM.
 *
 * Folded-call conventions (the only departures from the reference):
 *  - src_{A,B}_* must describe the whole stored matrix (srow = scol = 0,
 *    nrow x ncol = its full size): a 1D column layout with ld = nrow, as in
 *    examples/example_AB.c:85-98, concatenates to exactly that.
 *  - dst_C_* (if not all -1) may be any block of C; dst_C receives it.
 *  - C_out_{srow,scol,nrow,ncol} describe the union of all virtual ranks'
 *    C_out blocks, i.e. the whole m x n C, held in C_out_d (ld = m) when no
 *    dst_C block was given.  The other per-rank fields (A_2dmm_*, rank_m, ...)
 *    describe virtual rank 0; ca3dmm_engine_vrank_info returns any rank's.
 *  - dev_type DEV_TYPE_HOST is rejected like an invalid type (no CPU path).
 *  - Errors never exit(): they print, leave *engine_ == NULL (init) or set
 *    ca3dmm_engine_last_error() (exec).
 */
#ifndef CA3DMM_H
#define CA3DMM_H

#include "ca3dmm_vmpi.h"
#include "mat_redist.h"
#include "cannon.h"
#include "partition.h"
#include "dev_type.h"

/* GEMM modes (CA3DMM_GEMM_MODE env var or ca3dmm_engine_set_gemm_mode) */
#define CA3DMM_GEMM_PLAIN 0   /* FP64 DMMA tensor-core GEMM (env CA3DMM_PLAIN_MERGE_SLABS=0 at
                                 init keeps the kp-slab sum order instead of one GEMM over k) */
#define CA3DMM_GEMM_OZAKI 1   /* split precision: INT8 slices on tcgen05, FP64 recombination */
#define CA3DMM_GEMM_CRT   2   /* split precision, modular: P-bit row / column integers, their exact
                                 product from one INT8 tcgen05 GEMM per modulus (N moduli <= 256)
                                 and the Chinese remainder theorem, rounded once to FP64 */
#define CA3DMM_GEMM_AUTO  3   /* chosen at the first exec by the autotuner among plain, slice and
                                 modular configurations, split precision only where it passes
                                 the accuracy guard (include/ca3dmm_tune.h; env CA3DMM_AUTOTUNE,
                                 CA3DMM_TUNE_CACHE; CA3DMM_GEMM_MODE=auto at init) */

struct ca3dmm_engine {
    int m, n, k;                    /* Size of op(A) (m*k), op(B) (k*n), C (m*n) */
    int mp, np, kp, rp;             /* Process grid and idle ranks */
    int my_rank;                    /* 0 (the folded call acts for every virtual rank) */
    int n_proc;                     /* Number of virtual ranks p */
    int is_active;                  /* Virtual rank 0 is active */
    int rank_m, rank_n, rank_k;     /* Grid coordinates of virtual rank 0 */
    int trans_A, trans_B;           /* If A / B are transposed */
    int task_m_num, task_m_id;      /* m-dimension task count / id of rank 0 */
    int task_n_num, task_n_id;      /* n-dimension task count / id of rank 0 */
    int task_k_num, task_k_id;      /* k-dimension task count / id of rank 0 */
    int is_BTB;                     /* If this engine computes B^T * B */
    int use_ag, use_rsb;            /* Even allgather / reduce-scatter splits */
    int A_rd_srow, A_rd_scol;       /* Rank 0's op(A) block in redistribution */
    int B_rd_srow, B_rd_scol;       /* Rank 0's op(B) block in redistribution */
    int A_2dmm_srow, A_2dmm_scol;   /* Rank 0's op(A) block in the 2D matmul */
    int B_2dmm_srow, B_2dmm_scol;   /* Rank 0's op(B) block in the 2D matmul */
    int C_2dmm_srow, C_2dmm_scol;   /* Rank 0's C block in the 2D matmul */
    int C_out_srow, C_out_scol;     /* Folded output block: 0, 0 */
    int A_rd_nrow, A_rd_ncol;
    int B_rd_nrow, B_rd_ncol;
    int A_2dmm_nrow, A_2dmm_ncol;
    int B_2dmm_nrow, B_2dmm_ncol;
    int C_2dmm_nrow, C_2dmm_ncol;
    int C_out_nrow, C_out_ncol;     /* Folded output block: m, n */
    int alloc_workbuf;              /* If the work buffer is allocated by the engine */
    int *AB_agv_recvcnts;           /* Rank 0's allgather counts (reference layout) */
    int *AB_agv_displs;
    int *C_rs_recvcnts;             /* Rank 0's reduce-scatter counts */
    void *A_rd_recv_h;              /* Host aliases: unused (no host staging) */
    void *A_trans_h;
    void *A_2dmm_h;
    void *B_rd_recv_h;
    void *B_trans_h;
    void *B_2dmm_h;
    void *C_2dmm_h;
    void *C_out_h;
    void *A_rd_recv_d;              /* Packed op(A) blocks of every (task_m, task_k) */
    void *A_trans_d;                /* = A_rd_recv_d (transpose fused into the pack) */
    void *A_2dmm_d;                 /* = A_rd_recv_d (replication is shared reads) */
    void *B_rd_recv_d;              /* Packed op(B) blocks of every (task_k, task_n) */
    void *B_trans_d;
    void *B_2dmm_d;
    void *C_2dmm_d;                 /* kp partial C slabs (m x n each) when kp > 1 */
    void *C_out_d;                  /* Whole C (ld m) when no dst_C block was given */
    void *workbuf_h;
    void *workbuf_d;
    size_t rdA_workbuf_bytes;
    size_t rdB_workbuf_bytes;
    size_t rdC_workbuf_bytes;
    size_t cannon_workbuf_bytes;
    size_t self_workbuf_bytes;
    MPI_Comm comm_AB_agv;           /* NULL: replication needs no communicator */
    MPI_Comm comm_C_rs;             /* NULL */
    MPI_Comm comm_2dmm;             /* NULL */
    mat_redist_engine_p redist_A;   /* NULL: the batched pack lives in the plan */
    mat_redist_engine_p redist_B;
    mat_redist_engine_p redist_C;
    cannon_engine_p cannon_engine;  /* Rank 0's Cannon geometry (no work buffer) */
    dev_type_t dev_type;

    /* Statistic data (device time from CUDA events, ms) */
    int print_timing;
    double init_ms;
    double redist_ms;               /* pack of A, B and the dst_C copy */
    double agvAB_ms;                /* 0: replication is shared reads */
    double cannon_ms;               /* GEMM (plain or split precision) */
    double reduce_ms;               /* kp-slab reduction */
    double hd_trans_ms;             /* 0 */
    double exec_ms;
    int n_exec;

    /* ---- appended by this build ---- */
    int n_group;                    /* GEMM work groups = kp * task_m_num * task_n_num */
    int gemm_mode;                  /* CA3DMM_GEMM_PLAIN or CA3DMM_GEMM_OZAKI */
    int ozaki_slices;               /* INT8 slices per operand (split mode) */
    int last_error;                 /* CA3DMM_OK or the first error of the last call */
    void *stream;                   /* cudaStream_t of exec (NULL: legacy default stream) */
    int sync_exec;                  /* 1: exec returns with C complete (reference behaviour) */
    size_t workbuf_bytes;           /* device work buffer size */
    void *impl;                     /* opaque device plan */
    int raster;                     /* GEMM tile rows per raster band (tuning knob) */
    int btb_symmetric;              /* B^T B: compute the upper block triangle only, mirror it
                                       (env CA3DMM_BTB_SYMMETRIC=1 at init_BTB) */
    int crt_moduli;                 /* CA3DMM_GEMM_CRT: moduli (env CA3DMM_CRT_MODULI; 0 = the
                                       fewest that give 51-bit integers for this k) */
    int crt_bits;                   /* CA3DMM_GEMM_CRT: integer width P of the operands */
    int gemm_auto;                  /* CA3DMM_GEMM_AUTO: 1 until tuned, 2 after (gemm_mode then
                                       holds the choice) */
    double tune_ms;                 /* wall time of the tuning at the first exec */
};
typedef struct ca3dmm_engine ca3dmm_engine_s;
typedef struct ca3dmm_engine *ca3dmm_engine_p;

#ifdef __cplusplus
extern "C" {
#endif

/* src/ca3dmm.h:114-124 */
void ca3dmm_engine_init(const int m, const int n, const int k, const int trans_A,
                        const int trans_B, const int src_A_srow, const int src_A_nrow,
                        const int src_A_scol, const int src_A_ncol, const int src_B_srow,
                        const int src_B_nrow, const int src_B_scol, const int src_B_ncol,
                        const int dst_C_srow, const int dst_C_nrow, const int dst_C_scol,
                        const int dst_C_ncol, const int *proc_grid, MPI_Comm comm,
                        dev_type_t dev_type, ca3dmm_engine_p *engine_, size_t *workbuf_bytes);

/* src/ca3dmm.h:149-157 */
void ca3dmm_engine_init_BTB(const int n, const int k, const int src_B_srow, const int src_B_nrow,
                            const int src_B_scol, const int src_B_ncol, const int dst_C_srow,
                            const int dst_C_nrow, const int dst_C_scol, const int dst_C_ncol,
                            const int *proc_grid, MPI_Comm comm, dev_type_t dev_type,
                            ca3dmm_engine_p *engine_, size_t *workbuf_bytes);

/* src/ca3dmm.h:167 (workbuf_h may be NULL; workbuf_d is required) */
void ca3dmm_engine_attach_workbuf(ca3dmm_engine_p engine, void *workbuf_h, void *workbuf_d);

/* src/ca3dmm.h:170 */
void ca3dmm_engine_free(ca3dmm_engine_p *engine_);

/* src/ca3dmm.h:191-194 (device pointers; src_A ignored for BTB) */
void ca3dmm_engine_exec(ca3dmm_engine_p engine, const void *src_A, const int ldA,
                        const void *src_B, const int ldB, void *dst_C, const int ldC);

/* src/ca3dmm.h:197 */
void ca3dmm_engine_reset_stat(ca3dmm_engine_p engine);
/* src/ca3dmm.h:200 (src/ca3dmm.c:1390-1410 format) */
void ca3dmm_engine_print_stat(ca3dmm_engine_p engine);

/* ---- added entry points (no counterpart in the reference) ---- */

/* ca3dmm_engine_exec with HOST buffers: the same operands and output as
 * ca3dmm_engine_exec (a dst_C block is required), in host memory; page-locked
 * memory lets the copies run asynchronously.  The engine copies B in, then
 * op(A) in bands of output rows, and computes and copies C out band by band,
 * so that the host-device copies overlap the computation.  Device staging of
 * the size of A, B and C is allocated on the first call and kept until
 * ca3dmm_engine_free.  Synchronous; returns 0 or a CA3DMM_E* code (also in
 * ca3dmm_engine_last_error).  B^T B: A_h is ignored. */
int ca3dmm_engine_exec_host(ca3dmm_engine_p engine, const void *A_h, int ldA, const void *B_h,
                            int ldB, void *C_h, int ldC);

/* Diagnostic of the bounded device waits used by every kernel of the library
 * (each returns an error status instead of hanging when its partner never
 * arrives): one thread waits on a device barrier that is completed
 * (arrive != 0) or never completed (arrive == 0).  Returns CA3DMM_OK, or
 * CA3DMM_ETIMEOUT after about timeout_s (<= 60 s); the device stays usable. */
int ca3dmm_device_wait_check(double timeout_s, int arrive);

/* Kernels this library has launched since it was loaded, counted on the
 * host at each launch (a launch recorded into a CUDA graph counts once, at
 * capture; its replays do not). */
unsigned long long ca3dmm_kernel_launches(void);

/* Guard bands of the engine's device work buffer: 256-byte bands between its
 * regions (plan, packed operands, slab buffers, C, split-precision regions),
 * filled with the byte 0xA5 whenever the plan is uploaded.  With the
 * environment variable CA3DMM_CANARY=1 at init, every exec checks them on the
 * device afterwards and reports an overwritten band as CA3DMM_ECANARY (6),
 * printing its byte range -- a kernel that wrote past its region.  Writes up
 * to `max` band offsets (bytes into the work buffer) and returns the number
 * of bands (-1 for a NULL engine). */
int ca3dmm_engine_guard_bands(ca3dmm_engine_p engine, long long *offsets, int max);

/* First error of the last call on this engine (0 = none). */
int ca3dmm_engine_last_error(ca3dmm_engine_p engine);
/* Run exec on `stream` (cudaStream_t); sync = 0 makes exec asynchronous and
 * CUDA-graph capturable (the statistics are then not updated). */
void ca3dmm_engine_set_stream(ca3dmm_engine_p engine, void *stream, int sync);
/* Select the GEMM: CA3DMM_GEMM_PLAIN, CA3DMM_GEMM_OZAKI with `slices` INT8
 * slices per operand (2..8), CA3DMM_GEMM_CRT with `slices` moduli (8..18,
 * 0 = the fewest whose product admits 51-bit operand integers at this k; the
 * engine's crt_bits field then holds the integer width), or CA3DMM_GEMM_AUTO
 * (tuned at the next exec; the work buffer then covers every candidate;
 * `slices` ignored).  Must be called
 * before attach_workbuf when the caller allocates the work buffer (it changes
 * *workbuf_bytes, which ca3dmm_engine_workbuf_bytes reports). */
int ca3dmm_engine_set_gemm_mode(ca3dmm_engine_p engine, int mode, int slices);
size_t ca3dmm_engine_workbuf_bytes(ca3dmm_engine_p engine);
/* Tile rows per raster band of the GEMM launches (4, 8 or 16; L2 reuse). */
int ca3dmm_engine_set_raster(ca3dmm_engine_p engine, int raster);
/* Geometry of any virtual rank, same 34-int layout as the CPU oracle's
 * orc_rank_geometry: is_active, rank_m/n/k, task_{m,n,k}_{num,id},
 * A_2dmm/B_2dmm/C_2dmm/C_out/A_rd/B_rd (srow, scol, nrow, ncol). */
int ca3dmm_engine_vrank_info(ca3dmm_engine_p engine, int vrank, int *out34);

/* No counterpart in the reference.  C = A * B (column-major, device pointers,
 * no transposes) as kp k-slabs summed in slab order, for callers that may not
 * allocate device memory themselves: code living in a process whose device
 * memory belongs to another allocator (a serving framework's pool, a
 * memory-capped MPS client), or code that must not meet an allocation failure
 * in the middle of a job.  Allocates nothing: the partial slabs, plan and
 * status word live in one fixed device array of
 * ca3dmm_dgemm_kslab_noalloc_scratch_bytes() bytes (32 MiB) that every GPU
 * loading the library holds until exit; a problem needing more
 * (kp > 1: ~8 * m * n * kp bytes) is rejected with CA3DMM_EINVAL.  A, B must be
 * 16-byte aligned with even ldA >= m, ldB >= k; every slab start
 * k0 = calc_block_spos_size(k, kp, s) must be even; ldC >= m; 1 <= kp <= 64.
 * Calls that overlap on the GPU race on the shared array.  The call is
 * synchronous on `stream` (cudaStream_t, NULL = legacy default stream): it
 * waits for the stream before returning, so it must not be made while that
 * stream is being captured.  Returns 0 or a CA3DMM_E* code. */
int ca3dmm_dgemm_kslab_noalloc(int m, int n, int k, int kp, const double *A, int ldA,
                               const double *B, int ldB, double *C, int ldC, void *stream);
size_t ca3dmm_dgemm_kslab_noalloc_scratch_bytes(void);

#ifdef __cplusplus
}
#endif
#endif
