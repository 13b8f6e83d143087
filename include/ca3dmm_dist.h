/* CA3DMM over several GPUs, one rank per GPU, from C.
 *
 * The reference's multi-rank API is ca3dmm_engine_init / _init_BTB / exec /
 * free called by every rank of an MPI communicator with that rank's blocks
 * (src/ca3dmm.h:114-200; examples/example_AB.c:85-98 passes 1D column
 * blocks).  ca3dmm_dist_engine_* is that call with the communicator replaced
 * by a transport: two collectives the engine needs, as function pointers, so
 * that an MPI caller passes MPI_Allgather / MPI_Alltoallv_c through two
 * wrapper functions of a few lines, a C caller without MPI uses the built-in
 * NCCL transport, and ranks that are threads of one process use the built-in
 * thread transport.
 *
 * Each rank computes the reference's grid and every rank's cuboid for
 * p = the transport's size (the same arithmetic as ca3dmm_engine_init), and
 * an exec is two all-to-alls around the local GEMM:
 *   1. every rank sends every peer the intersection of its A and B blocks
 *      with the peer's op(A) panel (C_2dmm rows x slab k) and op(B) panel
 *      (slab k x C_2dmm columns) -- the panels the reference assembles by its
 *      redistribution, allgather and Cannon shifts (src/ca3dmm.c:977-1171,
 *      src/cannon.c:319-631);
 *   2. the local GEMM of the panels on this GPU (plain FP64 DMMA or split
 *      precision, the single-GPU engine);
 *   3. every rank sends every peer the intersection of its C_2dmm block with
 *      the peer's dst_C block; the receiver sums the kp slab partials in slab
 *      order 0 .. kp-1 (the reference's reduce-scatter over kp and its C
 *      redistribution, src/ca3dmm.c:1287-1372), the order in which the
 *      single-GPU engine sums its slabs, so that split-precision results are
 *      bit-identical to the single-GPU engine on the same grid.
 * A transport with device_buffers = 1 (NCCL) exchanges device memory (the
 * reference's DEV_TYPE_CUDA_MPI_DIRECT); otherwise the pieces are staged
 * through pinned host memory (its DEV_TYPE_CUDA).
 *
 * Rectangles are (srow, nrow, scol, ncol) of a column-major matrix, the
 * reference's argument order.  Blocks are device pointers of this rank's GPU.
 */
#ifndef CA3DMM_DIST_H
#define CA3DMM_DIST_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int rank, size;
    int device_buffers;   /* 1: alltoallv takes device pointers (stream-ordered on `stream`) */
    void *ctx;
    /* all[r * n + i] = rank r's mine[i] (host memory) */
    int (*allgather_ll)(void *ctx, const long long *mine, int n, long long *all);
    /* element counts and displacements per peer; send / recv are host or
     * device memory per device_buffers; returns 0 when the exchange is done
     * (device_buffers: enqueued on `stream`) */
    int (*alltoallv_d)(void *ctx, const double *send, const long long *scounts,
                       const long long *sdispls, double *recv, const long long *rcounts,
                       const long long *rdispls, void *stream);
} ca3dmm_transport_t;

/* Threads of one process as ranks: creates `size` transports sharing one
 * exchange area (host memory, a barrier per collective); transport r is used
 * by the thread acting as rank r.  Free once, after every rank is done. */
int ca3dmm_transport_threads_create(int size, ca3dmm_transport_t *per_rank);
void ca3dmm_transport_threads_free(ca3dmm_transport_t *per_rank);

/* NCCL (libnccl.so.2, loaded at run time): rank `rank` of `size`, one GPU
 * each, all ranks passing the same 128-byte id from ca3dmm_nccl_unique_id
 * (made by one rank, shared out of band).  The current CUDA device is the
 * rank's GPU.  device_buffers = 1. */
int ca3dmm_nccl_unique_id(unsigned char id[128]);
int ca3dmm_transport_nccl_create(int size, int rank, const unsigned char id[128],
                                 ca3dmm_transport_t *t);
void ca3dmm_transport_nccl_free(ca3dmm_transport_t *t);

typedef struct ca3dmm_dist_engine *ca3dmm_dist_engine_p;

/* Every rank calls it with its own blocks (src_A ignored for B^T B, where
 * btb = 1 computes C = B^T B with n = the column count of B).  proc_grid as in
 * ca3dmm_engine_init (NULL: the reference's choice for p = size).  gemm_mode
 * and slices as in ca3dmm_engine_set_gemm_mode for the local GEMM (modes 0, 1,
 * 2).  Ranks whose arguments disagree on m, n, k, transposes, mode or grid all
 * fail.  Makes no CUDA call: device buffers are made at the first exec. */
int ca3dmm_dist_engine_init(int m, int n, int k, int trans_A, int trans_B, int btb,
                            int src_A_srow, int src_A_nrow, int src_A_scol, int src_A_ncol,
                            int src_B_srow, int src_B_nrow, int src_B_scol, int src_B_ncol,
                            int dst_C_srow, int dst_C_nrow, int dst_C_scol, int dst_C_ncol,
                            const int *proc_grid, const ca3dmm_transport_t *transport,
                            int gemm_mode, int slices, ca3dmm_dist_engine_p *engine);
/* This rank's part of C = op(A) op(B) (or B^T B); every rank calls it.  A, B,
 * C: this rank's blocks (device, column-major, ld >= the block's rows; A may
 * be NULL for B^T B).  Synchronous.  Returns 0 or a CA3DMM_E* code. */
int ca3dmm_dist_engine_exec(ca3dmm_dist_engine_p engine, const double *A, int ldA,
                            const double *B, int ldB, double *C, int ldC);
/* grid and this rank's role: out[0..3] = mp, np, kp, rp; out[4] = active;
 * out[5] = slab; out[6..9] = C_2dmm block (srow, nrow, scol, ncol) */
int ca3dmm_dist_engine_info(ca3dmm_dist_engine_p engine, int out[10]);
/* elements this rank sends to / receives from each peer in the operand and C
 * exchanges (arrays of `size`; any may be NULL) */
int ca3dmm_dist_engine_counts(ca3dmm_dist_engine_p engine, long long *send_ab,
                              long long *recv_ab, long long *send_c, long long *recv_c);
/* accumulated wall time (ms) of the execs: [0] operand exchange, [1] local
 * GEMM, [2] C exchange and slab sum, [3] total; returns the exec count */
int ca3dmm_dist_engine_stats(ca3dmm_dist_engine_p engine, double out[4]);
void ca3dmm_dist_engine_free(ca3dmm_dist_engine_p *engine);

#ifdef __cplusplus
}
#endif
#endif
