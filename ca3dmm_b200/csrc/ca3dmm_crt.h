/* Internal C ABI of the modular split-precision GEMM (the CRT scheme).
 *
 * For one GEMM group C = op(A) op(B) over its k range:
 *   E_i = frexp exponent of max_l |a_il| (max < 2^E_i; 0 for a zero row),
 *   a'_il = rint(a_il 2^(P - E_i)), |a'| <= 2^P, likewise F_j, b'_lj for the
 *   columns of op(B);
 *   C'_ij = sum_l a'_il b'_lj, an integer with |C'| <= k 2^(2P).
 * The device never forms C' directly: for each of N pairwise coprime moduli
 * p_t <= 256 it multiplies the residues a' mod p_t and b' mod p_t (signed
 * bytes) with one exact INT8 tensor-core GEMM and reduces the INT32 sums mod
 * p_t; the Chinese remainder theorem then gives C' exactly (P is chosen so
 * that k 2^(2P+1) < prod p_t, at most 53), and
 *   C_ij = (C' rounded once to double) 2^(E_i + F_j - 2P).
 * Its error is that of rounding the operands to P bits below their row /
 * column maximum; N INT8 GEMMs replace the s(s+1)/2 slice products of the
 * slicing scheme (ca3dmm_ozaki.h).  Rows and columns holding an Inf or a NaN
 * are zero rows until ca3dmm_crt_run_nonfinite gives their entries the IEEE
 * value. */
#ifndef CA3DMM_CRT_H
#define CA3DMM_CRT_H

#include <stddef.h>
#include <cuda_runtime_api.h>
#include "ca3dmm_kernels.h"
#include "ca3dmm_ozaki.h"

#ifdef __cplusplus
extern "C" {
#endif

#define CA3DMM_CRT_MAX_MODULI 18
#define CA3DMM_CRT_MAX_K 131072   /* exact INT32 sums of residue products: k 2^14 < 2^31 */

/* One GEMM group: C (column-major, ldc) = op(A block a_blk) op(B block b_blk),
 * m x n over the blocks' k range (the same for both).  band: 128-row tile
 * rows per band of the GEMM's work list (0 = 8); within a band the moduli
 * run one after the other over the band's tiles, so a band of output rows is
 * one contiguous range of work items. */
typedef struct {
    int a_blk, b_blk;
    double *C;
    long long ldc;
    int m, n, k;
    int band;
    int tile_n;     /* GEMM tile columns: 128 or 256 (0 = 256); the same in every group */
} ca3dmm_crt_group_t;

typedef struct {
    int nmod, nA, nB, ngroup;
    int items;            /* GEMM work items (nmod x tiles over every group) */
    int exp_items[2];     /* exponent work items of the A / B blocks */
    int kc_tiles[2], rc_tiles[2];
    int p_min, p_max;     /* integer widths of the groups */
    long long n_exp;
    long long recon_items;  /* reconstruction items (4 rows x 1 column) over every group */
    int group_m, group_n;   /* the group's size when the plan has one group */
    int tile_n;             /* GEMM tile columns of every group */
    void *dev_plan;
    void *dev_work;
} ca3dmm_crt_plan_t;

/* Integer width P (<= 53) for nmod moduli and depth k: the largest P with
 * k 2^(2P+1) < prod p_t; below 2 the modulus count is too small. */
int ca3dmm_crt_bits(int nmod, long long k);
/* Modulus t of the list (256, 255, 253, 251, 247, 241, ...: pairwise coprime). */
int ca3dmm_crt_modulus(int t);

size_t ca3dmm_crt_plan_bytes(int nblk, int ngroup);
size_t ca3dmm_crt_work_bytes(int nA, const int *a_rows, const int *a_k, int nB, const int *b_k,
                             const int *b_cols, int ngroup, const int *g_m, const int *g_n,
                             int nmod);
/* Blocks as in ca3dmm_oz_plan_encode (alias >= 0: the A block is the
 * transpose of that B block and shares its residues). */
int ca3dmm_crt_plan_encode(ca3dmm_crt_plan_t *pl, int nmod, int nA, const ca3dmm_oz_blk_t *A,
                           const ca3dmm_oz_src_t *srcA, int nB, const ca3dmm_oz_blk_t *B,
                           const ca3dmm_oz_src_t *srcB, int ngroup, const ca3dmm_crt_group_t *G,
                           void *dev_work, size_t work_bytes, void *host_plan, void *dev_plan);
/* Exponents and residues of every block (clears the exponent arrays first). */
int ca3dmm_crt_run_pack(const ca3dmm_crt_plan_t *pl, const void *A, const void *B,
                        cudaStream_t stream);
/* Pieces for pipelined execution: clear; one side; an explicit descriptor list
 * (from ca3dmm_crt_encode_rows / _blocks, as for the slicing scheme). */
int ca3dmm_crt_clear(const ca3dmm_crt_plan_t *pl, cudaStream_t stream);
int ca3dmm_crt_pack_side(const ca3dmm_crt_plan_t *pl, int which, const void *src,
                         cudaStream_t stream);
int ca3dmm_crt_encode_rows(const void *host_plan, int ngroup, const int *blocks, int count, int r0,
                           int r1, void *out_descs, int ntiles[3]);
int ca3dmm_crt_encode_blocks(const void *host_plan, int ngroup, const int *descs, int count,
                             void *out_descs, int ntiles[3]);
int ca3dmm_crt_pack_descs(const ca3dmm_crt_plan_t *pl, const void *src, const void *dev_descs,
                          int ndesc, const int ntiles[3], cudaStream_t stream);
/* First work item and item count of group g, and of the band of tile rows
 * [tile_lo, tile_hi) of group g (read from the host copy of the plan). */
int ca3dmm_crt_group_items(const void *host_plan, int g, int tile_lo, int tile_hi, int *begin,
                           int *count);
/* The INT8 GEMMs (residue planes of C) over the work items of `ranges`
 * (NULL: all). */
int ca3dmm_crt_run_gemm(const ca3dmm_crt_plan_t *pl, const ca3dmm_tile_ranges_t *ranges,
                        int *dev_status, double timeout_s, cudaStream_t stream);
/* C from the residue planes, for groups [g0, g1) and rows [r0, r1) of each. */
int ca3dmm_crt_run_reconstruct(const ca3dmm_crt_plan_t *pl, int g0, int g1, int r0, int r1,
                               cudaStream_t stream);
/* The same with at most max_blocks blocks of 256 threads (0: 8 per SM), so
 * that it can share the SMs with a GEMM launch running beside it. */
int ca3dmm_crt_run_reconstruct_capped(const ca3dmm_crt_plan_t *pl, int g0, int g1, int r0, int r1,
                                      int max_blocks, cudaStream_t stream);
/* IEEE values of the entries in rows / columns holding an Inf or a NaN, for
 * groups [g0, g1) and rows [r0, r1); after the reconstruction.  Returns at once
 * on the device when no row or column was flagged. */
int ca3dmm_crt_run_nonfinite(const ca3dmm_crt_plan_t *pl, int g0, int g1, int r0, int r1,
                             const void *A, const void *B, cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif
