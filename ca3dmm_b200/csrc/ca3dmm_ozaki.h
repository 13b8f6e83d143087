/* Internal C ABI of the split-precision (Ozaki scheme, INT8 slices) GEMM.
 *
 * For op(A) rows i and op(B) columns j of one operand block over its k range:
 *   E_i = min{E : max_l |a_il| <= 2^E 127/128} (0 for a zero row),
 *   rint(a_il 2^(8s-1-E_i)) = sum_{t<s} qa_t,il 256^(s-1-t), balanced digits
 *   qa_t in [-128, 127], so a_il = sum_t qa_t,il 2^(E_i-7-8t) + r, |r| <= 2^(E_i-8s),
 * likewise F_j for the columns of op(B).  Then
 *   C_ij ~= 2^(E_i + F_j) sum_{d=s-1..0} 2^(-14 - 8d) sum_{t+u=d} (qa_t qb_u)_ij
 * where every inner sum is an exact INT32 tensor-core accumulation over k
 * chunks with s kc 2^14 < 2^31, and only the recombination over d (most
 * significant product last) and over chunks is done in FP64; the power of two
 * 2^(E_i + F_j) is applied once, at the store.  Rows and columns holding an
 * Inf or a NaN are sliced as zero rows (ca3dmm_oz_run_nonfinite). */
#ifndef CA3DMM_OZAKI_H
#define CA3DMM_OZAKI_H

#include <stddef.h>
#include <cuda_runtime_api.h>
#include "ca3dmm_kernels.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Block of op(A) or op(B).  alias >= 0 (A blocks only): this block is the
 * transpose of B block `alias` (same elements: B^T B), so it reuses that
 * block's slices and exponents instead of being sliced. */
typedef struct { int r0, c0, rows, cols, alias; } ca3dmm_oz_blk_t;

/* Where one operand block's source lives: op(X)(r, l) of the block's matrix
 * is read with leading dimension ld and transpose flag trans.  base == NULL:
 * offsets are relative to the pointer passed to ca3dmm_oz_run_pack (engine);
 * otherwise base is the block's matrix itself (batched problems). */
typedef struct {
    const void *base;
    long long ld;
    int trans, pad;
} ca3dmm_oz_src_t;

typedef struct {
    int a_blk, b_blk;     /* operand blocks */
    double *C;            /* output (column-major) */
    long long ldc;
    int m, n, k;
    int raster;           /* tile rows per raster band (0 = default) */
    int row0, col0;       /* first row of the group inside its A block (a multiple of 128) and
                             first column inside its B block (a multiple of 64) */
} ca3dmm_oz_group_t;

/* Work unit: nsub groups (group, group + sub_stride, ...) of equal m x n that
 * write the same C block (the k-slabs of one output block); each output tile
 * runs the groups in order, the first storing C and the others adding to it,
 * so the slab sum needs no separate reduction.  Without units every group is
 * its own unit. */
typedef struct {
    int group, nsub, sub_stride;
} ca3dmm_oz_unit_t;

typedef struct {
    int slices, nA, nB, ngroup, nunit, max_nsub;
    int tiles;            /* output tiles of the grouped INT8 launch (numbered per unit) */
    int max_rows, max_kpad;
    int exp_items[2];     /* exponent work items of the A / B blocks */
    int kc_tiles[2], rc_tiles[2];       /* slicing tiles of the A / B blocks: k-contiguous / rows-contiguous sources */
    long long n_exp;      /* rows with an exponent: E (int) then max bits (u64) arrays open the work region */
    void *dev_plan;       /* device copy of the plan (slice descriptors, tensor maps, groups) */
    void *dev_work;       /* slices and exponents */
} ca3dmm_oz_plan_t;

size_t ca3dmm_oz_plan_bytes(int ngroup);
size_t ca3dmm_oz_work_bytes(int nA, const int *a_rows, const int *a_k, int nB, const int *b_k,
                            const int *b_cols, int slices);
/* Build the plan into host memory host_plan (ca3dmm_oz_plan_bytes), which the
 * caller uploads to dev_plan before running.  A blocks: (r0, c0) = (first row
 * of op(A), first k), rows x cols = rows x kz; B blocks: (r0, c0) = (first k,
 * first column of op(B)), rows x cols = kz x cols. */
int ca3dmm_oz_plan_encode(ca3dmm_oz_plan_t *oz, int slices, int nA, const ca3dmm_oz_blk_t *A,
                          const ca3dmm_oz_src_t *srcA, int nB, const ca3dmm_oz_blk_t *B,
                          const ca3dmm_oz_src_t *srcB, int ngroup, const ca3dmm_oz_group_t *G,
                          int nunit, const ca3dmm_oz_unit_t *units, void *dev_work,
                          size_t work_bytes, void *host_plan, void *dev_plan);
/* Exponent extraction + slicing of every A and B block straight from the
 * caller's matrices (op(A)(i,l) = transA ? A[l + i*ldA] : A[i + l*ldA]). */
int ca3dmm_oz_run_pack(const ca3dmm_oz_plan_t *oz, const void *A, const void *B,
                       cudaStream_t stream);
/* Grouped INT8 tcgen05 GEMM with FP64 recombination into each group's C. */
int ca3dmm_oz_run_gemm(const ca3dmm_oz_plan_t *oz, int *dev_status, double timeout_s,
                       cudaStream_t stream);

/* Pieces of run_pack for pipelined execution: clear the exponent arrays
 * (once per exec, before any slicing); slice one operand side (0: every A
 * block, 1: every B block); or slice an explicit list of descriptors in device
 * memory, e.g. the A blocks restricted to a band of rows built by
 * ca3dmm_oz_encode_rows from the host copy of the plan (r0 a multiple of the
 * 128-row A tile, rows counted inside each listed A block; ntiles receives
 * the exponent item count and the KC and RC slicing tile counts). */
int ca3dmm_oz_clear(const ca3dmm_oz_plan_t *oz, cudaStream_t stream);
int ca3dmm_oz_slice_side(const ca3dmm_oz_plan_t *oz, int which, const void *src,
                         cudaStream_t stream);
size_t ca3dmm_oz_desc_bytes(void);
int ca3dmm_oz_encode_rows(const void *host_plan, int ngroup, const int *blocks, int count, int r0,
                          int r1, void *out_descs, int ntiles[3]);
/* Descriptors of whole blocks (indices into the plan's A then B blocks), with
 * their tile numbering restarted, for slicing those blocks alone. */
int ca3dmm_oz_encode_blocks(const void *host_plan, int ngroup, const int *descs, int count,
                            void *out_descs, int ntiles[3]);
int ca3dmm_oz_slice_descs(const ca3dmm_oz_plan_t *oz, const void *src, const void *dev_descs,
                          int ndesc, const int ntiles[3], cudaStream_t stream);
/* Non-finite inputs: rows of op(A) and columns of op(B) holding an Inf or a
 * NaN are sliced as zero rows; this pass then writes the IEEE value (NaN,
 * +Inf or -Inf, independent of the summation order) of every C entry in those
 * rows and columns, over the tiles of `ranges` (NULL: every tile).  Run it
 * after the GEMM over the same tiles and before any slab reduction, with the
 * operand pointers given to the slicing.  It returns at once on the device
 * when no row or column was flagged. */
int ca3dmm_oz_run_nonfinite(const ca3dmm_oz_plan_t *oz, const ca3dmm_tile_ranges_t *ranges,
                            const void *A, const void *B, cudaStream_t stream);
/* The GEMM over the tiles of `ranges` only (ca3dmm_kernels.h). */
int ca3dmm_oz_run_gemm_ranges(const ca3dmm_oz_plan_t *oz, const ca3dmm_tile_ranges_t *ranges,
                              int *dev_status, double timeout_s, cudaStream_t stream);

#ifdef __cplusplus
}
#endif
#endif
