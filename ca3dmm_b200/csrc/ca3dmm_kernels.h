/* Internal C ABI between the C host engine and the sm_100a kernels.
 * Plain pointers and sizes only; every launcher returns 0 or a CA3DMM_E*
 * error code and never exits the process. */
#ifndef CA3DMM_KERNELS_H
#define CA3DMM_KERNELS_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    CA3DMM_OK = 0,
    CA3DMM_EINVAL = 1,       /* bad argument (size, alignment, mode) */
    CA3DMM_ECUDA = 2,        /* a CUDA runtime / driver call failed */
    CA3DMM_ETIMEOUT = 3,     /* a device-side bounded wait ran out */
    CA3DMM_ENOMEM = 4,       /* work buffer too small / allocation failed */
    CA3DMM_ENODEV = 5,       /* no sm_100 device or driver entry point missing */
    CA3DMM_ECANARY = 6,      /* a guard band of the work buffer was overwritten */
};

/* ---- plain FP64 DMMA GEMM, grouped ---------------------------------------
 * One problem: C = alpha * op(A) op(B) + beta * C, where the operands are
 * packed by the pack kernels or read in place:
 *   A: op(A) stored M-major, element (i,l) at A[i + l*lda]   (lda even, A 16B-aligned)
 *      or, with a_kmajor, K-major: element (i,l) at A[l + i*lda] (the caller's
 *      transposed A read as it lies)
 *   B: op(B) stored K-major, element (l,j) at B[l + j*ldb]   (ldb even, B 16B-aligned)
 *   C: column-major, element (i,j) at C[i + j*ldc]           (any ldc >= m)      */
typedef struct {
    const double *A; long long lda;
    const double *B; long long ldb;
    double *C; long long ldc;
    int m, n, k;
    double alpha, beta;
    int raster;          /* tile rows per raster band (0 = default 8) */
    int a_kmajor;        /* 1: A is K-major (see above) */
} ca3dmm_dgemm_desc_t;

/* Bytes of the device plan for nprob problems (tensor maps + problem records). */
size_t ca3dmm_dgemm_plan_bytes(int nprob);
/* Encode the plan into host memory `host_plan` (size plan_bytes); the caller
 * copies it to device memory `dev_plan` before launching.  Tensor maps embed
 * the device addresses of A and B.  Returns the total tile count.  Every
 * problem of one plan has the same A layout (a_kmajor), which the launch
 * repeats. */
int ca3dmm_dgemm_plan_encode(const ca3dmm_dgemm_desc_t *probs, int nprob, void *host_plan,
                             int *total_tiles);
/* The same with output tiles of 128 x tile_n (tile_n = 128, the default, or
 * 64); the launch must be given the same tile_n. */
int ca3dmm_dgemm_plan_encode_tn(const ca3dmm_dgemm_desc_t *probs, int nprob, void *host_plan,
                                int *total_tiles, int tile_n);
/* Up to CA3DMM_MAX_RANGES contiguous ranges [begin, begin + len) of a grouped
 * plan's tile list (each problem's tiles are numbered in raster bands of
 * `raster` tile rows, so a band of output rows is one range per problem). */
#define CA3DMM_MAX_RANGES 8
#define CA3DMM_MAX_CANARIES 8
typedef struct {
    int n;
    int begin[CA3DMM_MAX_RANGES], len[CA3DMM_MAX_RANGES];
} ca3dmm_tile_ranges_t;

/* Persistent grouped launch over every tile of every problem. */
int ca3dmm_dgemm_launch(const void *dev_plan, int nprob, int total_tiles, int a_kmajor,
                        int *dev_status, double timeout_s, cudaStream_t stream);
/* The same over the tiles of `ranges` only. */
int ca3dmm_dgemm_launch_ranges(const void *dev_plan, int nprob, const ca3dmm_tile_ranges_t *ranges,
                               int a_kmajor, int *dev_status, double timeout_s,
                               cudaStream_t stream);
/* Both for a plan encoded with tile_n (ca3dmm_dgemm_plan_encode_tn). */
int ca3dmm_dgemm_launch_tn(const void *dev_plan, int nprob, int total_tiles, int a_kmajor,
                           int *dev_status, double timeout_s, cudaStream_t stream, int tile_n);
int ca3dmm_dgemm_launch_ranges_tn(const void *dev_plan, int nprob,
                                  const ca3dmm_tile_ranges_t *ranges, int a_kmajor,
                                  int *dev_status, double timeout_s, cudaStream_t stream,
                                  int tile_n);

/* ---- pack / transpose ----------------------------------------------------
 * Batched block copies between column-major matrices.  Descriptor j copies a
 * rows x cols block: dst[r + c*ldd] = trans ? src[c + r*lds] : src[r + c*lds],
 * with src = src_base + src_off (elements) and dst = dst_base + dst_off. */
typedef struct {
    long long src_off, lds;
    long long dst_off, ldd;
    int rows, cols, trans;
    int tile_begin;          /* first 64 x 64 tile of this block (set by ca3dmm_pack_tiles) */
} ca3dmm_pack_desc_t;

/* Transposing packs whose source blocks are 16-byte aligned with an even
 * leading dimension run staged through shared memory by TMA:
 * ca3dmm_pack_tma_prepare encodes one tensor map per descriptor into
 * host_tmaps (128 B each; the caller uploads them 64-byte aligned) and sets
 * the descriptors' tile_begin for that kernel's 64 x 16 tiles; it returns
 * CA3DMM_EINVAL when a descriptor is not eligible (then use
 * ca3dmm_pack_tiles + ca3dmm_pack_launch). */
int ca3dmm_pack_tma_prepare(ca3dmm_pack_desc_t *descs, int ndesc, const double *src_base,
                            void *host_tmaps, int *total_tiles);
int ca3dmm_pack_tma_launch(const void *dev_tmaps, const ca3dmm_pack_desc_t *dev_descs, int ndesc,
                           int total_tiles, double *dst_base, int *dev_status, double timeout_s,
                           cudaStream_t stream);

/* Assign each descriptor its range of 64 x 64 tiles; returns the total. */
int ca3dmm_pack_tiles(ca3dmm_pack_desc_t *descs, int ndesc);
/* One launch over the flat tile list of all descriptors (any mix of sizes and
 * transposes).  Element offsets are taken from src_base / dst_base; with a
 * NULL base the offset is an absolute address divided by 8 (batches whose
 * blocks live in unrelated allocations). */
int ca3dmm_pack_launch(const double *src_base, double *dst_base,
                       const ca3dmm_pack_desc_t *dev_descs, int ndesc, int total_tiles,
                       cudaStream_t stream);

/* One column-major block copy dst[r + c*ldd] = src[r + c*lds] (rows x cols),
 * stream-ordered, the geometry passed as kernel arguments. */
int ca3dmm_copy_block_launch(const double *src, long long lds, double *dst, long long ldd,
                             int rows, int cols, cudaStream_t stream);

/* ---- kp-slab reduction ---------------------------------------------------
 * out[i + j*ldo] = sum_{s=0}^{nslab-1} slab[s*slab_stride + i + j*lds]
 * (summed in slab order 0,1,...). */
/* C(i, j) = C(j, i) for i > j (n x n C, column-major). */
int ca3dmm_mirror_upper_launch(double *C, long long ldc, int n, cudaStream_t stream);
int ca3dmm_reduce_slabs_launch(const double *slab, long long slab_stride, long long lds,
                               int nslab, int m, int n, double *out, long long ldo,
                               cudaStream_t stream);

/* ---- work-buffer guard bands ----------------------------------------------
 * Checks n bands of `bytes` bytes at base + offsets[i] (each filled with
 * `pattern`); a band that differs sets *status to the canary code (first
 * writer wins) and records the band index in status[1]. */
typedef struct {
    int n, bytes, pattern, pad;
    long long off[CA3DMM_MAX_CANARIES];
} ca3dmm_guard_bands_t;
int ca3dmm_guard_check_launch(const void *base, const ca3dmm_guard_bands_t *bands, int *dev_status,
                              cudaStream_t stream);

/* ---- device properties (cached) ------------------------------------------ */
int ca3dmm_device_sm_count(void);

/* Adds n to the library's count of kernel launches (ca3dmm_kernel_launches). */
void ca3dmm_note_launch(int n);

#ifdef __cplusplus
}
#endif
#endif
