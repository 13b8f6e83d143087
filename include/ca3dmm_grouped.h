/* Batched independent FP64 GEMMs in one persistent launch.
 *
 * No counterpart in the reference, which runs one ca3dmm_engine_exec per
 * product.  A batch of nprob products C_i = op(A_i) op(B_i) of any sizes and
 * transposes is planned once; each exec packs every operand (one launch per
 * operand side), then runs ONE persistent grouped GEMM launch over the tiles
 * of all products -- the plain FP64 DMMA kernel, the split-precision
 * (Ozaki INT8 slices, tcgen05) kernel, or the modular split-precision kernel
 * (one INT8 product per modulus) with its reconstruction pass.  With set_stream(.., sync = 0) exec only
 * enqueues work on the stream, so a caller may capture it in a CUDA graph and
 * replay it; the plan is re-uploaded only when a pointer or leading dimension
 * changes between calls.
 */
#ifndef CA3DMM_GROUPED_H
#define CA3DMM_GROUPED_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ca3dmm_grouped *ca3dmm_grouped_p;

/* Plan nprob products (m[i] x n[i] x k[i], trans flags per product).
 * gemm_mode: 0 plain FP64 DMMA, 1 split precision with `slices` (2..8), 2
 * modular split precision with `slices` moduli (8..18; 0: the fewest that
 * give 51-bit operand integers for the deepest product; every k <= 131072).
 * *workbuf_bytes != NULL: the caller allocates and attaches the device work
 * buffer; NULL: the batch allocates it.  Returns 0 or a CA3DMM_E* code. */
int ca3dmm_grouped_init(int nprob, const int *m, const int *n, const int *k, const int *trans_A,
                        const int *trans_B, int gemm_mode, int slices, ca3dmm_grouped_p *g,
                        size_t *workbuf_bytes);
int ca3dmm_grouped_attach_workbuf(ca3dmm_grouped_p g, void *workbuf_d);
/* stream: cudaStream_t (NULL = legacy default); sync = 1 (default): exec
 * waits and checks the device status; 0: exec only enqueues. */
void ca3dmm_grouped_set_stream(ca3dmm_grouped_p g, void *stream, int sync);
/* A[i]: op(A_i) source (m x k, or k x m when trans), ldA[i] its leading
 * dimension; likewise B; C[i] column-major m x n with ldC[i] >= m.  Device
 * pointers.  Returns 0 or a CA3DMM_E* code. */
int ca3dmm_grouped_exec(ca3dmm_grouped_p g, const double *const *A, const int *ldA,
                        const double *const *B, const int *ldB, double *const *C,
                        const int *ldC);
/* Device milliseconds of the last synchronous exec (pack + GEMM). */
double ca3dmm_grouped_last_ms(ca3dmm_grouped_p g);
void ca3dmm_grouped_free(ca3dmm_grouped_p *g);

#ifdef __cplusplus
}
#endif
#endif
