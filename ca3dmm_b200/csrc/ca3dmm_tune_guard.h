/* Accuracy guard of the autotuner (k_tune_guard.cu): Dot2 values of a sample
 * of C's entries, and a candidate C's error on that sample. */
#ifndef CA3DMM_TUNE_GUARD_H
#define CA3DMM_TUNE_GUARD_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int m, n, k;
    int nr, nc;            /* sampled rows of op(A) / columns of op(B) */
    int nonfinite;         /* an operand holds an Inf or a NaN */
    float spread;          /* log2(max |x| / min nonzero |x|) over both operands */
    double truth_norm;     /* sum over the sample of |Dot2 value| */
    int *d_rows, *d_cols;
    double *d_truth, *d_absprod, *d_out;
    void *mem;             /* the one device allocation holding the arrays above */
} ca3dmm_guard_t;

/* Sample up to `samples` rows of op(A) and columns of op(B) (device operands,
 * column-major) and compute their entries' Dot2 values; synchronous on
 * `stream` (cudaStream_t). */
int ca3dmm_guard_create(ca3dmm_guard_t *g, int m, int n, int k, int trans_A, int trans_B,
                        const double *A, int ldA, const double *B, int ldB, int samples,
                        void *stream);
/* Error of C (device, ldC) on the sample: normwise sum |C - T| / sum |T| and
 * componentwise max |C - T| / (|A||B|)_ij; NaN when a sampled entry of C is
 * not finite. */
int ca3dmm_guard_error(const ca3dmm_guard_t *g, const double *C, long long ldC, double *normwise,
                       double *componentwise, void *stream);
void ca3dmm_guard_free(ca3dmm_guard_t *g);

#ifdef __cplusplus
}
#endif
#endif
