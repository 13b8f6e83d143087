/* Autotuner and learned cost model for the ca3dmm engine.
 *
 * No counterpart in the reference, which has no tuning: its only knobs are
 * the process grid (proc_grid / CA3DMM_REDUCE_KP) and CANNON_MIN_KBLK_SIZE.
 *
 * A configuration is (gemm mode, slices, k-slab split kp, tile raster).  The
 * tuner runs a candidate list through ca3dmm_engine_exec on the caller's
 * operands and times each on the device (exhaustive mode), or ranks the
 * candidates with the MLP cost model and times only the top-k (model mode).
 * The MLP (FP32, nin -> h1 -> h2 -> 1, ReLU, Adam on MSE) has hand-written
 * CUDA forward, backward and update kernels; it predicts log2(time in ms)
 * from ca3dmm_tune_features.
 */
#ifndef CA3DMM_TUNE_H
#define CA3DMM_TUNE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int gemm_mode;   /* 0 plain FP64 DMMA, 1 split precision */
    int slices;      /* INT8 slices (split precision) */
    int kp;          /* k-slab split: virtual grid 1 x 1 x kp */
    int raster;      /* tile rows grouped per raster band (L2 reuse): 4, 8 or 16 */
} ca3dmm_tune_cfg_t;

#define CA3DMM_TUNE_NFEAT 12

/* Cost-model features of (problem, configuration): log2 m, log2 n, log2 k,
 * trans_A, trans_B, gemm mode, slices, log2 kp, log2 raster, tile rows,
 * tile columns, operand exponent spread (log2 of max/min nonzero |x|). */
int ca3dmm_tune_features(int m, int n, int k, int trans_A, int trans_B,
                         const ca3dmm_tune_cfg_t *cfg, float exp_spread, float *feat);

/* Device time (ms, mean of reps after one warm-up) of one engine exec of
 * C = op(A) op(B) under cfg. */
int ca3dmm_tune_measure(int m, int n, int k, int trans_A, int trans_B, const double *A, int ldA,
                        const double *B, int ldB, double *C, int ldC,
                        const ca3dmm_tune_cfg_t *cfg, int reps, float *ms);

typedef struct ca3dmm_mlp *ca3dmm_mlp_p;

/* Pick the fastest of ncand candidates.  model == NULL: time all
 * (exhaustive).  Otherwise rank by the model and time the topk best-ranked.
 * measured_ms[i] receives the time of candidate i or -1 if not timed.
 * *best: index of the chosen candidate. */
int ca3dmm_autotune(int m, int n, int k, int trans_A, int trans_B, const double *A, int ldA,
                    const double *B, int ldB, double *C, int ldC, const ca3dmm_tune_cfg_t *cands,
                    int ncand, float exp_spread, ca3dmm_mlp_p model, int topk, int reps,
                    int *best, float *measured_ms);

/* ---- MLP cost model ---- */
int ca3dmm_mlp_create(int nin, int h1, int h2, unsigned long long seed, ca3dmm_mlp_p *mlp);
void ca3dmm_mlp_free(ca3dmm_mlp_p *mlp);
int ca3dmm_mlp_nparams(ca3dmm_mlp_p mlp);
int ca3dmm_mlp_get_params(ca3dmm_mlp_p mlp, float *host_params);
int ca3dmm_mlp_set_params(ca3dmm_mlp_p mlp, const float *host_params);
int ca3dmm_mlp_set_normalisation(ca3dmm_mlp_p mlp, const float *mean, const float *stdv);
/* One forward + backward on already-normalised features; loss = mean
 * 0.5 (y_hat - y)^2, gradients averaged over the batch (host arrays). */
int ca3dmm_mlp_fwd_bwd(ca3dmm_mlp_p mlp, const float *X, const float *y, int batch, float *loss,
                       float *grads);
/* Train with Adam on raw features (normalisation statistics computed here). */
int ca3dmm_mlp_train(ca3dmm_mlp_p mlp, const float *X, const float *y, int n, int epochs,
                     int batch, float lr, unsigned long long seed, float *final_loss);
int ca3dmm_mlp_predict(ca3dmm_mlp_p mlp, const float *X, int n, float *out);
int ca3dmm_mlp_save(ca3dmm_mlp_p mlp, const char *path);
int ca3dmm_mlp_load(const char *path, ca3dmm_mlp_p *mlp);

#ifdef __cplusplus
}
#endif
#endif
