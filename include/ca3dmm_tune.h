/* Autotuner and learned cost model for the ca3dmm engine.
 *
 * No counterpart in the reference, which has no tuning: its only knobs are
 * the process grid (proc_grid / CA3DMM_REDUCE_KP) and CANNON_MIN_KBLK_SIZE.
 *
 * A configuration is (gemm mode, slices or moduli, k-slab split kp, tile
 * raster or band, tile width).  The tuner runs a candidate list through the
 * engine on the caller's operands and times each on the device (exhaustive
 * mode), or ranks the candidates with the MLP cost model and times only the
 * top-k (model mode).  The MLP (FP32, nin -> h1 -> h2 -> 1, ReLU, Adam on MSE)
 * has hand-written CUDA forward, backward and update kernels; it predicts
 * log2(time in ms) from ca3dmm_tune_features.
 *
 * Accuracy guard: before a split-precision candidate is timed, its C is
 * compared on a sample of entries with Dot2 values of those entries
 * (compensated dot products from the operands); it is admissible only if its
 * normwise and componentwise errors on the sample are each within twice those
 * of the plain FP64 GEMM's C on the same sample (floored at 2^-53).  Half of
 * the sampled rows / columns are the ones with the largest ratio of maximum to
 * mean magnitude -- where rounding to P bits below the row maximum loses most.
 * Operands holding an Inf or a NaN admit only the plain GEMM.
 *
 * Engine wiring: an engine in CA3DMM_GEMM_AUTO mode (env CA3DMM_GEMM_MODE=auto
 * at init, or ca3dmm_engine_set_gemm_mode) runs ca3dmm_engine_autotune at its
 * first exec, on that exec's operands, then computes C with the choice.  Env:
 *   CA3DMM_AUTOTUNE   off | model | exhaustive (default model): off times
 *                     nothing (the model's best-ranked admissible candidate),
 *                     model times the top CA3DMM_TUNE_TOPK (default 2)
 *                     admissible candidates, exhaustive times all;
 *   CA3DMM_TUNE_CACHE a text file of earlier choices, keyed by problem and
 *                     grid; a hit is re-checked by the accuracy guard only;
 *   CA3DMM_COST_MODEL the MLP file (default: data/costmodel_b200.txt beside
 *                     the library).
 */
#ifndef CA3DMM_TUNE_H
#define CA3DMM_TUNE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int gemm_mode;   /* 0 plain FP64 DMMA, 1 INT8 slices, 2 modular (CRT) */
    int slices;      /* INT8 slices (mode 1); moduli (mode 2, 0 = the fewest for 51-bit integers) */
    int kp;          /* k-slab split: virtual grid 1 x 1 x kp (ca3dmm_autotune; the engine
                        tuner keeps the engine's grid and ignores it) */
    int raster;      /* modes 0, 1: tile rows per raster band (4, 8 or 16);
                        mode 2: tile rows per band of the work order (1 .. 1024) */
    int tile_n;      /* GEMM tile columns: mode 2: 128 or 256 (0 = 256); mode 0: 128 or
                        64 (0 = 128, or CA3DMM_PLAIN_TILE_N; 64 is refused for the
                        symmetric B^T B plan); mode 1 has one tile shape (128 x 64 per
                        slice) and takes 0 */
} ca3dmm_tune_cfg_t;

#define CA3DMM_TUNE_NFEAT 14

/* Cost-model features of (problem, configuration): log2 m, log2 n, log2 k,
 * trans_A, trans_B, [mode = 1], [mode = 2], slices or moduli (the count the
 * engine uses, 0 plain), log2 kp, log2 raster / band, tile rows, tile
 * columns, log2 output tiles of one slab (ceil(m / rows) ceil(n / cols)),
 * operand exponent spread (log2 of max / min nonzero |x|). */
int ca3dmm_tune_features(int m, int n, int k, int trans_A, int trans_B,
                         const ca3dmm_tune_cfg_t *cfg, float exp_spread, float *feat);

/* Device time (ms, mean of reps after one warm-up) of one engine exec of
 * C = op(A) op(B) under cfg. */
int ca3dmm_tune_measure(int m, int n, int k, int trans_A, int trans_B, const double *A, int ldA,
                        const double *B, int ldB, double *C, int ldC,
                        const ca3dmm_tune_cfg_t *cfg, int reps, float *ms);

typedef struct ca3dmm_mlp *ca3dmm_mlp_p;

/* Pick the fastest admissible of ncand candidates.  model == NULL: time all
 * (exhaustive).  Otherwise rank by the model and time the topk best-ranked
 * admissible ones.  One engine per kp serves every candidate with that kp.
 * measured_ms[i] receives the time of candidate i, -1 if not timed, -2 if
 * the accuracy guard rejected it; guard_err[i] (may be NULL) its normwise
 * error on the guard's sample (-1 if not run).  *best: the fastest timed
 * candidate; when none could be timed, the first plain candidate in the
 * model's order (the IEEE reference), else the model's first. */
int ca3dmm_autotune(int m, int n, int k, int trans_A, int trans_B, const double *A, int ldA,
                    const double *B, int ldB, double *C, int ldC, const ca3dmm_tune_cfg_t *cands,
                    int ncand, float exp_spread, ca3dmm_mlp_p model, int topk, int reps,
                    int *best, float *measured_ms, float *guard_err);

/* ---- the engine's own tuner ---- */
struct ca3dmm_engine;
/* Apply / read a configuration of an engine (cfg->kp is ignored). */
int ca3dmm_engine_set_tune(struct ca3dmm_engine *engine, const ca3dmm_tune_cfg_t *cfg);
int ca3dmm_engine_get_tune(struct ca3dmm_engine *engine, ca3dmm_tune_cfg_t *cfg);
/* Tune the engine on these operands (device pointers, as for exec; C is
 * overwritten) within its grid: how = 0 off, 1 model, 2 exhaustive (see
 * above; model falls back to exhaustive when no model file loads).  Applies
 * the choice and writes it to *chosen (may be NULL).  The engine's
 * statistics are reset afterwards. */
int ca3dmm_engine_autotune(struct ca3dmm_engine *engine, const void *A, int ldA, const void *B,
                           int ldB, void *C, int ldC, int how, ca3dmm_tune_cfg_t *chosen);
/* The candidates of the engine's last tuning: up to max of them with their
 * times (ms; -1 not timed, -2 rejected by the guard) and guard errors
 * (normwise; -1 not run).  Returns the number of candidates. */
int ca3dmm_engine_tune_report(struct ca3dmm_engine *engine, ca3dmm_tune_cfg_t *cfgs, float *ms,
                              float *err, int max);

/* ---- MLP cost model ---- */
int ca3dmm_mlp_create(int nin, int h1, int h2, unsigned long long seed, ca3dmm_mlp_p *mlp);
void ca3dmm_mlp_free(ca3dmm_mlp_p *mlp);
int ca3dmm_mlp_nparams(ca3dmm_mlp_p mlp);
int ca3dmm_mlp_inputs(ca3dmm_mlp_p mlp);   /* features per sample (nin) */
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
