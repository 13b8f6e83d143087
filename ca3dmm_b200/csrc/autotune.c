/* Autotuner for the ca3dmm engine: exhaustive timing of a candidate list, or
 * ranking by the learned cost model (ca3dmm_mlp_*) and timing only the best
 * top-k.  See include/ca3dmm_tune.h. */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <cuda_runtime_api.h>
#include "ca3dmm_util.h"
#include "ca3dmm_kernels.h"
#include "ca3dmm.h"
#include "ca3dmm_tune.h"

int ca3dmm_tune_features(int m, int n, int k, int trans_A, int trans_B,
                         const ca3dmm_tune_cfg_t *cfg, float exp_spread, float *f)
{
    if (!cfg || !f || m < 1 || n < 1 || k < 1) return CA3DMM_EINVAL;
    f[0] = (float) log2((double) m);
    f[1] = (float) log2((double) n);
    f[2] = (float) log2((double) k);
    f[3] = (float) (trans_A != 0);
    f[4] = (float) (trans_B != 0);
    f[5] = (float) cfg->gemm_mode;
    f[6] = cfg->gemm_mode ? (float) cfg->slices : 0.f;
    f[7] = (float) log2((double) (cfg->kp > 0 ? cfg->kp : 1));
    f[8] = (float) log2((double) (cfg->raster > 0 ? cfg->raster : 8));
    f[9] = 128.f;                                   /* tile rows of both GEMM kernels */
    f[10] = cfg->gemm_mode ? 64.f : 128.f;          /* tile columns */
    f[11] = exp_spread;
    return CA3DMM_OK;
}

int ca3dmm_tune_measure(int m, int n, int k, int trans_A, int trans_B, const double *A, int ldA,
                        const double *B, int ldB, double *C, int ldC,
                        const ca3dmm_tune_cfg_t *cfg, int reps, float *ms)
{
    if (!cfg || !ms || reps < 1 || cfg->kp < 1 || cfg->kp > k) return CA3DMM_EINVAL;
    MPI_Comm comm;
    if (ca3dmm_vcomm_create(cfg->kp, &comm)) return CA3DMM_EINVAL;
    const int grid[3] = {1, 1, cfg->kp};
    const int ar = trans_A ? k : m, ac = trans_A ? m : k, br = trans_B ? n : k, bc = trans_B ? k : n;
    ca3dmm_engine_p e = NULL;
    ca3dmm_engine_init(m, n, k, trans_A, trans_B, 0, ar, 0, ac, 0, br, 0, bc, 0, m, 0, n, grid,
                       comm, DEV_TYPE_CUDA, &e, NULL);
    int rc = e ? CA3DMM_OK : CA3DMM_EINVAL;
    if (!rc && cfg->gemm_mode) rc = ca3dmm_engine_set_gemm_mode(e, CA3DMM_GEMM_OZAKI, cfg->slices);
    if (!rc && cfg->raster) rc = ca3dmm_engine_set_raster(e, cfg->raster);
    if (!rc) {
        ca3dmm_engine_exec(e, A, ldA, B, ldB, C, ldC);     /* warm-up (plan upload) */
        rc = ca3dmm_engine_last_error(e);
    }
    if (!rc) {
        ca3dmm_engine_reset_stat(e);
        for (int r = 0; r < reps && !rc; r++) {
            ca3dmm_engine_exec(e, A, ldA, B, ldB, C, ldC);
            rc = ca3dmm_engine_last_error(e);
        }
    }
    if (!rc)
        *ms = (float) ((e->redist_ms + e->cannon_ms + e->reduce_ms) / (e->n_exec > 0 ? e->n_exec : 1));
    ca3dmm_engine_free(&e);
    ca3dmm_vcomm_free(&comm);
    return rc;
}

int ca3dmm_autotune(int m, int n, int k, int trans_A, int trans_B, const double *A, int ldA,
                    const double *B, int ldB, double *C, int ldC, const ca3dmm_tune_cfg_t *cands,
                    int ncand, float exp_spread, ca3dmm_mlp_p model, int topk, int reps, int *best,
                    float *measured_ms)
{
    if (!cands || ncand < 1 || !best) return CA3DMM_EINVAL;
    int *order = (int *) malloc(sizeof(int) * ncand);
    float *pred = (float *) malloc(sizeof(float) * ncand);
    float *feat = (float *) malloc(sizeof(float) * ncand * CA3DMM_TUNE_NFEAT);
    if (!order || !pred || !feat) { free(order); free(pred); free(feat); return CA3DMM_ENOMEM; }
    int rc = CA3DMM_OK, ntime = ncand;
    for (int i = 0; i < ncand; i++) order[i] = i;
    if (model) {
        for (int i = 0; i < ncand && !rc; i++)
            rc = ca3dmm_tune_features(m, n, k, trans_A, trans_B, &cands[i], exp_spread,
                                      feat + (size_t) i * CA3DMM_TUNE_NFEAT);
        if (!rc) rc = ca3dmm_mlp_predict(model, feat, ncand, pred);
        /* rank by predicted time (insertion sort; lists are short) */
        for (int i = 1; i < ncand && !rc; i++) {
            int v = order[i], j = i - 1;
            while (j >= 0 && pred[order[j]] > pred[v]) { order[j + 1] = order[j]; j--; }
            order[j + 1] = v;
        }
        ntime = topk < 1 ? 1 : (topk < ncand ? topk : ncand);
    }
    if (measured_ms)
        for (int i = 0; i < ncand; i++) measured_ms[i] = -1.f;
    float tbest = 0.f;
    *best = order[0];
    for (int r = 0; r < ntime && !rc; r++) {
        float t = 0.f;
        int i = order[r];
        int mrc = ca3dmm_tune_measure(m, n, k, trans_A, trans_B, A, ldA, B, ldB, C, ldC, &cands[i],
                                      reps, &t);
        if (mrc) continue;           /* an invalid candidate (e.g. kp > k) is skipped */
        if (measured_ms) measured_ms[i] = t;
        if (tbest == 0.f || t < tbest) { tbest = t; *best = i; }
    }
    free(order); free(pred); free(feat);
    return rc;
}
