/* Internal interface between the engine (ca3dmm.c) and its tuner
 * (autotune.c). */
#ifndef CA3DMM_TUNE_INTERNAL_H
#define CA3DMM_TUNE_INTERNAL_H

#include "ca3dmm.h"
#include "ca3dmm_tune.h"

#define CA3DMM_TUNE_MAX_CANDS 32

typedef struct {
    int n;
    ca3dmm_tune_cfg_t cfg[CA3DMM_TUNE_MAX_CANDS];
    float ms[CA3DMM_TUNE_MAX_CANDS];    /* -1 not timed, -2 rejected by the guard */
    float err[CA3DMM_TUNE_MAX_CANDS];   /* normwise guard error, -1 not run */
} ca3dmm_tune_report_t;

/* ca3dmm.c */
ca3dmm_tune_report_t *ca3dmm_engine_report_slot(ca3dmm_engine_p e);
/* reps device-exec calls; mean device time (ms) of one, from the engine's events */
int ca3dmm_engine_exec_reps(ca3dmm_engine_p e, const void *A, int ldA, const void *B, int ldB,
                            void *C, int ldC, int reps, float *ms);
/* where the whole C of the last exec is (dst_C, or the engine's own C) */
int ca3dmm_engine_full_c(ca3dmm_engine_p e, void *dst_C, int ldC, const double **C,
                         long long *ld);
/* the modular mode's moduli for a request (0: the fewest for 51-bit integers) */
int ca3dmm_engine_crt_resolve(ca3dmm_engine_p e, int want);
/* work-buffer bytes the engine's layout needs in (mode, count) */
size_t ca3dmm_engine_layout_bytes(ca3dmm_engine_p e, int mode, int count);
/* the candidates of the engine tuner, the largest work buffer among them */
int ca3dmm_engine_candidates(ca3dmm_engine_p e, ca3dmm_tune_cfg_t *cands, int max);

/* autotune.c: the tuning an auto-mode engine runs at its first exec (env
 * CA3DMM_AUTOTUNE, CA3DMM_TUNE_CACHE, CA3DMM_TUNE_TOPK, CA3DMM_TUNE_REPS) */
int ca3dmm_engine_autotune_env(ca3dmm_engine_p e, const void *A, int ldA, const void *B, int ldB,
                               void *C, int ldC);

#endif
