/* Autotuner for the ca3dmm engine: exhaustive timing of a candidate list, or
 * ranking by the learned cost model (ca3dmm_mlp_*) and timing only the best
 * top-k, with the accuracy guard of k_tune_guard.cu in front of every
 * split-precision candidate.  See include/ca3dmm_tune.h. */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>
#include <cuda_runtime_api.h>
#include "ca3dmm_util.h"
#include "ca3dmm_kernels.h"
#include "ca3dmm.h"
#include "ca3dmm_tune.h"
#include "ca3dmm_tune_guard.h"
#include "ca3dmm_tune_internal.h"
#include "ca3dmm_crt.h"

#define GUARD_SAMPLES 64
#define GUARD_FLOOR 0x1p-53

/* moduli the engine uses for a modular candidate (0: the fewest that give
 * 51-bit integers at this k; deeper k runs in slabs of CA3DMM_CRT_MAX_K) */
static int crt_count(int k, int want)
{
    if (want > 0) return want;
    const int ns = (k + CA3DMM_CRT_MAX_K - 1) / CA3DMM_CRT_MAX_K;
    const int kmax = (k + ns - 1) / ns;
    for (int nm = 8; nm <= CA3DMM_CRT_MAX_MODULI; nm++)
        if (ca3dmm_crt_bits(nm, kmax) >= 51) return nm;
    return CA3DMM_CRT_MAX_MODULI;
}

int ca3dmm_tune_features(int m, int n, int k, int trans_A, int trans_B,
                         const ca3dmm_tune_cfg_t *cfg, float exp_spread, float *f)
{
    if (!cfg || !f || m < 1 || n < 1 || k < 1) return CA3DMM_EINVAL;
    const int mode = cfg->gemm_mode;
    /* the tile each GEMM kernel computes: DMMA 128 x 128 or 128 x 64, slices
     * 128 x 64, modular 128 x tile_n */
    const int rows = 128;
    const int cols = mode == CA3DMM_GEMM_CRT ? (cfg->tile_n == 128 ? 128 : 256)
                     : mode == CA3DMM_GEMM_OZAKI ? 64 : (cfg->tile_n == 64 ? 64 : 128);
    const int raster = cfg->raster > 0 ? cfg->raster : (mode == CA3DMM_GEMM_CRT ? 32 : 8);
    f[0] = (float) log2((double) m);
    f[1] = (float) log2((double) n);
    f[2] = (float) log2((double) k);
    f[3] = (float) (trans_A != 0);
    f[4] = (float) (trans_B != 0);
    f[5] = (float) (mode == CA3DMM_GEMM_OZAKI);
    f[6] = (float) (mode == CA3DMM_GEMM_CRT);
    f[7] = mode == CA3DMM_GEMM_OZAKI ? (float) cfg->slices
           : mode == CA3DMM_GEMM_CRT ? (float) crt_count(k, cfg->slices) : 0.f;
    f[8] = (float) log2((double) (cfg->kp > 0 ? cfg->kp : 1));
    f[9] = (float) log2((double) raster);
    f[10] = (float) rows;
    f[11] = (float) cols;
    f[12] = (float) log2((double) ((m + rows - 1) / rows) * (double) ((n + cols - 1) / cols));
    f[13] = exp_spread;
    return CA3DMM_OK;
}

/* A 1 x 1 x kp engine over the whole operands (the tuner's own engine). */
static ca3dmm_engine_p make_engine(int m, int n, int k, int trans_A, int trans_B, int kp,
                                   MPI_Comm *comm)
{
    if (ca3dmm_vcomm_create(kp, comm)) return NULL;
    const int grid[3] = {1, 1, kp};
    const int ar = trans_A ? k : m, ac = trans_A ? m : k, br = trans_B ? n : k, bc = trans_B ? k : n;
    ca3dmm_engine_p e = NULL;
    ca3dmm_engine_init(m, n, k, trans_A, trans_B, 0, ar, 0, ac, 0, br, 0, bc, 0, m, 0, n, grid,
                       *comm, DEV_TYPE_CUDA, &e, NULL);
    if (!e) ca3dmm_vcomm_free(comm);
    return e;
}

int ca3dmm_tune_measure(int m, int n, int k, int trans_A, int trans_B, const double *A, int ldA,
                        const double *B, int ldB, double *C, int ldC,
                        const ca3dmm_tune_cfg_t *cfg, int reps, float *ms)
{
    if (!cfg || !ms || reps < 1 || cfg->kp < 1 || cfg->kp > k) return CA3DMM_EINVAL;
    MPI_Comm comm;
    ca3dmm_engine_p e = make_engine(m, n, k, trans_A, trans_B, cfg->kp, &comm);
    if (!e) return CA3DMM_EINVAL;
    int rc = ca3dmm_engine_set_tune(e, cfg);
    if (!rc) rc = ca3dmm_engine_exec_reps(e, A, ldA, B, ldB, C, ldC, 1, NULL);   /* warm-up */
    if (!rc) rc = ca3dmm_engine_exec_reps(e, A, ldA, B, ldB, C, ldC, reps, ms);
    ca3dmm_engine_free(&e);
    ca3dmm_vcomm_free(&comm);
    return rc;
}

/* ---------------------------------------------------------------------------
 * The candidate walk shared by ca3dmm_autotune and ca3dmm_engine_autotune. */

typedef struct {
    double ref_n, ref_c;       /* the plain GEMM's guard errors (thresholds / 2) */
    int have_ref;
} guard_ref_t;

/* One candidate on engine e: apply, run once (plan upload, warm-up) and check
 * the guard; then time `reps` execs when ntime.  *ms: time, -2 rejected, -1
 * not timed / failed; *err: normwise guard error or -1. */
static int try_candidate(ca3dmm_engine_p e, const ca3dmm_tune_cfg_t *c, const void *A, int ldA,
                         const void *B, int ldB, void *C, int ldC, const ca3dmm_guard_t *g,
                         guard_ref_t *ref, int timed, int reps, float *ms, float *err)
{
    *ms = -1.f;
    *err = -1.f;
    int rc = ca3dmm_engine_set_tune(e, c);
    if (rc) return rc;                                  /* e.g. no room in a caller's buffer */
    rc = ca3dmm_engine_exec_reps(e, A, ldA, B, ldB, C, ldC, 1, NULL);
    if (rc) return rc;
    if (g) {
        const double *Cf;
        long long ldf;
        double en = 0.0, ec = 0.0;
        ca3dmm_engine_full_c(e, C, ldC, &Cf, &ldf);
        rc = ca3dmm_guard_error(g, Cf, ldf, &en, &ec, e->stream);
        if (rc) return rc;
        *err = (float) en;
        if (c->gemm_mode == CA3DMM_GEMM_PLAIN) {
            if (!ref->have_ref) {
                ref->ref_n = en;
                ref->ref_c = ec;
                ref->have_ref = 1;
            }
        } else {
            const double tn = 2.0 * (ref->ref_n > GUARD_FLOOR ? ref->ref_n : GUARD_FLOOR);
            const double tc = 2.0 * (ref->ref_c > GUARD_FLOOR ? ref->ref_c : GUARD_FLOOR);
            if (g->nonfinite || !ref->have_ref || !(en <= tn) || !(ec <= tc)) {
                *ms = -2.f;
                return CA3DMM_OK;
            }
        }
    }
    if (timed) rc = ca3dmm_engine_exec_reps(e, A, ldA, B, ldB, C, ldC, reps, ms);
    return rc;
}

/* rank candidates by the model's predicted time (stable insertion sort) */
static int rank_by_model(ca3dmm_mlp_p model, int m, int n, int k, int tA, int tB,
                         const ca3dmm_tune_cfg_t *c, int nc, float spread, int *order)
{
    for (int i = 0; i < nc; i++) order[i] = i;
    if (!model) return CA3DMM_OK;
    float *feat = (float *) malloc(sizeof(float) * (size_t) nc * CA3DMM_TUNE_NFEAT);
    float *pred = (float *) malloc(sizeof(float) * (size_t) nc);
    int rc = (!feat || !pred) ? CA3DMM_ENOMEM : CA3DMM_OK;
    for (int i = 0; i < nc && !rc; i++)
        rc = ca3dmm_tune_features(m, n, k, tA, tB, &c[i], spread, feat + (size_t) i * CA3DMM_TUNE_NFEAT);
    if (!rc) rc = ca3dmm_mlp_predict(model, feat, nc, pred);
    for (int i = 1; i < nc && !rc; i++) {
        int v = order[i], j = i - 1;
        while (j >= 0 && pred[order[j]] > pred[v]) { order[j + 1] = order[j]; j--; }
        order[j + 1] = v;
    }
    free(feat);
    free(pred);
    return rc;
}

/* the tuner's engines, one per k split, each with its plain GEMM's guard
 * errors (run when the engine is made) */
typedef struct {
    int kp;
    ca3dmm_engine_p e;
    MPI_Comm comm;
    guard_ref_t ref;
} kp_engine_t;

static void drop_engines(kp_engine_t *pool, int *np)
{
    for (int i = 0; i < *np; i++) {
        ca3dmm_engine_free(&pool[i].e);
        ca3dmm_vcomm_free(&pool[i].comm);
    }
    *np = 0;
}

int ca3dmm_autotune(int m, int n, int k, int trans_A, int trans_B, const double *A, int ldA,
                    const double *B, int ldB, double *C, int ldC, const ca3dmm_tune_cfg_t *cands,
                    int ncand, float exp_spread, ca3dmm_mlp_p model, int topk, int reps, int *best,
                    float *measured_ms, float *guard_err)
{
    if (!cands || ncand < 1 || !best || reps < 1) return CA3DMM_EINVAL;
    int *order = (int *) malloc(sizeof(int) * ncand);
    float *ms = (float *) malloc(sizeof(float) * ncand), *er = (float *) malloc(sizeof(float) * ncand);
    if (!order || !ms || !er) { free(order); free(ms); free(er); return CA3DMM_ENOMEM; }
    ca3dmm_guard_t g;
    int rc = ca3dmm_guard_create(&g, m, n, k, trans_A, trans_B, A, ldA, B, ldB, GUARD_SAMPLES, NULL);
    if (rc) { free(order); free(ms); free(er); return rc; }
    if (model && ca3dmm_mlp_inputs(model) != CA3DMM_TUNE_NFEAT) rc = CA3DMM_EINVAL;
    if (!rc) rc = rank_by_model(model, m, n, k, trans_A, trans_B, cands, ncand, exp_spread, order);
    if (!model) {
        /* exhaustive: candidates of one k split together (stable), one engine at a time */
        for (int i = 1; i < ncand; i++) {
            int v = order[i], j = i - 1;
            while (j >= 0 && cands[order[j]].kp > cands[v].kp) { order[j + 1] = order[j]; j--; }
            order[j + 1] = v;
        }
    }
    for (int i = 0; i < ncand; i++) { ms[i] = -1.f; er[i] = -1.f; }
    const int ntime = model ? (topk < 1 ? 1 : topk) : ncand;
    kp_engine_t pool[8];
    int npool = 0, timed = 0;
    for (int r = 0; r < ncand && !rc && timed < ntime; r++) {
        const int i = order[r], kp = cands[i].kp;
        if (kp < 1 || kp > k) continue;
        int slot = -1;
        for (int q = 0; q < npool; q++) if (pool[q].kp == kp) slot = q;
        if (slot < 0) {
            if (!model || npool == 8) drop_engines(pool, &npool);
            kp_engine_t *pe = &pool[npool];
            pe->kp = kp;
            pe->e = make_engine(m, n, k, trans_A, trans_B, kp, &pe->comm);
            if (!pe->e) continue;
            memset(&pe->ref, 0, sizeof(pe->ref));
            const ca3dmm_tune_cfg_t plain = {CA3DMM_GEMM_PLAIN, 0, kp, 8, 0};
            float pm, pr;
            slot = npool++;
            rc = try_candidate(pe->e, &plain, A, ldA, B, ldB, C, ldC, &g, &pe->ref, 0, 1, &pm, &pr);
            if (rc) break;
        }
        const int crc = try_candidate(pool[slot].e, &cands[i], A, ldA, B, ldB, C, ldC, &g,
                                      &pool[slot].ref, 1, reps, &ms[i], &er[i]);
        if (crc == CA3DMM_EINVAL || crc == CA3DMM_ENOMEM) { ms[i] = -1.f; continue; }
        rc = crc;
        if (!rc && ms[i] >= 0.f) timed++;
    }
    drop_engines(pool, &npool);
    *best = -1;
    for (int i = 0; i < ncand; i++)
        if (ms[i] >= 0.f && (*best < 0 || ms[i] < ms[*best])) *best = i;
    /* nothing timed: the first plain candidate in the model's order (the IEEE
     * reference, admissible whatever the guard says), else the model's first */
    for (int r = 0; r < ncand && *best < 0; r++)
        if (cands[order[r]].gemm_mode == CA3DMM_GEMM_PLAIN && ms[order[r]] != -2.f) *best = order[r];
    if (*best < 0) *best = order[0];
    for (int i = 0; i < ncand; i++) {
        if (measured_ms) measured_ms[i] = ms[i];
        if (guard_err) guard_err[i] = er[i];
    }
    ca3dmm_guard_free(&g);
    free(order); free(ms); free(er);
    return rc;
}

/* ---------------------------------------------------------------------------
 * The engine's tuner. */

/* the shipped model: CA3DMM_COST_MODEL, else data/costmodel_b200.txt in the
 * library's directory */
static ca3dmm_mlp_p load_model(void)
{
    char path[4096];
    const char *env = getenv("CA3DMM_COST_MODEL");
    if (env && *env) {
        snprintf(path, sizeof(path), "%s", env);
    } else {
        Dl_info info;
        if (!dladdr((void *) &ca3dmm_engine_autotune, &info) || !info.dli_fname) return NULL;
        snprintf(path, sizeof(path), "%s", info.dli_fname);
        char *slash = strrchr(path, '/');
        if (slash) slash[1] = '\0'; else path[0] = '\0';
        strncat(path, "data/costmodel_b200.txt", sizeof(path) - strlen(path) - 1);
    }
    ca3dmm_mlp_p mdl = NULL;
    if (ca3dmm_mlp_load(path, &mdl) != CA3DMM_OK) return NULL;
    if (ca3dmm_mlp_inputs(mdl) != CA3DMM_TUNE_NFEAT) {
        WARNING_PRINTF("cost model %s takes %d features, not %d: not used\n", path,
                       ca3dmm_mlp_inputs(mdl), CA3DMM_TUNE_NFEAT);
        ca3dmm_mlp_free(&mdl);
        return NULL;
    }
    return mdl;
}

static void operands_of(ca3dmm_engine_p e, const void **A, int *ldA, const void *B, int ldB,
                        int *tA, int *tB)
{
    if (e->is_BTB) {         /* op(A) = B^T */
        *A = B;
        *ldA = ldB;
        *tA = 1;
        *tB = 0;
    } else {
        *tA = e->trans_A;
        *tB = e->trans_B;
    }
}

int ca3dmm_engine_autotune(ca3dmm_engine_p e, const void *A, int ldA, const void *B, int ldB,
                           void *C, int ldC, int how, ca3dmm_tune_cfg_t *chosen)
{
    if (!e || !B || how < 0 || how > 2) return CA3DMM_EINVAL;
    double t0 = ca3dmm_wtime_sec();
    const int auto_state = e->gemm_auto;      /* set_tune below clears it */
    int tA, tB;
    operands_of(e, &A, &ldA, B, ldB, &tA, &tB);
    ca3dmm_tune_report_t *rep = ca3dmm_engine_report_slot(e);
    ca3dmm_tune_cfg_t c[CA3DMM_TUNE_MAX_CANDS];
    const int nc = ca3dmm_engine_candidates(e, c, CA3DMM_TUNE_MAX_CANDS);
    int topk, reps;
    GET_ENV_INT_VAR(topk, "CA3DMM_TUNE_TOPK", "tune_topk", 2, 1, CA3DMM_TUNE_MAX_CANDS);
    GET_ENV_INT_VAR(reps, "CA3DMM_TUNE_REPS", "tune_reps", 2, 1, 100);
    ca3dmm_guard_t g;
    int rc = ca3dmm_guard_create(&g, e->m, e->n, e->k, tA, tB, (const double *) A, ldA,
                                 (const double *) B, ldB, GUARD_SAMPLES, e->stream);
    if (rc) return rc;
    ca3dmm_mlp_p model = how < 2 ? load_model() : NULL;
    if (how == 1 && !model) how = 2;            /* no model: time everything */
    int order[CA3DMM_TUNE_MAX_CANDS];
    rc = rank_by_model(model, e->m, e->n, e->k, tA, tB, c, nc, g.spread, order);
    if (model) ca3dmm_mlp_free(&model);
    rep->n = nc;
    for (int i = 0; i < nc; i++) { rep->cfg[i] = c[i]; rep->ms[i] = -1.f; rep->err[i] = -1.f; }
    guard_ref_t ref = {0.0, 0.0, 0};
    /* the plain GEMM (candidate 0) first: the guard's reference */
    float pm = -1.f, pe = -1.f;
    if (!rc) rc = try_candidate(e, &c[0], A, ldA, B, ldB, C, ldC, &g, &ref, 0, 1, &pm, &pe);
    if (!rc) rep->err[0] = pe;
    const int ntime = how == 2 ? nc : topk;
    int timed = 0, pick = -1;
    for (int r = 0; r < nc && !rc; r++) {
        const int i = order[r];
        if (how == 0) {
            /* no timing: the first admissible candidate in the model's order */
            float m0, e0;
            int crc = try_candidate(e, &c[i], A, ldA, B, ldB, C, ldC, &g, &ref, 0, 1, &m0, &e0);
            if (crc == CA3DMM_ENOMEM || crc == CA3DMM_EINVAL) continue;
            rc = crc;
            rep->err[i] = e0;
            rep->ms[i] = m0;
            if (!rc && m0 != -2.f) { pick = i; break; }
            continue;
        }
        if (timed >= ntime) break;
        int crc = try_candidate(e, &c[i], A, ldA, B, ldB, C, ldC, &g, &ref, 1, reps, &rep->ms[i],
                                &rep->err[i]);
        if (crc == CA3DMM_ENOMEM || crc == CA3DMM_EINVAL) continue;
        rc = crc;
        if (!rc && rep->ms[i] >= 0.f) {
            timed++;
            if (pick < 0 || rep->ms[i] < rep->ms[pick]) pick = i;
        }
    }
    ca3dmm_guard_free(&g);
    if (pick < 0) pick = 0;                     /* the plain GEMM is always admissible */
    if (!rc) rc = ca3dmm_engine_set_tune(e, &c[pick]);
    if (rc) {
        /* a failed tuning leaves the engine on the plain GEMM, still to be tuned */
        ca3dmm_engine_set_tune(e, &c[0]);
        e->gemm_auto = auto_state;
        ca3dmm_engine_reset_stat(e);
        return rc;
    }
    e->gemm_auto = auto_state == 1 ? 2 : auto_state;
    if (chosen) *chosen = c[pick];
    ca3dmm_engine_reset_stat(e);
    e->tune_ms = 1000.0 * (ca3dmm_wtime_sec() - t0);
    return rc;
}

/* ---------------------------------------------------------------------------
 * The tuning an auto-mode engine runs at its first exec: the cache, then the
 * tuner. */

static void cache_key(ca3dmm_engine_p e, char *key, size_t len)
{
    snprintf(key, len, "v1 %d %d %d %d %d %d %d %d %d %d", e->m, e->n, e->k, e->trans_A,
             e->trans_B, e->is_BTB, e->btb_symmetric, e->mp, e->np, e->kp);
}

static int cache_lookup(const char *path, const char *key, ca3dmm_tune_cfg_t *c)
{
    FILE *f = fopen(path, "r");
    if (!f) return 0;
    char line[512];
    int found = 0;
    const size_t kl = strlen(key);
    while (fgets(line, sizeof(line), f)) {
        if (strncmp(line, key, kl) != 0 || line[kl] != ' ' || line[kl + 1] != ':') continue;
        ca3dmm_tune_cfg_t t = {0, 0, 0, 0, 0};
        if (sscanf(line + kl + 2, "%d %d %d %d", &t.gemm_mode, &t.slices, &t.raster, &t.tile_n) == 4) {
            *c = t;          /* the last matching line wins */
            found = 1;
        }
    }
    fclose(f);
    return found;
}

static void cache_store(const char *path, const char *key, const ca3dmm_tune_cfg_t *c)
{
    FILE *f = fopen(path, "a");
    if (!f) {
        WARNING_PRINTF("CA3DMM_TUNE_CACHE: cannot append to %s\n", path);
        return;
    }
    fprintf(f, "%s : %d %d %d %d\n", key, c->gemm_mode, c->slices, c->raster, c->tile_n);
    fclose(f);
}

/* a cached split-precision choice still has to pass the guard on these operands */
static int cache_verify(ca3dmm_engine_p e, const ca3dmm_tune_cfg_t *c, const void *A, int ldA,
                        const void *B, int ldB, void *C, int ldC, int *ok)
{
    *ok = 1;
    if (c->gemm_mode == CA3DMM_GEMM_PLAIN) {
        /* a plain entry needs no guard, only to be valid for this engine */
        const int rc = ca3dmm_engine_set_tune(e, c);
        if (rc == CA3DMM_EINVAL || rc == CA3DMM_ENOMEM) *ok = 0;
        return rc == CA3DMM_EINVAL || rc == CA3DMM_ENOMEM ? CA3DMM_OK : rc;
    }
    int tA, tB;
    operands_of(e, &A, &ldA, B, ldB, &tA, &tB);
    ca3dmm_guard_t g;
    int rc = ca3dmm_guard_create(&g, e->m, e->n, e->k, tA, tB, (const double *) A, ldA,
                                 (const double *) B, ldB, GUARD_SAMPLES, e->stream);
    if (rc) return rc;
    guard_ref_t ref = {0.0, 0.0, 0};
    ca3dmm_tune_cfg_t plain = {CA3DMM_GEMM_PLAIN, 0, e->kp, 8, 0};
    float ms, er;
    rc = try_candidate(e, &plain, A, ldA, B, ldB, C, ldC, &g, &ref, 0, 1, &ms, &er);
    if (!rc) {
        const int crc = try_candidate(e, c, A, ldA, B, ldB, C, ldC, &g, &ref, 0, 1, &ms, &er);
        if (crc == CA3DMM_EINVAL || crc == CA3DMM_ENOMEM) *ok = 0;   /* not for this engine */
        else if (crc) rc = crc;
        else *ok = ms != -2.f;
    }
    ca3dmm_guard_free(&g);
    return rc;
}

int ca3dmm_engine_autotune_env(ca3dmm_engine_p e, const void *A, int ldA, const void *B, int ldB,
                               void *C, int ldC)
{
    enum cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing((cudaStream_t) e->stream, &cs) == cudaSuccess &&
        cs != cudaStreamCaptureStatusNone) {
        ERROR_PRINTF("CA3DMM_GEMM_AUTO: the first exec tunes and may not be captured\n");
        return CA3DMM_EINVAL;
    }
    int how = 1;
    const char *hs = getenv("CA3DMM_AUTOTUNE");
    if (hs) {
        if (!strcasecmp(hs, "off") || !strcmp(hs, "0")) how = 0;
        else if (!strcasecmp(hs, "model") || !strcmp(hs, "1")) how = 1;
        else if (!strcasecmp(hs, "exhaustive") || !strcmp(hs, "2")) how = 2;
        else WARNING_PRINTF("CA3DMM_AUTOTUNE=%s: expected off, model or exhaustive; using model\n", hs);
    }
    const char *cache = getenv("CA3DMM_TUNE_CACHE");
    char key[256];
    cache_key(e, key, sizeof(key));
    const double t0 = ca3dmm_wtime_sec();
    ca3dmm_tune_cfg_t c;
    if (cache && *cache && cache_lookup(cache, key, &c)) {
        const int auto_state = e->gemm_auto;
        int ok = 0;
        int rc = cache_verify(e, &c, A, ldA, B, ldB, C, ldC, &ok);
        if (!rc && ok) rc = ca3dmm_engine_set_tune(e, &c);
        e->gemm_auto = auto_state;
        if (rc == CA3DMM_EINVAL || rc == CA3DMM_ENOMEM) ok = 0;   /* an entry this engine cannot take */
        else if (rc) return rc;
        if (ok) {
            ca3dmm_tune_report_t *rep = ca3dmm_engine_report_slot(e);
            rep->n = 1;
            rep->cfg[0] = c;
            rep->ms[0] = -1.f;
            rep->err[0] = -1.f;
            e->gemm_auto = 2;
            ca3dmm_engine_reset_stat(e);
            e->tune_ms = 1000.0 * (ca3dmm_wtime_sec() - t0);
            return CA3DMM_OK;
        }
    }
    int rc = ca3dmm_engine_autotune(e, A, ldA, B, ldB, C, ldC, how, &c);
    if (rc) return rc;
    if (cache && *cache) cache_store(cache, key, &c);
    return CA3DMM_OK;
}
