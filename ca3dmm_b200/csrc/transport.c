/* Transports of the multi-GPU engine (include/ca3dmm_dist.h): threads of one
 * process exchanging through host memory, and NCCL loaded at run time. */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <errno.h>
#include <pthread.h>
#include <time.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <cuda_runtime_api.h>
#include <nccl.h>
#include "ca3dmm_util.h"
#include "ca3dmm_kernels.h"
#include "ca3dmm_dist.h"

/* ------------------------------------------------------------------ threads */

typedef struct {
    int size;
    pthread_mutex_t mu;         /* a barrier with a time limit: a rank that never */
    pthread_cond_t cv;          /* arrives fails the others' collective instead of */
    int arrived;                /* hanging them (CA3DMM_DIST_TIMEOUT seconds, 300) */
    unsigned long long phase;
    int broken;
    double limit_s;
    const void **ptr;           /* per rank: its send buffer / contribution */
    const long long **cnt, **dsp;
    int n;                      /* allgather: values per rank */
} thr_shared_t;

/* 0 when every rank arrived; nonzero when the limit passed first (the
 * exchange area is then broken and every later collective fails at once) */
static int thr_barrier(thr_shared_t *s)
{
    pthread_mutex_lock(&s->mu);
    if (s->broken) {
        pthread_mutex_unlock(&s->mu);
        return 1;
    }
    const unsigned long long ph = s->phase;
    if (++s->arrived == s->size) {
        s->arrived = 0;
        s->phase++;
        pthread_cond_broadcast(&s->cv);
        pthread_mutex_unlock(&s->mu);
        return 0;
    }
    struct timespec dl;
    clock_gettime(CLOCK_REALTIME, &dl);
    const double lim = s->limit_s;
    dl.tv_sec += (time_t) lim;
    dl.tv_nsec += (long) ((lim - (double) (time_t) lim) * 1e9);
    if (dl.tv_nsec >= 1000000000L) { dl.tv_sec++; dl.tv_nsec -= 1000000000L; }
    int rc = 0;
    while (s->phase == ph && !s->broken) {
        if (pthread_cond_timedwait(&s->cv, &s->mu, &dl) == ETIMEDOUT && s->phase == ph) {
            s->broken = 1;
            pthread_cond_broadcast(&s->cv);
            ERROR_PRINTF("thread transport: a rank did not arrive within %.0f s\n", lim);
            break;
        }
    }
    if (s->phase == ph) rc = 1;
    pthread_mutex_unlock(&s->mu);
    return rc;
}

typedef struct {
    thr_shared_t *sh;
    int rank;
} thr_rank_t;

static int thr_allgather(void *ctx, const long long *mine, int n, long long *all)
{
    thr_rank_t *t = (thr_rank_t *) ctx;
    thr_shared_t *s = t->sh;
    s->ptr[t->rank] = mine;
    if (thr_barrier(s)) return 1;
    for (int r = 0; r < s->size; r++)
        memcpy(all + (size_t) r * n, s->ptr[r], sizeof(long long) * (size_t) n);
    return thr_barrier(s);           /* no rank leaves while a peer still reads its values */
}

static int thr_alltoallv(void *ctx, const double *send, const long long *scounts,
                         const long long *sdispls, double *recv, const long long *rcounts,
                         const long long *rdispls, void *stream)
{
    (void) stream;
    thr_rank_t *t = (thr_rank_t *) ctx;
    thr_shared_t *s = t->sh;
    const int me = t->rank;
    s->ptr[me] = send;
    s->cnt[me] = scounts;
    s->dsp[me] = sdispls;
    if (thr_barrier(s)) return 1;
    int bad = 0;
    for (int q = 0; q < s->size; q++) {
        const long long c = s->cnt[q][me];
        if (c != rcounts[q]) {
            bad = 1;
            continue;
        }
        if (c > 0)
            memcpy(recv + rdispls[q], (const double *) s->ptr[q] + s->dsp[q][me],
                   sizeof(double) * (size_t) c);
    }
    if (thr_barrier(s)) return 1;
    return bad;
}

int ca3dmm_transport_threads_create(int size, ca3dmm_transport_t *per_rank)
{
    if (size < 1 || !per_rank) return CA3DMM_EINVAL;
    thr_shared_t *s = (thr_shared_t *) calloc(1, sizeof(thr_shared_t));
    thr_rank_t *ranks = (thr_rank_t *) calloc((size_t) size, sizeof(thr_rank_t));
    if (!s || !ranks) { free(s); free(ranks); return CA3DMM_ENOMEM; }
    s->size = size;
    s->ptr = (const void **) calloc((size_t) size, sizeof(void *));
    s->cnt = (const long long **) calloc((size_t) size, sizeof(void *));
    s->dsp = (const long long **) calloc((size_t) size, sizeof(void *));
    if (!s->ptr || !s->cnt || !s->dsp) {
        free(s->ptr); free(s->cnt); free(s->dsp); free(s); free(ranks);
        return CA3DMM_ENOMEM;
    }
    pthread_mutex_init(&s->mu, NULL);
    pthread_cond_init(&s->cv, NULL);
    int lim;
    GET_ENV_INT_VAR(lim, "CA3DMM_DIST_TIMEOUT", "dist_timeout", 300, 1, 1 << 20);
    s->limit_s = (double) lim;
    for (int r = 0; r < size; r++) {
        ranks[r].sh = s;
        ranks[r].rank = r;
        per_rank[r].rank = r;
        per_rank[r].size = size;
        per_rank[r].device_buffers = 0;
        per_rank[r].ctx = &ranks[r];
        per_rank[r].allgather_ll = thr_allgather;
        per_rank[r].alltoallv_d = thr_alltoallv;
    }
    return CA3DMM_OK;
}

void ca3dmm_transport_threads_free(ca3dmm_transport_t *per_rank)
{
    if (!per_rank || !per_rank[0].ctx) return;
    thr_rank_t *ranks = (thr_rank_t *) per_rank[0].ctx;
    thr_shared_t *s = ranks[0].sh;
    const int size = s->size;
    pthread_mutex_destroy(&s->mu);
    pthread_cond_destroy(&s->cv);
    free(s->ptr); free(s->cnt); free(s->dsp); free(s);
    free(ranks);
    for (int r = 0; r < size; r++) per_rank[r].ctx = NULL;
}

/* ------------------------------------------------------------------ NCCL */

typedef struct {
    void *so;
    ncclResult_t (*get_id)(ncclUniqueId *);
    ncclResult_t (*init_rank)(ncclComm_t *, int, ncclUniqueId, int);
    ncclResult_t (*destroy)(ncclComm_t);
    ncclResult_t (*group_start)(void);
    ncclResult_t (*group_end)(void);
    ncclResult_t (*send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
    ncclResult_t (*recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
    ncclResult_t (*allgather)(const void *, void *, size_t, ncclDataType_t, ncclComm_t,
                              cudaStream_t);
    const char *(*errstr)(ncclResult_t);
} nccl_api_t;

static nccl_api_t g_nccl;
static pthread_once_t g_nccl_once = PTHREAD_ONCE_INIT;

static void nccl_load(void)
{
    void *so = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!so) return;
#define LOAD(f, name) *(void **) (&g_nccl.f) = dlsym(so, name)
    LOAD(get_id, "ncclGetUniqueId");
    LOAD(init_rank, "ncclCommInitRank");
    LOAD(destroy, "ncclCommDestroy");
    LOAD(group_start, "ncclGroupStart");
    LOAD(group_end, "ncclGroupEnd");
    LOAD(send, "ncclSend");
    LOAD(recv, "ncclRecv");
    LOAD(allgather, "ncclAllGather");
    LOAD(errstr, "ncclGetErrorString");
#undef LOAD
    if (g_nccl.get_id && g_nccl.init_rank && g_nccl.destroy && g_nccl.group_start &&
        g_nccl.group_end && g_nccl.send && g_nccl.recv && g_nccl.allgather && g_nccl.errstr)
        g_nccl.so = so;
}

static int nccl_ok(void)
{
    pthread_once(&g_nccl_once, nccl_load);
    if (!g_nccl.so) ERROR_PRINTF("libnccl.so.2 could not be loaded\n");
    return g_nccl.so != NULL;
}

#define NCCL_TRY(call)                                                                      \
    do {                                                                                    \
        ncclResult_t r_ = (call);                                                           \
        if (r_ != ncclSuccess) {                                                            \
            ERROR_PRINTF("%s failed: %s\n", #call, g_nccl.errstr(r_));                      \
            return CA3DMM_ECUDA;                                                            \
        }                                                                                   \
    } while (0)

typedef struct {
    ncclComm_t comm;
    int rank, size;
    cudaStream_t stream;
} nccl_ctx_t;

int ca3dmm_nccl_unique_id(unsigned char id[128])
{
    if (!id || !nccl_ok()) return CA3DMM_EINVAL;
    ncclUniqueId u;
    NCCL_TRY(g_nccl.get_id(&u));
    memcpy(id, &u, sizeof(u) < 128 ? sizeof(u) : 128);
    return CA3DMM_OK;
}

static int nccl_allgather(void *ctx, const long long *mine, int n, long long *all)
{
    nccl_ctx_t *c = (nccl_ctx_t *) ctx;
    long long *d = NULL;
    const size_t b = sizeof(long long) * (size_t) n;
    CA3DMM_CUDA_TRY(cudaMalloc((void **) &d, b * (size_t) (c->size + 1)));
    int rc = CA3DMM_OK;
    if (cudaMemcpy(d, mine, b, cudaMemcpyHostToDevice) != cudaSuccess) rc = CA3DMM_ECUDA;
    if (!rc && g_nccl.allgather(d, d + n, (size_t) n, ncclInt64, c->comm, c->stream) != ncclSuccess)
        rc = CA3DMM_ECUDA;
    if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = CA3DMM_ECUDA;
    if (!rc && cudaMemcpy(all, d + n, b * (size_t) c->size, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = CA3DMM_ECUDA;
    cudaFree(d);
    return rc;
}

static int nccl_alltoallv(void *ctx, const double *send, const long long *scounts,
                          const long long *sdispls, double *recv, const long long *rcounts,
                          const long long *rdispls, void *stream)
{
    nccl_ctx_t *c = (nccl_ctx_t *) ctx;
    cudaStream_t st = stream ? (cudaStream_t) stream : c->stream;
    NCCL_TRY(g_nccl.group_start());
    for (int q = 0; q < c->size; q++) {
        if (scounts[q] > 0)
            NCCL_TRY(g_nccl.send(send + sdispls[q], (size_t) scounts[q], ncclFloat64, q, c->comm, st));
        if (rcounts[q] > 0)
            NCCL_TRY(g_nccl.recv(recv + rdispls[q], (size_t) rcounts[q], ncclFloat64, q, c->comm, st));
    }
    NCCL_TRY(g_nccl.group_end());
    CA3DMM_CUDA_TRY(cudaStreamSynchronize(st));
    return CA3DMM_OK;
}

int ca3dmm_transport_nccl_create(int size, int rank, const unsigned char id[128],
                                 ca3dmm_transport_t *t)
{
    if (!t || !id || size < 1 || rank < 0 || rank >= size || !nccl_ok()) return CA3DMM_EINVAL;
    nccl_ctx_t *c = (nccl_ctx_t *) calloc(1, sizeof(nccl_ctx_t));
    if (!c) return CA3DMM_ENOMEM;
    ncclUniqueId u;
    memcpy(&u, id, sizeof(u) < 128 ? sizeof(u) : 128);
    c->rank = rank;
    c->size = size;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        free(c);
        return CA3DMM_ECUDA;
    }
    if (g_nccl.init_rank(&c->comm, size, u, rank) != ncclSuccess) {
        cudaStreamDestroy(c->stream);
        free(c);
        return CA3DMM_ECUDA;
    }
    t->rank = rank;
    t->size = size;
    t->device_buffers = 1;
    t->ctx = c;
    t->allgather_ll = nccl_allgather;
    t->alltoallv_d = nccl_alltoallv;
    return CA3DMM_OK;
}

void ca3dmm_transport_nccl_free(ca3dmm_transport_t *t)
{
    if (!t || !t->ctx) return;
    nccl_ctx_t *c = (nccl_ctx_t *) t->ctx;
    if (g_nccl.so) g_nccl.destroy(c->comm);
    cudaStreamDestroy(c->stream);
    free(c);
    t->ctx = NULL;
}
