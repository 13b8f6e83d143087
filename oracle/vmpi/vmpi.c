/* vmpi: thread-backed MPI subset (see mpi.h).  TEST INFRASTRUCTURE ONLY.
 *
 * Every rank is a host thread.  Collectives meet on a per-communicator
 * barrier (mutex + condition variable with a timeout, so a rank that never
 * arrives makes the others return an error instead of hanging) and exchange
 * buffer pointers through per-member slots; point-to-point messages are
 * copied eagerly into the destination rank's mailbox. */
#define _GNU_SOURCE
#include <errno.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include "mpi.h"

#define TAG_NEIGHBOR 0x7ffffff0

struct vmpi_op {
    MPI_User_function *fn;   /* NULL: built-in sum */
};

struct vmpi_comm {
    int size, id;
    int *world;              /* member -> world rank */
    int *rank_of;            /* world rank -> member (or -1) */
    pthread_mutex_t mu;
    pthread_cond_t cv;
    int arrived;
    long long gen;
    /* collective slots, one per member */
    const void **ptr;
    const int **iptr;
    int *ival, *ival2;
    MPI_Comm *newc;
    /* topology */
    int dims[2];
    int *indeg, *outdeg, **src, **dst;
    int refs;
};

typedef struct msg {
    int comm_id, src, tag;
    size_t bytes;
    struct msg *next;
    char data[];
} msg_t;

typedef struct {
    pthread_mutex_t mu;
    pthread_cond_t cv;
    msg_t *head, *tail;
} mailbox_t;

struct vmpi_request {
    int is_recv;
    void *buf;
    size_t bytes;
    MPI_Comm comm;
    int src, tag;
};

static struct vmpi_op op_sum = {NULL};
MPI_Op vmpi_op_sum = &op_sum;
__thread MPI_Comm vmpi_world = NULL;
static __thread int my_world = -1;

static int world_size = 0;
static mailbox_t *mailboxes = NULL;
static double timeout_s = 60.0;
static volatile int failed = 0;
static int next_id = 1;
static pthread_mutex_t id_mu = PTHREAD_MUTEX_INITIALIZER;

static size_t dsize(MPI_Datatype t) { return t == MPI_DOUBLE ? 8 : 4; }

static void deadline(struct timespec *ts)
{
    clock_gettime(CLOCK_REALTIME, ts);
    long long ns = (long long) (timeout_s * 1e9);
    ts->tv_sec += ns / 1000000000LL;
    ts->tv_nsec += ns % 1000000000LL;
    if (ts->tv_nsec >= 1000000000L) { ts->tv_sec++; ts->tv_nsec -= 1000000000L; }
}

static MPI_Comm comm_new(int size, const int *world)
{
    MPI_Comm c = (MPI_Comm) calloc(1, sizeof(*c));
    c->size = size;
    pthread_mutex_lock(&id_mu);
    c->id = next_id++;
    pthread_mutex_unlock(&id_mu);
    c->world = (int *) malloc(sizeof(int) * size);
    memcpy(c->world, world, sizeof(int) * size);
    c->rank_of = (int *) malloc(sizeof(int) * world_size);
    for (int i = 0; i < world_size; i++) c->rank_of[i] = -1;
    for (int i = 0; i < size; i++) c->rank_of[world[i]] = i;
    pthread_mutex_init(&c->mu, NULL);
    pthread_cond_init(&c->cv, NULL);
    c->ptr = calloc(size, sizeof(void *));
    c->iptr = calloc(size, sizeof(int *));
    c->ival = calloc(size, sizeof(int));
    c->ival2 = calloc(size, sizeof(int));
    c->newc = calloc(size, sizeof(MPI_Comm));
    c->indeg = calloc(size, sizeof(int));
    c->outdeg = calloc(size, sizeof(int));
    c->src = calloc(size, sizeof(int *));
    c->dst = calloc(size, sizeof(int *));
    c->refs = size;
    return c;
}

static void comm_destroy(MPI_Comm c)
{
    for (int i = 0; i < c->size; i++) { free(c->src[i]); free(c->dst[i]); }
    free(c->world); free(c->rank_of); free(c->ptr); free(c->iptr); free(c->ival);
    free(c->ival2); free(c->newc); free(c->indeg); free(c->outdeg); free(c->src); free(c->dst);
    pthread_mutex_destroy(&c->mu);
    pthread_cond_destroy(&c->cv);
    free(c);
}

static int me(MPI_Comm c) { return c->rank_of[my_world]; }

/* barrier with timeout; a timeout marks the run failed */
static int barrier(MPI_Comm c)
{
    int rc = 0;
    pthread_mutex_lock(&c->mu);
    long long g = c->gen;
    if (++c->arrived == c->size) {
        c->arrived = 0;
        c->gen++;
        pthread_cond_broadcast(&c->cv);
    } else {
        struct timespec ts;
        deadline(&ts);
        while (c->gen == g) {
            if (pthread_cond_timedwait(&c->cv, &c->mu, &ts) == ETIMEDOUT) {
                /* a peer never arrived: like MPI's default fatal error
                 * handler, this rank stops (the run reports the failure) */
                failed = 1;
                c->arrived--;
                pthread_mutex_unlock(&c->mu);
                pthread_exit(NULL);
            }
        }
    }
    pthread_mutex_unlock(&c->mu);
    return rc;
}

int MPI_Init(int *argc, char ***argv) { (void) argc; (void) argv; return 0; }
int MPI_Finalize(void) { return 0; }

double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + ts.tv_nsec * 1e-9;
}

int MPI_Comm_rank(MPI_Comm c, int *r) { *r = me(c); return 0; }
int MPI_Comm_size(MPI_Comm c, int *s) { *s = c->size; return 0; }

int MPI_Comm_split(MPI_Comm c, int color, int key, MPI_Comm *out)
{
    const int r = me(c), n = c->size;
    c->ival[r] = color;
    c->ival2[r] = key;
    int rc = barrier(c);
    /* members of my colour ordered by (key, old rank) */
    int *mem = (int *) malloc(sizeof(int) * n), cnt = 0;
    for (int i = 0; i < n; i++)
        if (c->ival[i] == color) mem[cnt++] = i;
    for (int a = 1; a < cnt; a++) {
        int v = mem[a], b = a - 1;
        while (b >= 0 && (c->ival2[mem[b]] > c->ival2[v] ||
                          (c->ival2[mem[b]] == c->ival2[v] && mem[b] > v))) {
            mem[b + 1] = mem[b];
            b--;
        }
        mem[b + 1] = v;
    }
    if (mem[0] == r) {
        int *w = (int *) malloc(sizeof(int) * cnt);
        for (int i = 0; i < cnt; i++) w[i] = c->world[mem[i]];
        c->newc[r] = comm_new(cnt, w);
        free(w);
    }
    rc |= barrier(c);
    *out = c->newc[mem[0]];
    free(mem);
    rc |= barrier(c);
    return rc;
}

static int dup_comm(MPI_Comm c, MPI_Comm *out)
{
    const int r = me(c);
    int rc = barrier(c);
    if (r == 0) c->newc[0] = comm_new(c->size, c->world);
    rc |= barrier(c);
    *out = c->newc[0];
    rc |= barrier(c);
    return rc;
}

int MPI_Cart_create(MPI_Comm c, int ndims, const int *dims, const int *periods, int reorder,
                    MPI_Comm *cart)
{
    (void) periods; (void) reorder;
    int rc = dup_comm(c, cart);
    if (me(c) == 0) {
        (*cart)->dims[0] = dims[0];
        (*cart)->dims[1] = ndims > 1 ? dims[1] : 1;
    }
    rc |= barrier(c);
    return rc;
}

int MPI_Cart_coords(MPI_Comm c, int rank, int maxdims, int *coords)
{
    (void) maxdims;
    coords[0] = rank / c->dims[1];
    coords[1] = rank % c->dims[1];
    return 0;
}

int MPI_Dist_graph_create_adjacent(MPI_Comm c, int indeg, const int *sources, const int *sw,
                                   int outdeg, const int *dests, const int *dw, MPI_Info info,
                                   int reorder, MPI_Comm *graph)
{
    (void) sw; (void) dw; (void) info; (void) reorder;
    int rc = dup_comm(c, graph);
    MPI_Comm g = *graph;
    const int r = me(c);
    g->indeg[r] = indeg;
    g->outdeg[r] = outdeg;
    g->src[r] = (int *) malloc(sizeof(int) * (indeg > 0 ? indeg : 1));
    g->dst[r] = (int *) malloc(sizeof(int) * (outdeg > 0 ? outdeg : 1));
    memcpy(g->src[r], sources, sizeof(int) * indeg);
    memcpy(g->dst[r], dests, sizeof(int) * outdeg);
    rc |= barrier(c);
    return rc;
}

int MPI_Comm_free(MPI_Comm *c)
{
    if (!c || !*c) return 0;
    MPI_Comm x = *c;
    pthread_mutex_lock(&x->mu);
    int left = --x->refs;
    pthread_mutex_unlock(&x->mu);
    if (left == 0) comm_destroy(x);
    *c = NULL;
    return 0;
}

int MPI_Barrier(MPI_Comm c) { return barrier(c); }

int MPI_Allgatherv(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf,
                   const int *rcounts, const int *displs, MPI_Datatype rtype, MPI_Comm c)
{
    (void) scount; (void) stype;
    const int r = me(c);
    c->ptr[r] = sendbuf;
    int rc = barrier(c);
    const size_t es = dsize(rtype);
    for (int i = 0; i < c->size; i++)
        memcpy((char *) recvbuf + es * displs[i], c->ptr[i], es * rcounts[i]);
    rc |= barrier(c);
    return rc;
}

int MPI_Allgather(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf, int rcount,
                  MPI_Datatype rtype, MPI_Comm c)
{
    int *cnt = (int *) malloc(sizeof(int) * c->size), *dsp = (int *) malloc(sizeof(int) * c->size);
    for (int i = 0; i < c->size; i++) { cnt[i] = rcount; dsp[i] = i * rcount; }
    int rc = MPI_Allgatherv(sendbuf, scount, stype, recvbuf, cnt, dsp, rtype, c);
    free(cnt); free(dsp);
    return rc;
}

static void apply(MPI_Op op, const void *in, void *inout, int n, MPI_Datatype t)
{
    if (op && op->fn) { op->fn((void *) in, inout, &n, &t); return; }
    if (t == MPI_DOUBLE) for (int i = 0; i < n; i++) ((double *) inout)[i] += ((const double *) in)[i];
    else if (t == MPI_FLOAT) for (int i = 0; i < n; i++) ((float *) inout)[i] += ((const float *) in)[i];
    else for (int i = 0; i < n; i++) ((int *) inout)[i] += ((const int *) in)[i];
}

/* member r's result over [off, off + cnt): in_0 (+) in_1 (+) ... in rank order */
static void reduce_range(MPI_Comm c, MPI_Op op, MPI_Datatype t, size_t off, int cnt, void *tmp)
{
    const size_t es = dsize(t);
    memcpy(tmp, (const char *) c->ptr[0] + es * off, es * cnt);
    for (int i = 1; i < c->size; i++) apply(op, (const char *) c->ptr[i] + es * off, tmp, cnt, t);
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype t, MPI_Op op,
                  MPI_Comm c)
{
    const int r = me(c);
    c->ptr[r] = sendbuf == MPI_IN_PLACE ? recvbuf : sendbuf;
    int rc = barrier(c);
    void *tmp = malloc(dsize(t) * (count > 0 ? count : 1));
    reduce_range(c, op, t, 0, count, tmp);
    rc |= barrier(c);
    memcpy(recvbuf, tmp, dsize(t) * count);
    free(tmp);
    rc |= barrier(c);
    return rc;
}

int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype t, MPI_Op op, int root,
               MPI_Comm c)
{
    const int r = me(c);
    c->ptr[r] = sendbuf;
    int rc = barrier(c);
    if (r == root) reduce_range(c, op, t, 0, count, recvbuf);
    rc |= barrier(c);
    return rc;
}

int MPI_Reduce_scatter(const void *sendbuf, void *recvbuf, const int *rcounts, MPI_Datatype t,
                       MPI_Op op, MPI_Comm c)
{
    const int r = me(c);
    c->ptr[r] = sendbuf;
    int rc = barrier(c);
    size_t off = 0;
    for (int i = 0; i < r; i++) off += rcounts[i];
    void *tmp = malloc(dsize(t) * (rcounts[r] > 0 ? rcounts[r] : 1));
    reduce_range(c, op, t, off, rcounts[r], tmp);
    rc |= barrier(c);
    memcpy(recvbuf, tmp, dsize(t) * rcounts[r]);
    free(tmp);
    return rc;
}

int MPI_Reduce_scatter_block(const void *sendbuf, void *recvbuf, int rcount, MPI_Datatype t,
                             MPI_Op op, MPI_Comm c)
{
    int *cnt = (int *) malloc(sizeof(int) * c->size);
    for (int i = 0; i < c->size; i++) cnt[i] = rcount;
    int rc = MPI_Reduce_scatter(sendbuf, recvbuf, cnt, t, op, c);
    free(cnt);
    return rc;
}

static void post(MPI_Comm c, int dst, int tag, const void *buf, size_t bytes)
{
    msg_t *m = (msg_t *) malloc(sizeof(msg_t) + bytes);
    m->comm_id = c->id;
    m->src = me(c);
    m->tag = tag;
    m->bytes = bytes;
    m->next = NULL;
    memcpy(m->data, buf, bytes);
    mailbox_t *mb = &mailboxes[c->world[dst]];
    pthread_mutex_lock(&mb->mu);
    if (mb->tail) mb->tail->next = m; else mb->head = m;
    mb->tail = m;
    pthread_cond_broadcast(&mb->cv);
    pthread_mutex_unlock(&mb->mu);
}

static int take(MPI_Comm c, int src, int tag, void *buf, size_t maxbytes)
{
    mailbox_t *mb = &mailboxes[my_world];
    struct timespec ts;
    deadline(&ts);
    pthread_mutex_lock(&mb->mu);
    for (;;) {
        msg_t *prev = NULL;
        for (msg_t *m = mb->head; m; prev = m, m = m->next) {
            if (m->comm_id == c->id && m->src == src && m->tag == tag) {
                if (prev) prev->next = m->next; else mb->head = m->next;
                if (mb->tail == m) mb->tail = prev;
                pthread_mutex_unlock(&mb->mu);
                memcpy(buf, m->data, m->bytes < maxbytes ? m->bytes : maxbytes);
                free(m);
                return 0;
            }
        }
        if (pthread_cond_timedwait(&mb->cv, &mb->mu, &ts) == ETIMEDOUT) {
            failed = 1;
            pthread_mutex_unlock(&mb->mu);
            pthread_exit(NULL);
        }
    }
}

int MPI_Isend(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c,
              MPI_Request *req)
{
    post(c, dest, tag, buf, dsize(t) * count);
    *req = NULL;   /* eager: already complete */
    return 0;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm c,
              MPI_Request *req)
{
    struct vmpi_request *q = (struct vmpi_request *) malloc(sizeof(*q));
    q->is_recv = 1; q->buf = buf; q->bytes = dsize(t) * count; q->comm = c;
    q->src = source; q->tag = tag;
    *req = q;
    return 0;
}

int MPI_Wait(MPI_Request *req, MPI_Status *status)
{
    (void) status;
    if (!req || !*req) return 0;
    struct vmpi_request *q = *req;
    int rc = take(q->comm, q->src, q->tag, q->buf, q->bytes);
    free(q);
    *req = NULL;
    return rc;
}

int MPI_Sendrecv(const void *sendbuf, int scount, MPI_Datatype stype, int dest, int stag,
                 void *recvbuf, int rcount, MPI_Datatype rtype, int source, int rtag, MPI_Comm c,
                 MPI_Status *status)
{
    (void) status;
    post(c, dest, stag, sendbuf, dsize(stype) * scount);
    return take(c, source, rtag, recvbuf, dsize(rtype) * rcount);
}

int MPI_Neighbor_alltoallv(const void *sendbuf, const int *scounts, const int *sdispls,
                           MPI_Datatype stype, void *recvbuf, const int *rcounts,
                           const int *rdispls, MPI_Datatype rtype, MPI_Comm c)
{
    const int r = me(c);
    const size_t se = dsize(stype), re = dsize(rtype);
    for (int j = 0; j < c->outdeg[r]; j++)
        post(c, c->dst[r][j], TAG_NEIGHBOR, (const char *) sendbuf + se * sdispls[j],
             se * scounts[j]);
    int rc = 0;
    for (int i = 0; i < c->indeg[r]; i++)
        rc |= take(c, c->src[r][i], TAG_NEIGHBOR, (char *) recvbuf + re * rdispls[i],
                   re * rcounts[i]);
    return rc;
}

int MPI_Op_create(MPI_User_function *fn, int commute, MPI_Op *op)
{
    (void) commute;
    struct vmpi_op *o = (struct vmpi_op *) malloc(sizeof(*o));
    o->fn = fn;
    *op = o;
    return 0;
}

typedef struct {
    int rank;
    void (*fn)(int, void *);
    void *arg;
    MPI_Comm world;
} start_t;

static void *thread_main(void *p)
{
    start_t *s = (start_t *) p;
    my_world = s->rank;
    vmpi_world = s->world;
    s->fn(s->rank, s->arg);
    return NULL;
}

int vmpi_run(int p, void (*fn)(int rank, void *arg), void *arg, double timeout)
{
    if (p < 1) return 1;
    world_size = p;
    timeout_s = timeout > 0 ? timeout : 60.0;
    failed = 0;
    mailboxes = (mailbox_t *) calloc(p, sizeof(mailbox_t));
    for (int i = 0; i < p; i++) {
        pthread_mutex_init(&mailboxes[i].mu, NULL);
        pthread_cond_init(&mailboxes[i].cv, NULL);
    }
    int *w = (int *) malloc(sizeof(int) * p);
    for (int i = 0; i < p; i++) w[i] = i;
    MPI_Comm world = comm_new(p, w);
    free(w);
    pthread_t *th = (pthread_t *) malloc(sizeof(pthread_t) * p);
    start_t *st = (start_t *) malloc(sizeof(start_t) * p);
    pthread_attr_t attr;
    pthread_attr_init(&attr);
    pthread_attr_setstacksize(&attr, 64 << 20);
    for (int i = 0; i < p; i++) {
        st[i].rank = i; st[i].fn = fn; st[i].arg = arg; st[i].world = world;
        pthread_create(&th[i], &attr, thread_main, &st[i]);
    }
    for (int i = 0; i < p; i++) pthread_join(th[i], NULL);
    pthread_attr_destroy(&attr);
    for (int i = 0; i < p; i++) {
        msg_t *m = mailboxes[i].head;
        while (m) { msg_t *n = m->next; free(m); m = n; }
    }
    free(mailboxes);
    mailboxes = NULL;
    free(th); free(st);
    comm_destroy(world);
    return failed;
}
