/*
 * mpi_shim.c — a small shared-memory MPI for running the muMatScale
 * reference sources as N processes on one host.  Test infrastructure only
 * (the oracle and the timed CPU baseline); nothing in the product links it.
 *
 * Process model: MPI_Init forks MMSREF_NP-1 children (default 1 rank, no
 * fork).  All ranks share one anonymous MAP_SHARED region holding a
 * process-shared mutex/condvar/barrier, a message table and a first-fit
 * arena.  Sends copy into the arena and complete immediately; receives match
 * (source, tag) in send order.  Collectives publish per-rank arena blocks
 * between two barriers.  Reductions combine in rank order so results are
 * reproducible run to run.
 */
#define _GNU_SOURCE
#include "mpi.h"

#include <errno.h>
#include <pthread.h>
#include <signal.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/wait.h>
#include <time.h>
#include <unistd.h>

#define MAXNP 256
#define MAXMSG 8192
#define MAXTYPES 256

typedef struct {
    int used;
    int src, dst, tag;
    long seq;
    size_t off, len;
} shm_msg;

typedef struct {
    size_t size;   /* bytes of payload after the header */
    int free;
    int pad;
} arena_blk;

typedef struct {
    pthread_mutex_t mu;
    pthread_cond_t cv;
    long bar_count;
    long bar_gen;
    int np;
    int abort_flag;
    long seq;
    size_t arena_size;
    shm_msg msgs[MAXMSG];
    size_t coll_off[MAXNP];
    size_t coll_len[MAXNP];
} shm_hdr;

static shm_hdr *g_shm = NULL;
static char *g_arena = NULL;
static int g_rank = 0;
static int g_np = 1;
static pid_t g_children[MAXNP];
static int g_reaped[MAXNP];      /* rank 0: child already collected by waitpid */
static int g_child_status[MAXNP];
static int g_cart_dims[8];
static int g_cart_ndims = 0;

struct mmsref_req {
    int is_recv;
    void *buf;
    size_t maxlen;
    int src, tag;
};

/* ---- datatypes ---------------------------------------------------------- */
static size_t g_type_extent[MAXTYPES] = {0, 1, 4, 8, 8, 8, 8, 4, 4, 8};
static int g_ntypes = 10;

static size_t type_extent(MPI_Datatype t)
{
    if (t <= 0 || t >= g_ntypes) {
        fprintf(stderr, "mpi_shim: bad datatype %d\n", t);
        abort();
    }
    return g_type_extent[t];
}

int MPI_Type_create_struct(int count, const int blocklens[], const MPI_Aint disps[],
                           const MPI_Datatype types[], MPI_Datatype *newtype)
{
    size_t ext = 0;
    for (int i = 0; i < count; i++) {
        size_t end = (size_t)disps[i] + (size_t)blocklens[i] * type_extent(types[i]);
        if (end > ext) ext = end;
    }
    if (g_ntypes >= MAXTYPES) abort();
    g_type_extent[g_ntypes] = ext;
    *newtype = g_ntypes++;
    return MPI_SUCCESS;
}

int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *newtype)
{
    if (g_ntypes >= MAXTYPES) abort();
    g_type_extent[g_ntypes] = (size_t)count * type_extent(old);
    *newtype = g_ntypes++;
    return MPI_SUCCESS;
}

int MPI_Type_commit(MPI_Datatype *type) { (void)type; return MPI_SUCCESS; }
int MPI_Type_free(MPI_Datatype *type) { *type = MPI_DATATYPE_NULL; return MPI_SUCCESS; }
int MPI_Type_size(MPI_Datatype type, int *size) { *size = (int)type_extent(type); return MPI_SUCCESS; }

/* ---- arena (caller holds the mutex) ------------------------------------- */
static arena_blk *blk_at(size_t off) { return (arena_blk *)(g_arena + off); }

static size_t arena_alloc(size_t len)
{
    size_t need = (len + 63) & ~(size_t)63;
    size_t off = 0;
    while (off < g_shm->arena_size) {
        arena_blk *b = blk_at(off);
        if (b->free) {
            /* coalesce following free blocks */
            size_t nxt = off + sizeof(arena_blk) + b->size;
            while (nxt < g_shm->arena_size && blk_at(nxt)->free) {
                b->size += sizeof(arena_blk) + blk_at(nxt)->size;
                nxt = off + sizeof(arena_blk) + b->size;
            }
            if (b->size >= need) {
                if (b->size >= need + sizeof(arena_blk) + 64) {
                    size_t rest = b->size - need - sizeof(arena_blk);
                    b->size = need;
                    arena_blk *r = blk_at(off + sizeof(arena_blk) + need);
                    r->size = rest;
                    r->free = 1;
                }
                b->free = 0;
                return off + sizeof(arena_blk);
            }
        }
        off += sizeof(arena_blk) + b->size;
    }
    fprintf(stderr, "mpi_shim: arena exhausted (%zu bytes requested)\n", len);
    abort();
}

static void arena_free(size_t payload_off)
{
    blk_at(payload_off - sizeof(arena_blk))->free = 1;
}

static void lock(void) { pthread_mutex_lock(&g_shm->mu); }
static void unlock(void) { pthread_mutex_unlock(&g_shm->mu); }
static pid_t g_parent = 0;

/* Rank 0: collects children that have ended; returns 1 if one of them
 * ended abnormally (killed by a signal, or a non-zero exit). */
static int child_failed(void)
{
    int bad = 0;
    for (int r = 1; r < g_np; r++) {
        if (g_reaped[r]) continue;
        int st = 0;
        if (waitpid(g_children[r], &st, WNOHANG) == g_children[r]) {
            g_reaped[r] = 1;
            g_child_status[r] = st;
            if (!WIFEXITED(st) || WEXITSTATUS(st) != 0) bad = 1;
        }
    }
    return bad;
}

/* Waits on the shared condition variable for at most one second, then
 * returns.  A rank that sees the abort flag, or (as a child) finds rank 0
 * gone, exits instead of waiting forever; rank 0 raises the abort flag and
 * exits when a child rank has died (it would never reach the call being
 * waited for).  Caller holds the mutex. */
static void wait_or_die(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_REALTIME, &ts);
    ts.tv_sec += 1;
    pthread_cond_timedwait(&g_shm->cv, &g_shm->mu, &ts);
    if (g_rank == 0 && !g_shm->abort_flag && child_failed()) {
        g_shm->abort_flag = 1;
        pthread_cond_broadcast(&g_shm->cv);
        pthread_mutex_unlock(&g_shm->mu);
        fprintf(stderr, "mpi_shim: a rank died; ending the run\n");
        _exit(1);
    }
    if (g_shm->abort_flag || (g_rank != 0 && getppid() != g_parent)) {
        pthread_mutex_unlock(&g_shm->mu);
        _exit(1);
    }
}

/* ---- init / finalize ---------------------------------------------------- */
static void shm_setup(int np)
{
    size_t arena = (size_t)1 << 31;
    const char *a = getenv("MMSREF_ARENA_MB");
    if (a) arena = (size_t)atol(a) << 20;
    size_t total = sizeof(shm_hdr) + arena;
    void *p = mmap(NULL, total, PROT_READ | PROT_WRITE,
                   MAP_SHARED | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
    if (p == MAP_FAILED) {
        perror("mpi_shim: mmap");
        abort();
    }
    g_shm = (shm_hdr *)p;
    g_arena = (char *)p + sizeof(shm_hdr);
    memset(g_shm, 0, sizeof(shm_hdr));
    g_shm->np = np;
    g_shm->arena_size = arena;
    arena_blk *b = blk_at(0);
    b->size = arena - sizeof(arena_blk);
    b->free = 1;

    pthread_mutexattr_t ma;
    pthread_mutexattr_init(&ma);
    pthread_mutexattr_setpshared(&ma, PTHREAD_PROCESS_SHARED);
    pthread_mutex_init(&g_shm->mu, &ma);
    pthread_condattr_t ca;
    pthread_condattr_init(&ca);
    pthread_condattr_setpshared(&ca, PTHREAD_PROCESS_SHARED);
    pthread_cond_init(&g_shm->cv, &ca);
}

int MPI_Init_thread(int *argc, char ***argv, int required, int *provided)
{
    (void)argc; (void)argv;
    if (provided) *provided = required;
    const char *e = getenv("MMSREF_NP");
    int np = e ? atoi(e) : 1;
    if (np < 1 || np > MAXNP) np = 1;
    g_np = np;
    shm_setup(np);
    fflush(stdout);
    fflush(stderr);
    g_parent = getpid();
    for (int r = 1; r < np; r++) {
        pid_t pid = fork();
        if (pid < 0) {
            perror("mpi_shim: fork");
            abort();
        }
        if (pid == 0) {
            g_rank = r;
            return MPI_SUCCESS;
        }
        g_children[r] = pid;
    }
    g_rank = 0;
    return MPI_SUCCESS;
}

int MPI_Init(int *argc, char ***argv)
{
    int prov;
    return MPI_Init_thread(argc, argv, MPI_THREAD_SINGLE, &prov);
}

int MPI_Finalize(void)
{
    fflush(stdout);
    fflush(stderr);
    MPI_Barrier(MPI_COMM_WORLD);
    if (g_shm && g_shm->abort_flag) _exit(1);
    if (g_rank == 0) {
        int bad = 0;
        for (int r = 1; r < g_np; r++) {
            int st = g_child_status[r];
            if (!g_reaped[r]) waitpid(g_children[r], &st, 0);
            if (!WIFEXITED(st) || WEXITSTATUS(st) != 0) bad = 1;
        }
        if (bad) fprintf(stderr, "mpi_shim: a child rank exited abnormally\n");
    }
    return MPI_SUCCESS;
}

int MPI_Abort(MPI_Comm comm, int code)
{
    (void)comm;
    fflush(stdout);
    fflush(stderr);
    if (g_shm) {
        /* every rank polls this flag in its waits and exits */
        g_shm->abort_flag = 1;
        pthread_cond_broadcast(&g_shm->cv);
    }
    if (g_rank == 0) {
        for (int r = 1; r < g_np; r++) {
            int st;
            if (!g_reaped[r]) waitpid(g_children[r], &st, 0);
        }
    }
    _exit(code ? code : 1);
}

int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = g_np; return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = g_rank; return MPI_SUCCESS; }

int MPI_Barrier(MPI_Comm comm)
{
    (void)comm;
    if (g_np == 1) return MPI_SUCCESS;
    lock();
    long gen = g_shm->bar_gen;
    if (++g_shm->bar_count == g_np) {
        g_shm->bar_count = 0;
        g_shm->bar_gen++;
        pthread_cond_broadcast(&g_shm->cv);
    } else {
        while (g_shm->bar_gen == gen) wait_or_die();
    }
    unlock();
    return MPI_SUCCESS;
}

int MPI_Get_processor_name(char *name, int *len)
{
    gethostname(name, MPI_MAX_PROCESSOR_NAME - 1);
    name[MPI_MAX_PROCESSOR_NAME - 1] = 0;
    *len = (int)strlen(name);
    return MPI_SUCCESS;
}

double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int MPI_Cart_create(MPI_Comm old, int ndims, const int dims[], const int periods[],
                    int reorder, MPI_Comm *cart)
{
    (void)periods; (void)reorder;
    g_cart_ndims = ndims;
    for (int i = 0; i < ndims && i < 8; i++) g_cart_dims[i] = dims[i];
    *cart = old;
    return MPI_SUCCESS;
}

int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int coords[])
{
    (void)comm;
    int r = rank;
    for (int i = g_cart_ndims - 1; i >= 0; i--) {
        if (i < maxdims) coords[i] = r % g_cart_dims[i];
        r /= g_cart_dims[i];
    }
    return MPI_SUCCESS;
}

/* ---- point to point ----------------------------------------------------- */
int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag,
              MPI_Comm comm, MPI_Request *req)
{
    (void)comm;
    size_t len = (size_t)count * type_extent(type);
    lock();
    int slot = -1;
    for (int i = 0; i < MAXMSG; i++)
        if (!g_shm->msgs[i].used) { slot = i; break; }
    if (slot < 0) {
        unlock();
        fprintf(stderr, "mpi_shim: message table full\n");
        abort();
    }
    size_t off = arena_alloc(len ? len : 1);
    memcpy(g_arena + off, buf, len);
    shm_msg *m = &g_shm->msgs[slot];
    m->used = 1;
    m->src = g_rank;
    m->dst = dest;
    m->tag = tag;
    m->seq = g_shm->seq++;
    m->off = off;
    m->len = len;
    pthread_cond_broadcast(&g_shm->cv);
    unlock();
    if (req) *req = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}

int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm)
{
    MPI_Request r;
    return MPI_Isend(buf, count, type, dest, tag, comm, &r);
}

int MPI_Irecv(void *buf, int count, MPI_Datatype type, int src, int tag,
              MPI_Comm comm, MPI_Request *req)
{
    (void)comm;
    struct mmsref_req *r = (struct mmsref_req *)calloc(1, sizeof(*r));
    r->is_recv = 1;
    r->buf = buf;
    r->maxlen = (size_t)count * type_extent(type);
    r->src = src;
    r->tag = tag;
    *req = r;
    return MPI_SUCCESS;
}

static void complete_recv(struct mmsref_req *r, MPI_Status *st)
{
    lock();
    for (;;) {
        int best = -1;
        for (int i = 0; i < MAXMSG; i++) {
            shm_msg *m = &g_shm->msgs[i];
            if (!m->used || m->dst != g_rank) continue;
            if (r->src != MPI_ANY_SOURCE && m->src != r->src) continue;
            if (r->tag != MPI_ANY_TAG && m->tag != r->tag) continue;
            if (best < 0 || m->seq < g_shm->msgs[best].seq) best = i;
        }
        if (best >= 0) {
            shm_msg *m = &g_shm->msgs[best];
            if (m->len > r->maxlen) {
                unlock();
                fprintf(stderr, "mpi_shim: message truncated (%zu > %zu)\n", m->len, r->maxlen);
                abort();
            }
            memcpy(r->buf, g_arena + m->off, m->len);
            if (st) {
                st->MPI_SOURCE = m->src;
                st->MPI_TAG = m->tag;
                st->MPI_ERROR = 0;
                st->count = m->len;
            }
            arena_free(m->off);
            m->used = 0;
            break;
        }
        wait_or_die();
    }
    unlock();
}

int MPI_Wait(MPI_Request *req, MPI_Status *status)
{
    if (*req) {
        if ((*req)->is_recv) complete_recv(*req, status);
        free(*req);
        *req = MPI_REQUEST_NULL;
    }
    return MPI_SUCCESS;
}

int MPI_Waitall(int n, MPI_Request reqs[], MPI_Status statuses[])
{
    for (int i = 0; i < n; i++) MPI_Wait(&reqs[i], statuses ? &statuses[i] : NULL);
    return MPI_SUCCESS;
}

int MPI_Recv(void *buf, int count, MPI_Datatype type, int src, int tag,
             MPI_Comm comm, MPI_Status *status)
{
    MPI_Request r;
    MPI_Irecv(buf, count, type, src, tag, comm, &r);
    return MPI_Wait(&r, status);
}

int MPI_Sendrecv(const void *sbuf, int scount, MPI_Datatype stype, int dest, int stag,
                 void *rbuf, int rcount, MPI_Datatype rtype, int src, int rtag,
                 MPI_Comm comm, MPI_Status *status)
{
    MPI_Send(sbuf, scount, stype, dest, stag, comm);
    return MPI_Recv(rbuf, rcount, rtype, src, rtag, comm, status);
}

/* ---- collectives -------------------------------------------------------- */
/* Publish this rank's block, wait for everyone, run `fn` (reads peers'
 * blocks), wait again, free own block. */
static void publish(const void *data, size_t len)
{
    lock();
    size_t off = arena_alloc(len ? len : 1);
    unlock();
    if (len) memcpy(g_arena + off, data, len);
    g_shm->coll_off[g_rank] = off;
    g_shm->coll_len[g_rank] = len;
}

static void retire(void)
{
    MPI_Barrier(MPI_COMM_WORLD);
    lock();
    arena_free(g_shm->coll_off[g_rank]);
    unlock();
}

static const void *peer(int r) { return g_arena + g_shm->coll_off[r]; }

int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm)
{
    (void)comm;
    size_t len = (size_t)count * type_extent(type);
    publish(g_rank == root ? buf : NULL, g_rank == root ? len : 0);
    MPI_Barrier(MPI_COMM_WORLD);
    if (g_rank != root) memcpy(buf, peer(root), len);
    retire();
    return MPI_SUCCESS;
}

static void combine(void *acc, const void *x, int count, MPI_Datatype type, MPI_Op op)
{
    for (int i = 0; i < count; i++) {
        switch (type) {
#define CASE(T, CT)                                                          \
    case T: {                                                                \
        CT *a = (CT *)acc + i;                                               \
        CT b = ((const CT *)x)[i];                                           \
        if (op == MPI_SUM) *a = *a + b;                                      \
        else if (op == MPI_MAX) *a = *a > b ? *a : b;                        \
        else *a = *a < b ? *a : b;                                           \
        break;                                                               \
    }
            CASE(MPI_INT, int)
            CASE(MPI_DOUBLE, double)
            CASE(MPI_LONG_LONG_INT, long long)
            CASE(MPI_UNSIGNED_LONG, unsigned long)
            CASE(MPI_UNSIGNED_LONG_LONG, unsigned long long)
            CASE(MPI_FLOAT, float)
            CASE(MPI_UNSIGNED, unsigned)
            CASE(MPI_LONG, long)
#undef CASE
        default:
            fprintf(stderr, "mpi_shim: reduce on unsupported type %d\n", type);
            abort();
        }
    }
}

int MPI_Reduce(const void *sbuf, void *rbuf, int count, MPI_Datatype type, MPI_Op op,
               int root, MPI_Comm comm)
{
    (void)comm;
    size_t len = (size_t)count * type_extent(type);
    const void *mine = (sbuf == MPI_IN_PLACE) ? rbuf : sbuf;
    publish(mine, len);
    MPI_Barrier(MPI_COMM_WORLD);
    if (g_rank == root) {
        char *acc = (char *)malloc(len ? len : 1);
        memcpy(acc, peer(0), len);
        for (int r = 1; r < g_np; r++) combine(acc, peer(r), count, type, op);
        memcpy(rbuf, acc, len);
        free(acc);
    }
    retire();
    return MPI_SUCCESS;
}

int MPI_Allreduce(const void *sbuf, void *rbuf, int count, MPI_Datatype type, MPI_Op op,
                  MPI_Comm comm)
{
    (void)comm;
    size_t len = (size_t)count * type_extent(type);
    const void *mine = (sbuf == MPI_IN_PLACE) ? rbuf : sbuf;
    publish(mine, len);
    MPI_Barrier(MPI_COMM_WORLD);
    char *acc = (char *)malloc(len ? len : 1);
    memcpy(acc, peer(0), len);
    for (int r = 1; r < g_np; r++) combine(acc, peer(r), count, type, op);
    retire();
    memcpy(rbuf, acc, len);
    free(acc);
    return MPI_SUCCESS;
}

int MPI_Gather(const void *sbuf, int scount, MPI_Datatype stype, void *rbuf, int rcount,
               MPI_Datatype rtype, int root, MPI_Comm comm)
{
    (void)comm;
    size_t rl = (size_t)rcount * type_extent(rtype);
    if (sbuf == MPI_IN_PLACE)
        publish((char *)rbuf + (size_t)g_rank * rl, rl);
    else
        publish(sbuf, (size_t)scount * type_extent(stype));
    MPI_Barrier(MPI_COMM_WORLD);
    if (g_rank == root)
        for (int r = 0; r < g_np; r++) memcpy((char *)rbuf + (size_t)r * rl, peer(r), rl);
    retire();
    return MPI_SUCCESS;
}

int MPI_Allgather(const void *sbuf, int scount, MPI_Datatype stype, void *rbuf, int rcount,
                  MPI_Datatype rtype, MPI_Comm comm)
{
    (void)comm;
    size_t rl = (size_t)rcount * type_extent(rtype);
    if (sbuf == MPI_IN_PLACE)
        publish((char *)rbuf + (size_t)g_rank * rl, rl);
    else
        publish(sbuf, (size_t)scount * type_extent(stype));
    MPI_Barrier(MPI_COMM_WORLD);
    for (int r = 0; r < g_np; r++) memcpy((char *)rbuf + (size_t)r * rl, peer(r), rl);
    retire();
    return MPI_SUCCESS;
}

int MPI_Allgatherv(const void *sbuf, int scount, MPI_Datatype stype, void *rbuf,
                   const int rcounts[], const int displs[], MPI_Datatype rtype,
                   MPI_Comm comm)
{
    (void)comm;
    size_t ext = type_extent(rtype);
    if (sbuf == MPI_IN_PLACE)
        publish((char *)rbuf + (size_t)displs[g_rank] * ext, (size_t)rcounts[g_rank] * ext);
    else
        publish(sbuf, (size_t)scount * type_extent(stype));
    MPI_Barrier(MPI_COMM_WORLD);
    for (int r = 0; r < g_np; r++)
        memcpy((char *)rbuf + (size_t)displs[r] * ext, peer(r), (size_t)rcounts[r] * ext);
    retire();
    return MPI_SUCCESS;
}
