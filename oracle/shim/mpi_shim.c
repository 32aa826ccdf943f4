/* Forked-rank MPI stand-in (see mpi.h).  TEST INFRASTRUCTURE for oracle/_ref. */
#define _GNU_SOURCE
#include "mpi.h"
#include <pthread.h>
#include <sched.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/wait.h>
#include <time.h>
#include <unistd.h>

#define MAXMSG 200000
#define RED_BYTES (8u << 20)
#define WAIT_LIMIT_S 900.0

struct msg { int src, dst, tag, state; size_t off, bytes; };
struct shared {
  pthread_mutex_t lock;
  pthread_barrier_t bar;
  int P;
  size_t arena_size, arena_used;
  int nmsg;
  struct msg msgs[MAXMSG];
};
struct soi_mpi_req { int is_recv; int src, tag; void *buf; size_t bytes; };

static struct shared *g_sh;
static char *g_arena, *g_red;
static int g_rank, g_P = 1;

static size_t tsize(MPI_Datatype t)
{
  switch (t) { case MPI_CHAR: return 1; case MPI_INT: return 4; case MPI_FLOAT: return 4;
  case MPI_DOUBLE: return 8; case MPI_LONG: return 8; default: return 1; }
}
double MPI_Wtime(void)
{
  struct timespec ts; clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}
int MPI_Init(int *a, char ***b) { (void)a; (void)b; return MPI_SUCCESS; }
int MPI_Init_thread(int *a, char ***b, int req, int *prov) { (void)a; (void)b; *prov = req; return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = g_P; return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = g_rank; return MPI_SUCCESS; }

int MPI_Isend(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *r)
{
  (void)c;
  size_t bytes = (size_t)count * tsize(t);
  pthread_mutex_lock(&g_sh->lock);
  if (g_sh->nmsg >= MAXMSG || g_sh->arena_used + bytes > g_sh->arena_size) {
    pthread_mutex_unlock(&g_sh->lock);
    fprintf(stderr, "mpi shim: message arena exhausted\n");
    _exit(4);
  }
  size_t off = g_sh->arena_used;
  g_sh->arena_used += (bytes + 63) & ~(size_t)63;
  pthread_mutex_unlock(&g_sh->lock);
  memcpy(g_arena + off, buf, bytes);
  __sync_synchronize();
  pthread_mutex_lock(&g_sh->lock);
  struct msg *m = &g_sh->msgs[g_sh->nmsg++];
  m->src = g_rank; m->dst = dest; m->tag = tag; m->off = off; m->bytes = bytes; m->state = 1;
  pthread_mutex_unlock(&g_sh->lock);
  struct soi_mpi_req *q = (struct soi_mpi_req *)calloc(1, sizeof(*q));
  q->is_recv = 0;
  *r = q;
  return MPI_SUCCESS;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm c, MPI_Request *r)
{
  (void)c;
  struct soi_mpi_req *q = (struct soi_mpi_req *)calloc(1, sizeof(*q));
  q->is_recv = 1; q->src = source; q->tag = tag; q->buf = buf; q->bytes = (size_t)count * tsize(t);
  *r = q;
  return MPI_SUCCESS;
}

int MPI_Wait(MPI_Request *r, MPI_Status *st)
{
  (void)st;
  struct soi_mpi_req *q = *r;
  if (!q) return MPI_SUCCESS;
  if (q->is_recv) {
    double t0 = MPI_Wtime();
    for (;;) {
      int found = -1;
      pthread_mutex_lock(&g_sh->lock);
      for (int i = 0; i < g_sh->nmsg; ++i) {
        struct msg *m = &g_sh->msgs[i];
        if (m->state == 1 && m->dst == g_rank && m->src == q->src && m->tag == q->tag) {
          m->state = 2; found = i; break;
        }
      }
      pthread_mutex_unlock(&g_sh->lock);
      if (found >= 0) {
        struct msg *m = &g_sh->msgs[found];
        size_t n = m->bytes < q->bytes ? m->bytes : q->bytes;
        memcpy(q->buf, g_arena + m->off, n);
        break;
      }
      if (MPI_Wtime() - t0 > WAIT_LIMIT_S) {
        fprintf(stderr, "mpi shim: rank %d gave up waiting for (src %d, tag %d)\n", g_rank, q->src, q->tag);
        _exit(5);
      }
      sched_yield();
    }
  }
  free(q);
  *r = NULL;
  return MPI_SUCCESS;
}

int MPI_Waitall(int n, MPI_Request *r, MPI_Status *st)
{
  (void)st;
  for (int i = 0; i < n; ++i) MPI_Wait(&r[i], MPI_STATUS_IGNORE);
  return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm c)
{
  (void)c;
  if (g_P == 1) {
    int all = 1;
    for (int i = 0; i < g_sh->nmsg; ++i) if (g_sh->msgs[i].state == 1) all = 0;
    if (all) { g_sh->nmsg = 0; g_sh->arena_used = 0; }
    return MPI_SUCCESS;
  }
  int rc = pthread_barrier_wait(&g_sh->bar);
  if (rc == PTHREAD_BARRIER_SERIAL_THREAD) {
    int all = 1;
    for (int i = 0; i < g_sh->nmsg; ++i) if (g_sh->msgs[i].state == 1) all = 0;
    if (all) { g_sh->nmsg = 0; g_sh->arena_used = 0; }
  }
  pthread_barrier_wait(&g_sh->bar);
  return MPI_SUCCESS;
}

static void reduce_into(void *out, const char *slots, int count, MPI_Datatype t, MPI_Op op)
{
  size_t es = tsize(t);
  for (int e = 0; e < count; ++e) {
    if (t == MPI_INT) {
      int v = ((const int *)slots)[e];
      for (int p = 1; p < g_P; ++p) {
        int x = ((const int *)(slots + (size_t)p * count * es))[e];
        v = op == MPI_MAX ? (x > v ? x : v) : op == MPI_MIN ? (x < v ? x : v) : v + x;
      }
      ((int *)out)[e] = v;
    } else {
      double v = ((const double *)slots)[e];
      for (int p = 1; p < g_P; ++p) {
        double x = ((const double *)(slots + (size_t)p * count * es))[e];
        v = op == MPI_MAX ? (x > v ? x : v) : op == MPI_MIN ? (x < v ? x : v) : v + x;
      }
      ((double *)out)[e] = v;
    }
  }
}

int MPI_Allreduce(const void *in, void *out, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
  size_t es = tsize(t);
  if ((size_t)count * es * g_P > RED_BYTES) { fprintf(stderr, "mpi shim: reduction too large\n"); _exit(6); }
  memcpy(g_red + (size_t)g_rank * count * es, in, (size_t)count * es);
  MPI_Barrier(c);
  reduce_into(out, g_red, count, t, op);
  MPI_Barrier(c);
  return MPI_SUCCESS;
}

int MPI_Reduce(const void *in, void *out, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c)
{
  double tmp[4096];
  if (count > 512) { fprintf(stderr, "mpi shim: reduce too large\n"); _exit(6); }
  MPI_Allreduce(in, tmp, count, t, op, c);
  if (g_rank == root) memcpy(out, tmp, (size_t)count * tsize(t));
  return MPI_SUCCESS;
}

int MPI_Ialltoallv(const void *sb, const int *sc, const int *sd, MPI_Datatype st,
                   void *rb, const int *rc, const int *rd, MPI_Datatype rt, MPI_Comm c, MPI_Request *r)
{
  (void)sb; (void)sc; (void)sd; (void)st; (void)rb; (void)rc; (void)rd; (void)rt; (void)c; (void)r;
  fprintf(stderr, "mpi shim: MPI_Ialltoallv is not provided (reference builds without SOI_USE_I_ALL_TO_ALL)\n");
  return MPI_ERR_OTHER;
}
int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *newt) { (void)count; *newt = old; return MPI_SUCCESS; }
int MPI_Type_commit(MPI_Datatype *t) { (void)t; return MPI_SUCCESS; }
int MPI_Error_string(int code, char *s, int *len) { *len = snprintf(s, MPI_MAX_ERROR_STRING, "mpi shim error %d", code); return MPI_SUCCESS; }

int soi_mpi_run(int P, size_t arena_bytes, int (*body)(int, void *), void *arg)
{
  size_t total = sizeof(struct shared) + RED_BYTES + arena_bytes;
  void *mem = mmap(NULL, total, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
  if (mem == MAP_FAILED) { perror("mmap"); return -1; }
  g_sh = (struct shared *)mem;
  g_red = (char *)mem + sizeof(struct shared);
  g_arena = g_red + RED_BYTES;
  g_sh->P = P; g_sh->arena_size = arena_bytes; g_sh->arena_used = 0; g_sh->nmsg = 0;
  pthread_mutexattr_t ma; pthread_mutexattr_init(&ma);
  pthread_mutexattr_setpshared(&ma, PTHREAD_PROCESS_SHARED);
  pthread_mutex_init(&g_sh->lock, &ma);
  pthread_barrierattr_t ba; pthread_barrierattr_init(&ba);
  pthread_barrierattr_setpshared(&ba, PTHREAD_PROCESS_SHARED);
  pthread_barrier_init(&g_sh->bar, &ba, (unsigned)P);
  g_P = P;
  int rc = 0;
  if (P == 1) {
    g_rank = 0;
    rc = body(0, arg);
  } else {
    pid_t *pids = (pid_t *)calloc((size_t)P, sizeof(pid_t));
    for (int r = 0; r < P; ++r) {
      pid_t pid = fork();
      if (pid == 0) { g_rank = r; int x = body(r, arg); fflush(NULL); _exit(x); }
      pids[r] = pid;
    }
    for (int r = 0; r < P; ++r) {
      int status = 0;
      waitpid(pids[r], &status, 0);
      if (!WIFEXITED(status) || WEXITSTATUS(status) != 0) rc = 1;
    }
    free(pids);
  }
  munmap(mem, total);
  return rc;
}
