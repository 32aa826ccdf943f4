/* Minimal MPI stand-in covering the calls on the reference's compute_soi path
 * (soi.h:14; pfft.c:331-333,484-609,719; parallel_filter_subsampling.cpp:
 * 105-108,483,525).  Ranks are forked processes sharing one anonymous
 * MAP_SHARED region; sends are buffered into it, receives match (source, tag)
 * in posting order.  TEST INFRASTRUCTURE for oracle/_ref only. */
#ifndef SOI_SHIM_MPI_H
#define SOI_SHIM_MPI_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct soi_mpi_req *MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_CHAR 1
#define MPI_INT 2
#define MPI_FLOAT 3
#define MPI_DOUBLE 4
#define MPI_LONG 5
#define MPI_MAX 1
#define MPI_SUM 2
#define MPI_MIN 3
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3
#define MPI_MAX_ERROR_STRING 256
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
int MPI_Init(int *argc, char ***argv);
int MPI_Init_thread(int *argc, char ***argv, int required, int *provided);
int MPI_Finalize(void);
int MPI_Comm_size(MPI_Comm c, int *size);
int MPI_Comm_rank(MPI_Comm c, int *rank);
int MPI_Isend(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *r);
int MPI_Irecv(void *buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm c, MPI_Request *r);
int MPI_Wait(MPI_Request *r, MPI_Status *st);
int MPI_Waitall(int n, MPI_Request *r, MPI_Status *st);
int MPI_Barrier(MPI_Comm c);
int MPI_Allreduce(const void *in, void *out, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c);
int MPI_Reduce(const void *in, void *out, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c);
int MPI_Ialltoallv(const void *sb, const int *sc, const int *sd, MPI_Datatype st,
                   void *rb, const int *rc, const int *rd, MPI_Datatype rt, MPI_Comm c, MPI_Request *r);
int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *newt);
int MPI_Type_commit(MPI_Datatype *t);
int MPI_Error_string(int code, char *s, int *len);
double MPI_Wtime(void);

/* harness entry: run body(rank, arg) on P forked ranks (in-process for P=1);
 * returns 0 when every rank exited 0. */
int soi_mpi_run(int P, size_t arena_bytes, int (*body)(int rank, void *arg), void *arg);
#ifdef __cplusplus
}
#endif
#endif
