/*
 * mpi.h — minimal MPI interface used to compile the muMatScale reference
 * sources (src/*.c) as a CPU oracle.  This is test infrastructure, not part
 * of the product: it lets the unmodified reference run as N processes on one
 * host (fork + shared memory) so that its own outputs can pin the oracle and
 * serve as the timed CPU baseline.
 *
 * Only the entry points the reference calls are provided (ca_main.c,
 * calculate.c, face_util.c, distribute.c, grain.c, loop.c, functions.c,
 * profiler.c).  Sends are buffered (complete on return); receives match
 * (source, tag) in arrival order, like MPI's non-overtaking rule.
 */
#ifndef MMSREF_MPI_H
#define MMSREF_MPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPI_VERSION 3
#define MPI_SUBVERSION 0

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Errhandler;
typedef long MPI_Aint;
typedef struct mmsref_req *MPI_Request;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; size_t count; } MPI_Status;

#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_REQUEST_NULL ((MPI_Request)0)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)
#define MPI_ERRORS_RETURN 1
#define MPI_ERRORS_ARE_FATAL 0
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)

#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3

/* predefined datatypes: the handle indexes the shim's type table */
#define MPI_DATATYPE_NULL 0
#define MPI_BYTE 1
#define MPI_CHAR 1
#define MPI_INT 2
#define MPI_DOUBLE 3
#define MPI_LONG_LONG_INT 4
#define MPI_LONG_LONG 4
#define MPI_UNSIGNED_LONG 5
#define MPI_UNSIGNED_LONG_LONG 6
#define MPI_FLOAT 7
#define MPI_UNSIGNED 8
#define MPI_LONG 9

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

int MPI_Init(int *argc, char ***argv);
int MPI_Init_thread(int *argc, char ***argv, int required, int *provided);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Barrier(MPI_Comm comm);
int MPI_Get_processor_name(char *name, int *len);
double MPI_Wtime(void);

int MPI_Cart_create(MPI_Comm old, int ndims, const int dims[], const int periods[],
                    int reorder, MPI_Comm *cart);
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int coords[]);

int MPI_Type_create_struct(int count, const int blocklens[], const MPI_Aint disps[],
                           const MPI_Datatype types[], MPI_Datatype *newtype);
int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *newtype);
int MPI_Type_commit(MPI_Datatype *type);
int MPI_Type_free(MPI_Datatype *type);
int MPI_Type_size(MPI_Datatype type, int *size);

int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag,
             MPI_Comm comm);
int MPI_Irecv(void *buf, int count, MPI_Datatype type, int src, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Recv(void *buf, int count, MPI_Datatype type, int src, int tag,
             MPI_Comm comm, MPI_Status *status);
int MPI_Wait(MPI_Request *req, MPI_Status *status);
int MPI_Waitall(int n, MPI_Request reqs[], MPI_Status statuses[]);
int MPI_Sendrecv(const void *sbuf, int scount, MPI_Datatype stype, int dest, int stag,
                 void *rbuf, int rcount, MPI_Datatype rtype, int src, int rtag,
                 MPI_Comm comm, MPI_Status *status);

int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Reduce(const void *sbuf, void *rbuf, int count, MPI_Datatype type, MPI_Op op,
               int root, MPI_Comm comm);
int MPI_Allreduce(const void *sbuf, void *rbuf, int count, MPI_Datatype type, MPI_Op op,
                  MPI_Comm comm);
int MPI_Gather(const void *sbuf, int scount, MPI_Datatype stype, void *rbuf, int rcount,
               MPI_Datatype rtype, int root, MPI_Comm comm);
int MPI_Allgather(const void *sbuf, int scount, MPI_Datatype stype, void *rbuf, int rcount,
                  MPI_Datatype rtype, MPI_Comm comm);
int MPI_Allgatherv(const void *sbuf, int scount, MPI_Datatype stype, void *rbuf,
                   const int rcounts[], const int displs[], MPI_Datatype rtype,
                   MPI_Comm comm);

#ifdef __cplusplus
}
#endif
#endif
