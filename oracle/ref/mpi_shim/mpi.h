/*
 * Single-rank stand-in for <mpi.h>, written for this project so that the
 * reference's hot-path translation units compile and run as one MPI rank
 * without an MPI installation.  Test infrastructure only (oracle/_ref).
 * Every communicator has size 1; collectives copy their send buffer; point
 * to point calls accept only MPI_PROC_NULL partners.
 */
#ifndef APRL_ORACLE_MPI_SHIM_H
#define APRL_ORACLE_MPI_SHIM_H
#define MPI_H 1
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_COMM_NULL 0
#define MPI_PROC_NULL (-2)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)1)
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3

#define MPI_CHAR 1
#define MPI_INT 2
#define MPI_UNSIGNED 3
#define MPI_LONG 4
#define MPI_UNSIGNED_LONG 5
#define MPI_LONG_LONG 6
#define MPI_UNSIGNED_LONG_LONG 7
#define MPI_DOUBLE 8
#define MPI_LONG_DOUBLE 9
#define MPI_BYTE 10
#define MPI_UINT64_T 11
#define MPI_C_BOOL 12

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_LOR 4
#define MPI_LAND 5
#define MPI_MAXLOC 6
#define MPI_MINLOC 7
#define MPI_2INT 13
#define MPI_DOUBLE_INT 14

int MPI_Init(int*, char***);
int MPI_Init_thread(int*, char***, int, int*);
int MPI_Initialized(int*);
int MPI_Finalized(int*);
int MPI_Finalize(void);
int MPI_Query_thread(int*);
int MPI_Comm_rank(MPI_Comm, int*);
int MPI_Comm_size(MPI_Comm, int*);
int MPI_Abort(MPI_Comm, int);
int MPI_Barrier(MPI_Comm);
double MPI_Wtime(void);
int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm);
int MPI_Allreduce(const void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm);
int MPI_Reduce(const void*, void*, int, MPI_Datatype, MPI_Op, int, MPI_Comm);
int MPI_Allgather(const void*, int, MPI_Datatype, void*, int, MPI_Datatype, MPI_Comm);
int MPI_Gather(const void*, int, MPI_Datatype, void*, int, MPI_Datatype, int, MPI_Comm);
int MPI_Scatter(const void*, int, MPI_Datatype, void*, int, MPI_Datatype, int, MPI_Comm);
int MPI_Alltoall(const void*, int, MPI_Datatype, void*, int, MPI_Datatype, MPI_Comm);
int MPI_Alltoallv(const void*, const int*, const int*, MPI_Datatype, void*,
                  const int*, const int*, MPI_Datatype, MPI_Comm);
int MPI_Sendrecv(const void*, int, MPI_Datatype, int, int, void*, int,
                 MPI_Datatype, int, int, MPI_Comm, MPI_Status*);
int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm);
int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*);

#ifdef __cplusplus
}
#endif
#endif
