/* Single-rank stand-in for the MPI names the reference's particle-FMM path
 * uses.  A communicator has one rank; every collective copies the caller's
 * send buffer into its receive buffer (the one-rank result), point-to-point
 * messages to self are matched in order.  A datatype is its size in bytes. */
#ifndef PVFMM_REF_MPI_STUB_H
#define PVFMM_REF_MPI_STUB_H
#include <stddef.h>
#include <string.h>

typedef int MPI_Comm;
typedef long MPI_Datatype;
typedef int MPI_Fint;
typedef void(MPI_User_function)(void*, void*, int*, MPI_Datatype*);
typedef MPI_User_function* MPI_Op;
typedef struct {
  int MPI_SOURCE, MPI_TAG, MPI_ERROR;
  long count;
} MPI_Status;
typedef struct MPI_Request_s* MPI_Request;

#define MPI_COMM_WORLD 0
#define MPI_COMM_SELF 1
#define MPI_COMM_NULL (-1)
#define MPI_SUCCESS 0
#define MPI_THREAD_FUNNELED 1
#define MPI_IN_PLACE ((void*)1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_REQUEST_NULL ((MPI_Request)0)

#define MPI_CHAR ((MPI_Datatype)sizeof(char))
#define MPI_BYTE ((MPI_Datatype)1)
#define MPI_UNSIGNED_CHAR ((MPI_Datatype)sizeof(unsigned char))
#define MPI_SHORT ((MPI_Datatype)sizeof(short))
#define MPI_UNSIGNED_SHORT ((MPI_Datatype)sizeof(unsigned short))
#define MPI_INT ((MPI_Datatype)sizeof(int))
#define MPI_UNSIGNED ((MPI_Datatype)sizeof(unsigned))
#define MPI_LONG ((MPI_Datatype)sizeof(long))
#define MPI_UNSIGNED_LONG ((MPI_Datatype)sizeof(unsigned long))
#define MPI_LONG_LONG_INT ((MPI_Datatype)sizeof(long long))
#define MPI_LONG_LONG MPI_LONG_LONG_INT
#define MPI_UNSIGNED_LONG_LONG ((MPI_Datatype)sizeof(unsigned long long))
#define MPI_FLOAT ((MPI_Datatype)sizeof(float))
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))
#define MPI_LONG_DOUBLE ((MPI_Datatype)sizeof(long double))

#define MPI_MAX ((MPI_Op)0)
#define MPI_MIN ((MPI_Op)0)
#define MPI_SUM ((MPI_Op)0)

#ifdef __cplusplus
extern "C" {
#endif
int MPI_Init(int*, char***);
int MPI_Init_thread(int*, char***, int, int*);
int MPI_Initialized(int*);
int MPI_Finalize(void);
int MPI_Comm_size(MPI_Comm, int*);
int MPI_Comm_rank(MPI_Comm, int*);
int MPI_Comm_split(MPI_Comm, int, int, MPI_Comm*);
int MPI_Comm_free(MPI_Comm*);
MPI_Comm MPI_Comm_f2c(MPI_Fint);
int MPI_Barrier(MPI_Comm);
int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm);
int MPI_Allreduce(const void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm);
int MPI_Reduce(const void*, void*, int, MPI_Datatype, MPI_Op, int, MPI_Comm);
int MPI_Scan(const void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm);
int MPI_Allgather(const void*, int, MPI_Datatype, void*, int, MPI_Datatype, MPI_Comm);
int MPI_Allgatherv(const void*, int, MPI_Datatype, void*, const int*, const int*, MPI_Datatype, MPI_Comm);
int MPI_Alltoall(const void*, int, MPI_Datatype, void*, int, MPI_Datatype, MPI_Comm);
int MPI_Alltoallv(const void*, const int*, const int*, MPI_Datatype, void*, const int*, const int*, MPI_Datatype,
                  MPI_Comm);
int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm);
int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*);
int MPI_Sendrecv(const void*, int, MPI_Datatype, int, int, void*, int, MPI_Datatype, int, int, MPI_Comm,
                 MPI_Status*);
int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*);
int MPI_Issend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*);
int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*);
int MPI_Wait(MPI_Request*, MPI_Status*);
int MPI_Waitall(int, MPI_Request*, MPI_Status*);
int MPI_Type_contiguous(int, MPI_Datatype, MPI_Datatype*);
int MPI_Type_commit(MPI_Datatype*);
int MPI_Type_free(MPI_Datatype*);
int MPI_Op_create(MPI_User_function*, int, MPI_Op*);
int MPI_Op_free(MPI_Op*);
int MPI_Get_count(const MPI_Status*, MPI_Datatype, int*);
double MPI_Wtime(void);
#ifdef __cplusplus
}
#endif
#endif
