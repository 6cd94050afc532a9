/* Single-rank MPI stand-in used ONLY to compile the reference solver as a CPU
 * oracle (test infrastructure, never part of the product).  One process is
 * rank 0 of a world of size 1: reductions copy, all-to-all exchanges copy the
 * self segment, and point-to-point messages are matched rank-0 -> rank-0 by
 * tag in FIFO order.  Semantics follow the MPI-3.1 standard for a
 * one-process communicator. */
#ifndef ORACLE_SHIM_MPI_H
#define ORACLE_SHIM_MPI_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
#define MPI_VERSION 3
#define MPI_SUBVERSION 1
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct oracle_mpi_req *MPI_Request;
typedef struct MPI_Status {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
  long long oracle_bytes;
} MPI_Status;
#define MPI_COMM_WORLD ((MPI_Comm)1)
#define MPI_SUCCESS 0
#define MPI_CHAR ((MPI_Datatype)1)
#define MPI_BYTE ((MPI_Datatype)2)
#define MPI_INT ((MPI_Datatype)3)
#define MPI_DOUBLE ((MPI_Datatype)4)
#define MPI_INT64_T ((MPI_Datatype)5)
#define MPI_DOUBLE_INT ((MPI_Datatype)6)
#define MPI_LONG_LONG ((MPI_Datatype)7)
#define MPI_UNSIGNED_LONG_LONG ((MPI_Datatype)8)
#define MPI_UINT64_T ((MPI_Datatype)9)
#define MPI_LONG ((MPI_Datatype)10)
#define MPI_UNSIGNED ((MPI_Datatype)11)
#define MPI_FLOAT ((MPI_Datatype)12)
#define MPI_SUM ((MPI_Op)1)
#define MPI_MAX ((MPI_Op)2)
#define MPI_MIN ((MPI_Op)3)
#define MPI_MAXLOC ((MPI_Op)4)
#define MPI_MINLOC ((MPI_Op)5)
#define MPI_LOR ((MPI_Op)6)
#define MPI_LAND ((MPI_Op)7)
#define MPI_REQUEST_NULL ((MPI_Request)0)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)-1)
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)

int MPI_Init(int *argc, char ***argv);
int MPI_Initialized(int *flag);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm c, int *rank);
int MPI_Comm_size(MPI_Comm c, int *size);
int MPI_Barrier(MPI_Comm c);
double MPI_Wtime(void);
int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c);
int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c);
int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c);
int MPI_Gather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, int root, MPI_Comm c);
int MPI_Allgather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm c);
int MPI_Allgatherv(const void *s, int sn, MPI_Datatype st, void *r, const int *rn, const int *displs, MPI_Datatype rt, MPI_Comm c);
int MPI_Alltoall(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm c);
int MPI_Alltoallv(const void *s, const int *sn, const int *sd, MPI_Datatype st, void *r, const int *rn, const int *rd, MPI_Datatype rt, MPI_Comm c);
int MPI_Exscan(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c);
int MPI_Isend(const void *b, int n, MPI_Datatype t, int dst, int tag, MPI_Comm c, MPI_Request *req);
int MPI_Irecv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *req);
int MPI_Wait(MPI_Request *req, MPI_Status *st);
int MPI_Waitall(int n, MPI_Request *reqs, MPI_Status *sts);
int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *count);
int MPI_Abort(MPI_Comm c, int code);
#ifdef __cplusplus
}
#endif
#endif
