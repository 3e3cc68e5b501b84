/*
 * Single-rank MPI stand-in used only to compile and run the reference
 * (PIGFEM 4.6.1) serially as a CPU oracle.  Test infrastructure: nothing in
 * the product links it.
 *
 * Semantics: one process, rank 0, size 1.  Reductions, scans and broadcasts
 * copy the send buffer into the receive buffer.  Point-to-point calls are
 * never reached on the reference's serial code paths (Mesh::_serial); they
 * abort loudly if they are.
 */
#ifndef PG_REF_SHIM_MPI_H
#define PG_REF_SHIM_MPI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
/* A datatype carries its element size in bytes; that is all a single rank needs. */
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef long MPI_Aint;
typedef struct {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
    int count_bytes;
} MPI_Status;

#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_SUCCESS 0
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)1)

#define MPI_CHAR 1
#define MPI_UNSIGNED_CHAR 1
#define MPI_C_BOOL 1
#define MPI_BYTE 1
#define MPI_SHORT 2
#define MPI_INT 4
#define MPI_UNSIGNED 4
#define MPI_FLOAT 4
#define MPI_LONG 8
#define MPI_UNSIGNED_LONG 8
#define MPI_LONG_LONG 8
#define MPI_DOUBLE 8

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_LOR 4
#define MPI_LAND 5
#define MPI_PROD 6

int MPI_Init(int* argc, char*** argv);
int MPI_Initialized(int* flag);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int* rank);
int MPI_Comm_size(MPI_Comm comm, int* size);
int MPI_Barrier(MPI_Comm comm);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype dt, MPI_Op op, int root, MPI_Comm comm);
int MPI_Scan(const void* sendbuf, void* recvbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm comm);
int MPI_Exscan(const void* sendbuf, void* recvbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm comm);
int MPI_Bcast(void* buf, int count, MPI_Datatype dt, int root, MPI_Comm comm);
int MPI_Gather(const void* sendbuf, int sendcount, MPI_Datatype sdt, void* recvbuf, int recvcount, MPI_Datatype rdt, int root, MPI_Comm comm);
int MPI_Allgather(const void* sendbuf, int sendcount, MPI_Datatype sdt, void* recvbuf, int recvcount, MPI_Datatype rdt, MPI_Comm comm);
int MPI_Gatherv(const void* sendbuf, int sendcount, MPI_Datatype sdt, void* recvbuf, const int* recvcounts, const int* displs, MPI_Datatype rdt, int root, MPI_Comm comm);
int MPI_Allgatherv(const void* sendbuf, int sendcount, MPI_Datatype sdt, void* recvbuf, const int* recvcounts, const int* displs, MPI_Datatype rdt, MPI_Comm comm);
int MPI_Alltoall(const void* sendbuf, int sendcount, MPI_Datatype sdt, void* recvbuf, int recvcount, MPI_Datatype rdt, MPI_Comm comm);
int MPI_Isend(const void* buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm, MPI_Request* req);
int MPI_Send(const void* buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void* buf, int count, MPI_Datatype dt, int source, int tag, MPI_Comm comm, MPI_Status* status);
int MPI_Probe(int source, int tag, MPI_Comm comm, MPI_Status* status);
int MPI_Get_count(const MPI_Status* status, MPI_Datatype dt, int* count);
int MPI_Wait(MPI_Request* req, MPI_Status* status);
int MPI_Waitall(int count, MPI_Request* reqs, MPI_Status* statuses);
int MPI_Type_create_struct(int count, const int* blocklengths, const MPI_Aint* displs, const MPI_Datatype* types, MPI_Datatype* newtype);
int MPI_Type_commit(MPI_Datatype* dt);
int MPI_Type_free(MPI_Datatype* dt);
double MPI_Wtime(void);

#ifdef __cplusplus
}
#endif

#endif
