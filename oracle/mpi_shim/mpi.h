/*
 * Single-rank stand-in for <mpi.h>, written for this project so that the
 * reference library (which includes <mpi.h> unconditionally) can be compiled
 * without an MPI installation. Test infrastructure only: it is used solely by
 * oracle/Makefile to build the reference library into oracle/_ref/.
 *
 * Semantics are those of MPI_COMM_WORLD with exactly one process:
 *   - rank 0, size 1;
 *   - MPI_Allreduce copies the send buffer to the receive buffer (the sum over
 *     one rank is the identity);
 *   - MPI_Barrier, MPI_Isend, MPI_Irecv and MPI_Wait do nothing. With a
 *     {1,1,1,1} process grid the reference never calls the point-to-point
 *     routines (every neighbour is the calling rank itself, see
 *     src/qcu_communicator.cu:1374-1393 of the reference), so no message is
 *     ever lost.
 */
#ifndef QCU_ORACLE_MPI_SHIM_H
#define QCU_ORACLE_MPI_SHIM_H

#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD ((MPI_Comm)0)
#define MPI_DOUBLE ((MPI_Datatype)8)
#define MPI_SUM ((MPI_Op)1)
#define MPI_SUCCESS 0

static inline int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Allreduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op, MPI_Comm) {
  /* MPI_DOUBLE is the only datatype the reference reduces; its size is 8 bytes. */
  memcpy(recvbuf, sendbuf, (size_t)count * (size_t)type);
  return MPI_SUCCESS;
}
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* req) { *req = 0; return MPI_SUCCESS; }
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* req) { *req = 0; return MPI_SUCCESS; }
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { return MPI_SUCCESS; }

#endif
