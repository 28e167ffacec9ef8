/*
 * Single-rank MPI shim used only to compile the TIOGA reference sources into
 * the CPU oracle library (oracle/_ref).  It is test infrastructure, never
 * linked into the product library.
 *
 * Every communicator has exactly one rank (rank 0 of 1).  Collectives reduce
 * to copies; point-to-point messages are self-messages held in a FIFO
 * mailbox matched by tag (MPI's non-overtaking rule for one source).
 *
 * Datatype handles encode their size in bytes, which is all a one-rank
 * implementation needs.
 */
#ifndef TIOGA_ORACLE_MPI_SHIM_H
#define TIOGA_ORACLE_MPI_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Fint;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;

typedef struct MPI_Status {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
  int count_bytes;
} MPI_Status;

#define MPI_COMM_WORLD ((MPI_Comm)91)
#define MPI_COMM_NULL ((MPI_Comm)0)
#define MPI_SUCCESS 0

/* datatype handle == element size in bytes */
#define MPI_INT ((MPI_Datatype)4)
#define MPI_DOUBLE ((MPI_Datatype)8)

#define MPI_MAX ((MPI_Op)1)
#define MPI_MIN ((MPI_Op)2)
#define MPI_SUM ((MPI_Op)3)

#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
MPI_Comm MPI_Comm_f2c(MPI_Fint comm);
int MPI_Barrier(MPI_Comm comm);
int MPI_Abort(MPI_Comm comm, int code);
double MPI_Wtime(void);

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count,
                  MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count,
               MPI_Datatype type, MPI_Op op, int root, MPI_Comm comm);
int MPI_Allgather(const void *sendbuf, int scount, MPI_Datatype stype,
                  void *recvbuf, int rcount, MPI_Datatype rtype, MPI_Comm comm);
int MPI_Allgatherv(const void *sendbuf, int scount, MPI_Datatype stype,
                   void *recvbuf, const int *rcounts, const int *displs,
                   MPI_Datatype rtype, MPI_Comm comm);
int MPI_Alltoall(const void *sendbuf, int scount, MPI_Datatype stype,
                 void *recvbuf, int rcount, MPI_Datatype rtype, MPI_Comm comm);

int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest,
              int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag,
              MPI_Comm comm, MPI_Request *req);
int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *stats);

#ifdef __cplusplus
}
#endif

#endif
