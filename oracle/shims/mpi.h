/*
 * mpi.h -- single-process stand-in for the MPI subset the reference uses
 * (Types.h:7; MaterialGrid.cpp:257-271, 425-578, 1009-1045, 1214).
 * Project-written test infrastructure: it lets the reference's own sources
 * compile and run on one CPU core so they can serve as the parity oracle.
 * World size is 1 and rank is 0; MPI_Allreduce copies (and reports each call
 * to an optional hook so the harness can read the reference's reductions);
 * point-to-point calls are never reached with one rank and abort if they are.
 */
#ifndef VPFFT_SHIM_MPI_H
#define VPFFT_SHIM_MPI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
} MPI_Status;

#define MPI_COMM_WORLD ((MPI_Comm)0)
#define MPI_DOUBLE ((MPI_Datatype)1)
#define MPI_BYTE ((MPI_Datatype)2)
#define MPI_INT ((MPI_Datatype)3)
#define MPI_FLOAT ((MPI_Datatype)4)
#define MPI_SUM ((MPI_Op)1)
#define MPI_SUCCESS 0

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op,
                  MPI_Comm comm);
int MPI_Barrier(MPI_Comm comm);
int MPI_Send(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype dt, int src, int tag, MPI_Comm comm,
             MPI_Status *st);
int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm,
              MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int src, int tag, MPI_Comm comm,
              MPI_Request *req);
int MPI_Wait(MPI_Request *req, MPI_Status *st);

#ifdef __cplusplus
}
#endif

#endif
