/*
 * Single-rank stand-in for <mpi.h>, used only to compile the reference's CPU
 * sources into the test oracle (oracle/_ref). Test infrastructure, not product.
 *
 * The reference calls a handful of MPI routines on its hot path
 * (src/Flowfield.cpp:298-303 dt reduction, :846-848 halo exchange,
 * src/Reaction.cpp:971 Nchem gather, MPI_Abort on errors). With one rank every
 * neighbour is MPI_PROC_NULL, so sends/receives are never reached and the
 * collectives reduce to a copy of the local buffer.
 */
#pragma once
#include <cstddef>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int source, tag, error; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_PROC_NULL (-1)
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_MIN 3
#define MPI_MAX 4
#define MPI_SUM 5

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm, int *rank);
int MPI_Comm_size(MPI_Comm, int *size);
int MPI_Abort(MPI_Comm, int code);
int MPI_Barrier(MPI_Comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype, int root, MPI_Comm);
int MPI_Reduce(const void *send, void *recv, int count, MPI_Datatype, MPI_Op, int root, MPI_Comm);
int MPI_Gather(const void *send, int scount, MPI_Datatype stype, void *recv, int rcount,
               MPI_Datatype rtype, int root, MPI_Comm);
int MPI_Isend(const void *buf, int count, MPI_Datatype, int dest, int tag, MPI_Comm, MPI_Request *);
int MPI_Irecv(void *buf, int count, MPI_Datatype, int src, int tag, MPI_Comm, MPI_Request *);
int MPI_Waitall(int count, MPI_Request *, MPI_Status *);
