/*
 * Link-time stand-ins for the oracle/_ref build of the reference's CPU path.
 * Test infrastructure only.
 *
 * 1. A single-rank MPI (declared in ref_shim/mpi.h): rank 0 of 1, collectives copy
 *    the local buffer, point-to-point calls are unreachable with one rank
 *    (src/Flowfield.cpp:809-1117 guards every exchange with m_block_* > 1).
 * 2. The reference's CUDA-side entry points that its CPU objects still name after
 *    dead-branch elimination with use_cuda=false. The "chain" queries answer
 *    false (src/Flowfield.cpp:1132, :1334 then take the CPU branch); the GPU
 *    routines are never reached on the CPU path and abort if they are.
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cuda_runtime.h>
#include "mpi.h"

int MPI_Init(int *, char ***) { return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return 0; }
int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return 0; }
int MPI_Abort(MPI_Comm, int code)
{
    std::fprintf(stderr, "oracle/_ref: reference called MPI_Abort(%d)\n", code);
    std::abort();
}
int MPI_Barrier(MPI_Comm) { return 0; }
int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }

static size_t type_size(MPI_Datatype t) { return t == MPI_INT ? sizeof(int) : sizeof(double); }

int MPI_Reduce(const void *send, void *recv, int count, MPI_Datatype t, MPI_Op, int, MPI_Comm)
{
    std::memmove(recv, send, size_t(count) * type_size(t));
    return 0;
}
int MPI_Gather(const void *send, int scount, MPI_Datatype st, void *recv, int, MPI_Datatype, int, MPI_Comm)
{
    std::memmove(recv, send, size_t(scount) * type_size(st));
    return 0;
}
static int unreachable(const char *what)
{
    std::fprintf(stderr, "oracle/_ref: %s reached with a single rank\n", what);
    std::abort();
}
int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return unreachable("MPI_Isend"); }
int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return unreachable("MPI_Irecv"); }
int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return unreachable("MPI_Waitall"); }

/* include/FlowfieldCuda.cuh:71-72 */
void begin_muscl_upload_scope(bool) {}
void end_muscl_upload_scope() {}
/* include/ReactionCuda.cuh:279-282 */
bool ee_state_chain_enabled() { return false; }
bool ee_state_chain_pending() { return false; }
void publish_ee_state_rhs(const double *, int, int, int, int, int) { unreachable("publish_ee_state_rhs"); }
void post_advection_from_ee_host(const double *, const double *, const double *, int, int, int, int, int, double,
                                 const double *, const double *, const double *, const double *)
{
    unreachable("post_advection_from_ee_host");
}
/* include/TimeAdvCuda.cuh:6 */
cudaError_t launch_ee_cuda(const double *, const double *, const double *, const double *, const double *,
                           const double *, double *, int, int, int, int, int, double)
{
    unreachable("launch_ee_cuda");
    return cudaErrorUnknown;
}
