/* vmpi: a thread-backed subset of MPI, so that the reference's own CPU path
 * (src/ca3dmm.c, cannon.c, mat_redist.c, dev_type.c, mpi_op_omp.c) compiles
 * and runs unmodified in one process: each MPI rank is a host thread.
 * TEST INFRASTRUCTURE ONLY (the oracle's reference build); never part of the
 * product.  Exactly the calls and constants the reference uses. */
#ifndef VMPI_MPI_H
#define VMPI_MPI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct vmpi_comm *MPI_Comm;
typedef int MPI_Datatype;
typedef struct vmpi_op *MPI_Op;
typedef struct vmpi_request *MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
typedef int MPI_Info;
typedef void MPI_User_function(void *invec, void *inoutvec, int *len, MPI_Datatype *dtype);

#define MPI_DOUBLE ((MPI_Datatype) 1)
#define MPI_FLOAT ((MPI_Datatype) 2)
#define MPI_INT ((MPI_Datatype) 3)
#define MPI_SUCCESS 0
#define MPI_STATUS_IGNORE ((MPI_Status *) 0)
#define MPI_IN_PLACE ((void *) 1)
#define MPI_UNWEIGHTED ((int *) 2)
#define MPI_INFO_NULL 0
#define MPI_OP_NULL ((MPI_Op) 0)
extern MPI_Op vmpi_op_sum;
#define MPI_SUM vmpi_op_sum
extern __thread MPI_Comm vmpi_world;
#define MPI_COMM_WORLD vmpi_world

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
double MPI_Wtime(void);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm);
int MPI_Comm_free(MPI_Comm *comm);
int MPI_Cart_create(MPI_Comm comm, int ndims, const int *dims, const int *periods, int reorder,
                    MPI_Comm *cart);
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int *coords);
int MPI_Dist_graph_create_adjacent(MPI_Comm comm, int indegree, const int *sources,
                                   const int *sourceweights, int outdegree, const int *dests,
                                   const int *destweights, MPI_Info info, int reorder,
                                   MPI_Comm *graph);
int MPI_Barrier(MPI_Comm comm);
int MPI_Allgather(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf, int rcount,
                  MPI_Datatype rtype, MPI_Comm comm);
int MPI_Allgatherv(const void *sendbuf, int scount, MPI_Datatype stype, void *recvbuf,
                   const int *rcounts, const int *displs, MPI_Datatype rtype, MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dtype, MPI_Op op,
                  MPI_Comm comm);
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dtype, MPI_Op op,
               int root, MPI_Comm comm);
int MPI_Reduce_scatter(const void *sendbuf, void *recvbuf, const int *rcounts, MPI_Datatype dtype,
                       MPI_Op op, MPI_Comm comm);
int MPI_Reduce_scatter_block(const void *sendbuf, void *recvbuf, int rcount, MPI_Datatype dtype,
                             MPI_Op op, MPI_Comm comm);
int MPI_Isend(const void *buf, int count, MPI_Datatype dtype, int dest, int tag, MPI_Comm comm,
              MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype dtype, int source, int tag, MPI_Comm comm,
              MPI_Request *req);
int MPI_Wait(MPI_Request *req, MPI_Status *status);
int MPI_Sendrecv(const void *sendbuf, int scount, MPI_Datatype stype, int dest, int stag,
                 void *recvbuf, int rcount, MPI_Datatype rtype, int source, int rtag,
                 MPI_Comm comm, MPI_Status *status);
int MPI_Neighbor_alltoallv(const void *sendbuf, const int *scounts, const int *sdispls,
                           MPI_Datatype stype, void *recvbuf, const int *rcounts,
                           const int *rdispls, MPI_Datatype rtype, MPI_Comm comm);
int MPI_Op_create(MPI_User_function *fn, int commute, MPI_Op *op);

/* vmpi extensions: run fn(rank, arg) on p rank threads; a rank that waits
 * longer than timeout_s for a peer makes vmpi_run return nonzero. */
int vmpi_run(int p, void (*fn)(int rank, void *arg), void *arg, double timeout_s);

#ifdef __cplusplus
}
#endif
#endif
