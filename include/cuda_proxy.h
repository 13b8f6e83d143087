/* Device selection for one rank per GPU (replaces the one function of
 * src/cuda_proxy.h that the reference's example drivers call,
 * src/cuda_proxy.h:25-26; examples/example_AB.c:43-46).  The rest of that
 * header wraps cuBLAS / cuSOLVER / cudaMemcpy for the reference's own use and
 * has no counterpart here: the engines take device pointers directly. */
#ifndef CA3DMM_CUDA_PROXY_H
#define CA3DMM_CUDA_PROXY_H

#ifdef __cplusplus
extern "C" {
#endif

/* Make device (local rank mod device count) current for the calling thread.
 * The local rank is read from the launcher's environment: the first of
 * MPI_LOCALRANKID (MPICH / Intel MPI), MV2_COMM_WORLD_LOCAL_RANK (MVAPICH2),
 * OMPI_COMM_WORLD_NODE_RANK (Open MPI), SLURM_LOCALID, PBS_O_VNODENUM that is
 * set (a value that is not a non-negative number counts as 0); 0 when none is.  May be called before MPI_Init.  A CUDA error is printed (the
 * library does not exit) and leaves the current device unchanged. */
void select_cuda_device_by_mpi_local_rank(void);

/* The local rank select_cuda_device_by_mpi_local_rank reads (-1: none set). */
int ca3dmm_mpi_local_rank_env(void);

#ifdef __cplusplus
}
#endif
#endif
