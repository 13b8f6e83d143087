/* Virtual communicator: the MPI_Comm of the reference API, folded onto one GPU.
 *
 * The reference is an SPMD library: every MPI rank calls ca3dmm_engine_init /
 * _exec with its own block (src/ca3dmm.h:114-194).  This build runs the whole
 * mp x np x kp process grid as virtual ranks on one B200, so one host call
 * describes the whole problem and the communicator only carries the number of
 * virtual ranks p.  MPI_Comm, MPI_Datatype and MPI_DOUBLE keep their names so
 * callers written against the reference compile unchanged; they are not MPI.
 */
#ifndef CA3DMM_VMPI_H
#define CA3DMM_VMPI_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ca3dmm_vcomm_s *MPI_Comm;
typedef int MPI_Datatype;
#define MPI_DOUBLE ((MPI_Datatype) 1)
#define MPI_FLOAT  ((MPI_Datatype) 2)
#define MPI_INT    ((MPI_Datatype) 3)

/* Create a communicator of p >= 1 virtual ranks.  Returns 0 on success.
 * (No counterpart in the reference, which takes MPI_COMM_WORLD from MPI.) */
int ca3dmm_vcomm_create(int p, MPI_Comm *comm);
/* Free it and set *comm to NULL. */
void ca3dmm_vcomm_free(MPI_Comm *comm);
/* Number of virtual ranks (MPI_Comm_size). */
int ca3dmm_vcomm_size(MPI_Comm comm);

#ifdef __cplusplus
}
#endif
#endif
