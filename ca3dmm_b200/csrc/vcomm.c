/* Virtual communicator: carries the number of virtual ranks of a folded call. */
#include <stdlib.h>
#include "ca3dmm_vmpi.h"

struct ca3dmm_vcomm_s {
    int size;
};

int ca3dmm_vcomm_create(int p, MPI_Comm *comm)
{
    if (comm == NULL) return 1;
    *comm = NULL;
    if (p < 1) return 1;
    MPI_Comm c = (MPI_Comm) malloc(sizeof(struct ca3dmm_vcomm_s));
    if (c == NULL) return 1;
    c->size = p;
    *comm = c;
    return 0;
}

void ca3dmm_vcomm_free(MPI_Comm *comm)
{
    if (comm == NULL || *comm == NULL) return;
    free(*comm);
    *comm = NULL;
}

int ca3dmm_vcomm_size(MPI_Comm comm) { return comm ? comm->size : 0; }
