/* Empty stand-in: the reference's CA3DMM core calls no LAPACK routine. */
#ifndef VMPI_LAPACKE_H
#define VMPI_LAPACKE_H
#endif
