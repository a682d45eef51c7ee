/*
 * pvfmm_mpi_stub.h -- lets pvfmm.h compile without an MPI installation.
 *
 * The reference C interface takes an MPI_Comm (include/pvfmm.h:11, 254).  This
 * library runs one rank per GPU and ignores the communicator beyond checking
 * that it is a single-rank one.  Define PVFMM_B200_HAVE_MPI before including
 * pvfmm.h to use a real <mpi.h> instead.
 */
#ifndef PVFMM_B200_MPI_STUB_H_
#define PVFMM_B200_MPI_STUB_H_

#ifdef PVFMM_B200_HAVE_MPI
#include <mpi.h>
#else
#ifndef MPI_COMM_WORLD
typedef int MPI_Comm;
#define MPI_COMM_WORLD ((MPI_Comm)0x44000000)
#define MPI_COMM_SELF  ((MPI_Comm)0x44000001)
#endif
#endif

#endif /* PVFMM_B200_MPI_STUB_H_ */
