/*
 * pevsl-b200: lets a pEVSL driver that does `#include <mpi.h>` compile as a
 * single process without an MPI installation (add include/serial_mpi to the
 * include path).  See pevsl_serial_mpi.h.
 */
#ifndef PEVSL_SERIAL_MPI_SHIM_MPI_H
#define PEVSL_SERIAL_MPI_SHIM_MPI_H
#include "../pevsl_serial_mpi.h"
#endif
