/*
 * pevsl-b200: single-process stand-in for the MPI types and calls that the
 * pEVSL interface mentions.
 *
 * The pEVSL C API carries MPI_Comm in its structs and signatures
 * (INC/pevsl_struct.h:59-135, INC/pevsl.h:20-103 of the reference).  On one
 * B200 there is one process per GPU and no MPI library, so this header
 * supplies MPI_Comm as an opaque int together with the one-rank semantics
 * of the few calls that pEVSL drivers make (rank 0 of 1, collectives copy,
 * splits return the same communicator).  Build with -DPEVSL_USE_MPI to take
 * the types from a real <mpi.h> instead; the struct ABI then follows that
 * MPI's MPI_Comm (an int in MPICH, a pointer in Open MPI).
 */
#ifndef PEVSL_SERIAL_MPI_H
#define PEVSL_SERIAL_MPI_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Fint; /* Fortran handle: the same int as the C handle here */
typedef int MPI_Datatype; /* element size in bytes */
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct {
  int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_SUCCESS 0
#define MPI_UNDEFINED (-32766)
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))
#define MPI_INT ((MPI_Datatype)sizeof(int))
#define MPI_UNSIGNED_LONG ((MPI_Datatype)sizeof(unsigned long))
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

static inline int pevsl_serial_mpi_copy(const void *s, void *r, int n, MPI_Datatype t) {
  if (n > 0 && s != r) memmove(r, s, (size_t)n * (size_t)t);
  return MPI_SUCCESS;
}
static inline MPI_Comm MPI_Comm_f2c(MPI_Fint c) { return (MPI_Comm)c; }
static inline MPI_Fint MPI_Comm_c2f(MPI_Comm c) { return (MPI_Fint)c; }
static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return 0; }
static inline int MPI_Comm_split(MPI_Comm c, int color, int key, MPI_Comm *out) {
  (void)key;
  *out = color == MPI_UNDEFINED ? MPI_COMM_NULL : c;
  return 0;
}
static inline int MPI_Comm_free(MPI_Comm *c) { *c = MPI_COMM_NULL; return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
static inline int MPI_Abort(MPI_Comm c, int code) {
  (void)c;
  fprintf(stderr, "MPI_Abort(%d)\n", code);
  exit(code ? code : 1);
}
static inline double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op o,
                                MPI_Comm c) {
  (void)o; (void)c;
  return pevsl_serial_mpi_copy(s, r, n, t);
}
static inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op o, int root,
                             MPI_Comm c) {
  (void)o; (void)root; (void)c;
  return pevsl_serial_mpi_copy(s, r, n, t);
}
static inline int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c) {
  (void)b; (void)n; (void)t; (void)root; (void)c;
  return 0;
}

#endif
