/*
 * Single-process stand-in for the subset of MPI that the pEVSL reference
 * sources use.  TEST INFRASTRUCTURE ONLY: it exists so that the reference C
 * code under the read-only reference tree can be compiled, unmodified, into
 * oracle/_ref/ and run as a one-rank, one-group checker.  Nothing in the
 * product library includes or links this file.
 *
 * Semantics on one rank:
 *   - every communicator has size 1 and this process is rank 0;
 *   - reductions / gathers / all-to-alls copy the send buffer to the receive
 *     buffer (the identity for one participant);
 *   - broadcasts and barriers are no-ops;
 *   - point-to-point calls are never reached with one rank (the parcsr halo is
 *     empty) and succeed without moving data.
 * An MPI_Datatype value is the element size in bytes, which is all a
 * one-rank copy needs.
 */
#ifndef ORACLE_MPISTUB_MPI_H
#define ORACLE_MPISTUB_MPI_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
} MPI_Status;

#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_SUCCESS 0
#define MPI_UNDEFINED (-32766)
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))
#define MPI_INT ((MPI_Datatype)sizeof(int))
#define MPI_UNSIGNED_LONG ((MPI_Datatype)sizeof(unsigned long))
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

static inline int MPI_Init(int *argc, char ***argv) {
  (void)argc;
  (void)argv;
  return MPI_SUCCESS;
}
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r) {
  (void)c;
  *r = 0;
  return MPI_SUCCESS;
}
static inline int MPI_Comm_size(MPI_Comm c, int *s) {
  (void)c;
  *s = 1;
  return MPI_SUCCESS;
}
static inline int MPI_Comm_split(MPI_Comm c, int color, int key, MPI_Comm *out) {
  (void)key;
  *out = (color == MPI_UNDEFINED) ? MPI_COMM_NULL : c;
  return MPI_SUCCESS;
}
static inline int MPI_Comm_free(MPI_Comm *c) {
  *c = MPI_COMM_NULL;
  return MPI_SUCCESS;
}
static inline int MPI_Barrier(MPI_Comm c) {
  (void)c;
  return MPI_SUCCESS;
}
static inline int MPI_Abort(MPI_Comm c, int code) {
  (void)c;
  fprintf(stderr, "MPI_Abort (single-process stub), code %d\n", code);
  abort();
  return code;
}
static inline double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
/* One-rank collectives: the result equals the local contribution. */
static inline int oracle_mpistub_copy(const void *s, void *r, int cnt, MPI_Datatype t) {
  if (cnt > 0 && s != r) {
    memmove(r, s, (size_t)cnt * (size_t)t);
  }
  return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void *s, void *r, int cnt, MPI_Datatype t, MPI_Op op,
                                MPI_Comm c) {
  (void)op;
  (void)c;
  return oracle_mpistub_copy(s, r, cnt, t);
}
static inline int MPI_Reduce(const void *s, void *r, int cnt, MPI_Datatype t, MPI_Op op,
                             int root, MPI_Comm c) {
  (void)op;
  (void)root;
  (void)c;
  return oracle_mpistub_copy(s, r, cnt, t);
}
static inline int MPI_Bcast(void *b, int cnt, MPI_Datatype t, int root, MPI_Comm c) {
  (void)b;
  (void)cnt;
  (void)t;
  (void)root;
  (void)c;
  return MPI_SUCCESS;
}
static inline int MPI_Allgather(const void *s, int scnt, MPI_Datatype st, void *r, int rcnt,
                                MPI_Datatype rt, MPI_Comm c) {
  (void)rcnt;
  (void)rt;
  (void)c;
  return oracle_mpistub_copy(s, r, scnt, st);
}
static inline int MPI_Alltoall(const void *s, int scnt, MPI_Datatype st, void *r, int rcnt,
                               MPI_Datatype rt, MPI_Comm c) {
  (void)rcnt;
  (void)rt;
  (void)c;
  return oracle_mpistub_copy(s, r, scnt, st);
}
static inline int MPI_Alltoallv(const void *s, const int *scnt, const int *sdis, MPI_Datatype st,
                                void *r, const int *rcnt, const int *rdis, MPI_Datatype rt,
                                MPI_Comm c) {
  (void)rcnt;
  (void)rt;
  (void)c;
  return oracle_mpistub_copy((const char *)s + (size_t)sdis[0] * (size_t)st,
                             (char *)r + (size_t)rdis[0] * (size_t)st, scnt[0], st);
}
static inline int MPI_Isend(const void *b, int cnt, MPI_Datatype t, int dst, int tag, MPI_Comm c,
                            MPI_Request *req) {
  (void)b;
  (void)cnt;
  (void)t;
  (void)dst;
  (void)tag;
  (void)c;
  *req = 0;
  return MPI_SUCCESS;
}
static inline int MPI_Irecv(void *b, int cnt, MPI_Datatype t, int src, int tag, MPI_Comm c,
                            MPI_Request *req) {
  (void)b;
  (void)cnt;
  (void)t;
  (void)src;
  (void)tag;
  (void)c;
  *req = 0;
  return MPI_SUCCESS;
}
static inline int MPI_Waitall(int cnt, MPI_Request *req, MPI_Status *st) {
  (void)cnt;
  (void)req;
  (void)st;
  return MPI_SUCCESS;
}

#endif
