/*
 * pevsl-b200 — drop-in C interface of pEVSL's spectrum-slicing eigensolver,
 * implemented on one NVIDIA B200 (sm_100a).
 *
 * Every declaration below replaces the reference declaration cited next to
 * it (paths relative to the pEVSL project).  Struct layouts are field-for-
 * field those of the reference (INC/pevsl_struct.h) so that pEVSL drivers
 * compile and run unchanged; the documented differences are:
 *
 *   - One process per GPU.  Communicators are accepted and stored but the
 *     matrix is never row-partitioned: pEVSL_ParcsrSetup uploads the rows it
 *     is given as ONE device CSR (the diag/offd split and the halo exchange
 *     of SRC/parcsr.c / SRC/parcsrmv.c disappear).
 *   - The `data` arrays of pevsl_Parvec / pevsl_Parvecs created by this
 *     library live in CUDA managed memory: the host may read and write them
 *     between calls (as TESTS0/Matvec/test1.c does) and the kernels use them
 *     in place.  pevsl_Csr arrays reachable from a pevsl_Parcsr (diag) are
 *     device memory.  pevsl_Csr / pevsl_Coo built by the caller and handed to
 *     the host CSR utilities (pEVSL_CooToCsr, pEVSL_Matvec, ...) stay host
 *     memory, as in the reference.
 *   - A user matvec installed with pEVSL_SetAMatvec receives device (managed)
 *     pointers and must finish its work before returning; the built-in
 *     parcsr matvec is fused into the filter and moment kernels instead of
 *     being called through the pointer.
 *   - Nothing aborts the process: errors come back as return codes (the
 *     reference's codes where it has them, PEVSL_ERR_* below otherwise).
 *   - The generalized problem (SetGenEig): B-solve and L^{-T}-solve
 *     callbacks (SetBSol, SetLTSol) receive device (managed) pointers like
 *     a user matvec.  The library's own solvers -- least-squares
 *     polynomials (pEVSL_LSPolSol) and Chebyshev iterations
 *     (pevsl_itsol.h) -- run on the device; direct solvers (MUMPS, PARDISO)
 *     are not provided.
 */
#ifndef PEVSL_H
#define PEVSL_H

#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>

#ifdef PEVSL_USE_MPI
#include <mpi.h>
#else
#include "pevsl_serial_mpi.h"
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ constants
 * INC/pevsl_def.h:10-18,112 */
#define PEVSL_NOT_DEFINED -2
#define PEVSL_NOT_IMPLEMENT 11
#define PEVSL_MAX_LINE 2048
#define PEVSL_MAX(a, b) ((a) > (b) ? (a) : (b))
#define PEVSL_MIN(a, b) ((a) < (b) ? (a) : (b))
#define orthTol 1e-14
#ifndef PI
#define PI M_PI
#endif
#define NGS_MAX 2
#define PEVSL_FORT(name) name##_f90_

/* Error codes added by this implementation (never used by the reference). */
#define PEVSL_ERR_CUDA (-1001)     /* a CUDA runtime call failed            */
#define PEVSL_ERR_NOMEM (-1002)    /* device or host allocation failed      */
#define PEVSL_ERR_ARG (-1003)      /* bad size / pointer / layout argument  */
#define PEVSL_ERR_NOMATVEC (-1004) /* no matvec installed for A             */
#define PEVSL_ERR_NONFINITE (-1005) /* NaN/Inf met in a vector or scalar    */
#define PEVSL_ERR_EIG (-1006)      /* tridiagonal / dense eigensolver failed */

/* Helper macros that pEVSL drivers use (INC/pevsl_def.h:20-92); here they
 * report and exit instead of calling MPI_Abort on a communicator. */
#define PEVSL_ABORT(comm, errcode, msg)                    \
  {                                                        \
    fprintf(stderr, "PEVSL error: %s\n", msg);             \
    MPI_Abort(comm, errcode);                              \
  }
#ifdef PEVSL_DEBUG
#define PEVSL_CHKERR(ierr) \
  if (ierr) { PEVSL_ABORT(MPI_COMM_WORLD, 999, "Assertion failed") }
#else
#define PEVSL_CHKERR(ierr)
#endif
#define PEVSL_MALLOC(base, nmem, type)                                       \
  {                                                                          \
    (base) = (type *)malloc((size_t)(nmem) * sizeof(type));                  \
    if ((base) == NULL && (nmem) > 0) {                                      \
      PEVSL_ABORT(MPI_COMM_WORLD, -1, "out of host memory");                 \
    }                                                                        \
  }
#define PEVSL_CALLOC(base, nmem, type)                                       \
  {                                                                          \
    (base) = (type *)calloc((size_t)(nmem), sizeof(type));                   \
    if ((base) == NULL && (nmem) > 0) {                                      \
      PEVSL_ABORT(MPI_COMM_WORLD, -1, "out of host memory");                 \
    }                                                                        \
  }
#define PEVSL_REALLOC(base, nmem, type)                                      \
  {                                                                          \
    (base) = (type *)realloc((base), (size_t)(nmem) * sizeof(type));         \
    if ((base) == NULL && (nmem) > 0) {                                      \
      PEVSL_ABORT(MPI_COMM_WORLD, -1, "out of host memory");                 \
    }                                                                        \
  }
#define PEVSL_FREE(base) \
  {                      \
    if (base) {          \
      free(base);        \
    }                    \
    (base) = NULL;       \
  }
/* One process: the "sequential section" runs once, as rank 0 of 1. */
#define PEVSL_SEQ_BEGIN(MPI_COMM)   \
  {                                 \
    int size = 1, rank = 0, __i = 0; \
    (void)size;                     \
    (void)rank;                     \
    (void)__i;                      \
    {
#define PEVSL_SEQ_END(MPI_COMM) \
  }                             \
  }

/* ------------------------------------------------------------------ structs
 * Field order and types as INC/pevsl_struct.h:12-308. */

/* COO, 0-based (pevsl_struct.h:12-15). */
typedef struct _pevsl_cooMat {
  int nrows, ncols, nnz, *ir, *jc;
  double *vv;
} pevsl_Coo;

/* CSR, 0-based, nnz == ia[nrows] (pevsl_struct.h:23-26). */
typedef struct _pevsl_csrMat {
  int nrows, ncols, *ia, *ja;
  double *a;
} pevsl_Csr;

#define PEVSL_CSRNNZ(A) A->ia[A->nrows]

/* Halo-exchange plan of the reference (pevsl_struct.h:37-55).  Kept for the
 * layout of pevsl_Parcsr; on one GPU there is no halo and the pointer
 * pevsl_Parcsr.comm_handle refers to the library's device matrix instead. */
typedef struct _commHandle {
  int num_proc_send_to;
  int *proc_send_to;
  int *send_elmts_ids;
  int *send_elmts_ptr;
  int num_proc_recv_from;
  int *proc_recv_from;
  int *recv_elmts_ptr;
  double *send_buf;
  double *recv_buf;
  MPI_Request *send_recv_requests;
  MPI_Status *send_recv_status;
} commHandle;

/* Parallel CSR (pevsl_struct.h:59-103).  After pEVSL_ParcsrSetup: `diag`
 * describes the whole local matrix with DEVICE arrays, `offd` is empty. */
typedef struct _pevsl_parcsr {
  MPI_Comm comm;
  commHandle *comm_handle;
  int nrow_global;
  int ncol_global;
  int nrow_local;
  int ncol_local;
  int *row_starts;
  int *col_starts;
  int first_row;
  int first_col;
  pevsl_Csr *diag;
  pevsl_Csr *offd;
  int *col_map_offd;
} pevsl_Parcsr;

/* Parallel vector (pevsl_struct.h:109-116); data in managed memory. */
typedef struct _pevsl_parvec {
  MPI_Comm comm;
  int n_global;
  int n_local;
  int n_first;
  double *data;
} pevsl_Parvec;

/* Column-major multi-vector, leading dimension ld (pevsl_struct.h:125-135). */
typedef struct _pevsl_parvecs {
  MPI_Comm comm;
  int n_global;
  int n_local;
  int n_first;
  int n_vecs;
  int ld;
  double *data;
} pevsl_Parvecs;

/* Filter parameters and result (pevsl_struct.h:143-173). */
typedef struct _pevsl_polparams {
  int max_deg;
  int min_deg;
  int damping;
  double thresh_ext;
  double thresh_int;
  double intvtol;
  int type;
  double *mu;
  double cc;
  double dd;
  double gam;
  double bar;
  int deg;
} pevsl_Polparams;

/* Callback types (pevsl_struct.h:186-208). */
typedef void (*SVFuncC)(double *br, double *bz, double *xr, double *xz, void *data);
typedef void (*SVFunc)(double *b, double *x, void *data);
typedef void (*MVFunc)(double *x, double *y, void *data);

typedef struct _pevsl_Matvec {
  MVFunc func;
  void *data;
} pevsl_Matvec;

typedef struct _pevsl_Bsol {
  SVFunc func;
  void *data;
} pevsl_Bsol;

typedef struct _pevsl_LtSol {
  SVFunc func;
  void *data;
} pevsl_Ltsol;

/* Timers (seconds, from CUDA events / host clock) and counters
 * (pevsl_struct.h:241-272). */
typedef struct _pevsl_Stat {
  double t_setBsv;
  double t_setASigBsv;
  double t_eigbounds;
  double t_dos;
  double t_iter;
  double t_mvA;
  double t_mvB;
  double t_svB;
  double t_svLT;
  double t_svASigB;
  double t_reorth;
  double t_eig;
  double t_blas;
  double t_ritz;
  double t_polAv;
  double t_ratAv;
  double t_sth;
  size_t n_mvA;
  size_t n_mvB;
  size_t n_svB;
  size_t n_svLT;
  size_t n_svASigB;
  size_t n_polAv;
  size_t n_ratAv;
  size_t alloced;
  size_t alloced_total;
  size_t alloced_max;
} pevsl_Stat;

/* Instance (pevsl_struct.h:278-306).  Allocated by pEVSL_Start together
 * with the library's private GPU state; only pEVSL_Finish frees it. */
typedef struct _pevsl_Data {
  MPI_Comm comm;
  int N;
  int n;
  int nfirst;
  int ifGenEv;
  pevsl_Matvec *Amv;
  pevsl_Matvec *Bmv;
  pevsl_Bsol *Bsol;
  pevsl_Ltsol *LTsol;
  pevsl_Stat *stats;
  int nev_computed;
  double *eval_computed;
  pevsl_Parvecs *evec_computed;
  double sigma_mult;
} pevsl_Data;

/* ------------------------------------------------------------------ API */

/* Filter design — SRC/chebpol.c (INC/pevsl.h:12-14). */
void pEVSL_SetPolDef(pevsl_Polparams *pol);       /* chebpol.c:10   */
/* chebpol.c:359; the degree search runs from 2 to max_deg (or the forced
 * degree) as in the reference; a limit of 2 or less returns PEVSL_ERR_ARG */
int pEVSL_FindPol(double *intv, pevsl_Polparams *pol);
void pEVSL_FreePol(pevsl_Polparams *pol);         /* chebpol.c:491  */

/* KPM density of states — SRC/kpmdos.c:36 (INC/pevsl.h:17-18). */
int pEVSL_Kpmdos(pevsl_Data *pevsl, int Mdeg, int damping, int nvec, double *intv, int ngroups,
                 int groupid, MPI_Comm gl_comm, double *mu, double *ecnt);

/* Lanczos density of states — SRC/landos.c:40,331 (INC/pevsl.h:21-25). */
int pEVSL_LanDosG(pevsl_Data *pevsl, const int nvec, int msteps, int npts, double *xdos,
                  double *ydos, double *neig, double *intv, int ngroups, int groupid,
                  MPI_Comm gl_comm);
void pEVSL_SpslicerLan(double *xi, double *yi, int n_int, int npts, double *sli);

/* Spectrum bounds — SRC/lantrbnd.c:31 (INC/pevsl.h:28-30). */
int pEVSL_LanTrbounds(pevsl_Data *pevsl, int lanm, int maxit, double tol, pevsl_Parvec *vinit,
                      int bndtype, double *lammin, double *lammax, FILE *fstats);

/* Least-squares polynomial approximation of B^{-1/2} (or B^{-1}) applied
 * as a solve callback — SRC/lspolapprox.c (INC/pevsl.h:31-37).  B must be
 * a parcsr set up by this library; *vdata is NULL on failure.
 * pEVSL_SetupLSPol / pEVSL_SetupLSPolRec are exported by the reference's
 * library (SRC/lspolapprox.c:171,207) without a declaration in its header. */
void pEVSL_SetupLSPolSqrt(int max_deg, double tol, double lmin, double lmax, pevsl_Parcsr *B,
                          void **vdata);                        /* lspolapprox.c:221 */
void pEVSL_SetupLSPolRec(int max_deg, double tol, double lmin, double lmax, pevsl_Parcsr *B,
                         void **vdata);                         /* lspolapprox.c:207 */
void pEVSL_SetupLSPol(int max_deg, double tol, double lmin, double lmax, pevsl_Parcsr *B,
                      double (*ffun)(double), void **vdata);    /* lspolapprox.c:171 */
void pEVSL_LSPolSol(double *db, double *dx, void *data);        /* lspolapprox.c:296 */
void pEVSL_LSPolFree(void *vdata);                              /* lspolapprox.c:314 */

/* Instance — SRC/pevsl.c (INC/pevsl.h:41-52). */
int pEVSL_Start(MPI_Comm comm, pevsl_Data **data);                 /* pevsl.c:13  */
int pEVSL_Finish(pevsl_Data *pevsl_data);                          /* pevsl.c:52  */
int pEVSL_SetProbSizes(pevsl_Data *pevsl_data, int N, int n, int nfirst); /* :131 */
int pEVSL_SetAParcsr(pevsl_Data *pevsl_data, pevsl_Parcsr *A);     /* pevsl.c:81  */
int pEVSL_SetBParcsr(pevsl_Data *pevsl_data, pevsl_Parcsr *B);     /* pevsl.c:105 */
int pEVSL_SetAMatvec(pevsl_Data *pevsl_data, MVFunc func, void *data); /* :148 */
int pEVSL_SetBMatvec(pevsl_Data *pevsl_data, MVFunc func, void *data); /* :167 */
int pEVSL_SetBSol(pevsl_Data *pevsl_data, SVFunc func, void *data);    /* :184 */
int pEVSL_SetLTSol(pevsl_Data *pevsl_data, SVFunc func, void *data);   /* :201 */
int pEVSL_SetStdEig(pevsl_Data *pevsl_data);                       /* pevsl.c:216 */
int pEVSL_SetGenEig(pevsl_Data *pevsl_data);                       /* pevsl.c:228 */
int pEVSL_SetSigmaMult(pevsl_Data *pevsl_data, double mult);       /* pevsl.c:236 */

/* Parallel CSR — SRC/parcsr.c, SRC/parcsrmv.c (INC/pevsl.h:55-65). */
int pEVSL_ParcsrCreate(int nrow, int ncol, int *row_starts, int *col_starts, pevsl_Parcsr *A,
                       MPI_Comm comm);                              /* parcsr.c:24  */
int pEVSL_ParcsrSetup(pevsl_Csr *Ai, pevsl_Parcsr *A);             /* parcsr.c:70  */
void pEVSL_ParcsrFree(pevsl_Parcsr *A);                            /* parcsr.c:286 */
int pEVSL_ParcsrGetLocalMat(pevsl_Parcsr *A, int idx, pevsl_Coo *coo, pevsl_Csr *csr,
                            char stype);                            /* parcsr.c:319 */
int pEVSL_ParcsrNnz(pevsl_Parcsr *A);                              /* parcsr.c:408 */
int pEVSL_ParcsrLocalNnz(pevsl_Parcsr *A);                         /* parcsr.c:422 */
void pEVSL_ParcsrMatvec(pevsl_Parcsr *A, pevsl_Parvec *x, pevsl_Parvec *y); /* parcsrmv.c:84 */
/* The matvec callback installed by pEVSL_SetAParcsr (parcsrmv.c:66); x and
 * y are device or managed pointers, data is the pevsl_Parcsr. */
void pEVSL_ParcsrMatvec0(double *x, double *y, void *data);

/* Parallel vectors — SRC/parvec.c (INC/pevsl.h:68-86). */
void pEVSL_ParvecCreate(int nglobal, int nlocal, int nfirst, MPI_Comm comm, pevsl_Parvec *x);
void pEVSL_ParvecCreateShell(int nglobal, int nlocal, int nfirst, MPI_Comm comm, pevsl_Parvec *x,
                             double *data);
void pEVSL_ParvecDupl(pevsl_Parvec *x, pevsl_Parvec *y);
void pEVSL_ParvecFree(pevsl_Parvec *x);
void pEVSL_ParvecRand(pevsl_Parvec *x);
void pEVSL_ParvecDot(pevsl_Parvec *x, pevsl_Parvec *y, double *t);
void pEVSL_ParvecNrm2(pevsl_Parvec *x, double *t);
void pEVSL_ParvecCopy(pevsl_Parvec *x, pevsl_Parvec *y);
void pEVSL_ParvecSum(pevsl_Parvec *x, double *t);
void pEVSL_ParvecScal(pevsl_Parvec *x, double t);
void pEVSL_ParvecSetScalar(pevsl_Parvec *x, double t);
void pEVSL_ParvecSetZero(pevsl_Parvec *x);
void pEVSL_ParvecAxpy(double a, pevsl_Parvec *x, pevsl_Parvec *y);
int pEVSL_ParvecSameSize(pevsl_Parvec *x, pevsl_Parvec *y);
int pEVSL_ParvecWrite(pevsl_Parvec *x, const char *fn);

/* Parallel multi-vectors — SRC/parvecs.c (INC/pevsl.h:89-111). */
void pEVSL_ParvecsCreateShell(int nglobal, int nvecs, int ld, int nlocal, int nfirst,
                              MPI_Comm comm, pevsl_Parvecs *x, double *data);
void pEVSL_ParvecsCreate(int nglobal, int nvecs, int ld, int nlocal, int nfirst, MPI_Comm comm,
                         pevsl_Parvecs *x);
void pEVSL_ParvecsDuplParvec(pevsl_Parvec *x, int nvecs, int ld, pevsl_Parvecs *y);
void pEVSL_ParvecsFree(pevsl_Parvecs *x);
void pEVSL_ParvecsGetParvecShell(pevsl_Parvecs *X, int i, pevsl_Parvec *x);
void pEVSL_ParvecsGemv(double alp, pevsl_Parvecs *A, int nvecs, double *x, double bet,
                       pevsl_Parvec *y);
void pEVSL_ParvecsGemtvWithWspace(double alp, pevsl_Parvecs *A, int nvecs, pevsl_Parvec *x,
                                  double bet, double *y, double *w);
void pEVSL_ParvecsGemtv(double alp, pevsl_Parvecs *A, int nvecs, pevsl_Parvec *x, double bet,
                        double *y);

/* Host CSR / COO utilities — SRC/spmat.c (INC/pevsl.h:114-122).  These act
 * on host pevsl_Csr / pevsl_Coo as in the reference (matrix assembly by the
 * caller happens on the host before pEVSL_ParcsrSetup uploads it). */
void pEVSL_CsrResize(int nrow, int ncol, int nnz, pevsl_Csr *csr);
void pEVSL_FreeCsr(pevsl_Csr *csr);
void pEVSL_CooResize(int nrow, int ncol, int nnz, pevsl_Coo *coo);
void pEVSL_FreeCoo(pevsl_Coo *coo);
int pEVSL_CooToCsr(int cooidx, pevsl_Coo *coo, pevsl_Csr *csr);
int pEVSL_CsrToCoo(pevsl_Csr *csr, int cooidx, pevsl_Coo *coo);
int pEVSL_MatvecGen(double alp, pevsl_Csr *A, double *x, double bet, double *y);
int pEVSL_Matvec(pevsl_Csr *A, double *x, double *y);
void pEVSL_SortRow(pevsl_Csr *A);

/* Utilities — SRC/utils.c, SRC/vector.c (INC/pevsl.h:125-137). */
void pEVSL_SortInt(int *x, int n);
void pEVSL_SortDouble(int n, double *v, int *ind);
void pEVSL_LinSpace(double a, double b, int num, double *arr);
void pEVSL_Part1d(int len, int pnum, int *idx, int *j1, int *j2, int job);
int pEVSL_BinarySearch(int *x, int n, int key);
void pEVSL_Vecset(int n, double t, double *v);
double pEVSL_Wtime(void);
void linspace(double a, double b, int num, double *arr);
void vecset(int n, double t, double *v);
void sort_double(int n, double *v, int *ind);

/* Spectrum slicing by KPM — SRC/spslicer.c:62 (INC/pevsl.h:140). */
int pEVSL_SpslicerKpm(double *sli, double *mu, int Mdeg, double *intv, int n_int, int npts);

/* Statistics — SRC/stats.c:13,109 (INC/pevsl.h:143-144). */
void pEVSL_StatsReset(pevsl_Data *pevsl);
void pEVSL_StatsPrint(pevsl_Data *pevsl, FILE *fstats);

/* Filtered non-restarted Lanczos — SRC/cheblanNr.c:54 (INC/pevsl.h:147-149).
 * *lamo and *reso are host malloc; *Wo is a malloc'd pevsl_Parvecs whose
 * data is managed memory (free with pEVSL_ParvecsFree + free). */
int pEVSL_ChebLanNr(pevsl_Data *pevsl, double *intv, int maxit, double tol, pevsl_Parvec *vinit,
                    pevsl_Polparams *pol, int *nevOut, double **lamo, pevsl_Parvecs **Wo,
                    double **reso, FILE *fstats);

#ifdef __cplusplus
}
#endif

#endif
