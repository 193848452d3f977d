/*
 * Fortran binding: the entry points of the reference's FORTRAN/pevsl_f90.c
 * (lines 16-453), with its names (name_f90_, INC/pevsl_def.h:108), argument
 * meaning and defaults, over this library's C API.  Fortran passes every
 * argument by reference; objects (instance, matrices, filters, B-solvers)
 * travel as uintptr_t handles.
 *
 * Fortran arrays are host memory.  The entry points that hand such arrays
 * to device code (pevsl_parcsrmatvec, pevsl_bsv, pevsl_chebiter,
 * pevsl_lspolsol) stage them through managed buffers; callbacks installed
 * from Fortran (pevsl_setamv, ...) receive managed pointers, which a
 * Fortran routine reads and writes like its own arrays.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "internal.h"
#include "pevsl_f90.h"
#include "pevsl_itsol.h"

#define F90(name) name##_f90_

/* y = f(x) on host arrays of n doubles through managed staging */
static void staged(void (*f)(double *, double *, void *), void *data, int n, const double *x,
                   double *y) {
  const size_t bytes = sizeof(double) * (size_t)(n > 0 ? n : 1);
  double *xm = (double *)pEVSL_B200_ManagedAlloc(bytes);
  double *ym = (double *)pEVSL_B200_ManagedAlloc(bytes);
  if (xm && ym) {
    memcpy(xm, x, sizeof(double) * (size_t)n);
    memset(ym, 0, bytes);
    f(xm, ym, data);
    memcpy(y, ym, sizeof(double) * (size_t)n);
  }
  pEVSL_B200_ManagedFree(xm);
  pEVSL_B200_ManagedFree(ym);
}

static void free_saved_result(pevsl_Data *pevsl) {
  if (pevsl->eval_computed) free(pevsl->eval_computed);
  if (pevsl->evec_computed) {
    pEVSL_ParvecsFree(pevsl->evec_computed);
    free(pevsl->evec_computed);
  }
  pevsl->eval_computed = NULL;
  pevsl->evec_computed = NULL;
  pevsl->nev_computed = 0;
}

/* ---------------------------------------------------------------- instance */
void F90(pevsl_start)(MPI_Fint *Fcomm, uintptr_t *pevslf90) {
  pevsl_Data *pevsl = NULL;
  pEVSL_Start(MPI_Comm_f2c(*Fcomm), &pevsl);
  *pevslf90 = (uintptr_t)pevsl;
}

void F90(pevsl_finish)(uintptr_t *pevslf90) {
  pevsl_Data *pevsl = (pevsl_Data *)*pevslf90;
  free_saved_result(pevsl);
  pEVSL_Finish(pevsl);
}

void F90(pevsl_seta_parcsr)(uintptr_t *pevslf90, uintptr_t *Af90) {
  pEVSL_SetAParcsr((pevsl_Data *)*pevslf90, (pevsl_Parcsr *)*Af90);
}

void F90(pevsl_setb_parcsr)(uintptr_t *pevslf90, uintptr_t *Bf90) {
  pEVSL_SetBParcsr((pevsl_Data *)*pevslf90, (pevsl_Parcsr *)*Bf90);
}

/* nfirst < 0: not specified */
void F90(pevsl_setprobsizes)(uintptr_t *pevslf90, int *N, int *n, int *nfirst) {
  pEVSL_SetProbSizes((pevsl_Data *)*pevslf90, *N, *n, *nfirst);
}

void F90(pevsl_setamv)(uintptr_t *pevslf90, void *func, void *data) {
  pEVSL_SetAMatvec((pevsl_Data *)*pevslf90, (MVFunc)func, data);
}

void F90(pevsl_setbmv)(uintptr_t *pevslf90, void *func, void *data) {
  pEVSL_SetBMatvec((pevsl_Data *)*pevslf90, (MVFunc)func, data);
}

void F90(pevsl_setbsol)(uintptr_t *pevslf90, void *func, void *data) {
  pEVSL_SetBSol((pevsl_Data *)*pevslf90, (SVFunc)func, data);
}

void F90(pevsl_set_stdeig)(uintptr_t *pevslf90) { pEVSL_SetStdEig((pevsl_Data *)*pevslf90); }

void F90(pevsl_set_geneig)(uintptr_t *pevslf90) { pEVSL_SetGenEig((pevsl_Data *)*pevslf90); }

void F90(pevsl_set_sigmamult)(uintptr_t *pevslf90, double *mult) {
  pEVSL_SetSigmaMult((pevsl_Data *)*pevslf90, *mult);
}

/* ---------------------------------------------------------------- matrices */

/* ParcsrCreate + ParcsrSetup from this rank's rows in C-indexed CSR */
void F90(pevsl_parcsrcreate)(int *nrow, int *ncol, int *row_starts, int *col_starts, int *ia,
                             int *ja, double *aa, MPI_Fint *Fcomm, uintptr_t *matf90) {
  pevsl_Parcsr *mat = (pevsl_Parcsr *)calloc(1, sizeof(pevsl_Parcsr));
  *matf90 = 0;
  if (!mat) return;
  pEVSL_ParcsrCreate(*nrow, *ncol, row_starts, col_starts, mat, MPI_Comm_f2c(*Fcomm));
  pevsl_Csr loc;
  loc.nrows = mat->nrow_local;
  loc.ncols = mat->ncol_global;
  loc.ia = ia;
  loc.ja = ja;
  loc.a = aa;
  if (pEVSL_ParcsrSetup(&loc, mat)) {
    free(mat);
    return;
  }
  *matf90 = (uintptr_t)mat;
}

void F90(pevsl_parcsr_free)(uintptr_t *Af90) {
  pevsl_Parcsr *A = (pevsl_Parcsr *)*Af90;
  if (!A) return;
  pEVSL_ParcsrFree(A);
  free(A);
  *Af90 = 0;
}

void F90(pevsl_parcsrmatvec)(double *x, double *y, uintptr_t *matf90) {
  pevsl_Parcsr *mat = (pevsl_Parcsr *)*matf90;
  staged(pEVSL_ParcsrMatvec0, mat, mat->nrow_local, x, y);
}

void F90(pevsl_bsv)(uintptr_t *pevslf90, double *b, double *x) {
  pevsl_Data *pevsl = (pevsl_Data *)*pevslf90;
  if (!pevsl->Bsol || !pevsl->Bsol->func) return;
  staged(pevsl->Bsol->func, pevsl->Bsol->data, pevsl->n, b, x);
}

/* ---------------------------------------------------------------- solvers */

/* bounds by thick-restart Lanczos from a random vector; the reference
 * passes tol 1e-8 whatever *tol says (FORTRAN/pevsl_f90.c:216) */
void F90(pevsl_lanbounds)(uintptr_t *pevslf90, int *mlan, int *nsteps, double *tol, double *lmin,
                          double *lmax) {
  pevsl_Data *pevsl = (pevsl_Data *)*pevslf90;
  pevsl_Parvec vinit;
  (void)tol;
  pEVSL_ParvecCreate(pevsl->N, pevsl->n, pevsl->nfirst, pevsl->comm, &vinit);
  pEVSL_ParvecRand(&vinit);
  pEVSL_LanTrbounds(pevsl, *mlan, *nsteps, 1e-8, &vinit, 1, lmin, lmax, NULL);
  pEVSL_ParvecFree(&vinit);
}

/* filter with the defaults of FORTRAN/pevsl_f90.c:225-241: damping 2,
 * max_deg 50000, the given thresholds */
void F90(pevsl_findpol)(double *xintv, double *thresh_int, double *thresh_ext, uintptr_t *polf90) {
  pevsl_Polparams *pol = (pevsl_Polparams *)calloc(1, sizeof(pevsl_Polparams));
  *polf90 = 0;
  if (!pol) return;
  pEVSL_SetPolDef(pol);
  pol->damping = 2;
  pol->thresh_int = *thresh_int;
  pol->thresh_ext = *thresh_ext;
  pol->max_deg = 50000;
  pEVSL_FindPol(xintv, pol);
  fprintf(stdout, " polynomial deg %d, bar %e gam %e\n", pol->deg, pol->bar, pol->gam);
  *polf90 = (uintptr_t)pol;
}

void F90(pevsl_freepol)(uintptr_t *polf90) {
  pevsl_Polparams *pol = (pevsl_Polparams *)*polf90;
  if (!pol) return;
  pEVSL_FreePol(pol);
  free(pol);
  *polf90 = 0;
}

/* ChebLanNr from a random vector, statistics to stdout; the eigenpairs stay
 * in the instance for pevsl_get_nev / pevsl_copy_result */
void F90(pevsl_cheblannr)(uintptr_t *pevslf90, double *xintv, int *max_its, double *tol,
                          uintptr_t *polf90) {
  pevsl_Data *pevsl = (pevsl_Data *)*pevslf90;
  pevsl_Polparams *pol = (pevsl_Polparams *)*polf90;
  int nev2 = 0;
  double *lam = NULL, *res = NULL;
  pevsl_Parvecs *Y = NULL;
  pevsl_Parvec vinit;
  free_saved_result(pevsl);
  pEVSL_StatsReset(pevsl);
  pEVSL_ParvecCreate(pevsl->N, pevsl->n, pevsl->nfirst, pevsl->comm, &vinit);
  pEVSL_ParvecRand(&vinit);
  const int ierr = pEVSL_ChebLanNr(pevsl, xintv, *max_its, *tol, &vinit, pol, &nev2, &lam, &Y,
                                   &res, stdout);
  if (ierr) printf("ChebLanNr error %d\n", ierr);
  pEVSL_ParvecFree(&vinit);
  pEVSL_StatsPrint(pevsl, stdout);
  free(res);
  pevsl->nev_computed = nev2;
  pevsl->eval_computed = lam;
  pevsl->evec_computed = Y;
}

void F90(pevsl_get_nev)(uintptr_t *pevslf90, int *nev) {
  *nev = ((pevsl_Data *)*pevslf90)->nev_computed;
}

/* eigenvalues into val, eigenvectors into the columns of vec (leading
 * dimension *ld >= n); the saved results are released afterwards */
void F90(pevsl_copy_result)(uintptr_t *pevslf90, double *val, double *vec, int *ld) {
  pevsl_Data *pevsl = (pevsl_Data *)*pevslf90;
  const int nev = pevsl->nev_computed;
  if (nev > 0 && pevsl->eval_computed) memcpy(val, pevsl->eval_computed, sizeof(double) * nev);
  if (nev > 0 && pevsl->evec_computed)
    pEVSL_B200_CopyEigenvectors(pevsl->evec_computed, nev, vec, *ld);
  free_saved_result(pevsl);
}

void F90(pevsl_kpmdos_ecnt)(uintptr_t *pevslf90, int *Mdeg, int *damping, int *nvec, double *intv,
                            double *mu, double *ecnt) {
  pEVSL_Kpmdos((pevsl_Data *)*pevslf90, *Mdeg, *damping, *nvec, intv, 1, 0, MPI_COMM_NULL, mu,
               ecnt);
}

void F90(pevsl_landos_ecnt)(uintptr_t *pevslf90, int *nvec, int *msteps, int *npts, double *intv,
                            double *ecnt) {
  double *xdos = (double *)malloc(sizeof(double) * (size_t)(*npts > 0 ? *npts : 1));
  double *ydos = (double *)malloc(sizeof(double) * (size_t)(*npts > 0 ? *npts : 1));
  if (xdos && ydos)
    pEVSL_LanDosG((pevsl_Data *)*pevslf90, *nvec, *msteps, *npts, xdos, ydos, ecnt, intv, 1, 0,
                  MPI_COMM_NULL);
  free(xdos);
  free(ydos);
}

/* ---------------------------------------------------------------- B-solvers */
void F90(pevsl_setup_chebiter)(double *lmin, double *lmax, int *deg, uintptr_t *parcsrf90,
                               uintptr_t *chebf90) {
  void *cheb = NULL;
  pEVSL_ChebIterSetup(*lmin, *lmax, *deg, (pevsl_Parcsr *)*parcsrf90, &cheb);
  *chebf90 = (uintptr_t)cheb;
}

/* x = B^{-1} b by the first (*type == 1) or second kind */
void F90(pevsl_chebiter)(int *type, double *b, double *x, uintptr_t *chebf90) {
  void *cheb = (void *)*chebf90;
  staged(*type == 1 ? pEVSL_ChebIterSolv1 : pEVSL_ChebIterSolv2, cheb, pevsl_chebiter_size(cheb),
         b, x);
}

void F90(pevsl_chebiterstatsprint)(uintptr_t *chebf90) {
  pEVSL_ChebIterStatsPrint((void *)*chebf90, stdout);
}

void F90(pevsl_free_chebiterb)(uintptr_t *chebf90) {
  pEVSL_ChebIterFree((void *)*chebf90);
  *chebf90 = 0;
}

void F90(pevsl_setbsol_chebiter)(uintptr_t *pevslf90, int *type, uintptr_t *chebf90) {
  pEVSL_SetBSol((pevsl_Data *)*pevslf90, *type == 1 ? pEVSL_ChebIterSolv1 : pEVSL_ChebIterSolv2,
                (void *)*chebf90);
}

void F90(pevsl_setup_lspolsqrt)(double *lmin, double *lmax, int *maxdeg, double *tol,
                                uintptr_t *parcsrf90, uintptr_t *lspolf90) {
  void *lspol = NULL;
  pEVSL_SetupLSPolSqrt(*maxdeg, *tol, *lmin, *lmax, (pevsl_Parcsr *)*parcsrf90, &lspol);
  *lspolf90 = (uintptr_t)lspol;
}

void F90(pevsl_lspolsol)(double *b, double *x, uintptr_t *lspolf90) {
  void *lspol = (void *)*lspolf90;
  staged(pEVSL_LSPolSol, lspol, pevsl_lspol_size(lspol), b, x);
}

void F90(pevsl_free_lspol)(uintptr_t *lspolf90) {
  pEVSL_LSPolFree((void *)*lspolf90);
  *lspolf90 = 0;
}

void F90(pevsl_setltsol_lspol)(uintptr_t *pevslf90, uintptr_t *lspolf90) {
  pEVSL_SetLTSol((pevsl_Data *)*pevslf90, pEVSL_LSPolSol, (void *)*lspolf90);
}
