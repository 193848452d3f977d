/*
 * Fortran binding of pEVSL — the entry points of FORTRAN/pevsl_f90.c
 * (lines 16-453; names: INC/pevsl_def.h:108, name ## _f90_).  A Fortran
 * program calls e.g. `call pevsl_start_f90(comm, pevsl)`, which a Fortran
 * compiler with the usual trailing-underscore mangling resolves to
 * pevsl_start_f90_.  Every argument is passed by reference; handles
 * (instance, parcsr, filter, B-solver) are uintptr_t (INTEGER*8 on 64-bit
 * hosts).  CSR arrays given to pevsl_parcsrcreate are C-indexed.
 * Host arrays passed to pevsl_parcsrmatvec, pevsl_bsv, pevsl_chebiter and
 * pevsl_lspolsol are staged to the device and back; callbacks installed
 * from Fortran receive managed (host-accessible) arrays.
 */
#ifndef PEVSL_F90_H
#define PEVSL_F90_H

#include <stdint.h>

#include "pevsl.h"

#ifdef __cplusplus
extern "C" {
#endif

void pevsl_start_f90_(MPI_Fint *Fcomm, uintptr_t *pevslf90);                     /* :16  */
void pevsl_finish_f90_(uintptr_t *pevslf90);                                     /* :28  */
void pevsl_seta_parcsr_f90_(uintptr_t *pevslf90, uintptr_t *Af90);               /* :37  */
void pevsl_setb_parcsr_f90_(uintptr_t *pevslf90, uintptr_t *Bf90);               /* :47  */
void pevsl_setprobsizes_f90_(uintptr_t *pevslf90, int *N, int *n, int *nfirst);  /* :63  */
void pevsl_setamv_f90_(uintptr_t *pevslf90, void *func, void *data);             /* :76  */
void pevsl_setbmv_f90_(uintptr_t *pevslf90, void *func, void *data);             /* :89  */
void pevsl_setbsol_f90_(uintptr_t *pevslf90, void *func, void *data);            /* :98  */
void pevsl_set_stdeig_f90_(uintptr_t *pevslf90);                                 /* :107 */
void pevsl_set_geneig_f90_(uintptr_t *pevslf90);                                 /* :116 */
void pevsl_parcsrcreate_f90_(int *nrow, int *ncol, int *row_starts, int *col_starts, int *ia,
                             int *ja, double *aa, MPI_Fint *Fcomm, uintptr_t *matf90); /* :134 */
void pevsl_parcsr_free_f90_(uintptr_t *Af90);                                    /* :159 */
void pevsl_parcsrmatvec_f90_(double *x, double *y, uintptr_t *matf90);           /* :168 */
void pevsl_bsv_f90_(uintptr_t *pevslf90, double *b, double *x);                  /* :176 */
void pevsl_lanbounds_f90_(uintptr_t *pevslf90, int *mlan, int *nsteps, double *tol,
                          double *lmin, double *lmax);                           /* :193 */
void pevsl_findpol_f90_(double *xintv, double *thresh_int, double *thresh_ext,
                        uintptr_t *polf90);                                      /* :225 */
void pevsl_freepol_f90_(uintptr_t *polf90);                                      /* :243 */
void pevsl_cheblannr_f90_(uintptr_t *pevslf90, double *xintv, int *max_its, double *tol,
                          uintptr_t *polf90);                                    /* :253 */
void pevsl_get_nev_f90_(uintptr_t *pevslf90, int *nev);                          /* :296 */
void pevsl_copy_result_f90_(uintptr_t *pevslf90, double *val, double *vec, int *ld); /* :311 */
void pevsl_setup_chebiter_f90_(double *lmin, double *lmax, int *deg, uintptr_t *parcsrf90,
                               uintptr_t *chebf90);                              /* :333 */
void pevsl_chebiter_f90_(int *type, double *b, double *x, uintptr_t *chebf90);   /* :344 */
void pevsl_chebiterstatsprint_f90_(uintptr_t *chebf90);                          /* :357 */
void pevsl_free_chebiterb_f90_(uintptr_t *chebf90);                              /* :367 */
void pevsl_setbsol_chebiter_f90_(uintptr_t *pevslf90, int *type, uintptr_t *chebf90); /* :377 */
void pevsl_setup_lspolsqrt_f90_(double *lmin, double *lmax, int *maxdeg, double *tol,
                                uintptr_t *parcsrf90, uintptr_t *lspolf90);      /* :391 */
void pevsl_lspolsol_f90_(double *b, double *x, uintptr_t *lspolf90);             /* :402 */
void pevsl_free_lspol_f90_(uintptr_t *lspolf90);                                 /* :410 */
void pevsl_setltsol_lspol_f90_(uintptr_t *pevslf90, uintptr_t *lspolf90);        /* :420 */
void pevsl_kpmdos_ecnt_f90_(uintptr_t *pevslf90, int *Mdeg, int *damping, int *nvec,
                            double *intv, double *mu, double *ecnt);             /* :429 */
void pevsl_landos_ecnt_f90_(uintptr_t *pevslf90, int *nvec, int *msteps, int *npts,
                            double *intv, double *ecnt);                         /* :437 */
void pevsl_set_sigmamult_f90_(uintptr_t *pevslf90, double *mult);                /* :453 */

#ifdef __cplusplus
}
#endif

#endif
