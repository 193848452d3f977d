/*
 * Chebyshev iterations for B x = b, the iterative B-solvers of the
 * generalized problem — EXTERNAL/ITERSOL/pevsl_itsol.h:14-26 and
 * EXTERNAL/ITERSOL/chebiter.c.  A is a parcsr set up by this library and
 * [lmin, lmax] encloses its spectrum; deg iterations from a zero initial
 * guess.  Solv1 / Solv2 take device (managed) pointers and can be
 * installed with pEVSL_SetBSol; inside the solvers they are queued on the
 * library's stream, called directly they return with the result complete.
 */
#ifndef PEVSL_ITSOL_H
#define PEVSL_ITSOL_H

#include "pevsl.h"

#ifdef __cplusplus
extern "C" {
#endif

/* chebiter.c:77; returns 0, PEVSL_ERR_ARG (A not set up) or PEVSL_ERR_NOMEM */
int pEVSL_ChebIterSetup(double lmin, double lmax, int deg, pevsl_Parcsr *A, void **data);
/* first kind ("Templates ..." form), chebiter.c:121 */
void pEVSL_ChebIterSolv1(double *db, double *dx, void *data);
/* second kind (Saad, Iterative Methods, 2nd ed., p. 399), chebiter.c:204 */
void pEVSL_ChebIterSolv2(double *db, double *dx, void *data);
void pEVSL_ChebIterFree(void *vdata);                     /* chebiter.c:272 */
/* residual history: NULL, as the reference without SAVE_CONV_HIST */
double *pEVSL_ChebIterGetRes(void *data);                 /* chebiter.c:64  */
void pEVSL_ChebIterStatsPrint(void *data, FILE *fstats);  /* chebiter.c:287 */

#ifdef __cplusplus
}
#endif

#endif
