/*
 * Stand-in for the direct B-solver interface that TESTS/Gen_Lap/LapPLanN.c
 * includes (EXTERNAL/DIRECTSOL/pevsl_direct.h: MUMPS or PARDISO in the
 * reference).  Test infrastructure: bsol_cheb.c implements it with a
 * Chebyshev iteration of degree 40 on the driver's B, which solves to
 * rounding level, so the reference build and this library run the same
 * driver with the same B-solver.
 */
#ifndef PEVSL_DIRECT_H
#define PEVSL_DIRECT_H

int SetupBSolDirect(pevsl_Parcsr *B, void **data);
void BSolDirect(double *b, double *x, void *data);
void FreeBSolDirectData(void *data);

#endif
