/*
 * B-solver of the generalized-problem drivers (test infrastructure), for
 * both the reference build and this library: the Chebyshev iteration of
 * EXTERNAL/ITERSOL/pevsl_itsol.h (second kind) with degree 40 on the
 * spectrum enclosure [2, 6] of the driver's B, the 1D Laplacian with
 * diagonal 4 of TESTS/COMMON/lapl.c (Gershgorin: 4 -+ 2).  Its eigenvalues
 * lie inside (2, 6), so the error falls by at least
 * (sqrt(3) - 1) / (sqrt(3) + 1) = 0.27 per step: 40 steps solve to
 * rounding level.  The driver uses only the B-solve (its L^{-T} solve is
 * the library's least-squares polynomial).
 */
#include "pevsl.h"
#include "pevsl_direct.h"
#include "pevsl_itsol.h"

#define BSOL_LMIN 2.0
#define BSOL_LMAX 6.0
#define BSOL_DEG 40

int SetupBSolDirect(pevsl_Parcsr *B, void **data) {
  return pEVSL_ChebIterSetup(BSOL_LMIN, BSOL_LMAX, BSOL_DEG, B, data);
}

void BSolDirect(double *b, double *x, void *data) { pEVSL_ChebIterSolv2(b, x, data); }

void FreeBSolDirectData(void *data) { pEVSL_ChebIterFree(data); }
