/*
 * Least-squares Chebyshev approximation of a scalar function on an interval
 * [a, b] (host, scalar): the coefficients of the polynomial that
 * pEVSL_LSPolSol applies to B to approximate B^{-1} or B^{-1/2}
 * (SRC/lspolapprox.c:62-148).  The coefficients are Gauss-Chebyshev
 * quadratures of f on 4 max_deg nodes; the degree grows until the summed
 * relative error over 50 max_deg equispaced points of [-1, 1] falls below
 * tol.  The degree is a discrete output, so the arithmetic follows the
 * reference's order step by step.
 */
#include <math.h>
#include <stdlib.h>

#include "internal.h"

static double f_rec(double a) { return 1.0 / a; }
static double f_isqrt(double a) { return 1.0 / sqrt(a); }

int pevsl_lspol_coefs(double (*ffun)(double), int max_deg, double tol, double a, double b,
                      double *mu, int *deg, double *cc, double *dd) {
  if (max_deg <= 0 || !(b > a) || !ffun || !mu || !deg) return PEVSL_ERR_ARG;
  const double c = (a + b) / 2, h = (b - a) / 2;
  const int npts = max_deg * 4, nrm_pts = 50 * max_deg;
  double *th = (double *)malloc(sizeof(double) * (size_t)npts);
  double *gi = (double *)malloc(sizeof(double) * (size_t)npts);
  double *xe = (double *)malloc(sizeof(double) * (size_t)nrm_pts);
  double *fe = (double *)malloc(sizeof(double) * (size_t)nrm_pts);
  double *pe = (double *)malloc(sizeof(double) * (size_t)nrm_pts);
  int st = (!th || !gi || !xe || !fe || !pe) ? PEVSL_ERR_NOMEM : 0;
  if (!st) {
    /* Chebyshev nodes cos((2j+1) pi / (2 npts)) and f there */
    for (int j = 0; j < npts; j++) th[j] = (2 * j + 1) * (M_PI / (2 * npts));
    for (int j = 0; j < npts; j++) gi[j] = ffun(c + h * cos(th[j]));
    linspace(-1, 1, nrm_pts, xe);
    for (int j = 0; j < nrm_pts; j++) fe[j] = ffun(c + h * xe[j]);
    const double w0 = 1.0 / npts, w1 = 2.0 / npts;
    int k;
    for (k = 0; k < max_deg; k++) {
      double sum = 0;
      for (int j = 0; j < npts; j++) sum += cos(k * th[j]) * gi[j];
      mu[k] = (k == 0 ? w0 : w1) * sum;
      pevsl_chebxPltd(k, mu, nrm_pts, xe, pe);
      double err = 0;
      for (int j = 0; j < nrm_pts; j++) err += fabs((pe[j] - fe[j]) / fe[j]);
      if (err < tol) {
        k++;
        break;
      }
    }
    *deg = k - 1; /* mu[0..k-1] */
    if (cc) *cc = c;
    if (dd) *dd = h;
  }
  free(th);
  free(gi);
  free(xe);
  free(fe);
  free(pe);
  return st;
}

/* coefficients of 1/x (kind 0) or 1/sqrt(x) (kind 1): a host-only entry
 * point for checking the approximation without a device */
int pEVSL_B200_LSPolCoefs(int kind, int max_deg, double tol, double lmin, double lmax, double *mu,
                          int *deg, double *cc, double *dd) {
  if (kind != 0 && kind != 1) return PEVSL_ERR_ARG;
  return pevsl_lspol_coefs(kind ? f_isqrt : f_rec, max_deg, tol, lmin, lmax, mu, deg, cc, dd);
}

double (*pevsl_lspol_rec(void))(double) { return f_rec; }
double (*pevsl_lspol_isqrt(void))(double) { return f_isqrt; }
