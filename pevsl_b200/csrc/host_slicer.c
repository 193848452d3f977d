/*
 * Spectrum slicing (host, scalar): cut [a,b] into slices of equal estimated
 * eigenvalue count, from KPM moments (SRC/spslicer.c) or from a Lanczos DOS
 * curve (SRC/landos.c:331-355, SRC/simpson.c).  The moments and the DOS curve
 * come from the GPU; these O(Mdeg * npts) loops stay on the host because
 * slice endpoints are grid points whose choice must match the reference.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "internal.h"

/* Uniform grid with exact end points (SRC/vector.c:15-25). */
void linspace(double a, double b, int num, double *arr) {
  const double h = num == 1 ? 0 : (b - a) / (num - 1);
  arr[0] = a;
  arr[num - 1] = b;
  for (int i = 1; i < num - 1; i++) arr[i] = a + i * h;
}

void pEVSL_LinSpace(double a, double b, int num, double *arr) { linspace(a, b, num, arr); }

/* yi[j] = integral of the KPM density sum_k mu_k T_k(t)/sqrt(1-t^2) from
 * xi[0] to xi[j], in closed form via t = cos(theta) (SRC/spslicer.c:12-38). */
static int kpm_cumulative(int Mdeg, const double *mu, int npts, const double *xi, double *yi) {
  if (npts <= 0) return PEVSL_ERR_ARG;
  double *th = (double *)calloc((size_t)npts, sizeof(double));
  if (!th) return PEVSL_ERR_NOMEM;
  for (int j = 0; j < npts; j++) th[j] = acos(xi[j]);
  const double th0 = th[0];
  for (int j = 0; j < npts; j++) yi[j] = mu[0] * (th0 - th[j]);
  for (int k = 1; k <= Mdeg; k++) {
    const double base = sin(k * th0) / k;
    for (int j = 0; j < npts; j++) yi[j] += mu[k] * (base - sin(k * th[j]) / k);
  }
  free(th);
  return 0;
}

/* Equal-count slices from KPM moments (SRC/spslicer.c:62-156).  Returns 0,
 * -1 (invalid interval), 1 (ran out of grid), +2 (endpoints not monotone). */
int pEVSL_SpslicerKpm(double *sli, double *mu, int Mdeg, double *intv, int n_int, int npts) {
  if (pevsl_check_intv(intv, stdout) < 0) return -1;
  const double aa = PEVSL_MAX(intv[0], intv[2]), bb = PEVSL_MIN(intv[1], intv[3]);
  if (intv[0] < intv[2] || intv[1] > intv[3]) {
    fprintf(stdout, " warning: interval (%e, %e) is adjusted to (%e, %e)\n", intv[0], intv[1],
            aa, bb);
  }
  memset(sli, 0, (size_t)(n_int + 1) * sizeof(double));
  if (n_int == 1) {
    sli[0] = intv[0];
    sli[1] = intv[1];
    return 0;
  }
  const double ctr = (intv[3] + intv[2]) / 2, wid = (intv[3] - intv[2]) / 2;
  const double aL = PEVSL_MAX((aa - ctr) / wid, -1.0), bL = PEVSL_MIN((bb - ctr) / wid, 1.0);
  npts = PEVSL_MAX(npts, 2 * n_int + 1);
  double *xi = (double *)malloc((size_t)npts * sizeof(double));
  double *yi = (double *)malloc((size_t)npts * sizeof(double));
  if (!xi || !yi) {
    free(xi);
    free(yi);
    return PEVSL_ERR_NOMEM;
  }
  linspace(aL, bL, npts, xi);
  kpm_cumulative(Mdeg, mu, npts, xi, yi);
  /* walk the grid: each slice ends at the grid point nearest its target
   * share, and the remaining mass is re-split over the remaining slices */
  double target = yi[npts - 1] / (double)n_int;
  int ls = 0, ii = 0;
  sli[0] = intv[0];
  while (++ls < n_int) {
    while (ii < npts && yi[ii] < target) ii++;
    if (ii == npts) break;
    /* ii > 0: when the first grid point already reaches the target (a
     * moment set whose mass is not positive) the reference compares with
     * yi[-1], outside its array; here that grid point is kept */
    if (ii > 0 && target - yi[ii - 1] < yi[ii] - target) ii--;
    sli[ls] = ctr + wid * xi[ii];
    target = yi[ii] + (yi[npts - 1] - yi[ii]) / (n_int - ls);
  }
  sli[n_int] = intv[1];
  int err = ls != n_int ? 1 : 0;
  for (int i = 1; i <= n_int; i++) {
    if (sli[i] < sli[i - 1]) {
      err += 2;
      break;
    }
  }
  free(xi);
  free(yi);
  return err;
}

/* In-place running integral of yi over the grid xi: Simpson on each pair of
 * panels, trapezoid for the odd point and a trailing panel
 * (SRC/simpson.c:20-45). */
void pevsl_simpson(const double *xi, double *yi, int npts) {
  double acc = 0.0, held = yi[0];
  int i = 1;
  yi[0] = 0;
  while (i < npts - 1) {
    const double trap = (xi[i] - xi[i - 1]) * (held + yi[i]) / 2.0;
    const double mid = acc + trap;
    acc += (xi[i + 1] - xi[i - 1]) * (held + 4 * yi[i] + yi[i + 1]) / 6.0;
    yi[i] = mid;
    held = yi[i + 1];
    yi[i + 1] = acc;
    i += 2;
  }
  if (i == npts - 1) yi[i] = acc + (xi[i] - xi[i - 1]) * (yi[i] + held) / 2.0;
}

/* Equal-area slices of a sampled DOS (SRC/landos.c:331-355). */
void pEVSL_SpslicerLan(double *xi, double *yi, int n_int, int npts, double *sli) {
  pevsl_simpson(xi, yi, npts);
  double last = yi[0];
  const double want = (yi[npts - 1] - yi[0]) / (double)n_int;
  int ls = 0;
  sli[0] = xi[0];
  for (int k = 1; k < npts; k++) {
    if (yi[k] - last >= want) {
      ls++;
      if (ls <= n_int) sli[ls] = xi[k]; /* rounding can add a crossing past the end */
      last = yi[k];
    }
  }
  sli[n_int] = xi[npts - 1];
}
