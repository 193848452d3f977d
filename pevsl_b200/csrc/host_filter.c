/*
 * Polynomial filter design (host, scalar): the Chebyshev "delta-like" filter
 * of every slice and the damping factors shared with the KPM moments.
 * Same arithmetic as SRC/chebpol.c of the reference, so that degree, gam,
 * bar and coefficients agree to the last bit or two; the filter APPLICATION
 * (pEVSL_ChebAv) runs on the GPU (kernels_filter.cu).
 */
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "internal.h"

/* Defaults of a filter request (SRC/chebpol.c:10-19). */
void pEVSL_SetPolDef(pevsl_Polparams *pol) {
  pol->max_deg = 5000;
  pol->min_deg = 2;
  pol->damping = 2;
  pol->thresh_ext = 0.20;
  pol->thresh_int = 0.8;
  pol->mu = NULL;
  pol->deg = 0;
  pol->intvtol = 1e-9;
}

void pEVSL_FreePol(pevsl_Polparams *pol) {
  free(pol->mu);
  pol->mu = NULL;
}

/* Damping of a degree-m Chebyshev expansion (SRC/chebpol.c:34-61):
 * 0 none, 1 Jackson, 2 Lanczos sigma; jac[0] is 1/2 (the halved first term). */
void pevsl_dampcf(int m, int damping, double *jac) {
  const double dm = (double)m;
  double thetJ = 0.0, a1 = 0.0, a2 = 0.0, thetL = 0.0;
  if (damping == 1) {
    thetJ = M_PI / (dm + 2);
    a1 = 1 / (dm + 2);
    a2 = sin(thetJ);
  } else if (damping == 2) {
    thetL = M_PI / (dm + 1);
  }
  jac[0] = 0.5;
  for (int k = 1; k <= m; k++) {
    switch (damping) {
      case 0:
        jac[k] = 1.0;
        break;
      case 1: {
        const int k1 = k + 1;
        jac[k] = a1 * sin(k1 * thetJ) / a2 + (1 - k1 * a1) * cos(k * thetJ);
        break;
      }
      default:
        jac[k] = sin(k * thetL) / (k * thetL);
    }
  }
}

/* p(x) = sum_k mu[k] T_k(x) at npts points in [-1,1] by the three-term
 * recurrence (SRC/chebpol.c:100-131). */
void pevsl_chebxPltd(int m, const double *mu, int npts, const double *xi, double *yi) {
  double *buf = (double *)malloc((size_t)3 * (size_t)(npts > 0 ? npts : 1) * sizeof(double));
  double *tprev = buf, *tcur = buf + npts, *tnext = buf + 2 * npts;
  for (int j = 0; j < npts; j++) {
    tprev[j] = 0.0;
    tcur[j] = 1.0;
    yi[j] = mu[0];
  }
  for (int k = 0; k < m; k++) {
    const double two = k == 0 ? 1.0 : 2.0;
    for (int j = 0; j < npts; j++) tnext[j] = two * xi[j] * tcur[j] - tprev[j];
    double *r = tprev;
    tprev = tcur;
    tcur = tnext;
    tnext = r;
    for (int j = 0; j < npts; j++) yi[j] += mu[k + 1] * tcur[j];
  }
  free(buf);
}

/* End-interval filter (SRC/chebpol.c:166-255): the Chebyshev polynomial of
 * [a,b] (the part to damp) scaled to 1 at the outer spectrum end gam, kept in
 * the T_k basis of [-1,1] by a three-term recurrence on coefficient vectors;
 * the degree grows until p(x) drops below thresh_ext at the inner end x. */
static void end_interval_filter(pevsl_Polparams *pol, double aIn, double bIn) {
  int max_deg = pol->max_deg;
  double thresh = pol->thresh_ext;
  if (pol->deg > 0) { /* forced degree */
    thresh = -1.0;
    max_deg = pol->deg;
  }
  const double del = 0.1 * sqrt((bIn - aIn) * 0.5);
  double a, b, x, gam;
  if (bIn >= 1.0 - 1e-13) { /* right end of the spectrum */
    x = aIn;
    b = x - del;
    a = -1.0;
    gam = 1.0;
  } else { /* left end */
    x = bIn;
    a = x + del;
    b = 1.0;
    gam = -1.0;
  }
  const double e = (b - a) * 0.5, c = (b + a) * 0.5;
  const double sigma1 = e / (gam - c);
  double sigma = sigma1;
  const int m1 = max_deg + 1;
  double *coef = (double *)calloc((size_t)3 * (size_t)m1, sizeof(double));
  double *c0 = coef, *c1 = coef + m1, *cn = coef + 2 * m1;
  c0[0] = 1.0;
  c1[0] = -c * (sigma1 / e);
  c1[1] = sigma1 / e;
  double g0 = 1.0, g1 = (x - c) * sigma1 / e;
  int best = 0;
  if (g1 < thresh) {
    best = 1;
  } else {
    for (int k = 2; k <= max_deg; k++) {
      const double sigma_new = 1.0 / (2.0 / sigma1 - sigma);
      const double s1 = sigma_new / e, s2 = 2 * s1 * c, s3 = sigma * sigma_new;
      /* x T_j = (T_{j+1} + T_{j-1}) / 2, applied to the coefficients of c1 */
      for (int j = 2; j <= k; j++) cn[j - 1] = s1 * (c1[j] + c1[j - 2]);
      cn[1] = cn[1] + s1 * c1[0];
      cn[0] = s1 * c1[1];
      cn[k] = s1 * c1[k - 1];
      for (int j = 0; j <= k; j++) cn[j] = cn[j] - s2 * c1[j] - s3 * c0[j];
      for (int j = 0; j <= k; j++) {
        c0[j] = c1[j];
        c1[j] = cn[j];
      }
      const double gn = 2 * (x - c) * s1 * g1 - s3 * g0;
      g0 = g1;
      g1 = gn;
      best = k;
      if (g1 < thresh) break;
      sigma = sigma_new;
    }
  }
  memcpy(pol->mu, c1, (size_t)(best + 1) * sizeof(double));
  pol->deg = best;
  pol->bar = g1;
  pol->gam = gam;
  free(coef);
}

/* sum_j v[j] cos(j th) jac[j]: difference p(b) - p(a) of the balanced filter
 * as a function of the centre angle (SRC/chebpol.c:73-79). */
static double balance_fn(const double *v, int m, double th, const double *jac) {
  double f = 0.0;
  for (int j = 0; j <= m; j++) f += v[j] * cos(j * th) * jac[j];
  return f;
}

/* Centre angle thc making p(a) = p(b) (SRC/chebpol.c:284-332): safeguarded
 * Newton on balance_fn inside [thb, tha]; returns 1 if the sign condition
 * fails (degree too low), else writes mu[j] = cos(j thc) jac[j]. */
static int balance_centre(int m, const double *v, const double *jac, double tha, double thb,
                          double *mu, double *thc_out) {
  const double tolBal = fabs(tha - thb) * 1.e-13;
  double thc = 0.5 * (tha + thb);
  const double fb = balance_fn(v, m, thb, jac), fa = balance_fn(v, m, tha, jac);
  if (fa > 0 || fb < 0) return 1;
  for (int it = 0; it <= 30; it++) {
    const double f = balance_fn(v, m, thc, jac);
    double d = 0.0;
    for (int j = 1; j <= m; j++) d += jac[j] * j * sin(j * thc) * v[j];
    double thN = thc + f / d;
    if (fabs(f) < tolBal || fabs(thc - thN) < DBL_EPSILON * fabs(thc)) break;
    if (f > 0) {
      if (thN < thb || thN > tha) thN = 0.5 * (thc + tha);
      thb = thc;
    } else {
      if (thN < thb || thN > tha) thN = 0.5 * (thc + thb);
      tha = thc;
    }
    thc = thN;
  }
  for (int j = 0; j <= m; j++) mu[j] = cos(j * thc) * jac[j];
  *thc_out = thc;
  return 0;
}

/* Filter for the slice [intv0, intv1] of the spectrum [intv2, intv3]
 * (SRC/chebpol.c:359-484).  Returns -1 for an invalid interval, and
 * PEVSL_ERR_ARG when max_deg (or the forced degree) is 2 or less, which
 * leaves no degree to search (the reference then scales by t = 0).
 *
 * The degree search starts at 2 for every slice.  The reference writes its
 * start as 2 + (int) 0.5/(bb-aa) (SRC/chebpol.c:434), where the cast
 * applies to 0.5 alone, so its value is 2; the search here starts there too,
 * which gives the reference's degree whenever a degree below
 * 2 + 0.5/(bb-aa) already meets the threshold. */
int pEVSL_FindPol(double *intv, pevsl_Polparams *pol) {
  if (pevsl_check_intv(intv, stdout) < 0) return -1;
  int max_deg = pol->max_deg;
  const int cap = PEVSL_MAX(pol->max_deg, pol->deg) + 1;
  double *mu = (double *)malloc((size_t)cap * sizeof(double));
  double *v = (double *)malloc((size_t)cap * sizeof(double));
  double *jac = (double *)malloc((size_t)cap * sizeof(double));
  if (!mu || !v || !jac) {
    free(mu);
    free(v);
    free(jac);
    return PEVSL_ERR_NOMEM;
  }
  pol->mu = mu;
  double aa = PEVSL_MAX(intv[0], intv[2]), bb = PEVSL_MIN(intv[1], intv[3]);
  if (intv[0] < intv[2] || intv[1] > intv[3]) {
    fprintf(stdout, " warning: interval (%e, %e) is adjusted to (%e, %e)\n", intv[0], intv[1],
            aa, bb);
  }
  const double lmin = intv[2], lmax = intv[3];
  const double cc = 0.5 * (lmax + lmin), dd = 0.5 * (lmax - lmin);
  pol->cc = cc;
  pol->dd = dd;
  aa = PEVSL_MAX((aa - cc) / dd, -1.0);
  bb = PEVSL_MIN((bb - cc) / dd, 1.0);
  const double thb = acos(bb), tha = acos(aa);
  const double IntTol = pol->intvtol;
  if (aa - IntTol <= -1.0) {
    pol->type = 1;
    end_interval_filter(pol, -1.0, bb);
  } else if (bb + IntTol >= 1.0) {
    pol->type = 2;
    end_interval_filter(pol, aa, 1.0);
  } else {
    pol->type = 0;
    const double ends[2] = {aa, bb};
    double vals[2] = {0.0, 0.0}, t = 0.0, thc = 0.0, gam = 0.0;
    double thresh = pol->thresh_int;
    const int min_deg = 2;
    if (pol->deg > 0) {
      thresh = -1;
      max_deg = pol->deg;
    }
    if (max_deg <= min_deg) {
      fprintf(stdout, " FindPol: degree limit %d leaves no degree to search\n", max_deg);
      free(mu);
      free(v);
      free(jac);
      pol->mu = NULL;
      return PEVSL_ERR_ARG;
    }
    for (int j = 0; j < min_deg; j++) v[j] = cos(j * thb) - cos(j * tha);
    int m;
    for (m = min_deg; m < max_deg; m++) {
      pevsl_dampcf(m, pol->damping, jac);
      v[m] = cos(m * thb) - cos(m * tha);
      if (balance_centre(m, v, jac, tha, thb, mu, &thc)) continue;
      gam = cos(thc);
      pevsl_chebxPltd(m, mu, 1, &gam, &t);
      pevsl_chebxPltd(m, mu, 2, ends, vals);
      if (vals[0] <= t * thresh && vals[1] <= t * thresh) {
        m++;
        break;
      }
    }
    for (int j = 0; j <= m; j++) mu[j] /= t;
    pol->bar = PEVSL_MIN(vals[0], vals[1]) / t;
    pol->gam = gam;
    pol->deg = m - 1;
  }
  free(v);
  free(jac);
  return 0;
}
