/*
 * ORACLE — plain-C CPU restatement of pEVSL's spectrum-slicing path.
 *
 * TEST INFRASTRUCTURE ONLY.  The parity tests, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg use this file as the checker for the CUDA
 * path; the product library never links, loads or calls it.  It is pinned
 * against the reference itself (oracle/_ref, compiled from the reference's
 * own sources) by tests/test_oracle_pin.py and the fixtures in tests/golden/.
 *
 * Every routine restates one reference routine and cites it (paths are
 * relative to the reference project).  Scalar, single-threaded and written
 * for clarity: sums run in index order.  Third-party arithmetic that the
 * reference takes from LAPACK (DSTEV / DSYEV, SRC/miscla.c:29-66,161-198) is
 * restated from the published algorithms: the implicit symmetric tridiagonal
 * QR step with Wilkinson shift (Golub & Van Loan, Matrix Computations,
 * Alg. 8.3.2/8.3.3) and the cyclic Jacobi method for dense symmetric
 * matrices (Golub & Van Loan, Alg. 8.5.3).
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "philox_gauss.h"
#include "pipeline.h"

#define ORC_PI 3.14159265358979323846
#define ORC_ORTHTOL 1e-14 /* INC/pevsl_def.h:18 */
#define ORC_NGS_MAX 2     /* INC/pevsl_def.h:112 */

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static void *xcalloc(size_t n, size_t sz) {
  void *p = calloc(n ? n : 1, sz);
  if (!p) {
    fprintf(stderr, "oracle: out of memory\n");
    abort();
  }
  return p;
}

/* ------------------------------------------------------------------ BLAS1 */
static double dot(long n, const double *x, const double *y) {
  double s = 0.0;
  for (long i = 0; i < n; i++) s += x[i] * y[i];
  return s;
}
static double nrm2(long n, const double *x) { return sqrt(dot(n, x, x)); }
static void axpy(long n, double a, const double *x, double *y) {
  for (long i = 0; i < n; i++) y[i] += a * x[i];
}
static void scal(long n, double a, double *x) {
  for (long i = 0; i < n; i++) x[i] *= a;
}

/* ------------------------------------------------------------------ SpMV
 * y = A x, row loop of dcsrmv (SRC/spmat.c:184-194). */
void orc_matvec(int n, const int *ia, const int *ja, const double *a, const double *x, double *y) {
  for (int i = 0; i < n; i++) {
    double r = 0.0;
    for (int j = ia[i]; j < ia[i + 1]; j++) r += a[j] * x[ja[j]];
    y[i] = r;
  }
}

typedef struct {
  int n;
  const int *ia, *ja;
  const double *a;
} csr_t;

static void mv(const csr_t *A, const double *x, double *y) {
  orc_matvec(A->n, A->ia, A->ja, A->a, x, y);
}

/* ------------------------------------------------------------------ random vectors
 * glibc mode: (rand() - RAND_MAX/2) / (RAND_MAX/2) per element, as
 * pEVSL_ParvecRand (SRC/parvec.c:65-72); the stream is the C library's.
 * gauss mode: philox_gauss.h.  A draw counter numbers the vectors. */
static int g_mode = 0;
static uint64_t g_seed = 0, g_draw = 0;

void orc_set_rng(int mode, uint64_t seed) {
  g_mode = mode;
  g_seed = seed;
  g_draw = 0;
  srand((unsigned)seed);
}
uint64_t orc_rng_draws(void) { return g_draw; }

void orc_rand_vector(double *x, int n) {
  if (g_mode == 1) {
    orc_gauss_vector(x, n, g_seed, g_draw);
  } else {
    double t = ((double)RAND_MAX) / 2.0;
    for (int i = 0; i < n; i++) x[i] = (rand() - t) / t;
  }
  g_draw++;
}

/* ------------------------------------------------------------------ generators
 * 7-point (3D) / 5-point (nz == 1) Dirichlet Laplacian, rows in natural
 * order with ascending column indices: LocalLapGen (TESTS/COMMON/lapl.c:4-70).
 * ia needs n+1 entries, ja/a need 7n (3D) or 5n (2D); returns nnz. */
int orc_lap3(int nx, int ny, int nz, int *ia, int *ja, double *a) {
  int n = nx * ny * nz, nnz = 0;
  double d = nz > 1 ? 6.0 : 4.0;
  ia[0] = 0;
  for (int ii = 0; ii < n; ii++) {
    int k = ii / (nx * ny);
    int i = (ii - k * nx * ny) / nx;
    int j = ii - k * nx * ny - i * nx;
    if (k > 0) { ja[nnz] = ii - nx * ny; a[nnz++] = -1.0; }
    if (i > 0) { ja[nnz] = ii - nx; a[nnz++] = -1.0; }
    if (j > 0) { ja[nnz] = ii - 1; a[nnz++] = -1.0; }
    ja[nnz] = ii; a[nnz++] = d;
    if (j < nx - 1) { ja[nnz] = ii + 1; a[nnz++] = -1.0; }
    if (i < ny - 1) { ja[nnz] = ii + nx; a[nnz++] = -1.0; }
    if (k < nz - 1) { ja[nnz] = ii + nx * ny; a[nnz++] = -1.0; }
    ia[ii + 1] = nnz;
  }
  return nnz;
}

static int cmp_double(const void *p, const void *q) {
  double a = *(const double *)p, b = *(const double *)q;
  return a < b ? -1 : (a > b ? 1 : 0);
}

/* Analytic Laplacian eigenvalues in [a-eps, b+eps], ascending:
 * ExactEigLap3 (TESTS/COMMON/lapl.c:139-169).  out needs room for all n;
 * returns the count. */
int orc_exact_eig_lap3(int nx, int ny, int nz, double a, double b, double *out) {
  double thx = 0.5 * ORC_PI / (nx + 1.0), thy = 0.5 * ORC_PI / (ny + 1.0),
         thz = 0.5 * ORC_PI / (nz + 1.0);
  int l = 0;
  for (int i = 1; i <= nx; i++) {
    double tx = sin(i * thx);
    for (int j = 1; j <= ny; j++) {
      double ty = sin(j * thy);
      for (int k = 1; k <= nz; k++) {
        double tz = nz == 1 ? 0.0 : sin(k * thz);
        double ev = 4 * (tx * tx + ty * ty + tz * tz);
        if (ev >= a - DBL_EPSILON && ev <= b + DBL_EPSILON) out[l++] = ev;
      }
    }
  }
  qsort(out, (size_t)l, sizeof(double), cmp_double);
  return l;
}

/* ------------------------------------------------------------------ eigensolvers */

/* Eigen-decomposition of the symmetric tridiagonal matrix with diagonal
 * d[0..n) and off-diagonal e[0..n-1) (the job of DSTEV in SymmTridEig,
 * SRC/miscla.c:29-66).  Implicit QR sweeps with a Wilkinson shift chase a
 * bulge down each unreduced block; off-diagonals below
 * eps*(|d_i|+|d_i+1|) are set to zero.  On return w holds the eigenvalues in
 * ascending order and, if Z != NULL, Z (n x n, column major, ldz = n) the
 * matching orthonormal eigenvectors.  Returns 0, or 1 if a block did not
 * converge in 40 sweeps per eigenvalue. */
int orc_tridiag_eig(int n, const double *d_in, const double *e_in, double *w, double *Z) {
  if (n <= 0) return 0;
  double *d = w, *e = (double *)xcalloc((size_t)n, sizeof(double));
  memcpy(d, d_in, (size_t)n * sizeof(double));
  if (n > 1) memcpy(e, e_in, (size_t)(n - 1) * sizeof(double));
  if (Z) {
    memset(Z, 0, (size_t)n * (size_t)n * sizeof(double));
    for (int i = 0; i < n; i++) Z[(size_t)i * n + i] = 1.0;
  }
  int q = n - 1, sweeps = 0, status = 0;
  while (q > 0) {
    for (int i = 0; i < q; i++) {
      if (fabs(e[i]) <= DBL_EPSILON * (fabs(d[i]) + fabs(d[i + 1]))) e[i] = 0.0;
    }
    if (e[q - 1] == 0.0) {
      q--;
      continue;
    }
    int p = q - 1;
    while (p > 0 && e[p - 1] != 0.0) p--;
    if (++sweeps > 40 * n) {
      status = 1;
      break;
    }
    /* Wilkinson shift from the trailing 2x2 block of rows q-1, q */
    double dl = 0.5 * (d[q - 1] - d[q]);
    double b = e[q - 1];
    double den = dl + (dl >= 0.0 ? 1.0 : -1.0) * hypot(dl, b);
    double mu = d[q] - b * b / den;
    double x = d[p] - mu, z = e[p], bulge = 0.0;
    for (int k = p; k < q; k++) {
      double r = hypot(x, z), c, s;
      if (r == 0.0) {
        c = 1.0;
        s = 0.0;
      } else {
        c = x / r;
        s = z / r;
      }
      if (k > p) e[k - 1] = r;
      double a0 = d[k], b0 = e[k], a1 = d[k + 1];
      d[k] = a0 * c * c + 2.0 * b0 * c * s + a1 * s * s;
      d[k + 1] = a0 * s * s - 2.0 * b0 * c * s + a1 * c * c;
      e[k] = (a1 - a0) * c * s + b0 * (c * c - s * s);
      if (k + 1 < q) {
        double f = e[k + 1];
        bulge = s * f;
        e[k + 1] = c * f;
      }
      if (Z) {
        double *zk = Z + (size_t)k * n, *zk1 = Z + (size_t)(k + 1) * n;
        for (int i = 0; i < n; i++) {
          double u = zk[i], v = zk1[i];
          zk[i] = c * u + s * v;
          zk1[i] = -s * u + c * v;
        }
      }
      x = e[k];
      z = bulge;
    }
  }
  free(e);
  /* ascending order, eigenvectors follow their eigenvalues */
  for (int i = 0; i < n - 1; i++) {
    int m = i;
    for (int j = i + 1; j < n; j++)
      if (d[j] < d[m]) m = j;
    if (m != i) {
      double t = d[i];
      d[i] = d[m];
      d[m] = t;
      if (Z) {
        for (int r = 0; r < n; r++) {
          double u = Z[(size_t)i * n + r];
          Z[(size_t)i * n + r] = Z[(size_t)m * n + r];
          Z[(size_t)m * n + r] = u;
        }
      }
    }
  }
  return status;
}

/* Eigen-decomposition of a dense symmetric n x n matrix A (lda), the job of
 * DSYEV in SymEigenSolver (SRC/miscla.c:161-198): cyclic Jacobi rotations
 * until the off-diagonal mass is below eps^2 of the total.  Q (ldq) gets the
 * eigenvectors (columns), lam the eigenvalues, ascending. */
void orc_symeig(int n, const double *A, int lda, double *Q, int ldq, double *lam) {
  double *S = (double *)xcalloc((size_t)n * n, sizeof(double));
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) S[(size_t)j * n + i] = A[(size_t)j * lda + i];
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) Q[(size_t)j * ldq + i] = (i == j);
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0, tot = 0.0;
    for (int j = 0; j < n; j++)
      for (int i = 0; i < n; i++) {
        double v = S[(size_t)j * n + i] * S[(size_t)j * n + i];
        tot += v;
        if (i != j) off += v;
      }
    if (off <= DBL_EPSILON * DBL_EPSILON * tot) break;
    for (int p = 0; p < n - 1; p++) {
      for (int q = p + 1; q < n; q++) {
        double apq = S[(size_t)q * n + p];
        if (apq == 0.0) continue;
        double app = S[(size_t)p * n + p], aqq = S[(size_t)q * n + q];
        double theta = (aqq - app) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; k++) { /* columns p, q */
          double skp = S[(size_t)p * n + k], skq = S[(size_t)q * n + k];
          S[(size_t)p * n + k] = c * skp - s * skq;
          S[(size_t)q * n + k] = s * skp + c * skq;
        }
        for (int k = 0; k < n; k++) { /* rows p, q */
          double spk = S[(size_t)k * n + p], sqk = S[(size_t)k * n + q];
          S[(size_t)k * n + p] = c * spk - s * sqk;
          S[(size_t)k * n + q] = s * spk + c * sqk;
        }
        for (int k = 0; k < n; k++) {
          double qkp = Q[(size_t)p * ldq + k], qkq = Q[(size_t)q * ldq + k];
          Q[(size_t)p * ldq + k] = c * qkp - s * qkq;
          Q[(size_t)q * ldq + k] = s * qkp + c * qkq;
        }
      }
    }
  }
  for (int i = 0; i < n; i++) lam[i] = S[(size_t)i * n + i];
  free(S);
  for (int i = 0; i < n - 1; i++) {
    int m = i;
    for (int j = i + 1; j < n; j++)
      if (lam[j] < lam[m]) m = j;
    if (m != i) {
      double t = lam[i];
      lam[i] = lam[m];
      lam[m] = t;
      for (int r = 0; r < n; r++) {
        double u = Q[(size_t)i * ldq + r];
        Q[(size_t)i * ldq + r] = Q[(size_t)m * ldq + r];
        Q[(size_t)m * ldq + r] = u;
      }
    }
  }
}

/* ------------------------------------------------------------------ reorthogonalisation
 * Classical Gram-Schmidt against the first k columns of V (n x k, ld) with
 * the DGKS test: at most NGS_MAX passes, stop once the norm kept more than
 * 1/sqrt(2) of the previous one.  CGS_DGKS (SRC/miscla.c:211-240). */
static double cgs_dgks(int n, int k, const double *V, long ld, double *v, double *w) {
  double eta = 1.0 / sqrt(2.0), old_nrm = nrm2(n, v), new_nrm = old_nrm;
  for (int it = 0; it < ORC_NGS_MAX; it++) {
    for (int j = 0; j < k; j++) w[j] = dot(n, V + (size_t)j * ld, v);
    for (int j = 0; j < k; j++) axpy(n, -w[j], V + (size_t)j * ld, v);
    new_nrm = nrm2(n, v);
    if (new_nrm > eta * old_nrm) break;
    old_nrm = new_nrm;
  }
  return new_nrm;
}

/* ------------------------------------------------------------------ filter design */

/* Damping factors jac[0..m]: none / Jackson / Lanczos sigma, with jac[0]
 * halved for the first Chebyshev term.  dampcf (SRC/chebpol.c:34-61). */
void orc_dampcf(int m, int damping, double *jac) {
  double dm = (double)m, thetJ = 0, thetL = 0, a1 = 0, a2 = 0;
  if (damping == 1) {
    thetJ = ORC_PI / (dm + 2);
    a1 = 1 / (dm + 2);
    a2 = sin(thetJ);
  }
  if (damping == 2) thetL = ORC_PI / (dm + 1);
  jac[0] = 0.5;
  for (int k = 1; k <= m; k++) {
    if (damping == 0) {
      jac[k] = 1.0;
    } else if (damping == 1) {
      int k1 = k + 1;
      jac[k] = a1 * sin(k1 * thetJ) / a2 + (1 - k1 * a1) * cos(k * thetJ);
    } else {
      jac[k] = sin(k * thetL) / (k * thetL);
    }
  }
}

/* yi = sum_k mu[k] T_k(xi) by the three-term recurrence.
 * chebxPltd (SRC/chebpol.c:100-131). */
void orc_chebxPltd(int m, const double *mu, int npts, const double *xi, double *yi) {
  double *vkm1 = (double *)xcalloc((size_t)npts, sizeof(double));
  double *vk = (double *)xcalloc((size_t)npts, sizeof(double));
  double *vkp1 = (double *)xcalloc((size_t)npts, sizeof(double));
  for (int j = 0; j < npts; j++) {
    vk[j] = 1.0;
    yi[j] = mu[0];
  }
  for (int k = 0; k < m; k++) {
    double sc = k == 0 ? 1.0 : 2.0;
    for (int j = 0; j < npts; j++) vkp1[j] = sc * xi[j] * vk[j] - vkm1[j];
    double *t = vkm1;
    vkm1 = vk;
    vk = vkp1;
    vkp1 = t;
    for (int j = 0; j < npts; j++) yi[j] += mu[k + 1] * vk[j];
  }
  free(vkm1);
  free(vk);
  free(vkp1);
}

typedef struct {
  int max_deg, min_deg, damping;
  double thresh_ext, thresh_int, intvtol;
  int type, deg;
  double *mu, cc, dd, gam, bar;
} orc_pol;

/* Defaults of pEVSL_SetPolDef (SRC/chebpol.c:10-19). */
static void pol_defaults(orc_pol *p) {
  p->max_deg = 5000;
  p->min_deg = 2;
  p->damping = 2;
  p->thresh_ext = 0.20;
  p->thresh_int = 0.8;
  p->mu = NULL;
  p->deg = 0;
  p->intvtol = 1e-9;
}

/* End-interval filter: a scaled Chebyshev polynomial expressed in the
 * Chebyshev basis, degree raised until p(x) < thresh.  chext
 * (SRC/chebpol.c:166-255). */
static void chext(orc_pol *pol, double aIn, double bIn) {
  int max_deg = pol->max_deg;
  double thresh = pol->thresh_ext, *mu = pol->mu;
  double del = 0.1 * sqrt((bIn - aIn) * 0.5), eps = 1e-13;
  double a, b, x, gam;
  if (pol->deg > 0) {
    thresh = -1.0;
    max_deg = pol->deg;
  }
  if (bIn >= (1.0 - eps)) {
    x = aIn;
    b = x - del;
    a = -1.0;
    gam = 1.0;
  } else {
    x = bIn;
    a = x + del;
    b = 1.0;
    gam = -1.0;
  }
  double e = (b - a) * 0.5, c = (b + a) * 0.5;
  double sigma1 = e / (gam - c), sigma = sigma1;
  int m1 = max_deg + 1, mbest = 0;
  double *t0 = (double *)xcalloc((size_t)3 * m1, sizeof(double));
  double *t1 = t0 + m1, *tnew = t1 + m1;
  t0[0] = 1.0;
  t1[0] = -c * (sigma1 / e);
  t1[1] = sigma1 / e;
  double g0 = 1.0, g1 = (x - c) * sigma1 / e;
  if (g1 < thresh) {
    mbest = 1;
  } else {
    for (int k = 2; k <= max_deg; k++) {
      double sigma_new = 1.0 / (2.0 / sigma1 - sigma);
      double s1 = sigma_new / e, s2 = 2 * s1 * c, s3 = sigma * sigma_new;
      for (int j = 2; j <= k; j++) tnew[j - 1] = s1 * (t1[j] + t1[j - 2]);
      tnew[1] = tnew[1] + s1 * t1[0];
      tnew[0] = s1 * t1[1];
      tnew[k] = s1 * t1[k - 1];
      for (int j = 0; j <= k; j++) tnew[j] = tnew[j] - s2 * t1[j] - s3 * t0[j];
      for (int j = 0; j <= k; j++) {
        t0[j] = t1[j];
        t1[j] = tnew[j];
      }
      double gnew = 2 * (x - c) * s1 * g1 - s3 * g0;
      g0 = g1;
      g1 = gnew;
      mbest = k;
      if (g1 < thresh) break;
      sigma = sigma_new;
    }
  }
  memcpy(mu, t1, (size_t)(mbest + 1) * sizeof(double));
  pol->deg = mbest;
  pol->bar = g1;
  pol->gam = gam;
  free(t0);
}

static double dif_eval(const double *v, int m, double thc, const double *jac) {
  double f = 0.0;
  for (int j = 0; j <= m; j++) f += v[j] * cos(j * thc) * jac[j];
  return f;
}

/* Newton (with bisection safeguard) for the angle thc that balances the
 * filter at both ends, then mu[j] = cos(j thc) jac[j].  rootchb
 * (SRC/chebpol.c:284-332); returns 1 when no balanced root exists. */
static int rootchb(int m, const double *v, const double *jac, double tha, double thb, double *mu,
                   double *thcOut) {
  double tolBal = fabs(tha - thb) * 1.e-13, thc = 0.5 * (tha + thb);
  double fb = dif_eval(v, m, thb, jac), fa = dif_eval(v, m, tha, jac);
  if ((fa > 0) || (fb < 0)) return 1;
  for (int it = 0; it <= 30; it++) {
    double fval = dif_eval(v, m, thc, jac), d = 0.0;
    for (int j = 1; j <= m; j++) d += jac[j] * j * sin(j * thc) * v[j];
    double thN = thc + fval / d;
    if ((fabs(fval) < tolBal) || fabs(thc - thN) < DBL_EPSILON * fabs(thc)) break;
    if (fval > 0) {
      if ((thN < thb) || (thN > tha)) thN = 0.5 * (thc + tha);
      thb = thc;
      thc = thN;
    } else {
      if ((thN < thb) || (thN > tha)) thN = 0.5 * (thc + thb);
      tha = thc;
      thc = thN;
    }
  }
  for (int j = 0; j <= m; j++) mu[j] = cos(j * thc) * jac[j];
  *thcOut = thc;
  return 0;
}

static int check_intv(const double *intv) {
  double a = intv[0], b = intv[1], lmin = intv[2], lmax = intv[3];
  if (a >= b) return -1;
  if (a >= lmax || b <= lmin) return -2;
  return 0;
}

/* Filter for [intv0, intv1] inside the spectrum bounds [intv2, intv3]:
 * pEVSL_FindPol (SRC/chebpol.c:359-484).  pol->mu is allocated here
 * (max_deg+1 entries); caller frees. */
static int findpol(const double *intv, orc_pol *pol) {
  int max_deg = pol->max_deg, min_deg, damping = pol->damping, m, mbest, nitv;
  double t = 0.0, itv[2], vals[2] = {0, 0}, tha, thb, thc = 0.0, gam = 0.0, thresh;
  if (check_intv(intv) < 0) return -1;
  double *mu = (double *)xcalloc((size_t)max_deg + 1, sizeof(double));
  pol->mu = mu;
  double *v = (double *)xcalloc((size_t)max_deg + 1, sizeof(double));
  double *jac = (double *)xcalloc((size_t)max_deg + 1, sizeof(double));
  double IntTol = pol->intvtol;
  double aa = intv[0] > intv[2] ? intv[0] : intv[2];
  double bb = intv[1] < intv[3] ? intv[1] : intv[3];
  double lmin = intv[2], lmax = intv[3];
  double cc = 0.5 * (lmax + lmin), dd = 0.5 * (lmax - lmin);
  pol->cc = cc;
  pol->dd = dd;
  aa = (aa - cc) / dd;
  bb = (bb - cc) / dd;
  aa = aa > -1.0 ? aa : -1.0;
  bb = bb < 1.0 ? bb : 1.0;
  thb = acos(bb);
  tha = acos(aa);
  if (aa - IntTol <= -1.0) {
    nitv = 1;
    aa = -1.0;
    pol->type = 1;
  } else if (bb + IntTol >= 1.0) {
    nitv = 1;
    bb = 1;
    pol->type = 2;
  } else {
    itv[0] = aa;
    itv[1] = bb;
    nitv = 2;
    pol->type = 0;
  }
  if (nitv == 1) {
    chext(pol, aa, bb);
  } else {
    /* SRC/chebpol.c:434 writes 2 + (int) 0.5/(bb-aa): the cast applies to
     * 0.5, so the search starts at degree 2 */
    min_deg = 2;
    thresh = pol->thresh_int;
    if (pol->deg > 0) {
      thresh = -1;
      max_deg = pol->deg;
    }
    for (int j = 0; j < min_deg; j++) v[j] = cos(j * thb) - cos(j * tha);
    for (m = min_deg; m < max_deg; m++) {
      orc_dampcf(m, damping, jac);
      v[m] = cos(m * thb) - cos(m * tha);
      if (rootchb(m, v, jac, tha, thb, mu, &thc)) continue;
      gam = cos(thc);
      orc_chebxPltd(m, mu, 1, &gam, &t);
      orc_chebxPltd(m, mu, nitv, itv, vals);
      if (vals[0] <= t * thresh && vals[1] <= t * thresh) {
        m++;
        break;
      }
    }
    mbest = m - 1;
    for (int j = 0; j <= m; j++) mu[j] /= t;
    pol->bar = (vals[0] < vals[1] ? vals[0] : vals[1]) / t;
    pol->gam = gam;
    pol->deg = mbest;
  }
  free(v);
  free(jac);
  return 0;
}

/* Flat-argument form of findpol for the tests (mirrors oref_findpol). */
int orc_findpol(const double *intv, int max_deg, int damping, double thresh_int,
                double thresh_ext, int deg_in, int *type, int *deg, double *gam, double *bar,
                double *cc, double *dd, double *mu_out) {
  orc_pol pol;
  pol_defaults(&pol);
  pol.damping = damping;
  pol.thresh_int = thresh_int;
  pol.thresh_ext = thresh_ext;
  pol.max_deg = max_deg;
  pol.deg = deg_in;
  int ierr = findpol(intv, &pol);
  if (ierr) return ierr;
  *type = pol.type;
  *deg = pol.deg;
  *gam = pol.gam;
  *bar = pol.bar;
  *cc = pol.cc;
  *dd = pol.dd;
  memcpy(mu_out, pol.mu, (size_t)(pol.deg + 1) * sizeof(double));
  free(pol.mu);
  return 0;
}

/* ------------------------------------------------------------------ filter application
 * y = p((A - cc)/dd) v via the three-term recurrence with coefficients
 * mu[0..deg]; w is 3n of work.  pEVSL_ChebAv (SRC/chebpol.c:509-574). */
static void chebav(const csr_t *A, int deg, double cc, double dd, const double *mu,
                   const double *v, double *y, double *w) {
  int n = A->n;
  double *vk = w, *vkp1 = w + n, *vkm1 = w + 2 * (size_t)n, *tmp;
  double t1 = 1.0 / dd, t2 = 2.0 / dd;
  memcpy(vk, v, (size_t)n * sizeof(double));
  memcpy(y, vk, (size_t)n * sizeof(double));
  scal(n, mu[0], y);
  for (int k = 1; k <= deg; k++) {
    double t = k == 1 ? t1 : t2;
    mv(A, vk, vkp1);
    axpy(n, -cc, vk, vkp1);
    scal(n, t, vkp1);
    if (k > 1) axpy(n, -1.0, vkm1, vkp1);
    axpy(n, mu[k], vkp1, y);
    tmp = vkm1;
    vkm1 = vk;
    vk = vkp1;
    vkp1 = tmp;
  }
}

int orc_chebav(int n, const int *ia, const int *ja, const double *a, int deg, double cc,
               double dd, const double *mu, const double *v, double *y) {
  csr_t A = {n, ia, ja, a};
  double *w = (double *)xcalloc((size_t)3 * n, sizeof(double));
  chebav(&A, deg, cc, dd, mu, v, y, w);
  free(w);
  return 0;
}

/* ------------------------------------------------------------------ KPM density of states
 * Chebyshev moments mu[0..Mdeg] of the spectral density from nvec random
 * vectors, and the eigenvalue-count estimate for [intv0, intv1].
 * pEVSL_Kpmdos (SRC/kpmdos.c:36-197) with one group. */
static int kpmdos(const csr_t *A, int Mdeg, int damping, int nvec, const double *intv, double *mu,
                  double *ecnt) {
  int n = A->n;
  if (check_intv(intv) < 0) return -1;
  double aa = intv[0] > intv[2] ? intv[0] : intv[2];
  double bb = intv[1] < intv[3] ? intv[1] : intv[3];
  double ctr = (intv[3] + intv[2]) / 2.0, wid = (intv[3] - intv[2]) / 2.0, t;
  t = (aa - ctr) / wid;
  t = t > -1.0 + DBL_EPSILON ? t : -1.0 + DBL_EPSILON;
  double beta1 = acos(t);
  t = (bb - ctr) / wid;
  t = t < 1.0 - DBL_EPSILON ? t : 1.0 - DBL_EPSILON;
  double beta2 = acos(t);
  double *jac = (double *)xcalloc((size_t)Mdeg + 1, sizeof(double));
  orc_dampcf(Mdeg, damping, jac);
  jac[0] = 1.0;
  memset(mu, 0, (size_t)(Mdeg + 1) * sizeof(double));
  double tcnt = 0.0;
  double *buf = (double *)xcalloc((size_t)4 * n, sizeof(double));
  double *v = buf, *vkm1 = buf + n, *vk = buf + 2 * (size_t)n, *vkp1 = buf + 3 * (size_t)n, *tmp;
  for (int m = 0; m < nvec; m++) {
    orc_rand_vector(v, n);
    t = nrm2(n, v);
    scal(n, 1.0 / t, v);
    memcpy(vk, v, (size_t)n * sizeof(double));
    memset(vkm1, 0, (size_t)n * sizeof(double));
    mu[0] += jac[0];
    tcnt -= jac[0] * (beta2 - beta1);
    for (int k = 0; k < Mdeg; k++) {
      mv(A, vk, vkp1);
      double sc = (k == 0 ? 1.0 : 2.0) / wid;
      axpy(n, -ctr, vk, vkp1);
      scal(n, sc, vkp1);
      axpy(n, -1.0, vkm1, vkp1);
      tmp = vkm1;
      vkm1 = vk;
      vk = vkp1;
      vkp1 = tmp;
      int k1 = k + 1;
      t = dot(n, vk, v);
      t *= 2.0 * jac[k1];
      mu[k1] += t;
      tcnt -= t * (sin(k1 * beta2) - sin(k1 * beta1)) / k1;
    }
  }
  t = 1.0 / (((double)nvec) * ORC_PI);
  scal(Mdeg + 1, t, mu);
  tcnt *= t * ((double)n);
  *ecnt = tcnt;
  free(buf);
  free(jac);
  return 0;
}

int orc_kpmdos(int n, const int *ia, const int *ja, const double *a, int Mdeg, int damping,
               int nvec, const double *intv, double *mu, double *ecnt) {
  csr_t A = {n, ia, ja, a};
  return kpmdos(&A, Mdeg, damping, nvec, intv, mu, ecnt);
}

/* Integrals of the KPM density from xi[0] to xi[j]: intChx
 * (SRC/spslicer.c:12-38). */
static void intChx(int Mdeg, const double *mu, int npts, const double *xi, double *yi) {
  double *th = (double *)xcalloc((size_t)npts, sizeof(double));
  for (int j = 0; j < npts; j++) th[j] = acos(xi[j]);
  double th0 = th[0];
  for (int j = 0; j < npts; j++) yi[j] = mu[0] * (th0 - th[j]);
  for (int k = 1; k < Mdeg + 1; k++) {
    double val0 = sin(k * th0) / k;
    for (int j = 0; j < npts; j++) yi[j] += mu[k] * (val0 - sin(k * th[j]) / k);
  }
  free(th);
}

static void linspace(double a, double b, int num, double *arr) {
  double h = num == 1 ? 0 : (b - a) / (num - 1);
  arr[0] = a;
  arr[num - 1] = b;
  for (int i = 1; i < num - 1; i++) arr[i] = a + i * h;
}

/* Equal-count slicing of the KPM density on an npts grid:
 * pEVSL_SpslicerKpm (SRC/spslicer.c:62-156).  Returns 0, -1 (bad interval),
 * 1 (fewer slices found), +2 (non-monotone endpoints). */
int orc_spslicer_kpm(double *sli, const double *mu, int Mdeg, const double *intv, int n_int,
                     int npts) {
  if (check_intv(intv) < 0) return -1;
  double aa = intv[0] > intv[2] ? intv[0] : intv[2];
  double bb = intv[1] < intv[3] ? intv[1] : intv[3];
  memset(sli, 0, (size_t)(n_int + 1) * sizeof(double));
  if (n_int == 1) {
    sli[0] = intv[0];
    sli[1] = intv[1];
    return 0;
  }
  double ctr = (intv[3] + intv[2]) / 2, wid = (intv[3] - intv[2]) / 2;
  double aL = (aa - ctr) / wid, bL = (bb - ctr) / wid;
  aL = aL > -1.0 ? aL : -1.0;
  bL = bL < 1.0 ? bL : 1.0;
  npts = npts > 2 * n_int + 1 ? npts : 2 * n_int + 1;
  double *xi = (double *)xcalloc((size_t)npts, sizeof(double));
  double *yi = (double *)xcalloc((size_t)npts, sizeof(double));
  linspace(aL, bL, npts, xi);
  intChx(Mdeg, mu, npts, xi, yi);
  double target = yi[npts - 1] / (double)n_int;
  int ls = 0, ii = 0, err = 0;
  sli[ls] = intv[0];
  while (++ls < n_int) {
    while (ii < npts && yi[ii] < target) ii++;
    if (ii == npts) break;
    if ((target - yi[ii - 1]) < (yi[ii] - target)) ii--;
    sli[ls] = ctr + wid * xi[ii];
    target = yi[ii] + (yi[npts - 1] - yi[ii]) / (n_int - ls);
  }
  sli[n_int] = intv[1];
  if (ls != n_int) err = 1;
  for (ii = 1; ii <= n_int; ii++) {
    if (sli[ii] < sli[ii - 1]) {
      err += 2;
      break;
    }
  }
  free(xi);
  free(yi);
  return err;
}

/* ------------------------------------------------------------------ Lanczos DOS */

/* In-place cumulative Simpson integration: simpson (SRC/simpson.c:20-45). */
void orc_simpson(const double *xi, double *yi, int npts) {
  double tc = 0.0, ti, tm, ysav = yi[0];
  int i = 1;
  yi[0] = 0;
  while (i < npts - 1) {
    ti = (xi[i] - xi[i - 1]) * (ysav + yi[i]) / 2.0;
    tm = tc + ti;
    ti = (xi[i + 1] - xi[i - 1]) * (ysav + 4 * yi[i] + yi[i + 1]) / 6.0;
    tc += ti;
    yi[i] = tm;
    ysav = yi[i + 1];
    yi[i + 1] = tc;
    i += 2;
  }
  if (i == npts - 1) {
    ti = (xi[i] - xi[i - 1]) * (yi[i] + ysav) / 2.0;
    yi[i] = tc + ti;
  }
}

/* Equal-area slicing of a sampled DOS curve: pEVSL_SpslicerLan
 * (SRC/landos.c:331-355). */
void orc_spslicer_lan(const double *xi, double *yi, int n_int, int npts, double *sli) {
  orc_simpson(xi, yi, npts);
  double t = yi[0], want = (yi[npts - 1] - yi[0]) / (double)n_int;
  int ls = 0;
  sli[0] = xi[0];
  for (int k = 1; k < npts; k++) {
    if (yi[k] - t >= want) {
      ls = ls + 1;
      sli[ls] = xi[k];
      t = yi[k];
    }
  }
  sli[n_int] = xi[npts - 1];
}

/* Lanczos-quadrature DOS: msteps Lanczos steps with full reorthogonalisation
 * per random vector, Gaussians of width sigma placed at the Ritz values and
 * weighted by the squared first eigenvector components.  pEVSL_LanDosG
 * (SRC/landos.c:40-314), standard problem, one group. */
static int landos(const csr_t *A, int nvec, int msteps, int npts, double *xdos, double *ydos,
                  double *neig, const double *intv, double sigma_mult) {
  int n = A->n, maxit = msteps < n ? msteps : n;
  double *y = (double *)xcalloc((size_t)npts, sizeof(double));
  int *ind = (int *)xcalloc((size_t)npts, sizeof(int));
  double *gamma2 = (double *)xcalloc((size_t)maxit, sizeof(double));
  double *V = (double *)xcalloc((size_t)n * (maxit + 1), sizeof(double));
  double *dT = (double *)xcalloc((size_t)maxit, sizeof(double));
  double *eT = (double *)xcalloc((size_t)maxit, sizeof(double));
  double *EvalT = (double *)xcalloc((size_t)maxit, sizeof(double));
  double *EvecT = (double *)xcalloc((size_t)maxit * maxit, sizeof(double));
  double *warr = (double *)xcalloc((size_t)3 * maxit, sizeof(double));
  double *vinit = (double *)xcalloc((size_t)n, sizeof(double));
  double lm = intv[2], lM = intv[3];
  double aa = intv[0] > intv[2] ? intv[0] : intv[2];
  double bb = intv[1] < intv[3] ? intv[1] : intv[3];
  double kappa = 1.25;
  int M = msteps < 30 ? msteps : 30;
  double H = (lM - lm) / (M - 1);
  double sigma = H / sqrt(8 * log(kappa)) * sigma_mult;
  double sigma2 = 2 * sigma * sigma;
  double width = sigma * sqrt(-2.0 * log(1e-08));
  linspace(aa, bb, npts, xdos);
  for (int m = 0; m < nvec; m++) {
    orc_rand_vector(vinit, n);
    double t = 1.0 / nrm2(n, vinit);
    memcpy(V, vinit, (size_t)n * sizeof(double));
    scal(n, t, V);
    double wn = 0.0, alpha, beta = 0.0;
    int nwn = 0;
    for (int k = 0; k < maxit; k++) {
      double *v = V + (size_t)k * n, *vnew = V + (size_t)(k + 1) * n;
      mv(A, v, vnew);
      if (k > 0) axpy(n, -beta, V + (size_t)(k - 1) * n, vnew);
      alpha = dot(n, v, vnew);
      dT[k] = alpha;
      wn += fabs(alpha);
      axpy(n, -alpha, v, vnew);
      beta = cgs_dgks(n, k + 1, V, n, vnew, warr);
      wn += 2.0 * beta;
      nwn += 3;
      if (beta * nwn < ORC_ORTHTOL * wn) {
        orc_rand_vector(vnew, n);
        beta = cgs_dgks(n, k + 1, V, n, vnew, warr);
        scal(n, 1.0 / beta, vnew);
        beta = 0.0;
      } else {
        scal(n, 1.0 / beta, vnew);
      }
      eT[k] = beta;
    }
    orc_tridiag_eig(maxit, dT, eT, EvalT, EvecT);
    for (int i = 0; i < maxit; i++) gamma2[i] = EvecT[(size_t)i * maxit] * EvecT[(size_t)i * maxit];
    for (int i = 0; i < maxit; i++) {
      double th = EvalT[i];
      int numPlaced = 0;
      for (int j = 0; j < npts; j++)
        if (fabs(xdos[j] - th) < width) ind[numPlaced++] = j;
      for (int j = 0; j < numPlaced; j++)
        y[ind[j]] += gamma2[i] * exp(-((xdos[ind[j]] - th) * (xdos[ind[j]] - th)) / sigma2);
    }
  }
  double scaling = 1.0 / (nvec * sqrt(sigma2 * ORC_PI));
  scal(npts, scaling, y);
  memcpy(ydos, y, (size_t)npts * sizeof(double));
  orc_simpson(xdos, y, npts);
  *neig = y[npts - 1] * n;
  free(y);
  free(ind);
  free(gamma2);
  free(V);
  free(dT);
  free(eT);
  free(EvalT);
  free(EvecT);
  free(warr);
  free(vinit);
  return 0;
}

int orc_landos(int n, const int *ia, const int *ja, const double *a, int nvec, int msteps,
               int npts, double *xdos, double *ydos, double *neig, const double *intv) {
  csr_t A = {n, ia, ja, a};
  return landos(&A, nvec, msteps, npts, xdos, ydos, neig, intv, 1.0);
}

/* ------------------------------------------------------------------ spectrum bounds
 * Thick-restart Lanczos keeping the two extreme Ritz pairs; bounds are the
 * extreme Ritz values widened by |beta * last eigenvector component|
 * (bndtype 1) or the Kato-Temple term (bndtype 2).  pEVSL_LanTrbounds
 * (SRC/lantrbnd.c:31-408), standard problem.  Returns 0, or -3 if the
 * Krylov dimension is too small (the reference exits the process there). */
static int lantrbounds(const csr_t *A, int lanm, int maxit, double tol, const double *vinit,
                       int bndtype, double *lammin, double *lammax) {
  int N = A->n, n = A->n;
  double lmin = 0.0, lmax = 0.0, t1, t2;
  lanm = lanm < N ? lanm : N;
  int lanm1 = lanm + 1;
  if (lanm == N) maxit = maxit < N ? maxit : N;
  size_t L = (size_t)lanm1;
  int it = 0, trlen = 0, min_inner_step = 5;
  double *V = (double *)xcalloc((size_t)n * L, sizeof(double));
  double *T = (double *)xcalloc(L * L, sizeof(double));
  double *Rval = (double *)xcalloc((size_t)lanm, sizeof(double));
  double *Rvec = (double *)xcalloc((size_t)2 * n, sizeof(double));
  double *EvecT = (double *)xcalloc(L * L, sizeof(double));
  double *warr = (double *)xcalloc((size_t)3 * lanm, sizeof(double));
  double s[3] = {0, 0, 0};
  int status = 0;
  memcpy(V, vinit, (size_t)n * sizeof(double));
  scal(n, 1.0 / nrm2(n, V), V);
#define VC(j) (V + (size_t)(j) * n)
  while (it < maxit) {
    double wn = 0.0, beta = 0.0;
    int nwn = 0;
    int k = trlen > 0 ? trlen + 1 : 0;
    if (k + min_inner_step > lanm1) {
      status = -3;
      break;
    }
    if (trlen > 0) {
      int k1 = k - 1;
      double *v = VC(k1), *vnew = VC(k1 + 1);
      mv(A, v, vnew);
      for (int i = 0; i < trlen; i++) {
        T[i * L + i] = Rval[i];
        wn += fabs(Rval[i]);
      }
      s[k1] = dot(n, v, vnew);
      for (int j = 0; j < k; j++) axpy(n, -s[j], VC(j), vnew);
      for (int i = 0; i < k1; i++) {
        T[trlen * L + i] = s[i];
        T[i * L + trlen] = s[i];
        wn += 2.0 * fabs(s[i]);
      }
      T[trlen * L + trlen] = s[k1];
      wn += fabs(s[k1]);
      beta = nrm2(n, vnew);
      wn += 2.0 * beta;
      nwn += 3 * k;
      if (beta * nwn < ORC_ORTHTOL * wn) {
        orc_rand_vector(vnew, n);
        beta = cgs_dgks(n, k, V, n, vnew, warr);
        scal(n, 1.0 / beta, vnew);
        beta = 0.0;
      } else {
        scal(n, 1.0 / beta, vnew);
      }
      T[k1 * L + k] = beta;
      T[k * L + k1] = beta;
    }
    int have_old = k > 0;
    double *zold = have_old ? VC(k - 1) : NULL;
    while (k < lanm && it < maxit) {
      k++;
      double *v = VC(k - 1), *vnew = VC(k);
      mv(A, v, vnew);
      it++;
      if (zold) axpy(n, -beta, zold, vnew);
      double alpha = dot(n, v, vnew);
      T[(k - 1) * L + (k - 1)] = alpha;
      wn += fabs(alpha);
      axpy(n, -alpha, v, vnew);
      beta = cgs_dgks(n, k, V, n, vnew, warr);
      wn += 2.0 * beta;
      nwn += 3;
      zold = v;
      if (beta * nwn < ORC_ORTHTOL * wn) {
        orc_rand_vector(vnew, n);
        beta = cgs_dgks(n, k, V, n, vnew, warr);
        scal(n, 1.0 / beta, vnew);
        beta = 0.0;
      } else {
        scal(n, 1.0 / beta, vnew);
      }
      T[k * L + (k - 1)] = beta;
      T[(k - 1) * L + k] = beta;
    }
    orc_symeig(k, T, lanm1, EvecT, lanm1, Rval);
    s[0] = beta * EvecT[k - 1];
    s[1] = beta * EvecT[(k - 1) * L + (k - 1)];
    if (bndtype <= 1) {
      t1 = fabs(s[0]);
      t2 = fabs(s[1]);
    } else {
      t1 = 2.0 * s[0] * s[0] / (Rval[1] - Rval[0]);
      t2 = 2.0 * s[1] * s[1] / (Rval[k - 1] - Rval[k - 2]);
    }
    lmin = Rval[0] - t1;
    lmax = Rval[k - 1] + t2;
    /* two Ritz vectors become the thick-restart set */
    for (int c = 0; c < 2; c++) {
      const double *y = EvecT + (c == 0 ? 0 : (size_t)(k - 1) * L);
      double *r = Rvec + (size_t)c * n;
      memset(r, 0, (size_t)n * sizeof(double));
      for (int j = 0; j < k; j++) axpy(n, y[j], VC(j), r);
    }
    trlen = 2;
    memcpy(VC(0), Rvec, (size_t)n * sizeof(double));
    memcpy(VC(1), Rvec + n, (size_t)n * sizeof(double));
    Rval[1] = Rval[k - 1];
    if (t1 + t2 < tol * (fabs(lmin) + fabs(lmax))) break;
    memset(T, 0, L * L * sizeof(double));
    memcpy(VC(trlen), VC(k), (size_t)n * sizeof(double));
  }
#undef VC
  *lammin = lmin;
  *lammax = lmax;
  free(V);
  free(T);
  free(Rval);
  free(Rvec);
  free(EvecT);
  free(warr);
  return status;
}

int orc_lantrbounds(int n, const int *ia, const int *ja, const double *a, int lanm, int maxit,
                    double tol, const double *vinit, int bndtype, double *lmin, double *lmax) {
  csr_t A = {n, ia, ja, a};
  return lantrbounds(&A, lanm, maxit, tol, vinit, bndtype, lmin, lmax);
}

/* ------------------------------------------------------------------ filtered Lanczos
 * Non-restarted Lanczos on p(A) with full CGS-DGKS reorthogonalisation, the
 * restricted-trace convergence test every 20 steps from step 30, Ritz
 * extraction for Ritz values of p(A) >= bar, and acceptance of pairs whose
 * Rayleigh quotient lies in [a, b] and whose residual is below tol.
 * pEVSL_ChebLanNr (SRC/cheblanNr.c:54-448), FILTER_VINIT = 1, standard
 * problem.  Accepted pairs: lam/res (and W columns, n x cap) in the order
 * they are found; *its = Lanczos steps taken.  Returns 0, -1 (|gam| > 1),
 * 2 (zero Ritz vector). */
static int cheblannr(const csr_t *A, const double *intv, int maxit, double tol,
                     const double *vinit, const orc_pol *pol, int *nevOut, int *its, double *lam,
                     double *res, double *W, int cap) {
  int N = A->n, n = A->n;
  maxit = maxit < N ? maxit : N;
  double bar = pol->bar, gamB = pol->gam;
  *nevOut = 0;
  *its = 0;
  if (check_intv(intv) < 0) return 0;
  double aa = intv[0], bb = intv[1];
  if (gamB > 1.0 || gamB < -1.0) return -1;
  int Ntest = 30, cycle = 20, k, kdim = 0, count = 0, nconv = 0;
  double *V = (double *)xcalloc((size_t)n * (maxit + 1), sizeof(double));
  double *dT = (double *)xcalloc((size_t)maxit, sizeof(double));
  double *eT = (double *)xcalloc((size_t)maxit, sizeof(double));
  double *EvalT = (double *)xcalloc((size_t)maxit, sizeof(double));
  double *wk = (double *)xcalloc((size_t)3 * n, sizeof(double));
  double *warr = (double *)xcalloc((size_t)3 * maxit, sizeof(double));
  double *vrand = (double *)xcalloc((size_t)n, sizeof(double));
  double *u = (double *)xcalloc((size_t)n, sizeof(double));
  double *wv = (double *)xcalloc((size_t)n, sizeof(double));
#define VC(j) (V + (size_t)(j) * n)
  chebav(A, pol->deg, pol->cc, pol->dd, pol->mu, vinit, VC(0), wk);
  scal(n, 1.0 / nrm2(n, VC(0)), VC(0));
  double wn = 0.0, tr0 = 0, tr1, alpha, beta = 0.0;
  int nwn = 0;
  for (k = 0; k < maxit; k++) {
    double *z = VC(k), *znew = VC(k + 1);
    chebav(A, pol->deg, pol->cc, pol->dd, pol->mu, z, znew, wk);
    if (k > 0) axpy(n, -beta, VC(k - 1), znew);
    alpha = dot(n, z, znew);
    dT[k] = alpha;
    wn += fabs(alpha);
    axpy(n, -alpha, z, znew);
    beta = cgs_dgks(n, k + 1, V, n, znew, warr);
    wn += 2.0 * beta;
    nwn += 3;
    if (beta * nwn < ORC_ORTHTOL * wn) {
      orc_rand_vector(vrand, n);
      chebav(A, pol->deg, pol->cc, pol->dd, pol->mu, vrand, znew, wk);
      beta = cgs_dgks(n, k + 1, V, n, znew, warr);
      scal(n, 1.0 / beta, znew);
      beta = 0.0;
    } else {
      scal(n, 1.0 / beta, znew);
    }
    eT[k] = beta;
    if ((k < Ntest || (k - Ntest) % cycle != 0) && k != maxit - 1) continue;
    kdim = k + 1;
    orc_tridiag_eig(kdim, dT, eT, EvalT, NULL);
    count = kdim;
    tr1 = 0;
    nconv = 0;
    for (int i = 0; i < count; i++) {
      if (EvalT[i] + 5 * DBL_EPSILON >= bar) {
        tr1 += EvalT[i];
        nconv++;
      }
    }
    if ((fabs(tr1 - tr0) < 2e-12) || (fabs(tr1) + fabs(tr0) < 1e-10)) break;
    tr0 = tr1;
  }
  *its = kdim;
  double *EvecT = (double *)xcalloc((size_t)kdim * kdim, sizeof(double));
  orc_tridiag_eig(kdim, dT, eT, EvalT, EvecT);
  int nev = 0, status = 0;
  for (int i = 0; i < count; i++) {
    if (EvalT[i] < bar) continue;
    const double *y = EvecT + (size_t)i * kdim;
    memset(u, 0, (size_t)n * sizeof(double));
    for (int j = 0; j < kdim; j++) axpy(n, y[j], VC(j), u);
    double t = nrm2(n, u);
    if (t == 0.0) {
      status = 2;
      break;
    }
    scal(n, 1.0 / t, u);
    mv(A, u, wv);
    t = dot(n, wv, u);
    if (t < aa - DBL_EPSILON || t > bb + DBL_EPSILON) continue;
    axpy(n, -t, u, wv);
    double r0 = nrm2(n, wv);
    if (r0 < tol) {
      if (nev < cap) {
        lam[nev] = t;
        res[nev] = r0;
        if (W) memcpy(W + (size_t)nev * n, u, (size_t)n * sizeof(double));
      }
      nev++;
    }
  }
#undef VC
  *nevOut = nev;
  free(V);
  free(dT);
  free(eT);
  free(EvalT);
  free(EvecT);
  free(wk);
  free(warr);
  free(vrand);
  free(u);
  free(wv);
  return status;
}

/* Sort pairs ascending by eigenvalue (sort_double with indices,
 * SRC/vector.c:85-104), carrying residuals and vectors. */
static void sort_pairs(int m, double *lam, double *res, double *W, int n) {
  for (int i = 0; i < m - 1; i++) {
    int b = i;
    for (int j = i + 1; j < m; j++)
      if (lam[j] < lam[b]) b = j;
    if (b != i) {
      double t = lam[i];
      lam[i] = lam[b];
      lam[b] = t;
      t = res[i];
      res[i] = res[b];
      res[b] = t;
      if (W) {
        for (int r = 0; r < n; r++) {
          t = W[(size_t)i * n + r];
          W[(size_t)i * n + r] = W[(size_t)b * n + r];
          W[(size_t)b * n + r] = t;
        }
      }
    }
  }
}

int orc_cheblannr(int n, const int *ia, const int *ja, const double *a, const double *intv,
                  int maxit, double tol, const double *vinit, int deg, int ptype, double gam,
                  double bar, double cc, double dd, const double *mu, int *nev, int *its,
                  double *lam, double *res, double *W, int cap) {
  csr_t A = {n, ia, ja, a};
  orc_pol pol;
  pol_defaults(&pol);
  pol.deg = deg;
  pol.type = ptype;
  pol.gam = gam;
  pol.bar = bar;
  pol.cc = cc;
  pol.dd = dd;
  pol.mu = (double *)mu;
  int st = cheblannr(&A, intv, maxit, tol, vinit, &pol, nev, its, lam, res, W, cap);
  sort_pairs(*nev < cap ? *nev : cap, lam, res, W, n);
  return st;
}

/* ------------------------------------------------------------------ whole run
 * The driver sequence of TESTS/Lap/LapPLanN.c:118-296 with the bounds step
 * of TESTS/MM/MMPLanN.c:104-118: start vector first, bounds, DOS, slicer,
 * then every slice with nev = ev_int + 2 and mlan = min(max(5 nev, 300), n). */
int orc_pipeline(const orc_spec *s, orc_out *o) {
  csr_t A = {s->n, s->ia, s->ja, s->a};
  int n = s->n, nsl = s->nslices;
  double xintv[4], t0 = now_s(), t;
  o->status = 0;
  orc_set_rng(s->rng_mode, s->seed);
  double *vinit = (double *)xcalloc((size_t)n, sizeof(double));
  orc_rand_vector(vinit, n);
  t = now_s();
  if (s->bounds_mode == 1) {
    int st = lantrbounds(&A, s->lan_lanm, s->lan_maxit, s->lan_tol, vinit, s->lan_bndtype,
                         &o->lmin, &o->lmax);
    if (st) o->status = 400 - st;
  } else {
    o->lmin = s->lmin;
    o->lmax = s->lmax;
  }
  o->t_bounds = now_s() - t;
  xintv[0] = s->a_lo;
  xintv[1] = s->b_hi;
  xintv[2] = o->lmin;
  xintv[3] = o->lmax;
  t = now_s();
  if (s->dos_type == 0) {
    int ierr = kpmdos(&A, s->Mdeg, s->kpm_damping, s->nvec, xintv, o->mu, &o->ecount);
    o->t_dos = now_s() - t;
    if (ierr && !o->status) o->status = 100 + ierr;
    t = now_s();
    o->npts = (int)(10 * o->ecount);
    ierr = orc_spslicer_kpm(o->sli, o->mu, s->Mdeg, xintv, nsl, o->npts);
    if (ierr && !o->status) o->status = 200 + ierr;
    o->t_slicer = now_s() - t;
  } else {
    int npts = s->landos_npts;
    double *xdos = (double *)xcalloc((size_t)npts, sizeof(double));
    double *ydos = (double *)xcalloc((size_t)npts, sizeof(double));
    landos(&A, s->nvec, s->landos_msteps, npts, xdos, ydos, &o->ecount, xintv, 1.0);
    o->t_dos = now_s() - t;
    t = now_s();
    o->npts = npts;
    orc_spslicer_lan(xdos, ydos, nsl, npts, o->sli);
    o->t_slicer = now_s() - t;
    free(xdos);
    free(ydos);
  }
  int ev_int = (int)(1 + o->ecount / ((double)nsl));
  t = now_s();
  for (int sl = 0; sl < nsl; sl++) {
    orc_pol pol;
    int nev = ev_int + 2;
    int mlan = nev * 5 > s->mlan_min ? nev * 5 : s->mlan_min;
    mlan = mlan < n ? mlan : n;
    xintv[0] = o->sli[sl];
    xintv[1] = o->sli[sl + 1];
    xintv[2] = o->lmin;
    xintv[3] = o->lmax;
    pol_defaults(&pol);
    pol.damping = s->pol_damping;
    pol.thresh_int = s->thresh_int;
    pol.thresh_ext = s->thresh_ext;
    pol.max_deg = s->pol_max_deg;
    findpol(xintv, &pol);
    o->deg[sl] = pol.deg;
    o->ptype[sl] = pol.type;
    o->gam[sl] = pol.gam;
    o->bar[sl] = pol.bar;
    int nev2 = 0, its = 0;
    double *lam = o->lam + (size_t)sl * o->cap, *res = o->res + (size_t)sl * o->cap;
    int st = cheblannr(&A, xintv, mlan, s->tol, vinit, &pol, &nev2, &its, lam, res, NULL,
                       o->cap);
    if (st && !o->status) o->status = 300 + st;
    sort_pairs(nev2 < o->cap ? nev2 : o->cap, lam, res, NULL, n);
    o->nev[sl] = nev2;
    o->its[sl] = its;
    free(pol.mu);
  }
  o->t_slices = now_s() - t;
  free(vinit);
  o->t_total = now_s() - t0;
  return o->status;
}
