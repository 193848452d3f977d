/*
 * Small dense eigensolvers on the host (the reference calls LAPACK here):
 *
 *  - symmetric tridiagonal T (the Lanczos matrix; DSTEV in SymmTridEig,
 *    SRC/miscla.c:29-66): implicit QR sweeps with a Wilkinson shift, each
 *    chasing a bulge down an unreduced block by Givens rotations
 *    (Golub & Van Loan, Matrix Computations, Alg. 8.3.2-8.3.3).  Eigenvalues
 *    cost O(k^2).  Eigenvectors are formed only for the eigenvalues the
 *    caller selects: the rotations of the sweep are recorded and replayed,
 *    last to first, onto the unit vectors of the selected positions, which
 *    costs O(#rotations) per vector instead of the O(k^3) of accumulating the
 *    full eigenvector matrix.
 *  - dense symmetric (the thick-restart matrix of the bounds estimator; DSYEV
 *    in SymEigenSolver, SRC/miscla.c:161-198): cyclic Jacobi
 *    (Golub & Van Loan, Alg. 8.5.3).
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "internal.h"

typedef struct {
  int k;
  double c, s;
} rot_t;

typedef struct {
  rot_t *r;
  size_t n, cap;
  int failed;
} rotlog_t;

static void rotlog_push(rotlog_t *L, int k, double c, double s) {
  if (L->failed) return;
  if (L->n == L->cap) {
    size_t nc = L->cap ? 2 * L->cap : 4096;
    rot_t *p = (rot_t *)realloc(L->r, nc * sizeof(rot_t));
    if (!p) {
      L->failed = 1;
      return;
    }
    L->r = p;
    L->cap = nc;
  }
  L->r[L->n].k = k;
  L->r[L->n].c = c;
  L->r[L->n].s = s;
  L->n++;
}

/* Diagonalise T in place: d <- eigenvalues (unsorted).  Rotations go to L
 * when it is non-NULL.  Returns 0, or 1 if some block needed more than 40
 * sweeps per row. */
static int tridiag_qr(int n, double *d, double *e, rotlog_t *L) {
  int q = n - 1, sweeps = 0;
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
    if (++sweeps > 40 * n) return 1;
    /* shift: eigenvalue of the trailing 2x2 block closer to d[q] */
    const double half = 0.5 * (d[q - 1] - d[q]), b = e[q - 1];
    const double shift = d[q] - b * b / (half + copysign(hypot(half, b), half >= 0 ? 1.0 : -1.0));
    double x = d[p] - shift, z = e[p];
    for (int k = p; k < q; k++) {
      /* rotation in the (k, k+1) plane that zeroes z against x: the first
       * column of T - shift I at k == p, the bulge below e[k-1] after that */
      const double r = hypot(x, z);
      const double c = r == 0.0 ? 1.0 : x / r, s = r == 0.0 ? 0.0 : z / r;
      if (k > p) e[k - 1] = r;
      const double a0 = d[k], b0 = e[k], a1 = d[k + 1];
      d[k] = a0 * c * c + 2.0 * b0 * c * s + a1 * s * s;
      d[k + 1] = a0 * s * s - 2.0 * b0 * c * s + a1 * c * c;
      e[k] = (a1 - a0) * c * s + b0 * (c * c - s * s);
      double bulge = 0.0;
      if (k + 1 < q) {
        bulge = s * e[k + 1];
        e[k + 1] = c * e[k + 1];
      }
      if (L) rotlog_push(L, k, c, s);
      x = e[k];
      z = bulge;
    }
  }
  return 0;
}

/* order[i] = position (in the unsorted result) of the i-th smallest value */
static int *ascending_order(int n, const double *d) {
  int *ord = (int *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int));
  if (!ord) return NULL;
  for (int i = 0; i < n; i++) ord[i] = i;
  /* insertion sort: n is the Lanczos dimension, and ties keep position order */
  for (int i = 1; i < n; i++) {
    int v = ord[i], j = i - 1;
    while (j >= 0 && d[ord[j]] > d[v]) {
      ord[j + 1] = ord[j];
      j--;
    }
    ord[j + 1] = v;
  }
  return ord;
}

/* Eigenvalues w (ascending) and, if Z != NULL, all eigenvectors (n x n,
 * column major).  Returns 0 or PEVSL_ERR_EIG / PEVSL_ERR_NOMEM. */
int pevsl_tridiag_eig(int n, const double *d_in, const double *e_in, double *w, double *Z) {
  if (n <= 0) return 0;
  double *d = (double *)malloc((size_t)n * sizeof(double));
  double *e = (double *)calloc((size_t)n, sizeof(double));
  if (!d || !e) {
    free(d);
    free(e);
    return PEVSL_ERR_NOMEM;
  }
  memcpy(d, d_in, (size_t)n * sizeof(double));
  if (n > 1) memcpy(e, e_in, (size_t)(n - 1) * sizeof(double));
  rotlog_t L = {0};
  int st = tridiag_qr(n, d, e, Z ? &L : NULL);
  int *ord = ascending_order(n, d);
  if (!ord || L.failed) st = PEVSL_ERR_NOMEM;
  if (st == 0) {
    for (int i = 0; i < n; i++) w[i] = d[ord[i]];
    if (Z) {
      /* replay onto every unit vector: column i of Z is eigenvector ord[i] */
      memset(Z, 0, (size_t)n * (size_t)n * sizeof(double));
      for (int i = 0; i < n; i++) Z[(size_t)i * n + ord[i]] = 1.0;
      for (size_t r = L.n; r-- > 0;) {
        const int k = L.r[r].k;
        const double c = L.r[r].c, s = L.r[r].s;
        for (int i = 0; i < n; i++) {
          double *zc = Z + (size_t)i * n;
          const double xk = zc[k], xk1 = zc[k + 1];
          zc[k] = c * xk - s * xk1;
          zc[k + 1] = s * xk + c * xk1;
        }
      }
    }
  } else if (st == 1) {
    st = PEVSL_ERR_EIG;
  }
  free(L.r);
  free(ord);
  free(d);
  free(e);
  return st;
}

/* Eigenvalues w (ascending, all n) and the eigenvectors of the nsel
 * eigenvalues with ascending indices sel[] (Zsel, n x nsel column major). */
int pevsl_tridiag_eig_sel(int n, const double *d_in, const double *e_in, double *w, int nsel,
                          const int *sel, double *Zsel) {
  if (n <= 0) return 0;
  double *d = (double *)malloc((size_t)n * sizeof(double));
  double *e = (double *)calloc((size_t)n, sizeof(double));
  if (!d || !e) {
    free(d);
    free(e);
    return PEVSL_ERR_NOMEM;
  }
  memcpy(d, d_in, (size_t)n * sizeof(double));
  if (n > 1) memcpy(e, e_in, (size_t)(n - 1) * sizeof(double));
  rotlog_t L = {0};
  int st = tridiag_qr(n, d, e, nsel > 0 ? &L : NULL);
  int *ord = ascending_order(n, d);
  if (!ord || L.failed) st = PEVSL_ERR_NOMEM;
  if (st == 0) {
    for (int i = 0; i < n; i++) w[i] = d[ord[i]];
    if (nsel > 0) {
      /* rows of X are coordinates, columns the selected vectors: each
       * rotation touches two contiguous rows */
      double *X = (double *)calloc((size_t)n * (size_t)nsel, sizeof(double));
      if (!X) {
        st = PEVSL_ERR_NOMEM;
      } else {
        for (int j = 0; j < nsel; j++) X[(size_t)ord[sel[j]] * nsel + j] = 1.0;
        for (size_t r = L.n; r-- > 0;) {
          const int k = L.r[r].k;
          const double c = L.r[r].c, s = L.r[r].s;
          double *xk = X + (size_t)k * nsel, *xk1 = xk + nsel;
          for (int j = 0; j < nsel; j++) {
            const double a = xk[j], b = xk1[j];
            xk[j] = c * a - s * b;
            xk1[j] = s * a + c * b;
          }
        }
        for (int j = 0; j < nsel; j++)
          for (int i = 0; i < n; i++) Zsel[(size_t)j * n + i] = X[(size_t)i * nsel + j];
        free(X);
      }
    }
  } else if (st == 1) {
    st = PEVSL_ERR_EIG;
  }
  free(L.r);
  free(ord);
  free(d);
  free(e);
  return st;
}

/* Dense symmetric eigen-decomposition by cyclic Jacobi rotations; lam
 * ascending, Q columns the eigenvectors.  Returns 0 or PEVSL_ERR_NOMEM. */
int pevsl_dense_symeig(int n, const double *A, int lda, double *Q, int ldq, double *lam) {
  double *S = (double *)malloc((size_t)n * (size_t)n * sizeof(double));
  double *V = (double *)malloc((size_t)n * (size_t)n * sizeof(double));
  if (!S || !V) {
    free(S);
    free(V);
    return PEVSL_ERR_NOMEM;
  }
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) {
      S[(size_t)j * n + i] = A[(size_t)j * lda + i];
      V[(size_t)j * n + i] = i == j ? 1.0 : 0.0;
    }
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0, tot = 0.0;
    for (size_t t = 0; t < (size_t)n * n; t++) tot += S[t] * S[t];
    for (int j = 0; j < n; j++) off -= S[(size_t)j * n + j] * S[(size_t)j * n + j];
    off += tot;
    if (off <= DBL_EPSILON * DBL_EPSILON * tot) break;
    for (int p = 0; p < n - 1; p++) {
      for (int q = p + 1; q < n; q++) {
        const double apq = S[(size_t)q * n + p];
        if (apq == 0.0) continue;
        const double theta = (S[(size_t)q * n + q] - S[(size_t)p * n + p]) / (2.0 * apq);
        const double t = copysign(1.0, theta) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        double *sp = S + (size_t)p * n, *sq = S + (size_t)q * n;
        for (int k = 0; k < n; k++) {
          const double u = sp[k], v = sq[k];
          sp[k] = c * u - s * v;
          sq[k] = s * u + c * v;
        }
        for (int k = 0; k < n; k++) {
          double *col = S + (size_t)k * n;
          const double u = col[p], v = col[q];
          col[p] = c * u - s * v;
          col[q] = s * u + c * v;
        }
        double *vp = V + (size_t)p * n, *vq = V + (size_t)q * n;
        for (int k = 0; k < n; k++) {
          const double u = vp[k], v = vq[k];
          vp[k] = c * u - s * v;
          vq[k] = s * u + c * v;
        }
      }
    }
  }
  double *diag = (double *)malloc((size_t)n * sizeof(double));
  for (int i = 0; i < n; i++) diag[i] = S[(size_t)i * n + i];
  int *ord = ascending_order(n, diag);
  for (int i = 0; i < n; i++) {
    lam[i] = diag[ord[i]];
    memcpy(Q + (size_t)i * ldq, V + (size_t)ord[i] * n, (size_t)n * sizeof(double));
  }
  free(ord);
  free(diag);
  free(S);
  free(V);
  return 0;
}

/* Eigenpairs of a dense symmetric matrix (column major, both triangles set)
 * whose eigenvalues lie in [lo, hi]: Householder reduction to tridiagonal
 * form Q' H Q = T (Golub & Van Loan, Alg. 8.3.1, with the symmetric rank-2
 * update), the tridiagonal QR above for the eigenvalues and the selected
 * eigenvectors y, then x = Q y by applying the reflectors last to first
 * (Q is never formed).  lam (ascending) and Z (n x *m) must hold n
 * entries / columns.  O(n^3) for the reduction, O(n^2 *m) for the vectors. */
int pevsl_dense_symeig_range(int n, const double *H, int ldh, double lo, double hi, int *m,
                             double *lam, double *Z, int ldz) {
  *m = 0;
  if (n <= 0) return 0;
  double *A = (double *)malloc((size_t)n * (size_t)n * sizeof(double));
  double *d = (double *)malloc((size_t)n * sizeof(double));
  double *e = (double *)calloc((size_t)n, sizeof(double));
  double *beta = (double *)calloc((size_t)n, sizeof(double));
  double *p = (double *)malloc((size_t)n * sizeof(double));
  double *w = (double *)malloc((size_t)n * sizeof(double));
  int *sel = (int *)malloc((size_t)n * sizeof(int));
  int st = 0;
  if (!A || !d || !e || !beta || !p || !w || !sel) st = PEVSL_ERR_NOMEM;
  if (!st) {
    for (int j = 0; j < n; j++) memcpy(A + (size_t)j * n, H + (size_t)j * ldh, (size_t)n * sizeof(double));
    /* reflector k acts on rows/cols k+1..n-1; its vector v (v[0] = 1 is not
     * stored implicitly: the whole v is kept) replaces A(k+1:n, k) */
    for (int k = 0; k + 2 < n; k++) {
      double *x = A + (size_t)k * n + (k + 1);
      const int len = n - k - 1;
      double sig = 0.0;
      for (int i = 1; i < len; i++) sig += x[i] * x[i];
      if (sig == 0.0) {
        beta[k] = 0.0;
        e[k] = x[0];
        continue;
      }
      const double nx = sqrt(x[0] * x[0] + sig);
      const double alpha = x[0] > 0 ? -nx : nx;
      x[0] -= alpha; /* v = x - alpha e1 */
      const double vv = x[0] * x[0] + sig;
      const double b = 2.0 / vv;
      beta[k] = b;
      e[k] = alpha;
      /* p = b * A22 v */
      double *A22 = A + (size_t)(k + 1) * n + (k + 1);
      for (int i = 0; i < len; i++) p[i] = 0.0;
      for (int j = 0; j < len; j++) {
        const double vj = x[j];
        const double *col = A22 + (size_t)j * n;
        for (int i = 0; i < len; i++) p[i] += col[i] * vj;
      }
      double pv = 0.0;
      for (int i = 0; i < len; i++) {
        p[i] *= b;
        pv += p[i] * x[i];
      }
      /* w = p - (b/2)(p'v) v;  A22 -= v w' + w v' */
      const double c = 0.5 * b * pv;
      for (int i = 0; i < len; i++) w[i] = p[i] - c * x[i];
      for (int j = 0; j < len; j++) {
        double *col = A22 + (size_t)j * n;
        const double vj = x[j], wj = w[j];
        for (int i = 0; i < len; i++) col[i] -= x[i] * wj + w[i] * vj;
      }
    }
    for (int i = 0; i < n; i++) d[i] = A[(size_t)i * n + i];
    if (n >= 2) e[n - 2] = A[(size_t)(n - 2) * n + (n - 1)];
    for (int k = 0; k + 2 < n; k++)
      if (beta[k] == 0.0) e[k] = A[(size_t)k * n + (k + 1)];
    /* eigenvalues, then the vectors of those in [lo, hi] */
    st = pevsl_tridiag_eig(n, d, e, w, NULL);
    int ns = 0;
    for (int i = 0; !st && i < n; i++)
      if (w[i] >= lo && w[i] <= hi) sel[ns++] = i;
    if (!st && ns > 0) {
      double *Y = (double *)malloc((size_t)n * (size_t)ns * sizeof(double));
      if (!Y) st = PEVSL_ERR_NOMEM;
      if (!st) st = pevsl_tridiag_eig_sel(n, d, e, w, ns, sel, Y);
      for (int j = 0; !st && j < ns; j++) {
        double *y = Y + (size_t)j * n;
        for (int k = n - 3; k >= 0; k--) {
          if (beta[k] == 0.0) continue;
          const double *v = A + (size_t)k * n + (k + 1);
          double s = 0.0;
          for (int i = 0; i < n - k - 1; i++) s += v[i] * y[k + 1 + i];
          s *= beta[k];
          for (int i = 0; i < n - k - 1; i++) y[k + 1 + i] -= s * v[i];
        }
        lam[j] = w[sel[j]];
        memcpy(Z + (size_t)j * ldz, y, (size_t)n * sizeof(double));
      }
      free(Y);
      if (!st) *m = ns;
    }
  }
  free(A);
  free(d);
  free(e);
  free(beta);
  free(p);
  free(w);
  free(sel);
  return st;
}

/* Eigenpairs with eigenvalues in [lo, hi] of the pencil (H, G), G = P'P a
 * Gram matrix with unit diagonal, H = P' A P (both m x m, column major):
 * Cholesky G = L L' processed column by column, a column whose pivot falls
 * below 1e-10 (numerically dependent on the earlier ones) is dropped, then
 * C = L^-1 H L^-T on the kept columns, the ranged eigensolver above, and
 * Z = L^-T Zc scattered back to the m rows (dropped rows zero).  Returns
 * the eigenvalues (ascending) in lam and the m x *nout coefficients in Z. */
int pevsl_gen_symeig_range(int m, const double *H, const double *G, int ld, double lo, double hi,
                           int *nout, double *lam, double *Z, int ldz) {
  *nout = 0;
  if (m <= 0) return 0;
  double *L = (double *)calloc((size_t)m * m, sizeof(double)); /* kept x kept, column major */
  int *keep = (int *)malloc((size_t)m * sizeof(int));
  double *Cm = (double *)malloc((size_t)m * m * sizeof(double));
  double *Zc = (double *)malloc((size_t)m * m * sizeof(double));
  double *tmp = (double *)malloc((size_t)m * sizeof(double));
  int st = (!L || !keep || !Cm || !Zc || !tmp) ? PEVSL_ERR_NOMEM : 0;
  int q = 0;
  /* left-looking Cholesky over the kept columns */
  for (int j = 0; j < m && !st; j++) {
    /* row q of L for candidate column j: L(q, i) for i < q solve L(0:q,0:q) l = G(keep, j) */
    for (int i = 0; i < q; i++) {
      double s = G[(size_t)j * ld + keep[i]];
      for (int t = 0; t < i; t++) s -= L[(size_t)t * m + i] * tmp[t];
      tmp[i] = s / L[(size_t)i * m + i];
    }
    double d = G[(size_t)j * ld + j];
    for (int i = 0; i < q; i++) d -= tmp[i] * tmp[i];
    if (!(d > 1e-10 * G[(size_t)j * ld + j])) continue; /* dependent: drop */
    for (int i = 0; i < q; i++) L[(size_t)i * m + q] = tmp[i];
    L[(size_t)q * m + q] = sqrt(d);
    keep[q++] = j;
  }
  if (!st && q > 0) {
    /* C = L^-1 Hk L^-T, Hk = H(keep, keep): solve column by column */
    for (int c = 0; c < q; c++) {
      for (int r = 0; r < q; r++) Cm[(size_t)c * q + r] = H[(size_t)keep[c] * ld + keep[r]];
    }
    /* Cm <- L^-1 Cm (forward substitution on each column) */
    for (int c = 0; c < q; c++) {
      double *col = Cm + (size_t)c * q;
      for (int r = 0; r < q; r++) {
        double s = col[r];
        for (int t = 0; t < r; t++) s -= L[(size_t)t * m + r] * col[t];
        col[r] = s / L[(size_t)r * m + r];
      }
    }
    /* Cm <- Cm L^-T: rows of Cm solved against L, i.e. (L^-1 Cm^T)^T */
    for (int r = 0; r < q; r++) {
      for (int c = 0; c < q; c++) {
        double s = Cm[(size_t)c * q + r];
        for (int t = 0; t < c; t++) s -= L[(size_t)t * m + c] * Cm[(size_t)t * q + r];
        Cm[(size_t)c * q + r] = s / L[(size_t)c * m + c];
      }
    }
    for (int c = 0; c < q; c++)
      for (int r = 0; r < c; r++) {
        const double h = 0.5 * (Cm[(size_t)c * q + r] + Cm[(size_t)r * q + c]);
        Cm[(size_t)c * q + r] = Cm[(size_t)r * q + c] = h;
      }
    int ns = 0;
    st = pevsl_dense_symeig_range(q, Cm, q, lo, hi, &ns, lam, Zc, q);
    /* Z(keep, j) = L^-T zc (back substitution), other rows zero */
    for (int j = 0; j < ns && !st; j++) {
      double *zc = Zc + (size_t)j * q;
      for (int r = q - 1; r >= 0; r--) {
        double s = zc[r];
        for (int t = r + 1; t < q; t++) s -= L[(size_t)r * m + t] * zc[t];
        zc[r] = s / L[(size_t)r * m + r];
      }
      double *z = Z + (size_t)j * ldz;
      for (int r = 0; r < m; r++) z[r] = 0.0;
      for (int r = 0; r < q; r++) z[keep[r]] = zc[r];
    }
    if (!st) *nout = ns;
  }
  free(L);
  free(keep);
  free(Cm);
  free(Zc);
  free(tmp);
  return st;
}
