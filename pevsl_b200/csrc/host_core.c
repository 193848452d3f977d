/*
 * Host side of the pEVSL interface that involves no GPU work: instance
 * lifecycle and setters (SRC/pevsl.c), interval checks (INC/pevsl_int.h:
 * 174-193), sorting / partition / search utilities (SRC/utils.c,
 * SRC/vector.c), the host CSR/COO helpers that callers use to assemble a
 * matrix before pEVSL_ParcsrSetup uploads it (SRC/spmat.c), and the
 * statistics printout (SRC/stats.c).
 */
#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "internal.h"

double pevsl_now(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

double pEVSL_Wtime(void) { return pevsl_now(); }

/* 0 if [a,b] is a valid interval meeting [lmin,lmax]; -1 if a >= b; -2 if it
 * lies outside the bounds (INC/pevsl_int.h:174-193). */
int pevsl_check_intv(const double *intv, FILE *fstats) {
  const double a = intv[0], b = intv[1], lmin = intv[2], lmax = intv[3];
  if (a >= b) {
    if (fstats) fprintf(fstats, " error: invalid interval (%e, %e)\n", a, b);
    return -1;
  }
  if (a >= lmax || b <= lmin) {
    if (fstats)
      fprintf(fstats, " error: interval (%e, %e) is outside (%e %e) \n", a, b, lmin, lmax);
    return -2;
  }
  return 0;
}

/* ------------------------------------------------------------------ instance */

/* SRC/pevsl.c:13-45: sizes undefined, no operators, srand(rank) with rank 0. */
int pEVSL_Start(MPI_Comm comm, pevsl_Data **data) {
  pevsl_inst *inst = (pevsl_inst *)calloc(1, sizeof(pevsl_inst));
  if (!inst) return PEVSL_ERR_NOMEM;
  pevsl_Data *d = &inst->pub;
  d->comm = comm;
  d->N = PEVSL_NOT_DEFINED;
  d->n = PEVSL_NOT_DEFINED;
  d->nfirst = PEVSL_NOT_DEFINED;
  d->ifGenEv = 0;
  d->sigma_mult = 1.0;
  d->stats = &inst->stat;
  srand(0);
  *data = d;
  return 0;
}

int pEVSL_Finish(pevsl_Data *d) {
  if (d) free(pevsl_inst_of(d));
  return 0;
}

int pEVSL_SetProbSizes(pevsl_Data *d, int N, int n, int nfirst) {
  d->N = N;
  d->n = n;
  d->nfirst = nfirst < 0 ? PEVSL_NOT_DEFINED : nfirst;
  return 0;
}

/* SRC/pevsl.c:81-97: sizes from the matrix, A x by the built-in callback. */
int pEVSL_SetAParcsr(pevsl_Data *d, pevsl_Parcsr *A) {
  pevsl_inst *inst = pevsl_inst_of(d);
  d->N = A->ncol_global;
  d->n = A->ncol_local;
  d->nfirst = A->first_col;
  inst->amv.func = pEVSL_ParcsrMatvec0;
  inst->amv.data = (void *)A;
  d->Amv = &inst->amv;
  return 0;
}

int pEVSL_SetBParcsr(pevsl_Data *d, pevsl_Parcsr *B) {
  pevsl_inst *inst = pevsl_inst_of(d);
  d->N = B->ncol_global;
  d->n = B->ncol_local;
  d->nfirst = B->first_col;
  inst->bmv.func = pEVSL_ParcsrMatvec0;
  inst->bmv.data = (void *)B;
  d->Bmv = &inst->bmv;
  return 0;
}

int pEVSL_SetAMatvec(pevsl_Data *d, MVFunc func, void *data) {
  pevsl_inst *inst = pevsl_inst_of(d);
  inst->amv.func = func;
  inst->amv.data = data;
  d->Amv = &inst->amv;
  return 0;
}

int pEVSL_SetBMatvec(pevsl_Data *d, MVFunc func, void *data) {
  pevsl_inst *inst = pevsl_inst_of(d);
  inst->bmv.func = func;
  inst->bmv.data = data;
  d->Bmv = &inst->bmv;
  return 0;
}

int pEVSL_SetBSol(pevsl_Data *d, SVFunc func, void *data) {
  pevsl_inst *inst = pevsl_inst_of(d);
  inst->bsol.func = func;
  inst->bsol.data = data;
  d->Bsol = &inst->bsol;
  return 0;
}

int pEVSL_SetLTSol(pevsl_Data *d, SVFunc func, void *data) {
  pevsl_inst *inst = pevsl_inst_of(d);
  inst->ltsol.func = func;
  inst->ltsol.data = data;
  d->LTsol = &inst->ltsol;
  return 0;
}

int pEVSL_SetStdEig(pevsl_Data *d) {
  d->ifGenEv = 0;
  return 0;
}

int pEVSL_SetGenEig(pevsl_Data *d) {
  d->ifGenEv = 1;
  return 0;
}

int pEVSL_SetSigmaMult(pevsl_Data *d, double mult) {
  d->sigma_mult = mult;
  return 0;
}

int pEVSL_B200_SetPrecision(pevsl_Data *d, int precision) {
  if (precision != PEVSL_PREC_FP64 && precision != PEVSL_PREC_MIXED) return PEVSL_ERR_ARG;
  pevsl_inst_of(d)->precision = precision;
  return 0;
}

int pEVSL_B200_LastIterations(pevsl_Data *d) { return pevsl_inst_of(d)->last_its; }
int pEVSL_B200_LastNconv(pevsl_Data *d) { return pevsl_inst_of(d)->last_nconv; }
double pEVSL_B200_PhaseMs(pevsl_Data *d, int phase) {
  return (phase >= 0 && phase < 8) ? pevsl_inst_of(d)->phase_ms[phase] : 0.0;
}

/* ------------------------------------------------------------------ utilities */

static int cmp_int(const void *a, const void *b) {
  const int x = *(const int *)a, y = *(const int *)b;
  return (x > y) - (x < y);
}

static int cmp_dbl(const void *a, const void *b) {
  const double x = *(const double *)a, y = *(const double *)b;
  return (x > y) - (x < y);
}

typedef struct {
  int i;
  double d;
} dbl_idx;

static int cmp_dbl_idx(const void *a, const void *b) {
  const double x = ((const dbl_idx *)a)->d, y = ((const dbl_idx *)b)->d;
  return (x > y) - (x < y);
}

void pEVSL_SortInt(int *x, int n) { qsort(x, (size_t)n, sizeof(int), cmp_int); }

/* Ascending sort; ind (optional) receives the original positions
 * (SRC/vector.c:85-104, SRC/utils.c:58-75). */
void sort_double(int n, double *v, int *ind) {
  if (!ind) {
    qsort(v, (size_t)n, sizeof(double), cmp_dbl);
    return;
  }
  dbl_idx *t = (dbl_idx *)malloc((size_t)(n > 0 ? n : 1) * sizeof(dbl_idx));
  for (int i = 0; i < n; i++) {
    t[i].d = v[i];
    t[i].i = i;
  }
  qsort(t, (size_t)n, sizeof(dbl_idx), cmp_dbl_idx);
  for (int i = 0; i < n; i++) {
    v[i] = t[i].d;
    ind[i] = t[i].i;
  }
  free(t);
}

void pEVSL_SortDouble(int n, double *v, int *ind) { sort_double(n, v, ind); }

void vecset(int n, double t, double *v) {
  for (int i = 0; i < n; i++) v[i] = t;
}
void pEVSL_Vecset(int n, double t, double *v) { vecset(n, t, v); }

/* Balanced 1D partition of len items into pnum parts, the first len % pnum
 * parts one longer (SRC/utils.c:128-149).  job 1: range [j1,j2) of part
 * *idx; job 2: part *idx owning item *j1, and its size in *j2. */
void pEVSL_Part1d(int len, int pnum, int *idx, int *j1, int *j2, int job) {
  int size = (len + pnum - 1) / pnum;
  const int big = pnum - (size * pnum - len);
  if (job == 1) {
    if (*idx < big) {
      *j1 = *idx * size;
    } else {
      size--;
      *j1 = len - size * (pnum - *idx);
    }
    *j2 = *j1 + size;
  } else {
    if (*j1 < size * big) {
      *idx = *j1 / size;
    } else {
      *idx = big + (*j1 - size * big) / (size - 1);
      size--;
    }
    if (j2) *j2 = size;
  }
}

int pEVSL_BinarySearch(int *x, int n, int key) {
  int lo = 0, hi = n - 1;
  while (lo <= hi) {
    const int mid = lo + (hi - lo) / 2;
    if (x[mid] == key) return mid;
    if (x[mid] < key) {
      lo = mid + 1;
    } else {
      hi = mid - 1;
    }
  }
  return -1;
}

/* ------------------------------------------------------------------ host CSR / COO */

void pEVSL_CsrResize(int nrow, int ncol, int nnz, pevsl_Csr *csr) {
  csr->nrows = nrow;
  csr->ncols = ncol;
  csr->ia = (int *)malloc((size_t)(nrow + 1) * sizeof(int));
  csr->ja = (int *)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(int));
  csr->a = (double *)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(double));
}

void pEVSL_FreeCsr(pevsl_Csr *csr) {
  free(csr->ia);
  free(csr->ja);
  free(csr->a);
  csr->ia = NULL;
  csr->ja = NULL;
  csr->a = NULL;
}

void pEVSL_CooResize(int nrow, int ncol, int nnz, pevsl_Coo *coo) {
  coo->nrows = nrow;
  coo->ncols = ncol;
  coo->nnz = nnz;
  coo->ir = (int *)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(int));
  coo->jc = (int *)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(int));
  coo->vv = (double *)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(double));
}

void pEVSL_FreeCoo(pevsl_Coo *coo) {
  free(coo->ir);
  free(coo->jc);
  free(coo->vv);
  coo->ir = NULL;
  coo->jc = NULL;
  coo->vv = NULL;
}

/* Counting sort of the triples by row; entries keep their input order within
 * a row (SRC/spmat.c:56-86). */
int pEVSL_CooToCsr(int cooidx, pevsl_Coo *coo, pevsl_Csr *csr) {
  const int base = cooidx != 0, nnz = coo->nnz, nr = coo->nrows;
  pEVSL_CsrResize(nr, coo->ncols, nnz, csr);
  int *cnt = csr->ia;
  memset(cnt, 0, (size_t)(nr + 1) * sizeof(int));
  for (int i = 0; i < nnz; i++) cnt[coo->ir[i] - base + 1]++;
  for (int i = 0; i < nr; i++) cnt[i + 1] += cnt[i];
  int *next = (int *)malloc((size_t)(nr > 0 ? nr : 1) * sizeof(int));
  memcpy(next, cnt, (size_t)nr * sizeof(int));
  for (int i = 0; i < nnz; i++) {
    const int r = coo->ir[i] - base, k = next[r]++;
    csr->ja[k] = coo->jc[i] - base;
    csr->a[k] = coo->vv[i];
  }
  free(next);
  return 0;
}

int pEVSL_CsrToCoo(pevsl_Csr *csr, int cooidx, pevsl_Coo *coo) {
  const int base = cooidx != 0, nnz = csr->ia[csr->nrows];
  pEVSL_CooResize(csr->nrows, csr->ncols, nnz, coo);
  int k = 0;
  for (int i = 0; i < csr->nrows; i++) {
    for (int j = csr->ia[i]; j < csr->ia[i + 1]; j++, k++) {
      coo->ir[k] = i + base;
      coo->jc[k] = csr->ja[j] + base;
      coo->vv[k] = csr->a[j];
    }
  }
  return 0;
}

/* y = alp A x + bet y on a HOST csr (SRC/spmat.c:127-170). */
int pEVSL_MatvecGen(double alp, pevsl_Csr *A, double *x, double bet, double *y) {
  for (int i = 0; i < A->nrows; i++) {
    double r = 0.0;
    for (int j = A->ia[i]; j < A->ia[i + 1]; j++) r += A->a[j] * x[A->ja[j]];
    y[i] = bet * y[i] + alp * r;
  }
  return 0;
}

/* y = A x on a HOST csr (SRC/spmat.c:184-230). */
int pEVSL_Matvec(pevsl_Csr *A, double *x, double *y) {
  for (int i = 0; i < A->nrows; i++) {
    double r = 0.0;
    for (int j = A->ia[i]; j < A->ia[i + 1]; j++) r += A->a[j] * x[A->ja[j]];
    y[i] = r;
  }
  return 0;
}

/* Sort the column indices of every row, carrying the values
 * (SRC/spmat.c:287-305 does it by double transposition). */
void pEVSL_SortRow(pevsl_Csr *A) {
  for (int i = 0; i < A->nrows; i++) {
    for (int j = A->ia[i] + 1; j < A->ia[i + 1]; j++) {
      const int c = A->ja[j];
      const double v = A->a[j];
      int t = j - 1;
      while (t >= A->ia[i] && A->ja[t] > c) {
        A->ja[t + 1] = A->ja[t];
        A->a[t + 1] = A->a[t];
        t--;
      }
      A->ja[t + 1] = c;
      A->a[t + 1] = v;
    }
  }
}

/* ------------------------------------------------------------------ statistics */

void pEVSL_StatsReset(pevsl_Data *d) { memset(d->stats, 0, sizeof(pevsl_Stat)); }

/* Same layout as the reference printout (SRC/stats.c:13-103). */
void pEVSL_StatsPrint(pevsl_Data *d, FILE *f) {
  if (!f) return;
  const pevsl_Stat *s = d->stats;
  fprintf(f, "= = = = = = = = = = = = = = = = = = = Time & Memory Stats = = = = = = = = = = = = = "
             "= = = = = = =\n");
  fprintf(f, " Timing (sec):\n");
  if (s->t_setBsv) fprintf(f, "   Setup Solver for B        :  %f\n", s->t_setBsv);
  if (s->t_setASigBsv) fprintf(f, "   Setup Solver for A-SIG*B  :  %f\n", s->t_setASigBsv);
  if (s->t_eigbounds) fprintf(f, "   Compute Eigenvalue bounds :  %f\n", s->t_eigbounds);
  if (s->t_dos) fprintf(f, "   Compute DOS               :  %f\n", s->t_dos);
  if (s->t_iter) fprintf(f, "   Iteration time (tot)      :  %f\n", s->t_iter);
  fprintf(f, "   - - - - - - - - - - - - - - - - -\n");
  if (s->n_polAv)
    fprintf(f, "   Pol(A)*v                  :  %f (%8lu, avg %f)\n", s->t_polAv,
            (unsigned long)s->n_polAv, s->t_polAv / (double)s->n_polAv);
  if (s->n_mvA)
    fprintf(f, "   Matvec matrix A           :  %f (%8lu, avg %f)\n", s->t_mvA,
            (unsigned long)s->n_mvA, s->t_mvA / (double)s->n_mvA);
  if (s->t_reorth) fprintf(f, "   Reorthogonalization       :  %f\n", s->t_reorth);
  if (s->t_eig) fprintf(f, "   LAPACK eig                :  %f\n", s->t_eig);
  if (s->t_blas) fprintf(f, "   Other BLAS                :  %f\n", s->t_blas);
  if (s->t_ritz) fprintf(f, "   Compute Ritz vectors      :  %f\n", s->t_ritz);
  if (s->t_sth) fprintf(f, "   Other                     :  %f\n", s->t_sth);
  fprintf(f, "= = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = "
             "=\n");
}
