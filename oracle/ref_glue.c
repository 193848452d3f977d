/*
 * Glue that drives the pEVSL reference, compiled unmodified from its own
 * sources into oracle/_ref/libpevsl_ref.so (TEST INFRASTRUCTURE ONLY: the
 * parity tests and the CPU baseline call it; the product never does).
 *
 * Everything here calls the reference's public C API exactly as its drivers
 * do (TESTS/Lap/LapPLanN.c, TESTS/MM/MMPLanN.c, TESTS0/Matvec/test1.c):
 * one rank, one group (ngroups = 1, groupid = 0, gl_comm = MPI_COMM_NULL).
 *
 * Random vectors: the reference's pEVSL_ParvecRand (SRC/parvec.c:65-72) is
 * renamed at compile time to oref_glibc_ParvecRand and this file provides
 * pEVSL_ParvecRand, which either calls it (glibc mode: the reference's own
 * stream) or writes the next Philox Gaussian draw (see philox_gauss.h).
 */
#include "pevsl_int.h"

#include <stdint.h>
#include <unistd.h>

#include "philox_gauss.h"
#include "pipeline.h"

void oref_glibc_ParvecRand(pevsl_Parvec *x);

static int g_rng_mode = 0;
static uint64_t g_rng_seed = 0;
static uint64_t g_rng_draw = 0;

/* mode 0: srand(seed), glibc rand() stream; mode 1: Philox Gaussian, draw 0 */
void oref_set_rng(int mode, uint64_t seed) {
  g_rng_mode = mode;
  g_rng_seed = seed;
  g_rng_draw = 0;
  srand((unsigned)seed);
}

/* The unit wrappers below start their own pEVSL instance, and pEVSL_Start
 * reseeds glibc with srand(rank) (SRC/pevsl.c:36); they restart the stream
 * the caller asked for right after it. */
static int g_unit_mode = 0;
static uint64_t g_unit_seed = 0;
void oref_set_unit_rng(int mode, uint64_t seed) {
  g_unit_mode = mode;
  g_unit_seed = seed;
}
static void unit_reseed(void) { oref_set_rng(g_unit_mode, g_unit_seed); }

uint64_t oref_rng_draws(void) { return g_rng_draw; }

void pEVSL_ParvecRand(pevsl_Parvec *x) {
  if (g_rng_mode == 1) {
    orc_gauss_vector(x->data, x->n_local, g_rng_seed, g_rng_draw);
  } else {
    oref_glibc_ParvecRand(x);
  }
  g_rng_draw++;
}

/* One-rank parcsr from a full CSR (the diag block is the whole matrix). */
static void build_parcsr(int n, const int *ia, const int *ja, const double *a, pevsl_Parcsr *A) {
  pevsl_Csr csr;
  csr.nrows = n;
  csr.ncols = n;
  csr.ia = (int *)ia;
  csr.ja = (int *)ja;
  csr.a = (double *)a;
  pEVSL_ParcsrCreate(n, n, NULL, NULL, A, MPI_COMM_WORLD);
  pEVSL_ParcsrSetup(&csr, A);
}

static FILE *devnull(void) { return fopen("/dev/null", "w"); }

/* y = A x through pEVSL_ParcsrMatvec (TESTS0/Matvec/test1.c:74-80). */
int oref_matvec(int n, const int *ia, const int *ja, const double *a, const double *x,
                double *y) {
  pevsl_Parcsr A;
  pevsl_Parvec xv, yv;
  build_parcsr(n, ia, ja, a, &A);
  pEVSL_ParvecCreate(n, n, 0, MPI_COMM_WORLD, &xv);
  pEVSL_ParvecDupl(&xv, &yv);
  memcpy(xv.data, x, (size_t)n * sizeof(double));
  pEVSL_ParcsrMatvec(&A, &xv, &yv);
  memcpy(y, yv.data, (size_t)n * sizeof(double));
  pEVSL_ParvecFree(&xv);
  pEVSL_ParvecFree(&yv);
  pEVSL_ParcsrFree(&A);
  return 0;
}

/* pEVSL_Kpmdos with ngroups = 1 (LapPLanN.c:125-131). */
int oref_kpmdos(int n, const int *ia, const int *ja, const double *a, int Mdeg, int damping,
                int nvec, const double *intv, double *mu, double *ecnt) {
  pevsl_Parcsr A;
  pevsl_Data *pevsl;
  double xintv[4] = {intv[0], intv[1], intv[2], intv[3]};
  build_parcsr(n, ia, ja, a, &A);
  pEVSL_Start(MPI_COMM_WORLD, &pevsl);
  unit_reseed();
  pEVSL_SetAParcsr(pevsl, &A);
  int ierr = pEVSL_Kpmdos(pevsl, Mdeg, damping, nvec, xintv, 1, 0, MPI_COMM_NULL, mu, ecnt);
  pEVSL_Finish(pevsl);
  pEVSL_ParcsrFree(&A);
  return ierr;
}

int oref_spslicer_kpm(double *sli, double *mu, int Mdeg, const double *intv, int n_int, int npts) {
  double xintv[4] = {intv[0], intv[1], intv[2], intv[3]};
  return pEVSL_SpslicerKpm(sli, mu, Mdeg, xintv, n_int, npts);
}

/* pEVSL_SetPolDef + overrides + pEVSL_FindPol (LapPLanN.c:214-226).
 * mu_out needs max_deg+1 entries; returns FindPol's code. */
int oref_findpol(const double *intv, int max_deg, int damping, double thresh_int,
                 double thresh_ext, int deg_in, int *type, int *deg, double *gam, double *bar,
                 double *cc, double *dd, double *mu_out) {
  pevsl_Polparams pol;
  double xintv[4] = {intv[0], intv[1], intv[2], intv[3]};
  pEVSL_SetPolDef(&pol);
  pol.damping = damping;
  pol.thresh_int = thresh_int;
  pol.thresh_ext = thresh_ext;
  pol.max_deg = max_deg;
  pol.deg = deg_in;
  int ierr = pEVSL_FindPol(xintv, &pol);
  if (ierr) {
    return ierr;
  }
  *type = pol.type;
  *deg = pol.deg;
  *gam = pol.gam;
  *bar = pol.bar;
  *cc = pol.cc;
  *dd = pol.dd;
  memcpy(mu_out, pol.mu, (size_t)(pol.deg + 1) * sizeof(double));
  pEVSL_FreePol(&pol);
  return 0;
}

/* y = p(A) v with the filter given by (deg, cc, dd, mu): pEVSL_ChebAv. */
int oref_chebav(int n, const int *ia, const int *ja, const double *a, int deg, double cc,
                double dd, const double *mu, const double *v, double *y) {
  pevsl_Parcsr A;
  pevsl_Data *pevsl;
  pevsl_Parvec vv, yv, w[3];
  pevsl_Polparams pol;
  build_parcsr(n, ia, ja, a, &A);
  pEVSL_Start(MPI_COMM_WORLD, &pevsl);
  pEVSL_SetAParcsr(pevsl, &A);
  pEVSL_SetPolDef(&pol);
  pol.deg = deg;
  pol.cc = cc;
  pol.dd = dd;
  pol.mu = (double *)mu;
  pEVSL_ParvecCreate(n, n, 0, MPI_COMM_WORLD, &vv);
  pEVSL_ParvecDupl(&vv, &yv);
  for (int i = 0; i < 3; i++) {
    pEVSL_ParvecDupl(&vv, &w[i]);
  }
  memcpy(vv.data, v, (size_t)n * sizeof(double));
  pEVSL_ChebAv(pevsl, &pol, &vv, &yv, w);
  memcpy(y, yv.data, (size_t)n * sizeof(double));
  for (int i = 0; i < 3; i++) {
    pEVSL_ParvecFree(&w[i]);
  }
  pEVSL_ParvecFree(&vv);
  pEVSL_ParvecFree(&yv);
  pEVSL_Finish(pevsl);
  pEVSL_ParcsrFree(&A);
  return 0;
}

/* pEVSL_LanTrbounds from a given start vector (MMPLanN.c:111). */
int oref_lantrbounds(int n, const int *ia, const int *ja, const double *a, int lanm, int maxit,
                     double tol, const double *vinit, int bndtype, double *lmin, double *lmax) {
  pevsl_Parcsr A;
  pevsl_Data *pevsl;
  pevsl_Parvec v0;
  build_parcsr(n, ia, ja, a, &A);
  pEVSL_Start(MPI_COMM_WORLD, &pevsl);
  unit_reseed();
  pEVSL_SetAParcsr(pevsl, &A);
  pEVSL_ParvecCreate(n, n, 0, MPI_COMM_WORLD, &v0);
  memcpy(v0.data, vinit, (size_t)n * sizeof(double));
  FILE *fs = devnull();
  int ierr = pEVSL_LanTrbounds(pevsl, lanm, maxit, tol, &v0, bndtype, lmin, lmax, fs);
  fclose(fs);
  pEVSL_ParvecFree(&v0);
  pEVSL_Finish(pevsl);
  pEVSL_ParcsrFree(&A);
  return ierr;
}

/* pEVSL_LanDosG with ngroups = 1 (LapPLanN.c:158-165). */
int oref_landos(int n, const int *ia, const int *ja, const double *a, int nvec, int msteps,
                int npts, double *xdos, double *ydos, double *neig, const double *intv) {
  pevsl_Parcsr A;
  pevsl_Data *pevsl;
  double xintv[4] = {intv[0], intv[1], intv[2], intv[3]};
  build_parcsr(n, ia, ja, a, &A);
  pEVSL_Start(MPI_COMM_WORLD, &pevsl);
  unit_reseed();
  pEVSL_SetAParcsr(pevsl, &A);
  int ierr = pEVSL_LanDosG(pevsl, nvec, msteps, npts, xdos, ydos, neig, xintv, 1, 0,
                           MPI_COMM_NULL);
  pEVSL_Finish(pevsl);
  pEVSL_ParcsrFree(&A);
  return ierr;
}

void oref_spslicer_lan(double *xi, double *yi, int n_int, int npts, double *sli) {
  pEVSL_SpslicerLan(xi, yi, n_int, npts, sli);
}

/* Number of Lanczos steps from the ChebLanNr log: the last convergence test
 * printed is at step k and the loop leaves with kdim = k+1
 * (SRC/cheblanNr.c:298,323-331). */
static int parse_its(FILE *fs) {
  char line[512];
  int its = 0;
  rewind(fs);
  while (fgets(line, sizeof line, fs)) {
    int k, nconv;
    if (sscanf(line, " k %d: nconv %d", &k, &nconv) == 2) {
      its = k + 1;
    }
  }
  return its;
}

/* pEVSL_ChebLanNr on one slice.  lam/res receive up to cap pairs, sorted
 * ascending as the drivers do (LapPLanN.c:244-245); W (n x cap, column
 * major) receives the matching eigenvectors when non-NULL. */
int oref_cheblannr(int n, const int *ia, const int *ja, const double *a, const double *intv,
                   int maxit, double tol, const double *vinit, int deg, int ptype, double gam,
                   double bar, double cc, double dd, const double *mu, int *nev, int *its,
                   double *lam, double *res, double *W, int cap) {
  pevsl_Parcsr A;
  pevsl_Data *pevsl;
  pevsl_Parvec v0;
  pevsl_Polparams pol;
  double xintv[4] = {intv[0], intv[1], intv[2], intv[3]};
  build_parcsr(n, ia, ja, a, &A);
  pEVSL_Start(MPI_COMM_WORLD, &pevsl);
  unit_reseed();
  pEVSL_SetAParcsr(pevsl, &A);
  pEVSL_SetPolDef(&pol);
  pol.deg = deg;
  pol.type = ptype;
  pol.gam = gam;
  pol.bar = bar;
  pol.cc = cc;
  pol.dd = dd;
  pol.mu = (double *)mu;
  pEVSL_ParvecCreate(n, n, 0, MPI_COMM_WORLD, &v0);
  memcpy(v0.data, vinit, (size_t)n * sizeof(double));
  int nev2 = 0;
  double *lamo = NULL, *reso = NULL;
  pevsl_Parvecs *Y = NULL;
  FILE *fs = tmpfile();
  int ierr = pEVSL_ChebLanNr(pevsl, xintv, maxit, tol, &v0, &pol, &nev2, &lamo, &Y, &reso, fs);
  *its = parse_its(fs);
  fclose(fs);
  if (ierr == 0) {
    int *ind = (int *)malloc((size_t)(nev2 > 0 ? nev2 : 1) * sizeof(int));
    sort_double(nev2, lamo, ind);
    int m = nev2 < cap ? nev2 : cap;
    for (int i = 0; i < m; i++) {
      lam[i] = lamo[i];
      res[i] = reso[ind[i]];
      if (W) {
        memcpy(W + (size_t)i * n, Y->data + (size_t)ind[i] * Y->ld, (size_t)n * sizeof(double));
      }
    }
    free(ind);
    *nev = nev2;
  }
  if (lamo) free(lamo);
  if (reso) free(reso);
  if (Y) {
    pEVSL_ParvecsFree(Y);
    free(Y);
  }
  pEVSL_ParvecFree(&v0);
  pEVSL_Finish(pevsl);
  pEVSL_ParcsrFree(&A);
  return ierr;
}

/* The whole driver run (LapPLanN.c:118-296 with the bounds step of
 * MMPLanN.c:104-118): one pEVSL instance, one group, slices sl_lo..sl_hi-1
 * in order (bounds, DOS and slicing always run in full, so the slice ends
 * and filters are those of the whole run). */
static int pipeline_range(const orc_spec *s, orc_out *o, int sl_lo, int sl_hi) {
  pevsl_Parcsr A;
  pevsl_Data *pevsl;
  pevsl_Parvec vinit;
  double xintv[4];
  double t0 = pEVSL_Wtime(), t;
  int n = s->n;
  o->status = 0;
  build_parcsr(n, s->ia, s->ja, s->a, &A);
  pEVSL_Start(MPI_COMM_WORLD, &pevsl);
  oref_set_rng(s->rng_mode, s->seed);
  pEVSL_SetAParcsr(pevsl, &A);
  FILE *fs = devnull();
  /* the start vector is drawn first, as in MMPLanN.c:106-107 */
  pEVSL_ParvecCreate(A.ncol_global, A.ncol_local, A.first_col, MPI_COMM_WORLD, &vinit);
  pEVSL_ParvecRand(&vinit);
  t = pEVSL_Wtime();
  if (s->bounds_mode == 1) {
    pEVSL_LanTrbounds(pevsl, s->lan_lanm, s->lan_maxit, s->lan_tol, &vinit, s->lan_bndtype,
                      &o->lmin, &o->lmax, fs);
  } else {
    o->lmin = s->lmin;
    o->lmax = s->lmax;
  }
  o->t_bounds = pEVSL_Wtime() - t;
  xintv[0] = s->a_lo;
  xintv[1] = s->b_hi;
  xintv[2] = o->lmin;
  xintv[3] = o->lmax;
  t = pEVSL_Wtime();
  int nsl = s->nslices;
  if (s->dos_type == 0) {
    int ierr = pEVSL_Kpmdos(pevsl, s->Mdeg, s->kpm_damping, s->nvec, xintv, 1, 0, MPI_COMM_NULL,
                            o->mu, &o->ecount);
    o->t_dos = pEVSL_Wtime() - t;
    if (ierr) {
      o->status = 100 + ierr;
    }
    t = pEVSL_Wtime();
    o->npts = (int)(10 * o->ecount);
    ierr = pEVSL_SpslicerKpm(o->sli, o->mu, s->Mdeg, xintv, nsl, o->npts);
    if (ierr && !o->status) {
      o->status = 200 + ierr;
    }
    o->t_slicer = pEVSL_Wtime() - t;
  } else {
    int npts = s->landos_npts;
    double *xdos = (double *)calloc((size_t)npts, sizeof(double));
    double *ydos = (double *)calloc((size_t)npts, sizeof(double));
    pEVSL_LanDosG(pevsl, s->nvec, s->landos_msteps, npts, xdos, ydos, &o->ecount, xintv, 1, 0,
                  MPI_COMM_NULL);
    o->t_dos = pEVSL_Wtime() - t;
    t = pEVSL_Wtime();
    o->npts = npts;
    pEVSL_SpslicerLan(xdos, ydos, nsl, npts, o->sli);
    o->t_slicer = pEVSL_Wtime() - t;
    free(xdos);
    free(ydos);
  }
  int ev_int = (int)(1 + o->ecount / ((double)nsl));
  t = pEVSL_Wtime();
  for (int sl = sl_lo; sl < sl_hi && sl < nsl; sl++) {
    pevsl_Polparams pol;
    int nev = ev_int + 2;
    int mlan = nev * 5 > s->mlan_min ? nev * 5 : s->mlan_min;
    mlan = mlan < n ? mlan : n;
    xintv[0] = o->sli[sl];
    xintv[1] = o->sli[sl + 1];
    xintv[2] = o->lmin;
    xintv[3] = o->lmax;
    pEVSL_SetPolDef(&pol);
    pol.damping = s->pol_damping;
    pol.thresh_int = s->thresh_int;
    pol.thresh_ext = s->thresh_ext;
    pol.max_deg = s->pol_max_deg;
    pEVSL_FindPol(xintv, &pol);
    o->deg[sl] = pol.deg;
    o->ptype[sl] = pol.type;
    o->gam[sl] = pol.gam;
    o->bar[sl] = pol.bar;
    int nev2 = 0;
    double *lam = NULL, *res = NULL;
    pevsl_Parvecs *Y = NULL;
    FILE *ls = tmpfile();
    int ierr = pEVSL_ChebLanNr(pevsl, xintv, mlan, s->tol, &vinit, &pol, &nev2, &lam, &Y, &res,
                               ls);
    o->its[sl] = parse_its(ls);
    fclose(ls);
    if (ierr && !o->status) {
      o->status = 300 + ierr;
    }
    int *ind = (int *)malloc((size_t)(nev2 > 0 ? nev2 : 1) * sizeof(int));
    sort_double(nev2, lam, ind);
    o->nev[sl] = nev2;
    int m = nev2 < o->cap ? nev2 : o->cap;
    for (int i = 0; i < m; i++) {
      o->lam[(size_t)sl * o->cap + i] = lam[i];
      o->res[(size_t)sl * o->cap + i] = res[ind[i]];
    }
    free(ind);
    if (lam) free(lam);
    if (res) free(res);
    if (Y) {
      pEVSL_ParvecsFree(Y);
      free(Y);
    }
    pEVSL_FreePol(&pol);
  }
  o->t_slices = pEVSL_Wtime() - t;
  fclose(fs);
  pEVSL_ParvecFree(&vinit);
  pEVSL_Finish(pevsl);
  pEVSL_ParcsrFree(&A);
  o->t_total = pEVSL_Wtime() - t0;
  return o->status;
}

int oref_pipeline(const orc_spec *s, orc_out *o) { return pipeline_range(s, o, 0, s->nslices); }

/* One or a few slices of a whole run: several processes, each with its own
 * range, reproduce a long run slice by slice in parallel.  A slice draws
 * random vectors only on a breakdown restart (SRC/cheblanNr.c:248-281), so
 * the stream a slice sees equals the one-process run's unless an earlier
 * slice restarted. */
int oref_pipeline_slices(const orc_spec *s, orc_out *o, int sl_lo, int sl_hi) {
  return pipeline_range(s, o, sl_lo, sl_hi);
}

/* ------------------------------------------------------------ B-solvers */

/* exported by SRC/lspolapprox.c:207 without a declaration in INC/ */
void pEVSL_SetupLSPolRec(int max_deg, double tol, double lmin, double lmax, pevsl_Parcsr *B,
                         void **vdata);
int pEVSL_ChebIterSetup(double lmin, double lmax, int deg, pevsl_Parcsr *A, void **data);
void pEVSL_ChebIterSolv1(double *db, double *dx, void *data);
void pEVSL_ChebIterSolv2(double *db, double *dx, void *data);
void pEVSL_ChebIterFree(void *vdata);

/* The leading members of the private LSPol_Data of SRC/lspolapprox.c:10-22,
 * in their order, to read the degree and coefficients it computed. */
typedef struct {
  int N, n, nfirst, max_deg, deg;
  double intv[2];
  double cc, dd, tol;
  double *mu;
} oref_lspol_view;

/* pEVSL_SetupLSPolRec (kind 0) / pEVSL_SetupLSPolSqrt (kind 1) on B, then
 * x = pEVSL_LSPolSol(b); mu receives the max_deg coefficients. */
int oref_lspol(int kind, int max_deg, double tol, double lmin, double lmax, int n, const int *ia,
               const int *ja, const double *a, double *mu, int *deg, double *cc, double *dd,
               const double *b, double *x) {
  pevsl_Parcsr B;
  void *data = NULL;
  build_parcsr(n, ia, ja, a, &B);
  if (kind == 0)
    pEVSL_SetupLSPolRec(max_deg, tol, lmin, lmax, &B, &data);
  else
    pEVSL_SetupLSPolSqrt(max_deg, tol, lmin, lmax, &B, &data);
  const oref_lspol_view *L = (const oref_lspol_view *)data;
  *deg = L->deg;
  *cc = L->cc;
  *dd = L->dd;
  memcpy(mu, L->mu, (size_t)max_deg * sizeof(double));
  double *bb = (double *)malloc((size_t)n * sizeof(double));
  memcpy(bb, b, (size_t)n * sizeof(double));
  pEVSL_LSPolSol(bb, x, data);
  free(bb);
  pEVSL_LSPolFree(data);
  pEVSL_ParcsrFree(&B);
  return 0;
}

/* x = pEVSL_ChebIterSolv1 (kind 1) or Solv2 (kind 2) of b on A */
int oref_chebiter(int kind, double lmin, double lmax, int deg, int n, const int *ia, const int *ja,
                  const double *a, const double *b, double *x) {
  pevsl_Parcsr A;
  void *data = NULL;
  build_parcsr(n, ia, ja, a, &A);
  pEVSL_ChebIterSetup(lmin, lmax, deg, &A, &data);
  double *bb = (double *)malloc((size_t)n * sizeof(double));
  memcpy(bb, b, (size_t)n * sizeof(double));
  memset(x, 0, (size_t)n * sizeof(double));
  if (kind == 1)
    pEVSL_ChebIterSolv1(bb, x, data);
  else
    pEVSL_ChebIterSolv2(bb, x, data);
  free(bb);
  pEVSL_ChebIterFree(data);
  pEVSL_ParcsrFree(&A);
  return 0;
}

/* y = p(A B^{-1}) v through the reference's pEVSL_ChebAv with ifGenEv
 * (SRC/chebpol.c:538-546), B-solve pEVSL_LSPolSol of the least-squares
 * 1/x on [blo, bhi] (max degree lsdeg, tolerance lstol): the CPU sample of
 * the generalized filter. */
int oref_gen_chebav(int n, const int *ia, const int *ja, const double *a, const int *ib,
                    const int *jb, const double *b, int lsdeg, double lstol, double blo, double bhi,
                    int deg, double cc, double dd, const double *mu, const double *v, double *y) {
  pevsl_Parcsr A, B;
  pevsl_Data *pevsl;
  pevsl_Parvec vv, yv, w[4];
  pevsl_Polparams pol;
  void *bsol = NULL;
  build_parcsr(n, ia, ja, a, &A);
  build_parcsr(n, ib, jb, b, &B);
  pEVSL_SetupLSPolRec(lsdeg, lstol, blo, bhi, &B, &bsol);
  pEVSL_Start(MPI_COMM_WORLD, &pevsl);
  pEVSL_SetAParcsr(pevsl, &A);
  pEVSL_SetBParcsr(pevsl, &B);
  pEVSL_SetBSol(pevsl, pEVSL_LSPolSol, bsol);
  pEVSL_SetGenEig(pevsl);
  pEVSL_SetPolDef(&pol);
  pol.deg = deg;
  pol.cc = cc;
  pol.dd = dd;
  pol.mu = (double *)mu;
  pEVSL_ParvecCreate(n, n, 0, MPI_COMM_WORLD, &vv);
  pEVSL_ParvecDupl(&vv, &yv);
  for (int i = 0; i < 4; i++) pEVSL_ParvecDupl(&vv, &w[i]);
  memcpy(vv.data, v, (size_t)n * sizeof(double));
  pEVSL_ChebAv(pevsl, &pol, &vv, &yv, w);
  memcpy(y, yv.data, (size_t)n * sizeof(double));
  for (int i = 0; i < 4; i++) pEVSL_ParvecFree(&w[i]);
  pEVSL_ParvecFree(&vv);
  pEVSL_ParvecFree(&yv);
  pEVSL_Finish(pevsl);
  pEVSL_LSPolFree(bsol);
  pEVSL_ParcsrFree(&A);
  pEVSL_ParcsrFree(&B);
  return 0;
}
