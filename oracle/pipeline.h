/*
 * Shared description of one spectrum-slicing run, used by both CPU checkers
 * (TEST INFRASTRUCTURE ONLY):
 *   - oracle/ref_glue.c drives the reference pEVSL sources compiled into
 *     oracle/_ref/ through the reference's own public API;
 *   - oracle/pevsl_oracle.c is the plain-C restatement of the same path.
 * The run is the one the reference drivers perform: bounds (given, or
 * thick-restart Lanczos as in TESTS/MM/MMPLanN.c:111), density of states
 * (KPM as in TESTS/Lap/LapPLanN.c:125-151, or Lanczos DOS as in :157-176),
 * then FindPol + ChebLanNr on every slice (LapPLanN.c:197-240).
 */
#ifndef ORACLE_PIPELINE_H
#define ORACLE_PIPELINE_H

#include <stdint.h>

typedef struct {
  /* matrix: square CSR, 0-based, all rows (one rank) */
  int n;
  const int *ia;
  const int *ja;
  const double *a;
  /* interval of interest and number of slices */
  double a_lo, b_hi;
  int nslices;
  /* bounds: 0 = use lmin/lmax below, 1 = pEVSL_LanTrbounds */
  int bounds_mode;
  double lmin, lmax;
  int lan_lanm, lan_maxit, lan_bndtype;
  double lan_tol;
  /* density of states: 0 = KPM, 1 = Lanczos DOS */
  int dos_type;
  int Mdeg, kpm_damping, nvec;
  int landos_msteps, landos_npts;
  /* filter design (pEVSL_SetPolDef, then these overrides) */
  int pol_damping, pol_max_deg;
  double thresh_int, thresh_ext;
  /* ChebLanNr */
  double tol;
  int mlan_min; /* mlan = min(max(5*nev, mlan_min), n) */
  /* random vectors: 0 = glibc rand() after srand(seed), 1 = Philox Gaussian */
  int rng_mode;
  uint64_t seed;
} orc_spec;

typedef struct {
  /* caller-allocated outputs */
  int cap;      /* eigenpair capacity per slice */
  double *mu;   /* [Mdeg+1] KPM moments (unused for Lanczos DOS) */
  double *sli;  /* [nslices+1] slice endpoints */
  int *deg;     /* [nslices] filter degree */
  int *ptype;   /* [nslices] filter type 0/1/2 */
  double *gam;  /* [nslices] */
  double *bar;  /* [nslices] */
  int *nev;     /* [nslices] accepted eigenpairs */
  int *its;     /* [nslices] Lanczos steps taken (k+1 at exit) */
  double *lam;  /* [nslices*cap] eigenvalues, ascending within a slice */
  double *res;  /* [nslices*cap] residual norms matching lam */
  /* scalar outputs */
  double lmin, lmax, ecount;
  int npts;
  int status;
  double t_bounds, t_dos, t_slicer, t_slices, t_total;
} orc_out;

#endif
