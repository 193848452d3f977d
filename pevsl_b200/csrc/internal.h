/*
 * pevsl-b200 internal interfaces shared by the host C modules and the CUDA
 * modules.  Not installed; callers use include/pevsl.h and pevsl_b200.h.
 */
#ifndef PEVSL_B200_INTERNAL_H
#define PEVSL_B200_INTERNAL_H

#include <stdint.h>

#include "pevsl.h"
#include "pevsl_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ instance
 * pEVSL_Start allocates this block; the caller sees &inst->pub. */
typedef struct pevsl_inst {
  pevsl_Data pub; /* first member: pevsl_Data* <-> pevsl_inst* */
  pevsl_Stat stat;
  pevsl_Matvec amv, bmv;
  pevsl_Bsol bsol;
  pevsl_Ltsol ltsol;
  int last_its, last_nconv;
  double phase_ms[8];
  int precision; /* PEVSL_PREC_FP64 or PEVSL_PREC_MIXED */
  /* sum across the groups of a split KPM (pEVSL_B200_SetGroupReduce) */
  void (*group_reduce)(double *buf, int count, void *ctx);
  void *group_reduce_ctx;
} pevsl_inst;

static inline pevsl_inst *pevsl_inst_of(pevsl_Data *d) { return (pevsl_inst *)d; }

/* ------------------------------------------------------------------ device CSR
 * pevsl_Parcsr.comm_handle points at this block after pEVSL_ParcsrSetup; its
 * first member is a zeroed commHandle so the pointer type stays valid. */
#define PEVSL_DEVCSR_MAGIC 0x42323030u /* "B200" */
typedef struct pevsl_devcsr {
  commHandle zero_handle;
  uint32_t magic;
  int nrows, ncols;
  long long nnz;
  int *ia;    /* device, nrows+1 */
  int *ja;    /* device, nnz     */
  double *a;  /* device, nnz     */
  float *a32; /* device fp32 copy, made on first use */
  int max_row_nnz;
  double avg_row_nnz;
  int lanes; /* threads per row in the row-group SpMV kernels */
  int stream_r; /* rows per lane of the CSR-stream kernels, 0 until tuned */
  size_t bytes; /* size of the one device block holding a, ja, ia */
  /* packed copy of the entries (NULL when the matrix does not qualify):
   * pdj = column - 32 * (row / 32) as int16, pvi = index of the value in
   * pvtab (at most 256 distinct values, exact doubles; pvtab32 their FP32
   * roundings), all in one device block of pbytes bytes */
  short *pdj;
  unsigned char *pvi;
  double *pvtab;
  float *pvtab32;
  int pnv;
  size_t pbytes;
  /* the same packed entries in ELL layout (NULL unless every row has at
   * most ew <= 16 entries and the padding stays under a quarter): row r's
   * j-th entry at (r / 32) * 32 * ew + j * 32 + r % 32; padding has
   * edj = INT16_MIN.  A row's entries are addressed from r alone. */
  short *edj;
  unsigned char *evi;
  int ew;
  /* the filter-degree forms chosen for this matrix by timing both on the
   * GPU at set-up (filter_tune): one vector and groups of two on the ELL
   * copy (1) or on the packed CSR entries (0) */
  int ell1, ell2;
} pevsl_devcsr;

/* The device matrix behind a Parcsr, or NULL if it was never set up here. */
pevsl_devcsr *pevsl_devcsr_of(const pevsl_Parcsr *A);

/* The built-in matrix of an instance when Amv is the parcsr callback, else
 * NULL (a user matvec is installed). */
pevsl_devcsr *pevsl_builtin_A(pevsl_Data *pevsl);

/* ------------------------------------------------------------------ host helpers
 * (host C modules) */
double pevsl_now(void);
int pevsl_check_intv(const double *intv, FILE *fstats);
void pevsl_dampcf(int m, int damping, double *jac);
void pevsl_chebxPltd(int m, const double *mu, int npts, const double *xi, double *yi);
/* eigen-decomposition of a symmetric tridiagonal matrix; Z may be NULL */
int pevsl_tridiag_eig(int n, const double *d, const double *e, double *w, double *Z);
/* eigenvalues (ascending) + eigenvectors of the eigenvalues with ascending
 * indices sel[0..nsel) into Zsel (n x nsel, column major) */
int pevsl_tridiag_eig_sel(int n, const double *d, const double *e, double *w, int nsel,
                          const int *sel, double *Zsel);
/* eigen-decomposition of a dense symmetric matrix (column major) */
int pevsl_dense_symeig(int n, const double *A, int lda, double *Q, int ldq, double *lam);
/* eigenpairs with eigenvalues in [lo, hi] of a dense symmetric matrix
 * (Householder tridiagonalisation + tridiagonal QR); *m of them */
int pevsl_dense_symeig_range(int n, const double *H, int ldh, double lo, double hi, int *m,
                             double *lam, double *Z, int ldz);
/* eigenpairs with eigenvalues in [lo, hi] of the pencil (H, G), G a Gram
 * matrix with unit diagonal; dependent columns are dropped */
int pevsl_gen_symeig_range(int m, const double *H, const double *G, int ld, double lo, double hi,
                           int *nout, double *lam, double *Z, int ldz);
void pevsl_simpson(const double *xi, double *yi, int npts);
/* least-squares Chebyshev coefficients of ffun on [a, b] (mu has max_deg
 * entries; the polynomial has degree *deg) */
int pevsl_lspol_coefs(double (*ffun)(double), int max_deg, double tol, double a, double b,
                      double *mu, int *deg, double *cc, double *dd);
double (*pevsl_lspol_rec(void))(double);
double (*pevsl_lspol_isqrt(void))(double);

/* local vector length of a least-squares / Chebyshev-iteration B-solver */
int pevsl_lspol_size(const void *lspol);
int pevsl_chebiter_size(const void *cheb);

/* ------------------------------------------------------------------ generalized
 * problem (gpu_gen.cu): the ifGenEv branches of the solvers */
int pevsl_gen_kpm_moments(pevsl_Data *pevsl, int Mdeg, const double *jac, double ctr, double wid,
                          double beta1, double beta2, int vec_start, int vec_end, double *mu,
                          double *tcnt);
int pevsl_gen_landos_lanczos(pevsl_Data *pevsl, int maxit, const double *vinit, double *dT,
                             double *eT);
int pevsl_gen_lantrbounds(pevsl_Data *pevsl, int lanm, int maxit, double tol, pevsl_Parvec *vinit,
                          int bndtype, double *lammin, double *lammax, FILE *fstats);
int pevsl_gen_cheblannr(pevsl_Data *pevsl, double *intv, int maxit, double tol, pevsl_Parvec *vinit,
                        pevsl_Polparams *pol, int *nevOut, double **lamo, pevsl_Parvecs **Wo,
                        double **reso, int *its, FILE *fstats);
/* slices of one generalized problem in lockstep; 1 when not applicable */
int pevsl_gen_cheblannr_lockstep(pevsl_Data *pevsl, int ns, const double *intvs, const int *maxits,
                                 double tol, pevsl_Parvec *vinit, pevsl_Polparams *pols,
                                 int *nevOut, double **lamo, pevsl_Parvecs **Wo, double **reso,
                                 int *its, int *status, FILE *fstats);

/* RNG state (host side; rng.cu owns the device generator) */
int pevsl_rng_mode(void);
uint64_t pevsl_rng_seed(void);
uint64_t pevsl_rng_take(uint64_t ndraws); /* returns first draw index */
/* Fill n doubles at dev (device/managed) with the next random vector. */
int pevsl_rand_vector_dev(double *dev, int n);
/* Fill nv column-interleaved vectors X[i*ld + c], c < nv, with the next nv
 * draws (draw order = column order), row-interleaved layout. */
int pevsl_rand_block_dev(double *X, int n, int nv, int ld);

#ifdef __cplusplus
}
#endif

#endif
