/*
 * pevsl-b200 device runtime shared by the CUDA modules: the per-process GPU
 * context (one stream, reduction scratch, device scalars, cached
 * workspaces), launch accounting, and the host-callable wrappers of the
 * kernels.  Everything is enqueued on the context stream; wrappers return 0
 * or PEVSL_ERR_CUDA and never synchronise unless their name says so.
 */
#ifndef PEVSL_B200_GPU_CUH
#define PEVSL_B200_GPU_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "internal.h"

namespace pv {

constexpr int kThreads = 256;      /* block size of the streaming kernels      */
constexpr int kMaxRedBlocks = 1184; /* 8 x 148 SMs: partial sums per reduction */
constexpr int kMaxBatch = 16;       /* entries of one batched launch            */
constexpr int kMaxEntries = 256;    /* entries of one lockstep group / persistent filter */

/* per-entry pointers / scalars of a batched launch (kernel parameters) */
struct VPtrs {
  double *p[kMaxBatch];
};
struct CPtrs {
  const double *p[kMaxBatch];
};
struct BScal {
  double v[kMaxBatch];
};
/* per-entry filter data of a batched filter degree */
struct BatchParams {
  unsigned mask;          /* active entries */
  int deg[kMaxBatch];     /* filter degree of each entry */
  double cc[kMaxBatch];   /* centre of the spectrum bounds */
  double t1[kMaxBatch];   /* 1 / dd */
  double t2[kMaxBatch];   /* 2 / dd */
};

/* device scalar slots (doubles) */
enum Slot {
  S_ALPHA = 0,
  S_BETA = 1,
  S_NRM0 = 2,
  S_NRM = 3,
  S_TMP0 = 4,
  S_TMP1 = 5,
  S_TMP2 = 6,
  S_TMP3 = 7,
  S_COUNT = 64
};
/* device int flag slots */
enum Flag { F_PASS2 = 0, F_COUNT = 16 };
/* cached workspace slots */
enum Ws {
  WS_BASIS = 0, /* Lanczos basis                              */
  WS_CHEB,      /* three recurrence vectors                   */
  WS_VEC,       /* misc vectors                               */
  WS_KPM,       /* KPM blocks                                 */
  WS_MOM,       /* KPM moments                                */
  WS_PART,      /* CGS partial products                       */
  WS_SMALL,     /* small coefficient arrays                   */
  WS_RITZ,      /* Ritz vectors                               */
  WS_RITZ2,     /* A * Ritz vectors                           */
  WS_REF1,      /* refinement sweep: A P                      */
  WS_REF2,      /* refinement sweep: refined vectors          */
  WS_H,         /* refinement sweep: small projected matrices */
  WS_GEMM,      /* gemm_tn partial tiles                      */
  WS_FILT,      /* batched filter work vectors                */
  WS_MU,        /* filter coefficients on the device          */
  WS_GROUP,     /* per-entry coefficient vectors of a group   */
  WS_ZBASIS,    /* generalized problem: Z = B V               */
  WS_GEN,       /* generalized problem: filter / KPM vectors  */
  WS_IL,        /* interleaved filter: three n x S blocks     */
  WS_ILMU,      /* interleaved filter: per-degree coefficients */
  WS_COUNT
};

struct Ctx {
  bool ready = false;
  int device = 0;
  int sms = 148;
  cudaStream_t stream = nullptr;
  double *red = nullptr;       /* kMaxRedBlocks * 64 partial sums */
  unsigned *cnt = nullptr;     /* last-block counters, kept at 0  */
  double *dscal = nullptr;     /* S_COUNT device scalars          */
  double *hscal = nullptr;     /* pinned mirror of dscal          */
  int *dflag = nullptr;        /* F_COUNT device flags            */
  double *gscal = nullptr;     /* 4 * kMaxEntries per-entry device scalars */
  double *hgscal = nullptr;    /* pinned mirror of gscal          */
  int *gflag = nullptr;        /* kMaxEntries per-entry device flags       */
  void *htab = nullptr;        /* pinned staging of the persistent filter table, kTabSlots slots */
  void *dtab = nullptr;        /* device copies of those tables   */
  cudaEvent_t tab_ev[4] = {};  /* copy of slot i done             */
  int tab_next = 0;
  unsigned *bar = nullptr;     /* grid barrier: count, generation, error   */
  void *ws[WS_COUNT] = {};
  size_t wsz[WS_COUNT] = {};
  uint64_t launches = 0;
  int sticky_error = 0;
};

Ctx &ctx();
int ensure();                 /* initialise the context; 0 or PEVSL_ERR_CUDA */
int fail(cudaError_t e, const char *what);
int launched(const char *what); /* count a launch and check for errors */
/* point the L2 persisting window at [base, base+bytes) if enabled */
void l2_window(const void *base, size_t bytes);
int sync();
void *ws(int slot, size_t bytes);
int memcpy_async(void *dst, const void *src, size_t bytes);
/* scalar slots: copy device slots [first, first+count) to the pinned mirror
 * and wait; returns pointer into the mirror or NULL */
const double *fetch_scalars(int first, int count);

inline unsigned grid_for(long n, int per_thread = 1) {
  long b = (n + (long)kThreads * per_thread - 1) / ((long)kThreads * per_thread);
  if (b < 1) b = 1;
  if (b > kMaxRedBlocks) b = kMaxRedBlocks;
  return (unsigned)b;
}

/* ---------------------------------------------------------------- BLAS1 */
int vfill(double *x, long n, double v);
int vcopy(const double *x, double *y, long n);
int vscal(double *x, long n, double a);
int vaxpy(long n, double a, const double *x, double *y);
/* y += sign * (*coef) * x, coef in device memory */
int vaxpy_dev(long n, const double *coef, double sign, const double *x, double *y);
/* x *= 1 / (*s), s in device memory */
int vscal_inv_dev(long n, const double *s, double *x);
/* *out = <x, y> (deterministic); out in device memory */
int vdot(long n, const double *x, const double *y, double *out);
/* *out = ||x|| */
int vnrm2(long n, const double *x, double *out);
/* *out = sum x */
int vsum(long n, const double *x, double *out);
/* y -= (*coef) x  then  *nrm = ||y||  (one pass) */
int vaxpy_dev_nrm2(long n, const double *coef, const double *x, double *y, double *nrm);
/* out[c] = <X[:,c], Y[:,c]> for c < m, column-major with leading dims */
int vdot_cols(long n, int m, const double *X, long ldx, const double *Y, long ldy, double *out);
/* X[:,c] *= s[c] for c < m (s device) */
int vscal_cols(long n, int m, double *X, long ldx, const double *s);
/* Y[:,c] -= lam[c] X[:,c] (lam device) */
int vaxpy_cols(long n, int m, const double *lam, const double *X, long ldx, double *Y, long ldy);

/* ---------------------------------------------------------------- random */
/* Philox Gaussian draws m0 .. m0+nv-1 into columns of X: X[i*rs + c*cs]. */
int rand_gauss(double *X, long n, int nv, long rs, long cs, uint64_t seed, uint64_t m0);

/* ---------------------------------------------------------------- sparse */
int spmv(const pevsl_devcsr *A, const double *x, double *y);
/* One degree of the Chebyshev filter recurrence (fused SpMV):
 *   w = ((A vk - cc vk) * t) - vkm1   (vkm1 may be NULL)
 *   vkp1 = w;  y = first ? mu0 * vk + muk * w : y + muk * w            */
int cheb_step(const pevsl_devcsr *A, const double *vk, const double *vkm1, double *vkp1,
              double *y, double cc, double t, double mu0, double muk, int first);
/* The degree of the generalized filter (SRC/chebpol.c:543-546): the SpMV
 * reads x = B^{-1} vk, the recurrence uses vk; tmp (n doubles) is used
 * only by the row-group kernels. */
int cheb_step_x(const pevsl_devcsr *A, const double *x, const double *vk, const double *vkm1,
                double *vkp1, double *y, double cc, double t, double mu0, double muk, int first,
                double *tmp);
/* Fused steps of the Chebyshev iterations for B x = b
 * (EXTERNAL/ITERSOL/chebiter.c): first kind r = b - B x; p = bet p + r;
 * xnew = x + alp p.  Second kind x += d; r -= B d; dnew = c1 d + c2 r. */
int chebiter1_step(const pevsl_devcsr *B, const double *b, const double *x, double *p, double *xnew,
                   double bet, double alp, double *tmp);
int chebiter2_step(const pevsl_devcsr *B, const double *d, double *x, double *r, double *dnew,
                   double c1, double c2, double *tmp);
/* Same recurrence when A x is computed by a user callback: ax = A vk. */
int cheb_combine(long n, const double *ax, const double *vk, const double *vkm1, double *vkp1,
                 double *y, double cc, double t, double mu0, double muk, int first);
/* One KPM degree for s interleaved vectors (row-major n x ld blocks):
 *   Xkp1 = (A Xk - ctr Xk) sc - Xkm1;   mom[c] = <Xkp1[:,c], V0[:,c]>   */
int kpm_step(const pevsl_devcsr *A, int s, int ld, const double *Xk, const double *Xkm1,
             double *Xkp1, const double *V0, double ctr, double sc, double *mom);
/* out[c] = sum_b partials[b*s + c] over nb blocks, fixed order */
int col_reduce(const double *partials, int nb, int s, double *out);
/* Column sums of squares of an interleaved block: out[c] = sum_i X[i*ld+c]^2 */
int block_colnorm2(long n, int s, int ld, const double *X, double *out);
/* X[i*ld+c] *= 1/sqrt(nrm2[c]) */
int block_normalize(long n, int s, int ld, double *X, const double *nrm2);

/* ---------------------------------------------------------------- dense */
/* w[j] = sum_i V[i + j*ldv] v[i], j < k (two-stage, deterministic); kernels
 * return early when skip != NULL and *skip == 0 */
int gemvT(long n, int k, const double *V, long ldv, const double *v, double *w, const int *run);
/* v -= V w; *nrm = ||v||; if flag: *flag = (*nrm <= eta * *nrm_old), then
 * *nrm_old = *nrm.  Skipped when run != NULL and *run == 0. */
int gemv_sub_nrm(long n, int k, const double *V, long ldv, const double *w, double *v,
                 double *nrm, const int *run, int *flag_out, double *nrm_old, double eta);
/* ---------------------------------------------------------------- batched
 * Entry s of every call uses pointer p[s] / scalar v[s] and length
 * len.n[s] (leading dimension len.ld[s] for basis blocks); only entries
 * whose bit is set in mask run.  Per-entry outputs go to out[s]. */
struct BLen {
  long n[kMaxBatch];
  long ld[kMaxBatch];
};
BLen blen_uniform(long n, long ld, int S);
int b_axpy(const BLen &len, int S, CPtrs x, VPtrs y, BScal a, unsigned mask);
int b_scal(const BLen &len, int S, VPtrs x, BScal a, unsigned mask);
int b_dot(const BLen &len, int S, CPtrs x, CPtrs y, double *out, int fin, unsigned mask);
int b_axpy_dev_nrm2(const BLen &len, int S, const double *coef, CPtrs x, VPtrs y, double *nrm,
                    unsigned mask);
/* w[s*ldw + j] = <V_s(:,j), v_s>, j < k */
int b_gemvT(const BLen &len, int S, int k, CPtrs V, CPtrs v, double *w, long ldw, const int *run,
            unsigned mask);
/* v_s -= V_s w_s; nrm[s] = ||v_s||; flag/nrm_old per entry as gemv_sub_nrm */
int b_gemv_sub_nrm(const BLen &len, int S, int k, CPtrs V, const double *w, long ldw, VPtrs v,
                   double *nrm, const int *run, int *flag_out, double *nrm_old, double eta,
                   unsigned mask);
/* one filter degree (SRC/chebpol.c:538-568) for nb <= kMaxEntries
 * independent vectors, each on its own matrix A (entries on one matrix read
 * it once per launch): entry e's pointers are FP64 vectors, or FP32 ones
 * when fp32 (then the last degree sets yout, the FP64 result) */
struct ChebEntry {
  const pevsl_devcsr *A;
  const void *vk, *vkm1; /* vkm1 NULL at the first degree */
  void *vkp1, *y;        /* vkp1 may alias vkm1 */
  double *yout;
  double cc, t, mu0, muk;
  int first;
};
int cheb_step_batch(int nb, const ChebEntry *e, bool fp32);
/* the same degree for S in {2,4,8,16} vectors of one problem held
 * row-interleaved (X[i*S + s]); mu0[s], muk[s] on the device; Xkp1 may
 * alias Xkm1 */
int cheb_step_il(const pevsl_devcsr *A, int S, const double *Xk, const double *Xkm1, double *Xkp1,
                 double *Y, double cc, double t, const double *mu0, const double *muk, int first);
/* the same with the SpMV reading Xg instead of Xk (generalized filter) */
int cheb_step_il_x(const pevsl_devcsr *A, int S, const double *Xg, const double *Xk,
                   const double *Xkm1, double *Xkp1, double *Y, double cc, double t,
                   const double *mu0, const double *muk, int first);
/* degree k with a deferred accumulator: Y takes the terms of degrees
 * k-ny+1 .. k (ny in 0..3; 0 leaves Y untouched, neither read nor
 * written), whose vectors are X_k (Xkp1), X_{k-1} (Xk) and X_{k-2} (Xkm1);
 * their mu rows lie at muk, muk - S, muk - 2S.  fresh: Y holds nothing yet
 * and the sum starts from mu_0 X_0 (X_0 = Xk when ny = 1, Xkm1 when
 * ny = 2).  The multiply-adds run in degree order, so Y ends bit-identical
 * to the one-degree-at-a-time sum. */
int cheb_step_il_y(const pevsl_devcsr *A, int S, const double *Xg, const double *Xk,
                   const double *Xkm1, double *Xkp1, double *Y, double cc, double t,
                   const double *mu0, const double *muk, int ny, int fresh);
/* X[i*S + s] = xs[s][i] (S <= kMaxBatch), and ys[s][i] = X[i*S + s] for
 * the first cols columns */
int il_pack(long n, int S, const double *const *xs, double *X);
int il_unpack(long n, int S, int cols, const double *X, double *const *ys);
/* bytes per stored entry that the CSR-stream kernels read for A: 3 for the
 * packed form (int16 column offset + uint8 value index), else 12 (int32
 * column + FP64 value) or 8 (FP32 value) */
double entry_bytes(const pevsl_devcsr *A, bool fp32, bool batch = false);
/* bytes per entry the interleaved kernel reads for A (3 packed, 12 plain) */
double il_entry_bytes(const pevsl_devcsr *A);
/* L2 persistence window over the part of A the kernels read (if enabled) */
void matrix_window(const pevsl_devcsr *A);
/* choose the CSR-stream rows per lane of a matrix by timing (once) */
int stream_tune(pevsl_devcsr *A);
/* choose the CSR or ELL form of the one- and two-vector filter degrees of a
 * packed matrix with an ELL copy by timing both (at set-up) */
int filter_tune(pevsl_devcsr *A);

/* One entry of the persistent filter: y = p(A) x for its own matrix and
 * polynomial (mu on the device).  FP64 entries: b0, b1 are two work vectors
 * of n doubles and acc == y.  FP32 entries (a = the FP32 values): x is the
 * FP32 copy of the input, b0, b1, acc are FP32 and the last degree writes
 * y in FP64. */
struct FiltDev {
  const int *ia, *ja;
  const void *a;
  int n, deg, fp32, pad;
  double cc, t1, t2;
  const double *mu;
  const void *x;
  void *b0, *b1, *acc;
  double *y;
};
constexpr size_t kFiltTabBytes = sizeof(FiltDev) * kMaxEntries + sizeof(int) * (kMaxEntries + 8);
constexpr int kTabSlots = 4; /* staging slots: a slot is reused only after its copy ran */
/* All degrees of ne <= kMaxEntries filters in one cooperative launch: the
 * blocks sweep the (entry, 256-row block) items of every entry whose degree
 * has not been reached, then meet at a grid barrier before the next degree.
 * The entries must be sorted by non-increasing degree.  Returns 0,
 * PEVSL_ERR_CUDA, or PEVSL_ERR_ARG if the launch cannot be co-resident. */
int cheb_filter_persistent(int ne, const FiltDev *entries, int maxdeg);
/* the barrier's timeout flag of the last persistent filter (read after a sync) */
int persistent_filter_error();
void set_barrier_spins(unsigned spins);
int seed_barrier_arrivals(unsigned count);

/* ---------------------------------------------------------------- FP32 (mixed) */
int csr_make_fp32(pevsl_devcsr *A); /* FP32 copy of the values, once */
int kpm_step32(const pevsl_devcsr *A, int s, int ld, const float *Xk, const float *Xkm1,
               float *Xkp1, const float *V0, double ctr, double sc, double *mom);
int cvt_f64_f32(long n, const double *x, float *y);

/* C = V(:, 0:k)' W(:, 0:m)  (k x m, column-major ldc); deterministic */
int gemm_tn(long n, int k, int m, const double *V, long ldv, const double *W, long ldw, double *C,
            long ldc);
/* U = V(:, 0:k) Y  (n x m, V column-major ldv, Y k x m column-major ldy) */
int gemm_nn(long n, int k, int m, const double *V, long ldv, const double *Y, long ldy,
            double *U, long ldu);

}  // namespace pv

#endif
