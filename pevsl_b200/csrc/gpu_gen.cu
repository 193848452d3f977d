/*
 * The generalized problem A x = lambda B x (B symmetric positive definite)
 * on the GPU: the ifGenEv branches of the slicing path and the B-solvers
 * the reference offers without external libraries.
 *
 *   B^{-1}, B^{-1/2} by least squares   pEVSL_SetupLSPolSqrt/Rec, pEVSL_LSPolSol
 *                                       SRC/lspolapprox.c:161-322
 *   Chebyshev iteration for B x = b     pEVSL_ChebIterSetup/Solv1/Solv2
 *                                       EXTERNAL/ITERSOL/chebiter.c:77-308
 *   generalized filter                  SRC/chebpol.c:538-546
 *   KPM DOS                             SRC/kpmdos.c:104-137
 *   Lanczos DOS                         SRC/landos.c:134-262
 *   spectrum bounds                     SRC/lantrbnd.c:74-397
 *   filtered Lanczos                    SRC/cheblanNr.c:125-448
 *
 * The Lanczos solvers keep two bases, V and Z = B V, and orthogonalise in
 * the B inner product (CGS_DGKS2, SRC/miscla.c:248-263: two passes, no
 * test).  B^{-1} and L^{-T} are the installed solve callbacks (SetBSol,
 * SetLTSol) called with device pointers; the least-squares and Chebyshev
 * solvers of this file are recognised and run asynchronously on the
 * library stream: a least-squares solve is the fused Chebyshev-degree
 * kernel on B (the same recurrence as the filter), a Chebyshev iteration
 * one fused SpMV-plus-update kernel per step.
 */
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "gpu.cuh"
#include "pevsl_itsol.h"

using namespace pv;

/* ------------------------------------------------------------ solver data */
struct pevsl_lspol {
  int N, n, nfirst;
  int max_deg, deg;
  double intv[2], cc, dd, tol;
  double *mu;          /* host, max_deg */
  pevsl_devcsr *B;
  double *wk;          /* device: 3 n doubles */
  MPI_Comm comm;
};

struct pevsl_chebiter {
  double lb, ub;
  int deg;
  int N, n, nfirst;
  pevsl_devcsr *A;
  double *wk;          /* device: 4 n doubles (r, two p/d/x buffers, tmp) */
  MPI_Comm comm;
  size_t n_chebmv;
  double t_chebmv;     /* seconds of device time, of the solves read so far */
  cudaEvent_t ev[2 * 32]; /* start/stop pairs of up to 32 solves not yet read */
  int used;
  bool ev_ok;
};

namespace {

/* y = sum_k mu[k] T_k((M - cc)/dd) v on a device CSR: the filter
 * recurrence (pnav, SRC/lspolapprox.c:235-283).  w holds 3 n doubles; y
 * may alias v. */
int cheb_series(const pevsl_devcsr *M, const double *mu, int m, double cc, double dd,
                const double *v, double *y, double *w) {
  const long n = M->nrows;
  if (y == v) {
    if (vcopy(v, w + 2 * n, n)) return PEVSL_ERR_CUDA;
    v = w + 2 * n;
  }
  if (m <= 0) {
    if (vcopy(v, y, n)) return PEVSL_ERR_CUDA;
    return vscal(y, n, mu[0]);
  }
  double *buf[2] = {w, w + n};
  const double *vk = v, *vkm1 = nullptr;
  for (int k = 1; k <= m; k++) {
    double *vkp1 = k <= 2 ? buf[k - 1] : const_cast<double *>(vkm1);
    const double t = (k == 1 ? 1.0 : 2.0) / dd;
    if (cheb_step(M, vk, vkm1, vkp1, y, cc, t, mu[0], mu[k], k == 1)) return PEVSL_ERR_CUDA;
    vkm1 = vk;
    vk = vkp1;
  }
  return 0;
}

int lspol_apply(pevsl_lspol *L, const double *b, double *x) {
  if (!L || !L->B) return PEVSL_ERR_ARG;
  return cheb_series(L->B, L->mu, L->deg, L->cc, L->dd, b, x, L->wk);
}

/* Chebyshev iteration, first kind (EXTERNAL/ITERSOL/chebiter.c:121-197),
 * zero initial guess: x = alp b, then deg - 1 fused steps.  The last
 * residual of the reference (computed after the last update, used only for
 * its convergence history) is not formed. */
int chebiter1(pevsl_chebiter *C, const double *b, double *x) {
  const long n = C->n;
  if (C->deg < 1) return 0;
  const double d = (C->ub + C->lb) * 0.5, c = (C->ub - C->lb) * 0.5;
  double *p = C->wk, *xb[2] = {C->wk + n, C->wk + 2 * n}, *tmp = C->wk + 3 * n;
  double alp = 2.0 / d;
  if (vcopy(b, p, n)) return PEVSL_ERR_CUDA;
  double *xc = C->deg == 1 ? x : xb[0];
  if (vcopy(b, xc, n) || vscal(xc, n, alp)) return PEVSL_ERR_CUDA;
  for (int i = 1; i < C->deg; i++) {
    const double t = c * alp * 0.5, bet = t * t;
    alp = 1.0 / (d - bet);
    double *xn = i == C->deg - 1 ? x : xb[i & 1];
    if (chebiter1_step(C->A, b, xc, p, xn, bet, alp, tmp)) return PEVSL_ERR_CUDA;
    xc = xn;
    C->n_chebmv++;
  }
  return 0;
}

/* Chebyshev iteration, second kind (EXTERNAL/ITERSOL/chebiter.c:204-262):
 * x = 0, r = b, d = b / theta, then deg fused steps. */
int chebiter2(pevsl_chebiter *C, const double *b, double *x) {
  const long n = C->n;
  const double alpha = C->lb, beta = C->ub;
  const double theta = (beta + alpha) * 0.5, delta = (beta - alpha) * 0.5;
  const double sigma = theta / delta;
  double rho = 1.0 / sigma;
  double *r = C->wk, *db[2] = {C->wk + n, C->wk + 2 * n}, *tmp = C->wk + 3 * n;
  if (vfill(x, n, 0.0) || vcopy(b, r, n) || vcopy(r, db[0], n) || vscal(db[0], n, 1.0 / theta))
    return PEVSL_ERR_CUDA;
  for (int i = 0; i < C->deg; i++) {
    const double rho1 = 1.0 / (2.0 * sigma - rho);
    if (chebiter2_step(C->A, db[i & 1], x, r, db[(i + 1) & 1], rho1 * rho, 2.0 * rho1 / delta, tmp))
      return PEVSL_ERR_CUDA;
    rho = rho1;
    C->n_chebmv++;
  }
  return 0;
}

/* device time of the queued solves: read (one wait) when the 32 pairs
 * are used up, and before the statistics are printed */
void chebiter_flush(pevsl_chebiter *C) {
  if (!C->ev_ok || C->used == 0) return;
  cudaEventSynchronize(C->ev[2 * C->used - 1]);
  for (int i = 0; i < C->used; i++) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, C->ev[2 * i], C->ev[2 * i + 1]) == cudaSuccess)
      C->t_chebmv += 1e-3 * ms;
  }
  C->used = 0;
}

bool capturing() {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  return cudaStreamIsCapturing(ctx().stream, &cs) == cudaSuccess &&
         cs != cudaStreamCaptureStatusNone;
}

/* a solve inside a captured graph is not timed (its events would belong to
 * the capture) */
int chebiter_time(pevsl_chebiter *C, int (*f)(pevsl_chebiter *, const double *, double *),
                  const double *b, double *x) {
  const bool timed = C->ev_ok && !capturing();
  if (timed) {
    if (C->used == 32) chebiter_flush(C);
    cudaEventRecord(C->ev[2 * C->used], ctx().stream);
  }
  const int st = f(C, b, x);
  if (timed) cudaEventRecord(C->ev[2 * C->used++ + 1], ctx().stream);
  return st;
}

/* ------------------------------------------------------------ B operations */

/* y = F(x) through a solve callback: the library's own solvers are queued
 * on the stream; a user callback gets settled device pointers and must
 * finish before returning. */
int call_solver(SVFunc f, void *data, const double *x, double *y) {
  if (!f) return PEVSL_ERR_ARG;
  if (f == pEVSL_LSPolSol) return lspol_apply((pevsl_lspol *)data, x, y);
  if (f == pEVSL_ChebIterSolv1 || f == pEVSL_ChebIterSolv2) {
    pevsl_chebiter *C = (pevsl_chebiter *)data;
    if (!C || !C->A) return PEVSL_ERR_ARG;
    return chebiter_time(C, f == pEVSL_ChebIterSolv1 ? chebiter1 : chebiter2, x, y);
  }
  if (sync()) return PEVSL_ERR_CUDA;
  f(const_cast<double *>(x), y, data);
  return fail(cudaDeviceSynchronize(), "user solve");
}

int apply_B(pevsl_Data *pevsl, const double *x, double *y) {
  pevsl->stats->n_mvB++;
  if (!pevsl->Bmv || !pevsl->Bmv->func) return PEVSL_ERR_NOMATVEC;
  if (pevsl->Bmv->func == pEVSL_ParcsrMatvec0) {
    pevsl_devcsr *B = pevsl_devcsr_of((const pevsl_Parcsr *)pevsl->Bmv->data);
    if (B) return spmv(B, x, y);
  }
  if (sync()) return PEVSL_ERR_CUDA;
  pevsl->Bmv->func(const_cast<double *>(x), y, pevsl->Bmv->data);
  return fail(cudaDeviceSynchronize(), "user B matvec");
}

int solve_B(pevsl_Data *pevsl, const double *x, double *y) {
  pevsl->stats->n_svB++;
  if (!pevsl->Bsol) return PEVSL_ERR_ARG;
  return call_solver(pevsl->Bsol->func, pevsl->Bsol->data, x, y);
}

int solve_LT(pevsl_Data *pevsl, const double *x, double *y) {
  pevsl->stats->n_svLT++;
  if (!pevsl->LTsol) return PEVSL_ERR_ARG;
  return call_solver(pevsl->LTsol->func, pevsl->LTsol->data, x, y);
}

int apply_Ag(pevsl_Data *pevsl, const double *x, double *y) {
  pevsl_devcsr *A = pevsl_builtin_A(pevsl);
  pevsl->stats->n_mvA++;
  if (A) return spmv(A, x, y);
  if (!pevsl->Amv || !pevsl->Amv->func) return PEVSL_ERR_NOMATVEC;
  if (sync()) return PEVSL_ERR_CUDA;
  pevsl->Amv->func(const_cast<double *>(x), y, pevsl->Amv->data);
  return fail(cudaDeviceSynchronize(), "user matvec");
}

/* CGS_DGKS2 (SRC/miscla.c:248-263): two passes of v -= Q (P' v), P and Q
 * n x k column blocks with leading dimension ld */
int cgs2(long n, long ld, int k, const double *Q, const double *P, double *v) {
  double *w = (double *)ws(WS_SMALL, sizeof(double) * (size_t)(k + 1));
  if (!w) return PEVSL_ERR_NOMEM;
  double *junk = ctx().dscal + S_TMP3;
  for (int pass = 0; pass < 2; pass++) {
    if (gemvT(n, k, P, ld, v, w, nullptr)) return PEVSL_ERR_CUDA;
    if (gemv_sub_nrm(n, k, Q, ld, w, v, junk, nullptr, nullptr, nullptr, 0.0)) return PEVSL_ERR_CUDA;
  }
  return 0;
}

/* <x, y> to the host */
int dot_host(long n, const double *x, const double *y, double *out) {
  if (vdot(n, x, y, ctx().dscal + S_TMP0)) return PEVSL_ERR_CUDA;
  const double *h = fetch_scalars(S_TMP0, 1);
  if (!h) return PEVSL_ERR_CUDA;
  *out = h[0];
  return 0;
}

int nrm_host(long n, const double *x, double *out) {
  if (vnrm2(n, x, ctx().dscal + S_TMP0)) return PEVSL_ERR_CUDA;
  const double *h = fetch_scalars(S_TMP0, 1);
  if (!h) return PEVSL_ERR_CUDA;
  *out = h[0];
  return 0;
}

long gen_ld(long n) { return (n + 31) / 32 * 32; }

/* ------------------------------------------------ generalized filter counters
 * applications, algorithmic HBM bytes and device time (CUDA events around
 * each application) of the generalized filter: pEVSL_B200_GenCounters */
uint64_t g_gen_filters = 0, g_gen_degrees = 0;
double g_gen_bytes = 0.0, g_gen_ms = 0.0;

struct EvPool {
  static constexpr int kPairs = 64;
  cudaEvent_t ev[2 * kPairs];
  int used = 0;
  bool ok = false, init = false;
  void begin() {
    if (!init) {
      init = ok = true;
      for (int i = 0; i < 2 * kPairs && ok; i++) ok = cudaEventCreate(&ev[i]) == cudaSuccess;
    }
    if (!ok) return;
    if (used == kPairs) flush();
    cudaEventRecord(ev[2 * used], ctx().stream);
  }
  void end() {
    if (ok) cudaEventRecord(ev[2 * used++ + 1], ctx().stream);
  }
  void flush() {
    if (!ok || !used) return;
    cudaEventSynchronize(ev[2 * used - 1]);
    for (int i = 0; i < used; i++) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]) == cudaSuccess) g_gen_ms += ms;
    }
    used = 0;
  }
};
EvPool g_gen_ev;

/* algorithmic bytes: a matrix pass is entry_bytes (3 packed, 12 plain) per
 * entry + 4 (n + 1); a fused
 * Chebyshev degree adds v_k, v_{k-1}, y read and v_{k+1}, y written (the
 * first degree reads neither v_{k-1} nor y); a second-kind Chebyshev-
 * iteration step gathers d and reads/writes x and r, writes d_new */
double mat_bytes(const pevsl_devcsr *M) {
  return entry_bytes(M, false) * (double)M->nnz + 4.0 * (M->nrows + 1.0);
}

double solve_bytes(pevsl_Data *pevsl) {
  const SVFunc f = pevsl->Bsol ? pevsl->Bsol->func : nullptr;
  if (f == pEVSL_LSPolSol) {
    const pevsl_lspol *L = (const pevsl_lspol *)pevsl->Bsol->data;
    const double n = L->B->nrows;
    double b = 0.0;
    for (int k = 1; k <= L->deg; k++) b += mat_bytes(L->B) + (k == 1 ? 24.0 : 40.0) * n;
    return b;
  }
  if (f == pEVSL_ChebIterSolv1 || f == pEVSL_ChebIterSolv2) {
    const pevsl_chebiter *C = (const pevsl_chebiter *)pevsl->Bsol->data;
    const double n = C->A->nrows;
    return C->deg * (mat_bytes(C->A) + 48.0 * n) + 32.0 * n;
  }
  return 0.0;
}

/* The generalized filter (pEVSL_ChebAv with ifGenEv, SRC/chebpol.c:509-574):
 * y = p(A B^{-1}) v, each degree a B-solve then the fused degree kernel
 * whose SpMV reads B^{-1} v_k.  w holds 4 n doubles. */
int gen_filter(pevsl_Data *pevsl, const pevsl_Polparams *pol, const double *v, double *y,
               double *w, long n) {
  pevsl_devcsr *A = pevsl_builtin_A(pevsl);
  const int m = pol->deg;
  const double cc = pol->cc, dd = pol->dd;
  const double *mu = pol->mu;
  pevsl->stats->n_polAv++;
  if (m <= 0) {
    if (vcopy(v, y, n)) return PEVSL_ERR_CUDA;
    return vscal(y, n, mu[0]);
  }
  if (!A && (!pevsl->Amv || !pevsl->Amv->func)) return PEVSL_ERR_NOMATVEC;
  if (A) {
    const double sb = solve_bytes(pevsl);
    for (int k = 1; k <= m; k++) g_gen_bytes += sb + mat_bytes(A) + (k == 1 ? 32.0 : 48.0) * n;
  }
  g_gen_degrees += (uint64_t)m;
  g_gen_filters++;
  double *buf[2] = {w, w + n}, *w2 = w + 2 * n, *tmp = w + 3 * n;
  const double *vk = v, *vkm1 = nullptr;
  int st = 0;
  for (int k = 1; k <= m && !st; k++) {
    double *vkp1 = k <= 2 ? buf[k - 1] : const_cast<double *>(vkm1);
    const double t = (k == 1 ? 1.0 : 2.0) / dd;
    st = solve_B(pevsl, vk, w2);
    if (!st && A) {
      st = cheb_step_x(A, w2, vk, vkm1, vkp1, y, cc, t, mu[0], mu[k], k == 1, tmp);
      pevsl->stats->n_mvA++;
    } else if (!st) {
      st = apply_Ag(pevsl, w2, tmp);
      if (!st) st = cheb_combine(n, tmp, vk, vkm1, vkp1, y, cc, t, mu[0], mu[k], k == 1);
    }
    vkm1 = vk;
    vk = vkp1;
  }
  return st;
}

/* The library's own B-solvers enqueue a fixed sequence of launches with
 * no host synchronisation, so a generalized filter application (or a KPM
 * vector's degree loop) that uses one can be captured once in a CUDA graph
 * and replayed: at n ~ 10^5 a degree is 40+ short launches whose gaps would
 * otherwise cost as much as the kernels. */
bool graphable(pevsl_Data *pevsl) {
  if (!pevsl_builtin_A(pevsl) || !pevsl->Bsol) return false;
  const SVFunc f = pevsl->Bsol->func;
  if (f != pEVSL_LSPolSol && f != pEVSL_ChebIterSolv1 && f != pEVSL_ChebIterSolv2) return false;
  return !capturing() && getenv("PEVSL_B200_GEN_GRAPH_OFF") == nullptr;
}

/* choose the row kernels of A and of the B-solver's matrix before a
 * capture (the tuning times launches, which a capture cannot) */
void pretune(pevsl_Data *pevsl) {
  stream_tune(pevsl_builtin_A(pevsl));
  const SVFunc f = pevsl->Bsol->func;
  if (f == pEVSL_LSPolSol)
    stream_tune(((pevsl_lspol *)pevsl->Bsol->data)->B);
  else
    stream_tune(((pevsl_chebiter *)pevsl->Bsol->data)->A);
}

/* a captured launch sequence and the statistics one replay stands for */
struct GenGraph {
  cudaGraphExec_t exec = nullptr;
  size_t d_mvA = 0, d_svB = 0, d_polAv = 0, d_chebmv = 0;
  uint64_t d_launches = 0, d_filters = 0, d_degrees = 0;
  double d_bytes = 0.0;
  ~GenGraph() {
    if (exec) cudaGraphExecDestroy(exec);
  }
};

pevsl_chebiter *bsol_chebiter(pevsl_Data *pevsl) {
  const SVFunc f = pevsl->Bsol->func;
  return (f == pEVSL_ChebIterSolv1 || f == pEVSL_ChebIterSolv2) ? (pevsl_chebiter *)pevsl->Bsol->data
                                                                : nullptr;
}

/* capture body() into g (first call) and replay it */
template <class Body>
int graph_run(GenGraph &g, pevsl_Data *pevsl, Body body) {
  Ctx &c = ctx();
  pevsl_chebiter *C = bsol_chebiter(pevsl);
  if (!g.exec) {
    const size_t m0 = pevsl->stats->n_mvA, s0 = pevsl->stats->n_svB, p0 = pevsl->stats->n_polAv;
    const size_t c0 = C ? C->n_chebmv : 0;
    const uint64_t l0 = c.launches, f0 = g_gen_filters, dg0 = g_gen_degrees;
    const double b0 = g_gen_bytes;
    if (fail(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal), "BeginCapture"))
      return PEVSL_ERR_CUDA;
    const int st = body();
    cudaGraph_t gr = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(c.stream, &gr);
    if (st || fail(ec, "EndCapture")) {
      if (gr) cudaGraphDestroy(gr);
      return st ? st : PEVSL_ERR_CUDA;
    }
    const cudaError_t ei = cudaGraphInstantiate(&g.exec, gr, 0);
    cudaGraphDestroy(gr);
    if (fail(ei, "cudaGraphInstantiate")) {
      g.exec = nullptr;
      return PEVSL_ERR_CUDA;
    }
    /* the capture counted the statistics once; each replay adds them */
    g.d_mvA = pevsl->stats->n_mvA - m0;
    g.d_svB = pevsl->stats->n_svB - s0;
    g.d_polAv = pevsl->stats->n_polAv - p0;
    g.d_chebmv = C ? C->n_chebmv - c0 : 0;
    g.d_launches = c.launches - l0;
    g.d_filters = g_gen_filters - f0;
    g.d_degrees = g_gen_degrees - dg0;
    g.d_bytes = g_gen_bytes - b0;
    g_gen_filters = f0;
    g_gen_degrees = dg0;
    g_gen_bytes = b0;
    pevsl->stats->n_mvA = m0;
    pevsl->stats->n_svB = s0;
    pevsl->stats->n_polAv = p0;
    if (C) C->n_chebmv = c0;
    c.launches = l0;
  }
  pevsl->stats->n_mvA += g.d_mvA;
  pevsl->stats->n_svB += g.d_svB;
  pevsl->stats->n_polAv += g.d_polAv;
  if (C) C->n_chebmv += g.d_chebmv;
  c.launches += g.d_launches;
  g_gen_filters += g.d_filters;
  g_gen_degrees += g.d_degrees;
  g_gen_bytes += g.d_bytes;
  return fail(cudaGraphLaunch(g.exec, c.stream), "cudaGraphLaunch");
}

/* the generalized filter through a graph over the staging vectors xs, ys
 * (fixed addresses), with one copy in and one copy out */
int gen_filter_graphed(GenGraph &g, pevsl_Data *pevsl, const pevsl_Polparams *pol, const double *v,
                       double *y, double *w, double *xs, double *ys, long n) {
  if (memcpy_async(xs, v, sizeof(double) * (size_t)n)) return PEVSL_ERR_CUDA;
  const int st = graph_run(g, pevsl, [&]() { return gen_filter(pevsl, pol, xs, ys, w, n); });
  if (st) return st;
  return memcpy_async(y, ys, sizeof(double) * (size_t)n);
}

}  // namespace

/* ====================================================== generalized solvers */

/* KPM moments of the generalized problem for vectors [vec_start, vec_end)
 * (SRC/kpmdos.c:104-156): v random with unit 2-norm, w = L^{-T} v, v = B w,
 * the recurrence on w with v_{k+1} = B^{-1} A v_k; mu and tcnt are
 * accumulated in the reference's order. */
int pevsl_gen_kpm_moments(pevsl_Data *pevsl, int Mdeg, const double *jac, double ctr, double wid,
                          double beta1, double beta2, int vec_start, int vec_end, double *mu,
                          double *tcnt) {
  const long n = pevsl->n;
  double *buf = (double *)ws(WS_GEN, sizeof(double) * 5 * (size_t)n);
  double *ddot_ = (double *)ws(WS_MOM, sizeof(double) * (size_t)(Mdeg + 1));
  double *hdot = (double *)malloc(sizeof(double) * (size_t)(Mdeg + 1));
  int st = (!buf || !ddot_ || !hdot) ? PEVSL_ERR_NOMEM : 0;
  const bool use_graph = graphable(pevsl);
  if (use_graph) pretune(pevsl);
  GenGraph kg;
  for (int m = vec_start; m < vec_end && !st; m++) {
    double *v = buf, *vkm1 = buf + n, *vk = buf + 2 * n, *vkp1 = buf + 3 * n, *w = buf + 4 * n;
    double t = 0.0;
    st = pevsl_rand_vector_dev(v, (int)n);
    if (!st) st = nrm_host(n, v, &t);
    if (!st) st = vscal(v, n, 1.0 / t);
    if (!st) st = solve_LT(pevsl, v, w);
    if (!st) st = apply_B(pevsl, w, v);
    if (!st) st = vcopy(w, vk, n);
    if (!st) st = vfill(vkm1, n, 0.0);
    /* the degree loop touches only fixed buffers: one graph for every vector */
    auto degrees = [&]() -> int {
      double *a = vkm1, *bk = vk, *c = vkp1;
      int s2 = 0;
      for (int k = 0; k < Mdeg && !s2; k++) {
        const double sc = (k == 0 ? 1.0 : 2.0) / wid;
        s2 = apply_Ag(pevsl, bk, w);
        if (!s2) s2 = solve_B(pevsl, w, c);
        if (!s2) s2 = vaxpy(n, -ctr, bk, c);
        if (!s2) s2 = vscal(c, n, sc);
        if (!s2) s2 = vaxpy(n, -1.0, a, c);
        double *tmp = a;
        a = bk;
        bk = c;
        c = tmp;
        if (!s2) s2 = vdot(n, bk, v, ddot_ + k);
      }
      return s2;
    };
    if (!st) st = use_graph ? graph_run(kg, pevsl, degrees) : degrees();
    if (!st) st = memcpy_async(hdot, ddot_, sizeof(double) * (size_t)Mdeg);
    if (!st) st = sync();
    if (st) break;
    mu[0] += jac[0];
    *tcnt -= jac[0] * (beta2 - beta1);
    for (int k = 0; k < Mdeg; k++) {
      const int k1 = k + 1;
      const double tk = hdot[k] * 2.0 * jac[k1];
      mu[k1] += tk;
      *tcnt -= tk * (sin(k1 * beta2) - sin(k1 * beta1)) / k1;
    }
  }
  free(hdot);
  return st;
}

/* One Lanczos run of the generalized Lanczos DOS (SRC/landos.c:134-262):
 * v_0 = L^{-T} vinit with unit B-norm, the B-inner-product recurrence with
 * Z = B V, maxit steps; the tridiagonal matrix into dT, eT. */
int pevsl_gen_landos_lanczos(pevsl_Data *pevsl, int maxit, const double *vinit, double *dT,
                             double *eT) {
  const long n = pevsl->n, ld = gen_ld(n);
  double *V = (double *)ws(WS_BASIS, sizeof(double) * (size_t)ld * (size_t)(maxit + 1));
  double *Z = (double *)ws(WS_ZBASIS, sizeof(double) * (size_t)ld * (size_t)(maxit + 1));
  if (!V || !Z) return PEVSL_ERR_NOMEM;
  int st = solve_LT(pevsl, vinit, V);
  double t = 0.0;
  if (!st) st = apply_B(pevsl, V, Z);
  if (!st) st = dot_host(n, V, Z, &t);
  if (!st) {
    t = 1.0 / sqrt(t);
    st = vscal(Z, n, t);
  }
  if (!st) st = vscal(V, n, t);
  double wn = 0.0, beta = 0.0;
  int nwn = 0;
  for (int k = 0; k < maxit && !st; k++) {
    double *v = V + (size_t)k * ld, *z = Z + (size_t)k * ld;
    double *vnew = v + ld, *znew = z + ld;
    double alpha = 0.0;
    st = apply_Ag(pevsl, v, znew);
    if (!st && k > 0) st = vaxpy(n, -beta, z - ld, znew);
    if (!st) st = dot_host(n, v, znew, &alpha);
    if (st) break;
    dT[k] = alpha;
    wn += fabs(alpha);
    st = vaxpy(n, -alpha, z, znew);
    if (!st) st = cgs2(n, ld, k + 1, Z, V, znew);
    if (!st) st = solve_B(pevsl, znew, vnew);
    if (!st) st = dot_host(n, vnew, znew, &beta);
    if (st) break;
    beta = sqrt(beta);
    wn += 2.0 * beta;
    nwn += 3;
    if (beta * nwn < orthTol * wn) {
      st = pevsl_rand_vector_dev(vnew, (int)n);
      if (!st) st = cgs2(n, ld, k + 1, V, Z, vnew);
      if (!st) st = apply_B(pevsl, vnew, znew);
      if (!st) st = dot_host(n, vnew, znew, &beta);
      if (st) break;
      beta = sqrt(beta);
      t = 1.0 / beta;
      st = vscal(vnew, n, t);
      if (!st) st = vscal(znew, n, t);
      beta = 0.0;
    } else {
      t = 1.0 / beta;
      st = vscal(vnew, n, t);
      if (!st) st = vscal(znew, n, t);
    }
    eT[k] = beta;
  }
  return st;
}

/* pEVSL_LanTrbounds for the generalized problem (SRC/lantrbnd.c:31-408):
 * thick-restart Lanczos on B^{-1} A in the B inner product, two Ritz
 * vectors kept (with their B images) at each restart. */
int pevsl_gen_lantrbounds(pevsl_Data *pevsl, int lanm, int maxit, double tol, pevsl_Parvec *vinit,
                          int bndtype, double *lammin, double *lammax, FILE *fstats) {
  const int N = pevsl->N;
  const long n = pevsl->n, ld = gen_ld(n);
  lanm = PEVSL_MIN(lanm, N);
  const int lanm1 = lanm + 1;
  if (lanm == N) maxit = PEVSL_MIN(maxit, N);
  const size_t L = (size_t)lanm1;
  double *V = (double *)ws(WS_BASIS, sizeof(double) * (size_t)ld * L);
  double *Z = (double *)ws(WS_ZBASIS, sizeof(double) * (size_t)ld * L);
  double *R = (double *)ws(WS_RITZ, sizeof(double) * (size_t)ld * 4);
  double *dY = (double *)ws(WS_RITZ2, sizeof(double) * (L * 2 + L));
  double *T = (double *)calloc(L * L, sizeof(double));
  double *EvecT = (double *)calloc(L * L, sizeof(double));
  double *Rval = (double *)calloc(L, sizeof(double));
  double *hY = (double *)malloc(sizeof(double) * L * 2);
  if (!V || !Z || !R || !dY || !T || !EvecT || !Rval || !hY) {
    free(T);
    free(EvecT);
    free(Rval);
    free(hY);
    return PEVSL_ERR_NOMEM;
  }
  double *dS = dY + 2 * L;
  int st = 0, it = 0, trlen = 0;
  double lmin = 0.0, lmax = 0.0, s[3] = {0, 0, 0}, t = 0.0;
  if (fstats) fprintf(fstats, " LanTR for bounds: dim %d, maxits %d\n", lanm, maxit);
#define VC(j) (V + (size_t)(j) * ld)
#define ZC(j) (Z + (size_t)(j) * ld)
  st = vcopy(vinit->data, VC(0), n);
  if (!st) st = apply_B(pevsl, VC(0), ZC(0));
  if (!st) st = dot_host(n, VC(0), ZC(0), &t);
  if (!st) {
    t = 1.0 / sqrt(t);
    st = vscal(ZC(0), n, t);
  }
  if (!st) st = vscal(VC(0), n, t);
  while (it < maxit && !st) {
    double wn = 0.0, beta = 0.0;
    int nwn = 0;
    int k = trlen > 0 ? trlen + 1 : 0;
    if (k + 5 > lanm1) {
      fprintf(stderr, "Krylov dim too small for this problem. Try a larger dim\n");
      st = PEVSL_ERR_ARG;
      break;
    }
    if (trlen > 0) {
      const int k1 = k - 1;
      double *v = VC(k1), *vnew = VC(k1 + 1), *znew = ZC(k1 + 1);
      st = apply_Ag(pevsl, v, znew);
      for (int i = 0; i < trlen; i++) {
        T[i * L + i] = Rval[i];
        wn += fabs(Rval[i]);
      }
      if (!st) st = dot_host(n, v, znew, &s[k1]);
      if (!st) st = memcpy_async(dS, s, sizeof(double) * (size_t)k);
      if (!st) st = gemv_sub_nrm(n, k, Z, ld, dS, znew, ctx().dscal + S_TMP3, nullptr, nullptr,
                                 nullptr, 0.0);
      if (st) break;
      for (int i = 0; i < k1; i++) {
        T[trlen * L + i] = s[i];
        T[i * L + trlen] = s[i];
        wn += 2.0 * fabs(s[i]);
      }
      T[trlen * L + trlen] = s[k1];
      wn += fabs(s[k1]);
      st = solve_B(pevsl, znew, vnew);
      if (!st) st = dot_host(n, vnew, znew, &beta);
      if (st) break;
      beta = sqrt(beta);
      wn += 2.0 * beta;
      nwn += 3 * k;
      if (beta * nwn < orthTol * wn) {
        st = pevsl_rand_vector_dev(vnew, (int)n);
        if (!st) st = cgs2(n, ld, k, V, Z, vnew);
        if (!st) st = apply_B(pevsl, vnew, znew);
        if (!st) st = dot_host(n, vnew, znew, &beta);
        if (st) break;
        beta = sqrt(beta);
        const double ib = 1.0 / beta;
        st = vscal(vnew, n, ib);
        if (!st) st = vscal(znew, n, ib);
        beta = 0.0;
      } else {
        const double ib = 1.0 / beta;
        st = vscal(vnew, n, ib);
        if (!st) st = vscal(znew, n, ib);
      }
      T[k1 * L + k] = beta;
      T[k * L + k1] = beta;
    }
    const double *zold = k > 0 ? ZC(k - 1) : nullptr;
    while (k < lanm && it < maxit && !st) {
      k++;
      double *v = VC(k - 1), *z = ZC(k - 1), *vnew = VC(k), *znew = ZC(k);
      double alpha = 0.0;
      st = apply_Ag(pevsl, v, znew);
      it++;
      if (!st && zold) st = vaxpy(n, -beta, zold, znew);
      if (!st) st = dot_host(n, v, znew, &alpha);
      if (st) break;
      T[(k - 1) * L + (k - 1)] = alpha;
      wn += fabs(alpha);
      st = vaxpy(n, -alpha, z, znew);
      if (!st) st = cgs2(n, ld, k, Z, V, znew);
      if (!st) st = solve_B(pevsl, znew, vnew);
      if (!st) st = dot_host(n, vnew, znew, &beta);
      if (st) break;
      beta = sqrt(beta);
      wn += 2.0 * beta;
      nwn += 3;
      zold = z;
      if (beta * nwn < orthTol * wn) {
        if (fstats) fprintf(fstats, "it %4d: Lucky breakdown, beta = %.15e\n", it, beta);
        st = pevsl_rand_vector_dev(vnew, (int)n);
        if (!st) st = cgs2(n, ld, k, V, Z, vnew);
        if (!st) st = apply_B(pevsl, vnew, znew);
        if (!st) st = dot_host(n, vnew, znew, &beta);
        if (st) break;
        beta = sqrt(beta);
        const double ib = 1.0 / beta;
        st = vscal(vnew, n, ib);
        if (!st) st = vscal(znew, n, ib);
        beta = 0.0;
      } else {
        const double ib = 1.0 / beta;
        st = vscal(vnew, n, ib);
        if (!st) st = vscal(znew, n, ib);
      }
      T[k * L + (k - 1)] = beta;
      T[(k - 1) * L + k] = beta;
    }
    if (st) break;
    if (pevsl_dense_symeig(k, T, lanm1, EvecT, lanm1, Rval)) {
      st = PEVSL_ERR_EIG;
      break;
    }
    s[0] = beta * EvecT[k - 1];
    s[1] = beta * EvecT[(size_t)(k - 1) * L + (k - 1)];
    double t1, t2;
    if (bndtype <= 1) {
      t1 = fabs(s[0]);
      t2 = fabs(s[1]);
    } else {
      t1 = 2.0 * s[0] * s[0] / (Rval[1] - Rval[0]);
      t2 = 2.0 * s[1] * s[1] / (Rval[k - 1] - Rval[k - 2]);
    }
    lmin = Rval[0] - t1;
    lmax = Rval[k - 1] + t2;
    /* the extreme Ritz vectors and their B images become V, Z (:, 0:2) */
    memcpy(hY, EvecT, sizeof(double) * (size_t)k);
    memcpy(hY + k, EvecT + (size_t)(k - 1) * L, sizeof(double) * (size_t)k);
    st = memcpy_async(dY, hY, sizeof(double) * 2 * (size_t)k);
    if (!st) st = gemm_nn(n, k, 2, V, ld, dY, k, R, ld);
    if (!st) st = gemm_nn(n, k, 2, Z, ld, dY, k, R + 2 * ld, ld);
    if (!st) st = vcopy(R, VC(0), n);
    if (!st) st = vcopy(R + ld, VC(1), n);
    if (!st) st = vcopy(R + 2 * ld, ZC(0), n);
    if (!st) st = vcopy(R + 3 * ld, ZC(1), n);
    trlen = 2;
    Rval[1] = Rval[k - 1];
    if (fstats)
      fprintf(fstats, "it %4d, k %3d: ritz %.15e %.15e, t1,t2 %e %e, res %.15e %.15e\n", it, k,
              Rval[0], Rval[1], t1, t2, fabs(s[0]), fabs(s[1]));
    if (t1 + t2 < tol * (fabs(lmin) + fabs(lmax))) break;
    memset(T, 0, sizeof(double) * L * L);
    if (!st) st = vcopy(VC(k), VC(trlen), n);
    if (!st) st = vcopy(ZC(k), ZC(trlen), n);
  }
#undef VC
#undef ZC
  if (!st) st = sync();
  *lammin = lmin;
  *lammax = lmax;
  free(T);
  free(EvecT);
  free(Rval);
  free(hY);
  return st;
}

/* ---------------------------------------------------------------- ChebLanNr
 * pEVSL_ChebLanNr for the generalized problem (SRC/cheblanNr.c:54-448):
 * the filtered initial vector, the filter applied to z = B v (giving
 * B p(B^{-1}A) v), CGS_DGKS2 against (V, Z), v_{k+1} = B^{-1} z_{k+1},
 * the restricted-trace test every 20 steps from step 30, then Ritz pairs
 * normalised in the B-norm with residuals ||A u - lam B u||.  The state of
 * one slice lives in a GenSlice, so that slices can also advance in
 * lockstep with one interleaved filter application for all of them. */
namespace {

struct GenSlice {
  double intv[4];
  pevsl_Polparams *pol;
  int maxit;
  double *V, *Z; /* bases, ld x (maxit + 1) */
  std::vector<double> dT, eT, EvalT;
  double tr0 = 0.0, wn = 0.0, beta = 0.0;
  int nwn = 0, k = 0, kdim = 0, count = 0, nconv = 0;
  bool active = false, ran = false;
  int status = 0;
  int nev = 0;
  double *Lam = nullptr, *res = nullptr;
  pevsl_Parvecs *Rvec = nullptr;
};

const int kNtest = 30, kCycle = 20;

/* checks and header lines; active when the slice is to be solved */
void gs_begin(pevsl_Data *pevsl, GenSlice &S, FILE *fstats) {
  S.maxit = PEVSL_MIN(pevsl->N, S.maxit);
  S.active = false;
  S.status = 0;
  if (pevsl_check_intv(S.intv, fstats) < 0) return; /* no pairs, status 0 */
  if (fstats) {
    fprintf(fstats, " intv:[%e, %e, %e, %e]\n", S.intv[0], S.intv[1], S.intv[2], S.intv[3]);
    fprintf(fstats, " ** Cheb Poly of deg = %d, gam = %.15e, bar: %.15e\n", S.pol->deg,
            S.pol->gam, S.pol->bar);
  }
  if (S.pol->gam > 1.0 || S.pol->gam < -1.0) {
    fprintf(stdout, "gamB error %.15e\n", S.pol->gam);
    S.status = -1;
    return;
  }
  if (fstats) fprintf(fstats, " ** Cheb-LanNr \n");
  S.dT.assign((size_t)S.maxit + 1, 0.0);
  S.eT.assign((size_t)S.maxit + 1, 0.0);
  S.EvalT.assign((size_t)S.maxit + 1, 0.0);
  S.active = S.ran = true;
}

/* V(:,0) holds the filtered start vector: give it unit B-norm, Z(:,0) = B V(:,0) */
int gs_normalize0(pevsl_Data *pevsl, GenSlice &S, long n) {
  double t = 0.0;
  int st = apply_B(pevsl, S.V, S.Z);
  if (!st) st = dot_host(n, S.V, S.Z, &t);
  if (!st) {
    t = 1.0 / sqrt(t);
    st = vscal(S.Z, n, t);
  }
  if (!st) st = vscal(S.V, n, t);
  return st;
}

/* the rest of step k once Z(:,k+1) holds the filtered z; filter1(in, out)
 * is the one-vector filter (for a breakdown restart) */
template <class F1>
int gs_step(pevsl_Data *pevsl, GenSlice &S, long n, long ld, double *vrand, F1 filter1,
            FILE *fstats) {
  const int k = S.k;
  double *v = S.V + (size_t)k * ld, *z = S.Z + (size_t)k * ld;
  double *vnew = v + ld, *znew = z + ld;
  double alpha = 0.0, t = 0.0;
  int st = 0;
  if (k > 0) st = vaxpy(n, -S.beta, z - ld, znew);
  if (!st) st = dot_host(n, v, znew, &alpha);
  if (st) return st;
  S.dT[k] = alpha;
  S.wn += fabs(alpha);
  st = vaxpy(n, -alpha, z, znew);
  if (!st) st = cgs2(n, ld, k + 1, S.Z, S.V, znew);
  if (!st) st = solve_B(pevsl, znew, vnew);
  if (!st) st = dot_host(n, vnew, znew, &S.beta);
  if (st) return st;
  S.beta = sqrt(S.beta);
  S.wn += 2.0 * S.beta;
  S.nwn += 3;
  if (S.beta * S.nwn < orthTol * S.wn) {
    if (fstats) fprintf(fstats, "it %4d: Lucky breakdown, beta = %.15e\n", k, S.beta);
    st = pevsl_rand_vector_dev(vrand, (int)n);
    if (!st) st = filter1(vrand, vnew);
    if (!st) st = cgs2(n, ld, k + 1, S.V, S.Z, vnew);
    if (!st) st = apply_B(pevsl, vnew, znew);
    if (!st) st = dot_host(n, vnew, znew, &S.beta);
    if (st) return st;
    S.beta = sqrt(S.beta);
    t = 1.0 / S.beta;
    st = vscal(vnew, n, t);
    if (!st) st = vscal(znew, n, t);
    S.beta = 0.0;
  } else {
    t = 1.0 / S.beta;
    st = vscal(vnew, n, t);
    if (!st) st = vscal(znew, n, t);
  }
  if (st) return st;
  S.eT[k] = S.beta;
  S.k = k + 1;
  if ((k < kNtest || (k - kNtest) % kCycle != 0) && k != S.maxit - 1) {
    if (S.k >= S.maxit) S.active = false;
    return 0;
  }
  S.kdim = k + 1;
  if (pevsl_tridiag_eig(S.kdim, S.dT.data(), S.eT.data(), S.EvalT.data(), nullptr))
    return PEVSL_ERR_EIG;
  S.count = S.kdim;
  double tr1 = 0.0;
  S.nconv = 0;
  const double bar = S.pol->bar;
  for (int i = 0; i < S.count; i++)
    if (S.EvalT[i] + 5 * DBL_EPSILON >= bar) {
      tr1 += S.EvalT[i];
      S.nconv++;
    }
  if (fstats) fprintf(fstats, "  k %4d:   nconv %4d  tr1 %21.15e\n", k, S.nconv, tr1);
  if (fabs(tr1 - S.tr0) < 2e-12 || fabs(tr1) + fabs(S.tr0) < 1e-10) {
    S.active = false;
    S.k = k; /* the loop left at step k, as the reference's break */
    return 0;
  }
  S.tr0 = tr1;
  if (S.k >= S.maxit) S.active = false;
  return 0;
}

/* Ritz pairs of a finished slice: eigenvectors of T for the values >= bar */
int gs_finish(pevsl_Data *pevsl, GenSlice &S, pevsl_Parvec *vinit, long n, long ld, double tol,
              FILE *fstats) {
  if (S.k >= S.maxit && fstats)
    fprintf(fstats, "The max number of iterations [%d] has been reached. The eigenvalues "
                    "computed may not have converged\n", S.maxit);
  const int kdim = S.kdim, count = S.count;
  const double bar = S.pol->bar, aa = S.intv[0], bb = S.intv[1];
  if (kdim > 0 && pevsl_tridiag_eig(kdim, S.dT.data(), S.eT.data(), S.EvalT.data(), nullptr))
    return PEVSL_ERR_EIG;
  std::vector<int> sel;
  for (int i = 0; i < count; i++)
    if (S.EvalT[i] >= bar) sel.push_back(i);
  const int nsel = (int)sel.size();
  const int nout = PEVSL_MAX(S.nconv, nsel);
  double *Lam = (double *)malloc(sizeof(double) * (size_t)(nout > 0 ? nout : 1));
  double *res = (double *)malloc(sizeof(double) * (size_t)(nout > 0 ? nout : 1));
  pevsl_Parvecs *Rvec = (pevsl_Parvecs *)calloc(1, sizeof(pevsl_Parvecs));
  if (!Lam || !res || !Rvec) {
    free(Lam);
    free(res);
    free(Rvec);
    return PEVSL_ERR_NOMEM;
  }
  pEVSL_ParvecsDuplParvec(vinit, nout, (int)n, Rvec);
  int nev = 0, st = 0;
  if (nsel > 0) {
    std::vector<double> Y((size_t)kdim * nsel), hv(3 * (size_t)nsel);
    double *U = (double *)ws(WS_RITZ, sizeof(double) * (size_t)ld * (size_t)nsel);
    double *W = (double *)ws(WS_RITZ2, sizeof(double) * (size_t)ld * (size_t)nsel);
    double *BU = (double *)ws(WS_REF1, sizeof(double) * (size_t)ld * (size_t)nsel);
    double *dY = (double *)ws(WS_PART, sizeof(double) * (size_t)kdim * (size_t)nsel);
    double *dv = (double *)ws(WS_MOM, sizeof(double) * 3 * (size_t)nsel);
    if (!U || !W || !BU || !dY || !dv || (nout > 0 && !Rvec->data)) st = PEVSL_ERR_NOMEM;
    if (!st && pevsl_tridiag_eig_sel(kdim, S.dT.data(), S.eT.data(), S.EvalT.data(), nsel,
                                     sel.data(), Y.data()))
      st = PEVSL_ERR_EIG;
    if (!st) st = memcpy_async(dY, Y.data(), sizeof(double) * Y.size());
    if (!st) st = gemm_nn(n, kdim, nsel, S.V, ld, dY, kdim, U, ld);
    for (int j = 0; j < nsel && !st; j++) st = apply_B(pevsl, U + (size_t)j * ld, BU + (size_t)j * ld);
    if (!st) st = vdot_cols(n, nsel, U, ld, BU, ld, dv);
    if (!st) st = memcpy_async(hv.data(), dv, sizeof(double) * (size_t)nsel);
    if (!st) st = sync();
    for (int j = 0; j < nsel && !st; j++) {
      const double tn = sqrt(hv[j]);
      if (tn == 0.0) st = 2; /* zero eigenvector (SRC/cheblanNr.c:377-379) */
      hv[nsel + j] = st ? 0.0 : 1.0 / tn;
    }
    if (!st) st = memcpy_async(dv + nsel, hv.data() + nsel, sizeof(double) * (size_t)nsel);
    if (!st) st = vscal_cols(n, nsel, U, ld, dv + nsel);
    if (!st) st = vscal_cols(n, nsel, BU, ld, dv + nsel);
    for (int j = 0; j < nsel && !st; j++) st = apply_Ag(pevsl, U + (size_t)j * ld, W + (size_t)j * ld);
    if (!st) st = vdot_cols(n, nsel, W, ld, U, ld, dv);
    if (!st) st = vaxpy_cols(n, nsel, dv, BU, ld, W, ld);
    if (!st) st = vdot_cols(n, nsel, W, ld, W, ld, dv + 2 * nsel);
    if (!st) st = memcpy_async(hv.data(), dv, sizeof(double) * 3 * (size_t)nsel);
    if (!st) st = sync();
    for (int j = 0; j < nsel && !st; j++) {
      const double lam = hv[j];
      if (lam < aa - DBL_EPSILON || lam > bb + DBL_EPSILON) continue;
      const double r0 = sqrt(hv[2 * nsel + j]);
      if (r0 < tol) {
        Lam[nev] = lam;
        res[nev] = r0;
        st = vcopy(U + (size_t)j * ld, Rvec->data + (size_t)nev * Rvec->ld, n);
        nev++;
      }
    }
    if (!st) st = sync();
  }
  if (st) {
    free(Lam);
    free(res);
    pEVSL_ParvecsFree(Rvec);
    free(Rvec);
    return st;
  }
  S.nev = nev;
  S.Lam = Lam;
  S.res = res;
  S.Rvec = Rvec;
  return 0;
}

/* ------------------------------------------------------------ lockstep filter
 * The generalized filter for up to 16 slices of one problem at once, their
 * vectors row-interleaved: per degree, the least-squares B-solve as its
 * Chebyshev degrees on B (cheb_step_il, the same coefficients for every
 * column) and the A step (cheb_step_il_x: the SpMV reads B^{-1} X_k, the
 * recurrence X_k, each column with its slice's coefficients, zero past its
 * degree).  Per column the arithmetic is that of gen_filter, bit for bit.
 * The degree loop works on fixed blocks, so it is captured once in a CUDA
 * graph; packing the inputs and unpacking the outputs stay outside. */
struct GenIl {
  int S = 0, maxdeg = 0, degB = 0;
  long n = 0;
  const pevsl_devcsr *A = nullptr, *B = nullptr;
  double cc = 0, dd = 0, ccB = 0, ddB = 0;
  double *blk = nullptr; /* X0, B0, B1, Y, W, L0, L1: n x S each */
  double *smu = nullptr, *lmu = nullptr; /* coefficient tables on the device */
  GenGraph graph;
  bool use_graph = false;
  double *X(int i) const { return blk + (size_t)i * (size_t)n * (size_t)S; }
};

int genil_degrees(pevsl_Data *pevsl, GenIl &G) {
  const double *vk = G.X(0), *vkm1 = nullptr;
  int st = 0;
  for (int k = 1; k <= G.maxdeg && !st; k++) {
    /* W = the least-squares B^{-1} of X_k */
    const double *lk = vk, *lkm1 = nullptr;
    for (int j = 1; j <= G.degB && !st; j++) {
      double *lkp1 = j == 1 ? G.X(5) : j == 2 ? G.X(6) : const_cast<double *>(lkm1);
      st = cheb_step_il(G.B, G.S, lk, lkm1, lkp1, G.X(4), G.ccB, (j == 1 ? 1.0 : 2.0) / G.ddB,
                        G.lmu, G.lmu + (size_t)j * G.S, j == 1);
      lkm1 = lk;
      lk = lkp1;
    }
    double *vkp1 = k == 1 ? G.X(1) : k == 2 ? G.X(2) : const_cast<double *>(vkm1);
    if (!st)
      st = cheb_step_il_x(G.A, G.S, G.X(4), vk, vkm1, vkp1, G.X(3), G.cc,
                          (k == 1 ? 1.0 : 2.0) / G.dd, G.smu, G.smu + (size_t)k * G.S, k == 1);
    vkm1 = vk;
    vk = vkp1;
  }
  pevsl->stats->n_mvA += (size_t)G.maxdeg * G.S;
  pevsl->stats->n_svB += (size_t)G.maxdeg * G.S;
  g_gen_filters++;
  g_gen_degrees += (uint64_t)G.maxdeg;
  const double n = (double)G.n;
  g_gen_bytes += (double)G.maxdeg *
                 (G.degB * (il_entry_bytes(G.B) * G.B->nnz + 4.0 * (n + 1) + 40.0 * n * G.S) +
                  il_entry_bytes(G.A) * G.A->nnz + 4.0 * (n + 1) + 48.0 * n * G.S);
  return st;
}

/* one lockstep filter application: column c filters xs[c] into ys[c] */
int genil_apply(pevsl_Data *pevsl, GenIl &G, const double *const *xs, double *const *ys) {
  g_gen_ev.begin();
  int st = il_pack(G.n, G.S, xs, G.X(0));
  if (!st) {
    if (G.use_graph)
      st = graph_run(G.graph, pevsl, [&]() { return genil_degrees(pevsl, G); });
    else
      st = genil_degrees(pevsl, G);
  }
  if (!st) st = il_unpack(G.n, G.S, G.S, G.X(3), ys);
  g_gen_ev.end();
  return st;
}

}  // namespace

int pevsl_gen_cheblannr(pevsl_Data *pevsl, double *intv, int maxit, double tol, pevsl_Parvec *vinit,
                        pevsl_Polparams *pol, int *nevOut, double **lamo, pevsl_Parvecs **Wo,
                        double **reso, int *its, FILE *fstats) {
  *nevOut = 0;
  *lamo = nullptr;
  *Wo = nullptr;
  *reso = nullptr;
  if (its) *its = 0;
  const long n = pevsl->n, ld = gen_ld(n);
  GenSlice S;
  memcpy(S.intv, intv, sizeof S.intv);
  S.pol = pol;
  S.maxit = maxit;
  gs_begin(pevsl, S, fstats);
  if (!S.active) return S.status;
  double *V = (double *)ws(WS_BASIS, sizeof(double) * (size_t)ld * (size_t)(S.maxit + 1));
  double *Z = (double *)ws(WS_ZBASIS, sizeof(double) * (size_t)ld * (size_t)(S.maxit + 1));
  double *wf = (double *)ws(WS_GEN, sizeof(double) * 7 * (size_t)ld);
  if (!V || !Z || !wf) return PEVSL_ERR_NOMEM;
  S.V = V;
  S.Z = Z;
  double *vrand = wf + 4 * ld, *xs = wf + 5 * ld, *ys = wf + 6 * ld;
  const bool use_graph = graphable(pevsl);
  if (use_graph) pretune(pevsl);
  GenGraph fg;
  auto filter = [&](const double *in, double *out) -> int {
    g_gen_ev.begin();
    const int r = use_graph ? gen_filter_graphed(fg, pevsl, pol, in, out, wf, xs, ys, n)
                            : gen_filter(pevsl, pol, in, out, wf, n);
    g_gen_ev.end();
    return r;
  };
  /* filtered initial vector, unit B-norm */
  int st = filter(vinit->data, S.V);
  if (!st) st = gs_normalize0(pevsl, S, n);
  while (!st && S.active) {
    st = filter(S.Z + (size_t)S.k * ld, S.Z + (size_t)(S.k + 1) * ld);
    if (!st) st = gs_step(pevsl, S, n, ld, vrand, filter, fstats);
  }
  if (st) return st;
  if (its) *its = S.kdim;
  st = gs_finish(pevsl, S, vinit, n, ld, tol, fstats);
  if (st) return st;
  *nevOut = S.nev;
  *lamo = S.Lam;
  *Wo = S.Rvec;
  *reso = S.res;
  return 0;
}

/* Slices [0, ns) of one generalized problem in lockstep (the batched
 * entry points): one interleaved filter application per step for all
 * slices still iterating, the rest of each step per slice.  Applies when A
 * is the built-in matrix, the B-solve is the library's least-squares
 * polynomial, both matrices have short rows, 2 <= ns <= 16 and the filters
 * share the spectrum bounds; returns 1 (nothing done) otherwise.  Each
 * slice's result equals solving it alone (unless a breakdown restart draws
 * random vectors, whose order then differs). */
int pevsl_gen_cheblannr_lockstep(pevsl_Data *pevsl, int ns, const double *intvs, const int *maxits,
                                 double tol, pevsl_Parvec *vinit, pevsl_Polparams *pols,
                                 int *nevOut, double **lamo, pevsl_Parvecs **Wo, double **reso,
                                 int *its, int *status, FILE *fstats) {
  pevsl_devcsr *A = pevsl_builtin_A(pevsl);
  if (ns < 2 || ns > kMaxBatch || !A || A->lanes != 0 || !pevsl->Bsol ||
      pevsl->Bsol->func != pEVSL_LSPolSol || getenv("PEVSL_B200_GEN_LOCKSTEP_OFF"))
    return 1;
  const pevsl_lspol *L = (const pevsl_lspol *)pevsl->Bsol->data;
  if (!L || !L->B || L->B->lanes != 0 || L->deg < 1 || L->B->nrows != A->nrows) return 1;
  for (int s = 0; s < ns; s++)
    if (pols[s].cc != pols[0].cc || pols[s].dd != pols[0].dd || pols[s].deg < 1) return 1;
  const long n = pevsl->n, ld = gen_ld(n);
  std::vector<GenSlice> SL((size_t)ns);
  size_t basis = 0;
  for (int s = 0; s < ns; s++) {
    nevOut[s] = 0;
    lamo[s] = nullptr;
    Wo[s] = nullptr;
    reso[s] = nullptr;
    its[s] = 0;
    memcpy(SL[s].intv, intvs + 4 * (size_t)s, sizeof SL[s].intv);
    SL[s].pol = &pols[s];
    SL[s].maxit = maxits[s];
    gs_begin(pevsl, SL[s], fstats);
    status[s] = SL[s].status;
    if (SL[s].active) basis += (size_t)ld * (size_t)(SL[s].maxit + 1);
  }
  GenIl G;
  G.S = ns <= 2 ? 2 : ns <= 4 ? 4 : ns <= 8 ? 8 : 16;
  G.n = n;
  G.A = A;
  G.B = L->B;
  G.cc = pols[0].cc;
  G.dd = pols[0].dd;
  G.ccB = L->cc;
  G.ddB = L->dd;
  G.degB = L->deg;
  for (int s = 0; s < ns; s++) G.maxdeg = PEVSL_MAX(G.maxdeg, pols[s].deg);
  double *V = (double *)ws(WS_BASIS, sizeof(double) * (basis ? basis : 1));
  double *Z = (double *)ws(WS_ZBASIS, sizeof(double) * (basis ? basis : 1));
  /* four filter work vectors, a random vector, one scratch output per
   * padding or finished column */
  double *wf = (double *)ws(WS_GEN, sizeof(double) * (5 + kMaxBatch) * (size_t)ld);
  G.blk = (double *)ws(WS_IL, sizeof(double) * 7 * (size_t)n * (size_t)G.S);
  double *mu = (double *)ws(WS_ILMU, sizeof(double) * (size_t)(G.maxdeg + 1 + G.degB + 1) * G.S);
  if (!V || !Z || !wf || !G.blk || !mu) return PEVSL_ERR_NOMEM;
  G.smu = mu;
  G.lmu = mu + (size_t)(G.maxdeg + 1) * G.S;
  {
    std::vector<double> tab((size_t)(G.maxdeg + 1 + G.degB + 1) * G.S, 0.0);
    for (int s = 0; s < ns; s++)
      for (int k = 0; k <= pols[s].deg; k++) tab[(size_t)k * G.S + s] = pols[s].mu[k];
    for (int j = 0; j <= G.degB; j++)
      for (int c = 0; c < G.S; c++) tab[(size_t)(G.maxdeg + 1 + j) * G.S + c] = L->mu[j];
    int st0 = memcpy_async(mu, tab.data(), sizeof(double) * tab.size());
    if (!st0) st0 = sync();
    if (st0) return st0;
  }
  size_t off = 0;
  for (int s = 0; s < ns; s++)
    if (SL[s].active) {
      SL[s].V = V + off;
      SL[s].Z = Z + off;
      off += (size_t)ld * (size_t)(SL[s].maxit + 1);
    }
  double *vrand = wf + 4 * ld;
  auto dummy = [&](int c) { return wf + (5 + (size_t)c) * ld; };
  G.use_graph = graphable(pevsl);
  if (G.use_graph) pretune(pevsl);
  auto filter1 = [&](const pevsl_Polparams *pol, const double *in, double *out) -> int {
    return gen_filter(pevsl, pol, in, out, wf, n);
  };
  /* filtered initial vectors of every slice in one application */
  const double *xs[kMaxBatch];
  double *ys[kMaxBatch];
  for (int c = 0; c < G.S; c++) {
    xs[c] = vinit->data;
    ys[c] = c < ns && SL[c].active ? SL[c].V : dummy(c);
  }
  int st = genil_apply(pevsl, G, xs, ys);
  for (int s = 0; s < ns && !st; s++)
    if (SL[s].active) st = gs_normalize0(pevsl, SL[s], n);
  for (;;) {
    if (st) break;
    bool any = false;
    for (int c = 0; c < G.S; c++) {
      const bool on = c < ns && SL[c].active;
      any = any || on;
      xs[c] = on ? SL[c].Z + (size_t)SL[c].k * ld : vinit->data;
      ys[c] = on ? SL[c].Z + (size_t)(SL[c].k + 1) * ld : dummy(c);
    }
    if (!any) break;
    st = genil_apply(pevsl, G, xs, ys);
    for (int s = 0; s < ns && !st; s++) {
      if (!SL[s].active) continue;
      const pevsl_Polparams *pol = SL[s].pol;
      st = gs_step(pevsl, SL[s], n, ld, vrand,
                   [&](const double *in, double *out) { return filter1(pol, in, out); }, fstats);
    }
  }
  int first_err = st;
  for (int s = 0; s < ns && !st; s++) {
    if (!SL[s].ran || SL[s].status) continue;
    its[s] = SL[s].kdim;
    const int r = gs_finish(pevsl, SL[s], vinit, n, ld, tol, fstats);
    status[s] = r;
    if (r) {
      if (!first_err) first_err = r;
      continue;
    }
    nevOut[s] = SL[s].nev;
    lamo[s] = SL[s].Lam;
    Wo[s] = SL[s].Rvec;
    reso[s] = SL[s].res;
  }
  for (int s = 0; s < ns && !first_err; s++)
    if (status[s] && !first_err) first_err = status[s];
  return first_err;
}

/* ====================================================== C API */
extern "C" {

void pEVSL_SetupLSPol(int max_deg, double tol, double lmin, double lmax, pevsl_Parcsr *B,
                      double (*ffun)(double), void **vdata) {
  *vdata = nullptr;
  if (ensure() || !B) return;
  pevsl_devcsr *dB = pevsl_devcsr_of(B);
  pevsl_lspol *L = (pevsl_lspol *)calloc(1, sizeof(pevsl_lspol));
  if (!L || !dB) {
    free(L);
    return;
  }
  L->N = B->ncol_global;
  L->n = B->ncol_local;
  L->nfirst = B->first_col;
  L->max_deg = max_deg;
  L->intv[0] = lmin;
  L->intv[1] = lmax;
  L->tol = tol;
  L->comm = B->comm;
  L->B = dB;
  L->mu = (double *)calloc((size_t)(max_deg > 0 ? max_deg : 1), sizeof(double));
  if (!L->mu || fail(cudaMalloc(&L->wk, sizeof(double) * 3 * (size_t)(L->n > 0 ? L->n : 1)),
                     "cudaMalloc lspol")) {
    free(L->mu);
    free(L);
    return;
  }
  if (pevsl_lspol_coefs(ffun, max_deg, tol, lmin, lmax, L->mu, &L->deg, &L->cc, &L->dd)) {
    cudaFree(L->wk);
    free(L->mu);
    free(L);
    return;
  }
  *vdata = L;
}

void pEVSL_SetupLSPolRec(int max_deg, double tol, double lmin, double lmax, pevsl_Parcsr *B,
                         void **vdata) {
  pEVSL_SetupLSPol(max_deg, tol, lmin, lmax, B, pevsl_lspol_rec(), vdata);
}

void pEVSL_SetupLSPolSqrt(int max_deg, double tol, double lmin, double lmax, pevsl_Parcsr *B,
                          void **vdata) {
  pEVSL_SetupLSPol(max_deg, tol, lmin, lmax, B, pevsl_lspol_isqrt(), vdata);
}

void pEVSL_LSPolSol(double *db, double *dx, void *data) {
  if (lspol_apply((pevsl_lspol *)data, db, dx) == 0) sync();
}

void pEVSL_LSPolFree(void *vdata) {
  pevsl_lspol *L = (pevsl_lspol *)vdata;
  if (!L) return;
  if (L->wk) {
    cudaStreamSynchronize(ctx().stream);
    cudaFree(L->wk);
  }
  free(L->mu);
  free(L);
}

int pEVSL_B200_LSPolDegree(const void *vdata, double *mu_out, int cap) {
  const pevsl_lspol *L = (const pevsl_lspol *)vdata;
  if (!L) return PEVSL_ERR_ARG;
  for (int k = 0; mu_out && k <= L->deg && k < cap; k++) mu_out[k] = L->mu[k];
  return L->deg;
}

int pevsl_lspol_size(const void *lspol) { return lspol ? ((const pevsl_lspol *)lspol)->n : 0; }
int pevsl_chebiter_size(const void *cheb) { return cheb ? ((const pevsl_chebiter *)cheb)->n : 0; }

int pEVSL_ChebIterSetup(double lmin, double lmax, int deg, pevsl_Parcsr *A, void **data) {
  *data = nullptr;
  if (ensure()) return PEVSL_ERR_CUDA;
  pevsl_devcsr *dA = A ? pevsl_devcsr_of(A) : nullptr;
  if (!dA) return PEVSL_ERR_ARG;
  pevsl_chebiter *C = (pevsl_chebiter *)calloc(1, sizeof(pevsl_chebiter));
  if (!C) return PEVSL_ERR_NOMEM;
  C->lb = lmin;
  C->ub = lmax;
  C->deg = PEVSL_MAX(deg, 0);
  C->N = A->ncol_global;
  C->n = A->ncol_local;
  C->nfirst = A->first_col;
  C->A = dA;
  C->comm = A->comm;
  if (fail(cudaMalloc(&C->wk, sizeof(double) * 4 * (size_t)(C->n > 0 ? C->n : 1)),
           "cudaMalloc chebiter")) {
    free(C);
    return PEVSL_ERR_NOMEM;
  }
  C->ev_ok = true;
  for (int i = 0; i < 64 && C->ev_ok; i++) C->ev_ok = cudaEventCreate(&C->ev[i]) == cudaSuccess;
  *data = C;
  return 0;
}

/* called directly (not through an instance's solve slot): the result is
 * complete on return, as for a user callback */
void pEVSL_ChebIterSolv1(double *db, double *dx, void *data) {
  pevsl_chebiter *C = (pevsl_chebiter *)data;
  if (!C || !C->A) return;
  if (chebiter_time(C, chebiter1, db, dx) == 0) sync();
}

void pEVSL_ChebIterSolv2(double *db, double *dx, void *data) {
  pevsl_chebiter *C = (pevsl_chebiter *)data;
  if (!C || !C->A) return;
  if (chebiter_time(C, chebiter2, db, dx) == 0) sync();
}

void pEVSL_ChebIterFree(void *vdata) {
  pevsl_chebiter *C = (pevsl_chebiter *)vdata;
  if (!C) return;
  cudaStreamSynchronize(ctx().stream);
  cudaFree(C->wk);
  if (C->ev_ok)
    for (int i = 0; i < 64; i++) cudaEventDestroy(C->ev[i]);
  free(C);
}

/* the reference keeps no history unless built with SAVE_CONV_HIST */
double *pEVSL_ChebIterGetRes(void *data) { return nullptr; }

void pEVSL_ChebIterStatsPrint(void *data, FILE *fstats) {
  pevsl_chebiter *C = (pevsl_chebiter *)data;
  if (!C || !fstats) return;
  chebiter_flush(C);
  fprintf(fstats, "= = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = =\n");
  if (C->n_chebmv)
    fprintf(fstats, "   Matvec in ChebIter        :  %f (%8ld, avg %f)\n", C->t_chebmv,
            (long)C->n_chebmv, C->t_chebmv / C->n_chebmv);
  fprintf(fstats, "= = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = = =\n");
}

void pEVSL_B200_GenCounters(uint64_t *filters, uint64_t *degrees, double *bytes, double *ms) {
  g_gen_ev.flush();
  if (filters) *filters = g_gen_filters;
  if (degrees) *degrees = g_gen_degrees;
  if (bytes) *bytes = g_gen_bytes;
  if (ms) *ms = g_gen_ms;
}

void pEVSL_B200_ResetGenCounters(void) {
  g_gen_ev.flush();
  g_gen_filters = g_gen_degrees = 0;
  g_gen_bytes = g_gen_ms = 0.0;
}

/* y = p(A B^{-1}) v for the generalized problem (the filter of
 * SRC/chebpol.c:509-574 with ifGenEv), device or managed vectors */
int pEVSL_B200_ChebAvGen(pevsl_Data *pevsl, pevsl_Polparams *pol, const double *v, double *y) {
  if (ensure()) return PEVSL_ERR_CUDA;
  const long n = pevsl->n;
  double *w = (double *)ws(WS_GEN, sizeof(double) * 5 * (size_t)gen_ld(n));
  if (!w) return PEVSL_ERR_NOMEM;
  int st = gen_filter(pevsl, pol, v, y, w, n);
  if (!st) st = sync();
  return st;
}

}  // extern "C"
