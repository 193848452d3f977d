/*
 * The solvers of the slicing path, driven from the host with every vector
 * operation on the GPU:
 *
 *   filter application   pEVSL_ChebAv     SRC/chebpol.c:509-574
 *   KPM DOS              pEVSL_Kpmdos     SRC/kpmdos.c:36-197
 *   Lanczos DOS          pEVSL_LanDosG    SRC/landos.c:40-314
 *   spectrum bounds      pEVSL_LanTrbounds SRC/lantrbnd.c:31-408
 *   filtered Lanczos     pEVSL_ChebLanNr  SRC/cheblanNr.c:54-448
 *
 * The control flow (step counts, tests, breakdown restarts, acceptance) is
 * the reference's.  The host reads two scalars per Lanczos step (alpha,
 * beta); everything else stays on the device.  The DGKS second
 * Gram-Schmidt pass is decided on the device.  When A is the built-in
 * parcsr, the SpMV is fused into the recurrence kernels; a user matvec
 * (pEVSL_SetAMatvec) is called with device pointers instead.
 */
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <thread>
#include <vector>

#include "gpu.cuh"
#include "gpu_device.cuh"

using namespace pv;

namespace {

const double kEta = 0.70710678118654752440; /* 1/sqrt(2): DGKS threshold */

/* ------------------------------------------------------------ event timer
 * Sums the device time of repeated segments (filter applications,
 * reorthogonalisation) with a small pool of event pairs that is drained
 * whenever it fills; the pools live for the whole process. */
struct SegTimer {
  static constexpr int kPairs = 64;
  cudaEvent_t ev[2 * kPairs];
  int used = 0;
  double acc_ms = 0.0;
  bool ok = false;
  void init() {
    if (!ok) {
      ok = true;
      for (int i = 0; i < 2 * kPairs; i++)
        if (cudaEventCreate(&ev[i]) != cudaSuccess) ok = false;
    }
    used = 0;
    acc_ms = 0.0;
  }
  void begin() {
    if (!ok) return;
    if (used == kPairs) flush();
    cudaEventRecord(ev[2 * used], ctx().stream);
  }
  void end() {
    if (!ok) return;
    cudaEventRecord(ev[2 * used + 1], ctx().stream);
    used++;
  }
  void flush() {
    if (!ok || used == 0) return;
    cudaEventSynchronize(ev[2 * used - 1]);
    for (int i = 0; i < used; i++) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]) == cudaSuccess) acc_ms += ms;
    }
    used = 0;
  }
};
SegTimer g_t_pol, g_t_orth;

/* process-wide counters of the fused filter kernel (pEVSL_B200_FilterCounters) */
uint64_t g_filter_launches = 0;
uint64_t g_filter_persistent = 0; /* persistent filter launches (each covers many degrees) */
double g_filter_bytes = 0.0;
double g_filter_ms = 0.0;

/* algorithmic HBM bytes of one fused filter degree: the CSR (int32 column
 * indices, fp64 values, int32 row pointers) plus v_k read once, and
 * v_{k-1}, y read / v_{k+1}, y written (first degree: no v_{k-1}, y only
 * written) */
double cheb_step_bytes(const pevsl_devcsr *A, int first) {
  const double n = A->nrows;
  return entry_bytes(A, false) * (double)A->nnz + 4.0 * (n + 1) + (first ? 24.0 : 40.0) * n;
}

/* matvec through the installed operator: fused kernels use the device CSR
 * directly; this is for the plain y = A x steps. */
int apply_A(pevsl_Data *pevsl, const double *x, double *y) {
  pevsl_devcsr *A = pevsl_builtin_A(pevsl);
  pevsl->stats->n_mvA++;
  if (A) return spmv(A, x, y);
  if (!pevsl->Amv || !pevsl->Amv->func) return PEVSL_ERR_NOMATVEC;
  if (sync()) return PEVSL_ERR_CUDA;
  pevsl->Amv->func((double *)x, y, pevsl->Amv->data);
  return fail(cudaDeviceSynchronize(), "user matvec");
}

/* y = p((A - cc)/dd) v with mu[0..deg]; w3 holds 3n doubles. */
int cheb_apply(pevsl_Data *pevsl, const pevsl_Polparams *pol, const double *v, double *y,
               double *w3, long n) {
  pevsl_devcsr *A = pevsl_builtin_A(pevsl);
  const int m = pol->deg;
  const double cc = pol->cc, dd = pol->dd, t1 = 1.0 / dd, t2 = 2.0 / dd;
  const double *mu = pol->mu;
  pevsl->stats->n_polAv++;
  if (m <= 0) {
    if (vcopy(v, y, n)) return PEVSL_ERR_CUDA;
    return vscal(y, n, mu[0]);
  }
  if (!A && (!pevsl->Amv || !pevsl->Amv->func)) return PEVSL_ERR_NOMATVEC;
  double *buf[2] = {w3, w3 + n};
  double *ax = A ? nullptr : (double *)ws(WS_VEC, sizeof(double) * (size_t)n);
  if (!A && !ax) return PEVSL_ERR_NOMEM;
  const double *vk = v, *vkm1 = nullptr;
  for (int k = 1; k <= m; k++) {
    /* two work vectors: from degree 3 on, v_{k+1} replaces v_{k-1} in place */
    double *vkp1 = k <= 2 ? buf[k - 1] : const_cast<double *>(vkm1);
    const double t = k == 1 ? t1 : t2;
    int st;
    if (A) {
      st = cheb_step(A, vk, vkm1, vkp1, y, cc, t, mu[0], mu[k], k == 1);
      g_filter_launches++;
      g_filter_bytes += cheb_step_bytes(A, k == 1);
    } else {
      st = apply_A(pevsl, vk, ax);
      if (!st) st = cheb_combine(n, ax, vk, vkm1, vkp1, y, cc, t, mu[0], mu[k], k == 1);
      pevsl->stats->n_mvA--; /* counted below */
    }
    if (st) return st;
    vkm1 = vk;
    vk = vkp1;
  }
  pevsl->stats->n_mvA += (size_t)m;
  return 0;
}

/* One filter application of a batch: y = p(A) x (pEVSL_ChebAv,
 * SRC/chebpol.c:509-574) for entry e with its own device CSR, polynomial
 * and work space of 16 * ld bytes (two FP64 recurrence vectors, or, in
 * FP32, the FP32 copy of x, two FP32 recurrence vectors and the FP32
 * accumulator; the last degree writes y in FP64). */
struct FilterJob {
  pevsl_Data *pevsl;          /* statistics */
  const pevsl_devcsr *A;
  const double *x;
  double *y;
  const pevsl_Polparams *pol;
  const double *dmu;          /* pol->mu on the device (persistent form) */
  void *work;
  long ld;                    /* spacing of the work vectors: >= n, 256-byte multiple */
};

/* Form of the batched filter: 0 = one cheb_step_batch launch per degree
 * serving every entry (any matrices, up to kMaxEntries), 1 = one persistent
 * cooperative launch for all degrees and entries, 2 (default) = the
 * launches of form 0 captured in a CUDA graph per set of live slices and
 * replayed (filter_graphed).  One launch per degree beat the persistent
 * kernel (81 vs 119 us per degree for 4 slices at 10^6 rows, 4.1 vs 6.1 us
 * at 8000 rows): the grid barrier costs more than the gap between launches. */
static int g_filter_form_override = -1; /* -1: not read yet */
static int filter_form_setting() {
  if (g_filter_form_override < 0) {
    const char *e = getenv("PEVSL_B200_FILTER_FORM");
    const int v = e ? atoi(e) : 2;
    g_filter_form_override = (v >= 0 && v <= 2) ? v : 2;
  }
  return g_filter_form_override;
}
static int filter_form() { return filter_form_setting() == 1 ? 1 : 0; }

/* Interleaved form of the batched filter (PEVSL_B200_INTERLEAVE: 1 on, the
 * default; 0 off): the live slices of one problem on one matrix run with
 * their vectors row-interleaved, so one gather serves every slice
 * (cheb_step_il); the input is packed once and the result unpacked once per
 * filter application.  Applies to 2..16 FP64 slices on a short-row matrix
 * of at least 2^16 rows whose polynomials share the spectrum bounds
 * (cc, dd).  Measured per
 * degree against the grid-interleaved batch kernel: 100^3, 4 slices 52.6
 * vs 80.1 us (2 slices 34.0 vs 44.6, 16 slices 182 vs 310); random sparse
 * n = 2e6 with ~17 entries per row, 16 slices 758 vs 2160 us. */
static int interleave_setting() {
  static int v = -1;
  if (v < 0) {
    const char *e = getenv("PEVSL_B200_INTERLEAVE");
    v = e ? atoi(e) != 0 : 1;
  }
  return v;
}

static int il_width(int nlive) { return nlive <= 2 ? 2 : nlive <= 4 ? 4 : nlive <= 8 ? 8 : 16; }

/* Slices per interleaved group.  A group's whole filter application runs
 * before the next group's, and its working set from one degree to the next
 * -- three row-interleaved vector blocks (24 n bytes per slice) and the
 * matrix -- stays in the 126 MB L2 when it is at most half of it; wider
 * groups stream it from HBM at every degree.  So a group holds the most
 * slices (2, 4, 8 or 16) that fit in 64 MB, at least 2.  Measured per
 * degree at 100^3 (n = 1e6, packed matrix 25 MB): 2 slices 20.1 us (0.64 of
 * the HBM peak in algorithmic bytes, L2-resident), 4 slices 44.0-46.7 us.
 * PEVSL_B200_IL_MAXS caps it by hand (2..16). */
static int il_group_cap(const pevsl_devcsr *A) {
  const char *e = getenv("PEVSL_B200_IL_MAXS"); /* read per call: tests change it */
  const int env = e ? atoi(e) : 0;
  if (env >= 2) return PEVSL_MIN(env, kMaxBatch);
  const double mat = 3.0 * (double)A->nnz + 4.0 * (A->nrows + 1.0);
  int cap = 2;
  for (int S = 4; S <= kMaxBatch; S *= 2)
    if (24.0 * (double)A->nrows * S + mat <= 64.0 * 1024 * 1024) cap = S;
  return cap;
}

/* Degrees per accumulator update in the interleaved filter
 * (PEVSL_B200_IL_DEFER: 1, 2 or 3, the default).  With D > 1 a launch adds
 * the terms of the last D degrees to y (the first update at degree
 * min(D, 2), the last at the group's top degree) and the launches between
 * updates neither read nor write y: 24 instead of 40 bytes per row and
 * slice.  The sum is the same, term by term in degree order. */
static int il_defer_setting() {
  static int v = -1;
  if (v < 0) {
    const char *e = getenv("PEVSL_B200_IL_DEFER");
    v = e ? atoi(e) : 3;
    if (v < 1 || v > 3) v = 3;
  }
  return v;
}

/* terms that degree k of a group of top degree maxdeg adds to y when the
 * last update was at degree lastw (0: none yet), under deferral D */
static int il_terms(int k, int lastw, int maxdeg, int D) {
  const int span = lastw == 0 ? PEVSL_MIN(D, 2) : D;
  return (k == maxdeg || k - lastw == span) ? k - lastw : 0;
}

/* a set of slices the interleaved form serves together */
struct IlGroup {
  const pevsl_devcsr *A;
  int idx[kMaxBatch]; /* job indices, in job order */
  int cnt, S, maxdeg;
  double cc, dd;
  size_t ws_off, mu_off; /* in doubles, into WS_IL / WS_ILMU */
};

/* The entries the interleaved form takes: groups of 2..16 live FP64
 * entries on one short-row matrix of at least 2^16 rows with the same
 * spectrum bounds (cc, dd), in job order; the other entries stay with the
 * grid-interleaved batch kernel.  Below 2^16 rows the problem sits in L2
 * and the launch is latency-bound, where the batch kernel is faster (20^3,
 * 5 slices: the whole run 0.115 vs 0.125 s). */
static void il_partition(int ne, const FilterJob *jobs, bool fp32, std::vector<IlGroup> &g,
                         std::vector<char> &taken) {
  g.clear();
  taken.assign((size_t)ne, 0);
  if (fp32 || !interleave_setting()) return;
  std::vector<char> seen((size_t)ne, 0);
  size_t ws_off = 0, mu_off = 0;
  for (int e = 0; e < ne; e++) {
    const FilterJob &J = jobs[e];
    if (seen[e] || J.pol->deg <= 0) continue;
    const pevsl_devcsr *A = J.A;
    if (A->lanes != 0 || A->nrows < 65536) continue;
    std::vector<int> L;
    for (int f = e; f < ne; f++)
      if (!seen[f] && jobs[f].pol->deg > 0 && jobs[f].A == A && jobs[f].pol->cc == J.pol->cc &&
          jobs[f].pol->dd == J.pol->dd) {
        seen[f] = 1;
        L.push_back(f);
      }
    const size_t cap = (size_t)il_group_cap(A);
    for (size_t c0 = 0; c0 < L.size(); c0 += cap) {
      const int cnt = (int)PEVSL_MIN(cap, L.size() - c0);
      if (cnt < 2) continue;
      IlGroup G;
      G.A = A;
      G.cnt = cnt;
      G.S = il_width(cnt);
      G.maxdeg = 0;
      G.cc = J.pol->cc;
      G.dd = J.pol->dd;
      for (int i = 0; i < cnt; i++) {
        G.idx[i] = L[c0 + i];
        taken[(size_t)G.idx[i]] = 1;
        G.maxdeg = PEVSL_MAX(G.maxdeg, jobs[G.idx[i]].pol->deg);
      }
      G.ws_off = ws_off;
      G.mu_off = mu_off;
      ws_off += 4 * (size_t)A->nrows * (size_t)G.S;
      mu_off += (size_t)(G.maxdeg + 1) * (size_t)G.S;
      g.push_back(G);
    }
  }
}

static size_t il_ws_doubles(const std::vector<IlGroup> &g) {
  return g.empty() ? 0 : g.back().ws_off + 4 * (size_t)g.back().A->nrows * (size_t)g.back().S;
}
static size_t il_mu_doubles(const std::vector<IlGroup> &g) {
  return g.empty() ? 0 : g.back().mu_off + (size_t)(g.back().maxdeg + 1) * (size_t)g.back().S;
}

/* workspace and per-degree coefficient tables of the interleaved groups,
 * prepared outside any stream capture: row k of a group's table holds mu_k
 * of each of its slices (0 past a slice's degree, where its y then stays
 * unchanged) */
static int il_prepare(int ne, const FilterJob *jobs, bool fp32) {
  std::vector<IlGroup> g;
  std::vector<char> taken;
  il_partition(ne, jobs, fp32, g, taken);
  if (g.empty()) return 0;
  if (!ws(WS_IL, sizeof(double) * il_ws_doubles(g))) return PEVSL_ERR_NOMEM;
  double *dmu = (double *)ws(WS_ILMU, sizeof(double) * il_mu_doubles(g));
  if (!dmu) return PEVSL_ERR_NOMEM;
  std::vector<double> tab(il_mu_doubles(g), 0.0);
  for (const IlGroup &G : g)
    for (int c = 0; c < G.cnt; c++) {
      const pevsl_Polparams *pol = jobs[G.idx[c]].pol;
      for (int k = 0; k <= pol->deg; k++) tab[G.mu_off + (size_t)k * G.S + c] = pol->mu[k];
    }
  if (memcpy_async(dmu, tab.data(), sizeof(double) * tab.size())) return PEVSL_ERR_CUDA;
  return sync();
}

/* buffers of group G: packed input, two recurrence blocks, accumulator */
static void il_buffers(const IlGroup &G, double **X0, double **B0, double **B1, double **Y) {
  const size_t blk = (size_t)G.A->nrows * (size_t)G.S;
  *X0 = (double *)ctx().ws[WS_IL] + G.ws_off;
  *B0 = *X0 + blk;
  *B1 = *B0 + blk;
  *Y = *B1 + blk;
}

static double filter_bytes_degree(const pevsl_devcsr *A, int deg_k, bool fp32, bool last) {
  const double n = A->nrows, vb = fp32 ? 4.0 : 8.0;
  return (deg_k == 1 ? 3.0 : 5.0) * vb * n + (last ? 4.0 * n : 0.0);
}

static int cheb_filter_batch(int ne, const FilterJob *jobs, bool fp32) {
  if (ne <= 0) return 0;
  if (ne > kMaxEntries) return PEVSL_ERR_ARG;
  int st = 0, maxdeg = 0, nlive = 0;
  int live[kMaxEntries];
  for (int e = 0; e < ne && !st; e++) {
    const FilterJob &J = jobs[e];
    const pevsl_Polparams *pol = J.pol;
    const long n = J.A->nrows;
    if (fp32 && !J.A->a32) return PEVSL_ERR_ARG;
    J.pevsl->stats->n_polAv++;
    J.pevsl->stats->n_mvA += (size_t)PEVSL_MAX(pol->deg, 0);
    if (pol->deg <= 0) {
      st = vcopy(J.x, J.y, n);
      if (!st) st = vscal(J.y, n, pol->mu[0]);
      continue;
    }
    maxdeg = PEVSL_MAX(maxdeg, pol->deg);
    if (fp32) st = cvt_f64_f32(n, J.x, (float *)J.work);
    live[nlive++] = e;
  }
  if (st || !nlive) return st;
  /* matrix bytes: each distinct matrix once per degree, up to the largest
   * degree of its entries */
  double mat_bytes = 0.0;
  for (int i = 0; i < nlive; i++) {
    const pevsl_devcsr *A = jobs[live[i]].A;
    bool seen = false;
    for (int t = 0; t < i && !seen; t++) seen = jobs[live[t]].A == A;
    if (seen) continue;
    int dmax = 0;
    for (int t = i; t < nlive; t++)
      if (jobs[live[t]].A == A) dmax = PEVSL_MAX(dmax, jobs[live[t]].pol->deg);
    mat_bytes += (double)dmax * ((fp32 ? 8.0 : 12.0) * (double)A->nnz + 4.0 * (A->nrows + 1.0));
  }
  const int form = filter_form();
  if (form == 1) {
    /* table sorted by non-increasing degree (stable: ties keep their order) */
    FiltDev tab[kMaxEntries];
    int ord[kMaxEntries];
    for (int i = 0; i < nlive; i++) ord[i] = live[i];
    for (int i = 1; i < nlive; i++) {
      const int v = ord[i];
      int j = i - 1;
      while (j >= 0 && jobs[ord[j]].pol->deg < jobs[v].pol->deg) {
        ord[j + 1] = ord[j];
        j--;
      }
      ord[j + 1] = v;
    }
    double bytes = mat_bytes;
    for (int i = 0; i < nlive; i++) {
      const FilterJob &J = jobs[ord[i]];
      const pevsl_devcsr *A = J.A;
      FiltDev &E = tab[i];
      E.ia = A->ia;
      E.ja = A->ja;
      E.a = fp32 ? (const void *)A->a32 : (const void *)A->a;
      E.n = (int)A->nrows;
      E.deg = J.pol->deg;
      E.fp32 = fp32;
      E.pad = 0;
      E.cc = J.pol->cc;
      E.t1 = 1.0 / J.pol->dd;
      E.t2 = 2.0 / J.pol->dd;
      E.mu = J.dmu;
      if (fp32) {
        float *w = (float *)J.work;
        E.x = w;
        E.b0 = w + J.ld;
        E.b1 = w + 2 * J.ld;
        E.acc = w + 3 * J.ld;
      } else {
        double *w = (double *)J.work;
        E.x = J.x;
        E.b0 = w;
        E.b1 = w + J.ld;
        E.acc = J.y;
      }
      E.y = J.y;
      for (int k = 1; k <= E.deg; k++) bytes += filter_bytes_degree(A, k, fp32, fp32 && k == E.deg);
    }
    st = cheb_filter_persistent(nlive, tab, maxdeg);
    g_filter_launches += (uint64_t)maxdeg;
    g_filter_bytes += bytes;
    g_filter_persistent++;
    /* a barrier wait that ran out leaves the filter half applied: report it
     * before anything uses the result (one 16-byte read per application) */
    if (!st && persistent_filter_error()) {
      fprintf(stderr, "pevsl_b200: persistent filter barrier timed out\n");
      st = PEVSL_ERR_CUDA;
    }
    return st;
  }
  /* one launch per degree for all live entries; a matrix is read once per
   * launch for all entries on it.  Entries taken by interleaved groups run
   * as one interleaved launch per group and degree instead. */
  std::vector<IlGroup> ig;
  std::vector<char> taken;
  il_partition(ne, jobs, fp32, ig, taken);
  std::vector<std::array<const double *, 3>> ilv(ig.size()); /* vk, vkm1 per group */
  std::vector<int> ilw(ig.size(), 0);                          /* last degree added to y */
  const int defer = il_defer_setting();
  if (!ig.empty()) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(ctx().stream, &cs);
    /* inside a capture the caller prepared the workspace and coefficients */
    if (cs == cudaStreamCaptureStatusNone) st = il_prepare(ne, jobs, fp32);
    if (!st && (!ctx().ws[WS_IL] || ctx().wsz[WS_IL] < sizeof(double) * il_ws_doubles(ig) ||
                !ctx().ws[WS_ILMU] || ctx().wsz[WS_ILMU] < sizeof(double) * il_mu_doubles(ig)))
      st = PEVSL_ERR_ARG; /* il_prepare not run before the capture */
    for (size_t gi = 0; gi < ig.size() && !st; gi++) {
      const IlGroup &G = ig[gi];
      const double *xs[kMaxBatch];
      for (int c = 0; c < G.S; c++) xs[c] = jobs[G.idx[c < G.cnt ? c : 0]].x; /* padding: mu 0 */
      double *X0, *B0, *B1, *Y;
      il_buffers(G, &X0, &B0, &B1, &Y);
      st = il_pack(G.A->nrows, G.S, xs, X0);
      ilv[gi] = {X0, nullptr, nullptr};
    }
    if (st) return st;
  }
  std::vector<const void *> vk(nlive), vkm1(nlive);
  std::vector<void *> b0(nlive), b1(nlive), acc(nlive);
  for (int i = 0; i < nlive; i++) {
    const FilterJob &J = jobs[live[i]];
    if (fp32) {
      float *w = (float *)J.work;
      vk[i] = w;
      b0[i] = w + J.ld;
      b1[i] = w + 2 * J.ld;
      acc[i] = w + 3 * J.ld;
    } else {
      double *w = (double *)J.work;
      vk[i] = J.x;
      b0[i] = w;
      b1[i] = w + J.ld;
      acc[i] = J.y;
    }
    vkm1[i] = nullptr;
  }
  /* the interleaved groups one after another, each through all its
   * degrees, so that a group's working set stays in L2 between degrees
   * (il_group_cap); the groups are independent, so every slice's bits are
   * those of the degree-major order */
  for (size_t gi = 0; gi < ig.size() && !st; gi++) {
    const IlGroup &G = ig[gi];
    double *X0, *B0, *B1, *Y;
    il_buffers(G, &X0, &B0, &B1, &Y);
    const double *dmu = (const double *)ctx().ws[WS_ILMU] + G.mu_off;
    for (int k = 1; k <= G.maxdeg && !st; k++) {
      const double *gk = ilv[gi][0], *gkm1 = ilv[gi][1];
      double *gkp1 = k == 1 ? B0 : k == 2 ? B1 : const_cast<double *>(gkm1);
      const int ny = il_terms(k, ilw[gi], G.maxdeg, defer), fresh = ny > 0 && ilw[gi] == 0;
      st = cheb_step_il_y(G.A, G.S, gk, gk, gkm1, gkp1, Y, G.cc, (k == 1 ? 1.0 : 2.0) / G.dd, dmu,
                          dmu + (size_t)k * G.S, ny, fresh);
      if (ny > 0) ilw[gi] = k;
      /* read v_k, v_{k-1} (from degree 2), write v_{k+1}; y read unless
       * fresh and written when updated */
      const double vec = (k == 1 ? 16.0 : 24.0) + (ny > 0 ? (fresh ? 8.0 : 16.0) : 0.0);
      g_filter_bytes += il_entry_bytes(G.A) * (double)G.A->nnz + 4.0 * (G.A->nrows + 1.0) +
                        vec * (double)G.A->nrows * G.S;
      g_filter_launches++;
      ilv[gi][1] = gk;
      ilv[gi][0] = gkp1;
    }
  }
  bool others = false;
  for (int i = 0; i < nlive && !others; i++) others = !taken[(size_t)live[i]];
  std::vector<ChebEntry> en(nlive);
  for (int k = 1; k <= maxdeg && !st && others; k++) {
    int nb = 0;
    double bytes = 0.0;
    for (int i = 0; i < nlive; i++) {
      const FilterJob &J = jobs[live[i]];
      const pevsl_Polparams *pol = J.pol;
      if (taken[(size_t)live[i]]) continue;
      if (k > pol->deg) continue;
      /* two work vectors: from degree 3 on, v_{k+1} replaces v_{k-1} */
      void *vkp1 = k == 1 ? b0[i] : k == 2 ? b1[i] : const_cast<void *>(vkm1[i]);
      const bool last = fp32 && k == pol->deg;
      en[nb++] = ChebEntry{J.A, vk[i], vkm1[i], vkp1, acc[i], last ? J.y : nullptr,
                           pol->cc, (k == 1 ? 1.0 : 2.0) / pol->dd, pol->mu[0], pol->mu[k],
                           k == 1};
      bytes += filter_bytes_degree(J.A, k, fp32, last);
      vkm1[i] = vk[i];
      vk[i] = vkp1;
    }
    /* matrix bytes: each distinct matrix of this degree's entries once */
    for (int i = 0; i < nb; i++) {
      bool seen = false;
      for (int t = 0; t < i && !seen; t++) seen = en[t].A == en[i].A;
      if (!seen)
        bytes += entry_bytes(en[i].A, fp32, nb > 1) * (double)en[i].A->nnz +
                 4.0 * (en[i].A->nrows + 1.0);
    }
    if (nb == 0) {
      /* every live entry of this degree is in an interleaved group */
    } else if (nb == 1 && !fp32 && en[0].A->lanes == 0) {
      /* one live slice: the one-vector kernel (packed entries when the
       * matrix has them); the same arithmetic as the batch */
      const ChebEntry &c = en[0];
      st = cheb_step(c.A, (const double *)c.vk, (const double *)c.vkm1, (double *)c.vkp1,
                     (double *)c.y, c.cc, c.t, c.mu0, c.muk, c.first);
    } else {
      st = cheb_step_batch(nb, en.data(), fp32);
    }
    g_filter_launches++;
    g_filter_bytes += bytes;
  }
  for (size_t gi = 0; gi < ig.size() && !st; gi++) {
    const IlGroup &G = ig[gi];
    double *ys[kMaxBatch];
    for (int c = 0; c < G.cnt; c++) ys[c] = jobs[G.idx[c]].y;
    double *X0, *B0, *B1, *Y;
    il_buffers(G, &X0, &B0, &B1, &Y);
    st = il_unpack(G.A->nrows, G.S, G.cnt, Y, ys);
  }
  return st;
}

/* CUDA graph form of one batched filter application.  The degrees read the
 * input from, and accumulate into, two staging vectors in each slice's
 * work space (at 16 ld and 24 ld bytes), so that the launch sequence of a
 * given set of slices never changes: it is captured once (all degrees, the
 * FP32 conversion included) and replayed, with one copy in and one copy out
 * per slice around it.  A new set of live slices is captured anew. */
static bool filter_graph_enabled() { return filter_form_setting() == 2; }

struct FilterGraph {
  cudaGraphExec_t exec = nullptr;
  std::vector<char> key; /* live slices of the captured sequence */
  bool mixed = false;
  uint64_t launches = 0, kernel_launches = 0;
  double bytes = 0.0;
  ~FilterGraph() {
    if (exec) cudaGraphExecDestroy(exec);
  }
};

static int filter_graphed(FilterGraph &fg, const std::vector<char> &sel, std::vector<FilterJob> &jobs) {
  Ctx &c = ctx();
  const int ne = (int)jobs.size();
  std::vector<FilterJob> staged(jobs);
  int st = 0;
  for (int e = 0; e < ne && !st; e++) {
    double *xs = (double *)((char *)jobs[e].work + 16 * (size_t)jobs[e].ld);
    st = memcpy_async(xs, jobs[e].x, sizeof(double) * (size_t)jobs[e].A->nrows);
    staged[e].x = xs;
    staged[e].y = xs + jobs[e].ld;
  }
  if (st) return st;
  if (!fg.exec || fg.key != sel) {
    if (fg.exec) cudaGraphExecDestroy(fg.exec);
    fg.exec = nullptr;
    if (filter_form() == 0) {
      st = il_prepare(ne, staged.data(), fg.mixed);
      if (st) return st;
    }
    const uint64_t l0 = g_filter_launches, k0 = c.launches;
    const double b0 = g_filter_bytes;
    if (fail(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal), "BeginCapture"))
      return PEVSL_ERR_CUDA;
    st = cheb_filter_batch(ne, staged.data(), fg.mixed);
    cudaGraph_t gr = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(c.stream, &gr);
    if (st || fail(ec, "EndCapture")) {
      if (gr) cudaGraphDestroy(gr);
      return st ? st : PEVSL_ERR_CUDA;
    }
    const cudaError_t ei = cudaGraphInstantiate(&fg.exec, gr, 0);
    cudaGraphDestroy(gr);
    if (fail(ei, "cudaGraphInstantiate")) {
      fg.exec = nullptr;
      return PEVSL_ERR_CUDA;
    }
    fg.key = sel;
    fg.launches = g_filter_launches - l0;
    fg.kernel_launches = c.launches - k0;
    fg.bytes = g_filter_bytes - b0;
  } else {
    /* the statistics a direct call would have counted */
    for (int e = 0; e < ne; e++) {
      jobs[e].pevsl->stats->n_polAv++;
      jobs[e].pevsl->stats->n_mvA += (size_t)PEVSL_MAX(jobs[e].pol->deg, 0);
    }
    g_filter_launches += fg.launches;
    g_filter_bytes += fg.bytes;
    c.launches += fg.kernel_launches;
  }
  if (fail(cudaGraphLaunch(fg.exec, c.stream), "cudaGraphLaunch")) return PEVSL_ERR_CUDA;
  for (int e = 0; e < ne && !st; e++)
    st = memcpy_async(jobs[e].y, staged[e].y, sizeof(double) * (size_t)jobs[e].A->nrows);
  return st;
}

/* One CGS_DGKS (SRC/miscla.c:211-240) of v against V(:, 0:k).  On entry the
 * device slot S_NRM0 holds ||v||; on exit S_NRM holds the final norm.  The
 * second pass runs only if the first kept at most 1/sqrt(2) of the norm,
 * decided on the device. */
int cgs_dgks(const double *V, long ldv, int k, double *v, long n) {
  Ctx &c = ctx();
  double *w = (double *)ws(WS_SMALL, sizeof(double) * (size_t)(k + 1));
  if (!w) return PEVSL_ERR_NOMEM;
  int *run2 = c.dflag + F_PASS2;
  if (gemvT(n, k, V, ldv, v, w, nullptr)) return PEVSL_ERR_CUDA;
  if (gemv_sub_nrm(n, k, V, ldv, w, v, c.dscal + S_NRM, nullptr, run2, c.dscal + S_NRM0, kEta))
    return PEVSL_ERR_CUDA;
  if (gemvT(n, k, V, ldv, v, w, run2)) return PEVSL_ERR_CUDA;
  return gemv_sub_nrm(n, k, V, ldv, w, v, c.dscal + S_NRM, run2, nullptr, nullptr, kEta);
}

long round_ld(long n) { return (n + 31) / 32 * 32; }

}  // namespace

extern "C" {

/* Filter-kernel counters since the last reset: launches of the fused
 * Chebyshev degree kernel inside pEVSL_ChebLanNr, their algorithmic bytes,
 * and the device time of the filter applications that contain them (CUDA
 * events around each application, so launch gaps are included). */
void pEVSL_B200_FilterCounters(uint64_t *launches, double *bytes, double *ms) {
  if (launches) *launches = g_filter_launches;
  if (bytes) *bytes = g_filter_bytes;
  if (ms) *ms = g_filter_ms;
}

void pEVSL_B200_ResetFilterCounters(void) {
  g_filter_launches = 0;
  g_filter_persistent = 0;
  g_filter_bytes = 0.0;
  g_filter_ms = 0.0;
}

/* y = p(A) v (pEVSL_ChebAv, SRC/chebpol.c:509-574) on device or managed
 * vectors of length pevsl->n.  Extension entry point: the reference keeps
 * ChebAv internal. */
int pEVSL_B200_ChebAv(pevsl_Data *pevsl, pevsl_Polparams *pol, const double *v, double *y) {
  if (ensure()) return PEVSL_ERR_CUDA;
  matrix_window(pevsl_builtin_A(pevsl));
  const long n = pevsl->n;
  double *w3 = (double *)ws(WS_CHEB, sizeof(double) * 3 * (size_t)n);
  if (!w3) return PEVSL_ERR_NOMEM;
  int st = cheb_apply(pevsl, pol, v, y, w3, n);
  if (!st) st = sync();
  return st;
}

/* ================================================================ KPM DOS */

int pEVSL_Kpmdos(pevsl_Data *pevsl, int Mdeg, int damping, int nvec, double *intv, int ngroups,
                 int groupid, MPI_Comm gl_comm, double *mu, double *ecnt) {
  const double t0 = pevsl_now();
  if (ensure()) return PEVSL_ERR_CUDA;
  if (pevsl_check_intv(intv, stdout) < 0) return -1;
  const long n = pevsl->n;
  const double aa = PEVSL_MAX(intv[0], intv[2]), bb = PEVSL_MIN(intv[1], intv[3]);
  if (intv[0] < intv[2] || intv[1] > intv[3]) {
    fprintf(stdout, " warning: interval (%e, %e) is adjusted to (%e, %e)\n", intv[0], intv[1],
            aa, bb);
  }
  const double ctr = (intv[3] + intv[2]) / 2.0, wid = (intv[3] - intv[2]) / 2.0;
  const double beta1 = acos(PEVSL_MAX(-1.0 + DBL_EPSILON, (aa - ctr) / wid));
  const double beta2 = acos(PEVSL_MIN(1.0 - DBL_EPSILON, (bb - ctr) / wid));
  double *jac = (double *)malloc(sizeof(double) * (size_t)(Mdeg + 1));
  if (!jac) return PEVSL_ERR_NOMEM;
  pevsl_dampcf(Mdeg, damping, jac);
  jac[0] = 1.0;
  memset(mu, 0, sizeof(double) * (size_t)(Mdeg + 1));
  double tcnt = 0.0;
  int vec_start = 0, vec_end = nvec;
  if (ngroups > 1) pEVSL_Part1d(nvec, ngroups, &groupid, &vec_start, &vec_end, 1);
  /* counter-based Gaussian stream: a group starts at its first vector's
   * draw, so the groups' vectors are exactly one process's nvec vectors and
   * the summed moments equal the one-group moments (the C library stream is
   * per process, as the reference's per-rank srand) */
  if (ngroups > 1 && pevsl_rng_mode() == PEVSL_RNG_GAUSS && vec_start > 0)
    pevsl_rng_take((uint64_t)vec_start);
  pevsl_devcsr *A = pevsl_builtin_A(pevsl);
  int st = 0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, ctx().stream);
  const bool gen = pevsl->ifGenEv != 0;
  const bool mixed = !gen && A && pevsl_inst_of(pevsl)->precision == PEVSL_PREC_MIXED;
  if (mixed) st = csr_make_fp32(A);
  if (gen) {
    /* generalized problem: one vector at a time with B-solves */
    if (!st)
      st = pevsl_gen_kpm_moments(pevsl, Mdeg, jac, ctr, wid, beta1, beta2, vec_start, vec_end, mu,
                                 &tcnt);
  } else if (A && mixed && !st) {
    /* FP32 moments: blocks of up to 64 vectors drawn and normalised in FP64,
     * then rounded to FP32; FP32 recurrence and dots, one launch per degree */
    const int smax = 64;
    for (int m0 = vec_start; m0 < vec_end && !st; m0 += smax) {
      const int s = vec_end - m0 < smax ? vec_end - m0 : smax;
      const int ld = s;
      const size_t blk = (size_t)n * (size_t)ld;
      double *X = (double *)ws(WS_KPM, sizeof(double) * 4 * blk);
      double *mom = (double *)ws(WS_MOM, sizeof(double) * (size_t)(Mdeg + 1) * (size_t)s);
      double *nrm2 = (double *)ws(WS_SMALL, sizeof(double) * 64);
      double *hmom = (double *)malloc(sizeof(double) * (size_t)(Mdeg + 1) * (size_t)s);
      if (!X || !mom || !nrm2 || !hmom) {
        free(hmom);
        st = PEVSL_ERR_NOMEM;
        break;
      }
      double *V0d = X;
      float *V0 = (float *)(X + blk), *B[3] = {V0 + blk, V0 + 2 * blk, V0 + 3 * blk};
      st = pevsl_rand_block_dev(V0d, (int)n, s, ld);
      if (!st) st = block_colnorm2(n, s, ld, V0d, nrm2);
      if (!st) st = block_normalize(n, s, ld, V0d, nrm2);
      if (!st) st = cvt_f64_f32((long)blk, V0d, V0);
      for (int k = 0; k < Mdeg && !st; k++) {
        const double sc = (k == 0 ? 1.0 : 2.0) / wid;
        const float *Xk = k == 0 ? V0 : B[(k - 1) % 3];
        const float *Xkm1 = k == 0 ? nullptr : (k == 1 ? V0 : B[(k - 2) % 3]);
        st = kpm_step32(A, s, ld, Xk, Xkm1, B[k % 3], V0, ctr, sc, mom + (size_t)k * s);
      }
      if (!st) st = memcpy_async(hmom, mom, sizeof(double) * (size_t)Mdeg * (size_t)s);
      if (!st) st = sync();
      pevsl->stats->n_mvA += (size_t)Mdeg * (size_t)s;
      for (int c = 0; c < s && !st; c++) {
        mu[0] += jac[0];
        tcnt -= jac[0] * (beta2 - beta1);
        for (int k = 0; k < Mdeg; k++) {
          const int k1 = k + 1;
          const double t = hmom[(size_t)k * s + c] * 2.0 * jac[k1];
          mu[k1] += t;
          tcnt -= t * (sin(k1 * beta2) - sin(k1 * beta1)) / k1;
        }
      }
      free(hmom);
    }
  } else if (A && !st) {
    /* blocks of up to 64 vectors, row-interleaved; one launch per degree */
    const int smax = 64;
    for (int m0 = vec_start; m0 < vec_end && !st; m0 += smax) {
      const int s = vec_end - m0 < smax ? vec_end - m0 : smax;
      const int ld = s;
      const size_t blk = (size_t)n * (size_t)ld;
      double *X = (double *)ws(WS_KPM, sizeof(double) * 4 * blk);
      double *mom = (double *)ws(WS_MOM, sizeof(double) * (size_t)(Mdeg + 1) * (size_t)s);
      double *nrm2 = (double *)ws(WS_SMALL, sizeof(double) * 64);
      double *hmom = (double *)malloc(sizeof(double) * (size_t)(Mdeg + 1) * (size_t)s);
      if (!X || !mom || !nrm2 || !hmom) {
        free(hmom);
        st = PEVSL_ERR_NOMEM;
        break;
      }
      double *V0 = X, *B[3] = {X + blk, X + 2 * blk, X + 3 * blk};
      st = pevsl_rand_block_dev(V0, (int)n, s, ld);
      if (!st) st = block_colnorm2(n, s, ld, V0, nrm2);
      if (!st) st = block_normalize(n, s, ld, V0, nrm2);
      for (int k = 0; k < Mdeg && !st; k++) {
        const double sc = (k == 0 ? 1.0 : 2.0) / wid;
        const double *Xk = k == 0 ? V0 : B[(k - 1) % 3];
        const double *Xkm1 = k == 0 ? nullptr : (k == 1 ? V0 : B[(k - 2) % 3]);
        st = kpm_step(A, s, ld, Xk, Xkm1, B[k % 3], V0, ctr, sc, mom + (size_t)k * s);
      }
      if (!st) st = memcpy_async(hmom, mom, sizeof(double) * (size_t)Mdeg * (size_t)s);
      if (!st) st = sync();
      pevsl->stats->n_mvA += (size_t)Mdeg * (size_t)s;
      /* accumulate exactly as the reference: vector by vector, degree by degree */
      for (int c = 0; c < s && !st; c++) {
        mu[0] += jac[0];
        tcnt -= jac[0] * (beta2 - beta1);
        for (int k = 0; k < Mdeg; k++) {
          const int k1 = k + 1;
          const double t = hmom[(size_t)k * s + c] * 2.0 * jac[k1];
          mu[k1] += t;
          tcnt -= t * (sin(k1 * beta2) - sin(k1 * beta1)) / k1;
        }
      }
      free(hmom);
    }
  } else if (!st) {
    /* user matvec: one vector at a time, as the reference */
    double *buf = (double *)ws(WS_KPM, sizeof(double) * 4 * (size_t)n);
    double *hdot = (double *)malloc(sizeof(double) * (size_t)(Mdeg + 1));
    double *ddot_ = (double *)ws(WS_MOM, sizeof(double) * (size_t)(Mdeg + 1));
    if (!buf || !hdot || !ddot_) st = PEVSL_ERR_NOMEM;
    for (int m = vec_start; m < vec_end && !st; m++) {
      double *v = buf, *vkm1 = buf + n, *vk = buf + 2 * n, *vkp1 = buf + 3 * n, *tmp;
      st = pevsl_rand_vector_dev(v, (int)n);
      if (!st) st = vnrm2(n, v, ctx().dscal + S_TMP0);
      const double *h = st ? nullptr : fetch_scalars(S_TMP0, 1);
      if (!h) {
        st = st ? st : PEVSL_ERR_CUDA;
        break;
      }
      const double tn = h[0];
      if (!st) st = vscal(v, n, 1.0 / tn);
      if (!st) st = vcopy(v, vk, n);
      if (!st) st = vfill(vkm1, n, 0.0);
      for (int k = 0; k < Mdeg && !st; k++) {
        const double sc = (k == 0 ? 1.0 : 2.0) / wid;
        st = apply_A(pevsl, vk, vkp1);
        if (!st) st = vaxpy(n, -ctr, vk, vkp1);
        if (!st) st = vscal(vkp1, n, sc);
        if (!st) st = vaxpy(n, -1.0, vkm1, vkp1);
        tmp = vkm1;
        vkm1 = vk;
        vk = vkp1;
        vkp1 = tmp;
        if (!st) st = vdot(n, vk, v, ddot_ + k);
      }
      if (!st) st = memcpy_async(hdot, ddot_, sizeof(double) * (size_t)Mdeg);
      if (!st) st = sync();
      if (st) break;
      mu[0] += jac[0];
      tcnt -= jac[0] * (beta2 - beta1);
      for (int k = 0; k < Mdeg; k++) {
        const int k1 = k + 1;
        const double t = hdot[k] * 2.0 * jac[k1];
        mu[k1] += t;
        tcnt -= t * (sin(k1 * beta2) - sin(k1 * beta1)) / k1;
      }
    }
    free(hdot);
  }
  cudaEventRecord(e1, ctx().stream);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  pevsl_inst_of(pevsl)->phase_ms[1] = ms;
  free(jac);
  if (st) return st;
  if (ngroups > 1) {
    /* the groups' partial sums (SRC/kpmdos.c:160-176): through the
     * instance's reduction (one process per GPU) when one is installed,
     * else MPI on gl_comm */
    pevsl_inst *inst = pevsl_inst_of(pevsl);
    double *mu_g = (double *)malloc(sizeof(double) * (size_t)(Mdeg + 2));
    if (!mu_g) return PEVSL_ERR_NOMEM;
    if (inst->group_reduce) {
      memcpy(mu_g, mu, sizeof(double) * (size_t)(Mdeg + 1));
      mu_g[Mdeg + 1] = tcnt;
      inst->group_reduce(mu_g, Mdeg + 2, inst->group_reduce_ctx);
      memcpy(mu, mu_g, sizeof(double) * (size_t)(Mdeg + 1));
      tcnt = mu_g[Mdeg + 1];
    } else {
      double tcnt_g = 0.0;
      MPI_Allreduce(mu, mu_g, Mdeg + 1, MPI_DOUBLE, MPI_SUM, gl_comm);
      MPI_Allreduce(&tcnt, &tcnt_g, 1, MPI_DOUBLE, MPI_SUM, gl_comm);
      memcpy(mu, mu_g, sizeof(double) * (size_t)(Mdeg + 1));
      tcnt = tcnt_g;
    }
    free(mu_g);
  }
  const double t = 1.0 / (((double)nvec) * M_PI);
  for (int k = 0; k <= Mdeg; k++) mu[k] *= t;
  tcnt *= t * ((double)pevsl->N);
  *ecnt = tcnt;
  pevsl->stats->t_dos = pevsl_now() - t0;
  return 0;
}

/* ================================================================ Lanczos DOS */

/* one Lanczos run of pEVSL_LanDosG (SRC/landos.c:134-262): v_0 = vinit
 * normalised, maxit steps with full reorthogonalisation; the tridiagonal
 * matrix into dT, eT */
static int landos_lanczos(pevsl_Data *pevsl, int maxit, double *V, long ld, const double *vinit,
                          long n, double *dT, double *eT) {
  Ctx &c = ctx();
  int st = vnrm2(n, vinit, c.dscal + S_TMP0);
  const double *h = st ? nullptr : fetch_scalars(S_TMP0, 1);
  if (!h) return st ? st : PEVSL_ERR_CUDA;
  const double tinv = 1.0 / h[0];
  if (!st) st = vcopy(vinit, V, n);
  if (!st) st = vscal(V, n, tinv);
  double wn = 0.0, beta = 0.0;
  int nwn = 0;
  for (int k = 0; k < maxit && !st; k++) {
    double *v = V + (size_t)k * ld, *vnew = V + (size_t)(k + 1) * ld;
    st = apply_A(pevsl, v, vnew);
    if (!st && k > 0) st = vaxpy(n, -beta, V + (size_t)(k - 1) * ld, vnew);
    if (!st) st = vdot(n, v, vnew, c.dscal + S_ALPHA);
    if (!st) st = vaxpy_dev_nrm2(n, c.dscal + S_ALPHA, v, vnew, c.dscal + S_NRM0);
    if (!st) st = cgs_dgks(V, ld, k + 1, vnew, n);
    if (!st) st = memcpy_async(c.hscal + S_ALPHA, c.dscal + S_ALPHA, sizeof(double) * 4);
    if (!st) st = sync();
    if (st) break;
    const double alpha = c.hscal[S_ALPHA];
    beta = c.hscal[S_NRM];
    dT[k] = alpha;
    wn += fabs(alpha) + 2.0 * beta;
    nwn += 3;
    if (beta * nwn < orthTol * wn) {
      st = pevsl_rand_vector_dev(vnew, (int)n);
      if (!st) st = vnrm2(n, vnew, c.dscal + S_NRM0);
      if (!st) st = cgs_dgks(V, ld, k + 1, vnew, n);
      const double *hb = st ? nullptr : fetch_scalars(S_NRM, 1);
      if (!hb) return st ? st : PEVSL_ERR_CUDA;
      st = vscal(vnew, n, 1.0 / hb[0]);
      beta = 0.0;
    } else {
      st = vscal(vnew, n, 1.0 / beta);
    }
    eT[k] = beta;
  }
  return st;
}

int pEVSL_LanDosG(pevsl_Data *pevsl, const int nvec, int msteps, int npts, double *xdos,
                  double *ydos, double *neig, double *intv, int ngroups, int groupid,
                  MPI_Comm gl_comm) {
  if (ensure()) return PEVSL_ERR_CUDA;
  const double t0 = pevsl_now();
  const long n = pevsl->n, ld = round_ld(n);
  const int maxit = msteps < pevsl->N ? msteps : pevsl->N;
  double *V = (double *)ws(WS_BASIS, sizeof(double) * (size_t)ld * (size_t)(maxit + 1));
  double *vinit = (double *)ws(WS_VEC, sizeof(double) * (size_t)n);
  double *y = (double *)calloc((size_t)npts, sizeof(double));
  int *ind = (int *)malloc(sizeof(int) * (size_t)npts);
  double *dT = (double *)malloc(sizeof(double) * (size_t)maxit);
  double *eT = (double *)malloc(sizeof(double) * (size_t)maxit);
  double *EvalT = (double *)malloc(sizeof(double) * (size_t)maxit);
  double *EvecT = (double *)malloc(sizeof(double) * (size_t)maxit * (size_t)maxit);
  int st = (!V || !vinit || !y || !ind || !dT || !eT || !EvalT || !EvecT) ? PEVSL_ERR_NOMEM : 0;
  const double lm = intv[2], lM = intv[3];
  const double aa = PEVSL_MAX(intv[0], intv[2]), bb = PEVSL_MIN(intv[1], intv[3]);
  const int M = PEVSL_MIN(msteps, 30);
  const double H = (lM - lm) / (M - 1);
  const double sigma = H / sqrt(8 * log(1.25)) * pevsl->sigma_mult;
  const double sigma2 = 2 * sigma * sigma;
  const double width = sigma * sqrt(-2.0 * log(1e-08));
  if (!st) linspace(aa, bb, npts, xdos);
  int vec_start = 0, vec_end = nvec;
  if (ngroups > 1) pEVSL_Part1d(nvec, ngroups, &groupid, &vec_start, &vec_end, 1);
  for (int m = vec_start; m < vec_end && !st; m++) {
    st = pevsl_rand_vector_dev(vinit, (int)n);
    if (!st) st = pevsl->ifGenEv ? pevsl_gen_landos_lanczos(pevsl, maxit, vinit, dT, eT)
                                 : landos_lanczos(pevsl, maxit, V, ld, vinit, n, dT, eT);
    if (st) break;
    if (pevsl_tridiag_eig(maxit, dT, eT, EvalT, EvecT)) {
      st = PEVSL_ERR_EIG;
      break;
    }
    for (int i = 0; i < maxit; i++) {
      const double g2 = EvecT[(size_t)i * maxit] * EvecT[(size_t)i * maxit];
      const double th = EvalT[i];
      int np = 0;
      for (int j = 0; j < npts; j++)
        if (fabs(xdos[j] - th) < width) ind[np++] = j;
      for (int j = 0; j < np; j++)
        y[ind[j]] += g2 * exp(-((xdos[ind[j]] - th) * (xdos[ind[j]] - th)) / sigma2);
    }
  }
  if (!st && ngroups > 1) {
    double *yg = (double *)malloc(sizeof(double) * (size_t)npts);
    MPI_Allreduce(y, yg, npts, MPI_DOUBLE, MPI_SUM, gl_comm);
    memcpy(y, yg, sizeof(double) * (size_t)npts);
    free(yg);
  }
  if (!st) {
    const double scaling = 1.0 / (nvec * sqrt(sigma2 * M_PI));
    for (int j = 0; j < npts; j++) y[j] *= scaling;
    memcpy(ydos, y, sizeof(double) * (size_t)npts);
    pevsl_simpson(xdos, y, npts);
    *neig = y[npts - 1] * pevsl->N;
  }
  free(y);
  free(ind);
  free(dT);
  free(eT);
  free(EvalT);
  free(EvecT);
  pevsl->stats->t_dos = pevsl_now() - t0;
  return st;
}

/* ================================================================ bounds */

int pEVSL_LanTrbounds(pevsl_Data *pevsl, int lanm, int maxit, double tol, pevsl_Parvec *vinit,
                      int bndtype, double *lammin, double *lammax, FILE *fstats) {
  if (ensure()) return PEVSL_ERR_CUDA;
  const double t0 = pevsl_now();
  if (pevsl->ifGenEv) {
    const int st = pevsl_gen_lantrbounds(pevsl, lanm, maxit, tol, vinit, bndtype, lammin, lammax,
                                         fstats);
    pevsl->stats->t_eigbounds += pevsl_now() - t0;
    pevsl_inst_of(pevsl)->phase_ms[0] = 1e3 * (pevsl_now() - t0);
    return st;
  }
  const int N = pevsl->N;
  const long n = pevsl->n, ld = round_ld(n);
  lanm = PEVSL_MIN(lanm, N);
  const int lanm1 = lanm + 1;
  if (lanm == N) maxit = PEVSL_MIN(maxit, N);
  const size_t L = (size_t)lanm1;
  double *V = (double *)ws(WS_BASIS, sizeof(double) * (size_t)ld * L);
  double *R2 = (double *)ws(WS_RITZ, sizeof(double) * (size_t)ld * 2);
  double *dY = (double *)ws(WS_RITZ2, sizeof(double) * L * 2 + sizeof(double) * L);
  double *T = (double *)calloc(L * L, sizeof(double));
  double *EvecT = (double *)calloc(L * L, sizeof(double));
  double *Rval = (double *)calloc(L, sizeof(double));
  double *hY = (double *)malloc(sizeof(double) * L * 2);
  if (!V || !R2 || !dY || !T || !EvecT || !Rval || !hY) {
    free(T);
    free(EvecT);
    free(Rval);
    free(hY);
    return PEVSL_ERR_NOMEM;
  }
  double *dS = dY + 2 * L; /* coefficients s of the restart step */
  Ctx &c = ctx();
  int st = 0, it = 0, trlen = 0;
  double lmin = 0.0, lmax = 0.0, s[3] = {0, 0, 0};
  if (fstats) fprintf(fstats, " LanTR for bounds: dim %d, maxits %d\n", lanm, maxit);
  st = vcopy(vinit->data, V, n);
  if (!st) st = vnrm2(n, V, c.dscal + S_TMP0);
  const double *h0 = st ? nullptr : fetch_scalars(S_TMP0, 1);
  if (!h0) st = st ? st : PEVSL_ERR_CUDA;
  if (!st) st = vscal(V, n, 1.0 / h0[0]);
#define VC(j) (V + (size_t)(j) * ld)
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
      /* thick-restart step: arrowhead column of T (SRC/lantrbnd.c:150-223) */
      const int k1 = k - 1;
      double *v = VC(k1), *vnew = VC(k1 + 1);
      st = apply_A(pevsl, v, vnew);
      for (int i = 0; i < trlen; i++) {
        T[i * L + i] = Rval[i];
        wn += fabs(Rval[i]);
      }
      if (!st) st = vdot(n, v, vnew, c.dscal + S_TMP0);
      const double *hs = st ? nullptr : fetch_scalars(S_TMP0, 1);
      if (!hs) {
        st = st ? st : PEVSL_ERR_CUDA;
        break;
      }
      s[k1] = hs[0];
      if (!st) st = memcpy_async(dS, s, sizeof(double) * (size_t)k);
      if (!st) st = gemv_sub_nrm(n, k, V, ld, dS, vnew, c.dscal + S_NRM, nullptr, nullptr, nullptr,
                                 kEta);
      for (int i = 0; i < k1; i++) {
        T[trlen * L + i] = s[i];
        T[i * L + trlen] = s[i];
        wn += 2.0 * fabs(s[i]);
      }
      T[trlen * L + trlen] = s[k1];
      wn += fabs(s[k1]);
      const double *hb = st ? nullptr : fetch_scalars(S_NRM, 1);
      if (!hb) {
        st = st ? st : PEVSL_ERR_CUDA;
        break;
      }
      beta = hb[0];
      wn += 2.0 * beta;
      nwn += 3 * k;
      if (beta * nwn < orthTol * wn) {
        st = pevsl_rand_vector_dev(vnew, (int)n);
        if (!st) st = vnrm2(n, vnew, c.dscal + S_NRM0);
        if (!st) st = cgs_dgks(V, ld, k, vnew, n);
        const double *hb2 = st ? nullptr : fetch_scalars(S_NRM, 1);
        if (!hb2) {
          st = st ? st : PEVSL_ERR_CUDA;
          break;
        }
        st = vscal(vnew, n, 1.0 / hb2[0]);
        beta = 0.0;
      } else {
        st = vscal(vnew, n, 1.0 / beta);
      }
      T[k1 * L + k] = beta;
      T[k * L + k1] = beta;
    }
    const double *zold = k > 0 ? VC(k - 1) : nullptr;
    while (k < lanm && it < maxit && !st) {
      k++;
      double *v = VC(k - 1), *vnew = VC(k);
      st = apply_A(pevsl, v, vnew);
      it++;
      if (!st && zold) st = vaxpy(n, -beta, zold, vnew);
      if (!st) st = vdot(n, v, vnew, c.dscal + S_ALPHA);
      if (!st) st = vaxpy_dev_nrm2(n, c.dscal + S_ALPHA, v, vnew, c.dscal + S_NRM0);
      if (!st) st = cgs_dgks(V, ld, k, vnew, n);
      if (!st) st = memcpy_async(c.hscal + S_ALPHA, c.dscal + S_ALPHA, sizeof(double) * 4);
      if (!st) st = sync();
      if (st) break;
      const double alpha = c.hscal[S_ALPHA];
      beta = c.hscal[S_NRM];
      T[(k - 1) * L + (k - 1)] = alpha;
      wn += fabs(alpha) + 2.0 * beta;
      nwn += 3;
      zold = v;
      if (beta * nwn < orthTol * wn) {
        if (fstats) fprintf(fstats, "it %4d: Lucky breakdown, beta = %.15e\n", it, beta);
        st = pevsl_rand_vector_dev(vnew, (int)n);
        if (!st) st = vnrm2(n, vnew, c.dscal + S_NRM0);
        if (!st) st = cgs_dgks(V, ld, k, vnew, n);
        const double *hb = st ? nullptr : fetch_scalars(S_NRM, 1);
        if (!hb) {
          st = st ? st : PEVSL_ERR_CUDA;
          break;
        }
        st = vscal(vnew, n, 1.0 / hb[0]);
        beta = 0.0;
      } else {
        st = vscal(vnew, n, 1.0 / beta);
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
    /* the two extreme Ritz vectors become V(:,0:2) */
    memcpy(hY, EvecT, sizeof(double) * (size_t)k);
    memcpy(hY + k, EvecT + (size_t)(k - 1) * L, sizeof(double) * (size_t)k);
    st = memcpy_async(dY, hY, sizeof(double) * 2 * (size_t)k);
    if (!st) st = gemm_nn(n, k, 2, V, ld, dY, k, R2, ld);
    if (!st) st = vcopy(R2, VC(0), n);
    if (!st) st = vcopy(R2 + ld, VC(1), n);
    trlen = 2;
    Rval[1] = Rval[k - 1];
    if (fstats)
      fprintf(fstats, "it %4d, k %3d: ritz %.15e %.15e, t1,t2 %e %e, res %.15e %.15e\n", it, k,
              Rval[0], Rval[1], t1, t2, fabs(s[0]), fabs(s[1]));
    if (t1 + t2 < tol * (fabs(lmin) + fabs(lmax))) break;
    memset(T, 0, sizeof(double) * L * L);
    if (!st) st = vcopy(VC(k), VC(trlen), n);
  }
#undef VC
  if (!st) st = sync();
  *lammin = lmin;
  *lammax = lmax;
  free(T);
  free(EvecT);
  free(Rval);
  free(hY);
  pevsl->stats->t_eigbounds += pevsl_now() - t0;
  pevsl_inst_of(pevsl)->phase_ms[0] = 1e3 * (pevsl_now() - t0);
  return st;
}

/* ================================================================ filtered Lanczos
 * pEVSL_ChebLanNr (SRC/cheblanNr.c:54-448) for a batch of slices that
 * advance in lockstep: at every Lanczos step one fused filter kernel per
 * degree serves all slices (the matrix is read once per degree), the
 * Gram-Schmidt kernels run batched, and one host read fetches every slice's
 * alpha and beta.  Each slice keeps its own basis, tridiagonal matrix,
 * convergence test and stop; a single slice is a batch of one and follows
 * exactly the reference's sequence of operations. */

struct SliceState {
  /* inputs: the slice and the problem it belongs to */
  double intv[4];
  const pevsl_Polparams *pol;
  int maxit;
  pevsl_Data *pevsl;
  pevsl_devcsr *A; /* built-in device CSR, or NULL for a user matvec */
  pevsl_Parvec *vinit;
  long n, ld;
  /* state */
  double *V;      /* basis, ld x (maxit+1) */
  double *dT, *eT, *EvalT;
  double wn, tr0, beta;
  int nwn, kdim, count, nconv;
  int active, done;
  /* outputs */
  int status, nev, its;
  int short_pairs; /* mixed form: refined pairs in [a, b] above tol */
  double *Lam, *res;
  pevsl_Parvecs *Rvec;
};

/* Host threads for the per-slice host work of a lockstep group (the
 * tridiagonal eigenproblems of the convergence tests and the Ritz
 * extraction): PEVSL_B200_HOST_THREADS caps them (1: the calling thread
 * only; default: every hardware thread). */
static unsigned host_threads() {
  static unsigned v = 0;
  if (!v) {
    const char *e = getenv("PEVSL_B200_HOST_THREADS");
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int r = e ? atoi(e) : 0;
    v = r >= 1 ? std::min((unsigned)r, hw) : hw;
  }
  return v;
}

/* f(0), ..., f(m-1) on up to host_threads() threads, this one included,
 * when worth is set; else in order on this thread.  f must be host-only
 * code (no CUDA call) that writes nothing another index reads. */
extern "C++" {
template <class F>
static void host_parallel(size_t m, bool worth, F f) {
  const size_t nt = std::min<size_t>(m, host_threads());
  if (!worth || nt <= 1) {
    for (size_t i = 0; i < m; i++) f(i);
    return;
  }
  std::atomic<size_t> next{0};
  auto work = [&]() {
    for (size_t i = next.fetch_add(1); i < m; i = next.fetch_add(1)) f(i);
  };
  std::vector<std::thread> th;
  for (size_t t = 1; t < nt; t++) {
    try {
      th.emplace_back(work);
    } catch (...) {
      break; /* no more threads: this one does the rest */
    }
  }
  work();
  for (auto &x : th) x.join();
}
}  // extern "C++"

/* The host part of a slice's Ritz extraction: the eigenvalues of T again
 * and the eigenvectors of those >= bar.  Host arithmetic only, so the
 * slices of a group run it on host threads (host_parallel). */
struct RitzHost {
  int early = 0;  /* error that ends the extraction before any output */
  int sel_st = 0; /* the eigenvector step failed */
  int nsel = 0;
  int *sel = nullptr;
  double *Y = nullptr;
  double secs = 0.0;
};

static void ritz_host(SliceState *S, RitzHost *R) {
  const int kdim = S->kdim, count = S->count;
  const double bar = S->pol->bar;
  const double te = pevsl_now();
  /* eigenvalues again: the last convergence test may predate the last step
   * (a maxit exit), so more Ritz values than nconv may pass the bar test;
   * the outputs hold max(nconv, nsel) pairs */
  if (kdim > 0 && pevsl_tridiag_eig(kdim, S->dT, S->eT, S->EvalT, nullptr)) {
    R->early = PEVSL_ERR_EIG;
    return;
  }
  R->sel = (int *)malloc(sizeof(int) * (size_t)(kdim > 0 ? kdim : 1));
  if (!R->sel) {
    R->early = PEVSL_ERR_NOMEM;
    return;
  }
  for (int i = 0; i < count && kdim > 0; i++)
    if (S->EvalT[i] >= bar) R->sel[R->nsel++] = i;
  if (kdim > 0 && R->nsel > 0) {
    R->Y = (double *)malloc(sizeof(double) * (size_t)kdim * (size_t)R->nsel);
    if (!R->Y || pevsl_tridiag_eig_sel(kdim, S->dT, S->eT, S->EvalT, R->nsel, R->sel, R->Y))
      R->sel_st = PEVSL_ERR_EIG;
  }
  R->secs = pevsl_now() - te;
}

/* Ritz pairs of one finished slice (SRC/cheblanNr.c:339-413): eigenvectors
 * of T only for Ritz values >= bar (ritz_host, run before), U = V Y,
 * normalise, W = A U, Rayleigh quotients, interval check, residuals,
 * acceptance below tol.  Takes over R's buffers. */
static int ritz_extract(pevsl_Data *pevsl, SliceState *S, RitzHost *R, pevsl_Parvec *vinit,
                        long n, long ld, double tol) {
  Ctx &c = ctx();
  const int kdim = S->kdim;
  const double aa = S->intv[0], bb = S->intv[1];
  S->nev = 0;
  if (R->early) {
    free(R->sel);
    free(R->Y);
    R->sel = nullptr;
    R->Y = nullptr;
    return R->early;
  }
  int st = 0;
  const int nsel = R->nsel;
  int *sel = R->sel;
  double *Y = R->Y;
  R->sel = nullptr;
  R->Y = nullptr;
  const double te = pevsl_now();
  const int nout = PEVSL_MAX(S->nconv, nsel);
  S->Lam = (double *)malloc(sizeof(double) * (size_t)(nout > 0 ? nout : 1));
  S->res = (double *)malloc(sizeof(double) * (size_t)(nout > 0 ? nout : 1));
  S->Rvec = (pevsl_Parvecs *)calloc(1, sizeof(pevsl_Parvecs));
  if (!S->Lam || !S->res || !S->Rvec) {
    free(sel);
    free(Y);
    return PEVSL_ERR_NOMEM;
  }
  pEVSL_ParvecsDuplParvec(vinit, nout, (int)n, S->Rvec);
  if (nout > 0 && !S->Rvec->data) {
    free(sel);
    free(Y);
    return PEVSL_ERR_NOMEM;
  }
  if (kdim <= 0) {
    free(sel);
    free(Y);
    return 0;
  }
  st = R->sel_st;
  pevsl->stats->t_eig += R->secs + (pevsl_now() - te);
  if (!st && nsel > 0) {
    double *U = (double *)ws(WS_RITZ, sizeof(double) * (size_t)ld * (size_t)nsel);
    double *W = (double *)ws(WS_RITZ2, sizeof(double) * (size_t)ld * (size_t)nsel);
    double *dY = (double *)ws(WS_PART, sizeof(double) * (size_t)kdim * (size_t)nsel);
    double *dv = (double *)ws(WS_MOM, sizeof(double) * 3 * (size_t)nsel);
    double *hv = (double *)malloc(sizeof(double) * 3 * (size_t)nsel);
    if (!U || !W || !dY || !dv || !hv) st = PEVSL_ERR_NOMEM;
    if (!st) st = memcpy_async(dY, Y, sizeof(double) * (size_t)kdim * (size_t)nsel);
    if (!st) st = gemm_nn(n, kdim, nsel, S->V, ld, dY, kdim, U, ld);
    if (!st) st = vdot_cols(n, nsel, U, ld, U, ld, dv);
    if (!st) st = memcpy_async(hv, dv, sizeof(double) * (size_t)nsel);
    if (!st) st = sync();
    for (int j = 0; j < nsel && !st; j++) {
      const double t = sqrt(hv[j]);
      if (t == 0.0) {
        st = 2; /* zero eigenvector (SRC/cheblanNr.c:377-379) */
        break;
      }
      hv[nsel + j] = 1.0 / t;
    }
    if (!st) st = memcpy_async(dv + nsel, hv + nsel, sizeof(double) * (size_t)nsel);
    if (!st) st = vscal_cols(n, nsel, U, ld, dv + nsel);
    for (int j = 0; j < nsel && !st; j++) st = apply_A(pevsl, U + (size_t)j * ld, W + (size_t)j * ld);
    if (!st) st = vdot_cols(n, nsel, W, ld, U, ld, dv);
    if (!st) st = vaxpy_cols(n, nsel, dv, U, ld, W, ld);
    if (!st) st = vdot_cols(n, nsel, W, ld, W, ld, dv + 2 * nsel);
    if (!st) st = memcpy_async(hv, dv, sizeof(double) * 3 * (size_t)nsel);
    if (!st) st = sync();
    for (int j = 0; j < nsel && !st; j++) {
      const double lam = hv[j];
      if (lam < aa - DBL_EPSILON || lam > bb + DBL_EPSILON) continue;
      const double r0 = sqrt(hv[2 * nsel + j]);
      if (r0 < tol) {
        S->Lam[S->nev] = lam;
        S->res[S->nev] = r0;
        st = vcopy(U + (size_t)j * ld, S->Rvec->data + (size_t)S->nev * S->Rvec->ld, n);
        S->nev++;
      }
    }
    free(hv);
  }
  free(Y);
  free(sel);
  if (!st) st = sync();
  return st;
}

/* Ritz pairs of a slice whose Krylov basis came from the FP32 filter: one
 * FP64 filtered Rayleigh-Ritz sweep.  The FP32 recurrence leaves noise of
 * about 1e-6 relative in every direction of the basis, which Rayleigh-Ritz
 * on the basis alone cannot remove; one FP64 application of p(A) damps each
 * direction by p(lam_out)/p(lam_in), which is small except just outside the
 * slice, so those near-edge directions are taken into the subspace instead:
 * U = V Y for the Ritz values of p(A) >= guard * bar (guard < 1; the
 * reference keeps those >= bar, SRC/cheblanNr.c:350-365), P = p(A) U in
 * FP64 with unit columns, G = P'P, H = P'AP (gemm_tn), the pencil (H, G)
 * on the host (Cholesky dropping dependent columns), X = P Z, and the
 * reference's acceptance on the refined pairs (SRC/cheblanNr.c:366-405):
 * lam in [a, b] and ||A x - lam x|| < tol. */
static int ritz_refine(pevsl_Data *pevsl, SliceState *S, pevsl_Parvec *vinit, long n, long ld,
                       double tol, double guard, int passes) {
  pevsl_devcsr *A = pevsl_builtin_A(pevsl);
  const int kdim = S->kdim, count = S->count;
  const double bar = S->pol->bar, aa = S->intv[0], bb = S->intv[1];
  S->nev = 0;
  int m = 0, st = 0;
  int *sel = (int *)malloc(sizeof(int) * (size_t)(kdim > 0 ? kdim : 1));
  if (!sel) return PEVSL_ERR_NOMEM;
  if (kdim > 0 && pevsl_tridiag_eig(kdim, S->dT, S->eT, S->EvalT, nullptr)) st = PEVSL_ERR_EIG;
  int nbar = 0; /* Ritz values of p(A) above bar: the FP64 path's candidates */
  for (int i = 0; i < count && kdim > 0 && !st; i++) {
    if (S->EvalT[i] >= guard * bar) sel[m++] = i;
    if (S->EvalT[i] >= bar) nbar++;
  }
  S->short_pairs = nbar;
  S->Lam = (double *)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
  S->res = (double *)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
  S->Rvec = (pevsl_Parvecs *)calloc(1, sizeof(pevsl_Parvecs));
  if (!S->Lam || !S->res || !S->Rvec) st = PEVSL_ERR_NOMEM;
  if (st || m == 0) {
    if (S->Rvec) pEVSL_ParvecsDuplParvec(vinit, 0, (int)n, S->Rvec);
    free(sel);
    return st;
  }
  const size_t mm = (size_t)m * m;
  double *Y = (double *)malloc(sizeof(double) * (size_t)kdim * m);
  double *Hh = (double *)malloc(sizeof(double) * 2 * mm);
  double *Zh = (double *)malloc(sizeof(double) * mm);
  double *lam = (double *)malloc(sizeof(double) * (size_t)m);
  double *hv = (double *)malloc(sizeof(double) * (size_t)m);
  double *U = (double *)ws(WS_RITZ, sizeof(double) * (size_t)ld * m);
  double *P = (double *)ws(WS_RITZ2, sizeof(double) * (size_t)ld * m);
  double *W = (double *)ws(WS_REF1, sizeof(double) * (size_t)ld * m);
  double *X = (double *)ws(WS_REF2, sizeof(double) * (size_t)ld * m);
  void *fwork = ws(WS_FILT, 16 * (size_t)ld * kMaxBatch);
  double *dmu = (double *)ws(WS_MU, sizeof(double) * (size_t)(S->pol->deg + 1));
  if (dmu && memcpy_async(dmu, S->pol->mu, sizeof(double) * (size_t)(S->pol->deg + 1))) dmu = nullptr;
  /* small device matrices: Y | G | H | Z | 3 m scalars */
  double *dsm = (double *)ws(WS_H, sizeof(double) * ((size_t)kdim * m + 3 * mm + 3 * (size_t)m));
  if (!Y || !Hh || !Zh || !lam || !hv || !U || !P || !W || !X || !fwork || !dsm || !dmu)
    st = PEVSL_ERR_NOMEM;
  double *dY = dsm, *dG = dY + (size_t)kdim * m, *dH = dG + mm, *dZ = dH + mm, *dv = dZ + mm;
  if (!st && pevsl_tridiag_eig_sel(kdim, S->dT, S->eT, S->EvalT, m, sel, Y)) st = PEVSL_ERR_EIG;
  /* largest Ritz values first: the Cholesky of G then keeps the wanted
   * directions and drops guard columns that became dependent on them */
  for (int j = 0; j < m / 2 && !st; j++) {
    double *c1 = Y + (size_t)j * kdim, *c2 = Y + (size_t)(m - 1 - j) * kdim;
    for (int i = 0; i < kdim; i++) {
      const double t = c1[i];
      c1[i] = c2[i];
      c2[i] = t;
    }
  }
  /* U = V Y; P = p(A) U in FP64, unit columns */
  if (!st) st = memcpy_async(dY, Y, sizeof(double) * (size_t)kdim * m);
  if (!st) st = gemm_nn(n, kdim, m, S->V, ld, dY, kdim, U, ld);
  for (int pass = 0; pass < passes && !st; pass++) {
    double *src = pass % 2 == 0 ? U : P, *dst = pass % 2 == 0 ? P : U;
    for (int c0 = 0; c0 < m && !st; c0 += kMaxBatch) {
      const int cs = PEVSL_MIN(kMaxBatch, m - c0);
      FilterJob jobs[kMaxBatch];
      for (int e = 0; e < cs; e++)
        jobs[e] = FilterJob{pevsl, A, src + (size_t)(c0 + e) * ld, dst + (size_t)(c0 + e) * ld,
                            S->pol, dmu, (char *)fwork + 16 * (size_t)ld * e, ld};
      st = cheb_filter_batch(cs, jobs, false);
    }
    if (!st) st = vdot_cols(n, m, dst, ld, dst, ld, dv);
    if (!st) st = memcpy_async(hv, dv, sizeof(double) * m);
    if (!st) st = sync();
    for (int j = 0; j < m && !st; j++) hv[j] = hv[j] > 0 ? 1.0 / sqrt(hv[j]) : 0.0;
    if (!st) st = memcpy_async(dv, hv, sizeof(double) * m);
    if (!st) st = vscal_cols(n, m, dst, ld, dv);
  }
  if (!st && passes % 2 == 0) st = vcopy(U, P, (long)ld * m); /* filtered block in P */
  /* W = A P; G = P'P, H = P'W */
  for (int j = 0; j < m && !st; j++) st = spmv(A, P + (size_t)j * ld, W + (size_t)j * ld);
  pevsl->stats->n_mvA += (size_t)m;
  if (!st) st = gemm_tn(n, m, m, P, ld, P, ld, dG, m);
  if (!st) st = gemm_tn(n, m, m, P, ld, W, ld, dH, m);
  if (!st) st = memcpy_async(Hh, dG, sizeof(double) * 2 * mm);
  if (!st) st = sync();
  int q = 0;
  if (!st) {
    double *G = Hh, *H = Hh + mm;
    for (int i = 0; i < m; i++)
      for (int j = 0; j < i; j++) {
        const double g = 0.5 * (G[(size_t)j * m + i] + G[(size_t)i * m + j]);
        const double h = 0.5 * (H[(size_t)j * m + i] + H[(size_t)i * m + j]);
        G[(size_t)j * m + i] = G[(size_t)i * m + j] = g;
        H[(size_t)j * m + i] = H[(size_t)i * m + j] = h;
      }
    const double te = pevsl_now();
    st = pevsl_gen_symeig_range(m, H, G, m, aa - DBL_EPSILON, bb + DBL_EPSILON, &q, lam, Zh, m);
    pevsl->stats->t_eig += pevsl_now() - te;
  }
  pEVSL_ParvecsDuplParvec(vinit, q, (int)n, S->Rvec);
  if (!st && q > 0) {
    /* X = P Z, A X = W Z (into U), unit columns, R = A X - lam X */
    st = memcpy_async(dZ, Zh, sizeof(double) * (size_t)m * q);
    if (!st) st = gemm_nn(n, m, q, P, ld, dZ, m, X, ld);
    if (!st) st = gemm_nn(n, m, q, W, ld, dZ, m, U, ld);
    if (!st) st = vdot_cols(n, q, X, ld, X, ld, dv);
    if (!st) st = memcpy_async(hv, dv, sizeof(double) * q);
    if (!st) st = sync();
    for (int j = 0; j < q && !st; j++) hv[j] = hv[j] > 0 ? 1.0 / sqrt(hv[j]) : 0.0;
    if (!st) st = memcpy_async(dv, hv, sizeof(double) * q);
    if (!st) st = vscal_cols(n, q, X, ld, dv);
    if (!st) st = vscal_cols(n, q, U, ld, dv);
    if (!st) st = memcpy_async(dv + m, lam, sizeof(double) * q);
    if (!st) st = vaxpy_cols(n, q, dv + m, X, ld, U, ld);
    if (!st) st = vdot_cols(n, q, U, ld, U, ld, dv + 2 * m);
    if (!st) st = memcpy_async(hv, dv + 2 * m, sizeof(double) * q);
    if (!st) st = sync();
    double rmin = HUGE_VAL, rmax = 0.0;
    for (int j = 0; j < q && !st; j++) {
      const double r0 = sqrt(hv[j]);
      rmin = PEVSL_MIN(rmin, r0);
      rmax = PEVSL_MAX(rmax, r0);
      if (r0 < tol) {
        S->Lam[S->nev] = lam[j];
        S->res[S->nev] = r0;
        st = vcopy(X + (size_t)j * ld, S->Rvec->data + (size_t)S->nev * S->Rvec->ld, n);
        S->nev++;
      }
    }
    if (!st) st = sync();
    /* a refined pair in [a, b] short of the FP64 path's quality (residual
     * below tol, and below tol * |lam| for |lam| < 1) sends the slice back
     * to FP64 */
    int weak = 0;
    for (int j = 0; j < q; j++)
      if (!(sqrt(hv[j]) < tol * PEVSL_MIN(1.0, fabs(lam[j])))) weak++;
    S->short_pairs = PEVSL_MAX(weak, nbar - S->nev);
    if (getenv("PEVSL_B200_VERBOSE"))
      fprintf(stderr, "refine [%g, %g]: kdim %d, subspace %d, in [a,b] %d, accepted %d, res %.2e..%.2e\n",
              aa, bb, kdim, m, q, S->nev, rmin, rmax);
  } else if (getenv("PEVSL_B200_VERBOSE")) {
    fprintf(stderr, "refine [%g, %g]: kdim %d, subspace %d, in [a,b] %d, status %d\n", aa, bb, kdim,
            m, q, st);
  }
  free(sel);
  free(Y);
  free(Hh);
  free(Zh);
  free(lam);
  free(hv);
  return st;
}

static void free_slice_outputs(SliceState *S) {
  free(S->Lam);
  free(S->res);
  if (S->Rvec) {
    pEVSL_ParvecsFree(S->Rvec);
    free(S->Rvec);
  }
  S->Lam = S->res = nullptr;
  S->Rvec = nullptr;
}

/* Lockstep filtered Lanczos over ns <= kMaxBatch slices sharing vinit. */
static int g_fallbacks = 0; /* slices of the last call re-run in FP64 */

int pEVSL_B200_LastFallbacks(void) { return g_fallbacks; }

int pEVSL_B200_SetGroupReduce(pevsl_Data *pevsl, void (*reduce)(double *buf, int count, void *ctx),
                              void *ctx) {
  if (!pevsl) return PEVSL_ERR_ARG;
  pevsl_inst *inst = pevsl_inst_of(pevsl);
  inst->group_reduce = reduce;
  inst->group_reduce_ctx = ctx;
  return 0;
}

int pEVSL_B200_SetFilterForm(int form) {
  if (form < -1 || form > 2) return PEVSL_ERR_ARG;
  g_filter_form_override = form < 0 ? 2 : form;
  return 0;
}

int pEVSL_B200_SetBarrierSpins(unsigned spins) {
  set_barrier_spins(spins);
  return 0;
}

int pEVSL_B200_SeedBarrierArrivals(unsigned count) { return seed_barrier_arrivals(count); }

/* Filtered Lanczos in lockstep (pEVSL_ChebLanNr, SRC/cheblanNr.c:54-448) for
 * ns <= kMaxEntries slices, which may belong to different problems (each
 * entry carries its instance, matrix, length and start vector).  Every
 * step runs one filter application for all active slices (one launch per
 * degree, or one persistent launch), then the Lanczos recurrence and
 * CGS-DGKS as batched launches of up to kMaxBatch entries.  Per entry the
 * work decomposition is that of a one-slice run, so each slice's result is
 * bit-identical to solving it alone. */
static int cheblannr_group(SliceState *SL, int ns, double tol, FILE *fstats,
                           bool allow_mixed = true) {
  Ctx &c = ctx();
  if (ns <= 0) return 0;
  if (ns > kMaxEntries) return PEVSL_ERR_ARG;
  const bool mixed = allow_mixed && SL[0].A &&
                     pevsl_inst_of(SL[0].pevsl)->precision == PEVSL_PREC_MIXED;
  bool all_builtin = true;
  long nmax = 0;
  for (int s = 0; s < ns; s++) {
    all_builtin = all_builtin && SL[s].A != nullptr;
    nmax = PEVSL_MAX(nmax, SL[s].n);
  }
  /* the lockstep machinery also serves one slice when the filter is
   * graph-replayed (one captured launch sequence per filter application) */
  const bool batched = all_builtin && (ns > 1 || mixed || filter_graph_enabled());
  /* mixed form: trace tolerance per converged value, and the guard of the
   * refinement sweep (PEVSL_B200_MIXED_TRTOL / PEVSL_B200_MIXED_GUARD) */
  double trtol_mixed = 1e-9, guard = 0.3;
  int passes = 1;
  if (getenv("PEVSL_B200_MIXED_TRTOL")) trtol_mixed = atof(getenv("PEVSL_B200_MIXED_TRTOL"));
  if (getenv("PEVSL_B200_MIXED_GUARD")) guard = atof(getenv("PEVSL_B200_MIXED_GUARD"));
  if (getenv("PEVSL_B200_MIXED_PASSES")) passes = PEVSL_MAX(1, atoi(getenv("PEVSL_B200_MIXED_PASSES")));
  std::vector<char> act(ns, 0);
  int nact = 0;
  size_t basis_elems = 0, work_bytes = 0, mu_elems = 0;
  for (int s = 0; s < ns; s++) {
    SliceState *S = &SL[s];
    S->maxit = PEVSL_MIN(S->pevsl->N, S->maxit);
    S->status = 0;
    S->nev = 0;
    S->its = 0;
    S->short_pairs = 0;
    if (pevsl_check_intv(S->intv, fstats) < 0) {
      S->done = 1; /* invalid interval: no pairs, status 0 (SRC/cheblanNr.c:96-100) */
      continue;
    }
    if (fstats) {
      fprintf(fstats, " intv:[%e, %e, %e, %e]\n", S->intv[0], S->intv[1], S->intv[2], S->intv[3]);
      fprintf(fstats, " ** Cheb Poly of deg = %d, gam = %.15e, bar: %.15e\n", S->pol->deg,
              S->pol->gam, S->pol->bar);
    }
    if (S->pol->gam > 1.0 || S->pol->gam < -1.0) {
      fprintf(stdout, "gamB error %.15e\n", S->pol->gam);
      S->status = -1;
      S->done = 1;
      continue;
    }
    if (fstats) fprintf(fstats, " ** Cheb-LanNr \n");
    act[s] = 1;
    nact++;
    basis_elems += (size_t)S->ld * ((size_t)S->maxit + 1);
    work_bytes += 32 * (size_t)S->ld; /* filter work + the graph form's staging */
    mu_elems += (size_t)S->pol->deg + 1;
  }
  if (!nact) return 0;
  /* tune each matrix's stream kernels now: the filter may be captured */
  for (int s = 0; s < ns; s++)
    if (act[s] && SL[s].A && stream_tune(SL[s].A)) return PEVSL_ERR_CUDA;
  if (mixed)
    for (int s = 0; s < ns; s++)
      if (act[s] && csr_make_fp32(SL[s].A)) return PEVSL_ERR_NOMEM;
  /* bases of all active slices in one workspace; three FP64 vectors for
   * the one-slice filter and breakdown restarts; 16 ld bytes of batched
   * filter work per slice; the filter coefficients on the device */
  double *Vall = (double *)ws(WS_BASIS, sizeof(double) * basis_elems);
  double *w3 = (double *)ws(WS_CHEB, sizeof(double) * 3 * (size_t)nmax + (batched ? work_bytes : 0));
  double *vrand = (double *)ws(all_builtin ? WS_VEC : WS_RITZ2, sizeof(double) * (size_t)nmax);
  double *dmu_all = batched ? (double *)ws(WS_MU, sizeof(double) * mu_elems) : nullptr;
  if (!Vall || !w3 || !vrand || (batched && !dmu_all)) return PEVSL_ERR_NOMEM;
  char *bwork = (char *)(w3 + 3 * (size_t)nmax);
  std::vector<char *> work(ns, nullptr);
  std::vector<const double *> dmu(ns, nullptr);
  int st = 0;
  size_t off = 0, woff = 0, moff = 0;
  int maxit_all = 0;
  for (int s = 0; s < ns && !st; s++) {
    SliceState *S = &SL[s];
    if (!act[s]) continue;
    S->V = Vall + off;
    off += (size_t)S->ld * ((size_t)S->maxit + 1);
    if (batched) {
      work[s] = bwork + woff;
      woff += 32 * (size_t)S->ld;
      dmu[s] = dmu_all + moff;
      st = memcpy_async(dmu_all + moff, S->pol->mu, sizeof(double) * ((size_t)S->pol->deg + 1));
      moff += (size_t)S->pol->deg + 1;
    }
    S->dT = (double *)malloc(sizeof(double) * (size_t)S->maxit);
    S->eT = (double *)malloc(sizeof(double) * (size_t)S->maxit);
    S->EvalT = (double *)malloc(sizeof(double) * (size_t)S->maxit);
    if (!S->dT || !S->eT || !S->EvalT) return PEVSL_ERR_NOMEM;
    S->wn = S->tr0 = S->beta = 0.0;
    S->nwn = S->kdim = S->count = S->nconv = 0;
    maxit_all = PEVSL_MAX(maxit_all, S->maxit);
  }
  if (st) return st;
  SegTimer &t_pol = g_t_pol, &t_orth = g_t_orth;
  /* CUDA graph form of the batched filter: one captured launch sequence per
   * set of live slices, replayed every step */
  const bool graph_form = batched && filter_form() == 0 && filter_graph_enabled();
  FilterGraph fg;
  fg.mixed = mixed;
  /* y_s = p_s(A_s) x_s for the slices with sel[s]: x_s = V_s(:,kin) (or the
   * slice's start vector when xin), y_s = V_s(:,kout) */
  auto filter = [&](const std::vector<char> &sel, int kin, bool xin, int kout) -> int {
    t_pol.begin();
    int r = 0;
    if (!batched) {
      for (int s = 0; s < ns && !r; s++)
        if (sel[s])
          r = cheb_apply(SL[s].pevsl, SL[s].pol,
                         xin ? SL[s].vinit->data : SL[s].V + (size_t)kin * SL[s].ld,
                         SL[s].V + (size_t)kout * SL[s].ld, w3, SL[s].n);
    } else {
      std::vector<FilterJob> jobs;
      jobs.reserve(ns);
      for (int s = 0; s < ns; s++)
        if (sel[s])
          jobs.push_back(FilterJob{SL[s].pevsl, SL[s].A,
                                   xin ? SL[s].vinit->data : SL[s].V + (size_t)kin * SL[s].ld,
                                   SL[s].V + (size_t)kout * SL[s].ld, SL[s].pol, dmu[s], work[s],
                                   SL[s].ld});
      if (graph_form)
        r = filter_graphed(fg, sel, jobs);
      else
        r = cheb_filter_batch((int)jobs.size(), jobs.data(), mixed);
    }
    t_pol.end();
    return r;
  };
  /* a batched operation over the active entries, kMaxBatch at a time:
   * op(first entry, count, mask, lengths) */
  auto chunks = [&](const std::vector<char> &sel, auto &&op) -> int {
    for (int c0 = 0; c0 < ns; c0 += kMaxBatch) {
      const int cs = PEVSL_MIN(kMaxBatch, ns - c0);
      unsigned mask = 0;
      BLen len{};
      for (int i = 0; i < cs; i++) {
        len.n[i] = SL[c0 + i].n;
        len.ld[i] = SL[c0 + i].ld;
        if (sel[c0 + i]) mask |= 1u << i;
      }
      if (!mask) continue;
      const int r = op(c0, cs, mask, len);
      if (r) return r;
    }
    return 0;
  };
  /* per-entry device scalars: alpha, ||v|| before CGS, ||v|| after, and the
   * DGKS flag */
  double *dA = c.gscal, *dN0 = c.gscal + kMaxEntries, *dN = c.gscal + 2 * kMaxEntries;
  double *hA = c.hgscal, *hN = c.hgscal + 2 * kMaxEntries;
  int *dF = c.gflag;
  const long ldw = maxit_all + 1;
  double *dW = (double *)ws(WS_GROUP, sizeof(double) * (size_t)ns * (size_t)ldw);
  if (!dW) return PEVSL_ERR_NOMEM;
  for (int s = 0; s < ns; s++)
    if (act[s] && SL[s].A) matrix_window(SL[s].A);
  cudaEvent_t e_all0, e_all1;
  cudaEventCreate(&e_all0);
  cudaEventCreate(&e_all1);
  cudaEventRecord(e_all0, c.stream);
  /* filter the start vector, normalise (SRC/cheblanNr.c:164-194) */
  st = filter(act, 0, true, 0);
  if (!st)
    st = chunks(act, [&](int c0, int cs, unsigned mask, const BLen &len) {
      CPtrs x{};
      for (int i = 0; i < cs; i++) x.p[i] = SL[c0 + i].V;
      return b_dot(len, cs, x, x, dA + c0, FIN_SQRT, mask);
    });
  if (!st) st = memcpy_async(hA, dA, sizeof(double) * (size_t)ns);
  if (!st) st = sync();
  if (!st)
    st = chunks(act, [&](int c0, int cs, unsigned mask, const BLen &len) {
      BScal inv{};
      VPtrs y{};
      for (int i = 0; i < cs; i++) {
        inv.v[i] = 1.0 / hA[c0 + i];
        y.p[i] = SL[c0 + i].V;
      }
      return b_scal(len, cs, y, inv, mask);
    });
  int k;
  for (k = 0; nact > 0 && !st; k++) {
    st = filter(act, k, false, k + 1);
    auto col = [&](int s, int j) { return SL[s].V + (size_t)j * SL[s].ld; };
    if (!st && k > 0)
      st = chunks(act, [&](int c0, int cs, unsigned mask, const BLen &len) {
        CPtrs vprev{};
        VPtrs vnew{};
        BScal mb{};
        for (int i = 0; i < cs; i++) {
          vprev.p[i] = col(c0 + i, k - 1);
          vnew.p[i] = col(c0 + i, k + 1);
          mb.v[i] = -SL[c0 + i].beta;
        }
        return b_axpy(len, cs, vprev, vnew, mb, mask);
      });
    if (!st)
      st = chunks(act, [&](int c0, int cs, unsigned mask, const BLen &len) {
        CPtrs vk{}, vks{};
        for (int i = 0; i < cs; i++) {
          vk.p[i] = col(c0 + i, k);
          vks.p[i] = col(c0 + i, k + 1);
        }
        return b_dot(len, cs, vk, vks, dA + c0, FIN_ID, mask);
      });
    t_orth.begin();
    /* v -= alpha v_k, ||v||; CGS_DGKS: pass 1, then pass 2 where the first
     * kept <= 1/sqrt(2) of the norm */
    if (!st)
      st = chunks(act, [&](int c0, int cs, unsigned mask, const BLen &len) {
        CPtrs vk{}, Vc{}, vks{};
        VPtrs vnew{};
        for (int i = 0; i < cs; i++) {
          vk.p[i] = col(c0 + i, k);
          vnew.p[i] = col(c0 + i, k + 1);
          vks.p[i] = vnew.p[i];
          Vc.p[i] = SL[c0 + i].V;
        }
        int r = b_axpy_dev_nrm2(len, cs, dA + c0, vk, vnew, dN0 + c0, mask);
        double *w = dW + (size_t)c0 * ldw;
        if (!r) r = b_gemvT(len, cs, k + 1, Vc, vks, w, ldw, nullptr, mask);
        if (!r)
          r = b_gemv_sub_nrm(len, cs, k + 1, Vc, w, ldw, vnew, dN + c0, nullptr, dF + c0, dN0 + c0,
                             kEta, mask);
        if (!r) r = b_gemvT(len, cs, k + 1, Vc, vks, w, ldw, dF + c0, mask);
        if (!r)
          r = b_gemv_sub_nrm(len, cs, k + 1, Vc, w, ldw, vnew, dN + c0, dF + c0, nullptr, nullptr,
                             kEta, mask);
        return r;
      });
    t_orth.end();
    if (!st) st = memcpy_async(hA, dA, sizeof(double) * (size_t)ns);
    if (!st) st = memcpy_async(hN, dN, sizeof(double) * (size_t)ns);
    if (!st) st = sync();
    if (st) break;
    t_pol.flush();
    t_orth.flush();
    std::vector<char> scal_sel(ns, 0);
    std::vector<double> inv(ns, 0.0);
    for (int s = 0; s < ns && !st; s++) {
      if (!act[s]) continue;
      SliceState *S = &SL[s];
      const double alpha = hA[s];
      double beta = hN[s];
      if (!isfinite(alpha) || !isfinite(beta)) {
        S->status = PEVSL_ERR_NONFINITE;
        S->done = 1;
        act[s] = 0;
        nact--;
        continue;
      }
      S->dT[k] = alpha;
      S->wn += fabs(alpha);
      S->wn += 2.0 * beta;
      S->nwn += 3;
      double *znew = S->V + (size_t)(k + 1) * S->ld;
      if (beta * S->nwn < orthTol * S->wn) {
        /* lucky breakdown: restart from a new filtered random vector
         * (SRC/cheblanNr.c:248-281) */
        if (fstats) fprintf(fstats, "it %4d: Lucky breakdown, beta = %.15e\n", k, beta);
        st = pevsl_rand_vector_dev(vrand, (int)S->n);
        t_pol.begin();
        if (!st) st = cheb_apply(S->pevsl, S->pol, vrand, znew, w3, S->n);
        t_pol.end();
        if (!st) st = vnrm2(S->n, znew, c.dscal + S_NRM0);
        if (!st) st = cgs_dgks(S->V, S->ld, k + 1, znew, S->n);
        const double *hb = st ? nullptr : fetch_scalars(S_NRM, 1);
        if (!hb) {
          st = st ? st : PEVSL_ERR_CUDA;
          break;
        }
        st = vscal(znew, S->n, 1.0 / hb[0]);
        beta = 0.0;
      } else {
        inv[s] = 1.0 / beta;
        scal_sel[s] = 1;
      }
      S->beta = beta;
      S->eT[k] = beta;
    }
    if (!st)
      st = chunks(scal_sel, [&](int c0, int cs, unsigned mask, const BLen &len) {
        BScal v{};
        VPtrs sc{};
        for (int i = 0; i < cs; i++) {
          v.v[i] = inv[c0 + i];
          sc.p[i] = col(c0 + i, k + 1);
        }
        return b_scal(len, cs, sc, v, mask);
      });
    if (st) break;
    /* restricted-trace convergence test (SRC/cheblanNr.c:293-332); the
     * eigenvalues of the testing slices' T are computed first, on host
     * threads (each slice's own arithmetic, so the same values), then the
     * tests run in slice order */
    std::vector<int> tests;
    for (int s = 0; s < ns; s++)
      if (act[s] && !((k < 30 || (k - 30) % 20 != 0) && k != SL[s].maxit - 1)) tests.push_back(s);
    std::vector<int> eig_st(tests.size(), 0);
    std::vector<double> eig_secs(tests.size(), 0.0);
    host_parallel(tests.size(), k + 1 >= 64, [&](size_t i) {
      SliceState *S = &SL[tests[i]];
      const double te = pevsl_now();
      eig_st[i] = pevsl_tridiag_eig(k + 1, S->dT, S->eT, S->EvalT, nullptr);
      eig_secs[i] = pevsl_now() - te;
    });
    for (size_t ti = 0; ti < tests.size(); ti++) {
      const int s = tests[ti];
      SliceState *S = &SL[s];
      S->kdim = k + 1;
      if (eig_st[ti]) {
        st = PEVSL_ERR_EIG;
        break;
      }
      S->pevsl->stats->t_eig += eig_secs[ti];
      S->count = S->kdim;
      double tr1 = 0.0;
      S->nconv = 0;
      for (int i = 0; i < S->count; i++) {
        if (S->EvalT[i] + 5 * DBL_EPSILON >= S->pol->bar) {
          tr1 += S->EvalT[i];
          S->nconv++;
        }
      }
      if (fstats) fprintf(fstats, "  k %4d:   nconv %4d  tr1 %21.15e\n", k, S->nconv, tr1);
      /* FP64: the reference's test; mixed: differences at the FP32 noise
       * level of the filtered operator count as converged */
      const double trtol = mixed ? trtol_mixed * PEVSL_MAX(1, S->nconv) : 2e-12;
      const bool conv = fabs(tr1 - S->tr0) < trtol || fabs(tr1) + fabs(S->tr0) < 1e-10;
      S->tr0 = tr1;
      if (conv || k == S->maxit - 1) {
        if (!conv && fstats)
          fprintf(fstats, "The max number of iterations [%d] has been reached. The eigenvalues "
                          "computed may not have converged\n", S->maxit);
        act[s] = 0;
        nact--;
      }
    }
  }
  cudaEventRecord(e_all1, c.stream);
  const double tr_start = pevsl_now();
  /* the host part of every finished slice's Ritz extraction first, on host
   * threads; then the device part slice by slice */
  std::vector<RitzHost> rh((size_t)ns);
  if (!st && !mixed) {
    std::vector<int> fin;
    int kmax = 0;
    for (int s = 0; s < ns; s++)
      if (!SL[s].done && !SL[s].status) {
        fin.push_back(s);
        kmax = PEVSL_MAX(kmax, SL[s].kdim);
      }
    host_parallel(fin.size(), kmax >= 64, [&](size_t i) { ritz_host(&SL[fin[i]], &rh[fin[i]]); });
  }
  for (int s = 0; s < ns && !st; s++) {
    SliceState *S = &SL[s];
    if (S->done || S->status) continue;
    S->its = S->kdim;
    const int rs = mixed ? ritz_refine(S->pevsl, S, S->vinit, S->n, S->ld, tol, guard, passes)
                         : ritz_extract(S->pevsl, S, &rh[s], S->vinit, S->n, S->ld, tol);
    if (rs) S->status = rs;
  }
  for (RitzHost &R : rh) {
    free(R.sel);
    free(R.Y);
  }
  for (int s = 0; s < ns; s++) SL[s].pevsl->stats->t_ritz = pevsl_now() - tr_start;
  cudaEventSynchronize(e_all1);
  t_pol.flush();
  t_orth.flush();
  float ms_all = 0.f;
  cudaEventElapsedTime(&ms_all, e_all0, e_all1);
  cudaEventDestroy(e_all0);
  cudaEventDestroy(e_all1);
  for (int s = 0; s < ns; s++) {
    pevsl_inst *inst = pevsl_inst_of(SL[s].pevsl);
    if (s > 0 && SL[s].pevsl == SL[s - 1].pevsl) continue;
    inst->phase_ms[2] = ms_all;
    inst->phase_ms[3] = t_pol.acc_ms;
    inst->phase_ms[4] = t_orth.acc_ms;
    SL[s].pevsl->stats->t_polAv += 1e-3 * t_pol.acc_ms;
    SL[s].pevsl->stats->t_reorth += 1e-3 * t_orth.acc_ms;
  }
  if (all_builtin) g_filter_ms += t_pol.acc_ms;
  for (int s = 0; s < ns; s++) {
    free(SL[s].dT);
    free(SL[s].eT);
    free(SL[s].EvalT);
    SL[s].dT = SL[s].eT = SL[s].EvalT = nullptr;
  }
  if (mixed && !st) {
    /* a slice is run again in FP64 when a refined pair in [a, b] misses the
     * FP64 path's quality, or fewer pairs were accepted than the Lanczos
     * run had Ritz values above bar, so the mixed form never reports fewer
     * or worse pairs */
    std::vector<SliceState> R;
    std::vector<int> idx;
    for (int s = 0; s < ns; s++) {
      SliceState *S = &SL[s];
      if (S->done || S->status || S->short_pairs <= 0) continue;
      free_slice_outputs(S);
      SliceState r;
      memset(&r, 0, sizeof r);
      memcpy(r.intv, S->intv, sizeof S->intv);
      r.pol = S->pol;
      r.maxit = S->maxit;
      r.pevsl = S->pevsl;
      r.A = S->A;
      r.vinit = S->vinit;
      r.n = S->n;
      r.ld = S->ld;
      R.push_back(r);
      idx.push_back(s);
    }
    if (!R.empty()) {
      g_fallbacks += (int)R.size();
      pevsl_inst *inst = pevsl_inst_of(SL[0].pevsl);
      const float ms0 = inst->phase_ms[2], pol0 = inst->phase_ms[3], orth0 = inst->phase_ms[4];
      st = cheblannr_group(R.data(), (int)R.size(), tol, fstats, false);
      inst->phase_ms[2] += ms0;
      inst->phase_ms[3] += pol0;
      inst->phase_ms[4] += orth0;
      for (size_t r = 0; r < R.size(); r++) {
        SliceState *S = &SL[idx[r]];
        S->status = R[r].status;
        S->kdim = R[r].kdim;
        S->its = R[r].its;
        S->nconv = R[r].nconv;
        S->nev = R[r].nev;
        S->Lam = R[r].Lam;
        S->res = R[r].res;
        S->Rvec = R[r].Rvec;
        S->short_pairs = 0;
      }
    }
  }
  return st;
}

static void slice_bind(SliceState *S, pevsl_Data *pevsl, pevsl_Parvec *vinit) {
  S->pevsl = pevsl;
  S->A = pevsl_builtin_A(pevsl);
  S->vinit = vinit;
  S->n = pevsl->n;
  S->ld = round_ld(pevsl->n);
}

int pEVSL_ChebLanNr(pevsl_Data *pevsl, double *intv, int maxit, double tol, pevsl_Parvec *vinit,
                    pevsl_Polparams *pol, int *nevOut, double **lamo, pevsl_Parvecs **Wo,
                    double **reso, FILE *fstats) {
  const double tall = pevsl_now();
  *nevOut = 0;
  *lamo = nullptr;
  *Wo = nullptr;
  *reso = nullptr;
  if (ensure()) return PEVSL_ERR_CUDA;
  if (pevsl->ifGenEv) {
    int its = 0;
    const int st = pevsl_gen_cheblannr(pevsl, intv, maxit, tol, vinit, pol, nevOut, lamo, Wo, reso,
                                       &its, fstats);
    pevsl_inst_of(pevsl)->last_its = its;
    pevsl->stats->t_iter = pevsl_now() - tall;
    return st;
  }
  SliceState S;
  memset(&S, 0, sizeof S);
  memcpy(S.intv, intv, sizeof S.intv);
  S.pol = pol;
  S.maxit = maxit;
  slice_bind(&S, pevsl, vinit);
  g_t_pol.init();
  g_t_orth.init();
  g_fallbacks = 0;
  int st = cheblannr_group(&S, 1, tol, fstats);
  pevsl_inst *inst = pevsl_inst_of(pevsl);
  inst->last_its = S.kdim;
  inst->last_nconv = S.nconv;
  if (!st) st = S.status;
  if (st) {
    free_slice_outputs(&S);
    return st;
  }
  *nevOut = S.nev;
  *lamo = S.Lam;
  *Wo = S.Rvec;
  *reso = S.res;
  pevsl->stats->t_iter = pevsl_now() - tall;
  return 0;
}

/* outputs of a solved group into the caller's arrays at offset o */
static int group_outputs(SliceState *SL, int ns, int st, int o, int *nevOut, double **lamo,
                         pevsl_Parvecs **Wo, double **reso, int *its, int *status) {
  int first_err = 0;
  for (int s = 0; s < ns; s++) {
    SliceState *S = &SL[s];
    const int ss = st ? st : S->status;
    status[o + s] = ss;
    its[o + s] = S->kdim;
    if (ss) {
      free_slice_outputs(S);
      nevOut[o + s] = 0;
      lamo[o + s] = nullptr;
      Wo[o + s] = nullptr;
      reso[o + s] = nullptr;
      if (!first_err) first_err = ss;
    } else {
      nevOut[o + s] = S->nev;
      lamo[o + s] = S->Lam;
      Wo[o + s] = S->Rvec;
      reso[o + s] = S->res;
    }
  }
  return first_err;
}

int pEVSL_B200_ChebLanNrBatch(pevsl_Data *pevsl, int nslices, const double *intvs,
                              const int *maxits, double tol, pevsl_Parvec *vinit,
                              pevsl_Polparams *pols, int *nevOut, double **lamo,
                              pevsl_Parvecs **Wo, double **reso, int *its, int *status,
                              FILE *fstats) {
  const double tall = pevsl_now();
  if (ensure()) return PEVSL_ERR_CUDA;
  if (nslices < 0) return PEVSL_ERR_ARG;
  int first_err = 0;
  if (pevsl->ifGenEv) {
    /* generalized problem: in lockstep where the lockstep form applies,
     * else the slices one after the other */
    if (nslices >= 2 && nslices <= kMaxBatch) {
      const int r = pevsl_gen_cheblannr_lockstep(pevsl, nslices, intvs, maxits, tol, vinit, pols,
                                                 nevOut, lamo, Wo, reso, its, status, fstats);
      if (r != 1) {
        pevsl->stats->t_iter = pevsl_now() - tall;
        return r;
      }
    }
    for (int s = 0; s < nslices; s++) {
      double iv[4];
      memcpy(iv, intvs + 4 * (size_t)s, sizeof iv);
      status[s] = pevsl_gen_cheblannr(pevsl, iv, maxits[s], tol, vinit, &pols[s], &nevOut[s],
                                      &lamo[s], &Wo[s], &reso[s], &its[s], fstats);
      if (status[s] && !first_err) first_err = status[s];
    }
    pevsl->stats->t_iter = pevsl_now() - tall;
    return first_err;
  }
  g_t_pol.init();
  g_t_orth.init();
  g_fallbacks = 0;
  double ms_total = 0.0, pol_total = 0.0, orth_total = 0.0;
  for (int s0 = 0; s0 < nslices; s0 += kMaxEntries) {
    const int ns = PEVSL_MIN(kMaxEntries, nslices - s0);
    std::vector<SliceState> SL(ns);
    memset(SL.data(), 0, sizeof(SliceState) * (size_t)ns);
    for (int s = 0; s < ns; s++) {
      memcpy(SL[s].intv, intvs + 4 * (size_t)(s0 + s), sizeof SL[s].intv);
      SL[s].pol = &pols[s0 + s];
      SL[s].maxit = maxits[s0 + s];
      slice_bind(&SL[s], pevsl, vinit);
    }
    int st = cheblannr_group(SL.data(), ns, tol, fstats);
    pevsl_inst *inst = pevsl_inst_of(pevsl);
    ms_total += inst->phase_ms[2];
    pol_total += inst->phase_ms[3];
    orth_total += inst->phase_ms[4];
    const int e = group_outputs(SL.data(), ns, st, s0, nevOut, lamo, Wo, reso, its, status);
    if (!first_err) first_err = e;
  }
  pevsl_inst *inst = pevsl_inst_of(pevsl);
  inst->phase_ms[2] = ms_total;
  inst->phase_ms[3] = pol_total;
  inst->phase_ms[4] = orth_total;
  pevsl->stats->t_iter = pevsl_now() - tall;
  return first_err;
}

int pEVSL_B200_ChebLanNrMulti(int nprob, pevsl_Data **pevsls, const int *nslices,
                              const double *intvs, const int *maxits, double tol,
                              pevsl_Parvec **vinits, pevsl_Polparams *pols, int *nevOut,
                              double **lamo, pevsl_Parvecs **Wo, double **reso, int *its,
                              int *status, FILE *fstats) {
  if (ensure()) return PEVSL_ERR_CUDA;
  if (nprob < 0 || (nprob > 0 && (!pevsls || !nslices || !vinits))) return PEVSL_ERR_ARG;
  for (int p = 0; p < nprob; p++) {
    if (!pevsls[p] || nslices[p] < 0) return PEVSL_ERR_ARG;
  }
  g_t_pol.init();
  g_t_orth.init();
  g_fallbacks = 0;
  int first_err = 0;
  /* groups of up to kMaxEntries slices; a problem is kept in one group
   * where it fits, a problem with more slices fills groups of its own */
  std::vector<SliceState> SL;
  int o = 0, o0 = 0;
  auto flush = [&]() {
    if (SL.empty()) return;
    const int st = cheblannr_group(SL.data(), (int)SL.size(), tol, fstats);
    const int e = group_outputs(SL.data(), (int)SL.size(), st, o0, nevOut, lamo, Wo, reso, its,
                                status);
    if (!first_err) first_err = e;
    o0 += (int)SL.size();
    SL.clear();
  };
  for (int p = 0; p < nprob; p++) {
    if (pevsls[p]->ifGenEv) {
      /* a generalized problem: its slices one after the other */
      flush();
      for (int s = 0; s < nslices[p]; s++, o++) {
        double iv[4];
        memcpy(iv, intvs + 4 * (size_t)o, sizeof iv);
        status[o] = pevsl_gen_cheblannr(pevsls[p], iv, maxits[o], tol, vinits[p], &pols[o],
                                        &nevOut[o], &lamo[o], &Wo[o], &reso[o], &its[o], fstats);
        if (status[o] && !first_err) first_err = status[o];
      }
      o0 = o;
      continue;
    }
    if (!SL.empty() && (int)SL.size() + nslices[p] > kMaxEntries) flush();
    for (int s = 0; s < nslices[p]; s++, o++) {
      if ((int)SL.size() == kMaxEntries) flush();
      SliceState S;
      memset(&S, 0, sizeof S);
      memcpy(S.intv, intvs + 4 * (size_t)o, sizeof S.intv);
      S.pol = &pols[o];
      S.maxit = maxits[o];
      slice_bind(&S, pevsls[p], vinits[p]);
      SL.push_back(S);
    }
  }
  flush();
  return first_err;
}

}  // extern "C"
