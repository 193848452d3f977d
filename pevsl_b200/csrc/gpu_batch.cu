/*
 * Batched vector kernels: one launch serves up to kMaxBatch independent
 * vectors (the slices of an interval, advancing in lockstep), selected by a
 * bit mask, each with its own pointers and scalars.  blockIdx.y (or z) is the
 * batch entry; within an entry the work decomposition, and hence every
 * rounding, is the same as for a single vector, so a batched run gives the
 * same bits as running the entries one by one.  The single-vector wrappers
 * of gpu.cuh are these kernels with one entry.
 *
 *   b_dot / b_axpy_dev_nrm2  dots and norms: SRC/parvec.c:123-142
 *   b_gemvT / b_gemv_sub_nrm one CGS pass of CGS_DGKS: SRC/miscla.c:211-240
 *
 * Entries may differ in length (slices of different problems): entry s has
 * length len.n[s] and leading dimension len.ld[s], and is decomposed over
 * exactly the blocks a single-vector launch of that length would use (the
 * grid is as wide as the widest entry; the surplus blocks of a shorter
 * entry leave at once), so its reductions add in the same order.
 *
 * The batched filter degree is cheb_step_batch (gpu_sparse.cu).
 */
#include <cuda_runtime.h>

#include "gpu.cuh"
#include "gpu_device.cuh"

namespace pv {

#define PV_ACTIVE(mask, s) (((mask) >> (s)) & 1u)

/* per-entry decomposition of one launch */
struct BGeom {
  long n[kMaxBatch];
  long ld[kMaxBatch];
  unsigned nb[kMaxBatch]; /* blocks of entry s (x dimension) */
  int rows[kMaxBatch];    /* gemvT: rows per block of entry s */
};

/* grid_sum over the first nb blocks of the x dimension */
__device__ __forceinline__ double grid_sum_n(double part, double *partials, unsigned *counter,
                                             int fin, unsigned nb, bool *is_last) {
  __shared__ double sh[32];
  __shared__ bool am_last;
  const double s = block_sum(part, sh);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = s;
    __threadfence();
    am_last = atomicAdd(counter, 1u) == nb - 1;
  }
  __syncthreads();
  *is_last = am_last;
  if (!am_last) return 0.0;
  __threadfence();
  double t = 0.0;
  for (unsigned i = threadIdx.x; i < nb; i += blockDim.x) t += __ldcg(partials + i);
  t = block_sum(t, sh);
  if (threadIdx.x == 0) *counter = 0;
  return fin == FIN_SQRT ? sqrt(t) : t;
}

/* ---------------------------------------------------------------- level 1 */

__global__ void k_b_axpy(BGeom g, CPtrs x, VPtrs y, BScal a, unsigned mask) {
  const int s = blockIdx.y;
  if (!PV_ACTIVE(mask, s) || blockIdx.x >= g.nb[s]) return;
  const long n = g.n[s];
  const double c = a.v[s];
  const double *xs = x.p[s];
  double *ys = y.p[s];
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)g.nb[s] * blockDim.x)
    ys[i] += c * xs[i];
}

__global__ void k_b_scal(BGeom g, VPtrs x, BScal a, unsigned mask) {
  const int s = blockIdx.y;
  if (!PV_ACTIVE(mask, s) || blockIdx.x >= g.nb[s]) return;
  const long n = g.n[s];
  const double c = a.v[s];
  double *xs = x.p[s];
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)g.nb[s] * blockDim.x)
    xs[i] *= c;
}

__global__ void k_b_dot(BGeom g, CPtrs x, CPtrs y, double *partials, unsigned *counters, double *out,
                        int fin, unsigned mask) {
  const int s = blockIdx.y;
  if (!PV_ACTIVE(mask, s) || blockIdx.x >= g.nb[s]) return;
  const long n = g.n[s];
  const double *xs = x.p[s], *ys = y.p[s];
  double acc = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)g.nb[s] * blockDim.x)
    acc += xs[i] * ys[i];
  bool last;
  const double t =
      grid_sum_n(acc, partials + (size_t)s * kMaxRedBlocks, counters + s, fin, g.nb[s], &last);
  if (last && threadIdx.x == 0) out[s] = t;
}

/* y -= coef[s] x, then ||y|| */
__global__ void k_b_axpy_dev_nrm2(BGeom g, const double *coef, CPtrs x, VPtrs y, double *partials,
                                  unsigned *counters, double *nrm, unsigned mask) {
  const int s = blockIdx.y;
  if (!PV_ACTIVE(mask, s) || blockIdx.x >= g.nb[s]) return;
  const long n = g.n[s];
  const double a = -coef[s];
  const double *xs = x.p[s];
  double *ys = y.p[s];
  double acc = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)g.nb[s] * blockDim.x) {
    const double v = ys[i] + a * xs[i];
    ys[i] = v;
    acc += v * v;
  }
  bool last;
  const double t = grid_sum_n(acc, partials + (size_t)s * kMaxRedBlocks, counters + s, FIN_SQRT,
                              g.nb[s], &last);
  if (last && threadIdx.x == 0) nrm[s] = t;
}

/* ---------------------------------------------------------------- CGS pass */

constexpr int kGemvtCols = 4; /* columns per warp in gemvT */

static int gemvt_rows(long n) { return n < (1L << 16) ? 256 : 1024; }

/* partial[s][rb][j] = sum_{i in row block rb} V_s[i + j ld_s] v_s[i] (nb[s]
 * row blocks of rows[s] rows; the partials of entry s start at s*pstride) */
__global__ void __launch_bounds__(kThreads)
    k_b_gemvt_partial(BGeom g, int k, CPtrs V, CPtrs v, double *__restrict__ partial,
                      size_t pstride, const int *run, unsigned mask) {
  const int s = blockIdx.z;
  if (!PV_ACTIVE(mask, s) || (run && run[s] == 0) || blockIdx.x >= g.nb[s]) return;
  extern __shared__ double vsh[];
  const long n = g.n[s], ldv = g.ld[s];
  const int rows = g.rows[s];
  const long r0 = (long)blockIdx.x * rows;
  const int nr = (int)((n - r0) < rows ? (n - r0) : rows);
  const double *vs = v.p[s];
  for (int i = threadIdx.x; i < nr; i += blockDim.x) vsh[i] = vs[r0 + i];
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int cbase = blockIdx.y * wpb * kGemvtCols;
  double *ps = partial + (size_t)s * pstride;
#pragma unroll
  for (int q = 0; q < kGemvtCols; q++) {
    const int j = cbase + q * wpb + wib;
    if (j >= k) break;
    const double *col = V.p[s] + (size_t)j * ldv + r0;
    double acc = 0.0;
#pragma unroll 4
    for (int i = lane; i < nr; i += 32) acc = fma(col[i], vsh[i], acc);
    acc = warp_sum(acc);
    if (lane == 0) ps[(size_t)blockIdx.x * k + j] = acc;
  }
}

/* w[s*ldw + j] = sum_rb partial[s][rb][j], in row-block order */
__global__ void k_b_gemvt_reduce(BGeom g, int k, const double *__restrict__ partial, size_t pstride,
                                 double *__restrict__ w, long ldw, const int *run, unsigned mask) {
  const int s = blockIdx.y;
  if (!PV_ACTIVE(mask, s) || (run && run[s] == 0)) return;
  const double *ps = partial + (size_t)s * pstride;
  const unsigned nrb = g.nb[s];
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < k; j += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (unsigned b = 0; b < nrb; b++) acc += ps[(size_t)b * k + j];
    w[(size_t)s * ldw + j] = acc;
  }
}

/* v_s -= V_s w_s (thread per row, w_s in shared memory), ||v_s||, and the
 * DGKS flag for the next pass: flag[s] = ||v_s|| <= eta * nrm_old[s]. */
__global__ void __launch_bounds__(kThreads)
    k_b_gemv_sub_nrm(BGeom g, int k, CPtrs V, const double *__restrict__ w, long ldw, VPtrs v,
                     double *partials, unsigned *counters, double *nrm, const int *run,
                     int *flag_out, double *nrm_old, double eta, unsigned mask) {
  const int s = blockIdx.y;
  if (!PV_ACTIVE(mask, s) || (run && run[s] == 0) || blockIdx.x >= g.nb[s]) return;
  extern __shared__ double wsh[];
  for (int j = threadIdx.x; j < k; j += blockDim.x) wsh[j] = w[(size_t)s * ldw + j];
  __syncthreads();
  const long n = g.n[s], ldv = g.ld[s];
  const double *Vs = V.p[s];
  double *vs = v.p[s];
  double ss = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)g.nb[s] * blockDim.x) {
    const double *row = Vs + i;
    double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0, acc3 = 0.0;
    int j = 0;
    for (; j + 3 < k; j += 4) {
      acc0 = fma(row[(size_t)j * ldv], wsh[j], acc0);
      acc1 = fma(row[(size_t)(j + 1) * ldv], wsh[j + 1], acc1);
      acc2 = fma(row[(size_t)(j + 2) * ldv], wsh[j + 2], acc2);
      acc3 = fma(row[(size_t)(j + 3) * ldv], wsh[j + 3], acc3);
    }
    for (; j < k; j++) acc0 = fma(row[(size_t)j * ldv], wsh[j], acc0);
    const double nv = vs[i] - ((acc0 + acc1) + (acc2 + acc3));
    vs[i] = nv;
    ss = fma(nv, nv, ss);
  }
  bool last;
  const double t = grid_sum_n(ss, partials + (size_t)s * kMaxRedBlocks, counters + s, FIN_SQRT,
                              g.nb[s], &last);
  if (last && threadIdx.x == 0) {
    nrm[s] = t;
    if (flag_out) flag_out[s] = t <= eta * nrm_old[s] ? 1 : 0;
    if (nrm_old) nrm_old[s] = t;
  }
}

/* ---------------------------------------------------------------- host wrappers */

BLen blen_uniform(long n, long ld, int S) {
  BLen l{};
  for (int s = 0; s < S && s < kMaxBatch; s++) {
    l.n[s] = n;
    l.ld[s] = ld;
  }
  return l;
}

/* per-entry geometry: nb[s] = the single-vector grid of entry s; returns
 * the widest, or 0 when no active entry has work */
static unsigned geom(const BLen &len, int S, unsigned mask, int per_thread, BGeom *g) {
  unsigned gx = 0;
  for (int s = 0; s < S; s++) {
    g->n[s] = len.n[s];
    g->ld[s] = len.ld[s];
    g->nb[s] = len.n[s] > 0 ? grid_for(len.n[s], per_thread) : 0;
    g->rows[s] = 0;
    if (PV_ACTIVE(mask, s) && len.n[s] > 0 && g->nb[s] > gx) gx = g->nb[s];
  }
  return gx;
}

int b_axpy(const BLen &len, int S, CPtrs x, VPtrs y, BScal a, unsigned mask) {
  BGeom g;
  const unsigned gx = geom(len, S, mask, 4, &g);
  if (!gx) return 0;
  k_b_axpy<<<dim3(gx, S), kThreads, 0, ctx().stream>>>(g, x, y, a, mask);
  return launched("b_axpy");
}

int b_scal(const BLen &len, int S, VPtrs x, BScal a, unsigned mask) {
  BGeom g;
  const unsigned gx = geom(len, S, mask, 4, &g);
  if (!gx) return 0;
  k_b_scal<<<dim3(gx, S), kThreads, 0, ctx().stream>>>(g, x, a, mask);
  return launched("b_scal");
}

int b_dot(const BLen &len, int S, CPtrs x, CPtrs y, double *out, int fin, unsigned mask) {
  BGeom g;
  unsigned gx = geom(len, S, mask, 4, &g);
  if (!mask) return 0;
  for (int s = 0; s < S; s++)
    if (!g.nb[s]) g.nb[s] = 1; /* an empty entry still writes its (zero) result */
  if (!gx) gx = 1;
  k_b_dot<<<dim3(gx, S), kThreads, 0, ctx().stream>>>(g, x, y, ctx().red, ctx().cnt, out, fin, mask);
  return launched("b_dot");
}

int b_axpy_dev_nrm2(const BLen &len, int S, const double *coef, CPtrs x, VPtrs y, double *nrm,
                    unsigned mask) {
  BGeom g;
  unsigned gx = geom(len, S, mask, 4, &g);
  if (!mask) return 0;
  for (int s = 0; s < S; s++)
    if (!g.nb[s]) g.nb[s] = 1;
  if (!gx) gx = 1;
  k_b_axpy_dev_nrm2<<<dim3(gx, S), kThreads, 0, ctx().stream>>>(g, coef, x, y, ctx().red,
                                                                ctx().cnt, nrm, mask);
  return launched("b_axpy_dev_nrm2");
}

int b_gemvT(const BLen &len, int S, int k, CPtrs V, CPtrs v, double *w, long ldw, const int *run,
            unsigned mask) {
  if (k <= 0 || !mask) return 0;
  BGeom g;
  geom(len, S, mask, 1, &g);
  unsigned gx = 0;
  int maxrows = 0;
  for (int s = 0; s < S; s++) {
    const int rows = gemvt_rows(len.n[s]);
    g.rows[s] = rows;
    g.nb[s] = len.n[s] > 0 ? (unsigned)((len.n[s] + rows - 1) / rows) : 0;
    if (PV_ACTIVE(mask, s)) {
      gx = g.nb[s] > gx ? g.nb[s] : gx;
      maxrows = rows > maxrows ? rows : maxrows;
    }
  }
  if (!gx) return 0;
  const size_t pstride = (size_t)gx * (size_t)k;
  double *part = (double *)ws(WS_PART, sizeof(double) * (size_t)S * pstride);
  if (!part) return PEVSL_ERR_NOMEM;
  const int cols_per_block = (kThreads / 32) * kGemvtCols;
  dim3 g1(gx, (unsigned)((k + cols_per_block - 1) / cols_per_block), S);
  k_b_gemvt_partial<<<g1, kThreads, sizeof(double) * maxrows, ctx().stream>>>(g, k, V, v, part,
                                                                              pstride, run, mask);
  if (launched("b_gemvT_partial")) return PEVSL_ERR_CUDA;
  dim3 g2((unsigned)((k + kThreads - 1) / kThreads), S);
  k_b_gemvt_reduce<<<g2, kThreads, 0, ctx().stream>>>(g, k, part, pstride, w, ldw, run, mask);
  return launched("b_gemvT_reduce");
}

int b_gemv_sub_nrm(const BLen &len, int S, int k, CPtrs V, const double *w, long ldw, VPtrs v,
                   double *nrm, const int *run, int *flag_out, double *nrm_old, double eta,
                   unsigned mask) {
  if (!mask) return 0;
  if (k > 12288) return PEVSL_ERR_ARG; /* w must fit in shared memory */
  BGeom g;
  unsigned gx = geom(len, S, mask, 2, &g);
  for (int s = 0; s < S; s++)
    if (!g.nb[s]) g.nb[s] = 1;
  if (!gx) gx = 1;
  const size_t sh = sizeof(double) * (size_t)(k > 0 ? k : 1);
  static bool attr_done = false;
  if (!attr_done) {
    cudaFuncSetAttribute(k_b_gemv_sub_nrm, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
    attr_done = true;
  }
  k_b_gemv_sub_nrm<<<dim3(gx, S), kThreads, sh, ctx().stream>>>(g, k, V, w, ldw, v, ctx().red,
                                                                ctx().cnt, nrm, run, flag_out,
                                                                nrm_old, eta, mask);
  return launched("b_gemv_sub_nrm");
}

/* ---------------------------------------------------------------- single-vector forms */

int vdot(long n, const double *x, const double *y, double *out) {
  CPtrs a{}, b{};
  a.p[0] = x;
  b.p[0] = y;
  return b_dot(blen_uniform(n, n, 1), 1, a, b, out, FIN_ID, 1u);
}

int vnrm2(long n, const double *x, double *out) {
  CPtrs a{};
  a.p[0] = x;
  return b_dot(blen_uniform(n, n, 1), 1, a, a, out, FIN_SQRT, 1u);
}

int vaxpy_dev_nrm2(long n, const double *coef, const double *x, double *y, double *nrm) {
  CPtrs a{};
  VPtrs b{};
  a.p[0] = x;
  b.p[0] = y;
  return b_axpy_dev_nrm2(blen_uniform(n, n, 1), 1, coef, a, b, nrm, 1u);
}

int gemvT(long n, int k, const double *V, long ldv, const double *v, double *w, const int *run) {
  CPtrs a{}, b{};
  a.p[0] = V;
  b.p[0] = v;
  return b_gemvT(blen_uniform(n, ldv, 1), 1, k, a, b, w, 0, run, 1u);
}

int gemv_sub_nrm(long n, int k, const double *V, long ldv, const double *w, double *v, double *nrm,
                 const int *run, int *flag_out, double *nrm_old, double eta) {
  CPtrs a{};
  VPtrs b{};
  a.p[0] = V;
  b.p[0] = v;
  return b_gemv_sub_nrm(blen_uniform(n, ldv, 1), 1, k, a, w, 0, b, nrm, run, flag_out, nrm_old,
                        eta, 1u);
}

}  // namespace pv
