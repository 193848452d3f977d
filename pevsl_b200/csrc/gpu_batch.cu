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
 * The batched filter degree is cheb_step_batch (gpu_sparse.cu).
 */
#include <cuda_runtime.h>

#include "gpu.cuh"
#include "gpu_device.cuh"

namespace pv {

#define PV_ACTIVE(mask, s) (((mask) >> (s)) & 1u)

/* ---------------------------------------------------------------- level 1 */

__global__ void k_b_axpy(long n, CPtrs x, VPtrs y, BScal a, unsigned mask) {
  const int s = blockIdx.y;
  if (!PV_ACTIVE(mask, s)) return;
  const double c = a.v[s];
  const double *xs = x.p[s];
  double *ys = y.p[s];
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    ys[i] += c * xs[i];
}

__global__ void k_b_scal(long n, VPtrs x, BScal a, unsigned mask) {
  const int s = blockIdx.y;
  if (!PV_ACTIVE(mask, s)) return;
  const double c = a.v[s];
  double *xs = x.p[s];
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    xs[i] *= c;
}

__global__ void k_b_dot(long n, CPtrs x, CPtrs y, double *partials, unsigned *counters, double *out,
                        int fin, unsigned mask) {
  const int s = blockIdx.y;
  if (!PV_ACTIVE(mask, s)) return;
  const double *xs = x.p[s], *ys = y.p[s];
  double acc = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    acc += xs[i] * ys[i];
  bool last;
  const double t = grid_sum(acc, partials + (size_t)s * kMaxRedBlocks, counters + s, fin, &last);
  if (last && threadIdx.x == 0) out[s] = t;
}

/* y -= coef[s] x, then ||y|| */
__global__ void k_b_axpy_dev_nrm2(long n, const double *coef, CPtrs x, VPtrs y, double *partials,
                                  unsigned *counters, double *nrm, unsigned mask) {
  const int s = blockIdx.y;
  if (!PV_ACTIVE(mask, s)) return;
  const double a = -coef[s];
  const double *xs = x.p[s];
  double *ys = y.p[s];
  double acc = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double v = ys[i] + a * xs[i];
    ys[i] = v;
    acc += v * v;
  }
  bool last;
  const double t = grid_sum(acc, partials + (size_t)s * kMaxRedBlocks, counters + s, FIN_SQRT, &last);
  if (last && threadIdx.x == 0) nrm[s] = t;
}

/* ---------------------------------------------------------------- CGS pass */

constexpr int kGemvtCols = 4; /* columns per warp in gemvT */

static int gemvt_rows(long n) { return n < (1L << 16) ? 256 : 1024; }

/* partial[s][rb][j] = sum_{i in row block rb} V_s[i + j ldv] v_s[i] */
__global__ void __launch_bounds__(kThreads)
    k_b_gemvt_partial(long n, int k, CPtrs V, long ldv, CPtrs v, double *__restrict__ partial,
                      long nrb, int rows, const int *run, unsigned mask) {
  const int s = blockIdx.z;
  if (!PV_ACTIVE(mask, s) || (run && run[s] == 0)) return;
  extern __shared__ double vsh[];
  const long r0 = (long)blockIdx.x * rows;
  const int nr = (int)((n - r0) < rows ? (n - r0) : rows);
  const double *vs = v.p[s];
  for (int i = threadIdx.x; i < nr; i += blockDim.x) vsh[i] = vs[r0 + i];
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int cbase = blockIdx.y * wpb * kGemvtCols;
  double *ps = partial + (size_t)s * nrb * k;
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
__global__ void k_b_gemvt_reduce(int nrb, int k, const double *__restrict__ partial,
                                 double *__restrict__ w, long ldw, const int *run, unsigned mask) {
  const int s = blockIdx.y;
  if (!PV_ACTIVE(mask, s) || (run && run[s] == 0)) return;
  const double *ps = partial + (size_t)s * nrb * k;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < k; j += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int b = 0; b < nrb; b++) acc += ps[(size_t)b * k + j];
    w[(size_t)s * ldw + j] = acc;
  }
}

/* v_s -= V_s w_s (thread per row, w_s in shared memory), ||v_s||, and the
 * DGKS flag for the next pass: flag[s] = ||v_s|| <= eta * nrm_old[s]. */
__global__ void __launch_bounds__(kThreads)
    k_b_gemv_sub_nrm(long n, int k, CPtrs V, long ldv, const double *__restrict__ w, long ldw,
                     VPtrs v, double *partials, unsigned *counters, double *nrm, const int *run,
                     int *flag_out, double *nrm_old, double eta, unsigned mask) {
  const int s = blockIdx.y;
  if (!PV_ACTIVE(mask, s) || (run && run[s] == 0)) return;
  extern __shared__ double wsh[];
  for (int j = threadIdx.x; j < k; j += blockDim.x) wsh[j] = w[(size_t)s * ldw + j];
  __syncthreads();
  const double *Vs = V.p[s];
  double *vs = v.p[s];
  double ss = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
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
  const double t = grid_sum(ss, partials + (size_t)s * kMaxRedBlocks, counters + s, FIN_SQRT, &last);
  if (last && threadIdx.x == 0) {
    nrm[s] = t;
    if (flag_out) flag_out[s] = t <= eta * nrm_old[s] ? 1 : 0;
    if (nrm_old) nrm_old[s] = t;
  }
}


/* ---------------------------------------------------------------- host wrappers */

static unsigned col_grid(long n, int per_thread) { return grid_for(n, per_thread); }

int b_axpy(long n, int S, CPtrs x, VPtrs y, BScal a, unsigned mask) {
  if (n <= 0 || !mask) return 0;
  dim3 g(col_grid(n, 4), S);
  k_b_axpy<<<g, kThreads, 0, ctx().stream>>>(n, x, y, a, mask);
  return launched("b_axpy");
}

int b_scal(long n, int S, VPtrs x, BScal a, unsigned mask) {
  if (n <= 0 || !mask) return 0;
  dim3 g(col_grid(n, 4), S);
  k_b_scal<<<g, kThreads, 0, ctx().stream>>>(n, x, a, mask);
  return launched("b_scal");
}

int b_dot(long n, int S, CPtrs x, CPtrs y, double *out, int fin, unsigned mask) {
  if (!mask) return 0;
  dim3 g(col_grid(n, 4), S);
  k_b_dot<<<g, kThreads, 0, ctx().stream>>>(n, x, y, ctx().red, ctx().cnt, out, fin, mask);
  return launched("b_dot");
}

int b_axpy_dev_nrm2(long n, int S, const double *coef, CPtrs x, VPtrs y, double *nrm,
                    unsigned mask) {
  if (!mask) return 0;
  dim3 g(col_grid(n, 4), S);
  k_b_axpy_dev_nrm2<<<g, kThreads, 0, ctx().stream>>>(n, coef, x, y, ctx().red, ctx().cnt, nrm,
                                                      mask);
  return launched("b_axpy_dev_nrm2");
}

int b_gemvT(long n, int S, int k, CPtrs V, long ldv, CPtrs v, double *w, long ldw, const int *run,
            unsigned mask) {
  if (k <= 0 || !mask) return 0;
  const int rows = gemvt_rows(n);
  const long nrb = (n + rows - 1) / rows;
  double *part = (double *)ws(WS_PART, sizeof(double) * (size_t)S * (size_t)nrb * (size_t)k);
  if (!part) return PEVSL_ERR_NOMEM;
  const int cols_per_block = (kThreads / 32) * kGemvtCols;
  dim3 g((unsigned)nrb, (unsigned)((k + cols_per_block - 1) / cols_per_block), S);
  k_b_gemvt_partial<<<g, kThreads, sizeof(double) * rows, ctx().stream>>>(n, k, V, ldv, v, part, nrb,
                                                                           rows, run, mask);
  if (launched("b_gemvT_partial")) return PEVSL_ERR_CUDA;
  dim3 g2((unsigned)((k + kThreads - 1) / kThreads), S);
  k_b_gemvt_reduce<<<g2, kThreads, 0, ctx().stream>>>((int)nrb, k, part, w, ldw, run, mask);
  return launched("b_gemvT_reduce");
}

int b_gemv_sub_nrm(long n, int S, int k, CPtrs V, long ldv, const double *w, long ldw, VPtrs v,
                   double *nrm, const int *run, int *flag_out, double *nrm_old, double eta,
                   unsigned mask) {
  if (!mask) return 0;
  if (k > 12288) return PEVSL_ERR_ARG; /* w must fit in shared memory */
  const size_t sh = sizeof(double) * (size_t)(k > 0 ? k : 1);
  static bool attr_done = false;
  if (!attr_done) {
    cudaFuncSetAttribute(k_b_gemv_sub_nrm, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
    attr_done = true;
  }
  dim3 g(grid_for(n, 2), S);
  k_b_gemv_sub_nrm<<<g, kThreads, sh, ctx().stream>>>(n, k, V, ldv, w, ldw, v, ctx().red, ctx().cnt,
                                                      nrm, run, flag_out, nrm_old, eta, mask);
  return launched("b_gemv_sub_nrm");
}

/* ---------------------------------------------------------------- single-vector forms */

int vdot(long n, const double *x, const double *y, double *out) {
  CPtrs a{}, b{};
  a.p[0] = x;
  b.p[0] = y;
  return b_dot(n, 1, a, b, out, FIN_ID, 1u);
}

int vnrm2(long n, const double *x, double *out) {
  CPtrs a{};
  a.p[0] = x;
  return b_dot(n, 1, a, a, out, FIN_SQRT, 1u);
}

int vaxpy_dev_nrm2(long n, const double *coef, const double *x, double *y, double *nrm) {
  CPtrs a{};
  VPtrs b{};
  a.p[0] = x;
  b.p[0] = y;
  return b_axpy_dev_nrm2(n, 1, coef, a, b, nrm, 1u);
}

int gemvT(long n, int k, const double *V, long ldv, const double *v, double *w, const int *run) {
  CPtrs a{}, b{};
  a.p[0] = V;
  b.p[0] = v;
  return b_gemvT(n, 1, k, a, ldv, b, w, 0, run, 1u);
}

int gemv_sub_nrm(long n, int k, const double *V, long ldv, const double *w, double *v, double *nrm,
                 const int *run, int *flag_out, double *nrm_old, double eta) {
  CPtrs a{};
  VPtrs b{};
  a.p[0] = V;
  b.p[0] = v;
  return b_gemv_sub_nrm(n, 1, k, a, ldv, w, 0, b, nrm, run, flag_out, nrm_old, eta, 1u);
}

}  // namespace pv
