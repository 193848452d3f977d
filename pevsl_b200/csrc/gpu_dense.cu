/*
 * Dense kernels over the Lanczos basis V (n x k, column major, leading
 * dimension ldv):
 *
 *  - gemvT + gemv_sub_nrm: one classical Gram-Schmidt pass of CGS_DGKS
 *    (SRC/miscla.c:211-240 via SRC/parvecs.c:93-136): w = V' v, then
 *    v -= V w with ||v|| fused in; the DGKS decision whether a second pass
 *    runs is taken on the device (a flag the next pass reads), so no host
 *    round trip sits between the passes.  Both are HBM-bound (16 n k bytes
 *    per pass, 0.25 flop/byte).
 *  - gemm_nn: Ritz vectors U = V(:,0:k) Y (SRC/cheblanNr.c:363-365 does one
 *    GEMV per Ritz vector; here one pass over V serves 8 of them).
 */
#include <cuda_runtime.h>

#include "gpu.cuh"

namespace pv {

__device__ __forceinline__ double warp_sum32(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

constexpr int kGemvtCols = 4; /* columns per warp in gemvT */

/* partial[rb*k + j] = sum_{i in row block rb} V[i + j*ldv] v[i] */
__global__ void __launch_bounds__(kThreads)
    k_gemvt_partial(long n, int k, const double *__restrict__ V, long ldv,
                    const double *__restrict__ v, double *__restrict__ partial, int rows,
                    const int *run) {
  if (run && *run == 0) return;
  extern __shared__ double vsh[];
  const long r0 = (long)blockIdx.x * rows;
  const int nr = (int)((n - r0) < rows ? (n - r0) : rows);
  for (int i = threadIdx.x; i < nr; i += blockDim.x) vsh[i] = v[r0 + i];
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int cbase = blockIdx.y * wpb * kGemvtCols;
#pragma unroll
  for (int q = 0; q < kGemvtCols; q++) {
    const int j = cbase + q * wpb + wib;
    if (j >= k) break;
    const double *col = V + (size_t)j * ldv + r0;
    double s = 0.0;
#pragma unroll 4
    for (int i = lane; i < nr; i += 32) s = fma(col[i], vsh[i], s);
    s = warp_sum32(s);
    if (lane == 0) partial[(size_t)blockIdx.x * k + j] = s;
  }
}

/* w[j] = sum_rb partial[rb*k + j], in row-block order */
__global__ void k_gemvt_reduce(int nrb, int k, const double *__restrict__ partial,
                               double *__restrict__ w, const int *run) {
  if (run && *run == 0) return;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < k; j += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < nrb; b++) s += partial[(size_t)b * k + j];
    w[j] = s;
  }
}

static int gemvt_rows(long n) { return n < (1L << 16) ? 256 : 1024; }

int gemvT(long n, int k, const double *V, long ldv, const double *v, double *w, const int *run) {
  if (k <= 0) return 0;
  const int rows = gemvt_rows(n);
  const long nrb = (n + rows - 1) / rows;
  double *part = (double *)ws(WS_PART, sizeof(double) * (size_t)nrb * (size_t)k);
  if (!part) return PEVSL_ERR_NOMEM;
  const int cols_per_block = (kThreads / 32) * kGemvtCols;
  dim3 g((unsigned)nrb, (unsigned)((k + cols_per_block - 1) / cols_per_block));
  k_gemvt_partial<<<g, kThreads, sizeof(double) * rows, ctx().stream>>>(n, k, V, ldv, v, part, rows,
                                                                         run);
  if (launched("gemvT_partial")) return PEVSL_ERR_CUDA;
  k_gemvt_reduce<<<(k + kThreads - 1) / kThreads, kThreads, 0, ctx().stream>>>((int)nrb, k, part, w,
                                                                              run);
  return launched("gemvT_reduce");
}

/* v -= V w (thread per row, w staged in shared memory), ||v|| with the
 * last-block reduction, then the DGKS flag for the next pass. */
__global__ void __launch_bounds__(kThreads)
    k_gemv_sub_nrm(long n, int k, const double *__restrict__ V, long ldv,
                   const double *__restrict__ w, double *__restrict__ v, double *partials,
                   unsigned *counter, double *nrm, const int *run, int *flag_out, double *nrm_old,
                   double eta) {
  if (run && *run == 0) return;
  extern __shared__ double wsh[];
  __shared__ double red[kThreads / 32];
  __shared__ bool am_last;
  for (int j = threadIdx.x; j < k; j += blockDim.x) wsh[j] = w[j];
  __syncthreads();
  double ss = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double *row = V + i;
    double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0, acc3 = 0.0;
    int j = 0;
    for (; j + 3 < k; j += 4) {
      acc0 = fma(row[(size_t)j * ldv], wsh[j], acc0);
      acc1 = fma(row[(size_t)(j + 1) * ldv], wsh[j + 1], acc1);
      acc2 = fma(row[(size_t)(j + 2) * ldv], wsh[j + 2], acc2);
      acc3 = fma(row[(size_t)(j + 3) * ldv], wsh[j + 3], acc3);
    }
    for (; j < k; j++) acc0 = fma(row[(size_t)j * ldv], wsh[j], acc0);
    const double nv = v[i] - ((acc0 + acc1) + (acc2 + acc3));
    v[i] = nv;
    ss = fma(nv, nv, ss);
  }
  /* block sum, then the last block adds the block partials in order */
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  ss = warp_sum32(ss);
  if (lane == 0) red[wib] = ss;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) t += red[q];
    partials[blockIdx.x] = t;
    __threadfence();
    am_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (unsigned b = 0; b < gridDim.x; b++) t += __ldcg(partials + b);
    const double nn = sqrt(t);
    *nrm = nn;
    if (flag_out) *flag_out = nn <= eta * *nrm_old ? 1 : 0;
    if (nrm_old) *nrm_old = nn;
    *counter = 0;
  }
}

int gemv_sub_nrm(long n, int k, const double *V, long ldv, const double *w, double *v, double *nrm,
                 const int *run, int *flag_out, double *nrm_old, double eta) {
  if (k > 12288) return PEVSL_ERR_ARG; /* w must fit in shared memory */
  const size_t sh = sizeof(double) * (size_t)(k > 0 ? k : 1);
  if (sh > 48 * 1024) {
    static bool attr_done = false;
    if (!attr_done) {
      cudaFuncSetAttribute(k_gemv_sub_nrm, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
      attr_done = true;
    }
  }
  k_gemv_sub_nrm<<<grid_for(n, 2), kThreads, sh, ctx().stream>>>(n, k, V, ldv, w, v, ctx().red,
                                                                  ctx().cnt, nrm, run, flag_out,
                                                                  nrm_old, eta);
  return launched("gemv_sub_nrm");
}

/* U[:, c0:c0+8] = V(:, 0:k) Y[:, c0:c0+8]; thread per row, Y tile in smem */
constexpr int kGemmTile = 8;
__global__ void __launch_bounds__(kThreads)
    k_gemm_nn(long n, int k, int m, const double *__restrict__ V, long ldv,
              const double *__restrict__ Y, long ldy, double *__restrict__ U, long ldu) {
  extern __shared__ double ysh[]; /* k x kGemmTile */
  const int c0 = blockIdx.y * kGemmTile;
  const int mc = m - c0 < kGemmTile ? m - c0 : kGemmTile;
  for (int t = threadIdx.x; t < k * kGemmTile; t += blockDim.x) {
    const int j = t / kGemmTile, c = t % kGemmTile;
    ysh[t] = c < mc ? Y[(size_t)(c0 + c) * ldy + j] : 0.0;
  }
  __syncthreads();
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double acc[kGemmTile];
#pragma unroll
    for (int c = 0; c < kGemmTile; c++) acc[c] = 0.0;
    for (int j = 0; j < k; j++) {
      const double x = V[(size_t)j * ldv + i];
#pragma unroll
      for (int c = 0; c < kGemmTile; c++) acc[c] = fma(x, ysh[j * kGemmTile + c], acc[c]);
    }
#pragma unroll
    for (int c = 0; c < kGemmTile; c++)
      if (c < mc) U[(size_t)(c0 + c) * ldu + i] = acc[c];
  }
}

int gemm_nn(long n, int k, int m, const double *V, long ldv, const double *Y, long ldy, double *U,
            long ldu) {
  if (m <= 0 || n <= 0) return 0;
  const size_t sh = sizeof(double) * (size_t)k * kGemmTile;
  if (sh > 200 * 1024) return PEVSL_ERR_ARG;
  if (sh > 48 * 1024) {
    static bool attr_done = false;
    if (!attr_done) {
      cudaFuncSetAttribute(k_gemm_nn, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
      attr_done = true;
    }
  }
  dim3 g(grid_for(n, 1), (unsigned)((m + kGemmTile - 1) / kGemmTile));
  k_gemm_nn<<<g, kThreads, sh, ctx().stream>>>(n, k, m, V, ldv, Y, ldy, U, ldu);
  return launched("gemm_nn");
}

}  // namespace pv
