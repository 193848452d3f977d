/*
 * Dense kernel over the Lanczos basis V (n x k, column major, leading
 * dimension ldv); the Gram-Schmidt passes live in gpu_batch.cu.
 *
 *  - gemm_nn: Ritz vectors U = V(:,0:k) Y (SRC/cheblanNr.c:363-365 does one
 *    GEMV per Ritz vector; here one pass over V serves 8 of them).
 */
#include <cuda_runtime.h>

#include "gpu.cuh"

namespace pv {

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

/* C = V' W for tall V (n x k) and W (n x m): a block owns a 64 x 64 tile
 * of C and one chunk of rows; it stages 16 rows of the two 64-column
 * panels in shared memory and each thread accumulates a 4 x 4 subtile
 * (rows ty + 16 i, columns tx + 16 j, conflict-free).  Per-chunk tiles go
 * to partial[chunk], then k_gemm_tn_reduce adds them in chunk order. */
constexpr int kTnTile = 64, kTnRows = 16;
__global__ void __launch_bounds__(kThreads)
    k_gemm_tn_partial(long n, int k, int m, const double *__restrict__ V, long ldv,
                      const double *__restrict__ W, long ldw, long rows_per_chunk,
                      double *__restrict__ partial) {
  __shared__ double vs[kTnRows][kTnTile + 1], wsh[kTnRows][kTnTile + 1];
  const int ti = blockIdx.x, tj = blockIdx.y;
  const long r_beg = (long)blockIdx.z * rows_per_chunk;
  const long r_end = r_beg + rows_per_chunk < n ? r_beg + rows_per_chunk : n;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = 0.0;
  for (long r0 = r_beg; r0 < r_end; r0 += kTnRows) {
    /* 16 rows x 64 columns of each panel: thread t loads row t % 16 of
     * columns t / 16 + 16 q (16 consecutive rows of a column per half-warp) */
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int r = threadIdx.x & 15, c = (threadIdx.x >> 4) + 16 * q;
      const long row = r0 + r;
      const int cv = ti * kTnTile + c, cw = tj * kTnTile + c;
      vs[r][c] = (row < r_end && cv < k) ? V[(size_t)cv * ldv + row] : 0.0;
      wsh[r][c] = (row < r_end && cw < m) ? W[(size_t)cw * ldw + row] : 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int r = 0; r < kTnRows; r++) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = vs[r][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = wsh[r][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
  double *out = partial + (size_t)blockIdx.z * (size_t)k * (size_t)m;
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int ci = ti * kTnTile + ty + 16 * i, cj = tj * kTnTile + tx + 16 * j;
      if (ci < k && cj < m) out[(size_t)cj * k + ci] = acc[i][j];
    }
}

__global__ void k_gemm_tn_reduce(int k, int m, int nchunk, const double *__restrict__ partial,
                                 double *__restrict__ C, long ldc) {
  const long tot = (long)k * m;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int c = 0; c < nchunk; c++) s += partial[(size_t)c * tot + t];
    C[(t / k) * ldc + t % k] = s;
  }
}

int gemm_tn(long n, int k, int m, const double *V, long ldv, const double *W, long ldw, double *C,
            long ldc) {
  if (k <= 0 || m <= 0) return 0;
  const int tk = (k + kTnTile - 1) / kTnTile, tm = (m + kTnTile - 1) / kTnTile;
  /* enough row chunks for about four blocks per SM, at least 1024 rows each */
  long nchunk = (4L * 148 + tk * tm - 1) / (tk * tm);
  const long max_chunks = (n + 1023) / 1024;
  if (nchunk > max_chunks) nchunk = max_chunks;
  if (nchunk < 1) nchunk = 1;
  long rows = (n + nchunk - 1) / nchunk;
  rows = (rows + kTnRows - 1) / kTnRows * kTnRows;
  nchunk = n > 0 ? (n + rows - 1) / rows : 1;
  double *part = (double *)ws(WS_GEMM, sizeof(double) * (size_t)nchunk * (size_t)k * (size_t)m);
  if (!part) return PEVSL_ERR_NOMEM;
  dim3 g((unsigned)tk, (unsigned)tm, (unsigned)nchunk);
  k_gemm_tn_partial<<<g, kThreads, 0, ctx().stream>>>(n, k, m, V, ldv, W, ldw, rows, part);
  if (launched("gemm_tn_partial")) return PEVSL_ERR_CUDA;
  k_gemm_tn_reduce<<<grid_for((long)k * m, 1), kThreads, 0, ctx().stream>>>(k, m, (int)nchunk, part,
                                                                            C, ldc);
  return launched("gemm_tn_reduce");
}

}  // namespace pv
