/*
 * Dense kernels over the Lanczos basis V (n x k, column major, leading
 * dimension ldv), on the FP64 tensor cores (mma.sync m8n8k4 .f64); the
 * Gram-Schmidt passes live in gpu_batch.cu.
 *
 *  - gemm_nn: Ritz vectors U = V(:,0:k) Y (SRC/cheblanNr.c:363-365 does one
 *    GEMV per Ritz vector; here one pass over V serves 64 of them).
 *  - gemm_tn: Gram matrices C = V' W of the refinement sweep.
 */
#include <cuda_runtime.h>

#include "gpu.cuh"

namespace pv {

/* FP64 tensor-core product (DMMA): D = A B + C for an 8 x 4 tile of A and a
 * 4 x 8 tile of B.  Fragments per lane l: a = A[l / 4][l % 4],
 * b = B[l % 4][l / 4], c/d = C[l / 4][2 (l % 4) + {0, 1}]. */
__device__ __forceinline__ void dmma_8x8x4(double a, double b, double &c0, double &c1) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

/* U = V(:, 0:k) Y on the FP64 tensor cores: a block owns a 64 x 64 tile of
 * U (64 rows, 64 Ritz vectors) and walks k in panels of 16 columns of V,
 * staged in shared memory with the matching 16 rows of Y; each of the 8
 * warps accumulates 8 of the tile's 8 x 8 sub-tiles (warp w: sub-tile rows
 * w, sub-tile columns 0..7).  V is read m / 64 times instead of once per
 * eight Ritz vectors.  (SRC/cheblanNr.c:363-365 forms the Ritz vectors one
 * GEMV each.) */
constexpr int kNnTile = 64, kNnPanel = 16;
__global__ void __launch_bounds__(kThreads)
    k_gemm_nn_dmma(long n, int k, int m, const double *__restrict__ V, long ldv,
                   const double *__restrict__ Y, long ldy, double *__restrict__ U, long ldu) {
  __shared__ double vs[kNnPanel][kNnTile + 1]; /* vs[jj][i] = V[i0 + i, j + jj] */
  __shared__ double ys[kNnPanel][kNnTile + 1]; /* ys[jj][c] = Y[j + jj, c0 + c] */
  const long i0 = (long)blockIdx.x * kNnTile;
  const int c0 = blockIdx.y * kNnTile;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lr = lane >> 2, lc = lane & 3;
  double acc[8][2];
#pragma unroll
  for (int t = 0; t < 8; t++) acc[t][0] = acc[t][1] = 0.0;
  for (int j = 0; j < k; j += kNnPanel) {
    /* 64 rows x 16 columns of V (a column's 64 rows are contiguous) and 16
     * rows x 64 columns of Y, zero outside */
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int t = threadIdx.x + kThreads * q;
      const int i = t & 63, jj = t >> 6;
      const long row = i0 + i;
      vs[jj][i] = (row < n && j + jj < k) ? V[(size_t)(j + jj) * ldv + row] : 0.0;
      const int c = t >> 4, yj = t & 15;
      ys[yj][c] = (c0 + c < m && j + yj < k) ? Y[(size_t)(c0 + c) * ldy + j + yj] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kNnPanel; kk += 4) {
      const double a = vs[kk + lc][warp * 8 + lr];
#pragma unroll
      for (int t = 0; t < 8; t++) dmma_8x8x4(a, ys[kk + lc][t * 8 + lr], acc[t][0], acc[t][1]);
    }
    __syncthreads();
  }
  const long row = i0 + warp * 8 + lr;
  if (row < n) {
#pragma unroll
    for (int t = 0; t < 8; t++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int c = c0 + t * 8 + 2 * lc + h;
        if (c < m) U[(size_t)c * ldu + row] = acc[t][h];
      }
  }
}

int gemm_nn(long n, int k, int m, const double *V, long ldv, const double *Y, long ldy, double *U,
            long ldu) {
  if (m <= 0 || n <= 0) return 0;
  dim3 g((unsigned)((n + kNnTile - 1) / kNnTile), (unsigned)((m + kNnTile - 1) / kNnTile));
  k_gemm_nn_dmma<<<g, kThreads, 0, ctx().stream>>>(n, k, m, V, ldv, Y, ldy, U, ldu);
  return launched("gemm_nn_dmma");
}

/* C = V' W for tall V (n x k) and W (n x m) on the FP64 tensor cores: a
 * block owns a 64 x 64 tile of C and one chunk of rows; it stages 16 rows of
 * the two 64-column panels in shared memory, and each of the 8 warps
 * accumulates 8 of the tile's 8 x 8 sub-tiles (sub-tile row = warp) with
 * m8n8k4 DMMA over the panel's rows.  Per-chunk tiles go to partial[chunk],
 * then k_gemm_tn_reduce adds them in chunk order (deterministic).  These are
 * the block Gram products of the refinement sweep, the dense counterpart of
 * the reference's GemtvWithWspace (SRC/parvecs.c:117-136). */
constexpr int kTnTile = 64, kTnRows = 16;
__global__ void __launch_bounds__(kThreads)
    k_gemm_tn_partial(long n, int k, int m, const double *__restrict__ V, long ldv,
                      const double *__restrict__ W, long ldw, long rows_per_chunk,
                      double *__restrict__ partial) {
  __shared__ double vs[kTnRows][kTnTile + 1], wsh[kTnRows][kTnTile + 1];
  const int ti = blockIdx.x, tj = blockIdx.y;
  const long r_beg = (long)blockIdx.z * rows_per_chunk;
  const long r_end = r_beg + rows_per_chunk < n ? r_beg + rows_per_chunk : n;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lr = lane >> 2, lc = lane & 3;
  double acc[8][2];
#pragma unroll
  for (int t = 0; t < 8; t++) acc[t][0] = acc[t][1] = 0.0;
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
    /* A = V' (rows: columns of V, k: rows of the panel), B = W panel */
#pragma unroll
    for (int kk = 0; kk < kTnRows; kk += 4) {
      const double a = vs[kk + lc][warp * 8 + lr];
#pragma unroll
      for (int t = 0; t < 8; t++) dmma_8x8x4(a, wsh[kk + lc][t * 8 + lr], acc[t][0], acc[t][1]);
    }
    __syncthreads();
  }
  double *out = partial + (size_t)blockIdx.z * (size_t)k * (size_t)m;
  const int ci = ti * kTnTile + warp * 8 + lr;
  if (ci < k) {
#pragma unroll
    for (int t = 0; t < 8; t++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int cj = tj * kTnTile + t * 8 + 2 * lc + h;
        if (cj < m) out[(size_t)cj * k + ci] = acc[t][h];
      }
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

extern "C" {

int pEVSL_B200_GemmNN(long n, int k, int m, const double *V, long ldv, const double *Y, long ldy,
                      double *U, long ldu) {
  if (pv::ensure()) return PEVSL_ERR_CUDA;
  if (n < 0 || k < 0 || m < 0 || ldv < n || ldu < n || ldy < k) return PEVSL_ERR_ARG;
  return pv::gemm_nn(n, k, m, V, ldv, Y, ldy, U, ldu);
}

int pEVSL_B200_GemmTN(long n, int k, int m, const double *V, long ldv, const double *W, long ldw,
                      double *C, long ldc) {
  if (pv::ensure()) return PEVSL_ERR_CUDA;
  if (n < 0 || k < 0 || m < 0 || ldv < n || ldw < n || ldc < k) return PEVSL_ERR_ARG;
  return pv::gemm_tn(n, k, m, V, ldv, W, ldw, C, ldc);
}

}  // extern "C"
