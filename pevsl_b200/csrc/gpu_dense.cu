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

}  // namespace pv
