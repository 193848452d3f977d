/*
 * FP32 kernels of the mixed-precision form: the Chebyshev filter and the KPM
 * moments run on FP32 matrix values and FP32 vectors with FP32 accumulation,
 * halving the bytes per degree; the Lanczos basis, reorthogonalisation,
 * tridiagonal solves, Ritz vectors and residuals stay FP64 (gpu_solvers.cu).
 *
 *   kpm_step32     one KPM degree (SRC/kpmdos.c:129-156) for s <= 64
 *                  row-interleaved FP32 vectors with the moment dots fused
 *
 * The FP32 filter degree is the fp32 form of cheb_step_batch (gpu_sparse.cu).
 */
#include <cuda_runtime.h>

#include "gpu.cuh"
#include "gpu_device.cuh"

namespace pv {

__global__ void k_cvt_f64_f32(long n, const double *__restrict__ x, float *__restrict__ y) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    y[i] = (float)x[i];
}

int csr_make_fp32(pevsl_devcsr *A) {
  if (A->a32) return 0;
  float *p = nullptr;
  if (fail(cudaMalloc(&p, sizeof(float) * (size_t)(A->nnz > 0 ? A->nnz : 1)), "cudaMalloc a32"))
    return PEVSL_ERR_NOMEM;
  k_cvt_f64_f32<<<grid_for(A->nnz, 4), kThreads, 0, ctx().stream>>>(A->nnz, A->a, p);
  if (launched("cvt_f64_f32")) {
    cudaFree(p);
    return PEVSL_ERR_CUDA;
  }
  A->a32 = p;
  return 0;
}

/* FP32 KPM degree for s <= 32*CPL interleaved vectors (warp per row); the
 * per-block moment partials are FP32 sums, added across blocks in FP64. */
template <int CPL>
__global__ void __launch_bounds__(kThreads)
    k_kpm_step32(int n, int s, int ld, const int *__restrict__ ia, const int *__restrict__ ja,
                 const float *__restrict__ a, const float *__restrict__ Xk,
                 const float *__restrict__ Xkm1, float *__restrict__ Xkp1,
                 const float *__restrict__ V0, float ctr, float sc, double *partials,
                 unsigned *counter, double *mom) {
  __shared__ float acc_sh[kThreads / 32][32 * CPL];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  float acc[CPL];
#pragma unroll
  for (int q = 0; q < CPL; q++) acc[q] = 0.f;
  for (int row = blockIdx.x * wpb + wib; row < n; row += gridDim.x * wpb) {
    float r[CPL];
#pragma unroll
    for (int q = 0; q < CPL; q++) r[q] = 0.f;
    const int e = ia[row + 1];
    int j = ia[row];
    for (; j + 3 < e; j += 4) {
      const float a0 = a[j], a1 = a[j + 1], a2 = a[j + 2], a3 = a[j + 3];
      const float *x0 = Xk + (size_t)ja[j] * ld, *x1 = Xk + (size_t)ja[j + 1] * ld;
      const float *x2 = Xk + (size_t)ja[j + 2] * ld, *x3 = Xk + (size_t)ja[j + 3] * ld;
#pragma unroll
      for (int q = 0; q < CPL; q++) {
        const int c = lane + 32 * q;
        if (c < s) r[q] = fmaf(a3, x3[c], fmaf(a2, x2[c], fmaf(a1, x1[c], fmaf(a0, x0[c], r[q]))));
      }
    }
    for (; j < e; j++) {
      const float aj = a[j];
      const float *xr = Xk + (size_t)ja[j] * ld;
#pragma unroll
      for (int q = 0; q < CPL; q++) {
        const int c = lane + 32 * q;
        if (c < s) r[q] = fmaf(aj, xr[c], r[q]);
      }
    }
    const size_t base = (size_t)row * ld;
#pragma unroll
    for (int q = 0; q < CPL; q++) {
      const int c = lane + 32 * q;
      if (c < s) {
        float w = (r[q] - ctr * Xk[base + c]) * sc;
        if (Xkm1) w -= Xkm1[base + c];
        Xkp1[base + c] = w;
        acc[q] = fmaf(w, V0[base + c], acc[q]);
      }
    }
  }
#pragma unroll
  for (int q = 0; q < CPL; q++) acc_sh[wib][lane + 32 * q] = acc[q];
  __syncthreads();
  for (int c = threadIdx.x; c < s; c += blockDim.x) {
    float t = 0.f;
    for (int w = 0; w < wpb; w++) t += acc_sh[w][c];
    partials[(size_t)blockIdx.x * s + c] = (double)t;
  }
  /* the columns are added across blocks by k_col_reduce */
  (void)counter;
}

int kpm_step32(const pevsl_devcsr *A, int s, int ld, const float *Xk, const float *Xkm1,
               float *Xkp1, const float *V0, double ctr, double sc, double *mom) {
  if (s < 1 || s > 64 || !A->a32) return PEVSL_ERR_ARG;
  const long wpb = kThreads / 32;
  long g = (A->nrows + wpb - 1) / wpb;
  if (g > kMaxRedBlocks) g = kMaxRedBlocks;
  if (g < 1) g = 1;
  if (s <= 32) {
    k_kpm_step32<1><<<(unsigned)g, kThreads, 0, ctx().stream>>>(A->nrows, s, ld, A->ia, A->ja, A->a32, Xk, Xkm1, Xkp1, V0, (float)ctr, (float)sc, ctx().red, ctx().cnt, mom);
  } else {
    k_kpm_step32<2><<<(unsigned)g, kThreads, 0, ctx().stream>>>(A->nrows, s, ld, A->ia, A->ja, A->a32, Xk, Xkm1, Xkp1, V0, (float)ctr, (float)sc, ctx().red, ctx().cnt, mom);
  }
  if (launched("kpm_step32")) return PEVSL_ERR_CUDA;
  return col_reduce(ctx().red, (int)g, s, mom);
}

/* y = (float) x for an interleaved block */
int cvt_f64_f32(long n, const double *x, float *y) {
  if (n <= 0) return 0;
  k_cvt_f64_f32<<<grid_for(n, 4), kThreads, 0, ctx().stream>>>(n, x, y);
  return launched("cvt_f64_f32");
}

}  // namespace pv
