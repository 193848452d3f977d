/*
 * Device-side helpers shared by the CUDA modules: fixed-tree warp/block
 * sums, the last-block reduction used by every deterministic reduction, and
 * the Chebyshev recurrence epilogue with explicit rounding so that every
 * kernel that applies it (single vector or batched) gives identical bits.
 */
#ifndef PEVSL_B200_GPU_DEVICE_CUH
#define PEVSL_B200_GPU_DEVICE_CUH

#include <cuda_runtime.h>

namespace pv {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

/* Sum over the block with a fixed tree; valid in thread 0.  sh needs one
 * double per warp. */
__device__ __forceinline__ double block_sum(double v, double *sh) {
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  v = warp_sum(v);
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  v = (int)threadIdx.x < nw ? sh[threadIdx.x] : 0.0;
  if (w == 0) v = warp_sum(v);
  return v;
}

enum Fin { FIN_ID = 0, FIN_SQRT = 1 };

/* Deterministic grid reduction over gridDim.x blocks: this block's partial
 * goes to partials[blockIdx.x]; the last block to arrive (atomic ticket on
 * *counter) adds all partials in block order, applies fin, and returns the
 * total in thread 0 with *is_last set.  *counter is reset for reuse. */
__device__ __forceinline__ double grid_sum(double part, double *partials, unsigned *counter,
                                           int fin, bool *is_last) {
  __shared__ double sh[32];
  __shared__ bool am_last;
  const double s = block_sum(part, sh);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = s;
    __threadfence();
    am_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  *is_last = am_last;
  if (!am_last) return 0.0;
  __threadfence();
  double t = 0.0;
  for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x) t += __ldcg(partials + i);
  t = block_sum(t, sh);
  if (threadIdx.x == 0) *counter = 0;
  return fin == FIN_SQRT ? sqrt(t) : t;
}

/* One Chebyshev filter degree for one row (SRC/chebpol.c:549-559):
 *   w = (A v_k - cc v_k) t - v_{k-1};  y = first ? mu0 v_k + muk w : y + muk w
 * rounded as fma(-cc, x, r) * t, then subtractions and fma for y. */
__device__ __forceinline__ void cheb_update(double r, double x, const double *xm1, double cc,
                                            double t, double mu0, double muk, bool first,
                                            double *w_out, double *y) {
  double w = __dmul_rn(__fma_rn(-cc, x, r), t);
  if (xm1) w = __dsub_rn(w, *xm1);
  *w_out = w;
  *y = first ? __fma_rn(muk, w, __dmul_rn(mu0, x)) : __fma_rn(muk, w, *y);
}

/* cheb_update on values already loaded (xm1 used only when has_m1) */
__device__ __forceinline__ void cheb_update_v(double r, double x, double xm1, bool has_m1,
                                              double cc, double t, double mu0, double muk,
                                              bool first, double yold, double *w_out,
                                              double *y) {
  double w = __dmul_rn(__fma_rn(-cc, x, r), t);
  if (has_m1) w = __dsub_rn(w, xm1);
  *w_out = w;
  *y = first ? __fma_rn(muk, w, __dmul_rn(mu0, x)) : __fma_rn(muk, w, yold);
}

}  // namespace pv

#endif
