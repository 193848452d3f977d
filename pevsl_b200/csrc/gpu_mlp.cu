/*
 * Learned density of states: a small MLP (BF16 weights and activations,
 * FP32 accumulation and master weights) that maps KPM moments estimated from
 * a few random vectors to the moments of many vectors.  Training and
 * inference run on this file's kernels:
 *
 *   k_gemm_bf16   C = op(A) op(B) on the tensor cores (warp-level
 *                 mma.sync m16n8k16, BF16 inputs, FP32 accumulators), 64x64
 *                 tiles, operands staged in shared memory (either operand
 *                 may be transposed while staging), with fused epilogues:
 *                 bias + GELU (forward), bias (output layer), GELU'
 *                 (backward through an activation), plain store (weight
 *                 gradients);
 *   k_mse         dY = 2 (Y - T) / (B * nout) on the real outputs, and the
 *                 loss (deterministic block-ordered sum);
 *   k_colsum      bias gradients (column sums in row order);
 *   k_adam        Adam on the FP32 master weights, then the BF16 copies.
 *
 * Layer l maps K_l inputs to N_l outputs (dimensions padded to multiples of
 * 16 with zero weights); activations are row-major [batch][features].
 */
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gpu.cuh"

namespace pv {

typedef __nv_bfloat16 bf16;

constexpr int kGT = 64;    /* block tile (M and N) */
constexpr int kGK = 16;    /* K step = mma k */
constexpr int kGPad = 24;  /* shared row stride in bf16 (48 bytes): conflict-light, 4-byte aligned */

enum { EPI_STORE = 0, EPI_BIAS = 1, EPI_BIAS_GELU = 2, EPI_DGELU = 3 };

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
  return cdf + z * pdf;
}

__device__ __forceinline__ void mma_bf16_16816(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

/* C[m][n] = sum_k A'(m,k) B'(k,n) for m < M, n < N, with
 * A'(m,k) = TA ? A[k*lda + m] : A[m*lda + k] and
 * B'(k,n) = TB ? B[n*ldb + k] : B[k*ldb + n]; out-of-range elements are 0.
 * 128 threads: warp w owns rows 32*(w/2) .. +32 and columns 32*(w%2) .. +32
 * of the 64x64 tile, as 2 x 4 tiles of 16x8.  Epilogue (row m, column n):
 *   EPI_STORE      C = acc
 *   EPI_BIAS       C = acc + bias[n]
 *   EPI_BIAS_GELU  C = z = acc + bias[n];  act = bf16(gelu(z))
 *   EPI_DGELU      C = g = acc * gelu'(zp[m][n]);  act = bf16(g) */
template <bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(128)
    k_gemm_bf16(int M, int N, int K, const bf16 *__restrict__ A, int lda,
                const bf16 *__restrict__ B, int ldb, float *__restrict__ C, int ldc,
                const float *__restrict__ bias, bf16 *__restrict__ act, int ldact,
                const float *__restrict__ zp, int ldzp) {
  __shared__ __align__(16) bf16 As[kGT][kGPad];
  __shared__ __align__(16) bf16 Bs[kGT][kGPad]; /* [n][k] */
  const int m0 = blockIdx.y * kGT, n0 = blockIdx.x * kGT;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gid = lane >> 2, tig = lane & 3;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[i][j][q] = 0.f;
  const bf16 zero = __float2bfloat16(0.f);
  for (int k0 = 0; k0 < K; k0 += kGK) {
    /* stage 64 x 16 of A' and of B' (as [n][k]): 8 elements per thread each */
    for (int t = threadIdx.x; t < kGT * kGK; t += 128) {
      const int r = t / kGK, kk = t % kGK;
      const int m = m0 + r, n = n0 + r, k = k0 + kk;
      bf16 av = zero, bv = zero;
      if (m < M && k < K) av = TA ? A[(size_t)k * lda + m] : A[(size_t)m * lda + k];
      if (n < N && k < K) bv = TB ? B[(size_t)n * ldb + k] : B[(size_t)k * ldb + n];
      As[r][kk] = av;
      Bs[r][kk] = bv;
    }
    __syncthreads();
    uint32_t af[2][4], bfr[4][2];
#pragma unroll
    for (int i = 0; i < 2; i++) {
      const int r = wm + 16 * i + gid;
      af[i][0] = *reinterpret_cast<const uint32_t *>(&As[r][2 * tig]);
      af[i][1] = *reinterpret_cast<const uint32_t *>(&As[r + 8][2 * tig]);
      af[i][2] = *reinterpret_cast<const uint32_t *>(&As[r][2 * tig + 8]);
      af[i][3] = *reinterpret_cast<const uint32_t *>(&As[r + 8][2 * tig + 8]);
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int c = wn + 8 * j + gid;
      bfr[j][0] = *reinterpret_cast<const uint32_t *>(&Bs[c][2 * tig]);
      bfr[j][1] = *reinterpret_cast<const uint32_t *>(&Bs[c][2 * tig + 8]);
    }
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) mma_bf16_16816(acc[i][j], af[i], bfr[j]);
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int m = m0 + wm + 16 * i + gid + (q >= 2 ? 8 : 0);
        const int n = n0 + wn + 8 * j + 2 * tig + (q & 1);
        if (m >= M || n >= N) continue;
        float v = acc[i][j][q];
        if (EPI == EPI_BIAS || EPI == EPI_BIAS_GELU) v += bias[n];
        if (EPI == EPI_DGELU) v *= gelu_grad(zp[(size_t)m * ldzp + n]);
        C[(size_t)m * ldc + n] = v;
        if (EPI == EPI_BIAS_GELU) act[(size_t)m * ldact + n] = __float2bfloat16(gelu(v));
        if (EPI == EPI_DGELU) act[(size_t)m * ldact + n] = __float2bfloat16(v);
      }
}

/* dY = 2 (Y - T) / (B * nout) on columns < nout (0 elsewhere), bf16 copy,
 * and the mean squared error: per-block sums, the last block adds them in
 * block order */
__global__ void k_mse(int Bn, int ld, int nout, const float *__restrict__ Y,
                      const float *__restrict__ T, int ldt, float *__restrict__ dY,
                      bf16 *__restrict__ dYh, double *partials, unsigned *counter, float *loss) {
  __shared__ double sh[256];
  __shared__ bool am_last;
  const double scale = 2.0 / ((double)Bn * nout);
  double s = 0.0;
  const long tot = (long)Bn * ld;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < tot; i += (long)gridDim.x * blockDim.x) {
    const int m = (int)(i / ld), n = (int)(i % ld);
    float g = 0.f;
    if (n < nout) {
      const float d = Y[i] - T[(size_t)m * ldt + n];
      s += (double)d * d;
      g = (float)(scale * d);
    }
    dY[i] = g;
    dYh[i] = __float2bfloat16(g);
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = sh[0];
    __threadfence();
    am_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (am_last && threadIdx.x == 0) {
    __threadfence();
    double t = 0.0;
    for (unsigned b = 0; b < gridDim.x; b++) t += __ldcg(partials + b);
    *loss = (float)(t / ((double)Bn * nout));
    *counter = 0;
  }
}

/* db[n] = sum_m dZ[m][n], rows in order */
__global__ void k_colsum(int Bn, int N, const float *__restrict__ dZ, int ld, float *__restrict__ db) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.f;
  for (int m = 0; m < Bn; m++) s += dZ[(size_t)m * ld + n];
  db[n] = s;
}

/* Adam (Kingma & Ba, 2015) with bias correction on FP32 master weights;
 * entries with mask 0 (padding) stay 0 */
__global__ void k_adam(long np, float *__restrict__ p, const float *__restrict__ g,
                       float *__restrict__ m1, float *__restrict__ m2, const uint8_t *__restrict__ mask,
                       bf16 *__restrict__ ph, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < np; i += (long)gridDim.x * blockDim.x) {
    if (!mask[i]) {
      p[i] = 0.f;
      ph[i] = __float2bfloat16(0.f);
      continue;
    }
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.f - b1) * gi;
    const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    const float v = p[i] - lr * (a / c1) / (sqrtf(b / c2) + eps);
    p[i] = v;
    ph[i] = __float2bfloat16(v);
  }
}

__global__ void k_to_bf16(long n, const float *__restrict__ x, bf16 *__restrict__ y) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16(x[i]);
}

/* X [B][ld] (bf16, zero padding) from a row-major FP32 block [B][nin] */
__global__ void k_pack_input(int Bn, int nin, int ld, const float *__restrict__ x, bf16 *__restrict__ xh) {
  const long tot = (long)Bn * ld;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < tot; i += (long)gridDim.x * blockDim.x) {
    const int m = (int)(i / ld), n = (int)(i % ld);
    xh[i] = __float2bfloat16(n < nin ? x[(size_t)m * nin + n] : 0.f);
  }
}

template <bool TA, bool TB, int EPI>
static int gemm(int M, int N, int K, const bf16 *A, int lda, const bf16 *B, int ldb, float *C, int ldc,
                const float *bias, bf16 *act, int ldact, const float *zp, int ldzp) {
  if (M <= 0 || N <= 0) return 0;
  dim3 g((unsigned)((N + kGT - 1) / kGT), (unsigned)((M + kGT - 1) / kGT));
  k_gemm_bf16<TA, TB, EPI><<<g, 128, 0, ctx().stream>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, act,
                                                        ldact, zp, ldzp);
  return launched("gemm_bf16");
}

}  // namespace pv

using namespace pv;

/* ---------------------------------------------------------------- network */
struct pevsl_mlp {
  int nin, nout, width, layers; /* layers = number of linear maps */
  int kdim[8], ndim[8];         /* padded: K (inputs) and N (outputs) per layer */
  long woff[8], boff[8];        /* offsets of W_l (N x K, row-major) and b_l in the parameter block */
  long np;                      /* parameters incl. padding */
  float *p, *g, *m1, *m2;       /* device FP32: master, gradient, Adam moments */
  bf16 *ph;                     /* device BF16 copy of p */
  uint8_t *mask;                /* 1 for real parameters, 0 for padding */
  long step;
  int cap;                      /* batch capacity of the buffers */
  float *z[8];                  /* pre-activations [cap][N_l] */
  bf16 *a[9];                   /* a[0] = input, a[l+1] = gelu(z[l]) [cap][N_l] */
  float *dz;                    /* gradient of a pre-activation [cap][maxdim] (fp32) */
  bf16 *dzh[2];                 /* bf16 copies, ping-pong */
  float *loss;                  /* device scalar */
  double *partials;
  unsigned *counter;
};

static int pad16(int x) { return (x + 15) / 16 * 16; }

static void mlp_free_buffers(pevsl_mlp *net) {
  for (int l = 0; l < 8; l++) {
    cudaFree(net->z[l]);
    net->z[l] = nullptr;
  }
  for (int l = 0; l < 9; l++) {
    cudaFree(net->a[l]);
    net->a[l] = nullptr;
  }
  cudaFree(net->dz);
  cudaFree(net->dzh[0]);
  cudaFree(net->dzh[1]);
  net->dz = nullptr;
  net->dzh[0] = net->dzh[1] = nullptr;
  net->cap = 0;
}

static int mlp_reserve(pevsl_mlp *net, int batch) {
  if (batch <= net->cap) return 0;
  mlp_free_buffers(net);
  int maxd = net->kdim[0];
  for (int l = 0; l < net->layers; l++) maxd = PEVSL_MAX(maxd, net->ndim[l]);
  bool ok = true;
  ok = ok && cudaMalloc(&net->a[0], sizeof(bf16) * (size_t)batch * net->kdim[0]) == cudaSuccess;
  for (int l = 0; l < net->layers && ok; l++) {
    ok = ok && cudaMalloc(&net->z[l], sizeof(float) * (size_t)batch * net->ndim[l]) == cudaSuccess;
    ok = ok && cudaMalloc(&net->a[l + 1], sizeof(bf16) * (size_t)batch * net->ndim[l]) == cudaSuccess;
  }
  ok = ok && cudaMalloc(&net->dz, sizeof(float) * (size_t)batch * maxd) == cudaSuccess;
  ok = ok && cudaMalloc(&net->dzh[0], sizeof(bf16) * (size_t)batch * maxd) == cudaSuccess;
  ok = ok && cudaMalloc(&net->dzh[1], sizeof(bf16) * (size_t)batch * maxd) == cudaSuccess;
  if (!ok) {
    mlp_free_buffers(net);
    return PEVSL_ERR_NOMEM;
  }
  net->cap = batch;
  return 0;
}

/* forward pass on a[0] (already packed); outputs in z[layers-1] */
static int mlp_forward(pevsl_mlp *net, int B) {
  int st = 0;
  for (int l = 0; l < net->layers && !st; l++) {
    const int K = net->kdim[l], N = net->ndim[l];
    const bf16 *W = net->ph + net->woff[l];
    const float *b = net->p + net->boff[l];
    if (l + 1 < net->layers)
      st = gemm<false, true, EPI_BIAS_GELU>(B, N, K, net->a[l], K, W, K, net->z[l], N, b,
                                            net->a[l + 1], N, nullptr, 0);
    else
      st = gemm<false, true, EPI_BIAS>(B, N, K, net->a[l], K, W, K, net->z[l], N, b, nullptr, 0,
                                       nullptr, 0);
  }
  return st;
}

/* loss and gradients into net->g for targets T [B][ldt] (FP32, device) */
static int mlp_backward(pevsl_mlp *net, int B, const float *T, int ldt) {
  Ctx &c = ctx();
  const int L = net->layers;
  int st = fail(cudaMemsetAsync(net->g, 0, sizeof(float) * (size_t)net->np, c.stream), "memset g");
  const int NL = net->ndim[L - 1];
  const unsigned gb = grid_for((long)B * NL, 4) > 256 ? 256 : grid_for((long)B * NL, 4);
  if (!st) {
    k_mse<<<gb, 256, 0, c.stream>>>(B, NL, net->nout, net->z[L - 1], T, ldt, net->dz, net->dzh[0],
                                    net->partials, net->counter, net->loss);
    st = launched("mse");
  }
  int cur = 0;
  for (int l = L - 1; l >= 0 && !st; l--) {
    const int K = net->kdim[l], N = net->ndim[l];
    /* dW_l = dZ_l^T a_l (N x K), db_l = column sums of dZ_l */
    st = gemm<true, false, EPI_STORE>(N, K, B, net->dzh[cur], N, net->a[l], K, net->g + net->woff[l],
                                      K, nullptr, nullptr, 0, nullptr, 0);
    if (!st) {
      k_colsum<<<(N + 127) / 128, 128, 0, c.stream>>>(B, N, net->dz, N, net->g + net->boff[l]);
      st = launched("colsum");
    }
    if (l == 0 || st) break;
    /* dZ_{l-1} = (dZ_l W_l) * gelu'(z_{l-1}) */
    st = gemm<false, false, EPI_DGELU>(B, K, N, net->dzh[cur], N, net->ph + net->woff[l], K, net->dz,
                                       K, nullptr, net->dzh[1 - cur], K, net->z[l - 1], K);
    cur = 1 - cur;
  }
  return st;
}

extern "C" {

int pEVSL_B200_MlpCreate(pevsl_mlp **out, int nin, int width, int nout, int layers) {
  *out = nullptr;
  if (ensure()) return PEVSL_ERR_CUDA;
  if (nin <= 0 || nout <= 0 || width <= 0 || layers < 1 || layers > 8) return PEVSL_ERR_ARG;
  pevsl_mlp *net = (pevsl_mlp *)calloc(1, sizeof(pevsl_mlp));
  if (!net) return PEVSL_ERR_NOMEM;
  net->nin = nin;
  net->nout = nout;
  net->width = width;
  net->layers = layers;
  long off = 0;
  for (int l = 0; l < layers; l++) {
    net->kdim[l] = pad16(l == 0 ? nin : width);
    net->ndim[l] = pad16(l + 1 == layers ? nout : width);
    net->woff[l] = off;
    off += (long)net->kdim[l] * net->ndim[l];
    net->boff[l] = off;
    off += net->ndim[l];
  }
  net->np = off;
  bool ok = true;
  ok = ok && cudaMalloc(&net->p, sizeof(float) * off) == cudaSuccess;
  ok = ok && cudaMalloc(&net->g, sizeof(float) * off) == cudaSuccess;
  ok = ok && cudaMalloc(&net->m1, sizeof(float) * off) == cudaSuccess;
  ok = ok && cudaMalloc(&net->m2, sizeof(float) * off) == cudaSuccess;
  ok = ok && cudaMalloc(&net->ph, sizeof(bf16) * off) == cudaSuccess;
  ok = ok && cudaMalloc(&net->mask, off) == cudaSuccess;
  ok = ok && cudaMalloc(&net->loss, sizeof(float)) == cudaSuccess;
  ok = ok && cudaMalloc(&net->partials, sizeof(double) * 256) == cudaSuccess;
  ok = ok && cudaMalloc(&net->counter, sizeof(unsigned)) == cudaSuccess;
  if (ok) {
    cudaMemset(net->p, 0, sizeof(float) * off);
    cudaMemset(net->g, 0, sizeof(float) * off);
    cudaMemset(net->m1, 0, sizeof(float) * off);
    cudaMemset(net->m2, 0, sizeof(float) * off);
    cudaMemset(net->ph, 0, sizeof(bf16) * off);
    cudaMemset(net->counter, 0, sizeof(unsigned));
    /* mask of real entries */
    uint8_t *hm = (uint8_t *)calloc((size_t)off, 1);
    if (!hm) ok = false;
    for (int l = 0; l < layers && ok; l++) {
      const int kr = l == 0 ? nin : width, nr = l + 1 == layers ? nout : width;
      for (int n = 0; n < nr; n++) {
        memset(hm + net->woff[l] + (long)n * net->kdim[l], 1, (size_t)kr);
        hm[net->boff[l] + n] = 1;
      }
    }
    ok = ok && cudaMemcpy(net->mask, hm, (size_t)off, cudaMemcpyHostToDevice) == cudaSuccess;
    free(hm);
  }
  if (!ok) {
    pEVSL_B200_MlpFree(net);
    return PEVSL_ERR_NOMEM;
  }
  *out = net;
  return 0;
}

void pEVSL_B200_MlpFree(pevsl_mlp *net) {
  if (!net) return;
  mlp_free_buffers(net);
  cudaFree(net->p);
  cudaFree(net->g);
  cudaFree(net->m1);
  cudaFree(net->m2);
  cudaFree(net->ph);
  cudaFree(net->mask);
  cudaFree(net->loss);
  cudaFree(net->partials);
  cudaFree(net->counter);
  free(net);
}

long pEVSL_B200_MlpParamCount(const pevsl_mlp *net) { return net ? net->np : 0; }

int pEVSL_B200_MlpLayout(const pevsl_mlp *net, int *kdim, int *ndim, long *woff, long *boff) {
  if (!net) return PEVSL_ERR_ARG;
  for (int l = 0; l < net->layers; l++) {
    kdim[l] = net->kdim[l];
    ndim[l] = net->ndim[l];
    woff[l] = net->woff[l];
    boff[l] = net->boff[l];
  }
  return net->layers;
}

/* parameters (FP32 master, the padded layout above) from / to the host;
 * setting them resets the Adam state */
int pEVSL_B200_MlpSetParams(pevsl_mlp *net, const float *host) {
  if (!net || !host) return PEVSL_ERR_ARG;
  if (fail(cudaMemcpy(net->p, host, sizeof(float) * net->np, cudaMemcpyHostToDevice), "MlpSetParams"))
    return PEVSL_ERR_CUDA;
  cudaMemset(net->m1, 0, sizeof(float) * net->np);
  cudaMemset(net->m2, 0, sizeof(float) * net->np);
  net->step = 0;
  k_to_bf16<<<grid_for(net->np, 4), kThreads, 0, ctx().stream>>>(net->np, net->p, net->ph);
  if (launched("to_bf16")) return PEVSL_ERR_CUDA;
  return sync();
}

int pEVSL_B200_MlpGetParams(const pevsl_mlp *net, float *host) {
  if (!net || !host) return PEVSL_ERR_ARG;
  if (sync()) return PEVSL_ERR_CUDA;
  return fail(cudaMemcpy(host, net->p, sizeof(float) * net->np, cudaMemcpyDeviceToHost), "MlpGetParams")
             ? PEVSL_ERR_CUDA
             : 0;
}

/* Y [B][nout] = net(X [B][nin]); X, Y FP32 device (or managed) arrays */
int pEVSL_B200_MlpForward(pevsl_mlp *net, const float *X, float *Y, int B) {
  if (!net || B < 0) return PEVSL_ERR_ARG;
  if (B == 0) return 0;
  if (mlp_reserve(net, B)) return PEVSL_ERR_NOMEM;
  const int K0 = net->kdim[0];
  k_pack_input<<<grid_for((long)B * K0, 4), kThreads, 0, ctx().stream>>>(B, net->nin, K0, X, net->a[0]);
  if (launched("pack_input")) return PEVSL_ERR_CUDA;
  if (mlp_forward(net, B)) return PEVSL_ERR_CUDA;
  const int L = net->layers, NL = net->ndim[L - 1];
  if (fail(cudaMemcpy2DAsync(Y, sizeof(float) * net->nout, net->z[L - 1], sizeof(float) * NL,
                             sizeof(float) * net->nout, B, cudaMemcpyDefault, ctx().stream),
           "MlpForward copy"))
    return PEVSL_ERR_CUDA;
  return sync();
}

/* mean squared error of net(X) against T [B][nout] and its gradient (host
 * FP32, the parameter layout) without updating the weights */
int pEVSL_B200_MlpGradients(pevsl_mlp *net, const float *X, const float *T, int B, float *loss,
                            float *grad_host) {
  if (!net || B <= 0) return PEVSL_ERR_ARG;
  if (mlp_reserve(net, B)) return PEVSL_ERR_NOMEM;
  const int K0 = net->kdim[0];
  k_pack_input<<<grid_for((long)B * K0, 4), kThreads, 0, ctx().stream>>>(B, net->nin, K0, X, net->a[0]);
  if (launched("pack_input")) return PEVSL_ERR_CUDA;
  if (mlp_forward(net, B) || mlp_backward(net, B, T, net->nout)) return PEVSL_ERR_CUDA;
  if (sync()) return PEVSL_ERR_CUDA;
  if (loss && cudaMemcpy(loss, net->loss, sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
    return PEVSL_ERR_CUDA;
  if (grad_host &&
      cudaMemcpy(grad_host, net->g, sizeof(float) * net->np, cudaMemcpyDeviceToHost) != cudaSuccess)
    return PEVSL_ERR_CUDA;
  return 0;
}

/* one Adam step on the batch (X, T); the loss before the step in *loss
 * (may be NULL; reading it synchronises) */
int pEVSL_B200_MlpTrainStep(pevsl_mlp *net, const float *X, const float *T, int B, float lr,
                            float *loss) {
  if (!net || B <= 0) return PEVSL_ERR_ARG;
  if (mlp_reserve(net, B)) return PEVSL_ERR_NOMEM;
  Ctx &c = ctx();
  const int K0 = net->kdim[0];
  k_pack_input<<<grid_for((long)B * K0, 4), kThreads, 0, c.stream>>>(B, net->nin, K0, X, net->a[0]);
  if (launched("pack_input")) return PEVSL_ERR_CUDA;
  if (mlp_forward(net, B) || mlp_backward(net, B, T, net->nout)) return PEVSL_ERR_CUDA;
  net->step++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)net->step), c2 = 1.f - powf(b2, (float)net->step);
  k_adam<<<grid_for(net->np, 4), kThreads, 0, c.stream>>>(net->np, net->p, net->g, net->m1, net->m2,
                                                         net->mask, net->ph, lr, b1, b2, 1e-8f, c1, c2);
  if (launched("adam")) return PEVSL_ERR_CUDA;
  if (loss) {
    if (sync()) return PEVSL_ERR_CUDA;
    if (cudaMemcpy(loss, net->loss, sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
      return PEVSL_ERR_CUDA;
  }
  return 0;
}

}  // extern "C"
