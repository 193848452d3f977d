/*
 * Device runtime (context, workspaces, launch accounting), level-1 vector
 * kernels with deterministic reductions, the Philox Gaussian generator, and
 * the pEVSL vector API (SRC/parvec.c, SRC/parvecs.c) on device / managed
 * memory.
 *
 * Reductions are deterministic: each block reduces its grid-stride share with
 * a fixed shuffle tree, writes one partial, and the last block to finish (an
 * atomic ticket) adds the partials in block order.  The grid size depends
 * only on n, so a result never depends on scheduling.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gpu.cuh"
#include "gpu_device.cuh"

namespace pv {

static Ctx g_ctx;

Ctx &ctx() { return g_ctx; }

int fail(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return 0;
  fprintf(stderr, "pevsl-b200: CUDA error in %s: %s\n", what, cudaGetErrorString(e));
  g_ctx.sticky_error = PEVSL_ERR_CUDA;
  return PEVSL_ERR_CUDA;
}

static int g_req_device = -1;

int ensure() {
  if (g_ctx.ready) return 0;
  int dev = 0, ndev = 0;
  if (fail(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount")) return PEVSL_ERR_CUDA;
  /* device: pEVSL_B200_SetDevice, else PEVSL_B200_DEVICE, else the launcher's
   * LOCAL_RANK (one process per GPU), else 0 */
  int want = g_req_device;
  if (want < 0 && getenv("PEVSL_B200_DEVICE")) want = atoi(getenv("PEVSL_B200_DEVICE"));
  if (want < 0 && getenv("LOCAL_RANK")) want = atoi(getenv("LOCAL_RANK"));
  if (want >= 0 && ndev > 0) {
    if (fail(cudaSetDevice(want % ndev), "cudaSetDevice")) return PEVSL_ERR_CUDA;
  }
  if (fail(cudaGetDevice(&dev), "cudaGetDevice")) return PEVSL_ERR_CUDA;
  g_ctx.device = dev;
  cudaDeviceProp prop;
  if (fail(cudaGetDeviceProperties(&prop, dev), "cudaGetDeviceProperties")) return PEVSL_ERR_CUDA;
  g_ctx.sms = prop.multiProcessorCount;
  /* a blocking stream: work that a user callback puts on the legacy default
   * stream stays ordered with ours */
  if (fail(cudaStreamCreate(&g_ctx.stream), "cudaStreamCreate")) return PEVSL_ERR_CUDA;
  if (fail(cudaMalloc(&g_ctx.red, sizeof(double) * kMaxRedBlocks * 64), "cudaMalloc red"))
    return PEVSL_ERR_CUDA;
  if (fail(cudaMalloc(&g_ctx.cnt, sizeof(unsigned) * 4096), "cudaMalloc cnt")) return PEVSL_ERR_CUDA;
  if (fail(cudaMemset(g_ctx.cnt, 0, sizeof(unsigned) * 4096), "cudaMemset cnt")) return PEVSL_ERR_CUDA;
  if (fail(cudaMalloc(&g_ctx.dscal, sizeof(double) * S_COUNT), "cudaMalloc scal")) return PEVSL_ERR_CUDA;
  if (fail(cudaMemset(g_ctx.dscal, 0, sizeof(double) * S_COUNT), "cudaMemset scal"))
    return PEVSL_ERR_CUDA;
  if (fail(cudaMallocHost(&g_ctx.hscal, sizeof(double) * S_COUNT), "cudaMallocHost"))
    return PEVSL_ERR_CUDA;
  if (fail(cudaMalloc(&g_ctx.dflag, sizeof(int) * F_COUNT), "cudaMalloc flag")) return PEVSL_ERR_CUDA;
  if (fail(cudaMemset(g_ctx.dflag, 0, sizeof(int) * F_COUNT), "cudaMemset flag")) return PEVSL_ERR_CUDA;
  if (fail(cudaMalloc(&g_ctx.gscal, sizeof(double) * 4 * kMaxEntries), "cudaMalloc gscal"))
    return PEVSL_ERR_CUDA;
  if (fail(cudaMallocHost(&g_ctx.hgscal, sizeof(double) * 4 * kMaxEntries), "cudaMallocHost"))
    return PEVSL_ERR_CUDA;
  if (fail(cudaMalloc(&g_ctx.gflag, sizeof(int) * kMaxEntries), "cudaMalloc gflag"))
    return PEVSL_ERR_CUDA;
  if (fail(cudaMemset(g_ctx.gflag, 0, sizeof(int) * kMaxEntries), "cudaMemset gflag"))
    return PEVSL_ERR_CUDA;
  if (fail(cudaMallocHost(&g_ctx.htab, kFiltTabBytes * kTabSlots), "cudaMallocHost tab"))
    return PEVSL_ERR_CUDA;
  if (fail(cudaMalloc(&g_ctx.dtab, kFiltTabBytes * kTabSlots), "cudaMalloc tab")) return PEVSL_ERR_CUDA;
  for (int i = 0; i < kTabSlots; i++)
    if (fail(cudaEventCreateWithFlags(&g_ctx.tab_ev[i], cudaEventDisableTiming), "cudaEventCreate"))
      return PEVSL_ERR_CUDA;
  if (fail(cudaMalloc(&g_ctx.bar, sizeof(unsigned) * 4), "cudaMalloc bar")) return PEVSL_ERR_CUDA;
  if (fail(cudaMemset(g_ctx.bar, 0, sizeof(unsigned) * 4), "cudaMemset bar")) return PEVSL_ERR_CUDA;
  g_ctx.ready = true;
  return 0;
}

/* Optional L2 residency of the operator (environment variable
 * PEVSL_B200_L2PERSIST=1): reserve the persisting part of L2 and point the
 * library stream's access-policy window at the matrix block, so the matrix
 * stays on chip while the vectors stream through the rest of L2.  The limit
 * belongs to this process's context and ends with it. */
void l2_window(const void *base, size_t bytes) {
  static int enabled = -1;
  static size_t max_persist = 0, max_window = 0;
  if (enabled < 0) {
    const char *e = getenv("PEVSL_B200_L2PERSIST");
    enabled = e && atoi(e) != 0;
    if (enabled) {
      cudaDeviceProp prop;
      if (cudaGetDeviceProperties(&prop, g_ctx.device) == cudaSuccess) {
        max_persist = (size_t)prop.persistingL2CacheMaxSize;
        max_window = (size_t)prop.accessPolicyMaxWindowSize;
      }
      if (!max_persist || !max_window) enabled = 0;
    }
  }
  if (!enabled) return;
  const size_t win = bytes < max_window ? bytes : max_window;
  const size_t persist = win < max_persist ? win : max_persist;
  cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, persist);
  cudaStreamAttrValue attr;
  memset(&attr, 0, sizeof attr);
  attr.accessPolicyWindow.base_ptr = const_cast<void *>(base);
  attr.accessPolicyWindow.num_bytes = win;
  attr.accessPolicyWindow.hitRatio = (float)((double)persist / (double)win);
  attr.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
  attr.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
  cudaStreamSetAttribute(g_ctx.stream, cudaStreamAttributeAccessPolicyWindow, &attr);
  cudaGetLastError(); /* the window is a hint: ignore refusals */
}

int launched(const char *what) {
  g_ctx.launches++;
  return fail(cudaGetLastError(), what);
}

int sync() { return fail(cudaStreamSynchronize(g_ctx.stream), "cudaStreamSynchronize"); }

void *ws(int slot, size_t bytes) {
  if (ensure()) return nullptr;
  if (bytes == 0) bytes = 256;
  if (g_ctx.wsz[slot] >= bytes) return g_ctx.ws[slot];
  if (g_ctx.ws[slot]) {
    cudaStreamSynchronize(g_ctx.stream);
    cudaFree(g_ctx.ws[slot]);
    g_ctx.ws[slot] = nullptr;
    g_ctx.wsz[slot] = 0;
  }
  void *p = nullptr;
  if (fail(cudaMalloc(&p, bytes), "cudaMalloc workspace")) return nullptr;
  g_ctx.ws[slot] = p;
  g_ctx.wsz[slot] = bytes;
  return p;
}

int memcpy_async(void *dst, const void *src, size_t bytes) {
  if (bytes == 0) return 0;
  return fail(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, g_ctx.stream), "cudaMemcpyAsync");
}

const double *fetch_scalars(int first, int count) {
  if (memcpy_async(g_ctx.hscal + first, g_ctx.dscal + first, sizeof(double) * count)) return nullptr;
  if (sync()) return nullptr;
  return g_ctx.hscal + first;
}

/* ---------------------------------------------------------------- BLAS1 kernels */

__global__ void k_fill(double *x, long n, double v) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    x[i] = v;
}
__global__ void k_scal(double *x, long n, double a) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    x[i] *= a;
}
__global__ void k_axpy(long n, double a, const double *__restrict__ x, double *__restrict__ y) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    y[i] += a * x[i];
}
__global__ void k_axpy_dev(long n, const double *coef, double sign, const double *__restrict__ x,
                           double *__restrict__ y) {
  const double a = sign * *coef;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    y[i] += a * x[i];
}
__global__ void k_scal_inv_dev(long n, const double *s, double *x) {
  const double a = 1.0 / *s;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    x[i] *= a;
}
__global__ void k_sum(long n, const double *__restrict__ x, double *partials, unsigned *counter,
                      double *out) {
  double s = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    s += x[i];
  bool last;
  const double t = grid_sum(s, partials, counter, FIN_ID, &last);
  if (last && threadIdx.x == 0) *out = t;
}

/* per-column dot products: grid (bx, m); partials [m][bx] */
__global__ void k_dot_cols(long n, const double *__restrict__ X, long ldx,
                           const double *__restrict__ Y, long ldy, double *partials,
                           unsigned *counters, double *out) {
  const int c = blockIdx.y;
  const double *x = X + (size_t)c * ldx, *y = Y + (size_t)c * ldy;
  double s = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    s += x[i] * y[i];
  /* grid reduction over the blocks of this column */
  __shared__ bool am_last;
  __shared__ double sh[32];
  const double b = block_sum(s, sh);
  if (threadIdx.x == 0) {
    partials[(size_t)c * gridDim.x + blockIdx.x] = b;
    __threadfence();
    am_last = atomicAdd(counters + c, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  double t = 0.0;
  for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x)
    t += __ldcg(partials + (size_t)c * gridDim.x + i);
  t = block_sum(t, sh);
  if (threadIdx.x == 0) {
    out[c] = t;
    counters[c] = 0;
  }
}
__global__ void k_scal_cols(long n, double *X, long ldx, const double *s) {
  const int c = blockIdx.y;
  const double a = s[c];
  double *x = X + (size_t)c * ldx;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    x[i] *= a;
}
__global__ void k_axpy_cols(long n, const double *lam, const double *__restrict__ X, long ldx,
                            double *__restrict__ Y, long ldy) {
  const int c = blockIdx.y;
  const double a = -lam[c];
  const double *x = X + (size_t)c * ldx;
  double *y = Y + (size_t)c * ldy;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    y[i] += a * x[i];
}

int vfill(double *x, long n, double v) {
  if (n <= 0) return 0;
  k_fill<<<grid_for(n, 4), kThreads, 0, g_ctx.stream>>>(x, n, v);
  return launched("fill");
}
int vcopy(const double *x, double *y, long n) {
  if (n <= 0 || x == y) return 0;
  return memcpy_async(y, x, sizeof(double) * (size_t)n);
}
int vscal(double *x, long n, double a) {
  if (n <= 0) return 0;
  k_scal<<<grid_for(n, 4), kThreads, 0, g_ctx.stream>>>(x, n, a);
  return launched("scal");
}
int vaxpy(long n, double a, const double *x, double *y) {
  if (n <= 0) return 0;
  k_axpy<<<grid_for(n, 4), kThreads, 0, g_ctx.stream>>>(n, a, x, y);
  return launched("axpy");
}
int vaxpy_dev(long n, const double *coef, double sign, const double *x, double *y) {
  if (n <= 0) return 0;
  k_axpy_dev<<<grid_for(n, 4), kThreads, 0, g_ctx.stream>>>(n, coef, sign, x, y);
  return launched("axpy_dev");
}
int vscal_inv_dev(long n, const double *s, double *x) {
  if (n <= 0) return 0;
  k_scal_inv_dev<<<grid_for(n, 4), kThreads, 0, g_ctx.stream>>>(n, s, x);
  return launched("scal_inv_dev");
}
int vsum(long n, const double *x, double *out) {
  k_sum<<<grid_for(n, 4), kThreads, 0, g_ctx.stream>>>(n, x, g_ctx.red, g_ctx.cnt, out);
  return launched("sum");
}

static unsigned col_blocks(long n) {
  long b = (n + kThreads * 8 - 1) / (kThreads * 8);
  return (unsigned)(b < 1 ? 1 : (b > 64 ? 64 : b));
}

int vdot_cols(long n, int m, const double *X, long ldx, const double *Y, long ldy, double *out) {
  const unsigned bx = col_blocks(n);
  double *part = (double *)ws(WS_SMALL, sizeof(double) * (size_t)bx * 4096);
  if (!part) return PEVSL_ERR_NOMEM;
  for (int c0 = 0; c0 < m; c0 += 4096) {
    const int mc = m - c0 < 4096 ? m - c0 : 4096;
    dim3 g(bx, mc);
    k_dot_cols<<<g, kThreads, 0, g_ctx.stream>>>(n, X + (size_t)c0 * ldx, ldx, Y + (size_t)c0 * ldy,
                                                 ldy, part, g_ctx.cnt, out + c0);
    if (launched("dot_cols")) return PEVSL_ERR_CUDA;
  }
  return 0;
}
int vscal_cols(long n, int m, double *X, long ldx, const double *s) {
  for (int c0 = 0; c0 < m; c0 += 65535) {
    const int mc = m - c0 < 65535 ? m - c0 : 65535;
    dim3 g(col_blocks(n), mc);
    k_scal_cols<<<g, kThreads, 0, g_ctx.stream>>>(n, X + (size_t)c0 * ldx, ldx, s + c0);
    if (launched("scal_cols")) return PEVSL_ERR_CUDA;
  }
  return 0;
}
int vaxpy_cols(long n, int m, const double *lam, const double *X, long ldx, double *Y, long ldy) {
  for (int c0 = 0; c0 < m; c0 += 65535) {
    const int mc = m - c0 < 65535 ? m - c0 : 65535;
    dim3 g(col_blocks(n), mc);
    k_axpy_cols<<<g, kThreads, 0, g_ctx.stream>>>(n, lam + c0, X + (size_t)c0 * ldx, ldx,
                                                  Y + (size_t)c0 * ldy, ldy);
    if (launched("axpy_cols")) return PEVSL_ERR_CUDA;
  }
  return 0;
}

/* ---------------------------------------------------------------- Philox Gaussian
 * Counter-based generator of Salmon et al. (SC'11), 10 rounds; Box-Muller on
 * 53-bit uniforms.  Draw m, element pair p: counter {p, m}, key = seed. */
__device__ __forceinline__ void philox10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const uint32_t lo0 = 0xD2511F53u * c[0], hi0 = __umulhi(0xD2511F53u, c[0]);
    const uint32_t lo1 = 0xCD9E8D57u * c[2], hi1 = __umulhi(0xCD9E8D57u, c[2]);
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

__global__ void k_rand_gauss(double *X, long n, int nv, long rs, long cs, uint64_t seed, uint64_t m0) {
  const long npair = (n + 1) / 2;
  const int v = blockIdx.y;
  const uint64_t m = m0 + (uint64_t)v;
  const double two_pi = 6.283185307179586476925286766559;
  const double inv53 = 1.0 / 9007199254740992.0;
  for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < npair; p += (long)gridDim.x * blockDim.x) {
    uint32_t c[4] = {(uint32_t)p, (uint32_t)((uint64_t)p >> 32), (uint32_t)m, (uint32_t)(m >> 32)};
    philox10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const uint64_t a = ((((uint64_t)c[0]) << 32) | c[1]) >> 11;
    const uint64_t b = ((((uint64_t)c[2]) << 32) | c[3]) >> 11;
    const double u1 = ((double)a + 0.5) * inv53, u2 = (double)b * inv53;
    const double rad = sqrt(-2.0 * log(u1));
    double sn, cn;
    sincos(two_pi * u2, &sn, &cn);
    X[(2 * p) * rs + (long)v * cs] = rad * cn;
    if (2 * p + 1 < n) X[(2 * p + 1) * rs + (long)v * cs] = rad * sn;
  }
}

int rand_gauss(double *X, long n, int nv, long rs, long cs, uint64_t seed, uint64_t m0) {
  for (int v0 = 0; v0 < nv; v0 += 65535) {
    const int nb = nv - v0 < 65535 ? nv - v0 : 65535;
    dim3 g(grid_for((n + 1) / 2, 2), nb);
    k_rand_gauss<<<g, kThreads, 0, g_ctx.stream>>>(X + (long)v0 * cs, n, nb, rs, cs, seed,
                                                   m0 + (uint64_t)v0);
    if (launched("rand_gauss")) return PEVSL_ERR_CUDA;
  }
  return 0;
}

}  // namespace pv

/* ================================================================ C interface */
using namespace pv;

static int g_rng_mode = PEVSL_RNG_GLIBC;
static uint64_t g_rng_seed = 0, g_rng_draws = 0;

extern "C" {

int pEVSL_B200_SetRng(int mode, uint64_t seed) {
  if (mode != PEVSL_RNG_GLIBC && mode != PEVSL_RNG_GAUSS) return PEVSL_ERR_ARG;
  g_rng_mode = mode;
  g_rng_seed = seed;
  g_rng_draws = 0;
  srand((unsigned)seed);
  return 0;
}
uint64_t pEVSL_B200_RngDraws(void) { return g_rng_draws; }
int pevsl_rng_mode(void) { return g_rng_mode; }
uint64_t pevsl_rng_seed(void) { return g_rng_seed; }
uint64_t pevsl_rng_take(uint64_t k) {
  const uint64_t first = g_rng_draws;
  g_rng_draws += k;
  return first;
}

/* Host generation of the C library stream, uniform on [-1,1]: the element
 * formula of pEVSL_ParvecRand (SRC/parvec.c:65-72). */
static void glibc_fill(double *h, long n) {
  const double t = ((double)RAND_MAX) / 2.0;
  for (long i = 0; i < n; i++) h[i] = (rand() - t) / t;
}

int pevsl_rand_vector_dev(double *dev, int n) {
  if (ensure()) return PEVSL_ERR_CUDA;
  const uint64_t m = pevsl_rng_take(1);
  if (g_rng_mode == PEVSL_RNG_GAUSS) return rand_gauss(dev, n, 1, 1, 0, g_rng_seed, m);
  double *h = nullptr;
  if (fail(cudaMallocHost(&h, sizeof(double) * (size_t)(n > 0 ? n : 1)), "cudaMallocHost")) return PEVSL_ERR_CUDA;
  glibc_fill(h, n);
  int st = memcpy_async(dev, h, sizeof(double) * (size_t)n);
  if (!st) st = sync();
  cudaFreeHost(h);
  return st;
}

int pevsl_rand_block_dev(double *X, int n, int nv, int ld) {
  if (ensure()) return PEVSL_ERR_CUDA;
  const uint64_t m0 = pevsl_rng_take((uint64_t)nv);
  if (g_rng_mode == PEVSL_RNG_GAUSS) return rand_gauss(X, n, nv, ld, 1, g_rng_seed, m0);
  /* the C library stream is sequential: vector c is rand() draws
   * [c*n, (c+1)*n), laid out interleaved */
  const size_t tot = (size_t)n * (size_t)ld;
  double *h = nullptr, *col = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  if (!col || fail(cudaMallocHost(&h, sizeof(double) * (tot ? tot : 1)), "cudaMallocHost")) {
    free(col);
    return PEVSL_ERR_NOMEM;
  }
  memset(h, 0, sizeof(double) * tot);
  for (int c = 0; c < nv; c++) {
    glibc_fill(col, n);
    for (int i = 0; i < n; i++) h[(size_t)i * ld + c] = col[i];
  }
  int st = memcpy_async(X, h, sizeof(double) * tot);
  if (!st) st = sync();
  cudaFreeHost(h);
  free(col);
  return st;
}

uint64_t pEVSL_B200_LaunchCount(void) { return g_ctx.launches; }

/* Synchronous copy between host and library memory (device or managed), in
 * either direction. */
int pEVSL_B200_Memcpy(void *dst, const void *src, size_t bytes) {
  if (ensure()) return PEVSL_ERR_CUDA;
  if (memcpy_async(dst, src, bytes)) return PEVSL_ERR_CUDA;
  return sync();
}

int pEVSL_B200_CopyEigenvectors(const pevsl_Parvecs *W, int nvec, double *vec, long ld) {
  if (!W || nvec < 0 || nvec > W->n_vecs || (nvec > 0 && (!vec || ld < W->n_local)))
    return PEVSL_ERR_ARG;
  if (nvec == 0 || W->n_local == 0) return 0;
  if (ensure()) return PEVSL_ERR_CUDA;
  /* one strided copy: column i of W (ld W->ld) to vec + i * ld */
  if (fail(cudaMemcpy2DAsync(vec, sizeof(double) * (size_t)ld, W->data, sizeof(double) * (size_t)W->ld,
                             sizeof(double) * (size_t)W->n_local, (size_t)nvec, cudaMemcpyDefault,
                             g_ctx.stream),
           "cudaMemcpy2DAsync"))
    return PEVSL_ERR_CUDA;
  return sync();
}

int pEVSL_B200_SetDevice(int device) {
  if (g_ctx.ready) return g_ctx.device == device ? 0 : PEVSL_ERR_ARG;
  g_req_device = device;
  return ensure();
}

/* Events on the library stream, for timing a region of library work. */
static cudaEvent_t g_user_ev[16];
static bool g_user_ev_ok = false;

int pEVSL_B200_EventRecord(int slot) {
  if (ensure() || slot < 0 || slot >= 16) return PEVSL_ERR_ARG;
  if (!g_user_ev_ok) {
    for (int i = 0; i < 16; i++)
      if (fail(cudaEventCreate(&g_user_ev[i]), "cudaEventCreate")) return PEVSL_ERR_CUDA;
    g_user_ev_ok = true;
  }
  return fail(cudaEventRecord(g_user_ev[slot], g_ctx.stream), "cudaEventRecord");
}

double pEVSL_B200_EventElapsedMs(int a, int b) {
  if (!g_user_ev_ok || a < 0 || a >= 16 || b < 0 || b >= 16) return -1.0;
  if (fail(cudaEventSynchronize(g_user_ev[b]), "cudaEventSynchronize")) return -1.0;
  float ms = 0.f;
  if (fail(cudaEventElapsedTime(&ms, g_user_ev[a], g_user_ev[b]), "cudaEventElapsedTime")) return -1.0;
  return (double)ms;
}

/* write `bytes` (0: 256 MiB, twice the L2) of a scratch device buffer on
 * the library stream, so that the next timed work finds nothing of its own
 * in L2 */
int pEVSL_B200_FlushL2(size_t bytes) {
  static void *buf = nullptr;
  static size_t cap = 0;
  static int val = 0;
  if (ensure()) return PEVSL_ERR_CUDA;
  if (!bytes) bytes = (size_t)256 << 20;
  if (bytes > cap) {
    if (buf) cudaFree(buf);
    buf = nullptr;
    cap = 0;
    if (fail(cudaMalloc(&buf, bytes), "cudaMalloc flush")) return PEVSL_ERR_NOMEM;
    cap = bytes;
  }
  val = (val + 1) & 0xff;
  if (fail(cudaMemsetAsync(buf, val, bytes, g_ctx.stream), "cudaMemsetAsync flush")) return PEVSL_ERR_CUDA;
  return 0;
}

void *pEVSL_B200_HostAlloc(size_t bytes) {
  void *p = nullptr;
  if (ensure() || fail(cudaMallocHost(&p, bytes ? bytes : 1), "cudaMallocHost")) return nullptr;
  return p;
}

void pEVSL_B200_HostFree(void *p) {
  if (p) cudaFreeHost(p);
}

void *pEVSL_B200_ManagedAlloc(size_t bytes) {
  void *p = nullptr;
  if (ensure() || fail(cudaMallocManaged(&p, bytes ? bytes : 1), "cudaMallocManaged")) return nullptr;
  return p;
}

void pEVSL_B200_ManagedFree(void *p) {
  if (p) {
    cudaStreamSynchronize(g_ctx.stream);
    cudaFree(p);
  }
}

/* Wait for all work queued by the library. */
int pEVSL_B200_Sync(void) {
  if (ensure()) return PEVSL_ERR_CUDA;
  return sync();
}

int pEVSL_B200_LastError(void) {
  const int e = g_ctx.sticky_error;
  g_ctx.sticky_error = 0;
  return e;
}

void pEVSL_B200_ReleaseWorkspace(void) {
  if (!g_ctx.ready) return;
  cudaStreamSynchronize(g_ctx.stream);
  for (int i = 0; i < WS_COUNT; i++) {
    if (g_ctx.ws[i]) cudaFree(g_ctx.ws[i]);
    g_ctx.ws[i] = nullptr;
    g_ctx.wsz[i] = 0;
  }
}

int pEVSL_B200_Info(char *buf, int len) {
  if (!buf || len <= 0) return PEVSL_ERR_ARG;
  int dev = 0, rt = 0, drv = 0;
  cudaDeviceProp prop;
  memset(&prop, 0, sizeof prop);
  if (cudaGetDevice(&dev) == cudaSuccess) cudaGetDeviceProperties(&prop, dev);
  cudaRuntimeGetVersion(&rt);
  cudaDriverGetVersion(&drv);
  snprintf(buf, (size_t)len, "pevsl-b200 sm_100a build; device %d %s (cc %d.%d, %d SMs); runtime %d driver %d",
           dev, prop.name, prop.major, prop.minor, prop.multiProcessorCount, rt, drv);
  return 0;
}

/* ---------------------------------------------------------------- Parvec
 * SRC/parvec.c.  Data in managed memory (device memory when the environment
 * variable PEVSL_B200_PARVEC_MEM=device).  Every call completes before it
 * returns, like the reference's host BLAS. */

static double *alloc_vec(size_t count) {
  if (ensure()) return nullptr;
  void *p = nullptr;
  const size_t bytes = sizeof(double) * (count ? count : 1);
  const char *mode = getenv("PEVSL_B200_PARVEC_MEM");
  cudaError_t e = (mode && !strcmp(mode, "device")) ? cudaMalloc(&p, bytes)
                                                     : cudaMallocManaged(&p, bytes, cudaMemAttachGlobal);
  if (fail(e, "parvec allocation")) return nullptr;
  return (double *)p;
}

static void free_vec(double *p) {
  if (!p) return;
  cudaStreamSynchronize(g_ctx.stream);
  cudaFree(p);
}

void pEVSL_ParvecCreateShell(int nglobal, int nlocal, int nfirst, MPI_Comm comm, pevsl_Parvec *x,
                             double *data) {
  x->comm = comm;
  x->n_global = nglobal;
  x->n_local = nlocal;
  x->n_first = nfirst < 0 ? PEVSL_NOT_DEFINED : nfirst;
  x->data = data;
}

void pEVSL_ParvecCreate(int nglobal, int nlocal, int nfirst, MPI_Comm comm, pevsl_Parvec *x) {
  pEVSL_ParvecCreateShell(nglobal, nlocal, nfirst, comm, x, alloc_vec((size_t)nlocal));
}

void pEVSL_ParvecDupl(pevsl_Parvec *x, pevsl_Parvec *y) {
  pEVSL_ParvecCreate(x->n_global, x->n_local, x->n_first, x->comm, y);
}

void pEVSL_ParvecFree(pevsl_Parvec *x) {
  free_vec(x->data);
  x->data = nullptr;
}

void pEVSL_ParvecRand(pevsl_Parvec *x) {
  if (!pevsl_rand_vector_dev(x->data, x->n_local)) sync();
}

void pEVSL_ParvecDot(pevsl_Parvec *x, pevsl_Parvec *y, double *t) {
  *t = NAN;
  if (ensure() || vdot(x->n_local, x->data, y->data, g_ctx.dscal + S_TMP0)) return;
  const double *h = fetch_scalars(S_TMP0, 1);
  if (h) *t = h[0];
}

void pEVSL_ParvecNrm2(pevsl_Parvec *x, double *t) {
  *t = NAN;
  if (ensure() || vnrm2(x->n_local, x->data, g_ctx.dscal + S_TMP0)) return;
  const double *h = fetch_scalars(S_TMP0, 1);
  if (h) *t = h[0];
}

void pEVSL_ParvecSum(pevsl_Parvec *x, double *t) {
  *t = NAN;
  if (ensure() || vsum(x->n_local, x->data, g_ctx.dscal + S_TMP0)) return;
  const double *h = fetch_scalars(S_TMP0, 1);
  if (h) *t = h[0];
}

void pEVSL_ParvecCopy(pevsl_Parvec *x, pevsl_Parvec *y) {
  if (!ensure() && !vcopy(x->data, y->data, x->n_local)) sync();
}

void pEVSL_ParvecScal(pevsl_Parvec *x, double t) {
  if (!ensure() && !vscal(x->data, x->n_local, t)) sync();
}

void pEVSL_ParvecSetScalar(pevsl_Parvec *x, double t) {
  if (!ensure() && !vfill(x->data, x->n_local, t)) sync();
}

void pEVSL_ParvecSetZero(pevsl_Parvec *x) {
  if (!ensure() && !vfill(x->data, x->n_local, 0.0)) sync();
}

void pEVSL_ParvecAxpy(double a, pevsl_Parvec *x, pevsl_Parvec *y) {
  if (!ensure() && !vaxpy(x->n_local, a, x->data, y->data)) sync();
}

int pEVSL_ParvecSameSize(pevsl_Parvec *x, pevsl_Parvec *y) {
  return x->n_global == y->n_global && x->n_local == y->n_local && x->n_first == y->n_first;
}

/* Writes "% n_global" then one value per line (SRC/parvec.c:487-521). */
int pEVSL_ParvecWrite(pevsl_Parvec *x, const char *fn) {
  if (ensure()) return PEVSL_ERR_CUDA;
  double *h = (double *)malloc(sizeof(double) * (size_t)(x->n_local > 0 ? x->n_local : 1));
  if (!h) return PEVSL_ERR_NOMEM;
  int st = memcpy_async(h, x->data, sizeof(double) * (size_t)x->n_local);
  if (!st) st = sync();
  FILE *fp = fn ? fopen(fn, "w") : stdout;
  if (!st && fp) {
    fprintf(fp, "%% %d\n", x->n_global);
    for (int j = 0; j < x->n_local; j++) fprintf(fp, "%.15e\n", h[j]);
  }
  if (fn && fp) fclose(fp);
  free(h);
  return st;
}

/* ---------------------------------------------------------------- Parvecs
 * SRC/parvecs.c: column-major, leading dimension ld. */

void pEVSL_ParvecsCreateShell(int nglobal, int nvecs, int ld, int nlocal, int nfirst, MPI_Comm comm,
                              pevsl_Parvecs *x, double *data) {
  x->comm = comm;
  x->n_global = nglobal;
  x->n_local = nlocal;
  x->n_first = nfirst < 0 ? PEVSL_NOT_DEFINED : nfirst;
  x->n_vecs = nvecs;
  x->ld = ld;
  x->data = data;
}

void pEVSL_ParvecsCreate(int nglobal, int nvecs, int ld, int nlocal, int nfirst, MPI_Comm comm,
                         pevsl_Parvecs *x) {
  pEVSL_ParvecsCreateShell(nglobal, nvecs, ld, nlocal, nfirst, comm, x,
                           alloc_vec((size_t)ld * (size_t)nvecs));
}

void pEVSL_ParvecsDuplParvec(pevsl_Parvec *x, int nvecs, int ld, pevsl_Parvecs *y) {
  pEVSL_ParvecsCreate(x->n_global, nvecs, ld, x->n_local, x->n_first, x->comm, y);
}

void pEVSL_ParvecsFree(pevsl_Parvecs *x) {
  free_vec(x->data);
  x->data = nullptr;
}

void pEVSL_ParvecsGetParvecShell(pevsl_Parvecs *X, int i, pevsl_Parvec *x) {
  double *d = i < 0 ? nullptr : X->data + (size_t)X->ld * (size_t)i;
  pEVSL_ParvecCreateShell(X->n_global, X->n_local, X->n_first, X->comm, x, d);
}

/* y = alp A(:, 0:nvecs) x + bet y; x is a host array (SRC/parvecs.c:93-102) */
void pEVSL_ParvecsGemv(double alp, pevsl_Parvecs *A, int nvecs, double *x, double bet,
                       pevsl_Parvec *y) {
  if (ensure()) return;
  const long n = A->n_local;
  double *dx = (double *)ws(WS_SMALL, sizeof(double) * (size_t)(nvecs + 1));
  double *tmp = (double *)ws(WS_VEC, sizeof(double) * (size_t)(n > 0 ? n : 1));
  if (!dx || !tmp) return;
  if (memcpy_async(dx, x, sizeof(double) * (size_t)nvecs)) return;
  if (gemm_nn(n, nvecs, 1, A->data, A->ld, dx, nvecs, tmp, n)) return;
  if (bet == 0.0) {
    if (vfill(y->data, n, 0.0)) return; /* like BLAS: y is not read when beta is 0 */
  } else if (bet != 1.0 && vscal(y->data, n, bet)) {
    return;
  }
  if (vaxpy(n, alp, tmp, y->data)) return;
  sync();
}

/* y = alp A(:,0:nvecs)' x + bet y with y, w host arrays (SRC/parvecs.c:117-136) */
void pEVSL_ParvecsGemtvWithWspace(double alp, pevsl_Parvecs *A, int nvecs, pevsl_Parvec *x,
                                  double bet, double *y, double *w) {
  if (ensure()) return;
  double *dw = (double *)ws(WS_SMALL, sizeof(double) * (size_t)(nvecs + 1));
  if (!dw) return;
  if (gemvT(A->n_local, nvecs, A->data, A->ld, x->data, dw, nullptr)) return;
  if (memcpy_async(w, dw, sizeof(double) * (size_t)nvecs) || sync()) return;
  for (int j = 0; j < nvecs; j++) y[j] = bet * y[j] + alp * w[j];
}

void pEVSL_ParvecsGemtv(double alp, pevsl_Parvecs *A, int nvecs, pevsl_Parvec *x, double bet,
                        double *y) {
  double *w = (double *)malloc(sizeof(double) * (size_t)(2 * nvecs + 1));
  if (!w) return;
  pEVSL_ParvecsGemtvWithWspace(alp, A, nvecs, x, bet, y, w);
  free(w);
}

}  // extern "C"
