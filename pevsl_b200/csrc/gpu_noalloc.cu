/*
 * Allocation-free projection w = V(:, 0:k)' x.
 *
 * Some callers of this library cannot let it allocate device memory: code
 * that runs inside a host framework which owns every device allocation
 * through its own pool, latency-critical loops that cannot afford the device
 * synchronisation cudaMalloc/cudaFree imply, and programs that budget all
 * device memory up front and must not fail with out-of-memory in the middle
 * of a run.  pEVSL_B200_ParvecsGemtvNoAlloc serves them: it computes the
 * projection of pEVSL_ParvecsGemtv (the Gram-Schmidt coefficients of
 * SRC/parvecs.c:117-136) into caller-provided device memory and uses, as its
 * only scratch, a fixed array in this file that the library holds on every
 * GPU it is loaded on.  It never calls cudaMalloc, cudaFree, the library's
 * own context set-up or any allocating routine.
 */
#include <cuda_runtime.h>
#include <stdio.h>

#include <atomic>

#include "internal.h"

namespace {

constexpr int kNaRowBlocks = 128;      /* row blocks: partial sums per column */
constexpr int kNaMaxCols = 256;        /* largest k accepted                 */
constexpr int kNaThreads = 256;
constexpr int kNaColsPerBlock = kNaThreads / 32;

/* Scratch shared by every call on a device: kNaRowBlocks x kNaMaxCols
 * partial sums (256 KiB).  Each call overwrites every entry it later reads,
 * so nothing has to be cleared; calls that overlap on the GPU race on it. */
static __device__ __align__(256) double g_noalloc_partials[kNaRowBlocks * kNaMaxCols];

/* device address of the scratch array, looked up once per device; host
 * threads that race on the first lookup store the same address */
constexpr int kNaMaxDevices = 64;
std::atomic<double *> g_noalloc_ptr[kNaMaxDevices] = {};

/* partial[rb * k + j] = sum over the rows of block rb of V[i + j ld] x[i];
 * a warp per column, lanes across rows. */
__global__ void __launch_bounds__(kNaThreads)
    k_noalloc_partial(long n, int k, const double *__restrict__ V, long ld,
                      const double *__restrict__ x, long rows, double *__restrict__ partial) {
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int j = blockIdx.y * kNaColsPerBlock + wib;
  if (j >= k) return;
  const long r0 = (long)blockIdx.x * rows;
  const long r1 = r0 + rows < n ? r0 + rows : n;
  const double *col = V + (size_t)j * ld;
  double acc = 0.0;
  for (long i = r0 + lane; i < r1; i += 32) acc = fma(col[i], x[i], acc);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) partial[(size_t)blockIdx.x * k + j] = acc;
}

/* w[j] = sum of the kNaRowBlocks partials of column j, in block order */
__global__ void k_noalloc_reduce(int k, const double *__restrict__ partial, double *__restrict__ w) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= k) return;
  double acc = 0.0;
  for (int b = 0; b < kNaRowBlocks; b++) acc += partial[(size_t)b * k + j];
  w[j] = acc;
}

}  // namespace

extern "C" {

/* w = V(:, 0:k)' x on the GPU without allocating.
 *
 *   V      device pointer, column-major n x k, leading dimension ld >= n
 *   x      device pointer, n entries
 *   w      device pointer, k entries (output)
 *   stream cudaStream_t to run on, or NULL for the legacy default stream
 *
 * Accepts 0 < k <= 256 and n >= 0; anything else returns PEVSL_ERR_ARG with a
 * message on stderr.  The first call on a device looks up the device address
 * of the scratch array with cudaGetSymbolAddress (with that device current),
 * so make that first call on each device before any stream capture.  The
 * call is asynchronous on `stream`; w is ready when the stream is.  All calls
 * on one device share the scratch array: calls that may run concurrently on
 * the GPU (different streams without ordering between them) race on it and
 * must be serialised by the caller. */
int pEVSL_B200_ParvecsGemtvNoAlloc(const double *V, long n, long ld, int k, const double *x,
                                   double *w, void *stream) {
  if (k <= 0 || k > kNaMaxCols) {
    fprintf(stderr, "pEVSL_B200_ParvecsGemtvNoAlloc: k = %d is outside 1..%d\n", k, kNaMaxCols);
    return PEVSL_ERR_ARG;
  }
  if (n < 0 || ld < n || !V || !x || !w) {
    fprintf(stderr, "pEVSL_B200_ParvecsGemtvNoAlloc: bad sizes or pointers (n %ld, ld %ld)\n", n, ld);
    return PEVSL_ERR_ARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNaMaxDevices) return PEVSL_ERR_CUDA;
  double *scratch = g_noalloc_ptr[dev].load(std::memory_order_acquire);
  if (!scratch) {
    const cudaError_t e = cudaGetSymbolAddress((void **)&scratch, g_noalloc_partials);
    if (e != cudaSuccess) {
      fprintf(stderr, "pEVSL_B200_ParvecsGemtvNoAlloc: cudaGetSymbolAddress: %s\n",
              cudaGetErrorString(e));
      return PEVSL_ERR_CUDA;
    }
    g_noalloc_ptr[dev].store(scratch, std::memory_order_release);
  }
  cudaStream_t s = (cudaStream_t)stream;
  const long rows = n > 0 ? (n + kNaRowBlocks - 1) / kNaRowBlocks : 1;
  dim3 g(kNaRowBlocks, (unsigned)((k + kNaColsPerBlock - 1) / kNaColsPerBlock));
  k_noalloc_partial<<<g, kNaThreads, 0, s>>>(n, k, V, ld, x, rows, scratch);
  k_noalloc_reduce<<<(k + 127) / 128, 128, 0, s>>>(k, scratch, w);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "pEVSL_B200_ParvecsGemtvNoAlloc: launch failed: %s\n", cudaGetErrorString(e));
    return PEVSL_ERR_CUDA;
  }
  return 0;
}

}  // extern "C"
