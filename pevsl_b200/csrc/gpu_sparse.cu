/*
 * Sparse matrix on the GPU: the parcsr API (SRC/parcsr.c, SRC/parcsrmv.c)
 * collapsed onto one device CSR, the CSR SpMV, and the two fused hot kernels
 * of the path:
 *
 *  - cheb_step: one degree of the Chebyshev filter recurrence of
 *    pEVSL_ChebAv (SRC/chebpol.c:538-568) with the SpMV fused in, so that a
 *    degree reads A, v_k, v_{k-1}, y and writes v_{k+1}, y once;
 *  - kpm_step: one degree of the KPM recurrence of pEVSL_Kpmdos
 *    (SRC/kpmdos.c:129-156) for a block of s random vectors at once, with the
 *    moment dot products fused in, so that A is read once per degree for all
 *    vectors.
 *
 * Layout: CSR with int32 row pointers / column indices and fp64 values; a
 * row is handled by a group of L lanes (L = 1..32, a power of two picked from
 * the mean row length) that read the row's entries contiguously and reduce
 * with warp shuffles.  KPM blocks are row-interleaved (row i of all s vectors
 * contiguous), so the gather of x[col] is one coalesced 8*s-byte segment.
 */
#include <ctype.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <vector>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gpu.cuh"
#include "gpu_device.cuh"

namespace pv {

/* Programmatic dependent launch of the ELL filter-degree kernels.  A degree
 * launched with the stream-serialisation attribute may be scheduled while
 * the previous degree's last blocks still run: its blocks stage the value
 * table in shared memory, then wait (griddepcontrol.wait) until the
 * previous grid has completed and its writes are visible, and only then
 * read a vector.  A block lets the next degree be scheduled
 * (griddepcontrol.launch_dependents) only after its own wait, so the early
 * part of degree k+1 overlaps degree k and nothing older.  What the early
 * part reads, the value table, is written at set-up, followed by a device
 * synchronisation, and never again while the matrix lives.  Without the
 * attribute the wait returns at once.  (Loading the first entries of a row
 * before the wait as well took the one-vector kernel from 32 to 48
 * registers and measured slower.) */
__device__ __forceinline__ void pdl_wait_then_release() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

/* PEVSL_B200_PDL: 1 (default) launches the ELL filter degrees with the
 * attribute, 0 as plain stream-ordered launches */
static int pdl_mode() {
  static int v = -1;
  if (v < 0) {
    const char *e = getenv("PEVSL_B200_PDL");
    v = e ? atoi(e) != 0 : 1;
  }
  return v;
}

template <class... KA, class... AA>
static void launch_pdl(void (*k)(KA...), unsigned grid, cudaStream_t st, AA &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = pdl_mode();
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k, std::forward<AA>(args)...);
}

template <int L>
__device__ __forceinline__ unsigned group_mask() {
  if constexpr (L == 32) {
    return 0xffffffffu;
  } else {
    const unsigned lane = threadIdx.x & 31u;
    return ((1u << L) - 1u) << (lane & ~(unsigned)(L - 1));
  }
}

template <int L>
__device__ __forceinline__ double group_sum(double v, unsigned mask) {
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
  return v;
}

/* r = sum_{j in row} a[j] x[ja[j]], spread over the L lanes of the group */
template <int L>
__device__ __forceinline__ double row_dot(int row, const int *__restrict__ ia,
                                          const int *__restrict__ ja, const double *__restrict__ a,
                                          const double *__restrict__ x, int lane) {
  const int s = ia[row], e = ia[row + 1];
  double r = 0.0;
  for (int j = s + lane; j < e; j += L) r = fma(a[j], __ldg(x + ja[j]), r);
  return r;
}

template <int L>
__global__ void __launch_bounds__(kThreads) k_spmv(int n, const int *__restrict__ ia,
                                                   const int *__restrict__ ja,
                                                   const double *__restrict__ a,
                                                   const double *__restrict__ x,
                                                   double *__restrict__ y) {
  const long gt = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const int row = (int)(gt / L), lane = (int)(threadIdx.x & (L - 1));
  if (row >= n) return; /* the whole group leaves together */
  const unsigned mask = group_mask<L>();
  const double r = group_sum<L>(row_dot<L>(row, ia, ja, a, x, lane), mask);
  if (lane == 0) y[row] = r;
}

template <int L>
__global__ void __launch_bounds__(kThreads)
    k_cheb_step(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                const double *__restrict__ a, const double *__restrict__ vk,
                const double *__restrict__ vkm1, double *__restrict__ vkp1, double *__restrict__ y,
                double cc, double t, double mu0, double muk, int first) {
  const long gt = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const int row = (int)(gt / L), lane = (int)(threadIdx.x & (L - 1));
  if (row >= n) return;
  const unsigned mask = group_mask<L>();
  const double r = group_sum<L>(row_dot<L>(row, ia, ja, a, vk, lane), mask);
  if (lane == 0) {
    double w, yv = first ? 0.0 : y[row];
    cheb_update(r, vk[row], vkm1 ? vkm1 + row : nullptr, cc, t, mu0, muk, first, &w, &yv);
    vkp1[row] = w;
    y[row] = yv;
  }
}

__global__ void k_cheb_combine(long n, const double *__restrict__ ax, const double *__restrict__ vk,
                               const double *__restrict__ vkm1, double *__restrict__ vkp1,
                               double *__restrict__ y, double cc, double t, double mu0, double muk,
                               int first) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double w, yv = first ? 0.0 : y[i];
    cheb_update(ax[i], vk[i], vkm1 ? vkm1 + i : nullptr, cc, t, mu0, muk, first, &w, &yv);
    vkp1[i] = w;
    y[i] = yv;
  }
}

__global__ void k_chebiter1_combine(long n, const double *__restrict__ w, const double *__restrict__ b,
                                    const double *__restrict__ x, double *__restrict__ p,
                                    double *__restrict__ xnew, double bet, double alp) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double pn = __dadd_rn(__dmul_rn(p[i], bet), __dsub_rn(b[i], w[i]));
    p[i] = pn;
    xnew[i] = __fma_rn(alp, pn, x[i]);
  }
}

__global__ void k_chebiter2_combine(long n, const double *__restrict__ w, const double *__restrict__ d,
                                    double *__restrict__ x, double *__restrict__ r,
                                    double *__restrict__ dnew, double c1, double c2) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    x[i] = __dadd_rn(x[i], d[i]);
    const double rn = __dsub_rn(r[i], w[i]);
    r[i] = rn;
    dnew[i] = __fma_rn(c2, rn, __dmul_rn(d[i], c1));
  }
}

/* ---------------------------------------------------------------- CSR-stream
 * Short rows (the stencil matrices of this path have 5-16 entries): a warp
 * owns 32 consecutive rows.  Its lanes stream the rows' entries in
 * contiguous, independent 8-deep batches (column index, value, gathered x),
 * stage the products a[j]*x[ja[j]] in shared memory, and each lane then adds
 * its own row's products in index order -- the summation order of the
 * reference's row loop (SRC/spmat.c:188-193), so the result matches it to
 * the last bit when the products are not fused.  The epilogue runs one
 * thread per row, so the vector traffic is coalesced. */
constexpr int kStreamChunk = 256; /* staged entries per warp per pass */

__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

/* An epilogue loads what it needs of its row (pre) before the row's
 * products are formed, so those loads overlap the matrix and gather loads,
 * and then combines (operator()). */
struct EpiStore {
  double *y;
  struct Pre {};
  __device__ __forceinline__ Pre pre(int) const { return Pre{}; }
  __device__ __forceinline__ void operator()(int row, double r, const Pre &) const { y[row] = r; }
};

/* vkp1 may alias vkm1: the thread of a row reads v_{k-1} there first */
struct EpiCheb {
  const double *vk, *vkm1;
  double *vkp1, *y;
  double cc, t, mu0, muk;
  int first;
  struct Pre {
    double x, xm1, y;
  };
  __device__ __forceinline__ Pre pre(int row) const {
    return Pre{vk[row], vkm1 ? vkm1[row] : 0.0, first ? 0.0 : y[row]};
  }
  __device__ __forceinline__ void operator()(int row, double r, const Pre &p) const {
    double w, yv;
    cheb_update_v(r, p.x, p.xm1, vkm1 != nullptr, cc, t, mu0, muk, first, p.y, &w, &yv);
    vkp1[row] = w;
    y[row] = yv;
  }
};

/* FP32 degree of the mixed-precision filter; the last degree writes the
 * accumulated p(A) x to the FP64 output (yout) instead of y */
struct EpiCheb32 {
  const float *vk, *vkm1;
  float *vkp1, *y;
  double *yout;
  float cc, t, mu0, muk;
  int first;
  struct Pre {
    float x, xm1, y;
  };
  __device__ __forceinline__ Pre pre(int row) const {
    return Pre{vk[row], vkm1 ? vkm1[row] : 0.f, first ? 0.f : y[row]};
  }
  __device__ __forceinline__ void operator()(int row, float r, const Pre &p) const {
    float w = __fmul_rn(__fmaf_rn(-cc, p.x, r), t);
    if (vkm1) w = __fsub_rn(w, p.xm1);
    vkp1[row] = w;
    const float yv = first ? __fmaf_rn(muk, w, __fmul_rn(mu0, p.x)) : __fmaf_rn(muk, w, p.y);
    if (yout)
      yout[row] = (double)yv;
    else
      y[row] = yv;
  }
};

/* One step of the Chebyshev iteration for B x = b of
 * EXTERNAL/ITERSOL/chebiter.c:121-197 (first kind): with w = B x_i,
 *   r = b - w;  p = bet p + r;  x_{i+1} = x_i + alp p.
 * x_i is the gathered vector, so x_{i+1} goes to another buffer. */
struct EpiChebIter1 {
  const double *b, *x;
  double *p, *xnew;
  double bet, alp;
  struct Pre {
    double b, p, x;
  };
  __device__ __forceinline__ Pre pre(int row) const { return Pre{b[row], p[row], x[row]}; }
  __device__ __forceinline__ void operator()(int row, double w, const Pre &q) const {
    const double r = __dsub_rn(q.b, w);
    const double pn = __dadd_rn(__dmul_rn(q.p, bet), r);
    p[row] = pn;
    xnew[row] = __fma_rn(alp, pn, q.x);
  }
};

/* One step of EXTERNAL/ITERSOL/chebiter.c:204-262 (second kind): with
 * w = B d, x += d;  r -= w;  d_new = c1 d + c2 r  (c1 = rho1 rho,
 * c2 = 2 rho1 / delta).  d is the gathered vector: d_new goes to dnew. */
struct EpiChebIter2 {
  const double *d;
  double *x, *r, *dnew;
  double c1, c2;
  struct Pre {
    double d, x, r;
  };
  __device__ __forceinline__ Pre pre(int row) const { return Pre{d[row], x[row], r[row]}; }
  __device__ __forceinline__ void operator()(int row, double w, const Pre &q) const {
    x[row] = __dadd_rn(q.x, q.d);
    const double rn = __dsub_rn(q.r, w);
    r[row] = rn;
    dnew[row] = __fma_rn(c2, rn, __dmul_rn(q.d, c1));
  }
};

/* Rows [32 R (8 rblk + warp), +32 R) of y = A x, lane l owning rows
 * l + 32 j (j < R) so that the epilogue is coalesced.  Per pass a warp
 * stages 256 R consecutive entries of its rows: column indices and values
 * with independent coalesced loads, then the gathered products
 * a[j] * x[ja[j]] (unfused) into shared memory; each lane adds its rows'
 * products in index order -- the summation order of the reference's row
 * loop (SRC/spmat.c:188-193), so the result matches it to the last bit. */
/* Entry accessors of stream_rows: the plain CSR arrays, or the packed form
 * (int16 column offset from the row's 32-row group, uint8 index into a
 * table of the distinct values held in shared memory).  Both give the same
 * column and the same double (or float) for every entry. */
template <class T>
struct EntriesCSR {
  const int *__restrict__ ja;
  const T *__restrict__ a;
  __device__ __forceinline__ int col(long t, int) const { return __ldg(ja + t); }
  __device__ __forceinline__ T val(long t) const { return __ldg(a + t); }
};

template <class T>
struct EntriesPacked {
  const short *__restrict__ dj;
  const unsigned char *__restrict__ vi;
  const T *vt; /* shared memory */
  __device__ __forceinline__ int col(long t, int g0) const { return g0 + (int)__ldg(dj + t); }
  __device__ __forceinline__ T val(long t) const { return vt[__ldg(vi + t)]; }
};

/* R == 1 for the packed accessor: the column offsets are relative to the
 * warp's one 32-row group */
template <int R, class T, class Epi, bool NC, class Ent>
__device__ __forceinline__ void stream_rows_e(int n, const int *__restrict__ ia, const Ent &ent,
                                              const T *x, const Epi &epi, long rblk,
                                              T (*prod)[kStreamChunk * R]) {
  constexpr int CH = kStreamChunk * R, PL = CH / 32;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long r0l = (rblk * (kThreads / 32) + w) * 32 * R;
  if (r0l >= n) return; /* the whole warp leaves */
  const int r0 = (int)r0l;
  const int nr = n - r0 < 32 * R ? n - r0 : 32 * R;
  typename Epi::Pre pre[R];
  int rs[R], re[R];
  /* the matrix is read-only for every launch: the non-coherent path */
#pragma unroll
  for (int j = 0; j < R; j++) {
    const int row = r0 + lane + 32 * j;
    rs[j] = re[j] = 0;
    if (lane + 32 * j < nr) {
      pre[j] = epi.pre(row);
      rs[j] = __ldg(ia + row);
      re[j] = __ldg(ia + row + 1);
    }
  }
  const int base = __ldg(ia + r0), len = __ldg(ia + r0 + nr) - base;
  T acc[R];
#pragma unroll
  for (int j = 0; j < R; j++) {
    rs[j] -= base;
    re[j] -= base;
    acc[j] = T(0);
  }
  T *pw = prod[w];
  for (int c0 = 0; c0 < len; c0 += CH) {
    int col[PL];
    T val[PL];
#pragma unroll
    for (int q = 0; q < PL; q++) {
      const int t = c0 + q * 32 + lane;
      col[q] = t < len ? ent.col(base + t, r0) : -1;
      val[q] = t < len ? ent.val(base + t) : T(0);
    }
#pragma unroll
    for (int q = 0; q < PL; q++) {
      /* NC: x is read-only for the launch (non-coherent path); otherwise it
       * was written earlier in the same launch by other blocks */
      const T xv = col[q] >= 0 ? (NC ? __ldg(x + col[q]) : x[col[q]]) : T(0);
      pw[q * 32 + lane] = mul_rn(val[q], xv);
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < R; j++) {
      const int lo = rs[j] > c0 ? rs[j] : c0;
      const int hi = re[j] < c0 + CH ? re[j] : c0 + CH;
      for (int t = lo; t < hi; t++) acc[j] = add_rn(acc[j], pw[t - c0]);
    }
    __syncwarp();
  }
#pragma unroll
  for (int j = 0; j < R; j++)
    if (lane + 32 * j < nr) epi(r0 + lane + 32 * j, acc[j], pre[j]);
}

template <int R, class T, class Epi, bool NC = true>
__device__ __forceinline__ void stream_rows(int n, const int *__restrict__ ia,
                                            const int *__restrict__ ja, const T *__restrict__ a,
                                            const T *x, const Epi &epi, long rblk,
                                            T (*prod)[kStreamChunk * R]) {
  stream_rows_e<R, T, Epi, NC>(n, ia, EntriesCSR<T>{ja, a}, x, epi, rblk, prod);
}

/* the packed form: the block stages the value table in shared memory */
template <class T, class Epi>
__global__ void __launch_bounds__(kThreads, 5)
    k_csr_stream_packed(int n, const int *__restrict__ ia, const short *__restrict__ dj,
                        const unsigned char *__restrict__ vi, const T *__restrict__ vtab, int nv,
                        const T *__restrict__ x, Epi epi) {
  __shared__ T prod[kThreads / 32][kStreamChunk];
  __shared__ T vt[256];
  for (int i = threadIdx.x; i < nv; i += blockDim.x) vt[i] = vtab[i];
  __syncthreads();
  pdl_wait_then_release();
  stream_rows_e<1, T, Epi, true>(n, ia, EntriesPacked<T>{dj, vi, vt}, x, epi, blockIdx.x, prod);
}

/* R = 1 fits 48 registers (5 blocks per SM) without spilling */
template <int R, class T, class Epi>
__global__ void __launch_bounds__(kThreads, R == 1 ? 5 : 1)
    k_csr_stream(int n, const int *__restrict__ ia, const int *__restrict__ ja,
                 const T *__restrict__ a, const T *__restrict__ x, Epi epi) {
  __shared__ T prod[kThreads / 32][kStreamChunk * R];
  pdl_wait_then_release();
  stream_rows<R>(n, ia, ja, a, x, epi, blockIdx.x, prod);
}

/* Up to CAP independent products y_e = A_e x_e (x_e = epi[e].vk), each with
 * its own matrix and epilogue, in one launch.  With `shared` (all entries
 * on one matrix) block b serves entry b % nb on row block b / nb: the nb
 * blocks that read one stretch of the matrix are adjacent in launch order,
 * so the stretch comes from HBM once and from L2 for the other entries.
 * Otherwise block b serves the entry e with off[e] <= b < off[e+1], row
 * block b - off[e].  Each entry keeps its vectors in its own columns (no
 * interleaving, no copies), and its arithmetic is that of k_csr_stream, bit
 * for bit.  The table is a __grid_constant__ parameter (up to 32 KB). */
template <class T, class Epi, int CAP>
struct StreamBatch {
  const int *ia[CAP];
  const int *ja[CAP];
  const T *a[CAP];
  int n[CAP];
  int off[CAP + 1];
  Epi epi[CAP];
  int nb, shared;
};

/* SHARED: the one matrix comes as plain parameters (uniform operands, as in
 * k_csr_stream); otherwise per entry from the table. */
template <int R, class T, class Epi, int CAP, bool SHARED>
__global__ void __launch_bounds__(kThreads, R == 1 ? 4 : 1)
    k_csr_stream_batch(int n0, const int *__restrict__ ia0, const int *__restrict__ ja0,
                       const T *__restrict__ a0, const __grid_constant__ StreamBatch<T, Epi, CAP> b) {
  __shared__ T prod[kThreads / 32][kStreamChunk * R];
  pdl_wait_then_release();
  if constexpr (SHARED) {
    const int e = (int)(blockIdx.x % (unsigned)b.nb);
    stream_rows<R>(n0, ia0, ja0, a0, (const T *)b.epi[e].vk, b.epi[e],
                   (long)(blockIdx.x / (unsigned)b.nb), prod);
  } else {
    int lo = 0, hi = b.nb; /* off[lo] <= blockIdx.x < off[hi] */
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (b.off[mid] <= (int)blockIdx.x) lo = mid;
      else hi = mid;
    }
    stream_rows<R>(b.n[lo], b.ia[lo], b.ja[lo], b.a[lo], (const T *)b.epi[lo].vk, b.epi[lo],
                   (long)blockIdx.x - b.off[lo], prod);
  }
}

/* the shared-matrix batch on the packed form */
template <class T, class Epi, int CAP>
__global__ void __launch_bounds__(kThreads, 4)
    k_csr_stream_batch_packed(int n0, const int *__restrict__ ia0, const short *__restrict__ dj,
                              const unsigned char *__restrict__ vi, const T *__restrict__ vtab,
                              int nv, const __grid_constant__ StreamBatch<T, Epi, CAP> b) {
  __shared__ T prod[kThreads / 32][kStreamChunk];
  __shared__ T vt[256];
  for (int i = threadIdx.x; i < nv; i += blockDim.x) vt[i] = vtab[i];
  __syncthreads();
  pdl_wait_then_release();
  const int e = (int)(blockIdx.x % (unsigned)b.nb);
  stream_rows_e<1, T, Epi, true>(n0, ia0, EntriesPacked<T>{dj, vi, vt}, (const T *)b.epi[e].vk,
                                 b.epi[e], (long)(blockIdx.x / (unsigned)b.nb), prod);
}

/* ---------------------------------------------------------------- persistent filter */

constexpr unsigned kBarrierSpins = 1u << 24; /* ~2 s of polling before giving up */
static unsigned g_barrier_spins = kBarrierSpins;

/* Sense-counting grid barrier for a cooperative launch (all blocks are
 * co-resident).  bar[0] counts arrivals, bar[1] is the generation; the
 * waits are bounded: after `spins` polls the block sets bar[2] and
 * continues, and the kernel returns at its next check. */
__device__ __forceinline__ void grid_barrier(unsigned *bar, unsigned spins) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned *gen = bar + 1;
    const unsigned g = *gen;
    __threadfence();
    if (atomicAdd(bar, 1u) == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      unsigned it = 0;
      while (*gen == g) {
        if (++it > spins) {
          atomicExch(bar + 2, 1u);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

/* Operands of degree j of one entry (the two-buffer rotation of
 * cheb_apply: j = 1 reads x and writes b0, j = 2 reads b0 and x and writes
 * b1, then odd j write b0 over v_{j-1}, even j write b1). */
template <class T>
__device__ __forceinline__ void rotation(const FiltDev &E, int j, const T **vk, const T **vkm1,
                                         T **vkp1) {
  const T *x = (const T *)E.x;
  T *b0 = (T *)E.b0, *b1 = (T *)E.b1;
  if (j == 1) {
    *vk = x;
    *vkm1 = nullptr;
    *vkp1 = b0;
  } else if (j == 2) {
    *vk = b0;
    *vkm1 = x;
    *vkp1 = b1;
  } else if (j & 1) {
    *vk = b1;
    *vkm1 = b0;
    *vkp1 = b0;
  } else {
    *vk = b0;
    *vkm1 = b1;
    *vkp1 = b1;
  }
}

/* Work items of degree j: with `shared` (all entries on one matrix, nblk
 * row blocks each) item i is row block i / live of entry i % live, so the
 * entries reading one stretch of the matrix run together and share it in
 * L2; otherwise entry-major through the row-block offsets.  The table and,
 * per degree, every entry's mu[0] and mu[j] sit in shared memory, so an
 * item starts with the loads of its rows. */
template <class T, int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
    k_filter_persistent(const FiltDev *__restrict__ tab, int ne, const int *__restrict__ blk_off,
                        int maxdeg, int shared, unsigned *bar, unsigned spins) {
  __shared__ T prod[kThreads / 32][kStreamChunk];
  extern __shared__ double dyn[];
  FiltDev *s_tab = (FiltDev *)dyn;                /* ne entries */
  double *s_mu = (double *)(s_tab + ne);         /* 2 per entry: mu[0], mu[j] */
  int *s_off = (int *)(s_mu + 2 * ne);           /* ne + 1 */
  for (int i = threadIdx.x; i < ne * (int)(sizeof(FiltDev) / 8); i += blockDim.x)
    ((double *)s_tab)[i] = ((const double *)tab)[i];
  for (int i = threadIdx.x; i <= ne; i += blockDim.x) s_off[i] = blk_off[i];
  __syncthreads();
  int live = ne; /* entries sorted by non-increasing degree: a prefix is live */
  for (int j = 1; j <= maxdeg; j++) {
    while (live > 0 && s_tab[live - 1].deg < j) live--;
    for (int i = threadIdx.x; i < live; i += blockDim.x) {
      s_mu[2 * i] = s_tab[i].mu[0];
      s_mu[2 * i + 1] = s_tab[i].mu[j];
    }
    __syncthreads();
    const int total = s_off[live];
    for (int item = blockIdx.x; item < total; item += gridDim.x) {
      int lo;
      long rblk;
      if (shared) {
        lo = item % live;
        rblk = item / live;
      } else {
        int hi = live; /* s_off[lo] <= item < s_off[hi] */
        lo = 0;
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (s_off[mid] <= item) lo = mid;
          else hi = mid;
        }
        rblk = item - s_off[lo];
      }
      const FiltDev &E = s_tab[lo];
      const double t = j == 1 ? E.t1 : E.t2, mu0 = s_mu[2 * lo], muj = s_mu[2 * lo + 1];
      const T *vk, *vkm1;
      T *vkp1;
      rotation<T>(E, j, &vk, &vkm1, &vkp1);
      if constexpr (sizeof(T) == 8) {
        EpiCheb epi{vk, vkm1, vkp1, (double *)E.acc, E.cc, t, mu0, muj, j == 1};
        stream_rows<1, double, EpiCheb, false>(E.n, E.ia, E.ja, (const double *)E.a, vk, epi, rblk,
                                               prod);
      } else {
        EpiCheb32 epi{vk, vkm1, vkp1, (float *)E.acc, j == E.deg ? E.y : nullptr, (float)E.cc,
                      (float)t, (float)mu0, (float)muj, j == 1};
        stream_rows<1, float, EpiCheb32, false>(E.n, E.ia, E.ja, (const float *)E.a, vk, epi, rblk,
                                                prod);
      }
    }
    if (j < maxdeg) {
      grid_barrier(bar, spins); /* also orders the s_mu rewrite after every use */
      if (*(volatile unsigned *)(bar + 2)) return;
    }
  }
}

static_assert(sizeof(FiltDev) % 8 == 0, "the table is copied to shared memory in doubles");

static size_t persistent_smem(int ne) {
  return sizeof(FiltDev) * (size_t)ne + sizeof(double) * 2 * (size_t)ne +
         sizeof(int) * ((size_t)ne + 1);
}

static unsigned g_persist_grid = 0;

int cheb_filter_persistent(int ne, const FiltDev *entries, int maxdeg) {
  if (ne <= 0 || maxdeg <= 0) return 0;
  if (ne > kMaxEntries) return PEVSL_ERR_ARG;
  Ctx &c = ctx();
  /* co-resident grid for this table size (the dynamic shared memory grows
   * with the entries) */
  const size_t dsm = persistent_smem(ne);
  const bool fp32 = entries[0].fp32 != 0;
  /* blocks per SM the kernel is built for: 4 (64 registers) or 3
   * (PEVSL_B200_PERSIST_MINB=3, more registers, no spills) */
  static int minb = 0;
  if (!minb) {
    const char *e = getenv("PEVSL_B200_PERSIST_MINB");
    minb = e && atoi(e) == 3 ? 3 : 4;
  }
  const void *fn = fp32 ? (minb == 3 ? (const void *)k_filter_persistent<float, 3>
                                     : (const void *)k_filter_persistent<float, 4>)
                        : (minb == 3 ? (const void *)k_filter_persistent<double, 3>
                                     : (const void *)k_filter_persistent<double, 4>);
  static bool attr_done = false;
  if (!attr_done) {
    const void *all[4] = {(const void *)k_filter_persistent<float, 3>,
                          (const void *)k_filter_persistent<float, 4>,
                          (const void *)k_filter_persistent<double, 3>,
                          (const void *)k_filter_persistent<double, 4>};
    for (const void *f : all)
      if (fail(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)persistent_smem(kMaxEntries)),
               "cudaFuncSetAttribute"))
        return PEVSL_ERR_CUDA;
    attr_done = true;
  }
  int per_sm = 0;
  if (fail(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, dsm),
           "cudaOccupancyMaxActiveBlocksPerMultiprocessor"))
    return PEVSL_ERR_CUDA;
  if (per_sm < 1) return PEVSL_ERR_ARG;
  g_persist_grid = (unsigned)(per_sm * c.sms);
  /* table + row-block offsets staged in pinned memory, one copy; the slot
   * is rewritten only after its previous copy has run */
  const int slot = c.tab_next;
  c.tab_next = (c.tab_next + 1) % kTabSlots;
  if (fail(cudaEventSynchronize(c.tab_ev[slot]), "cudaEventSynchronize")) return PEVSL_ERR_CUDA;
  FiltDev *htab = (FiltDev *)((char *)c.htab + kFiltTabBytes * slot);
  int *hoff = (int *)(htab + kMaxEntries);
  memcpy(htab, entries, sizeof(FiltDev) * (size_t)ne);
  long total = 0;
  int shared = 1;
  for (int e = 0; e < ne; e++) {
    hoff[e] = (int)total;
    total += (entries[e].n + kThreads - 1) / kThreads;
    if (entries[e].ia != entries[0].ia || entries[e].a != entries[0].a) shared = 0;
  }
  hoff[ne] = (int)total;
  if (total <= 0) return 0;
  if (total > INT32_MAX) return PEVSL_ERR_ARG;
  const FiltDev *dtab = (const FiltDev *)((char *)c.dtab + kFiltTabBytes * slot);
  if (memcpy_async((void *)dtab, htab, kFiltTabBytes)) return PEVSL_ERR_CUDA;
  if (fail(cudaEventRecord(c.tab_ev[slot], c.stream), "cudaEventRecord")) return PEVSL_ERR_CUDA;
  unsigned grid = g_persist_grid;
  if ((long)grid > total) grid = (unsigned)total;
  const int *doff = (const int *)(dtab + kMaxEntries);
  unsigned *bar = c.bar;
  unsigned spins = g_barrier_spins;
  void *args[] = {(void *)&dtab,   (void *)&ne,     (void *)&doff, (void *)&maxdeg,
                  (void *)&shared, (void *)&bar,    (void *)&spins};
  if (fail(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kThreads), args, dsm, c.stream),
           "cudaLaunchCooperativeKernel"))
    return PEVSL_ERR_CUDA;
  return launched("filter_persistent");
}

/* polls before a barrier wait of the persistent filter gives up (0: the
 * default, about 2 s) */
void set_barrier_spins(unsigned spins) { g_barrier_spins = spins ? spins : kBarrierSpins; }

/* Preset the barrier's arrival counter so that no arrival completes it:
 * every wait then runs out after the spin limit and the kernel returns with
 * the timeout flag set (a fault injected from the host, for tests). */
int seed_barrier_arrivals(unsigned count) {
  if (ensure()) return PEVSL_ERR_CUDA;
  return fail(cudaMemcpy(ctx().bar, &count, sizeof count, cudaMemcpyHostToDevice), "cudaMemcpy")
             ? PEVSL_ERR_CUDA
             : 0;
}

int persistent_filter_error() {
  unsigned h[4] = {0, 0, 0, 0};
  if (cudaMemcpy(h, ctx().bar, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess) return 1;
  if (h[2]) {
    const unsigned z = 0;
    cudaMemcpy(ctx().bar + 2, &z, sizeof z, cudaMemcpyHostToDevice);
    cudaMemcpy(ctx().bar, &z, sizeof z, cudaMemcpyHostToDevice);
    return 1;
  }
  return 0;
}

/* Rows per lane of the CSR-stream kernels, per matrix: 1 until tuned */
static int stream_r(const pevsl_devcsr *A) { return A && A->stream_r == 2 ? 2 : 1; }

static unsigned stream_grid(int n, int R) {
  const long rows_per_block = (kThreads / 32) * 32L * R;
  return (unsigned)((n + rows_per_block - 1) / rows_per_block);
}


/* KPM degree for s <= 32*CPL interleaved vectors; one warp per row (grid
 * stride), lane c handles columns c, c+32, ...  Moments: per-block partial
 * sums in partials[block*s + c], the last block adds them in block order. */
template <int CPL>
__global__ void __launch_bounds__(kThreads)
    k_kpm_step(int n, int s, int ld, const int *__restrict__ ia, const int *__restrict__ ja,
               const double *__restrict__ a, const double *__restrict__ Xk,
               const double *__restrict__ Xkm1, double *__restrict__ Xkp1,
               const double *__restrict__ V0, double ctr, double sc, double *partials,
               unsigned *counter, double *mom) {
  __shared__ double acc_sh[kThreads / 32][32 * CPL];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  double acc[CPL];
#pragma unroll
  for (int q = 0; q < CPL; q++) acc[q] = 0.0;
  for (int row = blockIdx.x * wpb + wib; row < n; row += gridDim.x * wpb) {
    double r[CPL];
#pragma unroll
    for (int q = 0; q < CPL; q++) r[q] = 0.0;
    const int e = ia[row + 1];
    int j = ia[row];
    /* four entries per iteration: their loads are independent and in flight
     * together; each column still accumulates in entry order */
    for (; j + 3 < e; j += 4) {
      const double a0 = a[j], a1 = a[j + 1], a2 = a[j + 2], a3 = a[j + 3];
      const double *x0 = Xk + (size_t)ja[j] * ld, *x1 = Xk + (size_t)ja[j + 1] * ld;
      const double *x2 = Xk + (size_t)ja[j + 2] * ld, *x3 = Xk + (size_t)ja[j + 3] * ld;
#pragma unroll
      for (int q = 0; q < CPL; q++) {
        const int c = lane + 32 * q;
        if (c < s) {
          const double v0 = x0[c], v1 = x1[c], v2 = x2[c], v3 = x3[c];
          r[q] = fma(a3, v3, fma(a2, v2, fma(a1, v1, fma(a0, v0, r[q]))));
        }
      }
    }
    for (; j < e; j++) {
      const double aj = a[j];
      const double *xr = Xk + (size_t)ja[j] * ld;
#pragma unroll
      for (int q = 0; q < CPL; q++) {
        const int c = lane + 32 * q;
        if (c < s) r[q] = fma(aj, xr[c], r[q]);
      }
    }
    const size_t base = (size_t)row * ld;
#pragma unroll
    for (int q = 0; q < CPL; q++) {
      const int c = lane + 32 * q;
      if (c < s) {
        double w = (r[q] - ctr * Xk[base + c]) * sc;
        if (Xkm1) w -= Xkm1[base + c];
        Xkp1[base + c] = w;
        acc[q] = fma(w, V0[base + c], acc[q]);
      }
    }
  }
#pragma unroll
  for (int q = 0; q < CPL; q++) acc_sh[wib][lane + 32 * q] = acc[q];
  __syncthreads();
  for (int c = threadIdx.x; c < s; c += blockDim.x) {
    double t = 0.0;
    for (int w = 0; w < wpb; w++) t += acc_sh[w][c];
    partials[(size_t)blockIdx.x * s + c] = t;
  }
  /* the columns are added across blocks by k_col_reduce */
  (void)counter;
}

/* out[c] = sum_i X[i*ld + c]^2: per-block partials, last block adds them */
__global__ void k_block_colnorm2(long n, int s, int ld, const double *__restrict__ X,
                                 double *partials, unsigned *counter, double *out) {
  __shared__ double acc_sh[kThreads / 32][64];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  double acc[2] = {0.0, 0.0};
  for (long row = blockIdx.x * wpb + wib; row < n; row += (long)gridDim.x * wpb) {
    for (int q = 0; q < 2; q++) {
      const int c = lane + 32 * q;
      if (c < s) {
        const double v = X[row * ld + c];
        acc[q] = fma(v, v, acc[q]);
      }
    }
  }
  acc_sh[wib][lane] = acc[0];
  acc_sh[wib][lane + 32] = acc[1];
  __syncthreads();
  for (int c = threadIdx.x; c < s; c += blockDim.x) {
    double t = 0.0;
    for (int w = 0; w < wpb; w++) t += acc_sh[w][c];
    partials[(size_t)blockIdx.x * s + c] = t;
  }
  /* the columns are added across blocks by k_col_reduce */
  (void)counter;
}

__global__ void k_block_normalize(long n, int s, int ld, double *X, const double *nrm2) {
  const long tot = n * (long)ld;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < tot; i += (long)gridDim.x * blockDim.x) {
    const int c = (int)(i % ld);
    if (c < s) X[i] *= 1.0 / sqrt(nrm2[c]);
  }
}

#define PV_LANE_SWITCH(KERNEL, LANES, N, ...)                                                     \
  do {                                                                                           \
    const long _rows_per_block = kThreads / (LANES);                                             \
    const unsigned _g = (unsigned)(((N) + _rows_per_block - 1) / _rows_per_block);              \
    switch (LANES) {                                                                             \
      case 1: KERNEL<1><<<_g, kThreads, 0, ctx().stream>>>(__VA_ARGS__); break;                  \
      case 2: KERNEL<2><<<_g, kThreads, 0, ctx().stream>>>(__VA_ARGS__); break;                  \
      case 4: KERNEL<4><<<_g, kThreads, 0, ctx().stream>>>(__VA_ARGS__); break;                  \
      case 8: KERNEL<8><<<_g, kThreads, 0, ctx().stream>>>(__VA_ARGS__); break;                  \
      case 16: KERNEL<16><<<_g, kThreads, 0, ctx().stream>>>(__VA_ARGS__); break;                \
      default: KERNEL<32><<<_g, kThreads, 0, ctx().stream>>>(__VA_ARGS__); break;                \
    }                                                                                            \
  } while (0)

/* Autotuner of the CSR-stream kernels: on a matrix's first use, time one
 * Chebyshev degree with one and with two rows per lane (1 warm-up + 5 timed
 * launches each, CUDA events, scratch vectors of the matrix's size) and keep
 * the faster; two rows per lane must win by 3%.  Both give the same bits
 * (the per-row summation order is the same), so the choice never changes a
 * result.  PEVSL_B200_STREAM_R=1|2 fixes it; matrices under 4096 rows keep
 * one.  Must not run while the stream is being captured. */
int stream_tune(pevsl_devcsr *A) {
  if (!A || A->stream_r) return 0;
  const char *e = getenv("PEVSL_B200_STREAM_R");
  if (e && (atoi(e) == 1 || atoi(e) == 2)) {
    A->stream_r = atoi(e);
    return 0;
  }
  A->stream_r = 1;
  const long n = A->nrows;
  if (n < 4096) return 0;
  double *buf = nullptr;
  if (cudaMalloc(&buf, sizeof(double) * 4 * (size_t)n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  cudaStream_t st = ctx().stream;
  cudaMemsetAsync(buf, 0, sizeof(double) * 4 * (size_t)n, st);
  double *x = buf, *xm1 = buf + n, *xp1 = buf + 2 * n, *y = buf + 3 * n;
  const EpiCheb epi{x, xm1, xp1, y, 0.5, 0.5, 0.0, 0.5, 0};
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float ms[3] = {0.f, 0.f, 0.f};
  for (int R = 1; R <= 2; R++) {
    for (int it = 0; it < 6; it++) {
      if (it == 1) cudaEventRecord(e0, st);
      if (R == 2)
        launch_pdl(k_csr_stream<2, double, EpiCheb>, stream_grid(n, 2), st, A->nrows, A->ia, A->ja,
                   (const double *)A->a, x, epi);
      else
        launch_pdl(k_csr_stream<1, double, EpiCheb>, stream_grid(n, 1), st, A->nrows, A->ia, A->ja,
                   (const double *)A->a, x, epi);
    }
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms[R], e0, e1);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamSynchronize(st);
  cudaFree(buf);
  if (fail(cudaGetLastError(), "stream_tune")) return PEVSL_ERR_CUDA;
  ctx().launches += 12;
  if (ms[2] > 0.f && ms[2] < 0.97f * ms[1]) A->stream_r = 2;
  if (getenv("PEVSL_B200_VERBOSE"))
    fprintf(stderr, "stream_tune n=%ld: 1 row/lane %.2f us, 2 rows/lane %.2f us -> %d\n", n,
            ms[1] * 200.f, ms[2] * 200.f, A->stream_r);
  return 0;
}

/* one CSR-stream launch with the matrix's rows per lane (tuned on first use
 * when the stream is not being captured) */
/* Which kernels read the packed entries (PEVSL_B200_PACKED): 0 none, 1 the
 * one-vector kernels (default), 2 also the shared-matrix batch.  Measured
 * per filter degree at 100^3: one vector 22.3 vs 28.1 us, but 4 slices
 * 89.5 vs 79.9 us, and at 160^3 one vector 98.1 vs 99.4 us -- the kernels
 * are bound by the gathers and the vector streams more than by the matrix
 * bytes, so the packed form pays only where the working set nears L2. */
static int packed_mode() {
  static int on = -1;
  if (on < 0) {
    const char *e = getenv("PEVSL_B200_PACKED");
    on = e ? atoi(e) : 1;
    if (on < 0 || on > 2) on = 1;
  }
  return on;
}

static bool use_packed(const pevsl_devcsr *A) { return packed_mode() >= 1 && A->pdj != nullptr; }
static bool use_packed_batch(const pevsl_devcsr *A) {
  return packed_mode() == 2 && A->pdj != nullptr;
}

/* point the L2 persistence window (if enabled) at what the kernels read of
 * A's entries.  Measured with PEVSL_B200_L2PERSIST=1: no change at 100^3 or
 * 160^3 (20.2 vs 20.4 us, 96.8 vs 94.2 us per packed degree), so it stays
 * off by default. */
void matrix_window(const pevsl_devcsr *A) {
  if (!A) return;
  if (use_packed(A))
    l2_window(A->pdj, A->pbytes);
  else
    l2_window(A->a, A->bytes);
}

double entry_bytes(const pevsl_devcsr *A, bool fp32, bool batch) {
  return (batch ? use_packed_batch(A) : use_packed(A)) ? 3.0 : (fp32 ? 8.0 : 12.0);
}

template <class T>
static const T *packed_table(const pevsl_devcsr *A) {
  return sizeof(T) == 4 ? (const T *)(const void *)A->pvtab32 : (const T *)(const void *)A->pvtab;
}

template <class T, class Epi>
static void launch_stream(const pevsl_devcsr *A, const T *a, const T *x, const Epi &epi) {
  if (use_packed(A)) {
    launch_pdl(k_csr_stream_packed<T, Epi>, stream_grid(A->nrows, 1), ctx().stream, A->nrows,
               A->ia, A->pdj, A->pvi, packed_table<T>(A), A->pnv, x, epi);
    return;
  }
  if (!A->stream_r) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(ctx().stream, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone)
      stream_tune(const_cast<pevsl_devcsr *>(A));
  }
  if (stream_r(A) == 2)
    launch_pdl(k_csr_stream<2, T, Epi>, stream_grid(A->nrows, 2), ctx().stream, A->nrows, A->ia,
               A->ja, a, x, epi);
  else
    launch_pdl(k_csr_stream<1, T, Epi>, stream_grid(A->nrows, 1), ctx().stream, A->nrows, A->ia,
               A->ja, a, x, epi);
}

/* fill the table from the entries (matrices from e[i].A) and launch */
template <class T, class Epi, int CAP, class Make>
static int launch_stream_batch(int nb, const ChebEntry *en, Make make, const char *what) {
  static StreamBatch<T, Epi, CAP> b; /* host staging: the launch copies it */
  bool one = true;
  for (int i = 1; i < nb && one; i++) one = en[i].A == en[0].A;
  const int R = one ? stream_r(en[0].A) : 1;
  const long rows_per_block = (kThreads / 32) * 32L * R;
  b.nb = nb;
  b.shared = 1;
  long off = 0;
  for (int i = 0; i < nb; i++) {
    const pevsl_devcsr *A = en[i].A;
    b.ia[i] = A->ia;
    b.ja[i] = A->ja;
    b.a[i] = (const T *)(sizeof(T) == 4 ? (const void *)A->a32 : (const void *)A->a);
    b.n[i] = A->nrows;
    b.off[i] = (int)off;
    off += (A->nrows + rows_per_block - 1) / rows_per_block;
    b.epi[i] = make(en[i]);
    if (A != en[0].A) b.shared = 0;
  }
  b.off[nb] = (int)off;
  if (off <= 0) return 0;
  if (off > 0x7fffffffL) return PEVSL_ERR_ARG;
  const unsigned g = (unsigned)off;
  const int n0 = b.n[0];
  const int *ia0 = b.ia[0], *ja0 = b.ja[0];
  const T *a0 = b.a[0];
  if (b.shared && use_packed_batch(en[0].A)) {
    /* packed rows are grouped by 32 (one row group per warp) */
    const pevsl_devcsr *A = en[0].A;
    const long rb = (n0 + kThreads - 1) / kThreads;
    const unsigned gp = (unsigned)(rb * nb);
    launch_pdl(k_csr_stream_batch_packed<T, Epi, CAP>, gp, ctx().stream, n0, ia0, A->pdj, A->pvi,
               packed_table<T>(A), A->pnv, b);
  } else if (b.shared) {
    if (R == 2)
      launch_pdl(k_csr_stream_batch<2, T, Epi, CAP, true>, g, ctx().stream, n0, ia0, ja0, a0, b);
    else
      launch_pdl(k_csr_stream_batch<1, T, Epi, CAP, true>, g, ctx().stream, n0, ia0, ja0, a0, b);
  } else {
    if (R == 2)
      launch_pdl(k_csr_stream_batch<2, T, Epi, CAP, false>, g, ctx().stream, n0, ia0, ja0, a0, b);
    else
      launch_pdl(k_csr_stream_batch<1, T, Epi, CAP, false>, g, ctx().stream, n0, ia0, ja0, a0, b);
  }
  return launched(what);
}

int spmv(const pevsl_devcsr *A, const double *x, double *y) {
  if (A->nrows <= 0) return 0;
  if (A->lanes == 0) {
    launch_stream(A, (const double *)A->a, x, EpiStore{y});
    return launched("spmv_stream");
  }
  PV_LANE_SWITCH(k_spmv, A->lanes, A->nrows, A->nrows, A->ia, A->ja, A->a, x, y);
  return launched("spmv");
}

/* the ELL kernel and its switch (defined with the interleaved kernels) */
template <int S, int EW = 0>
__global__ void k_cheb_il_e(int n, const short *__restrict__ edj,
                            const unsigned char *__restrict__ evi, int ew_arg,
                            const double *__restrict__ vtab, int nv,
                            const double *__restrict__ Xk, const double *Xkm1, double *Xkp1,
                            double *Y, double cc, double t, const double *__restrict__ mu0,
                            const double *__restrict__ muk, double mu0s, double muks, int ny,
                            int fresh);
static bool ell_enabled(const pevsl_devcsr *A);
using Il1Kernel = decltype(&k_cheb_il_e<1, 0>);
static Il1Kernel il1_kernel(int ew);

int cheb_step(const pevsl_devcsr *A, const double *vk, const double *vkm1, double *vkp1, double *y,
              double cc, double t, double mu0, double muk, int first) {
  if (A->nrows <= 0) return 0;
  if (A->lanes == 0 && use_packed(A) && ell_enabled(A) && A->nrows >= 65536) {
    /* one lane per row on the ELL copy: the same bits as the stream kernel */
    const unsigned g = (unsigned)((A->nrows + kThreads - 1) / kThreads);
    launch_pdl(il1_kernel(A->ew), g, ctx().stream, A->nrows, A->edj, A->evi, A->ew, A->pvtab, A->pnv,
               vk, vkm1, vkp1, y, cc, t, nullptr, nullptr, mu0, muk, 1, first);
    return launched("cheb_step_ell");
  }
  if (A->lanes == 0) {
    launch_stream(A, (const double *)A->a, vk, EpiCheb{vk, vkm1, vkp1, y, cc, t, mu0, muk, first});
    return launched("cheb_step_stream");
  }
  PV_LANE_SWITCH(k_cheb_step, A->lanes, A->nrows, A->nrows, A->ia, A->ja, A->a, vk, vkm1, vkp1, y,
                 cc, t, mu0, muk, first);
  return launched("cheb_step");
}

int cheb_step_x(const pevsl_devcsr *A, const double *x, const double *vk, const double *vkm1,
                double *vkp1, double *y, double cc, double t, double mu0, double muk, int first,
                double *tmp) {
  if (A->nrows <= 0) return 0;
  if (A->lanes == 0) {
    launch_stream(A, (const double *)A->a, x, EpiCheb{vk, vkm1, vkp1, y, cc, t, mu0, muk, first});
    return launched("cheb_step_x");
  }
  if (spmv(A, x, tmp)) return PEVSL_ERR_CUDA;
  return cheb_combine(A->nrows, tmp, vk, vkm1, vkp1, y, cc, t, mu0, muk, first);
}

int chebiter1_step(const pevsl_devcsr *B, const double *b, const double *x, double *p, double *xnew,
                   double bet, double alp, double *tmp) {
  const long n = B->nrows;
  if (n <= 0) return 0;
  if (B->lanes == 0) {
    launch_stream(B, (const double *)B->a, x, EpiChebIter1{b, x, p, xnew, bet, alp});
    return launched("chebiter1_step");
  }
  if (spmv(B, x, tmp)) return PEVSL_ERR_CUDA;
  k_chebiter1_combine<<<grid_for(n, 4), kThreads, 0, ctx().stream>>>(n, tmp, b, x, p, xnew, bet, alp);
  return launched("chebiter1_combine");
}

int chebiter2_step(const pevsl_devcsr *B, const double *d, double *x, double *r, double *dnew,
                   double c1, double c2, double *tmp) {
  const long n = B->nrows;
  if (n <= 0) return 0;
  if (B->lanes == 0) {
    launch_stream(B, (const double *)B->a, d, EpiChebIter2{d, x, r, dnew, c1, c2});
    return launched("chebiter2_step");
  }
  if (spmv(B, d, tmp)) return PEVSL_ERR_CUDA;
  k_chebiter2_combine<<<grid_for(n, 4), kThreads, 0, ctx().stream>>>(n, tmp, d, x, r, dnew, c1, c2);
  return launched("chebiter2_combine");
}

/* ---------------------------------------------------------------- interleaved
 * One filter degree for S (2..16) vectors of one problem held row-interleaved
 * (X[i*S + s]): S lanes serve one row, lane s its vector s.  For each entry
 * the S lanes read x[col*S .. col*S+S-1] -- one contiguous segment -- so a
 * scattered column costs one L1/L2 access for all S vectors instead of one
 * per vector.  Lane s adds its row's products in entry order and applies
 * the recurrence of its own column (cheb_update_v's arithmetic with its own
 * mu), which is the arithmetic of the one-vector kernel, bit for bit.  X_{k+1} may alias
 * X_{k-1} (each lane reads its own element first).  The SpMV reads Xg,
 * which is Xk except in the generalized filter (Xg = B^{-1} X_k).
 *
 * The accumulator may be deferred (ny, fresh: cheb_step_il_y).  A launch
 * holds v_k (the new value), v_{k-1} and v_{k-2} in registers anyway, so
 * the terms of up to three degrees can be added in one launch: the launches
 * in between neither read nor write Y, 16 of 40 bytes per row and slice. */
template <int S>
__device__ __forceinline__ double il_accumulate(int ny, int fresh, double yold, double w,
                                                double x, double xm1, const double *mu0,
                                                const double *muk, int s) {
  double y = fresh ? __dmul_rn(mu0[s], ny == 1 ? x : xm1) : yold;
  if (ny >= 3) y = __fma_rn(muk[s - 2 * S], xm1, y);
  if (ny >= 2) y = __fma_rn(muk[s - S], x, y);
  return __fma_rn(muk[s], w, y);
}

template <int S>
__global__ void __launch_bounds__(kThreads)
    k_cheb_il(int n, const int *__restrict__ ia, const int *__restrict__ ja,
              const double *__restrict__ a, const double *__restrict__ Xg,
              const double *__restrict__ Xk, const double *Xkm1, double *Xkp1, double *Y, double cc,
              double t, const double *__restrict__ mu0, const double *__restrict__ muk, int ny,
              int fresh) {
  constexpr int RPW = 32 / S; /* rows per warp */
  const long gw = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31, s = lane % S;
  const long row = gw * RPW + lane / S;
  if (row >= n) return;
  const size_t me = (size_t)row * S + s;
  const double x = Xk[me];
  const double xm1 = Xkm1 ? Xkm1[me] : 0.0;
  const int e = __ldg(ia + row + 1);
  double r = 0.0;
  int j = __ldg(ia + row);
  for (; j + 3 < e; j += 4) {
    const int c0 = __ldg(ja + j), c1 = __ldg(ja + j + 1), c2 = __ldg(ja + j + 2), c3 = __ldg(ja + j + 3);
    const double a0 = __ldg(a + j), a1 = __ldg(a + j + 1), a2 = __ldg(a + j + 2), a3 = __ldg(a + j + 3);
    const double x0 = __ldg(Xg + (size_t)c0 * S + s), x1 = __ldg(Xg + (size_t)c1 * S + s);
    const double x2 = __ldg(Xg + (size_t)c2 * S + s), x3 = __ldg(Xg + (size_t)c3 * S + s);
    r = __dadd_rn(r, __dmul_rn(a0, x0));
    r = __dadd_rn(r, __dmul_rn(a1, x1));
    r = __dadd_rn(r, __dmul_rn(a2, x2));
    r = __dadd_rn(r, __dmul_rn(a3, x3));
  }
  for (; j < e; j++) r = __dadd_rn(r, __dmul_rn(__ldg(a + j), __ldg(Xg + (size_t)__ldg(ja + j) * S + s)));
  double w = __dmul_rn(__fma_rn(-cc, x, r), t);
  if (Xkm1) w = __dsub_rn(w, xm1);
  Xkp1[me] = w;
  /* y is loaded here, not before the gathers: held across the loop it
   * takes this kernel from 32 to 40 registers (6 instead of 8 blocks per
   * SM), and only the launches that update y load it */
  if (ny > 0) Y[me] = il_accumulate<S>(ny, fresh, fresh ? 0.0 : Y[me], w, x, xm1, mu0, muk, s);
}

/* k_cheb_il on the packed entries (int16 column offset from the row's
 * 32-row group, uint8 index into the value table staged in shared memory):
 * the same products in the same order */
template <int S>
__global__ void __launch_bounds__(kThreads)
    k_cheb_il_p(int n, const int *__restrict__ ia, const short *__restrict__ dj,
                const unsigned char *__restrict__ vi, const double *__restrict__ vtab, int nv,
                const double *__restrict__ Xg, const double *__restrict__ Xk, const double *Xkm1,
                double *Xkp1, double *Y, double cc, double t, const double *__restrict__ mu0,
                const double *__restrict__ muk, int ny, int fresh) {
  __shared__ double vt[256];
  for (int i = threadIdx.x; i < nv; i += blockDim.x) vt[i] = vtab[i];
  __syncthreads();
  pdl_wait_then_release();
  constexpr int RPW = 32 / S;
  const long gw = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31, s = lane % S;
  const long row = gw * RPW + lane / S;
  if (row >= n) return;
  const int g0 = (int)(row & ~31L);
  const size_t me = (size_t)row * S + s;
  const double x = Xk[me];
  const double xm1 = Xkm1 ? Xkm1[me] : 0.0;
  const double yold = (ny > 0 && !fresh) ? Y[me] : 0.0;
  const int e = __ldg(ia + row + 1);
  double r = 0.0;
  int j = __ldg(ia + row);
  for (; j + 3 < e; j += 4) {
    const int c0 = g0 + __ldg(dj + j), c1 = g0 + __ldg(dj + j + 1);
    const int c2 = g0 + __ldg(dj + j + 2), c3 = g0 + __ldg(dj + j + 3);
    const double a0 = vt[__ldg(vi + j)], a1 = vt[__ldg(vi + j + 1)];
    const double a2 = vt[__ldg(vi + j + 2)], a3 = vt[__ldg(vi + j + 3)];
    const double x0 = __ldg(Xg + (size_t)c0 * S + s), x1 = __ldg(Xg + (size_t)c1 * S + s);
    const double x2 = __ldg(Xg + (size_t)c2 * S + s), x3 = __ldg(Xg + (size_t)c3 * S + s);
    r = __dadd_rn(r, __dmul_rn(a0, x0));
    r = __dadd_rn(r, __dmul_rn(a1, x1));
    r = __dadd_rn(r, __dmul_rn(a2, x2));
    r = __dadd_rn(r, __dmul_rn(a3, x3));
  }
  for (; j < e; j++)
    r = __dadd_rn(r, __dmul_rn(vt[__ldg(vi + j)], __ldg(Xg + (size_t)(g0 + __ldg(dj + j)) * S + s)));
  double w = __dmul_rn(__fma_rn(-cc, x, r), t);
  if (Xkm1) w = __dsub_rn(w, xm1);
  Xkp1[me] = w;
  if (ny > 0) Y[me] = il_accumulate<S>(ny, fresh, yold, w, x, xm1, mu0, muk, s);
}

/* k_cheb_il_p on the ELL copy of the packed entries: row r's j-th entry
 * sits at (r / 32) * 32 * ew + j * 32 + r % 32, so a lane computes its
 * entries' addresses from its row alone and issues their loads together
 * with the vector loads -- the row-pointer load and the wait on it are
 * gone -- then up to eight gathers at once.  Padding (edj = INT16_MIN)
 * follows a row's entries and is skipped, never added, so the products are
 * added in the same order as k_cheb_il_p's: the same bits.  S = 1 is the
 * one-vector degree (y updated every degree with the scalar mu0s / muks,
 * the arithmetic of cheb_update_v). */
/* Idx: the type of the slot offsets -- 32-bit where the width is fixed at
 * compile time (every offset is b plus a constant), 64-bit in the loop over
 * any width (measured: 11.6 against 15.2 us per one-vector degree at 100^3
 * with 32-bit offsets there) */
template <int B, int S, class Idx>
__device__ __forceinline__ void il_entries(int j0, int ew, const short *__restrict__ edj,
                                           const unsigned char *__restrict__ evi, Idx b,
                                           const double *__restrict__ Xk, int g0, int s,
                                           const double *vt, double &r) {
  int dv[B];
  unsigned iv[B];
  double xv[B];
#pragma unroll
  for (int u = 0; u < B; u++) {
    dv[u] = INT16_MIN;
    iv[u] = 0;
    if (j0 + u < ew) {
      dv[u] = __ldg(edj + (b + (Idx)(j0 + u) * 32));
      iv[u] = __ldg(evi + (b + (Idx)(j0 + u) * 32));
    }
  }
#pragma unroll
  for (int u = 0; u < B; u++)
    xv[u] = dv[u] != INT16_MIN ? __ldg(Xk + ((size_t)(g0 + dv[u]) * S + s)) : 0.0;
#pragma unroll
  for (int u = 0; u < B; u++)
    if (dv[u] != INT16_MIN) r = __dadd_rn(r, __dmul_rn(vt[iv[u]], xv[u]));
}

/* EW > 0: the ELL width fixed at compile time, as in k_cheb_il2_e.  One
 * vector: built for eight blocks per SM (32 registers). */
template <int S, int EW>
__global__ void __launch_bounds__(kThreads, S == 1 ? 8 : 1)
    k_cheb_il_e(int n, const short *__restrict__ edj, const unsigned char *__restrict__ evi,
                int ew_arg, const double *__restrict__ vtab, int nv, const double *__restrict__ Xk,
                const double *Xkm1, double *Xkp1, double *Y, double cc, double t,
                const double *__restrict__ mu0, const double *__restrict__ muk, double mu0s,
                double muks, int ny, int fresh) {
  const int ew = EW > 0 ? EW : ew_arg;
  __shared__ double vt[256];
  for (int i = threadIdx.x; i < nv; i += blockDim.x) vt[i] = vtab[i];
  __syncthreads();
  pdl_wait_then_release();
  constexpr int RPW = 32 / S;
  const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31, s = lane % S;
  const int row = gw * RPW + lane / S;
  if (row >= n) return;
  const size_t me = (size_t)row * S + s;
  const bool read_y = S == 1 ? !fresh : (ny > 0 && !fresh);
  const double x = Xk[me];
  const double xm1 = Xkm1 ? Xkm1[me] : 0.0;
  const double yold = read_y ? Y[me] : 0.0;
  const int g0 = row & ~31;
  double r = 0.0;
  if constexpr (EW > 0) {
    const unsigned b = (unsigned)(row >> 5) * 32u * (unsigned)EW + (unsigned)(row & 31);
#pragma unroll
    for (int j0 = 0; j0 < EW; j0 += 8) il_entries<8, S>(j0, EW, edj, evi, b, Xk, g0, s, vt, r);
  } else {
    const size_t b = (size_t)(row >> 5) * 32 * (size_t)ew + (size_t)(row & 31);
    for (int j0 = 0; j0 < ew; j0 += 8) il_entries<8, S>(j0, ew, edj, evi, b, Xk, g0, s, vt, r);
  }
  double w = __dmul_rn(__fma_rn(-cc, x, r), t);
  if (Xkm1) w = __dsub_rn(w, xm1);
  Xkp1[me] = w;
  if (S == 1)
    Y[me] = fresh ? __fma_rn(muks, w, __dmul_rn(mu0s, x)) : __fma_rn(muks, w, yold);
  else if (ny > 0)
    Y[me] = il_accumulate<S>(ny, fresh, yold, w, x, xm1, mu0, muk, s);
}

/* Two interleaved vectors on the ELL copy with one thread per row: each
 * gather is one 16-byte load of both vectors' entries (X as double2), each
 * entry's offset and value index are loaded once for both, and the two
 * products of an entry go to two sums, each added in entry order -- the
 * bits of k_cheb_il_p<2>.  Four entries per batch of gathers, 48 registers,
 * five blocks per SM.  Measured per degree at 100^3 on one box: 19.8 us;
 * built for six blocks (40 registers, Y loaded after the gathers) 20.2-21.1
 * us, for eight (32 registers, spills) 24.7-28.1 us; eight entries per
 * batch (63 registers, spills) 28.3 us. */
template <int B>
__device__ __forceinline__ void il2_entries(int j0, int ew, const short *__restrict__ edj,
                                            const unsigned char *__restrict__ evi, unsigned b,
                                            const double2 *__restrict__ Xk, int g0,
                                            const double *vt, double &r0, double &r1) {
  int dv[B];
  unsigned iv[B];
  double2 xv[B];
#pragma unroll
  for (int u = 0; u < B; u++) {
    dv[u] = INT16_MIN;
    iv[u] = 0;
    if (j0 + u < ew) {
      dv[u] = __ldg(edj + (b + (unsigned)(j0 + u) * 32u));
      iv[u] = __ldg(evi + (b + (unsigned)(j0 + u) * 32u));
    }
  }
#pragma unroll
  for (int u = 0; u < B; u++)
    xv[u] = dv[u] != INT16_MIN ? __ldg(Xk + (g0 + dv[u])) : make_double2(0.0, 0.0);
#pragma unroll
  for (int u = 0; u < B; u++)
    if (dv[u] != INT16_MIN) {
      const double a = vt[iv[u]];
      r0 = __dadd_rn(r0, __dmul_rn(a, xv[u].x));
      r1 = __dadd_rn(r1, __dmul_rn(a, xv[u].y));
    }
}

/* EW > 0: the ELL width fixed at compile time (the common stencil widths
 * 5 and 7), so the entry loop unrolls completely, with no width tests, and
 * each entry's slot is b plus a constant; EW = 0: any width.  Offsets are
 * 32-bit: the set-up builds the ELL copy only below 2^31 slots.  Measured at
 * 100^3 (width 7), same box: 16.4-16.6 us per degree against 19.2-22.3 us
 * for the any-width build with 64-bit offsets; the whole C2 solve 30.4
 * against 35.3 s. */
template <int EW>
__global__ void __launch_bounds__(kThreads, 5)
    k_cheb_il2_e(int n, const short *__restrict__ edj, const unsigned char *__restrict__ evi,
                 int ew_arg, const double *__restrict__ vtab, int nv,
                 const double2 *__restrict__ Xk, const double2 *Xkm1, double2 *Xkp1, double2 *Y,
                 double cc, double t, const double *__restrict__ mu0,
                 const double *__restrict__ muk, int ny, int fresh) {
  const int ew = EW > 0 ? EW : ew_arg;
  __shared__ double vt[256];
  for (int i = threadIdx.x; i < nv; i += blockDim.x) vt[i] = vtab[i];
  __syncthreads();
  pdl_wait_then_release();
  const int row = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (row >= n) return;
  const double2 x = Xk[row];
  const double2 xm1 = Xkm1 ? Xkm1[row] : make_double2(0.0, 0.0);
  const double2 yold = (ny > 0 && !fresh) ? Y[row] : make_double2(0.0, 0.0);
  const unsigned b = (unsigned)(row >> 5) * 32u * (unsigned)ew + (unsigned)(row & 31);
  const int g0 = row & ~31;
  constexpr int B = 4;
  double r0 = 0.0, r1 = 0.0;
  if constexpr (EW > 0) {
#pragma unroll
    for (int j0 = 0; j0 < EW; j0 += B) il2_entries<B>(j0, EW, edj, evi, b, Xk, g0, vt, r0, r1);
  } else {
    for (int j0 = 0; j0 < ew; j0 += B) il2_entries<B>(j0, ew, edj, evi, b, Xk, g0, vt, r0, r1);
  }
  double w0 = __dmul_rn(__fma_rn(-cc, x.x, r0), t);
  double w1 = __dmul_rn(__fma_rn(-cc, x.y, r1), t);
  if (Xkm1) {
    w0 = __dsub_rn(w0, xm1.x);
    w1 = __dsub_rn(w1, xm1.y);
  }
  Xkp1[row] = make_double2(w0, w1);
  if (ny > 0)
    Y[row] = make_double2(il_accumulate<2>(ny, fresh, yold.x, w0, x.x, xm1.x, mu0, muk, 0),
                          il_accumulate<2>(ny, fresh, yold.y, w1, x.y, xm1.y, mu0, muk, 1));
}

/* PEVSL_B200_ELL_W: 1 (default) the ELL kernels compiled for the matrix's
 * width where it is a common stencil width (5 or 7), 0 the any-width
 * kernels.  Same results either way. */
static int ell_fixed_width() {
  static int v = -1;
  if (v < 0) {
    const char *e = getenv("PEVSL_B200_ELL_W");
    v = e ? atoi(e) != 0 : 1;
  }
  return v;
}

using Il2Kernel = decltype(&k_cheb_il2_e<0>);

static Il1Kernel il1_kernel(int ew) {
  if (ell_fixed_width() && ew == 7) return k_cheb_il_e<1, 7>;
  if (ell_fixed_width() && ew == 5) return k_cheb_il_e<1, 5>;
  return k_cheb_il_e<1, 0>;
}

static Il2Kernel il2_kernel(int ew) {
  if (ell_fixed_width() && ew == 7) return k_cheb_il2_e<7>;
  if (ell_fixed_width() && ew == 5) return k_cheb_il2_e<5>;
  return k_cheb_il2_e<0>;
}

/* Which filter-degree form runs, where the matrix has the ELL copy.  One
 * vector: k_cheb_il_e<1> or the CSR-stream kernel; groups of two:
 * k_cheb_il2_e or k_cheb_il_p<2> -- each chosen per matrix by timing both
 * on this GPU at set-up (filter_tune; measured at 100^3 with the any-width
 * ELL builds: one vector 11.8 against 20.8 us, groups of two 19.7-21.3
 * against 19.8-25.2 us from box to box; the width-7 builds: 11.4 and
 * 16.4-16.6 us).  Under a profiler that serialises launches the timings
 * are not a run's: force the forms there.  PEVSL_B200_ELL: 0 never ELL, 1 always (and k_cheb_il_e<S> for
 * wider groups, measured 21.0 against 19.8 us at two); PEVSL_B200_ELL2:
 * 0 / 1 forces the form of the groups of two. */
static int ell_mode() {
  static int v = -2;
  if (v == -2) {
    const char *e = getenv("PEVSL_B200_ELL");
    v = e ? atoi(e) : -1;
  }
  return v;
}
static int ell2_mode() {
  static int v = -2;
  if (v == -2) {
    const char *e = getenv("PEVSL_B200_ELL2");
    v = e ? (atoi(e) != 0) : -1;
  }
  return v;
}
static bool ell_enabled(const pevsl_devcsr *A) {
  if (!A->edj || ell_mode() == 0) return false;
  return ell_mode() > 0 || A->ell1;
}
static bool ell_multi(const pevsl_devcsr *A) { return ell_mode() > 0 && A->edj != nullptr; }
static bool ell_two(const pevsl_devcsr *A) {
  if (!A->edj || ell_mode() == 0) return false;
  if (ell2_mode() >= 0) return ell2_mode() == 1;
  return ell_mode() > 0 || A->ell2;
}

/* Choose the filter-degree forms of a packed matrix with an ELL copy by
 * timing both on this GPU: one vector (CSR-stream against k_cheb_il_e<1>)
 * and groups of two interleaved vectors (k_cheb_il_p<2> against
 * k_cheb_il2_e), ten launches each after three warm-up ones, two rounds in
 * alternating order, on scratch vectors.  Both forms give the same bits, so
 * the choice never changes a result.  Runs at set-up, outside any capture;
 * about 2 ms at 100^3. */
int filter_tune(pevsl_devcsr *A) {
  A->ell1 = A->ell2 = 0;
  if (!A->edj || A->nrows < 65536) return 0;
  if (ell_mode() == 0) return 0;
  if (ell_mode() > 0) {
    A->ell1 = A->ell2 = 1;
    return 0;
  }
  const long n = A->nrows;
  double *buf = nullptr;
  if (cudaMalloc(&buf, sizeof(double) * (8 * (size_t)n + 64)) != cudaSuccess) {
    cudaGetLastError();
    A->ell1 = A->ell2 = 1; /* untimed: the forms measured faster */
    return 0;
  }
  cudaStream_t st = ctx().stream;
  cudaMemsetAsync(buf, 0, sizeof(double) * (8 * (size_t)n + 64), st);
  double *X = buf, *Xm = buf + 2 * n, *Xp = buf + 4 * n, *Y = buf + 6 * n, *mu = buf + 8 * n;
  const unsigned g1 = (unsigned)((n + kThreads - 1) / kThreads);
  const unsigned g2 = (unsigned)((n + (kThreads / 2) - 1) / (kThreads / 2));
  const EpiCheb epi{X, Xm, Xp, Y, 0.5, 0.5, 0.0, 0.5, 0};
  auto one_csr = [&] {
    launch_pdl(k_csr_stream_packed<double, EpiCheb>, stream_grid(A->nrows, 1), st, A->nrows, A->ia,
               A->pdj, A->pvi, A->pvtab, A->pnv, X, epi);
  };
  auto one_ell = [&] {
    launch_pdl(il1_kernel(A->ew), g1, st, A->nrows, A->edj, A->evi, A->ew, A->pvtab, A->pnv, X, Xm,
               Xp, Y, 0.5, 0.5, nullptr, nullptr, 0.0, 0.5, 1, 0);
  };
  auto two_csr = [&] {
    k_cheb_il_p<2><<<g2, kThreads, 0, st>>>(A->nrows, A->ia, A->pdj, A->pvi, A->pvtab, A->pnv, X,
                                            X, Xm, Xp, Y, 0.5, 0.5, mu, mu + 2, 0, 0);
  };
  auto two_ell = [&] {
    launch_pdl(il2_kernel(A->ew), g1, st, A->nrows, A->edj, A->evi, A->ew, A->pvtab, A->pnv,
               (const double2 *)X, (const double2 *)Xm, (double2 *)Xp, (double2 *)Y, 0.5, 0.5, mu,
               mu + 2, 0, 0);
  };
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  auto timed = [&](auto &&launch) {
    for (int i = 0; i < 3; i++) launch();
    cudaEventRecord(e0, st);
    for (int i = 0; i < 10; i++) launch();
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms;
  };
  float t1c = 0.f, t1e = 0.f, t2c = 0.f, t2e = 0.f;
  for (int round = 0; round < 2; round++) {
    if (round == 0) {
      t1c += timed(one_csr);
      t1e += timed(one_ell);
      t2c += timed(two_csr);
      t2e += timed(two_ell);
    } else {
      t1e += timed(one_ell);
      t1c += timed(one_csr);
      t2e += timed(two_ell);
      t2c += timed(two_csr);
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamSynchronize(st);
  cudaFree(buf);
  if (fail(cudaGetLastError(), "filter_tune")) return PEVSL_ERR_CUDA;
  ctx().launches += 4 * 2 * 13;
  A->ell1 = t1e > 0.f && t1e < t1c;
  A->ell2 = t2e > 0.f && t2e < t2c;
  if (getenv("PEVSL_B200_VERBOSE"))
    fprintf(stderr,
            "filter_tune n=%ld: one vector CSR %.2f / ELL %.2f us, two vectors CSR %.2f / ELL "
            "%.2f us -> ell1 %d ell2 %d\n",
            n, t1c * 50.f, t1e * 50.f, t2c * 50.f, t2e * 50.f, A->ell1, A->ell2);
  return 0;
}

/* X[i*S + s] = x_s[i] and back */
__global__ void k_il_pack(long n, int S, CPtrs xs, double *X) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n * S;
       i += (long)gridDim.x * blockDim.x)
    X[i] = xs.p[i % S][i / S];
}

__global__ void k_il_unpack(long n, int S, int cols, const double *X, VPtrs ys) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n * S;
       i += (long)gridDim.x * blockDim.x)
    if ((int)(i % S) < cols) ys.p[i % S][i / S] = X[i];
}

int il_pack(long n, int S, const double *const *xs, double *X) {
  if (S < 1 || S > kMaxBatch) return PEVSL_ERR_ARG;
  CPtrs p{};
  for (int s = 0; s < S; s++) p.p[s] = xs[s];
  k_il_pack<<<grid_for(n * S, 4), kThreads, 0, ctx().stream>>>(n, S, p, X);
  return launched("il_pack");
}

int il_unpack(long n, int S, int cols, const double *X, double *const *ys) {
  if (S < 1 || S > kMaxBatch || cols < 1 || cols > S) return PEVSL_ERR_ARG;
  VPtrs p{};
  for (int s = 0; s < cols; s++) p.p[s] = ys[s];
  k_il_unpack<<<grid_for(n * S, 4), kThreads, 0, ctx().stream>>>(n, S, cols, X, p);
  return launched("il_unpack");
}

/* S is padded up to 2, 4, 8 or 16 by the caller (unused columns are zero) */
int cheb_step_il(const pevsl_devcsr *A, int S, const double *Xk, const double *Xkm1, double *Xkp1,
                 double *Y, double cc, double t, const double *mu0, const double *muk, int first) {
  return cheb_step_il_x(A, S, Xk, Xk, Xkm1, Xkp1, Y, cc, t, mu0, muk, first);
}

/* packed entries in the interleaved kernel (PEVSL_B200_IL_PACKED: 1 on, the
 * default; 0 off).  Measured per degree at 100^3: 2 slices 20.6 vs 33.7 us,
 * 4 slices 47.5 vs 51.1 us, 16 slices 172.8 vs 174.0 us; 160^3, 4 slices
 * 183.5 vs 200.8 us. */
static bool il_packed(const pevsl_devcsr *A) {
  static int v = -1;
  if (v < 0) {
    const char *e = getenv("PEVSL_B200_IL_PACKED");
    v = e ? atoi(e) != 0 : 1;
  }
  /* small matrices (the generalized path's lockstep, L2-resident) keep the
   * plain kernel: the table staging costs more than it saves there
   * (genlap24: 53.3 vs 49.5 us per degree) */
  return v && A->pdj != nullptr && packed_mode() >= 1 && A->nrows >= 65536;
}

double il_entry_bytes(const pevsl_devcsr *A) { return il_packed(A) ? 3.0 : 12.0; }

int cheb_step_il_x(const pevsl_devcsr *A, int S, const double *Xg, const double *Xk,
                   const double *Xkm1, double *Xkp1, double *Y, double cc, double t,
                   const double *mu0, const double *muk, int first) {
  return cheb_step_il_y(A, S, Xg, Xk, Xkm1, Xkp1, Y, cc, t, mu0, muk, 1, first);
}

int cheb_step_il_y(const pevsl_devcsr *A, int S, const double *Xg, const double *Xk,
                   const double *Xkm1, double *Xkp1, double *Y, double cc, double t,
                   const double *mu0, const double *muk, int ny, int fresh) {
  /* the terms must exist: ny - 1 earlier mu rows (from row 0 on) and the
   * vectors they multiply; a fresh sum starts at degree 1 or 2 */
  if (ny < 0 || ny > 3 || muk - (size_t)(ny > 0 ? ny - 1 : 0) * S < mu0) return PEVSL_ERR_ARG;
  if (ny == 3 && !Xkm1) return PEVSL_ERR_ARG;
  if (fresh && (ny < 1 || ny > 2 || (ny == 2 && !Xkm1) || muk != mu0 + (size_t)ny * S))
    return PEVSL_ERR_ARG;
  const long rows_per_block = (kThreads / 32) * (32 / S);
  const unsigned g = (unsigned)((A->nrows + rows_per_block - 1) / rows_per_block);
  cudaStream_t st = ctx().stream;
  if (Xg == Xk && il_packed(A) && S == 2 && ell_two(A)) {
    const unsigned g2 = (unsigned)((A->nrows + kThreads - 1) / kThreads);
    launch_pdl(il2_kernel(A->ew), g2, st, A->nrows, A->edj, A->evi, A->ew, A->pvtab, A->pnv,
               (const double2 *)Xk, (const double2 *)Xkm1, (double2 *)Xkp1, (double2 *)Y, cc, t,
               mu0, muk, ny, fresh);
    return launched("cheb_step_il2_ell");
  }
  if (Xg == Xk && il_packed(A) && ell_multi(A)) {
#define PV_IL_E(SS)                                                                             \
  launch_pdl(k_cheb_il_e<SS>, g, st, A->nrows, A->edj, A->evi, A->ew, A->pvtab, A->pnv, Xk, Xkm1, \
             Xkp1, Y, cc, t, mu0, muk, 0.0, 0.0, ny, fresh)
    switch (S) {
      case 2: PV_IL_E(2); break;
      case 4: PV_IL_E(4); break;
      case 8: PV_IL_E(8); break;
      case 16: PV_IL_E(16); break;
      default: return PEVSL_ERR_ARG;
    }
#undef PV_IL_E
    return launched("cheb_step_il_ell");
  }
  if (il_packed(A)) {
#define PV_IL_P(SS)                                                                          \
  k_cheb_il_p<SS><<<g, kThreads, 0, st>>>(A->nrows, A->ia, A->pdj, A->pvi, A->pvtab, A->pnv, \
                                          Xg, Xk, Xkm1, Xkp1, Y, cc, t, mu0, muk, ny, fresh)
    switch (S) {
      case 2: PV_IL_P(2); break;
      case 4: PV_IL_P(4); break;
      case 8: PV_IL_P(8); break;
      case 16: PV_IL_P(16); break;
      default: return PEVSL_ERR_ARG;
    }
#undef PV_IL_P
    return launched("cheb_step_il_packed");
  }
#define PV_IL(SS)                                                                            \
  k_cheb_il<SS><<<g, kThreads, 0, st>>>(A->nrows, A->ia, A->ja, A->a, Xg, Xk, Xkm1, Xkp1, Y, cc, \
                                        t, mu0, muk, ny, fresh)
  switch (S) {
    case 2: PV_IL(2); break;
    case 4: PV_IL(4); break;
    case 8: PV_IL(8); break;
    case 16: PV_IL(16); break;
    default: return PEVSL_ERR_ARG;
  }
#undef PV_IL
  return launched("cheb_step_il");
}

int cheb_step_batch(int nb, const ChebEntry *e, bool fp32) {
  if (nb <= 0) return 0;
  if (nb > kMaxEntries) return PEVSL_ERR_ARG;
  if (fp32) {
    for (int i = 0; i < nb; i++)
      if (!e[i].A->a32) return PEVSL_ERR_ARG;
    auto mk = [](const ChebEntry &c) {
      return EpiCheb32{(const float *)c.vk, (const float *)c.vkm1, (float *)c.vkp1, (float *)c.y,
                       c.yout, (float)c.cc, (float)c.t, (float)c.mu0, (float)c.muk, c.first};
    };
    return nb <= kMaxBatch
               ? launch_stream_batch<float, EpiCheb32, kMaxBatch>(nb, e, mk, "cheb_step_batch32")
               : launch_stream_batch<float, EpiCheb32, kMaxEntries>(nb, e, mk, "cheb_step_batch32");
  }
  auto mk = [](const ChebEntry &c) {
    return EpiCheb{(const double *)c.vk, (const double *)c.vkm1, (double *)c.vkp1, (double *)c.y,
                   c.cc, c.t, c.mu0, c.muk, c.first};
  };
  return nb <= kMaxBatch
             ? launch_stream_batch<double, EpiCheb, kMaxBatch>(nb, e, mk, "cheb_step_batch")
             : launch_stream_batch<double, EpiCheb, kMaxEntries>(nb, e, mk, "cheb_step_batch");
}

int cheb_combine(long n, const double *ax, const double *vk, const double *vkm1, double *vkp1,
                 double *y, double cc, double t, double mu0, double muk, int first) {
  if (n <= 0) return 0;
  k_cheb_combine<<<grid_for(n, 4), kThreads, 0, ctx().stream>>>(n, ax, vk, vkm1, vkp1, y, cc, t,
                                                                 mu0, muk, first);
  return launched("cheb_combine");
}

/* out[c] = sum over nb blocks of partials[b*s + c]: one block per column,
 * thread t adds blocks t, t + 256, ... and a fixed tree adds the threads */
__global__ void k_col_reduce(const double *__restrict__ partials, int nb, int s, double *out) {
  __shared__ double sh[32];
  const int c = blockIdx.x;
  double t = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) t += partials[(size_t)b * s + c];
  t = block_sum(t, sh);
  if (threadIdx.x == 0) out[c] = t;
}

int col_reduce(const double *partials, int nb, int s, double *out) {
  k_col_reduce<<<s, kThreads, 0, ctx().stream>>>(partials, nb, s, out);
  return launched("col_reduce");
}

static unsigned warp_row_grid(long n) {
  const long wpb = kThreads / 32;
  long g = (n + wpb - 1) / wpb;
  if (g > kMaxRedBlocks) g = kMaxRedBlocks;
  return (unsigned)(g < 1 ? 1 : g);
}

int kpm_step(const pevsl_devcsr *A, int s, int ld, const double *Xk, const double *Xkm1,
             double *Xkp1, const double *V0, double ctr, double sc, double *mom) {
  if (s < 1 || s > 64) return PEVSL_ERR_ARG;
  const unsigned g = warp_row_grid(A->nrows);
  if (s <= 32) {
    k_kpm_step<1><<<g, kThreads, 0, ctx().stream>>>(A->nrows, s, ld, A->ia, A->ja, A->a, Xk, Xkm1,
                                                    Xkp1, V0, ctr, sc, ctx().red, ctx().cnt, mom);
  } else {
    k_kpm_step<2><<<g, kThreads, 0, ctx().stream>>>(A->nrows, s, ld, A->ia, A->ja, A->a, Xk, Xkm1,
                                                    Xkp1, V0, ctr, sc, ctx().red, ctx().cnt, mom);
  }
  if (launched("kpm_step")) return PEVSL_ERR_CUDA;
  return col_reduce(ctx().red, (int)g, s, mom);
}

int block_colnorm2(long n, int s, int ld, const double *X, double *out) {
  if (s < 1 || s > 64) return PEVSL_ERR_ARG;
  const unsigned g = warp_row_grid(n);
  k_block_colnorm2<<<g, kThreads, 0, ctx().stream>>>(n, s, ld, X, ctx().red, ctx().cnt, out);
  if (launched("block_colnorm2")) return PEVSL_ERR_CUDA;
  return col_reduce(ctx().red, (int)g, s, out);
}

int block_normalize(long n, int s, int ld, double *X, const double *nrm2) {
  k_block_normalize<<<grid_for(n * ld, 4), kThreads, 0, ctx().stream>>>(n, s, ld, X, nrm2);
  return launched("block_normalize");
}

}  // namespace pv

/* ================================================================ parcsr API */
using namespace pv;

/* 0 selects the CSR-stream kernels (rows up to ~24 entries on average);
 * longer rows get a group of L lanes per row, L the next power of two. */
static int choose_lanes(double avg) {
  if (avg <= 24.0) return 0;
  int L = 1;
  while (L < 32 && L < avg) L <<= 1;
  return L;
}

static void *alloc_dev(size_t bytes) {
  void *p = nullptr;
  if (fail(cudaMalloc(&p, bytes ? bytes : 16), "cudaMalloc matrix")) return nullptr;
  return p;
}

extern "C" {

pevsl_devcsr *pevsl_devcsr_of(const pevsl_Parcsr *A) {
  if (!A || !A->comm_handle) return nullptr;
  pevsl_devcsr *d = (pevsl_devcsr *)A->comm_handle;
  return d->magic == PEVSL_DEVCSR_MAGIC ? d : nullptr;
}

pevsl_devcsr *pevsl_builtin_A(pevsl_Data *pevsl) {
  if (!pevsl->Amv || pevsl->Amv->func != pEVSL_ParcsrMatvec0) return nullptr;
  return pevsl_devcsr_of((const pevsl_Parcsr *)pevsl->Amv->data);
}

/* Sizes only; with one process the local block is the whole matrix unless
 * explicit starts say otherwise (SRC/parcsr.c:24-63). */
int pEVSL_ParcsrCreate(int nrow, int ncol, int *row_starts, int *col_starts, pevsl_Parcsr *A,
                       MPI_Comm comm) {
  memset(A, 0, sizeof(*A));
  A->comm = comm;
  A->nrow_global = nrow;
  A->ncol_global = ncol;
  A->nrow_local = row_starts ? row_starts[1] - row_starts[0] : nrow;
  A->ncol_local = col_starts ? col_starts[1] - col_starts[0] : ncol;
  A->first_row = row_starts ? row_starts[0] : 0;
  A->first_col = col_starts ? col_starts[0] : 0;
  if (row_starts) {
    A->row_starts = (int *)malloc(2 * sizeof(int));
    memcpy(A->row_starts, row_starts, 2 * sizeof(int));
  }
  if (col_starts) {
    A->col_starts = (int *)malloc(2 * sizeof(int));
    memcpy(A->col_starts, col_starts, 2 * sizeof(int));
  }
  return 0;
}

/* Upload the caller's host CSR (the local rows, global column indices) as
 * one device CSR (SRC/parcsr.c:70-283 without the split and halo plan). */
/* The packed copy of a matrix's entries, when every column lies within
 * int16 range of its row's 32-row group start and the matrix has at most
 * 256 distinct values (compared bit for bit, so each entry decodes to the
 * exact double it was): 3 bytes per entry instead of 12.  Stencil and
 * finite-element matrices with few coefficients qualify; the filter and SpMV
 * kernels then read a quarter of the bytes for the matrix, and the result is
 * bit-identical.  Returns 0 also when the matrix does not qualify. */
static int pack_entries(pevsl_devcsr *d, const pevsl_Csr *Ai) {
  const int nr = d->nrows;
  const long long nnz = d->nnz;
  if (nnz <= 0) return 0;
  std::vector<short> dj((size_t)nnz);
  std::vector<unsigned char> vi((size_t)nnz);
  std::vector<double> tab;
  tab.reserve(256);
  /* value bits -> table index: open addressing in 1024 slots */
  constexpr int kSlots = 1024;
  std::vector<uint64_t> hkey(kSlots);
  std::vector<int> hval(kSlots, -1);
  for (int i = 0; i < nr; i++) {
    const long g0 = (long)(i & ~31);
    for (int k = Ai->ia[i]; k < Ai->ia[i + 1]; k++) {
      const long off = (long)Ai->ja[k] - g0;
      /* INT16_MIN is kept free: it marks the ELL layout's padding */
      if (off <= -32768 || off > 32767) return 0;
      dj[(size_t)k] = (short)off;
      uint64_t key;
      memcpy(&key, &Ai->a[k], sizeof key);
      unsigned h = (unsigned)((key * 0x9E3779B97F4A7C15ull) >> 54) & (kSlots - 1);
      while (hval[h] >= 0 && hkey[h] != key) h = (h + 1) & (kSlots - 1);
      if (hval[h] < 0) {
        if (tab.size() == 256) return 0;
        hkey[h] = key;
        hval[h] = (int)tab.size();
        tab.push_back(Ai->a[k]);
      }
      vi[(size_t)k] = (unsigned char)hval[h];
    }
  }
  const size_t b_dj = ((sizeof(short) * (size_t)nnz + 255) / 256) * 256;
  const size_t b_vi = ((size_t)nnz + 255) / 256 * 256;
  const size_t b_tab = 256 * sizeof(double) + 256 * sizeof(float);
  /* ELL copy: width = the longest row, when that is at most 16 and pads
   * the entries by less than a quarter */
  const int ew = d->max_row_nnz;
  const size_t nslice = ((size_t)nr + 31) / 32;
  const size_t ecount = nslice * 32 * (size_t)ew;
  const bool ell = ew >= 1 && ew <= 16 && (double)ecount <= 1.25 * (double)nnz &&
                   ecount < ((size_t)1 << 31);
  const size_t b_edj = ell ? (sizeof(short) * ecount + 255) / 256 * 256 : 0;
  const size_t b_evi = ell ? (ecount + 255) / 256 * 256 : 0;
  char *base = (char *)alloc_dev(b_dj + b_vi + b_tab + b_edj + b_evi);
  if (!base) return PEVSL_ERR_NOMEM;
  std::vector<short> edj;
  std::vector<unsigned char> evi;
  if (ell) {
    edj.assign(ecount, (short)INT16_MIN);
    evi.assign(ecount, 0);
    for (int i = 0; i < nr; i++) {
      const size_t b = (size_t)(i / 32) * 32 * (size_t)ew + (size_t)(i % 32);
      for (int k = Ai->ia[i], j = 0; k < Ai->ia[i + 1]; k++, j++) {
        edj[b + (size_t)j * 32] = dj[(size_t)k];
        evi[b + (size_t)j * 32] = vi[(size_t)k];
      }
    }
    d->edj = (short *)(base + b_dj + b_vi + b_tab);
    d->evi = (unsigned char *)(base + b_dj + b_vi + b_tab + b_edj);
    d->ew = ew;
  }
  std::vector<float> tab32(tab.size());
  for (size_t t = 0; t < tab.size(); t++) tab32[t] = (float)tab[t];
  d->pdj = (short *)base;
  d->pvi = (unsigned char *)(base + b_dj);
  d->pvtab = (double *)(base + b_dj + b_vi);
  d->pvtab32 = (float *)(base + b_dj + b_vi + 256 * sizeof(double));
  d->pnv = (int)tab.size();
  d->pbytes = b_dj + b_vi + b_tab;
  int st = memcpy_async(d->pdj, dj.data(), sizeof(short) * (size_t)nnz);
  if (!st) st = memcpy_async(d->pvi, vi.data(), (size_t)nnz);
  if (!st && ell) st = memcpy_async(d->edj, edj.data(), sizeof(short) * ecount);
  if (!st && ell) st = memcpy_async(d->evi, evi.data(), ecount);
  if (!st) st = memcpy_async(d->pvtab, tab.data(), sizeof(double) * tab.size());
  if (!st) st = memcpy_async(d->pvtab32, tab32.data(), sizeof(float) * tab.size());
  if (!st) st = sync();
  if (!st && ell) st = filter_tune(d);
  return st;
}

int pEVSL_ParcsrSetup(pevsl_Csr *Ai, pevsl_Parcsr *A) {
  if (ensure()) return PEVSL_ERR_CUDA;
  const int nr = A->nrow_local;
  if (!Ai || Ai->nrows != nr || nr < 0) return PEVSL_ERR_ARG;
  const long long nnz = Ai->ia[nr];
  pevsl_devcsr *d = (pevsl_devcsr *)calloc(1, sizeof(pevsl_devcsr));
  if (!d) return PEVSL_ERR_NOMEM;
  d->magic = PEVSL_DEVCSR_MAGIC;
  d->nrows = nr;
  d->ncols = A->ncol_global;
  d->nnz = nnz;
  int maxr = 0;
  for (int i = 0; i < nr; i++) {
    const int r = Ai->ia[i + 1] - Ai->ia[i];
    if (r > maxr) maxr = r;
  }
  d->max_row_nnz = maxr;
  d->avg_row_nnz = nr ? (double)nnz / nr : 0.0;
  d->lanes = choose_lanes(d->avg_row_nnz);
  const char *lenv = getenv("PEVSL_B200_LANES");
  if (lenv) {
    const int L = atoi(lenv);
    if (L == 0 || L == 1 || L == 2 || L == 4 || L == 8 || L == 16 || L == 32) d->lanes = L;
  }
  /* one allocation [values | column indices | row pointers], 256-byte
   * aligned parts, so that a single L2 access-policy window can cover it */
  const size_t bytes_a = ((sizeof(double) * (size_t)nnz + 255) / 256) * 256;
  const size_t bytes_ja = ((sizeof(int) * (size_t)nnz + 255) / 256) * 256;
  const size_t bytes_ia = sizeof(int) * (size_t)(nr + 1);
  char *base = (char *)alloc_dev(bytes_a + bytes_ja + bytes_ia);
  if (!base) {
    free(d);
    return PEVSL_ERR_NOMEM;
  }
  d->a = (double *)base;
  d->ja = (int *)(base + bytes_a);
  d->ia = (int *)(base + bytes_a + bytes_ja);
  d->bytes = bytes_a + bytes_ja + bytes_ia;
  int st = memcpy_async(d->ia, Ai->ia, sizeof(int) * (size_t)(nr + 1));
  if (!st) st = memcpy_async(d->ja, Ai->ja, sizeof(int) * (size_t)nnz);
  if (!st) st = memcpy_async(d->a, Ai->a, sizeof(double) * (size_t)nnz);
  if (!st) st = sync();
  if (st) return st;
  st = pack_entries(d, Ai);
  if (st) return st;
  A->comm_handle = (commHandle *)d;
  A->diag = (pevsl_Csr *)calloc(1, sizeof(pevsl_Csr));
  A->offd = (pevsl_Csr *)calloc(1, sizeof(pevsl_Csr));
  A->diag->nrows = nr;
  A->diag->ncols = A->ncol_global;
  A->diag->ia = d->ia;
  A->diag->ja = d->ja;
  A->diag->a = d->a;
  /* an empty off-diagonal block: PEVSL_CSRNNZ(offd) reads ia[0] == 0 */
  A->offd->ia = (int *)calloc(1, sizeof(int));
  return 0;
}

void pEVSL_ParcsrFree(pevsl_Parcsr *A) {
  pevsl_devcsr *d = pevsl_devcsr_of(A);
  if (d) {
    cudaStreamSynchronize(ctx().stream);
    cudaFree(d->a); /* the whole [values | indices | pointers] block */
    if (d->a32) cudaFree(d->a32);
    if (d->pdj) cudaFree(d->pdj); /* the packed block */
    d->magic = 0;
    free(d);
  }
  A->comm_handle = nullptr;
  free(A->row_starts);
  free(A->col_starts);
  A->row_starts = A->col_starts = nullptr;
  if (A->diag) free(A->diag);
  if (A->offd) {
    free(A->offd->ia);
    free(A->offd);
  }
  A->diag = A->offd = nullptr;
  free(A->col_map_offd);
  A->col_map_offd = nullptr;
}

/* Local rows as host COO and/or CSR with global columns, optionally only
 * the lower ('L') or upper ('U') triangle, 0- or 1-based
 * (SRC/parcsr.c:319-401). */
int pEVSL_ParcsrGetLocalMat(pevsl_Parcsr *A, int idx, pevsl_Coo *coo, pevsl_Csr *csr, char stype) {
  pevsl_devcsr *d = pevsl_devcsr_of(A);
  if (!d) return PEVSL_ERR_ARG;
  stype = (char)toupper((unsigned char)stype);
  if (stype != 'L' && stype != 'U') stype = 'A';
  const int nr = d->nrows;
  const long long nnz = d->nnz;
  int *ia = (int *)malloc(sizeof(int) * (size_t)(nr + 1));
  int *ja = (int *)malloc(sizeof(int) * (size_t)(nnz ? nnz : 1));
  double *a = (double *)malloc(sizeof(double) * (size_t)(nnz ? nnz : 1));
  if (!ia || !ja || !a) {
    free(ia);
    free(ja);
    free(a);
    return PEVSL_ERR_NOMEM;
  }
  int st = memcpy_async(ia, d->ia, sizeof(int) * (size_t)(nr + 1));
  if (!st) st = memcpy_async(ja, d->ja, sizeof(int) * (size_t)nnz);
  if (!st) st = memcpy_async(a, d->a, sizeof(double) * (size_t)nnz);
  if (!st) st = sync();
  if (st) {
    free(ia);
    free(ja);
    free(a);
    return st;
  }
  pevsl_Csr loc;
  pEVSL_CsrResize(nr, A->ncol_global, (int)nnz, &loc);
  int k = 0;
  loc.ia[0] = 0;
  for (int i = 0; i < nr; i++) {
    const int grow = i + A->first_row;
    for (int j = ia[i]; j < ia[i + 1]; j++) {
      const int gcol = ja[j];
      if (stype == 'A' || (stype == 'L' && grow >= gcol) || (stype == 'U' && grow <= gcol)) {
        loc.ja[k] = gcol;
        loc.a[k] = a[j];
        k++;
      }
    }
    loc.ia[i + 1] = k;
  }
  free(ia);
  free(ja);
  free(a);
  pEVSL_SortRow(&loc);
  if (coo) pEVSL_CsrToCoo(&loc, idx, coo);
  if (csr) {
    if (idx) {
      for (int j = 0; j < loc.ia[nr]; j++) loc.ja[j]++;
      for (int i = 0; i <= nr; i++) loc.ia[i]++;
    }
    *csr = loc;
  } else {
    pEVSL_FreeCsr(&loc);
  }
  return 0;
}

int pEVSL_ParcsrNnz(pevsl_Parcsr *A) {
  pevsl_devcsr *d = pevsl_devcsr_of(A);
  return d ? (int)d->nnz : 0;
}

int pEVSL_ParcsrLocalNnz(pevsl_Parcsr *A) { return pEVSL_ParcsrNnz(A); }

void pEVSL_ParcsrMatvec0(double *x, double *y, void *data) {
  pevsl_devcsr *d = pevsl_devcsr_of((const pevsl_Parcsr *)data);
  if (!d || ensure()) return;
  if (!spmv(d, x, y)) sync();
}

void pEVSL_ParcsrMatvec(pevsl_Parcsr *A, pevsl_Parvec *x, pevsl_Parvec *y) {
  pEVSL_ParcsrMatvec0(x->data, y->data, (void *)A);
}

}  // extern "C"
