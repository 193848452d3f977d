/*
 * Staged interleaved filter degree for sm_100a: one degree of the Chebyshev
 * recurrence of pEVSL_ChebAv (SRC/chebpol.c:538-568) fused with the CSR
 * SpMV (SRC/spmat.c:184-206) for S row-interleaved vectors (X[i*S + s]) of
 * one matrix held in the packed form (int16 column offset from the row's
 * 32-row group start + uint8 index into a table of at most 256 values).
 *
 * The kernel is persistent and warp-specialised.  The matrix is cut into
 * row chunks (pevsl_devcsr.wchunk: at most 256 rows and 4096 entries, each
 * starting at a multiple of 4 rows).  Per block, one producer warp walks its
 * chunks and stages each chunk's contiguous streams -- the row pointers, the
 * packed column offsets and value indices, and the chunk's rows of X_k --
 * into shared memory with cp.async.bulk copies that complete on an mbarrier,
 * several chunks ahead (a ring of stages; the consumers hand a stage back on
 * a second mbarrier).  Eight consumer warps then find every operand of a row
 * in shared memory except the gathers of columns outside the chunk, which
 * are the only dependent global loads left; X_{k-1} and Y are read with
 * plain coalesced loads.  Per row the products are added in entry order and
 * the recurrence and the deferred sum use the arithmetic of the one-vector
 * kernel, so the results are bit-identical to k_cheb_il_p.
 *
 * Every mbarrier wait is bounded: a wait that runs out sets an error flag
 * (read by pv::il_tma_error) and the warp leaves its loop.  No copy reads
 * another GPU's memory and none uses multicast.
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "gpu.cuh"
#include "gpu_device.cuh"

namespace pv {

namespace {

constexpr int kCW = 8;              /* consumer warps                     */
constexpr int kWT = 32 * (kCW + 1); /* threads per block (+ one producer) */
constexpr int kRmax = PEVSL_WAVE_RMAX;
constexpr int kEmax = PEVSL_WAVE_EMAX;
constexpr unsigned kWaitSpins = 1u << 22; /* polls before a wait gives up (~0.5-1 s) */
constexpr unsigned kDepSpins = 1u << 20;  /* polls of a wavefront dependency (~0.1-0.5 s) */

/* one stage of the ring; every copied array starts on a 16-byte boundary */
template <int S>
struct __align__(128) Stage {
  double x[kRmax * S];          /* rows r0..r1-1 of X_k                      */
  int ia[kRmax + 8];            /* row pointers r0..r1 (copy rounded to 16 B) */
  short dj[kEmax + 16];         /* column offsets from entry jdj on          */
  unsigned char vi[kEmax + 32]; /* value indices from entry jvi on           */
  int r0, r1, jdj, jvi, big;    /* r0 < 0: no more chunks                     */
};

template <int S>
__host__ __device__ constexpr int stages_for() {
  return S >= 16 ? 2 : 3;
}
static_assert(sizeof(double) * kRmax % 16 == 0, "staged rows start on 16-byte boundaries");

template <int S>
__host__ __device__ constexpr size_t tma_smem() {
  return sizeof(Stage<S>) * stages_for<S>() + 2 * sizeof(uint64_t) * stages_for<S>() +
         256 * sizeof(double);
}

struct IlTmaArgs {
  int n, nc;
  const int *wchunk;
  const int *ia;
  const short *dj;
  const unsigned char *vi;
  const double *vtab;
  int nv;
  const double *Xk, *Xkm1;
  double *Xkp1, *Y;
  double cc, t;
  const double *mu0, *muk; /* per-vector coefficients (S >= 2) */
  double mu0s, muks;        /* the one vector's coefficients (S = 1) */
  int ny, fresh;
};

__device__ unsigned g_tma_err;
uint64_t g_tma_launches = 0, g_tma_checked = 0; /* host: launches, launches already checked */

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(
                   smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

/* bounded wait for the phase of the given parity; false (and the error flag
 * set) when it did not complete */
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
  for (unsigned i = 0; i < kWaitSpins; i++) {
    if (mbar_try(bar, parity)) return true;
    if (i > 16) __nanosleep(64);
  }
  atomicExch(&g_tma_err, 1u);
  return false;
}

/* bulk copy global -> this block's shared memory, completing on bar */
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ unsigned round16(unsigned b) { return (b + 15u) & ~15u; }

template <int S>
__global__ void __launch_bounds__(kWT) k_cheb_il_tma(const __grid_constant__ IlTmaArgs a) {
  constexpr int NST = stages_for<S>();
  extern __shared__ __align__(128) unsigned char smem[];
  Stage<S> *st = reinterpret_cast<Stage<S> *>(smem);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + sizeof(Stage<S>) * NST);
  uint64_t *empty = full + NST;
  double *vt = reinterpret_cast<double *>(empty + NST);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < NST; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kCW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = threadIdx.x; i < a.nv; i += blockDim.x) vt[i] = a.vtab[i];
  __syncthreads();

  if (warp == kCW) {
    /* producer: one thread stages chunk blockIdx.x + it * gridDim.x */
    if (lane != 0) return;
    int it = 0;
    for (int c = blockIdx.x;; c += gridDim.x, it++) {
      const int s = it % NST;
      Stage<S> &g = st[s];
      if (it >= NST && !mbar_wait(&empty[s], ((it / NST) - 1) & 1)) return;
      if (c >= a.nc) {
        g.r0 = -1;
        mbar_arrive(&full[s]);
        return;
      }
      const int r0 = __ldg(a.wchunk + 2 * c), e0 = __ldg(a.wchunk + 2 * c + 1);
      const int r1 = __ldg(a.wchunk + 2 * c + 2), e1 = __ldg(a.wchunk + 2 * c + 3);
      const int big = e1 - e0 > kEmax;
      const int jdj = e0 & ~7, jvi = e0 & ~15;
      const unsigned b_ia = round16(4u * (unsigned)(r1 + 1 - r0));
      /* S = 1: a chunk with an odd row count stages one row less (the copy
       * is a multiple of 16 bytes); its last row is read from global */
      const unsigned b_x = (8u * S * (unsigned)(r1 - r0)) & ~15u;
      const unsigned b_dj = big ? 0u : round16(2u * (unsigned)(e1 - jdj));
      const unsigned b_vi = big ? 0u : round16((unsigned)(e1 - jvi));
      g.r0 = r0;
      g.r1 = r1;
      g.jdj = jdj;
      g.jvi = jvi;
      g.big = big;
      mbar_arrive_tx(&full[s], b_ia + b_x + b_dj + b_vi);
      bulk_g2s(g.ia, a.ia + r0, b_ia, &full[s]);
      bulk_g2s(g.x, a.Xk + (size_t)r0 * S, b_x, &full[s]);
      if (!big) {
        bulk_g2s(g.dj, a.dj + jdj, b_dj, &full[s]);
        bulk_g2s(g.vi, a.vi + jvi, b_vi, &full[s]);
      }
    }
  }

  /* consumers: rows of the staged chunk, S lanes per row */
  const int tid = threadIdx.x;
  for (int it = 0;; it++) {
    const int s = it % NST;
    if (!mbar_wait(&full[s], (it / NST) & 1)) return;
    const Stage<S> &g = st[s];
    const int r0 = g.r0;
    if (r0 < 0) return;
    const int r1 = g.r1, jdj = g.jdj, jvi = g.jvi, big = g.big;
    const int nrows = r1 - r0;
    const int nr = S == 1 ? (nrows & ~1) : nrows; /* rows staged in g.x */
    for (int p = tid; p < nrows * S; p += kCW * 32) {
      const int lr = p / S, sl = p % S;
      const int row = r0 + lr;
      const size_t me = (size_t)row * S + sl;
      const double x = lr < nr ? g.x[p] : a.Xk[me];
      const double xm1 = a.Xkm1 ? a.Xkm1[me] : 0.0;
      const double yold = (a.ny > 0 && !a.fresh) ? a.Y[me] : 0.0;
      const int g0 = row & ~31;
      const int e = g.ia[lr + 1];
      int j = g.ia[lr];
      double r = 0.0;
      if (!big) {
        /* up to 8 entries' gathers in flight, then added in entry order
         * (an entry past the row end is skipped, never added as zero) */
        for (; j < e; j += 8) {
          double xv[8];
#pragma unroll
          for (int u = 0; u < 8; u++) {
            xv[u] = 0.0;
            if (j + u < e) {
              const int cu = g0 + g.dj[j + u - jdj];
              const unsigned lu = (unsigned)(cu - r0);
              xv[u] = lu < (unsigned)nr ? g.x[lu * S + sl] : __ldg(a.Xk + (size_t)cu * S + sl);
            }
          }
#pragma unroll
          for (int u = 0; u < 8; u++)
            if (j + u < e) r = __dadd_rn(r, __dmul_rn(vt[g.vi[j + u - jvi]], xv[u]));
        }
      } else {
        for (; j < e; j++) {
          const int c0 = g0 + __ldg(a.dj + j);
          r = __dadd_rn(r, __dmul_rn(vt[__ldg(a.vi + j)], __ldg(a.Xk + (size_t)c0 * S + sl)));
        }
      }
      double w = __dmul_rn(__fma_rn(-a.cc, x, r), a.t);
      if (a.Xkm1) w = __dsub_rn(w, xm1);
      a.Xkp1[me] = w;
      if (S == 1) {
        /* the one-vector recurrence (cheb_update_v): y updated every degree */
        a.Y[me] = a.fresh ? __fma_rn(a.muks, w, __dmul_rn(a.mu0s, x)) : __fma_rn(a.muks, w, yold);
      } else if (a.ny > 0) {
        /* the deferred sum of k_cheb_il: terms of degrees k-ny+1..k */
        double y = a.fresh ? __dmul_rn(a.mu0[sl], a.ny == 1 ? x : xm1) : yold;
        if (a.ny >= 3) y = __fma_rn(a.muk[sl - 2 * S], xm1, y);
        if (a.ny >= 2) y = __fma_rn(a.muk[sl - S], x, y);
        a.Y[me] = __fma_rn(a.muk[sl], w, y);
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }
}

/* resident blocks of each kernel and width (index log2 S), set by tma_init */
int g_grid_tma[5] = {0, 0, 0, 0, 0}, g_grid_wave[5] = {0, 0, 0, 0, 0};

constexpr int slot_of(int S) { return S == 1 ? 0 : S == 2 ? 1 : S == 4 ? 2 : S == 8 ? 3 : 4; }

/* dynamic shared memory above 48 KB and the resident grid of one kernel */
int setup_kernel(const void *fn, size_t smem, int *grid) {
  if (fail(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
           "cudaFuncSetAttribute"))
    return PEVSL_ERR_CUDA;
  int per_sm = 0;
  if (fail(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kWT, smem),
           "cudaOccupancyMaxActiveBlocksPerMultiprocessor"))
    return PEVSL_ERR_CUDA;
  if (per_sm < 1) return PEVSL_ERR_ARG;
  *grid = per_sm * ctx().sms;
  return 0;
}

/* ---------------------------------------------------------------- wavefront
 * Several degrees per launch.  Item (j, c) is degree k = k0 + j on chunk c;
 * it needs degree k - 1 done on the chunks of wdep[c] (its gathers, and the
 * readers of the rows it overwrites: T_k goes in place over T_{k-2}).  The
 * items are claimed through an atomic counter in the order of the skewed
 * time t = c + j * Lp (then j): with Lp above the dependency reach every
 * item depends only on items claimed before it, so the wait of the smallest
 * unfinished item always ends (no deadlock, whatever the number of resident
 * blocks), and the degrees of one launch sweep the rows as a wavefront a few
 * thousand rows wide -- the vectors, the accumulator and the matrix rows of
 * the wavefront stay in L2 between degrees instead of going to HBM for each.
 * done[c] counts the consumer warps that finished chunk c (kCW per degree,
 * released at gpu scope); data written in the launch is read through L2
 * (ld.global.cg) or by the bulk copies after a proxy fence. */
struct IlWaveArgs {
  int n, nc;
  const int *wchunk, *wdep;
  const int *ia;
  const short *dj;
  const unsigned char *vi;
  const double *vtab;
  int nv;
  const double *X0; /* T_0 (read only) */
  double *B0, *B1;  /* T_k for k >= 1: B0 for odd k, B1 for even k */
  double *Y;
  double cc, t1, t2;
  const double *mu; /* row k: mu_k of every vector (0 past a vector's degree) */
  int k0, D, maxdeg, defer, Lp;
  int *done;
  unsigned *ctr;
};

__device__ __forceinline__ const double *wave_buf(const IlWaveArgs &a, int k) {
  return k == 0 ? a.X0 : ((k & 1) ? a.B0 : a.B1);
}

/* items with time < t */
__host__ __device__ __forceinline__ long wave_before(long t, int nc, int D, int Lp) {
  long f = 0;
  for (int j = 0; j < D; j++) {
    const long v = t - (long)j * Lp;
    f += v <= 0 ? 0 : (v >= nc ? nc : v);
  }
  return f;
}

__host__ __device__ __forceinline__ void wave_item(long idx, int nc, int D, int Lp, int *j, int *c) {
  long lo = 0, hi = nc + (long)(D - 1) * Lp; /* before(lo) <= idx < before(hi) */
  while (hi - lo > 1) {
    const long mid = (lo + hi) >> 1;
    if (wave_before(mid, nc, D, Lp) <= idx) lo = mid;
    else hi = mid;
  }
  const long r = idx - wave_before(lo, nc, D, Lp);
  const long jmin = lo >= nc ? (lo - nc) / Lp + 1 : 0;
  *j = (int)(jmin + r);
  *c = (int)(lo - (jmin + r) * Lp);
}

/* terms of the deferred sum that degree k adds (the host's il_terms in
 * closed form): the first update at degree min(defer, 2), then every defer
 * degrees, and the last at maxdeg */
__host__ __device__ __forceinline__ int wave_terms(int k, int maxdeg, int defer, int *fresh) {
  const int first = defer < 2 ? defer : 2;
  *fresh = 0;
  if (k < first) {
    if (k == maxdeg) *fresh = 1;
    return k == maxdeg ? k : 0;
  }
  if (k == first) {
    *fresh = 1;
    return k;
  }
  const int m = (k - first) % defer;
  if (m == 0) return defer;
  return k == maxdeg ? m : 0;
}

__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void red_release_add(int *p, int v) {
  asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

/* the stage header of the wavefront kernel reuses Stage<S>: jvi/jdj as in
 * the staged kernel, r0 < 0 ends, and the degree in `big`'s upper bits */
template <int S>
__global__ void __launch_bounds__(kWT) k_cheb_il_wave(const __grid_constant__ IlWaveArgs a) {
  constexpr int NST = stages_for<S>();
  /* an earlier launch gave up: the application is reported failed, skip */
  if (*(volatile unsigned *)&g_tma_err) return;
  extern __shared__ __align__(128) unsigned char smem[];
  Stage<S> *st = reinterpret_cast<Stage<S> *>(smem);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + sizeof(Stage<S>) * NST);
  uint64_t *empty = full + NST;
  double *vt = reinterpret_cast<double *>(empty + NST);
  int *hdr_k = reinterpret_cast<int *>(vt + 256); /* degree and chunk of each stage */
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < NST; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kCW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = threadIdx.x; i < a.nv; i += blockDim.x) vt[i] = a.vtab[i];
  __syncthreads();
  const long total = (long)a.nc * a.D;

  if (warp == kCW) {
    /* producer warp: claim (one item ahead), wait for the dependencies,
     * stage.  A block holds at most two claimed items, the earlier one
     * staged first, so every wait still ends (items depend only on items
     * claimed before them). */
    unsigned next = 0;
    if (lane == 0) next = atomicAdd(a.ctr, 1u);
    next = __shfl_sync(0xffffffffu, next, 0);
    for (int it = 0;; it++) {
      const int s = it % NST;
      Stage<S> &g = st[s];
      const unsigned idx = next;
      if ((long)idx >= total) {
        int ok = 1;
        if (it >= NST && lane == 0) ok = mbar_wait(&empty[s], ((it / NST) - 1) & 1);
        if (lane == 0 && ok) {
          g.r0 = -1;
          mbar_arrive(&full[s]);
        }
        return;
      }
      int j, c;
      wave_item((long)idx, a.nc, a.D, a.Lp, &j, &c);
      const int k = a.k0 + j;
      /* the chunk's bounds (lanes 0..3), independent of the waits below */
      const int bnd = lane < 4 ? __ldg(a.wchunk + 2 * c + lane) : 0;
      if (j > 0) {
        /* degree k - 1 done on every chunk of the dependency range: each
         * lane reads its (up to 4) flags at once, then spins on the late */
        const int lo = __ldg(a.wdep + 2 * c), hi = __ldg(a.wdep + 2 * c + 1);
        const int need = kCW * (k - 1);
        int fine = 1;
        for (int q0 = lo; q0 <= hi && fine; q0 += 128) {
          int v[4];
#pragma unroll
          for (int u = 0; u < 4; u++) {
            const int q = q0 + lane + 32 * u;
            v[u] = q <= hi ? ld_acquire(a.done + q) : need;
          }
#pragma unroll
          for (int u = 0; u < 4; u++) {
            const int q = q0 + lane + 32 * u;
            unsigned spin = 0;
            while (v[u] < need) {
              if (++spin > kDepSpins) {
                atomicExch(&g_tma_err, 2u);
                fine = 0;
                break;
              }
              __nanosleep(32);
              v[u] = ld_acquire(a.done + q);
            }
          }
        }
        if (!__all_sync(0xffffffffu, fine)) {
          /* give up: end the consumers after what they hold */
          int ok = 1;
          if (it >= NST && lane == 0) ok = mbar_wait(&empty[s], ((it / NST) - 1) & 1);
          if (lane == 0 && ok) {
            g.r0 = -1;
            mbar_arrive(&full[s]);
          }
          return;
        }
      }
      /* the next claim overlaps the stage wait and the copies */
      if (lane == 0) next = atomicAdd(a.ctr, 1u);
      next = __shfl_sync(0xffffffffu, next, 0);
      const int r0 = __shfl_sync(0xffffffffu, bnd, 0), e0 = __shfl_sync(0xffffffffu, bnd, 1);
      const int r1 = __shfl_sync(0xffffffffu, bnd, 2), e1 = __shfl_sync(0xffffffffu, bnd, 3);
      int ok = 1;
      if (it >= NST && lane == 0) ok = mbar_wait(&empty[s], ((it / NST) - 1) & 1);
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) return;
      if (lane == 0) {
        fence_proxy_async_global();
        const int big = e1 - e0 > kEmax;
        const int jdj = e0 & ~7, jvi = e0 & ~15;
        const unsigned b_ia = round16(4u * (unsigned)(r1 + 1 - r0));
        /* S = 1: an odd row count stages one row less (16-byte copies) */
        const unsigned b_x = (8u * S * (unsigned)(r1 - r0)) & ~15u;
        const unsigned b_dj = big ? 0u : round16(2u * (unsigned)(e1 - jdj));
        const unsigned b_vi = big ? 0u : round16((unsigned)(e1 - jvi));
        g.r0 = r0;
        g.r1 = r1;
        g.jdj = jdj;
        g.jvi = jvi;
        g.big = big;
        hdr_k[2 * s] = k;
        hdr_k[2 * s + 1] = c;
        mbar_arrive_tx(&full[s], b_ia + b_x + b_dj + b_vi);
        bulk_g2s(g.ia, a.ia + r0, b_ia, &full[s]);
        bulk_g2s(g.x, wave_buf(a, k - 1) + (size_t)r0 * S, b_x, &full[s]);
        if (!big) {
          bulk_g2s(g.dj, a.dj + jdj, b_dj, &full[s]);
          bulk_g2s(g.vi, a.vi + jvi, b_vi, &full[s]);
        }
      }
      __syncwarp();
    }
  }

  /* consumers */
  const int tid = threadIdx.x;
  for (int it = 0;; it++) {
    const int s = it % NST;
    if (!mbar_wait(&full[s], (it / NST) & 1)) return;
    const Stage<S> &g = st[s];
    const int r0 = g.r0;
    if (r0 < 0) return;
    const int k = hdr_k[2 * s], c = hdr_k[2 * s + 1];
    const int r1 = g.r1, jdj = g.jdj, jvi = g.jvi, big = g.big;
    const int nrows = r1 - r0;
    const int nr = S == 1 ? (nrows & ~1) : nrows; /* rows staged in g.x */
    const double *Xg = wave_buf(a, k - 1);                 /* T_{k-1}: gathered  */
    const double *Xm = k >= 2 ? wave_buf(a, k - 2) : nullptr; /* T_{k-2}: own rows */
    double *Xo = const_cast<double *>(wave_buf(a, k));     /* T_k (over T_{k-2}) */
    const double t = k == 1 ? a.t1 : a.t2;
    const double *mu0 = a.mu, *muk = a.mu + (size_t)k * S;
    int fresh;
    const int ny = wave_terms(k, a.maxdeg, a.defer, &fresh);
    for (int p = tid; p < nrows * S; p += kCW * 32) {
      const int lr = p / S, sl = p % S;
      const int row = r0 + lr;
      const size_t me = (size_t)row * S + sl;
      const double x = lr < nr ? g.x[p] : __ldcg(Xg + me);
      const double xm1 = Xm ? __ldcg(Xm + me) : 0.0;
      const double yold = (ny > 0 && !fresh) ? __ldcg(a.Y + me) : 0.0;
      const int g0 = row & ~31;
      const int e = g.ia[lr + 1];
      int j = g.ia[lr];
      double r = 0.0;
      if (!big) {
        /* up to 8 entries' gathers in flight, added in entry order */
        for (; j < e; j += 8) {
          double xv[8];
#pragma unroll
          for (int u = 0; u < 8; u++) {
            xv[u] = 0.0;
            if (j + u < e) {
              const int cu = g0 + g.dj[j + u - jdj];
              const unsigned lu = (unsigned)(cu - r0);
              xv[u] = lu < (unsigned)nr ? g.x[lu * S + sl] : __ldcg(Xg + (size_t)cu * S + sl);
            }
          }
#pragma unroll
          for (int u = 0; u < 8; u++)
            if (j + u < e) r = __dadd_rn(r, __dmul_rn(vt[g.vi[j + u - jvi]], xv[u]));
        }
      } else {
        for (; j < e; j++) {
          const int c0 = g0 + __ldg(a.dj + j);
          r = __dadd_rn(r, __dmul_rn(vt[__ldg(a.vi + j)], __ldcg(Xg + (size_t)c0 * S + sl)));
        }
      }
      double w = __dmul_rn(__fma_rn(-a.cc, x, r), t);
      if (Xm) w = __dsub_rn(w, xm1);
      __stcg(Xo + me, w);
      if (ny > 0) {
        double y = fresh ? __dmul_rn(mu0[sl], ny == 1 ? x : xm1) : yold;
        if (ny >= 3) y = __fma_rn(muk[sl - 2 * S], xm1, y);
        if (ny >= 2) y = __fma_rn(muk[sl - S], x, y);
        __stcg(a.Y + me, __fma_rn(muk[sl], w, y));
      }
    }
    /* publish: this warp's rows of degree k on chunk c are written */
    fence_proxy_async_global();
    __syncwarp();
    if (lane == 0) {
      red_release_add(a.done + c, 1);
      mbar_arrive(&empty[s]);
    }
  }
}

template <int S>
constexpr size_t wave_smem() {
  return tma_smem<S>() + 2 * sizeof(int) * stages_for<S>();
}

template <int S>
int launch_il_wave(const IlWaveArgs &args, long total) {
  const int grid = g_grid_wave[slot_of(S)];
  if (grid < 1) return PEVSL_ERR_ARG; /* tma_init did not run */
  const unsigned g = (unsigned)(total < grid ? total : grid);
  k_cheb_il_wave<S><<<g, kWT, wave_smem<S>(), ctx().stream>>>(args);
  g_tma_launches++;
  return launched("cheb_il_wave");
}

template <int S>
int setup_width() {
  if (setup_kernel((const void *)k_cheb_il_tma<S>, tma_smem<S>(), &g_grid_tma[slot_of(S)]))
    return PEVSL_ERR_CUDA;
  return setup_kernel((const void *)k_cheb_il_wave<S>, wave_smem<S>(), &g_grid_wave[slot_of(S)]);
}

template <int S>
int launch_il_tma(const pevsl_devcsr *A, const IlTmaArgs &args) {
  const int grid = g_grid_tma[slot_of(S)];
  if (grid < 1) return PEVSL_ERR_ARG; /* tma_init did not run */
  const unsigned g = (unsigned)(A->wnc < grid ? A->wnc : grid);
  k_cheb_il_tma<S><<<g, kWT, tma_smem<S>(), ctx().stream>>>(args);
  g_tma_launches++;
  return launched("cheb_step_il_tma");
}

}  // namespace

/* the staged kernel applies to packed matrices with a chunk table, S >= 2,
 * and the standard (not generalized) filter: PEVSL_B200_IL_TMA=0 turns it
 * off */
bool il_tma_usable(const pevsl_devcsr *A, int S) {
  static int v = -1;
  if (v < 0) {
    const char *e = getenv("PEVSL_B200_IL_TMA");
    v = e ? atoi(e) != 0 : 1;
  }
  return v && A->pdj != nullptr && A->wchunk != nullptr && A->wnc > 0 &&
         (S == 1 || S == 2 || S == 4 || S == 8 || S == 16);
}

int cheb_step_il_tma(const pevsl_devcsr *A, int S, const double *Xk, const double *Xkm1,
                     double *Xkp1, double *Y, double cc, double t, const double *mu0,
                     const double *muk, int ny, int fresh) {
  IlTmaArgs args;
  args.n = A->nrows;
  args.nc = A->wnc;
  args.wchunk = A->wchunk;
  args.ia = A->ia;
  args.dj = A->pdj;
  args.vi = A->pvi;
  args.vtab = A->pvtab;
  args.nv = A->pnv;
  args.Xk = Xk;
  args.Xkm1 = Xkm1;
  args.Xkp1 = Xkp1;
  args.Y = Y;
  args.cc = cc;
  args.t = t;
  args.mu0 = mu0;
  args.muk = muk;
  args.mu0s = args.muks = 0.0;
  args.ny = ny;
  args.fresh = fresh;
  switch (S) {
    case 2: return launch_il_tma<2>(A, args);
    case 4: return launch_il_tma<4>(A, args);
    case 8: return launch_il_tma<8>(A, args);
    case 16: return launch_il_tma<16>(A, args);
    default: return PEVSL_ERR_ARG;
  }
}

int cheb_step_tma(const pevsl_devcsr *A, const double *vk, const double *vkm1, double *vkp1,
                  double *y, double cc, double t, double mu0, double muk, int first) {
  IlTmaArgs args;
  args.n = A->nrows;
  args.nc = A->wnc;
  args.wchunk = A->wchunk;
  args.ia = A->ia;
  args.dj = A->pdj;
  args.vi = A->pvi;
  args.vtab = A->pvtab;
  args.nv = A->pnv;
  args.Xk = vk;
  args.Xkm1 = vkm1;
  args.Xkp1 = vkp1;
  args.Y = y;
  args.cc = cc;
  args.t = t;
  args.mu0 = args.muk = nullptr;
  args.mu0s = mu0;
  args.muks = muk;
  args.ny = 1;
  args.fresh = first;
  return launch_il_tma<1>(A, args);
}

/* degrees per wavefront launch (PEVSL_B200_WAVE_D, default 8) and the skew's
 * slack in items per front (PEVSL_B200_WAVE_SLACK, default 1.0 x resident
 * blocks / D) */
static int wave_degrees() {
  static int v = 0;
  if (!v) {
    const char *e = getenv("PEVSL_B200_WAVE_D");
    v = e ? atoi(e) : 8;
    if (v < 1 || v > 64) v = 8;
  }
  return v;
}

static double wave_slack() {
  static double v = -1.0;
  if (v < 0) {
    const char *e = getenv("PEVSL_B200_WAVE_SLACK");
    v = e ? atof(e) : 1.0;
    if (!(v >= 0.0 && v <= 100.0)) v = 1.0;
  }
  return v;
}

bool il_wave_usable(const pevsl_devcsr *A, int S) {
  static int v = -1;
  if (v < 0) {
    const char *e = getenv("PEVSL_B200_IL_WAVE");
    v = e ? atoi(e) != 0 : 1;
  }
  return v && il_tma_usable(A, S) && A->wdep != nullptr;
}

size_t il_wave_ints(const pevsl_devcsr *A, int maxdeg) {
  return (size_t)A->wnc + (size_t)(maxdeg + wave_degrees() - 1) / wave_degrees() + 1;
}

int cheb_filter_il_wave(const pevsl_devcsr *A, int S, const double *X0, double *B0, double *B1,
                        double *Y, double cc, double dd, const double *mu, int maxdeg, int defer,
                        int *flags) {
  if (maxdeg <= 0) return 0;
  const int D = wave_degrees();
  const int nl = (maxdeg + D - 1) / D;
  int *done = flags;
  unsigned *ctr = (unsigned *)(flags + A->wnc);
  if (fail(cudaMemsetAsync(flags, 0, sizeof(int) * ((size_t)A->wnc + nl), ctx().stream),
           "cudaMemsetAsync"))
    return PEVSL_ERR_CUDA;
  if (S != 1 && S != 2 && S != 4 && S != 8 && S != 16) return PEVSL_ERR_ARG;
  const int grid = g_grid_wave[slot_of(S)];
  if (grid < 1) return PEVSL_ERR_ARG;
  IlWaveArgs a;
  a.n = A->nrows;
  a.nc = A->wnc;
  a.wchunk = A->wchunk;
  a.wdep = A->wdep;
  a.ia = A->ia;
  a.dj = A->pdj;
  a.vi = A->pvi;
  a.vtab = A->pvtab;
  a.nv = A->pnv;
  a.X0 = X0;
  a.B0 = B0;
  a.B1 = B1;
  a.Y = Y;
  a.cc = cc;
  a.t1 = 1.0 / dd;
  a.t2 = 2.0 / dd;
  a.mu = mu;
  a.maxdeg = maxdeg;
  a.defer = defer;
  a.done = done;
  for (int l = 0; l < nl; l++) {
    a.k0 = 1 + l * D;
    a.D = PEVSL_MIN(D, maxdeg - a.k0 + 1);
    /* skew: past the dependency reach by the items of one front in flight */
    a.Lp = A->wreach + 1 + (int)(wave_slack() * grid / a.D);
    a.ctr = ctr + l;
    const long total = (long)a.nc * a.D;
    int st;
    switch (S) {
      case 1: st = launch_il_wave<1>(a, total); break;
      case 2: st = launch_il_wave<2>(a, total); break;
      case 4: st = launch_il_wave<4>(a, total); break;
      case 8: st = launch_il_wave<8>(a, total); break;
      default: st = launch_il_wave<16>(a, total); break;
    }
    if (st) return st;
  }
  return 0;
}

int tma_init() {
  if (setup_width<1>() || setup_width<2>() || setup_width<4>() || setup_width<8>() ||
      setup_width<16>())
    return PEVSL_ERR_CUDA;
  return 0;
}

/* 1 (and the flag cleared) if a wait of the staged kernel ran out since the
 * last call; synchronises the context stream when the kernel ran since then
 * (not to be called inside a stream capture) */
int il_tma_error() {
  if (g_tma_launches == g_tma_checked) return 0;
  g_tma_checked = g_tma_launches;
  unsigned h = 0;
  if (cudaMemcpyFromSymbolAsync(&h, g_tma_err, sizeof h, 0, cudaMemcpyDeviceToHost,
                                ctx().stream) != cudaSuccess ||
      cudaStreamSynchronize(ctx().stream) != cudaSuccess)
    return 1;
  if (h) {
    const unsigned z = 0;
    cudaMemcpyToSymbolAsync(g_tma_err, &z, sizeof z, 0, cudaMemcpyHostToDevice, ctx().stream);
    cudaStreamSynchronize(ctx().stream);
    return 1;
  }
  return 0;
}

}  // namespace pv

extern "C" {

/* the wavefront's claim order and deferral schedule, on the host (the same
 * functions the kernel runs), for tests */
int pEVSL_B200_WaveItem(int nc, int D, int Lp, long idx, int *j, int *c) {
  if (nc <= 0 || D <= 0 || Lp <= 0 || idx < 0 || idx >= (long)nc * D || !j || !c)
    return PEVSL_ERR_ARG;
  pv::wave_item(idx, nc, D, Lp, j, c);
  return 0;
}

int pEVSL_B200_WaveTerms(int k, int maxdeg, int defer, int *fresh) {
  int f = 0;
  const int ny = pv::wave_terms(k, maxdeg, defer, &f);
  if (fresh) *fresh = f;
  return ny;
}

}  // extern "C"
