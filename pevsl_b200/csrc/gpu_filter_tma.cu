/*
 * Staged filter degree for sm_100a: one degree of the Chebyshev recurrence
 * of pEVSL_ChebAv (SRC/chebpol.c:538-568) fused with the CSR SpMV
 * (SRC/spmat.c:184-206) for S row-interleaved vectors (X[i*S + s]; S = 1 is
 * one plain vector) of one matrix held in the packed form (int16 column
 * offset from the row's 32-row group start + uint8 index into a table of at
 * most 256 values).
 *
 * The kernel is persistent and warp-specialised.  The matrix is cut into
 * row chunks (pevsl_devcsr.wchunk: at most 256 rows and 4096 entries, each
 * starting at a multiple of 4 rows).  Per block, one producer warp walks its
 * chunks and stages each chunk's contiguous streams -- the row pointers, the
 * packed column offsets and value indices, and the chunk's rows of X_k,
 * X_{k-1} and Y (the last two for S <= 4) -- into shared memory with
 * cp.async.bulk copies that complete on an mbarrier, a ring of stages ahead
 * (the consumers hand a stage back on a second mbarrier).  Sixteen consumer
 * warps then find every operand of a row in shared memory except the
 * gathers of columns outside the chunk, the only dependent global loads
 * left; each thread keeps up to eight of a row's gathers in flight and adds
 * the products in entry order afterwards.  The recurrence and the deferred
 * sum use the arithmetic of the one-thread-per-row kernels, so the results
 * are bit-identical to k_cheb_il_p / k_csr_stream_packed.
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

constexpr int kCW = 16;             /* consumer warps                     */
constexpr int kWT = 32 * (kCW + 1); /* threads per block (+ one producer) */
constexpr int kRmax = PEVSL_WAVE_RMAX;
constexpr int kEmax = PEVSL_WAVE_EMAX;
constexpr unsigned kWaitSpins = 1u << 22; /* polls before a wait gives up (~0.5-1 s) */

/* X_{k-1} and Y rows staged too, for the widths whose three vector blocks
 * of a chunk still leave room for two blocks per SM */
template <int S>
__host__ __device__ constexpr bool stage_all() {
  return S <= 4;
}
template <int S>
__host__ __device__ constexpr int rows_of() {
  return stage_all<S>() ? kRmax * S : 2;
}

/* one stage of the ring; every copied array starts on a 16-byte boundary */
template <int S>
struct __align__(128) Stage {
  double x[kRmax * S];          /* rows r0..r1-1 of X_k                      */
  double xm[rows_of<S>()];      /* ... of X_{k-1} (S <= 4)                   */
  double y[rows_of<S>()];       /* ... of Y (S <= 4, when Y is read)         */
  int ia[kRmax + 8];            /* row pointers r0..r1 (copy rounded to 16 B) */
  short dj[kEmax + 16];         /* column offsets from entry jdj on          */
  unsigned char vi[kEmax + 32]; /* value indices from entry jvi on           */
  int r0, r1, jdj, jvi, big;    /* r0 < 0: no more chunks                     */
};

/* stages in the ring: two where three would leave one block per SM (228 KB
 * of shared memory per SM, 1 KB of it reserved per block) */
template <int S>
__host__ __device__ constexpr int stages_for() {
  return S == 4 || S == 16 ? 2 : 3;
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
int g_grid_tma[5] = {0, 0, 0, 0, 0};             /* resident blocks per width, by tma_init */

__host__ __device__ constexpr int slot_of(int S) {
  return S == 1 ? 0 : S == 2 ? 1 : S == 4 ? 2 : S == 8 ? 3 : 4;
}

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
__global__ void __launch_bounds__(kWT, 2) k_cheb_il_tma(const __grid_constant__ IlTmaArgs a) {
  constexpr int NST = stages_for<S>();
  constexpr bool ALL = stage_all<S>();
  extern __shared__ __align__(128) unsigned char smem[];
  Stage<S> *st = reinterpret_cast<Stage<S> *>(smem);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + sizeof(Stage<S>) * NST);
  uint64_t *empty = full + NST;
  double *vt = reinterpret_cast<double *>(empty + NST);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  /* Y is read when the launch adds to a sum that holds terms already */
  const bool read_y = S == 1 ? !a.fresh : (a.ny > 0 && !a.fresh);
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
      /* S = 1: a chunk with an odd row count stages one row less (the copies
       * are multiples of 16 bytes); its last row is read from global */
      const unsigned b_x = (8u * S * (unsigned)(r1 - r0)) & ~15u;
      const unsigned b_xm = ALL && a.Xkm1 ? b_x : 0u;
      const unsigned b_y = ALL && read_y ? b_x : 0u;
      const unsigned b_dj = big ? 0u : round16(2u * (unsigned)(e1 - jdj));
      const unsigned b_vi = big ? 0u : round16((unsigned)(e1 - jvi));
      g.r0 = r0;
      g.r1 = r1;
      g.jdj = jdj;
      g.jvi = jvi;
      g.big = big;
      mbar_arrive_tx(&full[s], b_ia + b_x + b_xm + b_y + b_dj + b_vi);
      bulk_g2s(g.ia, a.ia + r0, b_ia, &full[s]);
      if (b_x) bulk_g2s(g.x, a.Xk + (size_t)r0 * S, b_x, &full[s]);
      if (b_xm) bulk_g2s(g.xm, a.Xkm1 + (size_t)r0 * S, b_xm, &full[s]);
      if (b_y) bulk_g2s(g.y, a.Y + (size_t)r0 * S, b_y, &full[s]);
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
    const int nr = S == 1 ? (nrows & ~1) : nrows; /* rows staged */
    for (int p = tid; p < nrows * S; p += kCW * 32) {
      const int lr = p / S, sl = p % S;
      const int row = r0 + lr;
      const size_t me = (size_t)row * S + sl;
      const bool staged = lr < nr;
      const double x = staged ? g.x[p] : a.Xk[me];
      double xm1 = 0.0, yold = 0.0;
      if (a.Xkm1) xm1 = ALL && staged ? g.xm[p] : a.Xkm1[me];
      if (read_y) yold = ALL && staged ? g.y[p] : a.Y[me];
      const int g0 = row & ~31;
      const int e = g.ia[lr + 1];
      int j = g.ia[lr];
      double r = 0.0;
      if (!big) {
        /* up to 8 entries' gathers in flight, then added in entry order (an
         * entry past the row end is skipped, never added as zero) */
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

/* dynamic shared memory above 48 KB and the resident grid of one width */
template <int S>
int setup_width() {
  const void *fn = (const void *)k_cheb_il_tma<S>;
  if (fail(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)tma_smem<S>()),
           "cudaFuncSetAttribute"))
    return PEVSL_ERR_CUDA;
  int per_sm = 0;
  if (fail(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kWT, tma_smem<S>()),
           "cudaOccupancyMaxActiveBlocksPerMultiprocessor"))
    return PEVSL_ERR_CUDA;
  if (per_sm < 1) return PEVSL_ERR_ARG;
  g_grid_tma[slot_of(S)] = per_sm * ctx().sms;
  return 0;
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

IlTmaArgs matrix_args(const pevsl_devcsr *A) {
  IlTmaArgs args;
  args.n = A->nrows;
  args.nc = A->wnc;
  args.wchunk = A->wchunk;
  args.ia = A->ia;
  args.dj = A->pdj;
  args.vi = A->pvi;
  args.vtab = A->pvtab;
  args.nv = A->pnv;
  return args;
}

}  // namespace

/* The staged kernel applies to packed matrices with a chunk table.  It is
 * off unless PEVSL_B200_IL_TMA=1: measured per degree at 100^3, its first
 * form (eight consumer warps, X_{k-1} and Y read from global) took 72.5 us
 * for 4 slices and 47.9 us for one vector against 44.0 and 22.0 us for the
 * one-thread-per-row kernels. */
bool il_tma_usable(const pevsl_devcsr *A, int S) {
  static int v = -1;
  if (v < 0) {
    const char *e = getenv("PEVSL_B200_IL_TMA");
    v = e ? atoi(e) != 0 : 0;
  }
  return v && A->pdj != nullptr && A->wchunk != nullptr && A->wnc > 0 &&
         (S == 1 || S == 2 || S == 4 || S == 8 || S == 16);
}

int cheb_step_il_tma(const pevsl_devcsr *A, int S, const double *Xk, const double *Xkm1,
                     double *Xkp1, double *Y, double cc, double t, const double *mu0,
                     const double *muk, int ny, int fresh) {
  IlTmaArgs args = matrix_args(A);
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
  IlTmaArgs args = matrix_args(A);
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
