/*
 * pevsl-b200 extensions: entry points beside the pEVSL API (pevsl.h) that
 * have no counterpart in the reference.  They select the random stream and
 * precision, expose per-call counters, and run all slices of an interval as
 * one batched solve on the GPU.
 */
#ifndef PEVSL_B200_H
#define PEVSL_B200_H

#include <stdint.h>

#include "pevsl.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Random vectors drawn by pEVSL_ParvecRand and by the solvers.
 *   PEVSL_RNG_GLIBC: the C library's rand(), uniform on [-1,1], exactly the
 *                    reference stream (SRC/parvec.c:65-72); generated on the
 *                    host, copied to the GPU.  srand(seed) is called.
 *   PEVSL_RNG_GAUSS: N(0,1) from Philox4x32-10 + Box-Muller, generated on the
 *                    GPU; vector number m of the stream is a pure function of
 *                    (seed, m), so batched draws equal sequential ones.
 * The draw counter restarts at 0.  pEVSL_Start calls srand(0) like the
 * reference but leaves the mode unchanged. */
#define PEVSL_RNG_GLIBC 0
#define PEVSL_RNG_GAUSS 1
int pEVSL_B200_SetRng(int mode, uint64_t seed);
uint64_t pEVSL_B200_RngDraws(void);

/* Arithmetic of the filter and the KPM moments on this instance.
 *   PEVSL_PREC_FP64 (default): everything in FP64, the drop-in behaviour.
 *   PEVSL_PREC_MIXED: the Chebyshev filter and the KPM moments run on FP32
 *     matrix values and FP32 vectors with FP32 accumulation; the Lanczos
 *     basis, reorthogonalisation, tridiagonal solves and Ritz vectors stay
 *     FP64.  The Lanczos convergence test allows the FP32 noise of the
 *     filter (PEVSL_B200_MIXED_TRTOL, default 1e-9 per converged Ritz
 *     value).  Before acceptance each slice gets one FP64 filtered
 *     Rayleigh-Ritz sweep: the Ritz vectors of p(A) with values
 *     >= guard * bar (PEVSL_B200_MIXED_GUARD, default 0.3; the extra ones
 *     hold the directions just outside the slice), the FP64 filter applied
 *     to them (PEVSL_B200_MIXED_PASSES times, default 1), Rayleigh-Ritz with
 *     A on the filtered block; acceptance (interval and residual < tol) is
 *     decided on the refined FP64 pairs.  A slice where a refined pair in
 *     [a, b] stays above tol is solved again in FP64, so the counts are
 *     those of the FP64 path; pEVSL_B200_LastFallbacks reports how many. */
#define PEVSL_PREC_FP64 0
#define PEVSL_PREC_MIXED 1
int pEVSL_B200_SetPrecision(pevsl_Data *pevsl, int precision);

/* Form of the batched filter: -1 automatic (= 2), 0 one launch per degree
 * serving every slice still filtering, 1 one persistent cooperative launch
 * running every degree of every slice (per-slice degree counters, a grid
 * barrier between degrees), 2 the launches of form 0 captured once per set
 * of live slices in a CUDA graph and replayed at every Lanczos step (the
 * slices' input and output pass through staging vectors in their work
 * space).  The results are the same bits in every form.
 * PEVSL_B200_FILTER_FORM sets the start value. */
int pEVSL_B200_SetFilterForm(int form);

/* Wait limit of the persistent filter's grid barrier (form 1), in polls of
 * about 64 ns; 0 restores the default (2^24 polls, about 2 s).  A wait that
 * runs out sets a flag and the kernel returns; the call that launched it
 * then returns PEVSL_ERR_CUDA (the flag is read after every filter
 * application), and the context stays usable. */
int pEVSL_B200_SetBarrierSpins(unsigned spins);

/* Fault injection for tests: preset the barrier's arrival counter to
 * `count`, so that (for count >= the grid size) no arrival completes the
 * next barrier and every wait runs out after the spin limit.  The timeout
 * report clears the counter again. */
int pEVSL_B200_SeedBarrierArrivals(unsigned count);

/* The cross-group sum of a split KPM: pEVSL_Kpmdos with ngroups > 1 computes
 * the moments of its group's share of the random vectors (pEVSL_Part1d)
 * and then, in place of MPI_Allreduce on gl_comm (SRC/kpmdos.c:160-176),
 * calls reduce(buf, Mdeg + 2, ctx) with buf = [partial moments mu[0..Mdeg],
 * partial count]; reduce must leave the sums over all groups in buf (with
 * one process per GPU: an all-reduce over the processes).  NULL restores
 * MPI. */
int pEVSL_B200_SetGroupReduce(pevsl_Data *pevsl, void (*reduce)(double *buf, int count, void *ctx),
                              void *ctx);

/* Slices of the last pEVSL_ChebLanNr / pEVSL_B200_ChebLanNrBatch /
 * pEVSL_B200_ChebLanNrMulti call that the mixed form solved again in FP64. */
int pEVSL_B200_LastFallbacks(void);

/* Lanczos steps taken by the last pEVSL_ChebLanNr on this instance, and the
 * number of Ritz values of p(A) above `bar` at its last convergence test. */
int pEVSL_B200_LastIterations(pevsl_Data *pevsl);
int pEVSL_B200_LastNconv(pevsl_Data *pevsl);

/* Number of this library's kernel launches since the process started. */
uint64_t pEVSL_B200_LaunchCount(void);

/* Device time (ms, CUDA events on the library stream) of the last call to
 * each phase: 0 bounds, 1 DOS, 2 filtered Lanczos (whole call), 3 filter
 * applications within it, 4 reorthogonalisation within it, 5 Ritz step. */
double pEVSL_B200_PhaseMs(pevsl_Data *pevsl, int phase);

/* Synchronous copy between host memory and library memory (device or
 * managed), either direction; and a wait for all queued library work. */
int pEVSL_B200_Memcpy(void *dst, const void *src, size_t bytes);

/* The first nvec eigenvectors of a pEVSL_ChebLanNr result (Wo) into the
 * caller's array: vector i (n_local values) to vec + i * ld, ld >= n_local;
 * vec may be host or device memory.  What the reference's Fortran
 * pevsl_copy_result does for its saved result (FORTRAN/pevsl_f90.c:311-331),
 * as one strided copy. */
int pEVSL_B200_CopyEigenvectors(const pevsl_Parvecs *W, int nvec, double *vec, long ld);
int pEVSL_B200_Sync(void);

/* Sticky CUDA error of the void entry points (pEVSL_Parvec*, ...): returns
 * the first PEVSL_ERR_* met since the last call, then clears it. */
int pEVSL_B200_LastError(void);

/* y = p(A) v for the filter in pol (what pEVSL_ChebAv, internal to the
 * reference at SRC/chebpol.c:509, computes); v and y are device or managed
 * vectors of length pevsl->n. */
int pEVSL_B200_ChebAv(pevsl_Data *pevsl, pevsl_Polparams *pol, const double *v, double *y);

/* The same for the generalized problem: y = p(A B^{-1}) v, each degree a
 * solve with the instance's B-solve callback (SRC/chebpol.c:543-546). */
int pEVSL_B200_ChebAvGen(pevsl_Data *pevsl, pevsl_Polparams *pol, const double *v, double *y);

/* Host only (no device needed): the least-squares Chebyshev coefficients
 * that pEVSL_SetupLSPolRec (kind 0, f = 1/x) or pEVSL_SetupLSPolSqrt
 * (kind 1, f = 1/sqrt(x)) computes for [lmin, lmax]: mu[0..*deg] (mu holds
 * max_deg entries), centre *cc and half-width *dd. */
int pEVSL_B200_LSPolCoefs(int kind, int max_deg, double tol, double lmin, double lmax, double *mu,
                          int *deg, double *cc, double *dd);
/* degree of a set-up least-squares solver; its coefficients into
 * mu_out[0..min(deg, cap-1)] when mu_out is not NULL */
int pEVSL_B200_LSPolDegree(const void *vdata, double *mu_out, int cap);

/* pEVSL_ChebLanNr for nslices slices at once.  The slices advance in
 * lockstep (up to 256 per group): one fused filter launch per polynomial
 * degree serves every slice still filtering (the matrix is read once per
 * degree for all of them), or (PEVSL_B200_FILTER_FORM=1) one persistent
 * launch runs every degree;
 * the reorthogonalisation kernels run batched, and one host read per Lanczos
 * step fetches all slices' recurrence scalars.  Slice s uses
 * intvs[4s..4s+3], pols[s], maxits[s]; its outputs are nevOut[s], lamo[s],
 * Wo[s], reso[s] (allocated as by pEVSL_ChebLanNr), its[s] (Lanczos steps)
 * and status[s] (pEVSL_ChebLanNr's return code).  Returns the first
 * nonzero status.  The results equal pEVSL_ChebLanNr called slice by slice,
 * except that a lucky-breakdown restart draws its random vector in lockstep
 * order rather than after the preceding slices have finished. */
int pEVSL_B200_ChebLanNrBatch(pevsl_Data *pevsl, int nslices, const double *intvs,
                              const int *maxits, double tol, pevsl_Parvec *vinit,
                              pevsl_Polparams *pols, int *nevOut, double **lamo,
                              pevsl_Parvecs **Wo, double **reso, int *its, int *status,
                              FILE *fstats);

/* pEVSL_B200_ChebLanNrBatch for several problems at once: problem p (its
 * own instance pevsls[p], matrix and start vector vinits[p]) has nslices[p]
 * slices, stored one after the other in intvs (4 doubles each), maxits,
 * pols and the per-slice outputs.  All slices of all problems advance in
 * lockstep (up to 256 per group); every filter degree of a step is one
 * launch over all slices still filtering, each with its own matrix,
 * polynomial and degree (or one persistent launch for all degrees, see
 * pEVSL_B200_SetFilterForm).  Each slice's result equals solving it
 * alone. */
int pEVSL_B200_ChebLanNrMulti(int nprob, pevsl_Data **pevsls, const int *nslices,
                              const double *intvs, const int *maxits, double tol,
                              pevsl_Parvec **vinits, pevsl_Polparams *pols, int *nevOut,
                              double **lamo, pevsl_Parvecs **Wo, double **reso, int *its,
                              int *status, FILE *fstats);

/* w = V(:, 0:k)' x (the projection of pEVSL_ParvecsGemtv) without any device
 * allocation; no counterpart in the reference.  For callers that must not
 * let the library allocate: a framework that owns all device memory through
 * its own pool, latency-critical loops that cannot take cudaMalloc's device
 * synchronisation, programs with a fixed memory budget.  V (column major,
 * n x k, leading dimension ld >= n), x (n) and w (k) are device pointers
 * owned by the caller; stream is a cudaStream_t or NULL (legacy default
 * stream).  The only workspace is a fixed 256 KiB array that the library
 * holds on every GPU it is loaded on, so k is limited to 1..256 (other
 * values return PEVSL_ERR_ARG).  The first call on a device looks up that
 * array's device address, so make it before any stream capture.  All calls
 * on a device share the array: calls that overlap on the GPU race. */
int pEVSL_B200_ParvecsGemtvNoAlloc(const double *V, long n, long ld, int k, const double *x,
                                   double *w, void *stream);

/* The two dense products of the solvers, on the FP64 tensor cores (DMMA,
 * mma.sync m8n8k4), for device pointers, column-major, on the library
 * stream: U = V(:, 0:k) Y (n x m; V n x k, leading dimension ldv; Y k x m,
 * ldy) -- the Ritz vectors (SRC/cheblanNr.c:363-365) -- and C = V' W (k x m;
 * W n x m, ldw) -- the Gram matrices of the refinement sweep, the block form
 * of GemtvWithWspace (SRC/parvecs.c:117-136).  Deterministic: a fixed
 * partition of the rows and a fixed order of the partial sums. */
int pEVSL_B200_GemmNN(long n, int k, int m, const double *V, long ldv, const double *Y, long ldy,
                      double *U, long ldu);
int pEVSL_B200_GemmTN(long n, int k, int m, const double *V, long ldv, const double *W, long ldw,
                      double *C, long ldc);

/* Release cached device workspaces (they are reused across calls). */
void pEVSL_B200_ReleaseWorkspace(void);

/* Device used by the library (call before any other entry point); by
 * default the environment variable PEVSL_B200_DEVICE, else LOCAL_RANK of a
 * one-process-per-GPU launcher, else device 0. */
int pEVSL_B200_SetDevice(int device);

/* CUDA events (slots 0..15) recorded on the library stream, and the device
 * time between two of them (waits for the second). */
int pEVSL_B200_EventRecord(int slot);
double pEVSL_B200_EventElapsedMs(int a, int b);

/* Page-locked host memory for fast host<->device copies of inputs. */
void *pEVSL_B200_HostAlloc(size_t bytes);
void pEVSL_B200_HostFree(void *p);
/* CUDA managed memory: the host may read and write it between library calls
 * (after pEVSL_B200_Sync) */
void *pEVSL_B200_ManagedAlloc(size_t bytes);
void pEVSL_B200_ManagedFree(void *p);

/* Counters of the fused Chebyshev filter kernel since the last reset:
 * launches inside pEVSL_ChebLanNr, their algorithmic bytes (CSR + vectors),
 * and the device time of the filter applications that contain them. */
void pEVSL_B200_FilterCounters(uint64_t *launches, double *bytes, double *ms);
void pEVSL_B200_ResetFilterCounters(void);

/* The generalized filter's counters since the last reset: filter
 * applications and degrees inside pEVSL_ChebLanNr with ifGenEv, their
 * algorithmic HBM bytes (per degree: the B-solve's matrix passes and
 * vectors, and the fused A step) and the device time of the applications
 * (CUDA events around each). */
void pEVSL_B200_GenCounters(uint64_t *filters, uint64_t *degrees, double *bytes, double *ms);

/* Benchmark helper: write `bytes` (0: 256 MiB, twice the L2) of a scratch
 * device buffer on the library stream, evicting earlier data from L2. */
int pEVSL_B200_FlushL2(size_t bytes);
void pEVSL_B200_ResetGenCounters(void);

/* Short build/device description into buf (NUL-terminated). */
int pEVSL_B200_Info(char *buf, int len);

/* ---------------------------------------------------------------- learned DOS
 * A small MLP with BF16 weights and activations and FP32 accumulation,
 * trained and run by this library's own GPU kernels (tensor-core BF16 GEMM
 * with fused bias/GELU epilogues, GELU' in the backward pass, Adam on FP32
 * master weights).  Layers: nin -> width -> ... -> width -> nout with GELU
 * between them ("layers" linear maps); dimensions are padded to multiples
 * of 16 inside.  The learned DOS maps KPM moments from a few random
 * vectors to the moments of many (pevsl_b200/learned.py drives it). */
typedef struct pevsl_mlp pevsl_mlp;
int pEVSL_B200_MlpCreate(pevsl_mlp **net, int nin, int width, int nout, int layers);
void pEVSL_B200_MlpFree(pevsl_mlp *net);
/* parameters incl. padding; per layer l: K_l, N_l (padded), and the offsets
 * of W_l (N_l x K_l, row-major) and b_l (N_l) in the parameter block;
 * returns the number of layers */
long pEVSL_B200_MlpParamCount(const pevsl_mlp *net);
int pEVSL_B200_MlpLayout(const pevsl_mlp *net, int *kdim, int *ndim, long *woff, long *boff);
/* FP32 master parameters from / to host memory (setting resets Adam) */
int pEVSL_B200_MlpSetParams(pevsl_mlp *net, const float *host);
int pEVSL_B200_MlpGetParams(const pevsl_mlp *net, float *host);
/* Y [B][nout] = net(X [B][nin]), row-major FP32 device arrays */
int pEVSL_B200_MlpForward(pevsl_mlp *net, const float *X, float *Y, int B);
/* mean squared error against T [B][nout] and its gradient (host FP32, the
 * parameter layout); the weights are not changed */
int pEVSL_B200_MlpGradients(pevsl_mlp *net, const float *X, const float *T, int B, float *loss,
                            float *grad_host);
/* one Adam step (beta 0.9 / 0.999) on (X, T); *loss = the loss before it */
int pEVSL_B200_MlpTrainStep(pevsl_mlp *net, const float *X, const float *T, int B, float lr,
                            float *loss);

#ifdef __cplusplus
}
#endif

#endif
