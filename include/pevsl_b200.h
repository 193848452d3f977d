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
int pEVSL_B200_Sync(void);

/* Sticky CUDA error of the void entry points (pEVSL_Parvec*, ...): returns
 * the first PEVSL_ERR_* met since the last call, then clears it. */
int pEVSL_B200_LastError(void);

/* y = p(A) v for the filter in pol (what pEVSL_ChebAv, internal to the
 * reference at SRC/chebpol.c:509, computes); v and y are device or managed
 * vectors of length pevsl->n. */
int pEVSL_B200_ChebAv(pevsl_Data *pevsl, pevsl_Polparams *pol, const double *v, double *y);

/* Release cached device workspaces (they are reused across calls). */
void pEVSL_B200_ReleaseWorkspace(void);

/* Short build/device description into buf (NUL-terminated). */
int pEVSL_B200_Info(char *buf, int len);

#ifdef __cplusplus
}
#endif

#endif
