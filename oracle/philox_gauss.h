/*
 * Counter-based Gaussian random vectors for the oracle (TEST INFRASTRUCTURE).
 *
 * The pEVSL reference draws its random vectors from glibc rand(), uniform on
 * [-1,1] (SRC/parvec.c:65-72), seeded once by srand(rank) (SRC/pevsl.c:36).
 * The seeded-Gaussian workloads instead use this generator, which the CUDA
 * path reproduces on the device:
 *
 *   draw m (0,1,2,... per process since the last reseed), element pair p:
 *     (r0,r1,r2,r3) = Philox4x32-10(counter = {p_lo, p_hi, m_lo, m_hi},
 *                                   key     = {seed_lo, seed_hi})
 *     u1 = ((r0:r1 >> 11) + 0.5) * 2^-53      in (0,1)
 *     u2 =  (r2:r3 >> 11)        * 2^-53      in [0,1)
 *     rad = sqrt(-2 log u1)
 *     x[2p] = rad cos(2 pi u2),  x[2p+1] = rad sin(2 pi u2)
 *
 * Philox4x32-10 is the counter-based generator of Salmon, Moraes, Dror and
 * Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC'11): ten rounds of
 * two 32x32->64 multiplies with multipliers 0xD2511F53 / 0xCD9E8D57 and a
 * Weyl key schedule with increments 0x9E3779B9 / 0xBB67AE85.  Box-Muller is
 * the classical polar-free transform.
 */
#ifndef ORACLE_PHILOX_GAUSS_H
#define ORACLE_PHILOX_GAUSS_H

#include <math.h>
#include <stdint.h>

static inline void orc_philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int round = 0; round < 10; round++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * (uint64_t)c[0];
    uint64_t p1 = (uint64_t)0xCD9E8D57u * (uint64_t)c[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c[1] ^ k0;
    uint32_t n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

/* Fill x[0..n) with draw number m of the Gaussian stream for this seed. */
static inline void orc_gauss_vector(double *x, long n, uint64_t seed, uint64_t m) {
  const double two_pi = 6.283185307179586476925286766559;
  const double inv53 = 1.0 / 9007199254740992.0; /* 2^-53 */
  for (long p = 0; 2 * p < n; p++) {
    uint32_t c[4] = {(uint32_t)p, (uint32_t)((uint64_t)p >> 32), (uint32_t)m,
                     (uint32_t)(m >> 32)};
    orc_philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    uint64_t a = (((uint64_t)c[0] << 32) | c[1]) >> 11;
    uint64_t b = (((uint64_t)c[2] << 32) | c[3]) >> 11;
    double u1 = ((double)a + 0.5) * inv53;
    double u2 = (double)b * inv53;
    double rad = sqrt(-2.0 * log(u1));
    double ang = two_pi * u2;
    x[2 * p] = rad * cos(ang);
    if (2 * p + 1 < n) {
      x[2 * p + 1] = rad * sin(ang);
    }
  }
}

#endif
