/*
 * trk_philox.h -- the random numbers of incoherent synchrotron radiation:
 * Philox4x32-10, the counter-based generator of Salmon, Moraes, Dror and
 * Shaw ("Parallel random numbers: as easy as 1, 2, 3", SC 2011), and a
 * standard normal deviate truncated at +-limit from two of its outputs by the
 * Box-Muller transform.  A deviate is a pure function of (seed, particle ID,
 * pass, element, kick, attempt), so a run does not depend on the launch
 * shape, the particle order or the number of GPUs, and the CPU oracle draws
 * the same numbers.  Compiles as CUDA device code and as host C.
 */
#ifndef TRK_PHILOX_H
#define TRK_PHILOX_H
#include <stdint.h>

#ifdef __CUDACC__
#define TRKPX_FN __host__ __device__ __forceinline__
#else
#define TRKPX_FN static inline
#endif

TRKPX_FN void trk_philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; r++) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
    c[1] = (uint32_t)p1;
    c[3] = (uint32_t)p0;
    c[0] = n0;
    c[2] = n2;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

/* uniform in (0, 1) from 53 bits of two words */
TRKPX_FN double trk_u53(uint32_t a, uint32_t b) {
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6) + 0.5) * (1.0 / 9007199254740992.0);
}

/* Standard normal truncated to |g| <= limit (limit > 0; the reference's
 * gauss_rn_lim redraws outside the limit, src/csbend.c:1651); at most 64
 * draws, then 0 (a chance of about 1e-160 at limit 3). */
TRKPX_FN double trk_isr_gauss(uint64_t seed, uint32_t id, uint32_t pass, uint32_t elem, uint32_t kick, double limit) {
  for (uint32_t attempt = 0; attempt < 64; attempt++) {
    uint32_t c[4] = {id, pass, elem, (kick << 6) | attempt};
    trk_philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const double u1 = trk_u53(c[0], c[1]), u2 = trk_u53(c[2], c[3]);
    const double g = sqrt(-2.0 * log(u1)) * cos(6.283185307179586476925287 * u2);
    if (!(limit > 0) || fabs(g) <= limit)
      return g;
  }
  return 0.0;
}
#endif
