/*
 * philox.h - Philox4x32-10 counter-based generator (Salmon, Moraes, Dror,
 * Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11).
 *
 * Used on the host (ssp_rng shim) and on the device (per realisation
 * streams). A draw is a pure function of (counter, key): realisation i of a
 * solve keyed by `seed` reads block Philox(ctr = {i_lo, i_hi, event, domain},
 * key = {seed_lo, seed_hi}); no state is stored between events.
 */
#ifndef SSOL_B200_PHILOX_H
#define SSOL_B200_PHILOX_H

#include <stdint.h>

#ifdef __CUDACC__
  #define PHILOX_HD __host__ __device__ __forceinline__
#else
  #define PHILOX_HD inline
#endif

namespace ssolb {

struct U32x4 { uint32_t v[4]; };

PHILOX_HD void philox_mulhilo(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo)
{
#ifdef __CUDA_ARCH__
  lo = a * b;
  hi = __umulhi(a, b);
#else
  const uint64_t p = (uint64_t)a * (uint64_t)b;
  lo = (uint32_t)p;
  hi = (uint32_t)(p >> 32);
#endif
}

PHILOX_HD U32x4 philox4x32_10
  (uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
   uint32_t k0, uint32_t k1)
{
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for(int r = 0; r < 10; ++r) {
    if(r) { k0 += W0; k1 += W1; }
    uint32_t hi0, lo0, hi1, lo1;
    philox_mulhilo(M0, c0, hi0, lo0);
    philox_mulhilo(M1, c2, hi1, lo1);
    const uint32_t n0 = hi1 ^ c1 ^ k0;
    const uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
  }
  U32x4 out;
  out.v[0] = c0; out.v[1] = c1; out.v[2] = c2; out.v[3] = c3;
  return out;
}

/* Uniform in [0, 1) with 24 significant bits: exactly representable in both
 * float and double, so the FP32 and FP64 builds see identical numbers */
PHILOX_HD float u01f(uint32_t x) { return (float)(x >> 8) * 0x1.0p-24f; }
PHILOX_HD double u01d(uint32_t x) { return (double)(x >> 8) * 0x1.0p-24; }

/* Stream domains of one realisation */
enum : uint32_t {
  RNG_PRIMARY = 0u, /* event 0: sample, 1: sun dir + wavelength, 2+: Buie */
  RNG_SCATTER = 1u, /* event j: j-th BSDF sample of the path */
  RNG_ROULETTE = 2u, /* event r: r-th Russian roulette draw */
  RNG_RETRY = 3u, /* event (j << 6) | k: k-th microfacet re-draw at bounce j */
  /* Renderers: stream id = pixel x samples per pixel + sample (path
   * tracer) or sample index (draft sub-pixel offsets, key 0) */
  RNG_DRAW_OFFSET = 4u, /* event 0: draft sub-pixel offset of sample i */
  RNG_DRAW_PIXEL = 5u, /* event 0: sub-pixel position of a camera sample */
  RNG_DRAW_WL = 6u, /* event a: wavelength of attempt a */
  RNG_DRAW_BSDF = 7u, /* event (a << 20) | b: BSDF sample at bounce b */
  RNG_DRAW_RR = 8u, /* event (a << 20) | b: roulette draw at bounce b */
  RNG_HOST = 0xffffffffu /* ssp_rng_get on the host */
};

} /* namespace ssolb */

#endif /* SSOL_B200_PHILOX_H */
