/*
 * ssp.h - minimal random number generator shim for the `ssol_solve` ABI.
 *
 * `ssol_solve` takes a `const struct ssp_rng*` (reference: src/ssol.h:1216,
 * where the type comes from Star-SP 0.12, a dependency that is not in the
 * reference tree). This header provides the subset of the Star-SP RNG API
 * that callers of the solver use (create, ref counting, draws, type query and
 * state (de)serialisation, as in src/test_ssol_solver1.c:115, 246-257).
 *
 * Every generator, whatever its type tag, is a counter-based Philox4x32-10
 * stream. Its state is (seed, position). `ssol_solve` uses the state as the
 * key of its per-realisation streams: realisation i of a solve started from
 * (seed, position) draws from Philox(key = seed, counter = position + i, ...).
 * The estimator's end state is (seed, position + realisations), so a solve
 * resumed from it never reuses a stream of the first one. The Star-SP
 * THREEFRY sequence itself is not reproduced.
 */
#ifndef SSP_H
#define SSP_H

#include <stdint.h>
#include <stdio.h>

#ifndef SSOL_RES_T_DEFINED
#define SSOL_RES_T_DEFINED
typedef int res_T;
#define RES_OK 0
#define RES_BAD_ARG 1
#define RES_MEM_ERR 2
#define RES_IO_ERR 3
#define RES_UNKNOWN_ERR 4
#define RES_BAD_OP 5
#define RES_EOF 6
#endif

#if defined(SSOL_SHARED_BUILD)
  #define SSP_API extern __attribute__((visibility("default")))
#else
  #define SSP_API extern
#endif

#ifdef __cplusplus
extern "C" {
#endif

struct mem_allocator;
struct ssp_rng;

/* Type tags accepted for source compatibility; all map to Philox4x32-10. */
enum ssp_rng_type {
  SSP_RNG_KISS,
  SSP_RNG_MT19937_64,
  SSP_RNG_RANLUX48,
  SSP_RNG_RANDOM_DEVICE,
  SSP_RNG_THREEFRY,
  SSP_RNG_AES,
  SSP_RNG_TYPES_COUNT__
};

SSP_API res_T ssp_rng_create
  (struct mem_allocator* allocator, const enum ssp_rng_type type,
   struct ssp_rng** rng);
SSP_API res_T ssp_rng_ref_get(struct ssp_rng* rng);
SSP_API res_T ssp_rng_ref_put(struct ssp_rng* rng);
SSP_API res_T ssp_rng_get_type
  (const struct ssp_rng* rng, enum ssp_rng_type* type);
/* Reset the stream: key = seed, position = 0 */
SSP_API res_T ssp_rng_set(struct ssp_rng* rng, const uint64_t seed);
/* 64 random bits */
SSP_API uint64_t ssp_rng_get(struct ssp_rng* rng);
/* Uniform in [0, 1) */
SSP_API double ssp_rng_canonical(struct ssp_rng* rng);
SSP_API float ssp_rng_canonical_float(struct ssp_rng* rng);
/* Skip `n` draws */
SSP_API res_T ssp_rng_discard(struct ssp_rng* rng, uint64_t n);
/* Text serialisation of (type, seed, position) */
SSP_API res_T ssp_rng_write(const struct ssp_rng* rng, FILE* stream);
SSP_API res_T ssp_rng_read(struct ssp_rng* rng, FILE* stream);

#ifdef __cplusplus
}
#endif

#endif /* SSP_H */
