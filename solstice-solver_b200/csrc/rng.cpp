/*
 * rng.cpp - the ssp_rng shim (see include/ssp.h): a Philox4x32-10 stream
 * keyed by a 64-bit seed with a 64-bit position.
 */
#include "objects.h"
#include "philox.h"

#include <cinttypes>
#include <new>

extern "C" res_T ssp_rng_create
  (struct mem_allocator* allocator, const enum ssp_rng_type type,
   ssp_rng** out)
{
  (void)allocator;
  if(!out || (unsigned)type >= SSP_RNG_TYPES_COUNT__) return RES_BAD_ARG;
  ssp_rng* r = new (std::nothrow) ssp_rng();
  if(!r) return RES_MEM_ERR;
  r->type = type;
  *out = r;
  return RES_OK;
}

extern "C" res_T ssp_rng_ref_get(ssp_rng* r)
{
  if(!r) return RES_BAD_ARG;
  r->ref.get();
  return RES_OK;
}

extern "C" res_T ssp_rng_ref_put(ssp_rng* r)
{
  if(!r) return RES_BAD_ARG;
  if(r->ref.put()) delete r;
  return RES_OK;
}

extern "C" res_T ssp_rng_get_type(const ssp_rng* r, enum ssp_rng_type* type)
{
  if(!r || !type) return RES_BAD_ARG;
  *type = r->type;
  return RES_OK;
}

extern "C" res_T ssp_rng_set(ssp_rng* r, const uint64_t seed)
{
  if(!r) return RES_BAD_ARG;
  r->seed = seed;
  r->position = 0;
  return RES_OK;
}

extern "C" uint64_t ssp_rng_get(ssp_rng* r)
{
  const ssolb::U32x4 x = ssolb::philox4x32_10
    ((uint32_t)r->position, (uint32_t)(r->position >> 32), 0u,
     ssolb::RNG_HOST, (uint32_t)r->seed, (uint32_t)(r->seed >> 32));
  ++r->position;
  return ((uint64_t)x.v[0] << 32) | x.v[1];
}

extern "C" double ssp_rng_canonical(ssp_rng* r)
{
  return (double)(ssp_rng_get(r) >> 11) * 0x1.0p-53;
}

extern "C" float ssp_rng_canonical_float(ssp_rng* r)
{
  return (float)(ssp_rng_get(r) >> 40) * 0x1.0p-24f;
}

extern "C" res_T ssp_rng_discard(ssp_rng* r, uint64_t n)
{
  if(!r) return RES_BAD_ARG;
  r->position += n;
  return RES_OK;
}

extern "C" res_T ssp_rng_write(const ssp_rng* r, FILE* stream)
{
  if(!r || !stream) return RES_BAD_ARG;
  if(fprintf(stream, "philox4x32-10 %d %" PRIu64 " %" PRIu64 "\n",
             (int)r->type, r->seed, r->position) < 0)
    return RES_IO_ERR;
  return RES_OK;
}

extern "C" res_T ssp_rng_read(ssp_rng* r, FILE* stream)
{
  if(!r || !stream) return RES_BAD_ARG;
  int type = 0;
  uint64_t seed = 0, pos = 0;
  if(fscanf(stream, " philox4x32-10 %d %" SCNu64 " %" SCNu64, &type, &seed,
            &pos) != 3)
    return RES_IO_ERR;
  if(type < 0 || type >= SSP_RNG_TYPES_COUNT__) return RES_IO_ERR;
  r->type = (ssp_rng_type)type;
  r->seed = seed;
  r->position = pos;
  return RES_OK;
}

res_T ssolb_rng_clone_advanced(const ssp_rng* src, uint64_t adv, ssp_rng** out)
{
  ssp_rng* r = new (std::nothrow) ssp_rng();
  if(!r) return RES_MEM_ERR;
  r->type = src->type;
  r->seed = src->seed;
  r->position = src->position + adv;
  *out = r;
  return RES_OK;
}
