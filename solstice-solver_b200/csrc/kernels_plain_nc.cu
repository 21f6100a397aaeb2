/*
 * kernels_plain_nc.cu - plain FP32 launches of the realisation kernel
 * without work counters (compiled apart so that the two sets of variants
 * build in parallel).
 */
#include "kernels_device.cuh"

namespace ssolb {

int launch_realisations_nocount_f32
  (const DScene<float>& S, const DTallies& T, uint64_t seed, uint64_t first,
   uint64_t count, const LaunchConfig& cfg, void* stream)
{ return launch_impl<float, FEAT_NOCOUNT>(S, T, seed, first, count, cfg, stream, nullptr); }

} /* namespace ssolb */
