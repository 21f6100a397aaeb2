/*
 * kernels_plain64.cu - plain all-FP64 launches of the realisation kernel.
 */
#include "kernels_device.cuh"

namespace ssolb {

int launch_realisations_f64
  (const DScene<double>& S, const DTallies& T, uint64_t seed, uint64_t first,
   uint64_t count, const LaunchConfig& cfg, void* stream, const DTrack* track)
{ return launch_impl<double>(S, T, seed, first, count, cfg, stream, track); }

} /* namespace ssolb */
