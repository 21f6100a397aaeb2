/*
 * kernels_batch_nc.cu - batched FP32 launches without work counters
 * (compiled apart so that the two sets of variants build in parallel).
 */
#include "kernels_device.cuh"

namespace ssolb {

int launch_batch_nocount_f32(const BatchLaunch<float>& b, const LaunchConfig& cfg,
                             void* stream)
{ return launch_batch_impl<float, FEAT_NOCOUNT>(b, cfg, stream); }

} /* namespace ssolb */
