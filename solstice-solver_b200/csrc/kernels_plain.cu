/*
 * kernels_plain.cu - plain FP32 launches of the realisation kernel, and the
 * per-device memory pool of the coherent order's scratch.
 */
#include "kernels_device.cuh"

namespace ssolb {

/* Per-device pool of the sort's scratch: stream-ordered allocations, so
 * that launches on different streams never share a buffer, kept by the pool
 * between launches */
cudaMemPool_t sort_pool(int dev)
{
  static cudaMemPool_t pools[64] = {};
  static std::mutex lock;
  if(dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> g(lock);
  if(!pools[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    if(cudaMemPoolCreate(&pools[dev], &props) != cudaSuccess) {
      pools[dev] = nullptr;
      return nullptr;
    }
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
  }
  return pools[dev];
}

int launch_realisations_f32
  (const DScene<float>& S, const DTallies& T, uint64_t seed, uint64_t first,
   uint64_t count, const LaunchConfig& cfg, void* stream, const DTrack* track)
{
  if(!track && !cfg.count_work)
    return launch_realisations_nocount_f32(S, T, seed, first, count, cfg, stream);
  return launch_impl<float>(S, T, seed, first, count, cfg, stream, track);
}


} /* namespace ssolb */
