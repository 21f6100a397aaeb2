/*
 * kernels_batch.cu - batched launches (several scenes in one persistent
 * launch), with and without library allocations.
 */
#include "kernels_device.cuh"

namespace ssolb {

int launch_batch_f32(const BatchLaunch<float>& b, const LaunchConfig& cfg,
                     void* stream)
{
  if(!cfg.count_work) return launch_batch_nocount_f32(b, cfg, stream);
  return launch_batch_impl<float>(b, cfg, stream);
}

int launch_batch_f64(const BatchLaunch<double>& b, const LaunchConfig& cfg,
                     void* stream)
{ return launch_batch_impl<double>(b, cfg, stream); }

/* Scratch of the no-allocation batched launch: one file-scope device array
 * holding the budget prefix sums (NOALLOC_MAX_ITEMS + 1 words), the
 * per-item first realisation ids (NOALLOC_MAX_ITEMS words), the per-item
 * work counters (NOALLOC_MAX_ITEMS words) and the launch counters (DStats):
 * 96 KiB. Every call on a device shares it. */
constexpr size_t NOALLOC_PREFIX = 0;
constexpr size_t NOALLOC_FIRSTS = NOALLOC_MAX_ITEMS + 1;
constexpr size_t NOALLOC_NEXT = 2 * NOALLOC_MAX_ITEMS + 1;
constexpr size_t NOALLOC_STATS = 3 * NOALLOC_MAX_ITEMS + 1;
constexpr size_t NOALLOC_WORDS =
  NOALLOC_STATS + sizeof(DStats) / sizeof(unsigned long long);
static __device__ __align__(256) unsigned long long
  g_noalloc_scratch[NOALLOC_WORDS];

/* Device address of the scratch array, resolved once per device with that
 * device current: the host-side name of a __device__ array is a stand-in,
 * not an address a kernel may be given */
static int noalloc_scratch_address(unsigned long long** out)
{
  /* Atomic entries: two host threads may make their first call on a device
   * at the same time (both then store the same address) */
  static std::atomic<unsigned long long*> cache[64] = {};
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if(err != cudaSuccess) return (int)err;
  if(dev < 0 || dev >= 64) return (int)cudaErrorInvalidDevice;
  unsigned long long* addr = cache[dev].load(std::memory_order_acquire);
  if(!addr) {
    void* ptr = nullptr;
    err = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if(err != cudaSuccess) return (int)err;
    addr = (unsigned long long*)ptr;
    cache[dev].store(addr, std::memory_order_release);
  }
  *out = addr;
  return 0;
}

template<class R, int MINB, int FEAT>
static int launch_batch_noalloc_variant
  (const DScene<R>* scenes, const DTallies* tallies, int nitems, uint64_t seed,
   const unsigned long long* h_prefix, const unsigned long long* h_firsts,
   const LaunchConfig& cfg, void* stream)
{
  if(nitems < 1 || nitems > NOALLOC_MAX_ITEMS) return (int)cudaErrorInvalidValue;
  unsigned long long* scratch = nullptr;
  int err = noalloc_scratch_address(&scratch);
  if(err) return err;
  const cudaStream_t s = (cudaStream_t)stream;
  int dev = 0;
  cudaGetDevice(&dev);
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int block = cfg.block_size > 0 ? cfg.block_size : MAX_BLOCK;
  if(block > MAX_BLOCK || block % 32) return (int)cudaErrorInvalidValue;
  const size_t smem = (size_t)((2 * NGLOBAL + PS_COUNT) * block) * sizeof(double)
                    + (size_t)SMEM_STACK * block * sizeof(int)
                    + (size_t)(block / 32) * 2 * (2 * NGLOBAL + cfg.rcv_doubles) * sizeof(double)
                    + (size_t)(block / 32) * 2 * sizeof(DScene<R>);
  raise_smem_limit<BatchTag<R, MINB, FEAT>>(batch_kernel<R, MINB, FEAT>, dev);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor
    (&per_sm, batch_kernel<R, MINB, FEAT>, block, smem);
  if(per_sm < 1) per_sm = 1;
  const uint64_t blocks = cfg.grid_blocks > 0
    ? (uint64_t)cfg.grid_blocks
    : (uint64_t)nsm * (uint64_t)per_sm * (uint64_t)(cfg.waves > 0 ? cfg.waves : 1);
  /* Budgets and stream offsets of this call; the work counter and launch
   * counters start at zero (the array keeps the previous call's values) */
  cudaError_t e;
  e = cudaMemcpyAsync(scratch + NOALLOC_PREFIX, h_prefix,
                      (size_t)(nitems + 1) * sizeof(unsigned long long),
                      cudaMemcpyHostToDevice, s);
  if(e != cudaSuccess) return (int)e;
  e = cudaMemcpyAsync(scratch + NOALLOC_FIRSTS, h_firsts,
                      (size_t)nitems * sizeof(unsigned long long),
                      cudaMemcpyHostToDevice, s);
  if(e != cudaSuccess) return (int)e;
  e = cudaMemsetAsync(scratch + NOALLOC_NEXT, 0,
                      (NOALLOC_WORDS - NOALLOC_NEXT) * sizeof(unsigned long long), s);
  if(e != cudaSuccess) return (int)e;
  batch_kernel<R, MINB, FEAT><<<(unsigned)blocks, block, smem, s>>>
    (scenes, tallies, scratch + NOALLOC_PREFIX, scratch + NOALLOC_FIRSTS, nitems,
     seed, cfg.max_segments, scratch + NOALLOC_NEXT,
     reinterpret_cast<DStats*>(scratch + NOALLOC_STATS), cfg.rcv_doubles,
     nullptr, nullptr, nullptr); /* id order: the coherent order needs scratch */
  return (int)cudaGetLastError();
}

template<class R>
static int launch_batch_noalloc_impl
  (const DScene<R>* scenes, const DTallies* tallies, int nitems, uint64_t seed,
   const unsigned long long* h_prefix, const unsigned long long* h_firsts,
   const LaunchConfig& cfg, void* stream)
{
  if(sizeof(R) == sizeof(float) && cfg.features == 0) {
    switch(cfg.min_blocks) {
      case 1: return launch_batch_noalloc_variant<R, 1, 0>
        (scenes, tallies, nitems, seed, h_prefix, h_firsts, cfg, stream);
      case 3: return launch_batch_noalloc_variant<R, 3, 0>
        (scenes, tallies, nitems, seed, h_prefix, h_firsts, cfg, stream);
      default: return launch_batch_noalloc_variant<R, 2, 0>
        (scenes, tallies, nitems, seed, h_prefix, h_firsts, cfg, stream);
    }
  }
  switch(cfg.min_blocks) {
    case 1: return launch_batch_noalloc_variant<R, 1, FEAT_ALL>
      (scenes, tallies, nitems, seed, h_prefix, h_firsts, cfg, stream);
    case 3: return launch_batch_noalloc_variant<R, 3, FEAT_ALL>
      (scenes, tallies, nitems, seed, h_prefix, h_firsts, cfg, stream);
    default: return launch_batch_noalloc_variant<R, 2, FEAT_ALL>
      (scenes, tallies, nitems, seed, h_prefix, h_firsts, cfg, stream);
  }
}

int launch_batch_noalloc_f32
  (const DScene<float>* scenes, const DTallies* tallies, int nitems,
   uint64_t seed, const unsigned long long* h_prefix,
   const unsigned long long* h_firsts, const LaunchConfig& cfg, void* stream)
{
  return launch_batch_noalloc_impl<float>
    (scenes, tallies, nitems, seed, h_prefix, h_firsts, cfg, stream);
}

int launch_batch_noalloc_f64
  (const DScene<double>* scenes, const DTallies* tallies, int nitems,
   uint64_t seed, const unsigned long long* h_prefix,
   const unsigned long long* h_firsts, const LaunchConfig& cfg, void* stream)
{
  return launch_batch_noalloc_impl<double>
    (scenes, tallies, nitems, seed, h_prefix, h_firsts, cfg, stream);
}

} /* namespace ssolb */

namespace ssolb {

/*******************************************************************************
 * Tracking batches: re-aimed heliostats and refitted BVHs, built per item on
 * the device from one snapshot
 ******************************************************************************/

/* FP64 arithmetic rounded operation by operation (no FMA contraction), in
 * the order the host builds a scene's transforms and vertices, so that a
 * re-aimed triangle gets the FP32 vertices a host snapshot of the re-aimed
 * scene would */
__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ds(double a, double b) { return __dsub_rn(a, b); }

__device__ __forceinline__ void unit3(double v[3])
{
  const double l = sqrt(da(da(dm(v[0], v[0]), dm(v[1], v[1])), dm(v[2], v[2])));
  v[0] = __ddiv_rn(v[0], l);
  v[1] = __ddiv_rn(v[1], l);
  v[2] = __ddiv_rn(v[2], l);
}

/* Rotation of a heliostat at `pos` aiming at `aim` under the sun toward
 * `to_sun`: its local +z (the mirror normal) bisects the directions to the
 * sun and to the aim point, its local x axis is horizontal, up x n (or +x
 * when the normal is vertical), y = n x x. Columns x, y, n. */
__device__ void tracking_frame(const double pos[3], const double aim[3],
                               const double to_sun[3], double X[3], double Y[3],
                               double N[3])
{
  double a[3] = {ds(aim[0], pos[0]), ds(aim[1], pos[1]), ds(aim[2], pos[2])};
  unit3(a);
  N[0] = da(to_sun[0], a[0]);
  N[1] = da(to_sun[1], a[1]);
  N[2] = da(to_sun[2], a[2]);
  unit3(N);
  unit3(N);
  /* up x N with up = (0, 0, 1) */
  X[0] = -N[1];
  X[1] = N[0];
  X[2] = 0.0;
  if(da(dm(X[0], X[0]), dm(X[1], X[1])) < 1e-12) {
    X[0] = 1.0;
    X[1] = 0.0;
  }
  unit3(X);
  Y[0] = ds(dm(N[1], X[2]), dm(N[2], X[1]));
  Y[1] = ds(dm(N[2], X[0]), dm(N[0], X[2]));
  Y[2] = ds(dm(N[0], X[1]), dm(N[1], X[0]));
}

template<class R>
__global__ void __launch_bounds__(256) track_triangles_kernel(const TrackArgs A)
{
  const size_t total = (size_t)A.nitems * (size_t)A.ntracked;
  for(size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < total;
      g += (size_t)gridDim.x * blockDim.x) {
    const int item = (int)(g / (size_t)A.ntracked);
    const int t = (int)(g % (size_t)A.ntracked);
    const int h = A.tri_helio[t];
    double X[3], Y[3], N[3];
    tracking_frame(A.helio + 6 * h, A.helio + 6 * h + 3, A.to_sun + 3 * item, X, Y, N);
    const double* p = A.helio + 6 * h;
    const double* l = A.local + 9 * (size_t)t;
    float vf[3][3];
    for(int k = 0; k < 3; ++k) {
      const double* q = l + 3 * k;
      vf[k][0] = (float)da(da(da(dm(X[0], q[0]), dm(Y[0], q[1])), dm(N[0], q[2])), p[0]);
      vf[k][1] = (float)da(da(da(dm(X[1], q[0]), dm(Y[1], q[1])), dm(N[1], q[2])), p[1]);
      vf[k][2] = (float)da(da(da(dm(X[2], q[0]), dm(Y[2], q[1])), dm(N[2], q[2])), p[2]);
    }
    DTri<R>* tris = (DTri<R>*)A.tris + (size_t)item * A.tri_stride;
    DTri<R>& T = tris[A.tri_index[t]];
    for(int c = 0; c < 3; ++c) {
      T.v0[c] = (R)vf[0][c];
      T.v1[c] = (R)vf[1][c];
      T.v2[c] = (R)vf[2][c];
    }
    const int si = A.tri_samp[t];
    if(si < 0) continue;
    /* The sampled triangle as a snapshot builds it: FP64 normal from the
     * FP32 vertices, e2 x e1, normalised and rounded through FP32 */
    double e1[3], e2[3], n[3];
    for(int c = 0; c < 3; ++c) {
      e1[c] = ds((double)vf[1][c], (double)vf[0][c]);
      e2[c] = ds((double)vf[2][c], (double)vf[0][c]);
    }
    n[0] = ds(dm(e2[1], e1[2]), dm(e2[2], e1[1]));
    n[1] = ds(dm(e2[2], e1[0]), dm(e2[0], e1[2]));
    n[2] = ds(dm(e2[0], e1[1]), dm(e2[1], e1[0]));
    const double len = sqrt(da(da(dm(n[0], n[0]), dm(n[1], n[1])), dm(n[2], n[2])));
    DSampTri<R>* samp = (DSampTri<R>*)A.samp + (size_t)item * A.samp_stride;
    DSampTri<R>& st = samp[si];
    for(int c = 0; c < 3; ++c) {
      st.v0[c] = T.v0[c];
      st.e1[c] = T.v1[c] - T.v0[c];
      st.e2[c] = T.v2[c] - T.v0[c];
      st.n[c] = (R)(float)(len > 0 ? __ddiv_rn(n[c], len) : 0.0);
    }
  }
}

/* Box of the triangles of a BVH leaf slot; quadric patches (never tracked)
 * keep the slot's box from the snapshot */
template<class R>
__device__ void leaf_box(const DNode<R>& node, int k, const DTri<R>* tris,
                         const uint32_t* primrefs, R lo[3], R hi[3])
{
  const int cnt = node.count[k];
  bool quad = false;
  for(int c = 0; c < 3; ++c) { lo[c] = rmax<R>(); hi[c] = -rmax<R>(); }
  for(int i = 0; i < cnt; ++i) {
    const uint32_t ref = cnt == 1 ? (uint32_t)node.child[k] : primrefs[node.child[k] + i];
    if(primref_kind(ref) != PRIM_TRIANGLE) { quad = true; continue; }
    const DTri<R>& T = tris[primref_index(ref)];
    for(int c = 0; c < 3; ++c) {
      lo[c] = fmin(lo[c], fmin(T.v0[c], fmin(T.v1[c], T.v2[c])));
      hi[c] = fmax(hi[c], fmax(T.v0[c], fmax(T.v1[c], T.v2[c])));
    }
  }
  if(quad)
    for(int c = 0; c < 3; ++c) {
      lo[c] = fmin(lo[c], node.lo[k][c]);
      hi[c] = fmax(hi[c], node.hi[k][c]);
    }
}

/* One block per item: the BVH's child boxes level by level, deepest first,
 * so that a node's children are final before their parent reads them */
template<class R>
__global__ void __launch_bounds__(256) track_refit_kernel(const TrackArgs A)
{
  const int item = blockIdx.x;
  DNode<R>* nodes = (DNode<R>*)A.nodes + (size_t)item * A.node_stride;
  const DTri<R>* tris = (const DTri<R>*)A.tris + (size_t)item * A.tri_stride;
  for(int L = 0; L < A.nlevels; ++L) {
    for(int i = A.level_first[L] + threadIdx.x; i < A.level_first[L + 1]; i += blockDim.x) {
      DNode<R>& node = nodes[A.level_nodes[i]];
      for(int k = 0; k < 2; ++k) {
        const int cnt = node.count[k];
        if(cnt < 0) continue;
        R lo[3], hi[3];
        if(cnt > 0) {
          leaf_box(node, k, tris, A.primrefs, lo, hi);
        } else {
          const DNode<R>& ch = nodes[node.child[k]];
          for(int c = 0; c < 3; ++c) { lo[c] = rmax<R>(); hi[c] = -rmax<R>(); }
          for(int j = 0; j < 2; ++j) {
            if(ch.count[j] < 0) continue;
            for(int c = 0; c < 3; ++c) {
              lo[c] = fmin(lo[c], ch.lo[j][c]);
              hi[c] = fmax(hi[c], ch.hi[j][c]);
            }
          }
        }
        for(int c = 0; c < 3; ++c) {
          node.lo[k][c] = lo[c];
          node.hi[k][c] = hi[c];
        }
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) gather_globals_kernel
  (const DTallies* tallies, int nitems, double* out)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int item = k / 13, q = k % 13;
  if(item >= nitems) return;
  const DTallies& T = tallies[item];
  out[k] = q < 2 * NGLOBAL ? T.global[q] : (double)T.counters[0];
}

int launch_gather_globals(const DTallies* tallies, int nitems, double* out, void* stream)
{
  const int total = 13 * nitems;
  if(total > 0)
    gather_globals_kernel<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>
      (tallies, nitems, out);
  return (int)cudaGetLastError();
}

template<class R>
static int launch_track(const TrackArgs& A, void* stream)
{
  const cudaStream_t s = (cudaStream_t)stream;
  const size_t total = (size_t)A.nitems * (size_t)A.ntracked;
  if(total) {
    const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, 148 * 16);
    track_triangles_kernel<R><<<blocks, 256, 0, s>>>(A);
  }
  if(A.nitems) track_refit_kernel<R><<<(unsigned)A.nitems, 256, 0, s>>>(A);
  return (int)cudaGetLastError();
}

int launch_track_f32(const TrackArgs& A, void* stream) { return launch_track<float>(A, stream); }
int launch_track_f64(const TrackArgs& A, void* stream) { return launch_track<double>(A, stream); }

} /* namespace ssolb */
