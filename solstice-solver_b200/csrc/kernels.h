/*
 * kernels.h - host-callable launchers of the realisation kernel
 * (kernels_*.cu). Plain C++ types only, so that host code compiled by the
 * system C++ compiler can call them.
 */
#ifndef SSOL_B200_KERNELS_H
#define SSOL_B200_KERNELS_H

#include "device_scene.h"

#include <stddef.h>

namespace ssolb {

struct LaunchConfig {
  int block_size; /* threads per block, <= 256; 0 => 256 */
  int grid_blocks; /* 0 => SMs x resident blocks x waves */
  int waves; /* persistent grid multiplier, 0 => 1 */
  unsigned long long max_segments; /* per path segment budget */
  int min_blocks; /* register budget: 1 (255 regs), 2 (128) or 3 (85) */
  int rcv_doubles = 0; /* batched launches: largest item receiver-sum array
                        * (nrcv x 10 x 2); 0 => receiver sums go straight
                        * to device memory */
  bool coherent = true; /* plain launches of at least 2^24 realisations run
                         * in the order of their sampled primitives */
  /* Plain launches: stop handing out realisations once this many paths
   * have failed (~0: never), or once the host sets the tallies' abort word
   * (when `abortable`) */
  unsigned long long max_failed = ~0ull;
  bool abortable = false;
  /* FEAT_* bits the scene needs; the launch picks the smallest variant
   * that covers them */
  int features = FEAT_ALL;
  /* Count rays, node visits and primitive tests into the launch's stats
   * (FP32 plain launches without tracking and FP32 batched launches can
   * leave them out; the others always count) */
  bool count_work = true;
};

/* Enqueue the realisations [first, first + count) of the stream keyed by
 * `seed` on `stream` (a cudaStream_t); tallies accumulate into T; `track`
 * (may be NULL) records the paths of the first track->npaths of them.
 * Returns a cudaError_t value. */
int launch_realisations_f32
  (const DScene<float>& S, const DTallies& T, uint64_t seed, uint64_t first,
   uint64_t count, const LaunchConfig& cfg, void* stream,
   const DTrack* track = nullptr);
int launch_realisations_f64
  (const DScene<double>& S, const DTallies& T, uint64_t seed, uint64_t first,
   uint64_t count, const LaunchConfig& cfg, void* stream,
   const DTrack* track = nullptr);
/* The FP32 variants without work counters (kernels_plain_nc.cu), which
 * launch_realisations_f32 calls when cfg.count_work is false */
int launch_realisations_nocount_f32
  (const DScene<float>& S, const DTallies& T, uint64_t seed, uint64_t first,
   uint64_t count, const LaunchConfig& cfg, void* stream);

/* Batched launch: device arrays of per-item scenes and tallies, the item
 * budgets as an inclusive prefix (nitems + 1 entries; the last one is the
 * launch total) and the first realisation index of each item */
/* Realisations per warp segment of the coherent order */
constexpr uint32_t SORT_SEGMENT = 256;

/* Coherent order of a batched launch (sorted_off null: id order). Per item,
 * from prefix[item] on, sorted_off / sorted_draw hold its realisations'
 * offsets in the item and primary draws (4 words each) in the order of their
 * sampled primitive; seg_mul[item] is the stride of the order in which its
 * warp segments are handed out (coprime with its number of full segments);
 * bin_base[item] is its first histogram bin, nbins the bins of all items.
 * hist and bin_off are the presort's histogram and ranges (nbins each). */
struct BatchOrder {
  uint32_t* sorted_off = nullptr;
  uint32_t* sorted_draw = nullptr;
  uint32_t* hist = nullptr;
  uint32_t* bin_off = nullptr;
  const uint32_t* bin_base = nullptr;
  const uint32_t* seg_mul = nullptr;
  uint32_t nbins = 0;
};

template<class R> struct BatchLaunch {
  const DScene<R>* scenes;
  const DTallies* tallies;
  const unsigned long long* prefix;
  const unsigned long long* firsts;
  int nitems;
  uint64_t seed;
  unsigned long long* next_items; /* per-item work counters (scratch) */
  DStats* stats;
  BatchOrder order;
};

int launch_batch_f32(const BatchLaunch<float>& b, const LaunchConfig& cfg,
                     void* stream);
/* The FP32 batched variants without work counters (kernels_batch_nc.cu),
 * which launch_batch_f32 calls when cfg.count_work is false */
int launch_batch_nocount_f32(const BatchLaunch<float>& b, const LaunchConfig& cfg,
                             void* stream);

/* Largest item count of the no-allocation batched launch: its scratch is a
 * static device array sized for this many items */
constexpr int NOALLOC_MAX_ITEMS = 4096;

/* Batched launch whose scratch (budget prefix, per-item first ids, work
 * counter, launch counters) lives in a static device array instead of
 * caller or library allocations; h_prefix (nitems + 1) and h_firsts
 * (nitems) are host arrays copied into it */
int launch_batch_noalloc_f32
  (const DScene<float>* scenes, const DTallies* tallies, int nitems,
   uint64_t seed, const unsigned long long* h_prefix,
   const unsigned long long* h_firsts, const LaunchConfig& cfg, void* stream);
int launch_batch_noalloc_f64
  (const DScene<double>* scenes, const DTallies* tallies, int nitems,
   uint64_t seed, const unsigned long long* h_prefix,
   const unsigned long long* h_firsts, const LaunchConfig& cfg, void* stream);
int launch_batch_f64(const BatchLaunch<double>& b, const LaunchConfig& cfg,
                     void* stream);

/* Per item of a batch, its 12 global sums and its failure count (as a
 * double), 13 doubles per item into `out` (device) */
int launch_gather_globals(const DTallies* tallies, int nitems, double* out, void* stream);

/* Tracking batches (one snapshot, one item per sun position): per item,
 * each tracked heliostat turns toward the item's sun, its triangles and
 * sampled triangles are rewritten, and the BVH is refitted. Device arrays:
 * helio (per heliostat: position, aim point), to_sun (per item: unit vector
 * toward the sun), per tracked triangle its heliostat, its index in tris, its
 * index in samp (-1 if not sampled) and its 9 local vertex coordinates; the
 * items' tris, samp and nodes arrays (item i at base + i x stride elements,
 * already holding copies of the snapshot's); the BVH's node indices grouped
 * by depth, deepest first (level_first: nlevels + 1 offsets). */
struct TrackArgs {
  int nitems, ntracked, nlevels;
  const double* helio;
  const double* to_sun;
  const int32_t* tri_helio;
  const int32_t* tri_index;
  const int32_t* tri_samp;
  const double* local;
  void* tris; size_t tri_stride;
  void* samp; size_t samp_stride;
  void* nodes; size_t node_stride;
  const uint32_t* primrefs;
  const int32_t* level_nodes;
  const int32_t* level_first;
};
int launch_track_f32(const TrackArgs& A, void* stream);
int launch_track_f64(const TrackArgs& A, void* stream);

/* Device-built linear BVH (lbvh.cu) over n >= 2 primitive boxes (device
 * array of 6 R per primitive: lo xyz, hi xyz, already rounded outward) and
 * their references; writes the n - 1 nodes of DNode<R> (root 0, one
 * primitive per leaf) and the tree depth (device int). The scratch pointers
 * come from lbvh_bind_scratch over lbvh_scratch_bytes(n) bytes. */
struct LbvhArgs {
  int n;
  const void* box;
  const uint32_t* ref;
  void* nodes;
  void* cbounds;
  int32_t* depth;
  uint32_t* keys;
  uint32_t* vals;
  int32_t* parent;
  uint32_t* flags;
  int32_t* height;
  float* cost;
  int32_t* ninner;
  int32_t* newidx;
  int32_t* level_nodes;
  int32_t* level_first; /* MAX_LEVELS + 1 offsets, then the largest height */
  void* tmp_nodes;
  int optimize; /* treelet restructuring of every node's subtree */
};
size_t lbvh_scratch_bytes(int n);
void lbvh_bind_scratch(LbvhArgs& A, void* scratch);
int launch_lbvh_f32(const LbvhArgs& A, void* stream);
int launch_lbvh_f64(const LbvhArgs& A, void* stream);

/* Arguments of the adjoint passes (adjoint.cuh). Device pointers: inst_slot
 * (parameter slot per instance, -1 if none), axes (per slot: centre, e_x,
 * e_y), map (nx * ny cell sums of pass 0, read by pass 1), sums (sum w,
 * sum w^2, hits), grad_abs and grad_spill (2 per slot), counters (rays,
 * nodes, triangles, quadrics). */
struct AdjointArgs {
  const int* inst_slot;
  const double* axes;
  int rcv_instance;
  int rcv_side; /* the receiver's receiving side: 1 front (+z), 2 back */
  int rcv_mtl; /* material of that side (device index) */
  double w2l[12]; /* the receiver's world -> local transform, rows x, y, z */
  double upper[2]; /* far corner of the map (its near corner is `lower`) */
  double edge; /* width of the ramp that smooths the receiver's boundary */
  double lower[2], inv_cell[2];
  int nx, ny;
  double* map;
  double* sums;
  double* grad_abs;
  double* grad_spill;
  unsigned long long* counters;
  double target; /* uniform target flux density */
  double inv_n; /* 1 / realisations */
  double map_scale; /* 1 / (realisations x cell area) */
};

/* One adjoint pass (0: objective and map, 1: gradients) */
int launch_adjoint_f32
  (const DScene<float>& S, const AdjointArgs& A, uint64_t seed, uint64_t first,
   uint64_t count, int pass, void* stream);
int launch_adjoint_f64
  (const DScene<double>& S, const AdjointArgs& A, uint64_t seed, uint64_t first,
   uint64_t count, int pass, void* stream);

/* Arguments of the renderers (draw.cuh). The camera basis is FP32 as in
 * src/ssol_camera.h; pix_w and pix_h are 1 / width and 1 / height in FP32;
 * offsets (draft: 2 per sample) and pixels (width x height x 3) are device
 * arrays; counters (device, 6): rays, BVH nodes, triangle tests, quadric
 * tests, shaded bounces, camera samples. */
struct DrawArgs {
  float cam_x[3], cam_y[3], cam_z[3], cam_pos[3];
  float pix_w, pix_h;
  int width, height, spp;
  const float* offsets;
  float up[3];
  uint64_t seed;
  double* pixels;
  unsigned long long* counters;
};

int launch_draft_f32(const DScene<float>& S, const DrawArgs& A, void* stream);
int launch_draft_f64(const DScene<double>& S, const DrawArgs& A, void* stream);
int launch_pt_f32(const DScene<float>& S, const DrawArgs& A, void* stream);
int launch_pt_f64(const DScene<double>& S, const DrawArgs& A, void* stream);

} /* namespace ssolb */

#endif /* SSOL_B200_KERNELS_H */
