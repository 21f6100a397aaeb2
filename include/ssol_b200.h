/*
 * ssol_b200.h - B200 extensions of the ssol_* C API.
 *
 * None of these entry points has a counterpart in the reference; they expose
 * what a GPU solver adds around `ssol_solve` (src/ssol.h:1216-1223):
 *  - solve options: arithmetic precision of geometry/sampling/BSDFs (FP32 or
 *    all-FP64; tallies are FP64 in both), launch shape, BVH leaf size, and
 *    whether the BVH is built on the host or the device;
 *  - plans: a scene snapshot resident in device memory that can be launched
 *    many times on a caller's CUDA stream and read back once, which is how
 *    `ssol_solve` itself is built (create, reset, launch, finish);
 *  - per-solve device timing and work counters for roofline reporting.
 * Plain C: CUDA streams travel as `void*` (a cudaStream_t).
 */
#ifndef SSOL_B200_H
#define SSOL_B200_H

#include "ssol.h"
#include "ssp.h"

#ifdef __cplusplus
extern "C" {
#endif

enum ssol_b200_precision {
  SSOL_B200_FP32 = 0, /* FP32 geometry, sampling and BSDFs; FP64 tallies */
  SSOL_B200_FP64 = 1 /* everything in FP64 on identical random numbers */
};

/* Who builds the ray-tracing BVH of a plan's snapshot (the reference builds
 * its Star-3D view on every solve, src/ssol_scene.c:347-433):
 *  - SSOL_B200_BVH_SAH: binned-SAH tree on the host threads, uploaded with
 *    the snapshot; leaves of bvh_leaf_size primitives; the fastest to trace;
 *  - SSOL_B200_BVH_LBVH: linear BVH built on the device from the uploaded
 *    primitive boxes (Morton codes, radix sort, Karras' hierarchy, bottom-up
 *    boxes, treelet restructuring for a lower SAH cost, depth-first node
 *    order), one primitive per leaf (bvh_leaf_size is ignored); the fastest
 *    to build. A tree deeper than the traversal stack allows (more than 30
 *    levels) is rebuilt on the host with the SAH builder, with a warning;
 *  - SSOL_B200_BVH_AUTO (the default): ssol_solve and ssol_solve_ex use the
 *    device builder for solves of at most SSOL_B200_BVH_AUTO_MAX_PATHS
 *    realisations, where building is a large part of the call. Larger solves
 *    start on the device's tree and, after their first 6e6 realisations,
 *    trace on the SAH tree that the host threads built meanwhile. Plans,
 *    which do not know how many realisations they will trace, use the SAH
 *    builder.
 * Both trees find the same closest hits; only the time to build them and to
 * traverse them differs. Batches and the renderers always use the SAH
 * builder. */
enum ssol_b200_bvh_builder {
  SSOL_B200_BVH_AUTO = 0,
  SSOL_B200_BVH_SAH = 1,
  SSOL_B200_BVH_LBVH = 2
};
#define SSOL_B200_BVH_AUTO_MAX_PATHS (1ull << 24)

struct ssol_b200_options {
  enum ssol_b200_precision precision;
  int block_size; /* threads per block, <= 256; 0 => 256 */
  int grid_blocks; /* 0 => one persistent wave sized from occupancy */
  int waves; /* persistent grid multiplier when grid_blocks == 0 */
  int bvh_leaf_size; /* primitives per BVH leaf; 0 => 1 */
  unsigned long long max_segments; /* path segment budget; 0 => 1e6 */
  int min_blocks_per_sm; /* register budget of the kernel variant: 1, 2, 3;
                          * 0 => 3 in FP32, 2 in FP64 */
  enum ssol_b200_bvh_builder bvh_builder; /* plans and ssol_solve_ex */
  /* Nonzero: count rays, BVH node visits and primitive tests into the stats
   * (ssol_b200_stats rays .. quadric_tests). 0 (the default): leave them out
   * of the FP32 plain and batched kernels, which are about 1-2 % faster
   * without them; they then read 0. The FP64 build, path tracking, the
   * no-allocation batched launch, the adjoint and the renderers always
   * count. */
  int count_work;
};
#define SSOL_B200_OPTIONS_DEFAULT__ { SSOL_B200_FP32, 256, 0, 1, 0, 0, 0, SSOL_B200_BVH_AUTO, 0 }
static const struct ssol_b200_options SSOL_B200_OPTIONS_DEFAULT =
  SSOL_B200_OPTIONS_DEFAULT__;

/* Device work of the last solve (or of a plan's launches since its reset) */
struct ssol_b200_stats {
  double kernel_ms; /* CUDA-event time of the realisation launches */
  /* rays cast (shadow + scattered), BVH nodes fetched, triangle and quadric
   * tests: counted when the options ask for it (count_work) */
  unsigned long long rays;
  unsigned long long node_visits;
  unsigned long long triangle_tests;
  unsigned long long quadric_tests;
  unsigned long long bounces; /* surface interactions that were shaded */
  unsigned long long paths;
  unsigned long long killed; /* paths ended by the Russian roulette */
  unsigned long long scene_bytes; /* host -> device bytes of the snapshot */
  unsigned long long tally_bytes; /* device -> host bytes of the tallies */
  unsigned long long bvh_nodes; /* BVH nodes of the plan's snapshot */
  unsigned long long bvh_depth; /* levels of internal nodes */
  unsigned long long bvh_device; /* 1 if the BVH was built on the device */
};

/* ssol_solve with explicit options (NULL => defaults) */
SSOL_API res_T ssol_solve_ex
  (struct ssol_scene* scn,
   const struct ssp_rng* rng,
   const size_t realisations_count,
   const size_t max_failed_count,
   const struct ssol_path_tracker* tracker,
   const struct ssol_b200_options* options,
   struct ssol_estimator** estimator);

SSOL_API res_T ssol_estimator_get_b200_stats
  (const struct ssol_estimator* estimator, struct ssol_b200_stats* stats);

/* Plans */
struct ssol_b200_plan;

/* Snapshot `scn` (flatten, build the BVH, upload); device memory stays
 * allocated until the last reference is released */
SSOL_API res_T ssol_b200_plan_create
  (struct ssol_scene* scn, const struct ssol_b200_options* options,
   struct ssol_b200_plan** plan);
SSOL_API res_T ssol_b200_plan_ref_get(struct ssol_b200_plan* plan);
SSOL_API res_T ssol_b200_plan_ref_put(struct ssol_b200_plan* plan);
/* Zero the device tallies, asynchronously on `stream` (NULL => the plan's
 * own stream), and clear an abort request (call it once the plan's earlier
 * launches have completed) */
SSOL_API res_T ssol_b200_plan_reset
  (struct ssol_b200_plan* plan, void* stream);
/* Host-side stop of a long solve, from any thread: the plan's running and
 * queued launches take no new realisations (paths in flight finish). The
 * call copies a flag into the plan's device tallies on a stream of its own
 * (a copy-engine transfer, which runs beside the plan's kernels) and
 * returns once it has landed; the kernels' work fetch polls it, so it takes
 * effect within microseconds. It stays until ssol_b200_plan_reset.
 * ssol_b200_plan_finish then builds the estimator of the realisations that
 * ran (realisation count below the one asked for) and returns RES_BAD_OP, as
 * the reference's solve returns the error that stopped its loop with a valid
 * estimator (src/ssol_solver.c:1229, 1339). */
SSOL_API res_T ssol_b200_plan_abort(struct ssol_b200_plan* plan);
/* Enqueue realisations [first, first + count) of the streams keyed by `rng`;
 * tallies accumulate. Asynchronous. */
SSOL_API res_T ssol_b200_plan_launch
  (struct ssol_b200_plan* plan, const struct ssp_rng* rng,
   const uint64_t first, const uint64_t count, void* stream);
/* Wait for `stream`, read the tallies back and build an estimator for
 * `realisations_count` realisations; same failure rule as ssol_solve */
SSOL_API res_T ssol_b200_plan_finish
  (struct ssol_b200_plan* plan, const struct ssp_rng* rng,
   const uint64_t realisations_count, const size_t max_failed_count,
   void* stream, struct ssol_estimator** estimator);
SSOL_API res_T ssol_b200_plan_get_stats
  (const struct ssol_b200_plan* plan, struct ssol_b200_stats* stats);

/* Tallies across GPUs. The reference merges its per-thread sums inside
 * ssol_solve (src/ssol_solver.c:1254-1333); several GPUs tracing disjoint
 * realisations of one scene merge theirs the same way, by adding them.
 * ssol_b200_plan_get_tallies gives device pointers to the plan's FP64 sums
 * (`nsums` doubles: sum w and sum w^2 of every estimate) and its 64-bit
 * counts (`ncounts`: samples per sampled instance, failures, launch
 * counters). Adding the vectors of the plans of one scene element-wise, for
 * instance by an in-place all-reduce over their GPUs, leaves in each the
 * tallies of all their realisations; ssol_b200_plan_finish with the total
 * realisation count then builds the merged estimator. */
SSOL_API res_T ssol_b200_plan_get_tallies
  (struct ssol_b200_plan* plan, double** sums, size_t* nsums, uint64_t** counts,
   size_t* ncounts);
/* The same vectors on the host, where no GPU is needed: their sizes for a
 * scene, and the estimator of `realisations_count` realisations of `scn`
 * built from (merged) host copies, with ssol_b200_plan_finish's rules
 * (failure limit, RNG end state). RES_BAD_ARG if the sizes do not match the
 * scene. */
SSOL_API res_T ssol_b200_tallies_size
  (struct ssol_scene* scn, size_t* nsums, size_t* ncounts);
SSOL_API res_T ssol_b200_estimator_create_from_tallies
  (struct ssol_scene* scn, const struct ssp_rng* rng, const uint64_t realisations_count,
   const size_t max_failed_count, const double* sums, const size_t nsums,
   const uint64_t* counts, const size_t ncounts, struct ssol_estimator** estimator);

/* Autotuner: times `trial_paths` realisations of `scn` for every launch
 * shape in {block 128, 256} x {register budget 1, 2, 3 blocks per SM} x
 * {1, 2 persistent waves} on each BVH leaf size in {1, 2, 4} (one snapshot
 * per leaf size), after one untimed launch of each, and writes the fastest
 * into `options` (its precision and max_segments are kept). `best_ms`, if
 * not NULL, receives that launch's CUDA-event time. Synchronous; tallies of
 * the trials are discarded. */
SSOL_API res_T ssol_b200_autotune
  (struct ssol_scene* scn, const struct ssp_rng* rng, const uint64_t trial_paths,
   struct ssol_b200_options* options, double* best_ms);

/* Adjoint (no counterpart in the reference): gradients of a receiver flux
 * objective with respect to the aim of heliostats.
 *
 * Only first-bounce paths count: sampled on a mirror, not shadowed, reflected
 * once and reaching the `receiver` first on a receiving side with a mirror or
 * matte material. Their weight w there includes the atmosphere and the
 * receiver's absorptivity. Objectives:
 *   absorbed = (1/N) sum w                               (W)
 *   spillage = sum_c (M_c - target)^2                    (W^2/m^4)
 * M_c is the flux density of cell c of an nx x ny grid over
 * [lower, upper] in the receiver's local x, y, each hit splatted with
 * bilinear weights on the cell centres. Parameters: for each listed
 * heliostat, rotations theta_x, theta_y about its instance's local x and y
 * axes through its translation, at theta = 0. Gradients follow the paths
 * (reparameterised sampling, replayed from the Philox keys of `rng`).
 * The receiver's boundary, taken as the map's rectangle (so the map should
 * cover the receiver exactly), is differentiated through a smoothed
 * receiver: a linear ramp of width `edge_band` across each side, so that
 * the reflected rays that cross the receiver's plane within half a band of
 * its boundary, unblocked, carry the derivative of the flux entering or
 * leaving it (bias O(edge_band); 0 selects half a map cell). The changes of
 * shadowing and blocking are not differentiated. */
struct ssol_b200_adjoint_map {
  struct ssol_instance* receiver; /* a mesh instance */
  double lower[2], upper[2]; /* receiver-local x, y extent of the grid */
  unsigned nx, ny;
  double target; /* uniform target flux density, W/m^2 */
  double edge_band; /* width of the boundary ramp, m; 0 => half a cell */
};

struct ssol_b200_adjoint_result {
  double absorbed, absorbed_se; /* first-bounce absorbed power and its SE */
  double spillage;
  unsigned long long hits; /* first-bounce paths that reached the receiver */
  double kernel_ms; /* both passes */
  /* device work of both passes */
  unsigned long long rays, node_visits, triangle_tests, quadric_tests;
};

/* d_absorbed and d_spillage receive 2 x nheliostats values (theta_x, theta_y
 * of each listed heliostat, in order) and may be NULL when nheliostats is 0;
 * flux_map (optional) receives the nx x ny flux densities, row by row. */
SSOL_API res_T ssol_solve_adjoint
  (struct ssol_scene* scn, const struct ssp_rng* rng, const size_t realisations_count,
   struct ssol_instance* const* heliostats, const size_t nheliostats,
   const struct ssol_b200_adjoint_map* map, const struct ssol_b200_options* options,
   struct ssol_b200_adjoint_result* result, double* d_absorbed, double* d_spillage,
   double* flux_map);

/* Batches: several scenes (typically one per sun position, each with its own
 * re-aimed field and sun) traced by one persistent kernel launch replayed
 * from a captured CUDA graph, each item with its own budget and tallies */
struct ssol_b200_batch;

SSOL_API res_T ssol_b200_batch_create
  (struct ssol_scene* const* scenes, const size_t nscenes,
   const struct ssol_b200_options* options, struct ssol_b200_batch** batch);
/* A tracking field over several sun positions, as one batch built on the
 * device: item i is `scn` with its sun's direction and DNI set to suns[i]
 * (its sunshape and spectrum kept) and every listed heliostat turned to
 * track that sun. A heliostat instance keeps its translation p and gets the
 * rotation whose columns are x, y, n: n the unit bisector of the direction
 * to the sun (-direction, normalised as ssol_sun_set_direction does) and the
 * unit direction from p to its aim point (aim_points, 3 per heliostat); x
 * the unit vector of up x n, up = +z (+x when n is vertical); y = n x x.
 * Its object's mirror normal is thus its local +z. The scene is snapshot
 * once on the host; per item the device rewrites the heliostats' triangles
 * and sampled triangles, in the arithmetic and rounding of a host snapshot
 * of the re-aimed scene, and refits the BVH built for `scn` (the tree keeps
 * its topology; every child box is recomputed). Heliostats must be mesh
 * instances of `scn`, and the scene must have no vertex normals and no
 * shaders baked per vertex (RES_BAD_ARG otherwise). The other batch calls
 * apply; finish returns one estimator per sun. */
struct ssol_b200_sun_position {
  double direction[3]; /* from the sun toward the scene */
  double dni; /* W/m^2, > 0 */
};
SSOL_API res_T ssol_b200_batch_create_tracking
  (struct ssol_scene* scn, struct ssol_instance* const* heliostats,
   const size_t nheliostats, const double* aim_points,
   const struct ssol_b200_sun_position* suns, const size_t nsuns,
   const struct ssol_b200_options* options, struct ssol_b200_batch** batch);
SSOL_API res_T ssol_b200_batch_ref_get(struct ssol_b200_batch* batch);
SSOL_API res_T ssol_b200_batch_ref_put(struct ssol_b200_batch* batch);
/* Zero every item's tallies and realisation counts */
SSOL_API res_T ssol_b200_batch_reset(struct ssol_b200_batch* batch, void* stream);
/* One launch: budgets[i] more realisations of item i, continuing its own
 * stream (realisation ids position + k of `rng`, k counted per item since
 * the last reset). Returns when the launch has completed. A launch of at
 * least 2^22 and at most 2^29 realisations in all runs them in the order of
 * their sampled primitives (the same paths, only the order of the FP64 sums
 * changes); for that the batch keeps a device scratch of 20 bytes per
 * realisation of its largest such launch (plus a quarter), released with
 * the batch. */
SSOL_API res_T ssol_b200_batch_launch
  (struct ssol_b200_batch* batch, const struct ssp_rng* rng,
   const uint64_t* budgets, void* stream);
/* No counterpart in the reference. The same launch as
 * ssol_b200_batch_launch for callers that must not have device memory
 * allocated on their behalf while they launch: code that owns every device
 * allocation through its own pool, or a real-time loop whose rules forbid
 * allocating (an allocation can block, or fail, at any time). The batch
 * (scenes in, tallies out) is created beforehand; this call allocates
 * nothing: no cudaMalloc/cudaFree and no CUDA graph. The kernel's scratch
 * (budget prefix sums, per-item first realisation ids, per-item work
 * counters and launch counters) lives in a static device array sized for
 * at most 4096 items (96 KiB), which every GPU that loads the library keeps
 * until the process exits; batches with more items get RES_BAD_ARG. The
 * first call on a device looks up that array's device address, with that
 * device current, and keeps
 * it for later calls (make that first call before any stream capture; after
 * a cudaDeviceReset the kept address is stale and the process must not call
 * this entry point again on that device). All calls share the array, so
 * calls that overlap on the GPU race; each call sets it up anew. The call
 * copies the budgets from host memory and waits for `stream` before it
 * returns, so it is made outside any capture of `stream` (RES_BAD_ARG
 * otherwise). Work counters of these launches are not reported in
 * ssol_b200_stats. */
SSOL_API res_T ssol_b200_batch_launch_noalloc
  (struct ssol_b200_batch* batch, const struct ssp_rng* rng,
   const uint64_t* budgets, void* stream);
/* The global estimates of every item (nscenes entries), as
 * ssol_estimator_get_mc_global gives them on the item's estimator, without
 * building estimators: a device gather and a read of 13 doubles per item.
 * For pilots that size each item's next budget. */
SSOL_API res_T ssol_b200_batch_get_mc_global
  (struct ssol_b200_batch* batch, void* stream, struct ssol_mc_global* globals);
/* One estimator per item (nscenes entries), as ssol_solve would return for
 * the realisations the item received */
SSOL_API res_T ssol_b200_batch_finish
  (struct ssol_b200_batch* batch, const struct ssp_rng* rng,
   const size_t max_failed_count, void* stream,
   struct ssol_estimator** estimators);

/* Shaders (ssol_shader_getter_T) for materials whose properties are the
 * same everywhere. No counterpart in the reference, whose callers write such
 * callbacks themselves. ssol_b200_shader_param0 / _param1 return the first /
 * second double of the material's parameter buffer (ssol_param_buffer_get,
 * 0 without a buffer); ssol_b200_shader_Ns returns the fragment's shading
 * normal. Being plain C, they cost nothing when the scene is snapshot from
 * several host threads, unlike callbacks into an interpreter that must take
 * its lock on every call. */
SSOL_API void ssol_b200_shader_param0
  (struct ssol_device* dev, struct ssol_param_buffer* buf, const double wavelength,
   const struct ssol_surface_fragment* frag, double* val);
SSOL_API void ssol_b200_shader_param1
  (struct ssol_device* dev, struct ssol_param_buffer* buf, const double wavelength,
   const struct ssol_surface_fragment* frag, double* val);
SSOL_API void ssol_b200_shader_Ns
  (struct ssol_device* dev, struct ssol_param_buffer* buf, const double wavelength,
   const struct ssol_surface_fragment* frag, double* val);

/* Renderers into device memory. No counterpart in the reference: its
 * ssol_draw_draft / ssol_draw_pt (src/ssol.h:1225-1244) hand tiles to a host
 * writer, which the ssol.h versions here still do. These leave the image in
 * a caller's device buffer (a headless device image), width x height
 * pixels of 3 doubles, row after row (row pitch width x 24 bytes), and
 * return when it is written. `options` (NULL => defaults) selects the
 * arithmetic precision and the BVH leaf size; `stats` (may be NULL)
 * receives the kernel time and work counters (bounces = shaded surface
 * interactions, paths = camera samples). ssol_b200_draw_pt_device keys its
 * random streams by `seed`; ssol_draw_pt uses seed 0. */
SSOL_API res_T ssol_b200_draw_draft_device
  (struct ssol_scene* scn, struct ssol_camera* cam, const size_t width,
   const size_t height, const size_t spp,
   const struct ssol_b200_options* options, double* device_pixels,
   struct ssol_b200_stats* stats);
SSOL_API res_T ssol_b200_draw_pt_device
  (struct ssol_scene* scn, struct ssol_camera* cam, const size_t width,
   const size_t height, const size_t spp, const double up[3],
   const uint64_t seed, const struct ssol_b200_options* options,
   double* device_pixels, struct ssol_b200_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* SSOL_B200_H */
