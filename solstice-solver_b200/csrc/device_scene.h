/*
 * device_scene.h - flat, device-resident scene layout of one `ssol_solve`.
 *
 * Compiled by both the host C++ compiler and nvcc. Everything is plain data:
 * arrays of PODs addressed by 32-bit indices, built once per solve by
 * scene_flatten.cpp and uploaded to HBM in one contiguous allocation.
 *
 * The layout replaces the reference's Star-3D scene views and hash maps
 * (src/ssol_scene.c:347-433, src/ssol_solver.c:254-258, 374-378):
 *  - every instance x shaded shape x triangle becomes one world-space
 *    triangle; every instance x punched shaded shape becomes one analytic
 *    quadric patch with its world->local transform precomputed;
 *  - both kinds share one binary BVH whose nodes hold their two children's
 *    boxes (one 64-byte node per visit in the FP32 build);
 *  - the sampled proxy triangles form an alias table (O(1) area-weighted
 *    primitive choice, replacing Star-3D's scene_view_sample);
 *  - receiver tallies are flat FP64 arrays addressed by precomputed slots.
 */
#ifndef SSOL_B200_DEVICE_SCENE_H
#define SSOL_B200_DEVICE_SCENE_H

#include <stdint.h>

#ifdef __CUDACC__
  #define SSOL_HD __host__ __device__ __forceinline__
#else
  #define SSOL_HD inline
#endif

namespace ssolb {

/* Primitive kinds referenced from BVH leaves */
enum : uint32_t {
  PRIM_TRIANGLE = 0u,
  PRIM_QUADRIC = 1u
};
/* prim reference = kind in bit 31, index in bits 0..30 */
SSOL_HD uint32_t primref_make(uint32_t kind, uint32_t idx)
{ return (kind << 31) | idx; }
SSOL_HD uint32_t primref_kind(uint32_t ref) { return ref >> 31; }
SSOL_HD uint32_t primref_index(uint32_t ref) { return ref & 0x7fffffffu; }

/* Material kinds, same order as enum ssol_material_type */
enum : int32_t {
  MTL_DIELECTRIC = 0,
  MTL_MATTE = 1,
  MTL_MIRROR = 2,
  MTL_THIN_DIELECTRIC = 3,
  MTL_VIRTUAL = 4
};

enum : int32_t { DISTRIB_BECKMANN = 0, DISTRIB_PILLBOX = 1 };

/* Sun shapes */
enum : int32_t {
  SUN_DIRAC = 0,
  SUN_PILLBOX = 1,
  SUN_GAUSSIAN = 2,
  SUN_BUIE = 3
};

/* Quadric kinds, same order as enum ssol_quadric_type */
enum : int32_t {
  QUAD_PLANE = 0,
  QUAD_PARABOL = 1,
  QUAD_PARABOL2F = 2,
  QUAD_HYPERBOL = 3,
  QUAD_PCYLINDER = 4,
  QUAD_HEMISPHERE = 5
};

/* Number of tallied quantities per receiver side, per sampled x receiver and
 * per primitive (the MC_RECEIVER_DATA list, src/ssol_estimator_c.h:44-54) */
constexpr int NRCV_Q = 10;
/* Global quantities (struct ssol_mc_global, src/ssol.h:388-395) */
enum : int {
  G_COS = 0, G_ABS_RCV = 1, G_SHADOW = 2, G_MISSING = 3, G_ATM = 4,
  G_OTHER = 5, NGLOBAL = 6
};

/* Scalar data: a constant or a piecewise linear spectrum */
struct DData {
  int32_t spectrum; /* -1 => constant `real`; else index into spectra */
  int32_t pad;
  double real;
};

struct DSpectrum {
  int32_t first; /* into wavelengths/values */
  int32_t count;
};

/* Medium: extinction and refractive index (struct ssol_medium) */
struct DMedium {
  DData extinction;
  DData refractive_index;
};

/* Per material constants; shader callbacks are tabulated per sun wavelength
 * node (`nodes` entries starting at `table`) */
struct alignas(16) DMaterial {
  int32_t type;
  int32_t distrib;
  int32_t in_medium; /* index into media */
  int32_t out_medium;
  int32_t table; /* into shader_tab: (reflectivity, roughness) pairs */
  int32_t slab_medium; /* thin dielectric */
  double thickness;
};

/* Instance x shaded shape record: what a hit resolves to */
struct alignas(16) DShadedInst {
  int32_t instance; /* index of the instance in attach order */
  int32_t mtl[2]; /* [0] front, [1] back */
  int32_t receiver_mask; /* SSOL_FRONT | SSOL_BACK bits */
  int32_t rcv_slot[2]; /* receiver-side slot for front/back, -1 if none */
  int32_t prim_base[2]; /* per-primitive tally base slot, -1 if none */
  int32_t sampled; /* index among sampled instances, -1 if not sampled */
  int32_t is_punched;
  int32_t quadric; /* quadric patch index when punched */
  int32_t virtual_mask; /* bit0: front material virtual, bit1: back */
  int32_t pad[3];
};

/* World-space triangle, stored as its three vertices (the watertight test
 * needs the shared vertices of neighbours bit-identical). The front-face
 * normal follows Star-3D: Ng = (v2 - v0) x (v1 - v0) = e2 x e1. */
template<typename R> struct alignas(16) DTri {
  R v0[3]; R v1[3]; R v2[3]; /* world vertices, FP32-rounded like Star-3D's */
  int32_t sinst; /* DShadedInst index */
  int32_t prim; /* triangle index inside its shape */
  int32_t gid; /* global triangle index (self-hit test) */
};

/* Shading attributes of a mesh triangle, present only in scenes that need
 * them: world-space vertex normals (n[0] is NaN when the mesh has none) and,
 * per side (front, back), the offset in DScene::bake_tab of shader values
 * baked at the three vertices (-1: the material's tabulated constants).
 * A baked block is [vertex 0..2][wavelength node][reflectivity, roughness]. */
template<typename R> struct alignas(16) DTriShade {
  R n[9];
  int32_t bake[2];
};

/* Analytic punched quadric patch */
template<typename R> struct alignas(16) DQuadric {
  R w2l[12]; /* world -> local: rows 0..2 of a 3x4 affine map (row major) */
  R l2w[12]; /* local -> world, same layout */
  R param[4]; /* kind specific constants, see quadric_eval in kernels */
  /* The same surface as an axis-aligned quadric in local coordinates,
   * F = kx x^2 + ky y^2 + kz (z - z0)^2 + lz z + m = 0, in FP64:
   * {kx, ky, kz, z0, lz, m, s, h}; the front normal is s grad F, and the
   * surface's height above (x, y) is the root z0 + h sqrt(...) when kz != 0 */
  double gen[8];
  R carve_lo[2], carve_hi[2]; /* AABB of the AND carvings (local xy) */
  R grid_delta; /* cell size of the RT tessellation grid */
  int32_t type;
  int32_t sinst;
  int32_t carve_first; /* into carvings */
  int32_t carve_count; /* 0: the AABB alone is the domain */
  int32_t grid_n[2]; /* grid cells along x and y (per-primitive tallies) */
};

/* Carving polygon: `count` vertices at carve_verts[first..] (local xy) */
struct DCarving {
  int32_t first;
  int32_t count;
  int32_t op; /* 0 AND, 1 SUB */
  int32_t pad;
};

/* Binary BVH node holding its children's boxes. count == 0: child is a node
 * index; count == 1: child is the leaf's prim reference itself; count > 1:
 * child is the leaf's first entry in primrefs; count < 0: empty slot. */
template<typename R> struct alignas(16) DNode {
  R lo[2][3];
  R hi[2][3];
  int32_t child[2];
  int32_t count[2];
};

/* Sampled flat proxy triangle (world space) */
template<typename R> struct alignas(16) DSampTri {
  R v0[3]; R e1[3]; R e2[3];
  R n[3]; /* normalised proxy normal (Star-3D orientation) */
  int32_t sinst;
  int32_t prim; /* RT triangle id for meshes */
  int32_t gid; /* global RT triangle index for meshes, -1 otherwise */
  int32_t pad;
};

/* Scene features a kernel variant handles (set per launch from the
 * snapshot): a variant without a feature drops its code from the hot loop */
enum : int32_t {
  FEAT_QUADRIC = 1, /* punched quadric patches */
  FEAT_DIELECTRIC = 2, /* dielectric or thin-dielectric materials */
  FEAT_ATTRIBUTES = 4, /* per-triangle shading attributes (DScene::tshade) */
  FEAT_ALL = 7,
  /* Not a scene feature: the plain kernel variant that does not count rays,
   * node visits and primitive tests (one instruction per node visit) */
  FEAT_NOCOUNT = 8
};

/* Counters for the roofline model (see kernels_device.cuh) */
struct DStats {
  unsigned long long rays;
  unsigned long long node_visits;
  unsigned long long tri_tests;
  unsigned long long quad_tests;
  unsigned long long bounces;
  unsigned long long paths;
};

/* Everything a launch reads, as device pointers */
template<typename R> struct DScene {
  const DNode<R>* nodes;
  const uint32_t* primrefs;
  const DTri<R>* tris;
  const DQuadric<R>* quads;
  const DCarving* carvings;
  const R* carve_verts; /* xy pairs */
  const DShadedInst* sinsts;
  const DMaterial* mtls;
  const DMedium* media;
  const DSpectrum* spectra;
  const double* spec_wl;
  const double* spec_val;
  const R* shader_tab; /* per material: nodes x (reflectivity, roughness) */
  const double* shader_wl; /* sun spectrum wavelength nodes */
  int32_t shader_nodes;

  const DSampTri<R>* samp;
  const float* alias_prob;
  const int32_t* alias_idx;
  int32_t nsamp;

  /* sun */
  int32_t sun_type;
  R sun_dir[3]; /* main direction (from the sun toward the scene) */
  R sun_basis[9]; /* columns: X, Y, sun_dir */
  R sun_param; /* sin^2(theta_max) for pillbox, sigma for gaussian */
  double buie[8];
  double dni;
  /* sun wavelength distribution */
  int32_t wl_count; /* 1 => Dirac */
  const double* wl_nodes;
  const double* wl_pdf; /* intensities */
  const double* wl_cdf; /* cumulative, normalised, wl_count entries */

  int32_t air_medium;
  double area_proxy; /* sampled_area_proxy */
  double area_rt; /* sampled_area */

  const DTriShade<R>* tshade; /* per triangle, or nullptr */
  const R* bake_tab; /* baked per-vertex shader values */

  int32_t nrcv; /* receiver-side slots */
  int32_t nsampled; /* sampled instances */
  int32_t nprim_slots; /* per-primitive tally slots */
};

/* Device tally buffers (all FP64 sums of (w, w^2)) */
struct DTallies {
  double* global; /* NGLOBAL x 2 */
  double* rcv; /* nrcv x NRCV_Q x 2 */
  double* samp; /* nsampled x 2(cos, shadow) x 2 */
  double* samp_rcv; /* nsampled x nrcv x NRCV_Q x 2 */
  double* prim; /* nprim_slots x NRCV_Q x 2 */
  unsigned long long* nb_samples; /* nsampled */
  unsigned long long* counters; /* [0] failed, [1] killed, [2] overflow,
                                   [3] work counter, [4] stop word,
                                   [5] abort word */
  DStats* stats;
};

/* Early stop of a plain launch (src/ssol_solver.c:1229, 1240-1248): once
 * `max_failed` paths have failed, the kernel sets the device word `stop`
 * and its warps take no new realisations; `abort` (device memory, or null)
 * is a word the host may set at any time, by a copy on a stream of its own,
 * for the same effect. Paths in flight always finish. `stop` null disables
 * the failure limit. */
struct DControl {
  unsigned long long max_failed;
  unsigned long long* stop;
  const unsigned long long* abort;
};

/* Path tracking (ssol_path_tracker): the realisations of launch index
 * below npaths record their vertices, each appended through a counter with
 * its path slot and its rank in the path; the host groups them back */
struct TrackVertex {
  uint32_t slot, seq;
  double pos[3];
  double weight;
};

struct DTrack {
  TrackVertex* verts;
  unsigned long long* nverts; /* vertices appended (may exceed cap) */
  unsigned long long cap; /* capacity of verts */
  int32_t* path_type; /* per slot: ssol_path_type, -1 if not registered */
  int32_t* path_nv; /* per slot: vertices the path produced */
  unsigned long long npaths; /* tracked launch indices [0, npaths) */
  double sun_len, inf_len; /* lengths of the sun and infinite segments */
};

} /* namespace ssolb */

#endif /* SSOL_B200_DEVICE_SCENE_H */
