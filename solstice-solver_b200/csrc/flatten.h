/*
 * flatten.h - snapshot of an ssol_scene into the flat arrays of
 * device_scene.h (host side, one precision R per snapshot).
 *
 * Restates the set-up half of ssol_solve: scene_check
 * (src/ssol_scene.c:539-558), the sampled/RT view creation and the sampled
 * areas (src/ssol_scene.c:347-433), the sun samplers' set-up
 * (src/ssol_sun.c:214-279, src/ssol_ranst_sun_dir.c:362-419,
 * src/ssol_ranst_sun_wl.c:154-188) and the estimator's receiver and sampled
 * registries (src/ssol_estimator.c:30-60).
 */
#ifndef SSOL_B200_FLATTEN_H
#define SSOL_B200_FLATTEN_H

#include "bvh.h"
#include "device_scene.h"
#include "objects.h"

#include <array>
#include <vector>

namespace ssolb {

/* Precision independent bookkeeping that maps tally slots back to API
 * objects when the estimator is built */
struct FlatMeta {
  std::vector<const ssol_instance*> sampled; /* sampled index -> instance */
  struct RcvSide { const ssol_instance* inst; int side; /* 0 front, 1 back */ };
  std::vector<RcvSide> rcv; /* receiver-side slot -> (instance, side) */
  struct PrimRange {
    int rcv_slot;
    const ssol_shape* shape;
    int base;
    int ntris;
  };
  std::vector<PrimRange> prims;
  int nprim_slots = 0;
  double sampled_area = 0;
  double sampled_area_proxy = 0;
  size_t scene_bytes = 0; /* bytes uploaded to the device */
  double aabb_lo[3] = {0, 0, 0}, aabb_hi[3] = {0, 0, 0}; /* ray-traced geometry */
  int features = 0; /* FEAT_* bits of the snapshot (kernel variant) */
  /* Where each (instance, mesh shaded shape) landed: its triangles
   * [tri_first, tri_first + ntris) and, for sampled instances, its sampled
   * triangles from samp_first (-1 otherwise), in the same order */
  struct MeshRange {
    const ssol_instance* inst;
    const ssol_shape* shape;
    int tri_first, ntris, samp_first;
  };
  std::vector<MeshRange> meshes;
  /* Per instance (attach order): device material indices of the front and
   * back of its first shaded shape, -1 if it has none */
  std::vector<std::array<int, 2>> inst_mtl;
};

template<class R> struct FlatScene {
  FlatMeta meta;
  BvhResult bvh;
  std::vector<DNode<R>> nodes;
  /* Device-built BVH (BvhBuildParams::device): the primitives' boxes rounded
   * outward (6 per primitive) and their references; `nodes` then holds the
   * n - 1 zeroed nodes the device builder fills, and bvh.depth is unknown
   * (0) until it has run */
  bool device_bvh = false;
  std::vector<R> prim_box;
  std::vector<uint32_t> prim_ref;
  std::vector<DTri<R>> tris;
  std::vector<DQuadric<R>> quads;
  std::vector<DCarving> carvings;
  std::vector<R> carve_verts;
  std::vector<DShadedInst> sinsts;
  std::vector<DMaterial> mtls;
  std::vector<DMedium> media;
  std::vector<DSpectrum> spectra;
  std::vector<double> spec_wl, spec_val;
  std::vector<R> shader_tab;
  std::vector<double> shader_wl;
  std::vector<DTriShade<R>> tshade; /* empty when no triangle needs it */
  std::vector<R> bake_tab;
  std::vector<DSampTri<R>> samp;
  std::vector<float> alias_prob;
  std::vector<int32_t> alias_idx;
  std::vector<double> wl_nodes, wl_pdf, wl_cdf;
  /* scalars copied into DScene<R> */
  int32_t sun_type = SUN_DIRAC;
  R sun_dir[3] = {0, 0, 0};
  R sun_basis[9] = {};
  R sun_param = 0;
  double buie[8] = {};
  double dni = 0;
  int32_t air_medium = 0;
};

/* for_draw: snapshot for the renderers, which sample no instance (no
 * "nothing to sample" error, no receiver warning) */
res_T flatten_scene
  (ssol_scene* scn, const BvhBuildParams& bvh, FlatScene<float>& out,
   bool for_draw = false);
res_T flatten_scene
  (ssol_scene* scn, const BvhBuildParams& bvh, FlatScene<double>& out,
   bool for_draw = false);

/* The sun's frame as a snapshot stores it (columns X, Y, dir), from its
 * unit direction */
void sun_frame(const double dir[3], double out[9]);

/* Vose's alias method over non-negative weights (deterministic) */
void build_alias(const std::vector<double>& w, std::vector<float>& prob,
                 std::vector<int32_t>& alias);

} /* namespace ssolb */

#endif /* SSOL_B200_FLATTEN_H */
