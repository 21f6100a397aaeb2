/*
 * bvh.h - binned-SAH binary BVH over world-space primitive boxes, emitted in
 * the "children boxes in the parent" layout of DNode (device_scene.h).
 * Replaces the Star-3D acceleration structure (src/ssol_scene.c:410-413).
 */
#ifndef SSOL_B200_BVH_H
#define SSOL_B200_BVH_H

#include "device_scene.h"

#include <cstdint>
#include <vector>

namespace ssolb {

struct PrimBox {
  double lo[3], hi[3];
  uint32_t ref; /* primref_make(kind, index) */
};

struct BvhBuildParams {
  int max_leaf = 4; /* primitives per leaf */
  int bins = 16; /* SAH bins per axis */
  int max_depth = 30; /* the device traversal stack holds 32 entries */
  int threads = 1; /* host threads for the subtrees of large scenes */
  /* Leave the tree to the device builder (lbvh.cu): the snapshot keeps the
   * primitive boxes instead (scenes of at least 2 primitives) */
  bool device = false;
};

struct BvhResult {
  std::vector<double> lo, hi; /* per node child boxes: node*2+k, 3 each */
  std::vector<int32_t> child, count; /* per node*2+k */
  std::vector<uint32_t> primrefs;
  int depth = 0;
};

void build_bvh(std::vector<PrimBox> prims, const BvhBuildParams& params,
               BvhResult& out);

/* A primitive's box in precision R, rounded outward: lo xyz, hi xyz */
template<class R> void round_box_outward(const PrimBox& b, R out[6]);

/* Convert to device nodes of precision R, rounding boxes outward */
template<class R> std::vector<DNode<R>> bvh_nodes(const BvhResult& b);

} /* namespace ssolb */

#endif /* SSOL_B200_BVH_H */
