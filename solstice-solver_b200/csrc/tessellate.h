/*
 * tessellate.h - host-side discretisation of punched surfaces.
 *
 * A punched surface is a quadric clipped in its local xy plane by carving
 * polygons. The GPU intersects the quadric analytically; this discretisation
 * only provides what the reference derives from its tessellated proxies
 * (src/ssol_shape.c:493-652, 691-811, 1611-1699):
 *  - the flat sampling proxy (z = 0) whose area is `sampled_area_proxy`;
 *  - the z-displaced RT triangulation whose area is the instance area and
 *    whose triangles index the per-primitive receiver tallies.
 * The grid and its slice count follow the reference; the clipping against
 * the carvings is this project's own convex-polygon Boolean code.
 */
#ifndef SSOL_B200_TESSELLATE_H
#define SSOL_B200_TESSELLATE_H

#include "objects.h"

struct PunchedInput {
  ssol_quadric quadric;
  std::vector<Carving> carvings;
};

struct PunchedMesh {
  double qparam[4] = {0, 0, 0, 0};
  double lower[2] = {0, 0}, upper[2] = {0, 0};
  double hemi_radius = 0;
  /* Rectangular grid of the tessellation; `grid_exact` when no carving cut a
   * grid triangle, so that triangle ids follow from (x, y) arithmetically */
  size_t grid_n[2] = {0, 0};
  double grid_delta = 0;
  bool grid_exact = false;
  std::vector<double> flat_xy; /* quadric local xy, 2 per vertex */
  std::vector<float> rt_pos; /* object space, z displaced, 3 per vertex */
  std::vector<float> samp_pos; /* object space, z = 0, 3 per vertex */
  std::vector<float> uv; /* 2 per vertex */
  std::vector<uint32_t> ids; /* 3 per triangle */
};

res_T ssolb_tessellate_punched(const PunchedInput& in, PunchedMesh& out);

/* Quadric height z(x, y) in its local frame */
double ssolb_quadric_z(int type, const double qparam[4], double x, double y);

/* Even-odd point in carved domain test (local xy) */
bool ssolb_in_carvings
  (const std::vector<Carving>& carvings, double x, double y);

#endif /* SSOL_B200_TESSELLATE_H */
