/*
 * tessellate.cpp - grid discretisation of punched surfaces and clipping of
 * the grid against the carving polygons.
 *
 * Grid and slice count: src/ssol_shape.c:493-574 (build_triangulated_plane)
 * and :1352-1403 (slice count). Quadric heights: src/ssol_shape.c:236-285.
 * Hyperboloid constants: src/ssol_shape.c:1283-1299.
 *
 * The clipping is a small convex-polygon Boolean kernel: each grid triangle
 * is intersected with every AND carving and has every SUB carving removed;
 * non-convex carvings are first split into triangles by ear clipping.
 */
#include "tessellate.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <map>

namespace {

using Pt = std::pair<double, double>;
using Poly = std::vector<Pt>;

double cross(const Pt& o, const Pt& a, const Pt& b)
{
  return (a.first - o.first) * (b.second - o.second)
       - (a.second - o.second) * (b.first - o.first);
}

double signed_area(const Poly& p)
{
  double a = 0;
  for(size_t i = 0; i < p.size(); ++i) {
    const Pt& u = p[i];
    const Pt& v = p[(i + 1) % p.size()];
    a += u.first * v.second - v.first * u.second;
  }
  return 0.5 * a;
}

bool is_convex_ccw(const Poly& p)
{
  if(p.size() < 3) return false;
  for(size_t i = 0; i < p.size(); ++i) {
    if(cross(p[i], p[(i + 1) % p.size()], p[(i + 2) % p.size()]) < 0)
      return false;
  }
  return true;
}

/* Keep the part of `in` on the left of the directed line a->b (CCW inside) */
Poly clip_halfplane(const Poly& in, const Pt& a, const Pt& b, bool keep_left)
{
  Poly out;
  const size_t n = in.size();
  if(!n) return out;
  auto side = [&](const Pt& p) {
    const double c = cross(a, b, p);
    return keep_left ? c : -c;
  };
  for(size_t i = 0; i < n; ++i) {
    const Pt& p = in[i];
    const Pt& q = in[(i + 1) % n];
    const double sp = side(p), sq = side(q);
    if(sp >= 0) out.push_back(p);
    if((sp >= 0) != (sq >= 0)) {
      const double t = sp / (sp - sq);
      out.emplace_back(p.first + t * (q.first - p.first),
                       p.second + t * (q.second - p.second));
    }
  }
  return out;
}

/* Intersection of a convex polygon with a convex CCW polygon */
Poly intersect_convex(Poly a, const Poly& b)
{
  for(size_t i = 0; i < b.size() && a.size() >= 3; ++i)
    a = clip_halfplane(a, b[i], b[(i + 1) % b.size()], true);
  return a;
}

/* Convex `a` minus convex CCW `b`, as disjoint convex pieces */
std::vector<Poly> subtract_convex(const Poly& a, const Poly& b)
{
  std::vector<Poly> pieces;
  Poly rest = a;
  for(size_t i = 0; i < b.size() && rest.size() >= 3; ++i) {
    const Pt& p = b[i];
    const Pt& q = b[(i + 1) % b.size()];
    Poly outside = clip_halfplane(rest, p, q, false);
    if(outside.size() >= 3 && std::fabs(signed_area(outside)) > 0)
      pieces.push_back(outside);
    rest = clip_halfplane(rest, p, q, true);
  }
  return pieces;
}

/* Ear clipping of a simple CCW polygon into triangles */
std::vector<Poly> ear_clip(Poly p)
{
  std::vector<Poly> tris;
  size_t guard = 0;
  while(p.size() > 3 && guard++ < 100000) {
    bool cut = false;
    for(size_t i = 0; i < p.size(); ++i) {
      const Pt& a = p[(i + p.size() - 1) % p.size()];
      const Pt& b = p[i];
      const Pt& c = p[(i + 1) % p.size()];
      if(cross(a, b, c) <= 0) continue;
      bool inside = false;
      for(size_t k = 0; k < p.size() && !inside; ++k) {
        const Pt& q = p[k];
        if(q == a || q == b || q == c) continue;
        inside = cross(a, b, q) >= 0 && cross(b, c, q) >= 0
              && cross(c, a, q) >= 0;
      }
      if(inside) continue;
      tris.push_back({a, b, c});
      p.erase(p.begin() + (long)i);
      cut = true;
      break;
    }
    if(!cut) break; /* degenerate input: give up on the remainder */
  }
  if(p.size() == 3) tris.push_back(p);
  return tris;
}

/* A carving as a list of convex CCW parts */
std::vector<Poly> convex_parts(const Carving& c)
{
  Poly p;
  for(size_t i = 0; i + 1 < c.xy.size(); i += 2) {
    const Pt v(c.xy[i], c.xy[i + 1]);
    if(p.empty() || p.back() != v) p.push_back(v);
  }
  while(p.size() > 1 && p.front() == p.back()) p.pop_back();
  if(p.size() < 3) return {};
  if(signed_area(p) < 0) std::reverse(p.begin(), p.end());
  if(is_convex_ccw(p)) return {p};
  return ear_clip(p);
}

}

double ssolb_quadric_z(int type, const double q[4], double x, double y)
{
  switch(type) {
    case SSOL_QUADRIC_PLANE: return 0;
    case SSOL_QUADRIC_PARABOL: return (x * x + y * y) * q[1];
    case SSOL_QUADRIC_PARABOL2F: return x * x * q[0] + y * y * q[1];
    case SSOL_QUADRIC_HYPERBOL: {
      /* q = (g/2, |b|, a^2/b^2, 1/a^2) */
      const double z0 = q[0] + q[1];
      return q[1] * std::sqrt(1 + (x * x + y * y) * q[3]) + q[0] - z0;
    }
    case SSOL_QUADRIC_PARABOLIC_CYLINDER: return y * y * q[1];
    case SSOL_QUADRIC_HEMISPHERE: {
      /* q = (r, r^2) */
      const double z2 = q[1] - (x * x + y * y);
      return z2 > 0 ? -std::sqrt(z2) + q[0] : q[0];
    }
    default: return 0;
  }
}

bool ssolb_in_carvings(const std::vector<Carving>& carvings, double x, double y)
{
  bool any_and = false;
  for(const Carving& c : carvings) {
    const size_t n = c.xy.size() / 2;
    bool in = false;
    for(size_t i = 0, j = n - 1; i < n; j = i++) {
      const double xi = c.xy[2 * i], yi = c.xy[2 * i + 1];
      const double xj = c.xy[2 * j], yj = c.xy[2 * j + 1];
      if(((yi > y) != (yj > y))
      && (x < (xj - xi) * (y - yi) / (yj - yi) + xi))
        in = !in;
    }
    if(c.op == SSOL_AND) {
      any_and = true;
      if(!in) return false;
    } else if(in) {
      return false;
    }
  }
  return any_and || carvings.empty();
}

static void quadric_constants(const ssol_quadric& q, double out[4])
{
  out[0] = out[1] = out[2] = out[3] = 0;
  switch(q.type) {
    case SSOL_QUADRIC_PARABOL:
      out[0] = q.data.parabol.focal;
      out[1] = 1 / (4.0 * q.data.parabol.focal);
      break;
    case SSOL_QUADRIC_PARABOL2F:
      out[0] = 1 / (4.0 * q.data.parabol2f.focal_x);
      out[1] = 1 / (4.0 * q.data.parabol2f.focal_y);
      break;
    case SSOL_QUADRIC_HYPERBOL: {
      const double g = q.data.hyperbol.real_focal + q.data.hyperbol.img_focal;
      const double f = q.data.hyperbol.real_focal / g;
      const double a2 = g * g * (f - f * f);
      out[0] = g * 0.5;
      out[1] = g * std::fabs(f - 0.5);
      out[2] = a2 / (out[1] * out[1]);
      out[3] = 1 / a2;
      break;
    }
    case SSOL_QUADRIC_PARABOLIC_CYLINDER:
      out[0] = q.data.parabolic_cylinder.focal;
      out[1] = 1 / (4.0 * q.data.parabolic_cylinder.focal);
      break;
    case SSOL_QUADRIC_HEMISPHERE:
      out[0] = q.data.hemisphere.radius;
      out[1] = q.data.hemisphere.radius * q.data.hemisphere.radius;
      break;
    default: break;
  }
}

res_T ssolb_tessellate_punched(const PunchedInput& in, PunchedMesh& out)
{
  const ssol_quadric& q = in.quadric;
  quadric_constants(q, out.qparam);

  std::vector<Poly> cells; /* convex pieces to emit, in grid order */
  size_t nslices = 0;

  if(q.type == SSOL_QUADRIC_HEMISPHERE) {
    /* Disk of radius min(carvings radius, r) (src/ssol_shape.c:1640-1644) */
    double r2 = -1;
    for(const Carving& c : in.carvings) {
      if(c.op == SSOL_SUB) continue;
      for(size_t i = 0; i + 1 < c.xy.size(); i += 2)
        r2 = std::max(r2, c.xy[i] * c.xy[i] + c.xy[i + 1] * c.xy[i + 1]);
    }
    double radius = r2 >= 0 ? std::sqrt(r2) : q.data.hemisphere.radius;
    radius = std::min(radius, q.data.hemisphere.radius);
    out.hemi_radius = radius;
    out.lower[0] = out.lower[1] = -radius;
    out.upper[0] = out.upper[1] = radius;
    nslices = q.slices_count_hint != SIZE_MAX
      ? q.slices_count_hint
      : (size_t)(5.5 + 11 * radius / q.data.hemisphere.radius);
    if(!nslices) return RES_BAD_ARG;
    /* Polar grid: `nslices` rings, enough sectors to follow the rim */
    const size_t nsect = std::max<size_t>(64, 8 * nslices);
    for(size_t k = 0; k < nslices; ++k) {
      const double ra = radius * std::sin(0.5 * M_PI * (double)k / nslices);
      const double rb = radius * std::sin(0.5 * M_PI * (double)(k+1)/nslices);
      for(size_t s = 0; s < nsect; ++s) {
        const double a0 = 2 * M_PI * (double)s / nsect;
        const double a1 = 2 * M_PI * (double)(s + 1) / nsect;
        const Pt p00(ra * std::cos(a0), ra * std::sin(a0));
        const Pt p01(ra * std::cos(a1), ra * std::sin(a1));
        const Pt p10(rb * std::cos(a0), rb * std::sin(a0));
        const Pt p11(rb * std::cos(a1), rb * std::sin(a1));
        if(k == 0) {
          cells.push_back({Pt(0, 0), p10, p11});
        } else {
          cells.push_back({p00, p10, p11});
          cells.push_back({p00, p11, p01});
        }
      }
    }
  } else {
    /* AABB of the non-SUB carvings (src/ssol_shape.c:392-415) */
    double lo[2] = {DBL_MAX, DBL_MAX}, hi[2] = {-DBL_MAX, -DBL_MAX};
    for(const Carving& c : in.carvings) {
      if(c.op == SSOL_SUB) continue;
      for(size_t i = 0; i + 1 < c.xy.size(); i += 2) {
        lo[0] = std::min(lo[0], c.xy[i]); hi[0] = std::max(hi[0], c.xy[i]);
        lo[1] = std::min(lo[1], c.xy[i+1]); hi[1] = std::max(hi[1], c.xy[i+1]);
      }
    }
    if(lo[0] >= hi[0] || lo[1] >= hi[1]) return RES_BAD_ARG;
    out.lower[0] = lo[0]; out.lower[1] = lo[1];
    out.upper[0] = hi[0]; out.upper[1] = hi[1];

    /* Slice count (src/ssol_shape.c:1352-1395) */
    if(q.slices_count_hint != SIZE_MAX) {
      nslices = q.slices_count_hint;
    } else if(q.type == SSOL_QUADRIC_PLANE) {
      nslices = 1;
    } else {
      const double zmax = std::max
        (ssolb_quadric_z(q.type, out.qparam, lo[0], lo[1]),
         ssolb_quadric_z(q.type, out.qparam, hi[0], hi[1]));
      nslices = std::min<size_t>(50, (size_t)(3 + std::sqrt(zmax) * 6));
    }
    if(!nslices) return RES_BAD_ARG;

    /* Grid (src/ssol_shape.c:493-574) */
    const double size[2] = {hi[0] - lo[0], hi[1] - lo[1]};
    const double size_min = std::min(size[0], size[1]);
    if(std::fabs(size_min) <= 1e-6) return RES_BAD_ARG;
    const double delta = size_min / (double)nslices;
    const size_t nx = (size_t)std::ceil(size[0] / delta);
    const size_t ny = (size_t)std::ceil(size[1] / delta);
    out.grid_n[0] = nx;
    out.grid_n[1] = ny;
    out.grid_delta = delta;
    auto vtx = [&](size_t ix, size_t iy) {
      return Pt(std::min(lo[0] + (double)ix * delta, hi[0]),
                std::min(lo[1] + (double)iy * delta, hi[1]));
    };
    for(size_t ix = 0; ix < nx; ++ix) {
      for(size_t iy = 0; iy < ny; ++iy) {
        const Pt v0 = vtx(ix, iy), v1 = vtx(ix + 1, iy);
        const Pt v2 = vtx(ix, iy + 1), v3 = vtx(ix + 1, iy + 1);
        cells.push_back({v0, v3, v1});
        cells.push_back({v0, v2, v3});
      }
    }
  }

  /* Clip every cell triangle against the carvings */
  std::vector<std::vector<Poly>> and_parts, sub_parts;
  for(const Carving& c : in.carvings) {
    std::vector<Poly> parts = convex_parts(c);
    if(c.op == SSOL_AND) and_parts.push_back(parts);
    else sub_parts.push_back(parts);
  }

  std::vector<Poly> tris_out;
  size_t kept_intact = 0;
  for(const Poly& tri : cells) {
    /* Work in CCW order, remember the original winding to restore it */
    const bool ccw = signed_area(tri) > 0;
    Poly t = tri;
    if(!ccw) std::reverse(t.begin(), t.end());
    std::vector<Poly> pieces = {t};
    for(const std::vector<Poly>& parts : and_parts) {
      std::vector<Poly> next;
      for(const Poly& piece : pieces)
        for(const Poly& part : parts) {
          Poly r = intersect_convex(piece, part);
          if(r.size() >= 3 && signed_area(r) > 0) next.push_back(r);
        }
      pieces.swap(next);
    }
    for(const std::vector<Poly>& parts : sub_parts) {
      for(const Poly& part : parts) {
        std::vector<Poly> next;
        for(const Poly& piece : pieces) {
          std::vector<Poly> r = subtract_convex(piece, part);
          next.insert(next.end(), r.begin(), r.end());
        }
        pieces.swap(next);
      }
    }
    for(Poly& piece : pieces) {
      /* Unchanged triangle: keep its vertex order */
      if(piece.size() == 3 && pieces.size() == 1
      && std::is_permutation(piece.begin(), piece.end(), t.begin())) {
        tris_out.push_back(tri);
        ++kept_intact;
        continue;
      }
      for(size_t k = 1; k + 1 < piece.size(); ++k) {
        Poly f = {piece[0], piece[k], piece[k + 1]};
        if(std::fabs(signed_area(f)) <= 0) continue;
        if(!ccw) std::reverse(f.begin(), f.end());
        tris_out.push_back(f);
      }
    }
  }

  out.grid_exact = q.type != SSOL_QUADRIC_HEMISPHERE
    && kept_intact == cells.size() && tris_out.size() == cells.size();

  /* Emit with shared vertices */
  std::map<Pt, uint32_t> index;
  out.ids.clear();
  out.flat_xy.clear();
  for(const Poly& t : tris_out) {
    for(const Pt& p : t) {
      auto it = index.find(p);
      uint32_t id;
      if(it == index.end()) {
        id = (uint32_t)(out.flat_xy.size() / 2);
        index.emplace(p, id);
        out.flat_xy.push_back(p.first);
        out.flat_xy.push_back(p.second);
      } else {
        id = it->second;
      }
      out.ids.push_back(id);
    }
  }

  /* Object-space positions (src/ssol_shape.c:202-390, quadric_mesh_*_get_pos)
   * and uv (src/ssol_shape.c:177-190) */
  const double* T = q.transform;
  const size_t nv = out.flat_xy.size() / 2;
  out.rt_pos.resize(nv * 3);
  out.samp_pos.resize(nv * 3);
  out.uv.resize(nv * 2);
  for(size_t v = 0; v < nv; ++v) {
    const double x = out.flat_xy[2 * v], y = out.flat_xy[2 * v + 1];
    const double z = ssolb_quadric_z(q.type, out.qparam, x, y);
    const double xf = (float)x, yf = (float)y;
    for(int c = 0; c < 3; ++c) {
      out.rt_pos[v * 3 + c] =
        (float)(T[c] * x + T[3 + c] * y + T[6 + c] * z + T[9 + c]);
      out.samp_pos[v * 3 + c] = (float)(T[c] * xf + T[3 + c] * yf + T[9 + c]);
    }
    out.uv[2 * v] = (float)((x - out.lower[0]) / (out.upper[0] - out.lower[0]));
    out.uv[2 * v + 1] =
      (float)((y - out.lower[1]) / (out.upper[1] - out.lower[1]));
  }
  if(out.ids.empty()) return RES_BAD_ARG;
  return RES_OK;
}
