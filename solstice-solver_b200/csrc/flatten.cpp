/*
 * flatten.cpp - ssol_scene -> FlatScene<R> (see flatten.h).
 */
#include "flatten.h"
#include "tessellate.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <limits>
#include <map>
#include <set>

void ssolb_d33_invtrans(double out[9], const double m[9]); /* objects.cpp */

namespace ssolb {

namespace {

/* 3x4 column-major affine helpers (the ssol_instance / ssol_quadric
 * transform convention: R in [0..8] column major, T in [9..11]) */
void compose(double out[12], const double a[12], const double b[12])
{
  double r[12];
  for(int c = 0; c < 3; ++c)
    for(int row = 0; row < 3; ++row)
      r[c * 3 + row] = a[row] * b[c * 3] + a[3 + row] * b[c * 3 + 1]
                     + a[6 + row] * b[c * 3 + 2];
  for(int row = 0; row < 3; ++row)
    r[9 + row] = a[row] * b[9] + a[3 + row] * b[10] + a[6 + row] * b[11]
               + a[9 + row];
  for(int i = 0; i < 12; ++i) out[i] = r[i];
}

bool invert(double out[12], const double m[12])
{
  const double a = m[0], b = m[3], c = m[6];
  const double d = m[1], e = m[4], f = m[7];
  const double g = m[2], h = m[5], k = m[8];
  const double A = e * k - f * h, B = -(d * k - f * g), C = d * h - e * g;
  const double det = a * A + b * B + c * C;
  if(det == 0) return false;
  const double inv = 1.0 / det;
  /* row-major inverse entries */
  const double i00 = A * inv, i01 = -(b * k - c * h) * inv, i02 = (b * f - c * e) * inv;
  const double i10 = B * inv, i11 = (a * k - c * g) * inv, i12 = -(a * f - c * d) * inv;
  const double i20 = C * inv, i21 = -(a * h - b * g) * inv, i22 = (a * e - b * d) * inv;
  out[0] = i00; out[3] = i01; out[6] = i02;
  out[1] = i10; out[4] = i11; out[7] = i12;
  out[2] = i20; out[5] = i21; out[8] = i22;
  for(int row = 0; row < 3; ++row)
    out[9 + row] = -(out[row] * m[9] + out[3 + row] * m[10]
                   + out[6 + row] * m[11]);
  return true;
}

void apply(const double m[12], const double p[3], double out[3])
{
  for(int r = 0; r < 3; ++r)
    out[r] = m[r] * p[0] + m[3 + r] * p[1] + m[6 + r] * p[2] + m[9 + r];
}

/* Column-major 3x4 -> row-major 3x4 of precision R */
template<class R> void to_rows(R out[12], const double m[12])
{
  for(int r = 0; r < 3; ++r) {
    for(int c = 0; c < 3; ++c) out[r * 4 + c] = (R)m[c * 3 + r];
    out[r * 4 + 3] = (R)m[9 + r];
  }
}

/* Buie sunshape constants (src/ssol_ranst_sun_dir.c:82-222): the Buie et al.
 * (2003) circumsolar profile with its published CSR calibration */
double buie_chi(double csr)
{
  if(csr > 0.145)
    return -0.04419909985804843 + csr * (1.401323894233574
      + csr * (-0.3639746714505299 + csr * (-0.9579768560161194
      + 1.1550475450828657 * csr)));
  if(csr > 0.035)
    return 0.022652077593662934 + csr * (0.5252380349996234
      + csr * (2.5484334534423887 - 0.8763755326550412 * csr));
  return 0.004733749294807862 + csr * (4.716738065192151
    + csr * (-463.506669149804 + csr * (24745.88727411664
    + csr * (-606122.7511711778 + 5521693.445014727 * csr))));
}

void buie_state(double csr, double out[8])
{
  const double thetaSD = 0.00465, thetaCS = 0.0436;
  const double integralA = 9.224724736098827E-6;
  const double chi = buie_chi(csr);
  const double k = 0.9 * std::log(13.5 * chi) * std::pow(chi, -0.3);
  const double gamma = 2.2 * std::log(0.52 * chi) * std::pow(chi, 0.43) - 0.1;
  const double ek1000g = std::exp(k) * std::pow(1000, gamma);
  const double g2 = gamma + 2.0;
  const double integralB = ek1000g / g2
    * (std::pow(thetaCS, g2) - std::pow(thetaSD, g2));
  const double alpha = 1 / (integralA + integralB);
  auto pdf = [&](double t) {
    const double phi = t < thetaSD ? std::cos(326 * t) / std::cos(308 * t)
                                   : ek1000g * std::pow(t, gamma);
    return alpha * phi * std::sin(t);
  };
  const double h1 = 1.001 * pdf(0.0038915695846209047);
  const double h2 = pdf(thetaSD);
  const double d = thetaCS - thetaSD;
  out[0] = thetaSD;
  out[1] = d;
  out[2] = gamma;
  out[3] = ek1000g;
  out[4] = alpha;
  out[5] = h1;
  out[6] = h2;
  out[7] = (thetaSD * h1) / (thetaSD * h1 + d * h2);
}

/* Orthonormal basis, same construction as the device (Duff et al. 2017) */
void basis(const double n[3], double out[9])
{
  const double sgn = n[2] >= 0 ? 1.0 : -1.0;
  const double a = -1.0 / (sgn + n[2]);
  const double b = n[0] * n[1] * a;
  const double b1[3] = {1 + sgn * n[0] * n[0] * a, sgn * b, -sgn * n[0]};
  const double b2[3] = {b, sgn + n[1] * n[1] * a, -n[1]};
  for(int c = 0; c < 3; ++c) {
    out[c] = b1[c];
    out[3 + c] = b2[c];
    out[6 + c] = n[c];
  }
}

struct Interner {
  std::vector<ssol_medium> media;
  std::map<const ssol_spectrum*, int> spectra;
};

template<class R>
int intern_spectrum(FlatScene<R>& out, Interner& in, const ssol_spectrum* s)
{
  auto it = in.spectra.find(s);
  if(it != in.spectra.end()) return it->second;
  DSpectrum d;
  d.first = (int32_t)out.spec_wl.size();
  d.count = (int32_t)s->wavelengths.size();
  out.spec_wl.insert(out.spec_wl.end(), s->wavelengths.begin(),
                     s->wavelengths.end());
  out.spec_val.insert(out.spec_val.end(), s->intensities.begin(),
                      s->intensities.end());
  const int id = (int)out.spectra.size();
  out.spectra.push_back(d);
  in.spectra.emplace(s, id);
  return id;
}

template<class R>
DData to_ddata(FlatScene<R>& out, Interner& in, const ssol_data& d)
{
  DData r;
  r.pad = 0;
  if(d.type == SSOL_DATA_SPECTRUM) {
    r.spectrum = intern_spectrum(out, in, d.value.spectrum);
    r.real = 0;
  } else {
    r.spectrum = -1;
    r.real = d.value.real;
  }
  return r;
}

/* Media compare by value (media_ceq, src/ssol_material.c:730-736) */
template<class R>
int intern_medium(FlatScene<R>& out, Interner& in, const ssol_medium& m)
{
  for(size_t i = 0; i < in.media.size(); ++i)
    if(ssolb_media_ceq(in.media[i], m)) return (int)i;
  DMedium d;
  d.extinction = to_ddata(out, in, m.extinction);
  d.refractive_index = to_ddata(out, in, m.refractive_index);
  out.media.push_back(d);
  in.media.push_back(m);
  return (int)in.media.size() - 1;
}

/* Evaluate shader callbacks once per sun wavelength node on a canonical
 * fragment; shaders may vary with the wavelength, not with the position */
template<class R>
bool tabulate_shaders(FlatScene<R>& out, ssol_material* m, ssol_device* dev)
{
  ssol_surface_fragment frag = SSOL_SURFACE_FRAGMENT_NULL;
  frag.dir[2] = -1;
  frag.Ng[2] = 1;
  frag.Ns[2] = 1;
  frag.dPdu[0] = 1;
  frag.dPdv[1] = 1;
  for(double wl : out.shader_wl) {
    double refl = 0, rough = 0;
    if(m->reflectivity) m->reflectivity(dev, m->buf, wl, &frag, &refl);
    if(m->roughness) m->roughness(dev, m->buf, wl, &frag, &rough);
    out.shader_tab.push_back((R)refl);
    out.shader_tab.push_back((R)rough);
  }
  if(m->normal) {
    /* Normal shaders are evaluated per hit by the reference
     * (src/ssol_material.c:551-655); the device uses Ns, so any other
     * normal is refused rather than silently replaced */
    ssol_surface_fragment tilted = frag;
    tilted.Ns[0] = 0.6; tilted.Ns[2] = 0.8;
    const ssol_surface_fragment* probes[2] = {&frag, &tilted};
    for(const ssol_surface_fragment* f : probes) {
      double n[3] = {0, 0, 0};
      m->normal(dev, m->buf, out.shader_wl[0], f, n);
      if(n[0] != f->Ns[0] || n[1] != f->Ns[1] || n[2] != f->Ns[2]) {
        dev->log_error("normal shaders other than the shading normal Ns are "
                       "not supported on the device.\n");
        return false;
      }
    }
  }
  return true;
}

/* Fragments of the three vertices of mesh triangle t seen from `side`
 * (0 front, 1 back), with the fields of surface_fragment_setup
 * (src/ssol_material.c:551-655): P the vertex, Ng the side's unit normal, dir
 * = -Ng, uv the vertex texcoord or Star-3D's default (1,0), (0,1), (0,0), Ns
 * the vertex normal through the inverse transpose of the instance (or Ng),
 * turned toward -dir, dPdu and dPdv of the triangle. */
void vertex_fragments(const ssol_shape* shape, int t, const double T[12],
                      const double Rn[9], int side, ssol_surface_fragment f[3])
{
  double v[3][3];
  for(int k = 0; k < 3; ++k) {
    const uint32_t id = shape->ids[(size_t)t * 3 + k];
    const double p[3] = {shape->pos[id * 3 + 0], shape->pos[id * 3 + 1],
                         shape->pos[id * 3 + 2]};
    apply(T, p, v[k]);
  }
  double e1[3], e2[3], n[3];
  for(int c = 0; c < 3; ++c) { e1[c] = v[1][c] - v[0][c]; e2[c] = v[2][c] - v[0][c]; }
  n[0] = e2[1] * e1[2] - e2[2] * e1[1];
  n[1] = e2[2] * e1[0] - e2[0] * e1[2];
  n[2] = e2[0] * e1[1] - e2[1] * e1[0];
  double len = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  if(!(len > 0)) len = 1;
  const double sgn = side == 0 ? 1.0 : -1.0;
  double ng[3];
  for(int c = 0; c < 3; ++c) ng[c] = sgn * n[c] / len;
  double uv[3][2] = {{1, 0}, {0, 1}, {0, 0}};
  if(!shape->uv.empty())
    for(int k = 0; k < 3; ++k) {
      const uint32_t id = shape->ids[(size_t)t * 3 + k];
      uv[k][0] = shape->uv[id * 2 + 0];
      uv[k][1] = shape->uv[id * 2 + 1];
    }
  const double duv1[2] = {uv[1][0] - uv[0][0], uv[1][1] - uv[0][1]};
  const double duv2[2] = {uv[2][0] - uv[0][0], uv[2][1] - uv[0][1]};
  const double det = duv1[0] * duv2[1] - duv1[1] * duv2[0];
  double dpdu[3], dpdv[3];
  if(det == 0) {
    /* any orthonormal tangents of Ng (Duff et al. basis) */
    const double s2 = ng[2] >= 0 ? 1.0 : -1.0;
    const double a = -1.0 / (s2 + ng[2]), b = ng[0] * ng[1] * a;
    dpdu[0] = 1 + s2 * ng[0] * ng[0] * a; dpdu[1] = s2 * b; dpdu[2] = -s2 * ng[0];
    dpdv[0] = b; dpdv[1] = s2 + ng[1] * ng[1] * a; dpdv[2] = -ng[1];
  } else {
    for(int c = 0; c < 3; ++c) {
      dpdu[c] = (e1[c] * duv2[1] - e2[c] * duv1[1]) / det;
      dpdv[c] = (e2[c] * duv1[0] - e1[c] * duv2[0]) / det;
    }
  }
  for(int k = 0; k < 3; ++k) {
    ssol_surface_fragment& fr = f[k];
    fr = SSOL_SURFACE_FRAGMENT_NULL;
    for(int c = 0; c < 3; ++c) {
      fr.P[c] = v[k][c];
      fr.Ng[c] = ng[c];
      fr.dir[c] = -ng[c];
      fr.Ns[c] = ng[c];
      fr.dPdu[c] = dpdu[c];
      fr.dPdv[c] = dpdv[c];
    }
    fr.uv[0] = uv[k][0];
    fr.uv[1] = uv[k][1];
    if(!shape->nrm.empty()) {
      const uint32_t id = shape->ids[(size_t)t * 3 + k];
      const double m[3] = {shape->nrm[id * 3 + 0], shape->nrm[id * 3 + 1],
                           shape->nrm[id * 3 + 2]};
      double w[3], l = 0;
      for(int c = 0; c < 3; ++c) {
        w[c] = Rn[c] * m[0] + Rn[3 + c] * m[1] + Rn[6 + c] * m[2];
        l += w[c] * w[c];
      }
      l = std::sqrt(l);
      if(l > 0) {
        double d = 0;
        for(int c = 0; c < 3; ++c) { w[c] /= l; d += fr.dir[c] * w[c]; }
        for(int c = 0; c < 3; ++c) fr.Ns[c] = d > 0 ? -w[c] : w[c];
      }
    }
  }
}

/* Matrix that takes vertex normals to world space: the inverse transpose of
 * the instance's linear part, except when one of its three columns, in FP32,
 * equals the identity's, where src/ssol_material.c:632-646 keeps the normal
 * as it is */
void normal_matrix(const double T[12], double Rn[9])
{
  bool any_id = false;
  for(int c = 0; c < 3; ++c) {
    bool eq = true;
    for(int r = 0; r < 3; ++r)
      eq = eq && (float)T[3 * c + r] == (r == c ? 1.f : 0.f);
    any_id = any_id || eq;
  }
  if(any_id) {
    for(int k = 0; k < 9; ++k) Rn[k] = (k % 4 == 0) ? 1.0 : 0.0;
  } else {
    ssolb_d33_invtrans(Rn, T);
  }
}

/* Whether a mirror or matte material's shaders give other values at the
 * vertex fragments of a shape than at the reference fragment used for the
 * per-material table (then they are baked per vertex) */
bool material_varies(ssol_material* m, const ssol_surface_fragment* f, int nf,
                     double wl, ssol_device* dev)
{
  if(m->type != SSOL_MATERIAL_MIRROR && m->type != SSOL_MATERIAL_MATTE) return false;
  ssol_surface_fragment ref = SSOL_SURFACE_FRAGMENT_NULL;
  ref.dir[2] = -1; ref.Ng[2] = 1; ref.Ns[2] = 1; ref.dPdu[0] = 1; ref.dPdv[1] = 1;
  double r0 = 0, g0 = 0;
  if(m->reflectivity) m->reflectivity(dev, m->buf, wl, &ref, &r0);
  if(m->roughness) m->roughness(dev, m->buf, wl, &ref, &g0);
  for(int i = 0; i < nf; ++i) {
    double r = 0, g = 0;
    if(m->reflectivity) m->reflectivity(dev, m->buf, wl, &f[i], &r);
    if(m->roughness) m->roughness(dev, m->buf, wl, &f[i], &g);
    if(r != r0 || g != g0) return true;
  }
  return false;
}

/* Whether a mirror or matte material's shaders read the fragment's
 * incoming direction: at each probe fragment, the values with dir = -Ng and
 * with dir tilted toward dPdu differ. The reference evaluates the shaders
 * per hit with the ray's direction (src/ssol_material.c:551-655); the device
 * tables and per-vertex bakes cannot hold that. */
bool material_reads_dir(ssol_material* m, const ssol_surface_fragment* f, int nf,
                        double wl, ssol_device* dev)
{
  if(m->type != SSOL_MATERIAL_MIRROR && m->type != SSOL_MATERIAL_MATTE) return false;
  for(int i = 0; i < nf; ++i) {
    ssol_surface_fragment g = f[i];
    double t[3], l = 0;
    for(int c = 0; c < 3; ++c) { t[c] = g.dir[c] + 0.5 * g.dPdu[c]; l += t[c] * t[c]; }
    l = std::sqrt(l);
    if(!(l > 0)) continue;
    for(int c = 0; c < 3; ++c) g.dir[c] = t[c] / l;
    double r0 = 0, g0 = 0, r1 = 0, g1 = 0;
    if(m->reflectivity) {
      m->reflectivity(dev, m->buf, wl, &f[i], &r0);
      m->reflectivity(dev, m->buf, wl, &g, &r1);
    }
    if(m->roughness) {
      m->roughness(dev, m->buf, wl, &f[i], &g0);
      m->roughness(dev, m->buf, wl, &g, &g1);
    }
    if(r0 != r1 || g0 != g1) return true;
  }
  return false;
}

/* Fragments at a 3 x 3 grid of points of a punched surface (the carving's
 * box, points outside the carvings skipped; its centre always kept), seen
 * from `side`: P on the quadric through the local -> world map M, Ng = Ns the
 * side's unit normal, dir = -Ng, dPdu and dPdv the local x and y axes */
static int punched_fragments(const ssol_shape* shape, const double M[12], int side,
                             ssol_surface_fragment f[9])
{
  int n = 0;
  for(int j = 0; j < 3; ++j)
    for(int i = 0; i < 3; ++i) {
      const double x = shape->carve_lo[0] + 0.5 * i * (shape->carve_hi[0] - shape->carve_lo[0]);
      const double y = shape->carve_lo[1] + 0.5 * j * (shape->carve_hi[1] - shape->carve_lo[1]);
      if(!(i == 1 && j == 1) && !ssolb_in_carvings(shape->carvings, x, y)) continue;
      const double h = 1e-4 * std::max(1.0, shape->carve_hi[0] - shape->carve_lo[0]);
      const double z = ssolb_quadric_z(shape->quadric.type, shape->qparam, x, y);
      const double zx = (ssolb_quadric_z(shape->quadric.type, shape->qparam, x + h, y)
                       - ssolb_quadric_z(shape->quadric.type, shape->qparam, x - h, y)) / (2 * h);
      const double zy = (ssolb_quadric_z(shape->quadric.type, shape->qparam, x, y + h)
                       - ssolb_quadric_z(shape->quadric.type, shape->qparam, x, y - h)) / (2 * h);
      const double pl[3] = {x, y, z}, tu[3] = {1, 0, zx}, tv[3] = {0, 1, zy};
      ssol_surface_fragment& fr = f[n++];
      fr = SSOL_SURFACE_FRAGMENT_NULL;
      double pw[3], du[3], dv[3], ng[3];
      apply(M, pl, pw);
      for(int c = 0; c < 3; ++c) {
        du[c] = M[c] * tu[0] + M[3 + c] * tu[1] + M[6 + c] * tu[2];
        dv[c] = M[c] * tv[0] + M[3 + c] * tv[1] + M[6 + c] * tv[2];
      }
      ng[0] = du[1] * dv[2] - du[2] * dv[1];
      ng[1] = du[2] * dv[0] - du[0] * dv[2];
      ng[2] = du[0] * dv[1] - du[1] * dv[0];
      double l = std::sqrt(ng[0] * ng[0] + ng[1] * ng[1] + ng[2] * ng[2]);
      if(!(l > 0)) l = 1;
      const double sg = side == 0 ? 1.0 : -1.0;
      for(int c = 0; c < 3; ++c) {
        fr.P[c] = pw[c];
        fr.Ng[c] = fr.Ns[c] = sg * ng[c] / l;
        fr.dir[c] = -fr.Ng[c];
        fr.dPdu[c] = du[c];
        fr.dPdv[c] = dv[c];
      }
    }
  return n;
}

/* The patch's surface as F = kx x^2 + ky y^2 + kz (z - z0)^2 + lz z + m
 * over its (rounded) kind constants, with the sign that turns grad F into
 * the front normal of src/ssol_shape.c:236-285 and the side of z0 its
 * height is taken on (DQuadric::gen) */
template<class R>
static void quadric_general(DQuadric<R>& q)
{
  const double p0 = (double)q.param[0], p1 = (double)q.param[1], p3 = (double)q.param[3];
  double* g = q.gen;
  for(int k = 0; k < 8; ++k) g[k] = 0;
  switch(q.type) {
    case QUAD_PLANE: g[4] = 1; g[6] = 1; break;
    case QUAD_PARABOL: g[0] = g[1] = 1; g[4] = -4 * p0; g[6] = -1; break;
    case QUAD_PARABOL2F: g[0] = p0; g[1] = p1; g[4] = -1; g[6] = -1; break;
    case QUAD_HYPERBOL:
      g[0] = g[1] = p1 * p1 * p3; g[2] = -1; g[3] = -p1; g[5] = p1 * p1; g[6] = 1;
      g[7] = 1; /* upper sheet */
      break;
    case QUAD_PCYLINDER: g[1] = 1; g[4] = -4 * p0; g[6] = -1; break;
    case QUAD_HEMISPHERE:
      g[0] = g[1] = g[2] = 1; g[3] = p0; g[5] = -p1; g[6] = -1;
      g[7] = -1; /* the half below the centre */
      break;
    default: g[4] = 1; g[6] = 1; break;
  }
}

/* Quadric patch bounds: local z range over the carving AABB */
void quadric_z_range(const ssol_shape* s, double& zlo, double& zhi)
{
  const double* lo = s->carve_lo;
  const double* hi = s->carve_hi;
  const int t = s->quadric.type;
  if(t == SSOL_QUADRIC_PLANE) { zlo = zhi = 0; return; }
  /* All supported heights are monotonic in |x| and |y| */
  const double xmin = (lo[0] <= 0 && hi[0] >= 0) ? 0
                    : std::min(std::fabs(lo[0]), std::fabs(hi[0]));
  const double ymin = (lo[1] <= 0 && hi[1] >= 0) ? 0
                    : std::min(std::fabs(lo[1]), std::fabs(hi[1]));
  const double xmax = std::max(std::fabs(lo[0]), std::fabs(hi[0]));
  const double ymax = std::max(std::fabs(lo[1]), std::fabs(hi[1]));
  zlo = ssolb_quadric_z(t, s->qparam, xmin, ymin);
  zhi = ssolb_quadric_z(t, s->qparam, xmax, ymax);
  if(zlo > zhi) std::swap(zlo, zhi);
}

} /* namespace */

void sun_frame(const double dir[3], double out[9]) { basis(dir, out); }

void build_alias(const std::vector<double>& w, std::vector<float>& prob,
                 std::vector<int32_t>& alias)
{
  const size_t n = w.size();
  prob.assign(n, 1.0f);
  alias.resize(n);
  double total = 0;
  for(double x : w) total += x;
  std::vector<double> p(n);
  std::vector<int32_t> small, large;
  for(size_t i = 0; i < n; ++i) {
    alias[i] = (int32_t)i;
    p[i] = total > 0 ? w[i] * (double)n / total : 1.0;
    if(p[i] < 1.0) small.push_back((int32_t)i);
    else large.push_back((int32_t)i);
  }
  while(!small.empty() && !large.empty()) {
    const int32_t s = small.back(); small.pop_back();
    const int32_t l = large.back(); large.pop_back();
    prob[s] = (float)p[s];
    alias[s] = l;
    p[l] = (p[l] + p[s]) - 1.0;
    if(p[l] < 1.0) small.push_back(l); else large.push_back(l);
  }
  for(int32_t i : small) prob[i] = 1.0f;
  for(int32_t i : large) prob[i] = 1.0f;
}

template<class R>
static res_T flatten_impl
  (ssol_scene* scn, const BvhBuildParams& bvh_params, FlatScene<R>& out,
   bool for_draw)
{
  ssol_device* dev = scn->dev;
  out = FlatScene<R>();

  /* scene_check (src/ssol_scene.c:539-558) */
  if(!scn->sun) { dev->log_error("no sun attached.\n"); return RES_BAD_ARG; }
  const ssol_sun* sun = scn->sun;
  if(!sun->spectrum || sun->spectrum->wavelengths.empty()) {
    dev->log_error("sun's spectrum undefined.\n");
    return RES_BAD_ARG;
  }
  if(sun->dni <= 0) {
    dev->log_error("sun's DNI undefined.\n");
    return RES_BAD_ARG;
  }

  Interner in;
  /* Air: vacuum with the atmosphere's extinction (src/ssol_solver.c:1180) */
  ssol_medium air = SSOL_MEDIUM_VACUUM;
  if(scn->atmosphere) air.extinction = scn->atmosphere->extinction;
  out.air_medium = intern_medium(out, in, air);

  /* Sun */
  for(int c = 0; c < 3; ++c) out.sun_dir[c] = (R)sun->direction[c];
  double B[9];
  basis(sun->direction, B);
  for(int c = 0; c < 9; ++c) out.sun_basis[c] = (R)B[c];
  out.dni = sun->dni;
  switch(sun->kind) {
    case SUNK_DIRECTIONAL: out.sun_type = SUN_DIRAC; break;
    case SUNK_PILLBOX: {
      if(!(sun->half_angle > 0)) {
        dev->log_error("pillbox half angle undefined.\n");
        return RES_BAD_ARG;
      }
      out.sun_type = SUN_PILLBOX;
      const double s = std::sin(sun->half_angle);
      out.sun_param = (R)(s * s);
      break;
    }
    case SUNK_GAUSSIAN:
      if(!(sun->std_dev > 0)) return RES_BAD_ARG;
      out.sun_type = SUN_GAUSSIAN;
      out.sun_param = (R)sun->std_dev;
      break;
    case SUNK_BUIE:
      /* ranst_sun_dir_buie_setup accepts CSR in [1e-6, 0.849] */
      if(sun->csr < 1e-6 || sun->csr > 0.849) return RES_BAD_ARG;
      out.sun_type = SUN_BUIE;
      buie_state(sun->csr, out.buie);
      break;
  }
  /* Wavelength distribution (src/ssol_ranst_sun_wl.c:154-188) */
  out.wl_nodes = sun->spectrum->wavelengths;
  out.wl_pdf = sun->spectrum->intensities;
  {
    const size_t n = out.wl_nodes.size();
    out.wl_cdf.assign(n, 0.0);
    for(size_t i = 1; i < n; ++i)
      out.wl_cdf[i] = out.wl_cdf[i - 1] + 0.5 * (out.wl_pdf[i] + out.wl_pdf[i - 1])
                    * (out.wl_nodes[i] - out.wl_nodes[i - 1]);
    if(n > 1) {
      const double total = out.wl_cdf[n - 1];
      if(!(total > 0)) return RES_BAD_ARG;
      for(double& c : out.wl_cdf) c /= total;
      out.wl_cdf[n - 1] = 1.0;
    }
  }
  out.shader_wl = out.wl_nodes;

  /* Materials */
  std::map<const ssol_material*, int> mtl_index;
  bool bad_shader = false;
  auto material_id = [&](ssol_material* m) {
    auto it = mtl_index.find(m);
    if(it != mtl_index.end()) return it->second;
    DMaterial d;
    d.type = m->type;
    d.distrib = m->distrib == SSOL_MICROFACET_PILLBOX ? DISTRIB_PILLBOX
                                                      : DISTRIB_BECKMANN;
    d.in_medium = intern_medium(out, in, m->in_medium);
    d.out_medium = intern_medium(out, in, m->out_medium);
    d.slab_medium = intern_medium(out, in, m->slab_medium);
    d.thickness = m->thickness;
    d.table = (int32_t)out.shader_tab.size();
    if(!tabulate_shaders(out, m, dev)) bad_shader = true;
    const int id = (int)out.mtls.size();
    out.mtls.push_back(d);
    mtl_index.emplace(m, id);
    return id;
  };

  /* Receivers and sampled instances, in attach order */
  bool has_sampled = false, has_receiver = false;
  std::vector<PrimBox> boxes;
  /* Shading attributes (vertex normals, baked spatially varying shaders),
   * one record per triangle, kept only if some triangle needs one */
  std::vector<DTriShade<R>> tsh;
  bool need_tshade = false;
  std::map<std::pair<const ssol_material*, const ssol_shape*>, bool> varies;
  std::set<std::pair<const ssol_material*, const ssol_shape*>> punched_checked;
  std::vector<double> samp_area;
  for(size_t ii = 0; ii < scn->instances.size(); ++ii) {
    ssol_instance* inst = scn->instances[ii];
    const ssol_object* obj = inst->object;
    if(obj->shaded.empty()) out.meta.inst_mtl.push_back({-1, -1});
    int rcv_slot[2] = {-1, -1};
    for(int side = 0; side < 2; ++side) {
      if(inst->receiver_mask & (side == 0 ? SSOL_FRONT : SSOL_BACK)) {
        rcv_slot[side] = (int)out.meta.rcv.size();
        out.meta.rcv.push_back({inst, side});
      }
    }
    if(inst->receiver_mask) has_receiver = true;
    int sampled_idx = -1;
    if(inst->sample) {
      sampled_idx = (int)out.meta.sampled.size();
      out.meta.sampled.push_back(inst);
      out.meta.sampled_area += obj->rt_area;
      out.meta.sampled_area_proxy += obj->samp_area;
      has_sampled = true;
    }
    for(const ShadedShape& ss : obj->shaded) {
      const ssol_shape* shape = ss.shape;
      if(!shape->ready) continue;
      DShadedInst si;
      si.instance = (int32_t)ii;
      si.mtl[0] = material_id(ss.front);
      si.mtl[1] = material_id(ss.back);
      if(out.meta.inst_mtl.size() == ii) out.meta.inst_mtl.push_back({si.mtl[0], si.mtl[1]});
      si.receiver_mask = inst->receiver_mask & (SSOL_FRONT | SSOL_BACK);
      si.rcv_slot[0] = rcv_slot[0];
      si.rcv_slot[1] = rcv_slot[1];
      si.prim_base[0] = si.prim_base[1] = -1;
      si.sampled = sampled_idx;
      si.is_punched = shape->kind == SHAPE_PUNCHED;
      si.quadric = -1;
      si.virtual_mask = (ss.front->type == SSOL_MATERIAL_VIRTUAL ? 1 : 0)
                      | (ss.back->type == SSOL_MATERIAL_VIRTUAL ? 2 : 0);
      const int ntris = (int)(shape->ids.size() / 3);
      if(inst->per_primitive) {
        if(si.is_punched && !shape->grid_exact) {
          dev->log_error("per-primitive tallies on a punched surface need a "
                         "carving equal to its bounding rectangle.\n");
          return RES_BAD_ARG;
        }
        for(int side = 0; side < 2; ++side) {
          if(rcv_slot[side] < 0) continue;
          si.prim_base[side] = out.meta.nprim_slots;
          out.meta.prims.push_back({rcv_slot[side], shape,
                                    out.meta.nprim_slots, ntris});
          out.meta.nprim_slots += ntris;
        }
      }
      const int sinst_id = (int)out.sinsts.size();
      const double* T = inst->transform;

      if(shape->kind == SHAPE_MESH) {
        const int first_gid = (int)out.tris.size();
        /* Normals go through the inverse transpose of the instance
         * (src/ssol_material.c:632-646); a side's shaders are baked per vertex
         * when they vary over the shape */
        double Rn[9];
        normal_matrix(T, Rn);
        ssol_material* side_mtl[2] = {ss.front, ss.back};
        bool bake_side[2] = {false, false};
        for(int sd = 0; sd < 2; ++sd) {
          const auto key = std::make_pair((const ssol_material*)side_mtl[sd],
                                          (const ssol_shape*)shape);
          auto found = varies.find(key);
          if(found == varies.end()) {
            /* Probe the vertices of up to 8 triangles spread over the mesh
             * at both ends of the wavelength grid */
            const int nprobe = std::min(ntris, 8);
            std::vector<ssol_surface_fragment> fr((size_t)nprobe * 3);
            for(int i = 0; i < nprobe; ++i) {
              const int t = nprobe > 1 ? (int)((long long)i * (ntris - 1) / (nprobe - 1)) : 0;
              vertex_fragments(shape, t, T, Rn, sd, fr.data() + 3 * i);
            }
            const bool v = ntris > 0
              && (material_varies(side_mtl[sd], fr.data(), 3 * nprobe,
                                  out.shader_wl.front(), dev)
                  || material_varies(side_mtl[sd], fr.data(), 3 * nprobe,
                                     out.shader_wl.back(), dev));
            if(ntris > 0
            && (material_reads_dir(side_mtl[sd], fr.data(), 3 * nprobe,
                                   out.shader_wl.front(), dev)
                || material_reads_dir(side_mtl[sd], fr.data(), 3 * nprobe,
                                      out.shader_wl.back(), dev))) {
              dev->log_error("shaders that read the incoming direction are not "
                             "supported on the device.\n");
              return RES_BAD_ARG;
            }
            found = varies.emplace(key, v).first;
          }
          bake_side[sd] = found->second;
        }
        const bool has_n = !shape->nrm.empty();
        const bool attrs = has_n || bake_side[0] || bake_side[1];
        if(attrs) need_tshade = true;
        out.meta.meshes.push_back({inst, shape, first_gid, ntris,
                                   inst->sample ? (int)out.samp.size() : -1});
        for(int t = 0; t < ntris; ++t) {
          double v[3][3];
          float vf[3][3];
          for(int k = 0; k < 3; ++k) {
            const double p[3] = {shape->pos[shape->ids[t * 3 + k] * 3 + 0],
                                 shape->pos[shape->ids[t * 3 + k] * 3 + 1],
                                 shape->pos[shape->ids[t * 3 + k] * 3 + 2]};
            apply(T, p, v[k]);
            for(int c = 0; c < 3; ++c) vf[k][c] = (float)v[k][c];
          }
          DTri<R> tri;
          PrimBox box;
          for(int c = 0; c < 3; ++c) {
            /* Vertices go through FP32 like the reference's Star-3D scene */
            const R a = (R)vf[0][c], b = (R)vf[1][c], d = (R)vf[2][c];
            tri.v0[c] = a;
            tri.v1[c] = b;
            tri.v2[c] = d;
            box.lo[c] = std::min({(double)vf[0][c], (double)vf[1][c],
                                  (double)vf[2][c]});
            box.hi[c] = std::max({(double)vf[0][c], (double)vf[1][c],
                                  (double)vf[2][c]});
          }
          tri.sinst = sinst_id;
          tri.prim = t;
          tri.gid = first_gid + t;
          box.ref = primref_make(PRIM_TRIANGLE, (uint32_t)out.tris.size());
          out.tris.push_back(tri);
          boxes.push_back(box);
          DTriShade<R> ts;
          for(int c = 0; c < 9; ++c) ts.n[c] = R(0);
          ts.n[0] = std::numeric_limits<R>::quiet_NaN();
          ts.bake[0] = ts.bake[1] = -1;
          if(has_n) {
            for(int k = 0; k < 3; ++k) {
              const uint32_t id = shape->ids[(size_t)t * 3 + k];
              const double m[3] = {shape->nrm[id * 3 + 0], shape->nrm[id * 3 + 1],
                                   shape->nrm[id * 3 + 2]};
              for(int c = 0; c < 3; ++c)
                ts.n[3 * k + c] = (R)(Rn[c] * m[0] + Rn[3 + c] * m[1] + Rn[6 + c] * m[2]);
            }
          }
          for(int sd = 0; sd < 2 && attrs; ++sd) {
            if(!bake_side[sd]) continue;
            ssol_surface_fragment fr[3];
            vertex_fragments(shape, t, T, Rn, sd, fr);
            ts.bake[sd] = (int32_t)out.bake_tab.size();
            ssol_material* m = side_mtl[sd];
            for(int k = 0; k < 3; ++k)
              for(double wl : out.shader_wl) {
                double refl = 0, rough = 0;
                if(m->reflectivity) m->reflectivity(dev, m->buf, wl, &fr[k], &refl);
                if(m->roughness) m->roughness(dev, m->buf, wl, &fr[k], &rough);
                out.bake_tab.push_back((R)refl);
                out.bake_tab.push_back((R)rough);
              }
          }
          tsh.push_back(ts);
          if(inst->sample) {
            DSampTri<R> st;
            double n[3], e1[3], e2[3];
            for(int c = 0; c < 3; ++c) {
              e1[c] = (double)vf[1][c] - vf[0][c];
              e2[c] = (double)vf[2][c] - vf[0][c];
            }
            /* Star-3D front normal: e2 x e1 */
            n[0] = e2[1] * e1[2] - e2[2] * e1[1];
            n[1] = e2[2] * e1[0] - e2[0] * e1[2];
            n[2] = e2[0] * e1[1] - e2[1] * e1[0];
            const double len = std::sqrt(n[0]*n[0] + n[1]*n[1] + n[2]*n[2]);
            for(int c = 0; c < 3; ++c) {
              st.v0[c] = tri.v0[c];
              st.e1[c] = tri.v1[c] - tri.v0[c];
              st.e2[c] = tri.v2[c] - tri.v0[c];
              /* normalised in FP32 like f3_normalize */
              st.n[c] = (R)(float)(len > 0 ? n[c] / len : 0);
            }
            st.sinst = sinst_id;
            st.prim = t;
            st.gid = tri.gid;
            st.pad = 0;
            out.samp.push_back(st);
            samp_area.push_back(0.5 * len);
          }
        }
      } else {
        /* Punched: one analytic patch + flat sampling proxy */
        double M[12], W[12];
        compose(M, T, shape->quadric.transform);
        if(!invert(W, M)) {
          dev->log_error("singular instance transform.\n");
          return RES_BAD_ARG;
        }
        /* The device evaluates a punched surface's shaders from the
         * per-material table: shaders that vary over it, or read the
         * incoming direction, are refused */
        ssol_material* pside[2] = {ss.front, ss.back};
        for(int sd = 0; sd < 2; ++sd) {
          const auto key = std::make_pair((const ssol_material*)pside[sd],
                                          (const ssol_shape*)shape);
          if(punched_checked.count(key)) continue;
          punched_checked.insert(key);
          ssol_surface_fragment fr[9];
          const int nf = punched_fragments(shape, M, sd, fr);
          for(const double wl : {out.shader_wl.front(), out.shader_wl.back()}) {
            if(material_varies(pside[sd], fr, nf, wl, dev)) {
              dev->log_error("shaders that vary over a punched surface are not "
                             "supported on the device.\n");
              return RES_BAD_ARG;
            }
            if(material_reads_dir(pside[sd], fr, nf, wl, dev)) {
              dev->log_error("shaders that read the incoming direction are not "
                             "supported on the device.\n");
              return RES_BAD_ARG;
            }
          }
        }
        DQuadric<R> q;
        to_rows(q.w2l, W);
        to_rows(q.l2w, M);
        for(int c = 0; c < 4; ++c) q.param[c] = (R)shape->qparam[c];
        if(shape->quadric.type == SSOL_QUADRIC_HEMISPHERE)
          q.param[2] = (R)(shape->hemi_radius * shape->hemi_radius);
        q.type = shape->quadric.type;
        quadric_general(q);
        q.carve_lo[0] = (R)shape->carve_lo[0];
        q.carve_lo[1] = (R)shape->carve_lo[1];
        q.carve_hi[0] = (R)shape->carve_hi[0];
        q.carve_hi[1] = (R)shape->carve_hi[1];
        q.grid_delta = (R)shape->grid_delta;
        q.type = shape->quadric.type;
        q.sinst = sinst_id;
        q.grid_n[0] = (int32_t)shape->grid_n[0];
        q.grid_n[1] = (int32_t)shape->grid_n[1];
        /* A single AND rectangle equal to the AABB needs no polygon test */
        bool aabb_only = shape->carvings.size() == 1
          && shape->carvings[0].op == SSOL_AND
          && shape->carvings[0].xy.size() == 8;
        if(aabb_only) {
          const std::vector<double>& xy = shape->carvings[0].xy;
          for(int v = 0; v < 4 && aabb_only; ++v) {
            const double x = xy[2 * v], y = xy[2 * v + 1];
            aabb_only = (x == shape->carve_lo[0] || x == shape->carve_hi[0])
                     && (y == shape->carve_lo[1] || y == shape->carve_hi[1]);
          }
        }
        q.carve_first = (int32_t)out.carvings.size();
        q.carve_count = 0;
        if(!aabb_only) {
          for(const Carving& c : shape->carvings) {
            DCarving d;
            d.first = (int32_t)(out.carve_verts.size() / 2);
            d.count = (int32_t)(c.xy.size() / 2);
            d.op = c.op == SSOL_AND ? 0 : 1;
            d.pad = 0;
            for(double x : c.xy) out.carve_verts.push_back((R)x);
            out.carvings.push_back(d);
            ++q.carve_count;
          }
        }
        /* World box of the patch: local box corners through M */
        double zlo, zhi;
        quadric_z_range(shape, zlo, zhi);
        if(shape->quadric.type == SSOL_QUADRIC_HEMISPHERE) {
          zlo = 0;
          zhi = shape->qparam[0];
        }
        PrimBox box;
        for(int c = 0; c < 3; ++c) {
          box.lo[c] = std::numeric_limits<double>::max();
          box.hi[c] = -std::numeric_limits<double>::max();
        }
        for(int corner = 0; corner < 8; ++corner) {
          const double p[3] = {
            (corner & 1) ? shape->carve_hi[0] : shape->carve_lo[0],
            (corner & 2) ? shape->carve_hi[1] : shape->carve_lo[1],
            (corner & 4) ? zhi : zlo};
          double w[3];
          apply(M, p, w);
          for(int c = 0; c < 3; ++c) {
            box.lo[c] = std::min(box.lo[c], w[c]);
            box.hi[c] = std::max(box.hi[c], w[c]);
          }
        }
        double ext = 0;
        for(int c = 0; c < 3; ++c) ext = std::max(ext, box.hi[c] - box.lo[c]);
        for(int c = 0; c < 3; ++c) {
          const double pad = 1e-5 * ext + 1e-6 * std::max(std::fabs(box.lo[c]),
                                                          std::fabs(box.hi[c]));
          box.lo[c] -= pad;
          box.hi[c] += pad;
        }
        si.quadric = (int32_t)out.quads.size();
        box.ref = primref_make(PRIM_QUADRIC, (uint32_t)out.quads.size());
        out.quads.push_back(q);
        boxes.push_back(box);

        if(inst->sample) {
          for(size_t t = 0; t + 2 < shape->samp_ids.size(); t += 3) {
            float vf[3][3];
            for(int k = 0; k < 3; ++k) {
              const uint32_t id = shape->samp_ids[t + k];
              const double p[3] = {(double)(float)shape->samp_xy[id * 2],
                                   (double)(float)shape->samp_xy[id * 2 + 1],
                                   0.0};
              double w[3];
              apply(M, p, w);
              for(int c = 0; c < 3; ++c) vf[k][c] = (float)w[c];
            }
            DSampTri<R> st;
            double n[3], e1[3], e2[3];
            for(int c = 0; c < 3; ++c) {
              e1[c] = (double)vf[1][c] - vf[0][c];
              e2[c] = (double)vf[2][c] - vf[0][c];
            }
            n[0] = e2[1] * e1[2] - e2[2] * e1[1];
            n[1] = e2[2] * e1[0] - e2[0] * e1[2];
            n[2] = e2[0] * e1[1] - e2[1] * e1[0];
            const double len = std::sqrt(n[0]*n[0] + n[1]*n[1] + n[2]*n[2]);
            for(int c = 0; c < 3; ++c) {
              st.v0[c] = (R)vf[0][c];
              st.e1[c] = (R)((R)vf[1][c] - (R)vf[0][c]);
              st.e2[c] = (R)((R)vf[2][c] - (R)vf[0][c]);
              st.n[c] = (R)(float)(len > 0 ? n[c] / len : 0);
            }
            st.sinst = sinst_id;
            st.prim = (int32_t)(t / 3);
            st.gid = -1;
            st.pad = 0;
            out.samp.push_back(st);
            samp_area.push_back(0.5 * len);
          }
        }
      }
      out.sinsts.push_back(si);
    }
  }
  if(bad_shader) return RES_BAD_ARG;
  if(!for_draw && (!has_sampled || out.samp.empty())) {
    dev->log_error("No solstice instance to sample.\n");
    return RES_BAD_ARG;
  }
  if(!for_draw && !has_receiver) dev->log_warning("No receiver is defined.\n");

  build_alias(samp_area, out.alias_prob, out.alias_idx);
  if(need_tshade) out.tshade = std::move(tsh);
  /* Features the kernel variant must handle */
  out.meta.features = 0;
  if(!out.quads.empty()) out.meta.features |= FEAT_QUADRIC;
  for(const DMaterial& d : out.mtls)
    if(d.type == MTL_DIELECTRIC || d.type == MTL_THIN_DIELECTRIC)
      out.meta.features |= FEAT_DIELECTRIC;
  if(!out.tshade.empty()) out.meta.features |= FEAT_ATTRIBUTES;

  /* Bounding box of the ray-traced geometry (src/ssol_solver.c:563-570 uses
   * the scene view's box for the tracked segments to and from infinity) */
  for(int c = 0; c < 3; ++c) {
    out.meta.aabb_lo[c] = boxes.empty() ? 0.0 : DBL_MAX;
    out.meta.aabb_hi[c] = boxes.empty() ? 0.0 : -DBL_MAX;
  }
  for(const PrimBox& b : boxes)
    for(int c = 0; c < 3; ++c) {
      out.meta.aabb_lo[c] = std::min(out.meta.aabb_lo[c], b.lo[c]);
      out.meta.aabb_hi[c] = std::max(out.meta.aabb_hi[c], b.hi[c]);
    }
  if(bvh_params.device && boxes.size() >= 2) {
    const size_t n = boxes.size();
    out.device_bvh = true;
    out.prim_box.resize(6 * n);
    out.prim_ref.resize(n);
    for(size_t i = 0; i < n; ++i) {
      round_box_outward<R>(boxes[i], out.prim_box.data() + 6 * i);
      out.prim_ref[i] = boxes[i].ref;
    }
    out.bvh = BvhResult();
    out.nodes.assign(n - 1, DNode<R>());
    return RES_OK;
  }
  build_bvh(boxes, bvh_params, out.bvh);
  out.nodes = bvh_nodes<R>(out.bvh);
  return RES_OK;
}

res_T flatten_scene
  (ssol_scene* scn, const BvhBuildParams& bvh, FlatScene<float>& out,
   bool for_draw)
{ return flatten_impl<float>(scn, bvh, out, for_draw); }

res_T flatten_scene
  (ssol_scene* scn, const BvhBuildParams& bvh, FlatScene<double>& out,
   bool for_draw)
{ return flatten_impl<double>(scn, bvh, out, for_draw); }

} /* namespace ssolb */
