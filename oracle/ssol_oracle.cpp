/*
 * ssol_oracle.cpp - CPU oracle of the ssol_solve realisation loop.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker for the B200 library:
 * tests/, __graft_entry__.smoke() and bench.py's CPU baseline may load it;
 * the product never does. It is an independent C++17 + OpenMP restatement of
 * the reference algorithm, exporting the same C API (include/ssol.h,
 * include/ssp.h) so that one scene description drives both libraries.
 *
 * Followed files (reference paths relative to the reference tree):
 *   src/ssol_solver.c:148-1361      point, init, shade, tallies, roulette,
 *                                   loop, OpenMP schedule, per-thread merge
 *   src/ssol_scene.c:347-558        views, sampled areas, hit filter, checks
 *   src/ssol_shape.c:236-1494       quadric heights, roots, gradients,
 *                                   projection, grid discretisation
 *   src/ssol_estimator_c.h:33-126   deferred mc_data accumulators
 *   src/ssol_estimator.c:112-268    read-out formulas
 *   src/ssol_mc_receiver.c:32-173   per receiver / per primitive read-out
 *   src/ssol_ranst_sun_dir.c        sun direction samplers
 *   src/ssol_ranst_sun_wl.c         wavelength sampler
 *   src/ssol_spectrum.c:57-89       spectrum interpolation
 *   src/ssol_material.c:82-736      BSDF choice, media rules
 * Third-party arithmetic that the reference takes from Star-SF 0.6 / Star-SP
 * 0.12 / Star-3D 0.8 (not in the reference tree) is restated from published
 * methods, with the same choices as the B200 library so that both consume
 * identical random numbers: Philox4x32-10 streams keyed (seed, realisation),
 * Vose alias sampling of the sampled triangles, the sqrt-parameterised
 * uniform triangle point, a Duff et al. orthonormal basis, Fresnel
 * equations, Beckmann / pillbox microfacet normal sampling (Walter et al.
 * 2007), Malley cosine sampling and the thin-slab multiple-reflection sums.
 *
 * Parity pins: tests/test_oracle_pins.py checks this oracle against the
 * closed-form answers of the reference's own solver tests
 * (src/test_ssol_solver1.c, 4, 5, 6, 9, 10, 12, by_receiver_integration).
 */
#include "../include/ssol.h"
#include "../include/ssp.h"

#include <omp.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cfloat>
#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <vector>

#define API extern "C" __attribute__((visibility("default")))

/*******************************************************************************
 * Philox4x32-10 (Salmon et al., SC'11)
 ******************************************************************************/
namespace {

struct Block { uint32_t x[4]; };

Block philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
             uint32_t k0, uint32_t k1)
{
  for(int round = 0; round < 10; ++round) {
    if(round > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    const uint32_t n1 = (uint32_t)p1;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    const uint32_t n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
  }
  Block b = {{c0, c1, c2, c3}};
  return b;
}

inline double unif(uint32_t x) { return (double)(x >> 8) * (1.0 / 16777216.0); }

enum { DOM_PRIMARY = 0, DOM_SCATTER = 1, DOM_ROULETTE = 2, DOM_RETRY = 3 };
const uint32_t DOM_HOST = 0xffffffffu;

struct PathRng {
  uint64_t id;
  uint64_t seed;
  Block get(uint32_t event, uint32_t domain) const
  {
    return philox((uint32_t)id, (uint32_t)(id >> 32), event, domain,
                  (uint32_t)seed, (uint32_t)(seed >> 32));
  }
};

/*******************************************************************************
 * Small 3D helpers (double)
 ******************************************************************************/
struct V { double x, y, z; };
inline V v3(double x, double y, double z) { V r = {x, y, z}; return r; }
inline V operator+(V a, V b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V operator-(V a, V b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V operator-(V a) { return v3(-a.x, -a.y, -a.z); }
inline V operator*(V a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
inline double dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V cross(V a, V b)
{ return v3(a.y*b.z - a.z*b.y, a.z*b.x - a.x*b.z, a.x*b.y - a.y*b.x); }
inline V unit(V a)
{ const double l = std::sqrt(dot(a, a)); return l > 0 ? a * (1 / l) : a; }

void onb(V n, V& b1, V& b2)
{
  const double s = n.z >= 0 ? 1.0 : -1.0;
  const double a = -1.0 / (s + n.z);
  const double b = n.x * n.y * a;
  b1 = v3(1 + s * n.x * n.x * a, s * b, -s * n.x);
  b2 = v3(b, s + n.y * n.y * a, -n.y);
}

/* Affine 3x4, column major (ssol convention) */
struct Affine { double m[12]; };
V xpoint(const Affine& a, V p)
{
  return v3(a.m[0]*p.x + a.m[3]*p.y + a.m[6]*p.z + a.m[9],
            a.m[1]*p.x + a.m[4]*p.y + a.m[7]*p.z + a.m[10],
            a.m[2]*p.x + a.m[5]*p.y + a.m[8]*p.z + a.m[11]);
}
V xvec(const Affine& a, V p)
{
  return v3(a.m[0]*p.x + a.m[3]*p.y + a.m[6]*p.z,
            a.m[1]*p.x + a.m[4]*p.y + a.m[7]*p.z,
            a.m[2]*p.x + a.m[5]*p.y + a.m[8]*p.z);
}
/* Transpose of the linear part applied to p */
V xvec_t(const Affine& a, V p)
{
  return v3(a.m[0]*p.x + a.m[1]*p.y + a.m[2]*p.z,
            a.m[3]*p.x + a.m[4]*p.y + a.m[5]*p.z,
            a.m[6]*p.x + a.m[7]*p.y + a.m[8]*p.z);
}
Affine compose(const Affine& a, const Affine& b)
{
  Affine r;
  for(int c = 0; c < 3; ++c) {
    const V col = xvec(a, v3(b.m[c*3], b.m[c*3+1], b.m[c*3+2]));
    r.m[c*3] = col.x; r.m[c*3+1] = col.y; r.m[c*3+2] = col.z;
  }
  const V t = xpoint(a, v3(b.m[9], b.m[10], b.m[11]));
  r.m[9] = t.x; r.m[10] = t.y; r.m[11] = t.z;
  return r;
}
bool inverse(const Affine& a, Affine& r)
{
  const V c0 = v3(a.m[0], a.m[1], a.m[2]);
  const V c1 = v3(a.m[3], a.m[4], a.m[5]);
  const V c2 = v3(a.m[6], a.m[7], a.m[8]);
  const V r0 = cross(c1, c2), r1 = cross(c2, c0), r2 = cross(c0, c1);
  const double det = dot(c0, r0);
  if(det == 0) return false;
  const double inv = 1 / det;
  /* rows of the inverse are r0, r1, r2 / det */
  r.m[0] = r0.x * inv; r.m[3] = r0.y * inv; r.m[6] = r0.z * inv;
  r.m[1] = r1.x * inv; r.m[4] = r1.y * inv; r.m[7] = r1.z * inv;
  r.m[2] = r2.x * inv; r.m[5] = r2.y * inv; r.m[8] = r2.z * inv;
  const V t = xvec(r, v3(a.m[9], a.m[10], a.m[11]));
  r.m[9] = -t.x; r.m[10] = -t.y; r.m[11] = -t.z;
  return true;
}

struct Ref {
  std::atomic<int> n{1};
  void get() { n.fetch_add(1); }
  bool put() { return n.fetch_sub(1) == 1; }
};

} /* namespace */

/*******************************************************************************
 * Object model
 ******************************************************************************/
struct ssp_rng { Ref ref; ssp_rng_type type; uint64_t seed = 0, pos = 0; };
struct ssol_device { Ref ref; int verbose = 0; unsigned nthreads = 1; };
struct ssol_spectrum {
  Ref ref; ssol_device* dev;
  std::vector<double> wl, val;
  uint64_t sum[2] = {0, 0};
};
struct OCarving { int op; std::vector<double> xy; };
struct ssol_shape {
  Ref ref; ssol_device* dev; bool punched; bool ready = false;
  std::vector<float> pos; /* RT positions, shape space */
  std::vector<float> nrm, uv; /* optional vertex normals and texcoords */
  std::vector<unsigned> ids;
  double rt_area = 0, samp_area = 0;
  /* punched */
  ssol_quadric quad{};
  double q[4] = {0, 0, 0, 0};
  std::vector<OCarving> carv;
  double lo[2] = {0, 0}, hi[2] = {0, 0};
  double disk2 = 0;
  std::vector<double> flat; /* local xy per vertex */
  size_t gnx = 0, gny = 0;
  double gdelta = 0;
  bool gexact = false;
};
struct ssol_param_buffer {
  Ref ref; ssol_device* dev; std::vector<unsigned char> mem;
  size_t cap = 0, used = 0;
};
struct ssol_material {
  Ref ref; ssol_device* dev; ssol_material_type type;
  ssol_shader_getter_T refl = nullptr, rough = nullptr, normal = nullptr;
  ssol_microfacet_distribution distrib = SSOL_MICROFACET_BECKMANN;
  ssol_medium out = SSOL_MEDIUM_VACUUM__, in = SSOL_MEDIUM_VACUUM__;
  ssol_medium slab = SSOL_MEDIUM_VACUUM__;
  double thickness = 0;
  ssol_param_buffer* buf = nullptr;
};
struct OShaded { ssol_shape* shape; ssol_material* front; ssol_material* back; };
struct ssol_object {
  Ref ref; ssol_device* dev; std::vector<OShaded> shaded;
  double rt_area = 0, samp_area = 0;
};
struct ssol_instance {
  Ref ref; ssol_device* dev; ssol_object* obj; uint32_t id;
  Affine xf = {{1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0}};
  int mask = 0, per_prim = 0, sample = 1;
};
struct ssol_sun {
  Ref ref; ssol_device* dev; int kind; double dir[3] = {0, 0, 0};
  double dni = 0; ssol_spectrum* spec = nullptr; double param = 0;
  ssol_scene* scn = nullptr;
};
struct ssol_atmosphere {
  Ref ref; ssol_device* dev; ssol_data ext = SSOL_DATA_NULL__;
  ssol_scene* scn = nullptr;
};
struct ssol_scene {
  Ref ref; ssol_device* dev; std::vector<ssol_instance*> inst;
  ssol_sun* sun = nullptr; ssol_atmosphere* atm = nullptr;
};

/* Deferred MC accumulator (src/ssol_estimator_c.h:33-126) */
struct McData {
  size_t ireal = SIZE_MAX;
  double tmp = 0, w = 0, w2 = 0;
  void flush() { w += tmp; w2 += tmp * tmp; tmp = 0; }
  void add(size_t i, double x)
  {
    if(i != ireal) { flush(); ireal = i; }
    tmp += x;
  }
  void factor(size_t i, double f) { if(i == ireal) tmp *= f; }
  void accum(McData& src) { flush(); src.flush(); w += src.w; w2 += src.w2; }
};
struct McRcv1 {
  McData q[10];
  std::map<const ssol_shape*, std::map<unsigned, std::vector<McData>>> prims;
};
struct McRcv { McRcv1 side[2]; };
struct McSamp {
  McData cos, shadow;
  size_t nb = 0;
  std::map<const ssol_instance*, McRcv> rcv;
};

struct OPath { ssol_path_type type; std::vector<ssol_path_vertex> v; };

struct ssol_estimator {
  Ref ref; ssol_device* dev;
  size_t nreal = 0, nfail = 0;
  McData g[6];
  std::map<const ssol_instance*, McRcv> rcv;
  std::map<const ssol_instance*, McSamp> samp;
  double sampled_area = 0;
  ssp_rng* rng = nullptr;
  std::vector<OPath> paths;
};

namespace {

uint32_t next_id() { static std::atomic<uint32_t> n{1}; return n++; }

bool data_ceq(const ssol_data& a, const ssol_data& b)
{
  if(a.type != b.type) return false;
  if(a.type == SSOL_DATA_REAL) return a.value.real == b.value.real;
  return a.value.spectrum->sum[0] == b.value.spectrum->sum[0]
      && a.value.spectrum->sum[1] == b.value.spectrum->sum[1];
}
bool media_ceq(const ssol_medium& a, const ssol_medium& b)
{ return data_ceq(a.refractive_index, b.refractive_index)
      && data_ceq(a.extinction, b.extinction); }

double interp(const std::vector<double>& w, const std::vector<double>& v,
              double x)
{
  const size_t i = (size_t)(std::lower_bound(w.begin(), w.end(), x) - w.begin());
  if(i == w.size()) return v.back();
  if(i == 0) return v[0];
  const double s = (v[i] - v[i - 1]) / (w[i] - w[i - 1]);
  return v[i - 1] + (x - w[i - 1]) * s;
}

double data_value(const ssol_data& d, double wl)
{
  if(d.type == SSOL_DATA_REAL) return d.value.real;
  return interp(d.value.spectrum->wl, d.value.spectrum->val, wl);
}

uint64_t fnv(const void* p, size_t n)
{
  const unsigned char* c = (const unsigned char*)p;
  uint64_t h = 0xcbf29ce484222325ull;
  for(size_t i = 0; i < n; ++i) { h ^= c[i]; h *= 0x100000001b3ull; }
  return h;
}

bool spectrum_ok(const ssol_spectrum* s, double lo, double hi)
{
  if(!s || s->val.empty() || s->val.size() != s->wl.size()) return false;
  double cur = 0;
  for(size_t i = 0; i < s->val.size(); ++i) {
    if(s->val[i] < lo || s->val[i] > hi || s->wl[i] <= 0 || s->wl[i] <= cur)
      return false;
    cur = s->wl[i];
  }
  return true;
}

bool medium_ok(const ssol_medium* m)
{
  if(!m) return false;
  if(m->extinction.type == SSOL_DATA_REAL) {
    if(m->extinction.value.real < 0) return false;
  } else if(!spectrum_ok(m->extinction.value.spectrum, 0, DBL_MAX)) return false;
  if(m->refractive_index.type == SSOL_DATA_REAL) {
    if(m->refractive_index.value.real <= 0) return false;
  } else if(!spectrum_ok(m->refractive_index.value.spectrum, DBL_EPSILON,
                         DBL_MAX)) return false;
  return true;
}

/* Quadric heights and gradients in the local frame */
double qz(int t, const double* q, double x, double y)
{
  switch(t) {
    case SSOL_QUADRIC_PARABOL: return (x * x + y * y) * q[1];
    case SSOL_QUADRIC_PARABOL2F: return x * x * q[0] + y * y * q[1];
    case SSOL_QUADRIC_HYPERBOL:
      return q[1] * std::sqrt(1 + (x * x + y * y) * q[3]) - q[1];
    case SSOL_QUADRIC_PARABOLIC_CYLINDER: return y * y * q[1];
    case SSOL_QUADRIC_HEMISPHERE: {
      const double z2 = q[1] - (x * x + y * y);
      return z2 > 0 ? q[0] - std::sqrt(z2) : q[0];
    }
    default: return 0;
  }
}

V qgrad(int t, const double* q, V p)
{
  switch(t) {
    case SSOL_QUADRIC_PARABOL: return v3(-p.x, -p.y, 2 * q[0]);
    case SSOL_QUADRIC_PARABOL2F: return v3(-p.x * 4 * q[0], -p.y * 4 * q[1], 2);
    case SSOL_QUADRIC_HYPERBOL: return v3(p.x, p.y, -(p.z + q[1]) * q[2]);
    case SSOL_QUADRIC_PARABOLIC_CYLINDER: return v3(0, -p.y, 2 * q[0]);
    case SSOL_QUADRIC_HEMISPHERE: return v3(-p.x, -p.y, q[0] - p.z);
    default: return v3(0, 0, 1);
  }
}

void qcoef(int t, const double* q, V o, V d, double& a, double& b, double& c)
{
  switch(t) {
    case SSOL_QUADRIC_PLANE: a = 0; b = d.z; c = o.z; break;
    case SSOL_QUADRIC_PARABOL:
      a = d.x * d.x + d.y * d.y;
      b = 2 * o.x * d.x + 2 * o.y * d.y - 4 * q[0] * d.z;
      c = o.x * o.x + o.y * o.y - 4 * q[0] * o.z;
      break;
    case SSOL_QUADRIC_PARABOL2F:
      a = d.x * d.x * q[0] + d.y * d.y * q[1];
      b = 2 * o.x * d.x * q[0] + 2 * o.y * d.y * q[1] - d.z;
      c = o.x * o.x * q[0] + o.y * o.y * q[1] - o.z;
      break;
    case SSOL_QUADRIC_HYPERBOL: {
      const double b2 = q[1] * q[1], b2a2 = b2 * q[3], zz = o.z + q[1];
      a = b2a2 * (d.x * d.x + d.y * d.y) - d.z * d.z;
      b = 2 * (b2a2 * (o.x * d.x + o.y * d.y) - zz * d.z);
      c = b2a2 * (o.x * o.x + o.y * o.y) + b2 - zz * zz;
      break;
    }
    case SSOL_QUADRIC_PARABOLIC_CYLINDER:
      a = d.y * d.y;
      b = 2 * o.y * d.y - 4 * q[0] * d.z;
      c = o.y * o.y - 4 * q[0] * o.z;
      break;
    case SSOL_QUADRIC_HEMISPHERE: {
      const double z0 = -q[0];
      a = dot(d, d);
      b = 2 * (dot(o, d) + z0 * d.z);
      c = dot(o, o) - q[1] + 2 * z0 * o.z + z0 * z0;
      break;
    }
    default: a = b = c = 0;
  }
}

bool point_in_polygon(const std::vector<double>& xy, double x, double y)
{
  const size_t n = xy.size() / 2;
  bool in = false;
  for(size_t i = 0, j = n - 1; i < n; j = i++) {
    const double xi = xy[2*i], yi = xy[2*i+1], xj = xy[2*j], yj = xy[2*j+1];
    if(((yi > y) != (yj > y)) && (x < (xj - xi) * (y - yi) / (yj - yi) + xi))
      in = !in;
  }
  return in;
}

bool in_domain(const ssol_shape* s, double x, double y)
{
  if(s->quad.type == SSOL_QUADRIC_HEMISPHERE && x * x + y * y > s->disk2)
    return false;
  if(x < s->lo[0] || x > s->hi[0] || y < s->lo[1] || y > s->hi[1])
    return false;
  for(const OCarving& c : s->carv) {
    const bool in = point_in_polygon(c.xy, x, y);
    if(c.op == SSOL_AND ? !in : in) return false;
  }
  return true;
}

/* Sutherland-Hodgman style clipping of a convex polygon by a half-plane */
typedef std::vector<std::pair<double, double>> Poly;
double orient(const std::pair<double,double>& a, const std::pair<double,double>& b,
              const std::pair<double,double>& p)
{ return (b.first - a.first) * (p.second - a.second)
       - (b.second - a.second) * (p.first - a.first); }
double poly_area(const Poly& p)
{
  double s = 0;
  for(size_t i = 0; i < p.size(); ++i) {
    const size_t j = (i + 1) % p.size();
    s += p[i].first * p[j].second - p[j].first * p[i].second;
  }
  return 0.5 * s;
}
Poly half_clip(const Poly& in, const std::pair<double,double>& a,
               const std::pair<double,double>& b, double sign)
{
  Poly out;
  for(size_t i = 0; i < in.size(); ++i) {
    const auto& p = in[i];
    const auto& q = in[(i + 1) % in.size()];
    const double sp = sign * orient(a, b, p), sq = sign * orient(a, b, q);
    if(sp >= 0) out.push_back(p);
    if((sp >= 0) != (sq >= 0)) {
      const double t = sp / (sp - sq);
      out.push_back({p.first + t * (q.first - p.first),
                     p.second + t * (q.second - p.second)});
    }
  }
  return out;
}

} /* namespace */

/*******************************************************************************
 * API: device, rng, spectrum, data
 ******************************************************************************/
API res_T ssol_device_create(logger*, mem_allocator*, const unsigned nthreads,
                             const int verbose, ssol_device** out)
{
  if(!nthreads || !out) return RES_BAD_ARG;
  ssol_device* d = new ssol_device();
  d->verbose = verbose;
  d->nthreads = std::min<unsigned>(nthreads, (unsigned)omp_get_num_procs());
  *out = d;
  return RES_OK;
}
API res_T ssol_device_ref_get(ssol_device* d)
{ if(!d) return RES_BAD_ARG; d->ref.get(); return RES_OK; }
API res_T ssol_device_ref_put(ssol_device* d)
{ if(!d) return RES_BAD_ARG; if(d->ref.put()) delete d; return RES_OK; }

API res_T ssp_rng_create(mem_allocator*, const ssp_rng_type t, ssp_rng** out)
{
  if(!out || (unsigned)t >= SSP_RNG_TYPES_COUNT__) return RES_BAD_ARG;
  ssp_rng* r = new ssp_rng();
  r->type = t;
  *out = r;
  return RES_OK;
}
API res_T ssp_rng_ref_get(ssp_rng* r)
{ if(!r) return RES_BAD_ARG; r->ref.get(); return RES_OK; }
API res_T ssp_rng_ref_put(ssp_rng* r)
{ if(!r) return RES_BAD_ARG; if(r->ref.put()) delete r; return RES_OK; }
API res_T ssp_rng_get_type(const ssp_rng* r, ssp_rng_type* t)
{ if(!r || !t) return RES_BAD_ARG; *t = r->type; return RES_OK; }
API res_T ssp_rng_set(ssp_rng* r, const uint64_t seed)
{ if(!r) return RES_BAD_ARG; r->seed = seed; r->pos = 0; return RES_OK; }
API uint64_t ssp_rng_get(ssp_rng* r)
{
  const Block b = philox((uint32_t)r->pos, (uint32_t)(r->pos >> 32), 0,
                         DOM_HOST, (uint32_t)r->seed,
                         (uint32_t)(r->seed >> 32));
  ++r->pos;
  return ((uint64_t)b.x[0] << 32) | b.x[1];
}
API double ssp_rng_canonical(ssp_rng* r)
{ return (double)(ssp_rng_get(r) >> 11) * (1.0 / 9007199254740992.0); }
API float ssp_rng_canonical_float(ssp_rng* r)
{ return (float)(ssp_rng_get(r) >> 40) * (1.0f / 16777216.0f); }
API res_T ssp_rng_discard(ssp_rng* r, uint64_t n)
{ if(!r) return RES_BAD_ARG; r->pos += n; return RES_OK; }
API res_T ssp_rng_write(const ssp_rng* r, FILE* f)
{
  if(!r || !f) return RES_BAD_ARG;
  return fprintf(f, "philox4x32-10 %d %" PRIu64 " %" PRIu64 "\n", (int)r->type,
                 r->seed, r->pos) < 0 ? RES_IO_ERR : RES_OK;
}
API res_T ssp_rng_read(ssp_rng* r, FILE* f)
{
  if(!r || !f) return RES_BAD_ARG;
  int t; uint64_t s, p;
  if(fscanf(f, " philox4x32-10 %d %" SCNu64 " %" SCNu64, &t, &s, &p) != 3)
    return RES_IO_ERR;
  r->type = (ssp_rng_type)t; r->seed = s; r->pos = p;
  return RES_OK;
}

API res_T ssol_spectrum_create(ssol_device* d, ssol_spectrum** out)
{
  if(!d || !out) return RES_BAD_ARG;
  ssol_spectrum* s = new ssol_spectrum();
  s->dev = d; d->ref.get();
  *out = s;
  return RES_OK;
}
API res_T ssol_spectrum_ref_get(ssol_spectrum* s)
{ if(!s) return RES_BAD_ARG; s->ref.get(); return RES_OK; }
API res_T ssol_spectrum_ref_put(ssol_spectrum* s)
{
  if(!s) return RES_BAD_ARG;
  if(s->ref.put()) { ssol_device* d = s->dev; delete s; ssol_device_ref_put(d); }
  return RES_OK;
}
API res_T ssol_spectrum_setup(ssol_spectrum* s,
  void (*get)(const size_t, double*, double*, void*), const size_t n, void* ctx)
{
  if(!s || !n || !get) return RES_BAD_ARG;
  std::vector<double> w(n), v(n);
  double cur = 0;
  for(size_t i = 0; i < n; ++i) {
    get(i, &w[i], &v[i], ctx);
    if(w[i] <= cur || v[i] < 0) {
      s->wl.clear(); s->val.clear(); s->sum[0] = s->sum[1] = 0;
      return RES_BAD_ARG;
    }
    cur = w[i];
  }
  s->wl = w; s->val = v;
  s->sum[0] = fnv(w.data(), n * sizeof(double));
  s->sum[1] = fnv(v.data(), n * sizeof(double));
  return RES_OK;
}

API ssol_data* ssol_data_clear(ssol_data* d)
{
  if(d->type == SSOL_DATA_SPECTRUM) {
    ssol_spectrum_ref_put(d->value.spectrum);
    *d = SSOL_DATA_NULL;
  }
  return d;
}
API ssol_data* ssol_data_set_real(ssol_data* d, const double r)
{ ssol_data_clear(d); d->type = SSOL_DATA_REAL; d->value.real = r; return d; }
API ssol_data* ssol_data_set_spectrum(ssol_data* d, ssol_spectrum* s)
{
  if(d->type == SSOL_DATA_SPECTRUM && d->value.spectrum == s) return d;
  ssol_data_clear(d);
  d->type = SSOL_DATA_SPECTRUM; d->value.spectrum = s; s->ref.get();
  return d;
}
API ssol_data* ssol_data_copy(ssol_data* dst, const ssol_data* src)
{
  if(dst == src) return dst;
  if(src->type == SSOL_DATA_SPECTRUM) ssol_data_set_spectrum(dst, src->value.spectrum);
  else ssol_data_set_real(dst, src->value.real);
  return dst;
}
API double ssol_data_get_value(const ssol_data* d, const double wl)
{ return data_value(*d, wl); }

/*******************************************************************************
 * API: shapes
 ******************************************************************************/
static double tri_area_f(const std::vector<float>& p, const std::vector<unsigned>& ids)
{
  double a = 0;
  for(size_t t = 0; t + 2 < ids.size(); t += 3) {
    const V v0 = v3(p[ids[t]*3], p[ids[t]*3+1], p[ids[t]*3+2]);
    const V v1 = v3(p[ids[t+1]*3], p[ids[t+1]*3+1], p[ids[t+1]*3+2]);
    const V v2 = v3(p[ids[t+2]*3], p[ids[t+2]*3+1], p[ids[t+2]*3+2]);
    const V n = cross(v1 - v0, v2 - v0);
    a += std::sqrt(dot(n, n));
  }
  return 0.5 * a;
}

static res_T shape_new(ssol_device* d, ssol_shape** out, bool punched)
{
  if(!d || !out) return RES_BAD_ARG;
  ssol_shape* s = new ssol_shape();
  s->dev = d; d->ref.get(); s->punched = punched;
  *out = s;
  return RES_OK;
}
API res_T ssol_shape_create_mesh(ssol_device* d, ssol_shape** o)
{ return shape_new(d, o, false); }
API res_T ssol_shape_create_punched_surface(ssol_device* d, ssol_shape** o)
{ return shape_new(d, o, true); }
API res_T ssol_shape_ref_get(ssol_shape* s)
{ if(!s) return RES_BAD_ARG; s->ref.get(); return RES_OK; }
API res_T ssol_shape_ref_put(ssol_shape* s)
{
  if(!s) return RES_BAD_ARG;
  if(s->ref.put()) { ssol_device* d = s->dev; delete s; ssol_device_ref_put(d); }
  return RES_OK;
}
API res_T ssol_shape_get_vertices_count(const ssol_shape* s, unsigned* n)
{ if(!s || !n) return RES_BAD_ARG; *n = (unsigned)(s->pos.size() / 3); return RES_OK; }
API res_T ssol_shape_get_triangles_count(const ssol_shape* s, unsigned* n)
{ if(!s || !n) return RES_BAD_ARG; *n = (unsigned)(s->ids.size() / 3); return RES_OK; }
API res_T ssol_shape_get_triangle_indices(const ssol_shape* s, const unsigned i,
                                          unsigned ids[3])
{
  if(!s || !ids || i >= s->ids.size() / 3) return RES_BAD_ARG;
  for(int k = 0; k < 3; ++k) ids[k] = s->ids[i * 3 + k];
  return RES_OK;
}
API res_T ssol_shape_get_vertex_attrib(const ssol_shape* s, const unsigned iv,
  const ssol_attrib_usage u, double v[])
{
  if(!s || (unsigned)u >= SSOL_ATTRIBS_COUNT__ || !v || u != SSOL_POSITION
  || iv >= s->pos.size() / 3)
    return RES_BAD_ARG;
  for(int c = 0; c < 3; ++c) v[c] = s->pos[iv * 3 + c];
  if(s->punched) {
    Affine a; std::memcpy(a.m, s->quad.transform, sizeof(a.m));
    const V w = xpoint(a, v3(v[0], v[1], v[2]));
    v[0] = w.x; v[1] = w.y; v[2] = w.z;
  }
  return RES_OK;
}

API res_T ssol_mesh_setup(ssol_shape* s, const unsigned ntris,
  void (*get_ids)(const unsigned, unsigned[3], void*), const unsigned nverts,
  const ssol_vertex_data attribs[], const unsigned nattribs, void* data)
{
  if(!s || s->punched || !get_ids || !ntris || !nverts || !attribs || !nattribs)
    return RES_BAD_ARG;
  if(nattribs > SSOL_ATTRIBS_COUNT__) return RES_MEM_ERR;
  const ssol_vertex_data* pos = nullptr;
  const ssol_vertex_data* nrm = nullptr;
  const ssol_vertex_data* tex = nullptr;
  for(unsigned i = 0; i < nattribs; ++i) {
    if(attribs[i].usage == SSOL_POSITION) pos = &attribs[i];
    else if(attribs[i].usage == SSOL_NORMAL) nrm = &attribs[i];
    else if(attribs[i].usage == SSOL_TEXCOORD) tex = &attribs[i];
  }
  if(!pos || !pos->get) return RES_BAD_ARG;
  s->nrm.clear(); s->uv.clear();
  if(nrm && nrm->get) {
    s->nrm.resize(nverts * 3);
    for(unsigned v = 0; v < nverts; ++v) nrm->get(v, &s->nrm[v * 3], data);
  }
  if(tex && tex->get) {
    s->uv.resize(nverts * 2);
    for(unsigned v = 0; v < nverts; ++v) tex->get(v, &s->uv[v * 2], data);
  }
  std::vector<unsigned> ids(ntris * 3);
  for(unsigned t = 0; t < ntris; ++t) {
    get_ids(t, &ids[t * 3], data);
    for(int k = 0; k < 3; ++k) if(ids[t * 3 + k] >= nverts) return RES_BAD_ARG;
  }
  std::vector<float> p(nverts * 3);
  for(unsigned v = 0; v < nverts; ++v) pos->get(v, &p[v * 3], data);
  s->ids = ids; s->pos = p;
  s->rt_area = s->samp_area = tri_area_f(p, ids);
  s->ready = true;
  return RES_OK;
}

/* Punched surface discretisation: the reference's grid
 * (src/ssol_shape.c:493-574, 1352-1403) clipped by convex carvings */
API res_T ssol_punched_surface_setup(ssol_shape* s, const ssol_punched_surface* ps)
{
  if(!s || !s->punched || !ps || !ps->quadric) return RES_BAD_ARG;
  const ssol_quadric& q = *ps->quadric;
  bool ok = true;
  switch(q.type) {
    case SSOL_QUADRIC_PLANE: break;
    case SSOL_QUADRIC_PARABOL: ok = q.data.parabol.focal > 0; break;
    case SSOL_QUADRIC_PARABOL2F:
      ok = q.data.parabol2f.focal_x > 0 && q.data.parabol2f.focal_y > 0; break;
    case SSOL_QUADRIC_HYPERBOL:
      ok = q.data.hyperbol.img_focal > 0 && q.data.hyperbol.real_focal > 0; break;
    case SSOL_QUADRIC_PARABOLIC_CYLINDER:
      ok = q.data.parabolic_cylinder.focal > 0; break;
    case SSOL_QUADRIC_HEMISPHERE: ok = q.data.hemisphere.radius > 0; break;
    default: ok = false;
  }
  if(!ok) return RES_BAD_ARG;
  if(ps->nb_carvings == 0 && q.type != SSOL_QUADRIC_HEMISPHERE) return RES_BAD_ARG;
  if(ps->nb_carvings && !ps->carvings) return RES_BAD_ARG;
  std::vector<OCarving> carv;
  for(size_t i = 0; i < ps->nb_carvings; ++i) {
    const ssol_carving& c = ps->carvings[i];
    if(!c.get || !c.nb_vertices || (unsigned)c.operation >= SSOL_CLIPPING_OPS_COUNT__)
      return RES_BAD_ARG;
    OCarving oc; oc.op = c.operation; oc.xy.resize(c.nb_vertices * 2);
    for(size_t v = 0; v < c.nb_vertices; ++v) c.get(v, &oc.xy[v * 2], c.context);
    carv.push_back(oc);
  }
  double qp[4] = {0, 0, 0, 0};
  switch(q.type) {
    case SSOL_QUADRIC_PARABOL:
      qp[0] = q.data.parabol.focal; qp[1] = 1 / (4.0 * q.data.parabol.focal); break;
    case SSOL_QUADRIC_PARABOL2F:
      qp[0] = 1 / (4.0 * q.data.parabol2f.focal_x);
      qp[1] = 1 / (4.0 * q.data.parabol2f.focal_y); break;
    case SSOL_QUADRIC_HYPERBOL: {
      /* src/ssol_shape.c:1283-1299 */
      const double g = q.data.hyperbol.real_focal + q.data.hyperbol.img_focal;
      const double f = q.data.hyperbol.real_focal / g;
      const double a2 = g * g * (f - f * f);
      qp[0] = g * 0.5; qp[1] = g * std::fabs(f - 0.5);
      qp[2] = a2 / (qp[1] * qp[1]); qp[3] = 1 / a2; break;
    }
    case SSOL_QUADRIC_PARABOLIC_CYLINDER:
      qp[0] = q.data.parabolic_cylinder.focal;
      qp[1] = 1 / (4.0 * q.data.parabolic_cylinder.focal); break;
    case SSOL_QUADRIC_HEMISPHERE:
      qp[0] = q.data.hemisphere.radius;
      qp[1] = qp[0] * qp[0]; break;
    default: break;
  }
  std::vector<Poly> cells;
  double lo[2], hi[2];
  size_t nslices;
  size_t gnx = 0, gny = 0;
  double delta = 0;
  double disk2 = 0;
  if(q.type == SSOL_QUADRIC_HEMISPHERE) {
    double r2 = -1;
    for(const OCarving& c : carv) if(c.op != SSOL_SUB)
      for(size_t i = 0; i + 1 < c.xy.size(); i += 2)
        r2 = std::max(r2, c.xy[i] * c.xy[i] + c.xy[i+1] * c.xy[i+1]);
    const double r = std::min(r2 >= 0 ? std::sqrt(r2) : qp[0], qp[0]);
    disk2 = r * r;
    lo[0] = lo[1] = -r; hi[0] = hi[1] = r;
    nslices = q.slices_count_hint != SIZE_MAX ? q.slices_count_hint
            : (size_t)(5.5 + 11 * r / qp[0]);
    if(!nslices) return RES_BAD_ARG;
    const size_t ns = std::max<size_t>(64, 8 * nslices);
    for(size_t k = 0; k < nslices; ++k) {
      const double ra = r * std::sin(0.5 * M_PI * (double)k / nslices);
      const double rb = r * std::sin(0.5 * M_PI * (double)(k + 1) / nslices);
      for(size_t j = 0; j < ns; ++j) {
        const double a0 = 2 * M_PI * (double)j / ns, a1 = 2 * M_PI * (double)(j + 1) / ns;
        const std::pair<double,double> p00(ra*std::cos(a0), ra*std::sin(a0));
        const std::pair<double,double> p01(ra*std::cos(a1), ra*std::sin(a1));
        const std::pair<double,double> p10(rb*std::cos(a0), rb*std::sin(a0));
        const std::pair<double,double> p11(rb*std::cos(a1), rb*std::sin(a1));
        if(k == 0) cells.push_back({{0.0, 0.0}, p10, p11});
        else { cells.push_back({p00, p10, p11}); cells.push_back({p00, p11, p01}); }
      }
    }
  } else {
    lo[0] = lo[1] = DBL_MAX; hi[0] = hi[1] = -DBL_MAX;
    for(const OCarving& c : carv) if(c.op != SSOL_SUB)
      for(size_t i = 0; i + 1 < c.xy.size(); i += 2) {
        lo[0] = std::min(lo[0], c.xy[i]); hi[0] = std::max(hi[0], c.xy[i]);
        lo[1] = std::min(lo[1], c.xy[i+1]); hi[1] = std::max(hi[1], c.xy[i+1]);
      }
    if(lo[0] >= hi[0] || lo[1] >= hi[1]) return RES_BAD_ARG;
    if(q.slices_count_hint != SIZE_MAX) nslices = q.slices_count_hint;
    else if(q.type == SSOL_QUADRIC_PLANE) nslices = 1;
    else {
      const double zmax = std::max(qz(q.type, qp, lo[0], lo[1]),
                                   qz(q.type, qp, hi[0], hi[1]));
      nslices = std::min<size_t>(50, (size_t)(3 + std::sqrt(zmax) * 6));
    }
    if(!nslices) return RES_BAD_ARG;
    const double sx = hi[0] - lo[0], sy = hi[1] - lo[1];
    const double smin = std::min(sx, sy);
    if(std::fabs(smin) <= 1e-6) return RES_BAD_ARG;
    delta = smin / (double)nslices;
    gnx = (size_t)std::ceil(sx / delta);
    gny = (size_t)std::ceil(sy / delta);
    auto at = [&](size_t i, size_t j) {
      return std::pair<double,double>(std::min(lo[0] + (double)i * delta, hi[0]),
                                      std::min(lo[1] + (double)j * delta, hi[1]));
    };
    for(size_t i = 0; i < gnx; ++i)
      for(size_t j = 0; j < gny; ++j) {
        cells.push_back({at(i, j), at(i + 1, j + 1), at(i + 1, j)});
        cells.push_back({at(i, j), at(i, j + 1), at(i + 1, j + 1)});
      }
  }
  /* Clip: convex carvings only (each AND keeps the inside, each SUB removes
   * it by splitting along its edges) */
  auto ccw = [](Poly p) { if(poly_area(p) < 0) std::reverse(p.begin(), p.end()); return p; };
  std::vector<Poly> ands, subs;
  for(const OCarving& c : carv) {
    Poly p;
    for(size_t i = 0; i + 1 < c.xy.size(); i += 2) p.push_back({c.xy[i], c.xy[i+1]});
    (c.op == SSOL_AND ? ands : subs).push_back(ccw(p));
  }
  std::vector<Poly> outp;
  size_t intact = 0;
  for(const Poly& cell : cells) {
    const bool cell_ccw = poly_area(cell) > 0;
    std::vector<Poly> pieces = {ccw(cell)};
    for(const Poly& a : ands) {
      std::vector<Poly> nx;
      for(Poly pc : pieces) {
        for(size_t e = 0; e < a.size() && pc.size() >= 3; ++e)
          pc = half_clip(pc, a[e], a[(e + 1) % a.size()], 1.0);
        if(pc.size() >= 3 && poly_area(pc) > 0) nx.push_back(pc);
      }
      pieces = nx;
    }
    for(const Poly& sb : subs) {
      std::vector<Poly> nx;
      for(const Poly& pc : pieces) {
        Poly rest = pc;
        for(size_t e = 0; e < sb.size() && rest.size() >= 3; ++e) {
          Poly outside = half_clip(rest, sb[e], sb[(e + 1) % sb.size()], -1.0);
          if(outside.size() >= 3 && std::fabs(poly_area(outside)) > 0) nx.push_back(outside);
          rest = half_clip(rest, sb[e], sb[(e + 1) % sb.size()], 1.0);
        }
      }
      pieces = nx;
    }
    if(pieces.size() == 1 && pieces[0].size() == 3
    && std::is_permutation(pieces[0].begin(), pieces[0].end(), ccw(cell).begin())) {
      outp.push_back(cell);
      ++intact;
      continue;
    }
    for(const Poly& pc : pieces)
      for(size_t k = 1; k + 1 < pc.size(); ++k) {
        Poly t = {pc[0], pc[k], pc[k + 1]};
        if(std::fabs(poly_area(t)) <= 0) continue;
        if(!cell_ccw) std::reverse(t.begin(), t.end());
        outp.push_back(t);
      }
  }
  if(outp.empty()) return RES_BAD_ARG;
  std::map<std::pair<double,double>, unsigned> index;
  std::vector<double> flat;
  std::vector<unsigned> ids;
  for(const Poly& t : outp)
    for(const auto& p : t) {
      auto it = index.find(p);
      unsigned id;
      if(it == index.end()) {
        id = (unsigned)(flat.size() / 2);
        index.emplace(p, id);
        flat.push_back(p.first); flat.push_back(p.second);
      } else id = it->second;
      ids.push_back(id);
    }
  Affine T; std::memcpy(T.m, q.transform, sizeof(T.m));
  const size_t nv = flat.size() / 2;
  std::vector<float> rt(nv * 3), sp(nv * 3);
  for(size_t v = 0; v < nv; ++v) {
    const double x = flat[2*v], y = flat[2*v+1];
    const V a = xpoint(T, v3(x, y, qz(q.type, qp, x, y)));
    const V b = xpoint(T, v3((float)x, (float)y, 0));
    rt[v*3] = (float)a.x; rt[v*3+1] = (float)a.y; rt[v*3+2] = (float)a.z;
    sp[v*3] = (float)b.x; sp[v*3+1] = (float)b.y; sp[v*3+2] = (float)b.z;
  }
  s->quad = q;
  for(int k = 0; k < 4; ++k) s->q[k] = qp[k];
  s->carv = carv;
  s->lo[0] = lo[0]; s->lo[1] = lo[1]; s->hi[0] = hi[0]; s->hi[1] = hi[1];
  s->disk2 = disk2;
  s->flat = flat; s->ids = ids; s->pos = rt;
  s->rt_area = tri_area_f(rt, ids);
  s->samp_area = tri_area_f(sp, ids);
  s->gnx = gnx; s->gny = gny; s->gdelta = delta;
  s->gexact = q.type != SSOL_QUADRIC_HEMISPHERE && intact == cells.size()
           && outp.size() == cells.size();
  s->ready = true;
  return RES_OK;
}

/*******************************************************************************
 * API: materials, param buffers
 ******************************************************************************/
static res_T mtl_new(ssol_device* d, ssol_material** o, ssol_material_type t)
{
  if(!d || !o) return RES_BAD_ARG;
  ssol_material* m = new ssol_material();
  m->dev = d; d->ref.get(); m->type = t;
  *o = m;
  return RES_OK;
}
API res_T ssol_material_create_dielectric(ssol_device* d, ssol_material** o)
{ return mtl_new(d, o, SSOL_MATERIAL_DIELECTRIC); }
API res_T ssol_material_create_mirror(ssol_device* d, ssol_material** o)
{ return mtl_new(d, o, SSOL_MATERIAL_MIRROR); }
API res_T ssol_material_create_matte(ssol_device* d, ssol_material** o)
{ return mtl_new(d, o, SSOL_MATERIAL_MATTE); }
API res_T ssol_material_create_virtual(ssol_device* d, ssol_material** o)
{ return mtl_new(d, o, SSOL_MATERIAL_VIRTUAL); }
API res_T ssol_material_create_thin_dielectric(ssol_device* d, ssol_material** o)
{ return mtl_new(d, o, SSOL_MATERIAL_THIN_DIELECTRIC); }
API res_T ssol_material_get_type(const ssol_material* m, ssol_material_type* t)
{ if(!m || !t) return RES_BAD_ARG; *t = m->type; return RES_OK; }
API res_T ssol_material_ref_get(ssol_material* m)
{ if(!m) return RES_BAD_ARG; m->ref.get(); return RES_OK; }
API res_T ssol_param_buffer_ref_put(ssol_param_buffer* b);
API res_T ssol_material_ref_put(ssol_material* m)
{
  if(!m) return RES_BAD_ARG;
  if(m->ref.put()) {
    ssol_device* d = m->dev;
    ssol_medium_clear(&m->in); ssol_medium_clear(&m->out);
    ssol_medium_clear(&m->slab);
    if(m->buf) ssol_param_buffer_ref_put(m->buf);
    delete m;
    ssol_device_ref_put(d);
  }
  return RES_OK;
}
API res_T ssol_material_set_param_buffer(ssol_material* m, ssol_param_buffer* b)
{
  if(!m || !b) return RES_BAD_ARG;
  b->ref.get();
  if(m->buf) ssol_param_buffer_ref_put(m->buf);
  m->buf = b;
  return RES_OK;
}
API res_T ssol_dielectric_setup(ssol_material* m, const ssol_dielectric_shader* sh,
  const ssol_medium* out, const ssol_medium* in)
{
  if(!m || m->type != SSOL_MATERIAL_DIELECTRIC || !sh || !sh->normal
  || !medium_ok(out) || !medium_ok(in)) return RES_BAD_ARG;
  ssol_medium_copy(&m->out, out); ssol_medium_copy(&m->in, in);
  m->normal = sh->normal;
  return RES_OK;
}
API res_T ssol_mirror_setup(ssol_material* m, const ssol_mirror_shader* sh,
  const ssol_microfacet_distribution d)
{
  if(!m || m->type != SSOL_MATERIAL_MIRROR || !sh || !sh->normal
  || !sh->reflectivity || !sh->roughness
  || (unsigned)d >= SSOL_MICROFACET_DISTRIBUTIONS_COUNT__) return RES_BAD_ARG;
  m->normal = sh->normal; m->refl = sh->reflectivity; m->rough = sh->roughness;
  m->distrib = d;
  return RES_OK;
}
API res_T ssol_matte_setup(ssol_material* m, const ssol_matte_shader* sh)
{
  if(!m || m->type != SSOL_MATERIAL_MATTE || !sh || !sh->normal || !sh->reflectivity)
    return RES_BAD_ARG;
  m->normal = sh->normal; m->refl = sh->reflectivity;
  return RES_OK;
}
API res_T ssol_thin_dielectric_setup(ssol_material* m,
  const ssol_thin_dielectric_shader* sh, const ssol_medium* out,
  const ssol_medium* slab, const double thickness)
{
  if(!m || m->type != SSOL_MATERIAL_THIN_DIELECTRIC || !sh || !sh->normal
  || !medium_ok(out) || !medium_ok(slab) || thickness < 0) return RES_BAD_ARG;
  ssol_medium_copy(&m->slab, slab); m->thickness = thickness;
  ssol_medium_copy(&m->out, out); ssol_medium_copy(&m->in, out);
  m->normal = sh->normal;
  return RES_OK;
}
API res_T ssol_param_buffer_create(ssol_device* d, const size_t cap,
                                   ssol_param_buffer** o)
{
  if(!d || !cap || !o) return RES_BAD_ARG;
  ssol_param_buffer* b = new ssol_param_buffer();
  b->dev = d; d->ref.get(); b->mem.resize(cap + 64); b->cap = cap;
  *o = b;
  return RES_OK;
}
API res_T ssol_param_buffer_ref_get(ssol_param_buffer* b)
{ if(!b) return RES_BAD_ARG; b->ref.get(); return RES_OK; }
API res_T ssol_param_buffer_ref_put(ssol_param_buffer* b)
{
  if(!b) return RES_BAD_ARG;
  if(b->ref.put()) { ssol_device* d = b->dev; delete b; ssol_device_ref_put(d); }
  return RES_OK;
}
static unsigned char* pbase(ssol_param_buffer* b)
{ return (unsigned char*)(((uintptr_t)b->mem.data() + 63) & ~(uintptr_t)63); }
API void* ssol_param_buffer_allocate(ssol_param_buffer* b, const size_t sz,
                                     const size_t al, void (*)(void*))
{
  if(!b || !sz || !al || (al & (al - 1)) || al > 64) return nullptr;
  const size_t off = (b->used + al - 1) & ~(al - 1);
  if(off + sz > b->cap) return nullptr;
  b->used = off + sz;
  return pbase(b) + off;
}
API void* ssol_param_buffer_get(ssol_param_buffer* b)
{ return b && b->used ? pbase(b) : nullptr; }
API res_T ssol_param_buffer_clear(ssol_param_buffer* b)
{ if(!b) return RES_BAD_ARG; b->used = 0; return RES_OK; }

/*******************************************************************************
 * API: objects and instances
 ******************************************************************************/
API res_T ssol_object_create(ssol_device* d, ssol_object** o)
{
  if(!d || !o) return RES_BAD_ARG;
  ssol_object* ob = new ssol_object();
  ob->dev = d; d->ref.get();
  *o = ob;
  return RES_OK;
}
API res_T ssol_object_ref_get(ssol_object* o)
{ if(!o) return RES_BAD_ARG; o->ref.get(); return RES_OK; }
API res_T ssol_object_clear(ssol_object* o)
{
  if(!o) return RES_BAD_ARG;
  for(OShaded& s : o->shaded) {
    ssol_shape_ref_put(s.shape);
    ssol_material_ref_put(s.front);
    ssol_material_ref_put(s.back);
  }
  o->shaded.clear(); o->rt_area = o->samp_area = 0;
  return RES_OK;
}
API res_T ssol_object_ref_put(ssol_object* o)
{
  if(!o) return RES_BAD_ARG;
  if(o->ref.put()) {
    ssol_device* d = o->dev; ssol_object_clear(o); delete o; ssol_device_ref_put(d);
  }
  return RES_OK;
}
API res_T ssol_object_add_shaded_shape(ssol_object* o, ssol_shape* s,
                                       ssol_material* f, ssol_material* b)
{
  if(!o || !s || !f || !b) return RES_BAD_ARG;
  for(const OShaded& x : o->shaded) if(x.shape == s) return RES_OK;
  s->ref.get(); f->ref.get(); b->ref.get();
  o->shaded.push_back({s, f, b});
  o->rt_area += s->rt_area; o->samp_area += s->samp_area;
  return RES_OK;
}
API res_T ssol_object_get_area(const ssol_object* o, double* a)
{ if(!o || !a) return RES_BAD_ARG; *a = o->rt_area; return RES_OK; }
API res_T ssol_object_instantiate(ssol_object* o, ssol_instance** out)
{
  if(!o || !out) return RES_BAD_ARG;
  ssol_instance* i = new ssol_instance();
  i->dev = o->dev; o->dev->ref.get(); i->obj = o; o->ref.get(); i->id = next_id();
  *out = i;
  return RES_OK;
}
API res_T ssol_instance_ref_get(ssol_instance* i)
{ if(!i) return RES_BAD_ARG; i->ref.get(); return RES_OK; }
API res_T ssol_instance_ref_put(ssol_instance* i)
{
  if(!i) return RES_BAD_ARG;
  if(i->ref.put()) {
    ssol_device* d = i->dev; ssol_object_ref_put(i->obj); delete i;
    ssol_device_ref_put(d);
  }
  return RES_OK;
}
API res_T ssol_instance_set_transform(ssol_instance* i, const double t[12])
{ if(!i || !t) return RES_BAD_ARG; std::memcpy(i->xf.m, t, sizeof(i->xf.m)); return RES_OK; }
API res_T ssol_instance_set_receiver(ssol_instance* i, const int mask, const int pp)
{ if(!i) return RES_BAD_ARG; i->mask = mask; i->per_prim = pp; return RES_OK; }
API res_T ssol_instance_is_receiver(ssol_instance* i, int* mask, int* pp)
{ if(!i || !mask || !pp) return RES_BAD_ARG; *mask = i->mask; *pp = i->per_prim; return RES_OK; }
API res_T ssol_instance_sample(ssol_instance* i, const int s)
{ if(!i) return RES_BAD_ARG; i->sample = s; return RES_OK; }
API res_T ssol_instance_get_id(const ssol_instance* i, uint32_t* id)
{ if(!i || !id) return RES_BAD_ARG; *id = i->id; return RES_OK; }
API res_T ssol_instance_get_area(const ssol_instance* i, double* a)
{ if(!i || !a) return RES_BAD_ARG; *a = i->obj->rt_area; return RES_OK; }
API res_T ssol_instance_get_shaded_shapes_count(const ssol_instance* i, size_t* n)
{ if(!i || !n) return RES_BAD_ARG; *n = i->obj->shaded.size(); return RES_OK; }

/*******************************************************************************
 * API: sun, atmosphere, scene
 ******************************************************************************/
static res_T sun_new(ssol_device* d, ssol_sun** o, int k)
{
  if(!d || !o) return RES_BAD_ARG;
  ssol_sun* s = new ssol_sun();
  s->dev = d; d->ref.get(); s->kind = k;
  *o = s;
  return RES_OK;
}
API res_T ssol_sun_create_directional(ssol_device* d, ssol_sun** o) { return sun_new(d, o, 0); }
API res_T ssol_sun_create_pillbox(ssol_device* d, ssol_sun** o) { return sun_new(d, o, 1); }
API res_T ssol_sun_create_gaussian(ssol_device* d, ssol_sun** o) { return sun_new(d, o, 2); }
API res_T ssol_sun_create_buie(ssol_device* d, ssol_sun** o) { return sun_new(d, o, 3); }
API res_T ssol_sun_ref_get(ssol_sun* s) { if(!s) return RES_BAD_ARG; s->ref.get(); return RES_OK; }
API res_T ssol_sun_ref_put(ssol_sun* s)
{
  if(!s) return RES_BAD_ARG;
  if(s->ref.put()) {
    ssol_device* d = s->dev;
    if(s->spec) ssol_spectrum_ref_put(s->spec);
    delete s; ssol_device_ref_put(d);
  }
  return RES_OK;
}
API res_T ssol_sun_set_direction(ssol_sun* s, const double d[3])
{
  if(!s || !d) return RES_BAD_ARG;
  const double l = std::sqrt(d[0]*d[0] + d[1]*d[1] + d[2]*d[2]);
  if(l == 0) return RES_BAD_ARG;
  for(int c = 0; c < 3; ++c) s->dir[c] = d[c] / l;
  return RES_OK;
}
API res_T ssol_sun_get_direction(const ssol_sun* s, double d[3])
{ if(!s || !d) return RES_BAD_ARG; for(int c = 0; c < 3; ++c) d[c] = s->dir[c]; return RES_OK; }
API res_T ssol_sun_set_dni(ssol_sun* s, const double dni)
{ if(!s || dni <= 0) return RES_BAD_ARG; s->dni = dni; return RES_OK; }
API res_T ssol_sun_get_dni(const ssol_sun* s, double* dni)
{ if(!s || !dni) return RES_BAD_ARG; *dni = s->dni; return RES_OK; }
API res_T ssol_sun_set_spectrum(ssol_sun* s, ssol_spectrum* sp)
{
  if(!s || !sp) return RES_BAD_ARG;
  if(sp == s->spec) return RES_OK;
  sp->ref.get();
  if(s->spec) ssol_spectrum_ref_put(s->spec);
  s->spec = sp;
  return RES_OK;
}
API res_T ssol_sun_pillbox_set_half_angle(ssol_sun* s, const double a)
{ if(!s || a <= 0 || a > M_PI * 0.5 || s->kind != 1) return RES_BAD_ARG; s->param = a; return RES_OK; }
API res_T ssol_sun_gaussian_set_std_dev(ssol_sun* s, const double sd)
{ if(!s || sd <= 0 || s->kind != 2) return RES_BAD_ARG; s->param = sd; return RES_OK; }
API res_T ssol_sun_set_buie_param(ssol_sun* s, const double c)
{ if(!s || c <= 0 || c >= 1 || s->kind != 3) return RES_BAD_ARG; s->param = c; return RES_OK; }

API res_T ssol_atmosphere_create(ssol_device* d, ssol_atmosphere** o)
{
  if(!d || !o) return RES_BAD_ARG;
  ssol_atmosphere* a = new ssol_atmosphere();
  a->dev = d; d->ref.get();
  *o = a;
  return RES_OK;
}
API res_T ssol_atmosphere_ref_get(ssol_atmosphere* a)
{ if(!a) return RES_BAD_ARG; a->ref.get(); return RES_OK; }
API res_T ssol_atmosphere_ref_put(ssol_atmosphere* a)
{
  if(!a) return RES_BAD_ARG;
  if(a->ref.put()) { ssol_device* d = a->dev; ssol_data_clear(&a->ext); delete a; ssol_device_ref_put(d); }
  return RES_OK;
}
API res_T ssol_atmosphere_set_extinction(ssol_atmosphere* a, ssol_data* e)
{
  if(!a || !e) return RES_BAD_ARG;
  if(e->type == SSOL_DATA_REAL) {
    if(e->value.real < 0 || e->value.real > 1) return RES_BAD_ARG;
  } else if(!spectrum_ok(e->value.spectrum, 0, 1)) return RES_BAD_ARG;
  ssol_data_copy(&a->ext, e);
  return RES_OK;
}

API res_T ssol_scene_create(ssol_device* d, ssol_scene** o)
{
  if(!d || !o) return RES_BAD_ARG;
  ssol_scene* s = new ssol_scene();
  s->dev = d; d->ref.get();
  *o = s;
  return RES_OK;
}
API res_T ssol_scene_ref_get(ssol_scene* s) { if(!s) return RES_BAD_ARG; s->ref.get(); return RES_OK; }
API res_T ssol_scene_detach_sun(ssol_scene* s, ssol_sun* sun)
{
  if(!s || !sun || !s->sun || sun->scn != s) return RES_BAD_ARG;
  sun->scn = nullptr; s->sun = nullptr; ssol_sun_ref_put(sun);
  return RES_OK;
}
API res_T ssol_scene_detach_atmosphere(ssol_scene* s, ssol_atmosphere* a)
{
  if(!s || !a || !s->atm || a->scn != s) return RES_BAD_ARG;
  a->scn = nullptr; s->atm = nullptr; ssol_atmosphere_ref_put(a);
  return RES_OK;
}
API res_T ssol_scene_clear(ssol_scene* s)
{
  if(!s) return RES_BAD_ARG;
  for(ssol_instance* i : s->inst) ssol_instance_ref_put(i);
  s->inst.clear();
  if(s->sun) ssol_scene_detach_sun(s, s->sun);
  if(s->atm) ssol_scene_detach_atmosphere(s, s->atm);
  return RES_OK;
}
API res_T ssol_scene_ref_put(ssol_scene* s)
{
  if(!s) return RES_BAD_ARG;
  if(s->ref.put()) { ssol_device* d = s->dev; ssol_scene_clear(s); delete s; ssol_device_ref_put(d); }
  return RES_OK;
}
API res_T ssol_scene_attach_instance(ssol_scene* s, ssol_instance* i)
{
  if(!s || !i) return RES_BAD_ARG;
  if(std::find(s->inst.begin(), s->inst.end(), i) != s->inst.end()) return RES_OK;
  i->ref.get(); s->inst.push_back(i);
  return RES_OK;
}
API res_T ssol_scene_detach_instance(ssol_scene* s, ssol_instance* i)
{
  if(!s || !i) return RES_BAD_ARG;
  auto it = std::find(s->inst.begin(), s->inst.end(), i);
  if(it == s->inst.end()) return RES_BAD_ARG;
  s->inst.erase(it); ssol_instance_ref_put(i);
  return RES_OK;
}
API res_T ssol_scene_attach_sun(ssol_scene* s, ssol_sun* sun)
{
  if(!s || !sun) return RES_BAD_ARG;
  if(sun->scn || s->sun) return (sun->scn == s && s->sun == sun) ? RES_OK : RES_BAD_ARG;
  sun->ref.get(); s->sun = sun; sun->scn = s;
  return RES_OK;
}
API res_T ssol_scene_attach_atmosphere(ssol_scene* s, ssol_atmosphere* a)
{
  if(!s || !a) return RES_BAD_ARG;
  if(a->scn || s->atm) return (a->scn == s && s->atm == a) ? RES_OK : RES_BAD_ARG;
  a->ref.get(); s->atm = a; a->scn = s;
  return RES_OK;
}

/*******************************************************************************
 * Solver
 ******************************************************************************/
namespace {

struct OTri { V v0, v1, v2; int sinst; unsigned prim; int gid; int attr = -1; };
/* Fragment inputs of a mesh triangle (src/ssol_material.c:551-655): world
 * vertex normals through the inverse transpose of the instance, texcoords
 * (or Star-3D's default (1,0), (0,1), (0,0)), dP/du and dP/dv, and per side
 * the material whose shaders vary over the shape (evaluated per fragment) */
struct OTriAttr {
  bool has_n = false; V n[3];
  double uv[3][2];
  V dpdu, dpdv;
  const ssol_material* vary[2] = {nullptr, nullptr};
};
struct OQuad {
  Affine l2w, w2l; const ssol_shape* shape; int sinst;
};
struct OSInst {
  const ssol_instance* inst; const ssol_shape* shape;
  const ssol_material* mtl[2]; bool punched; int quad;
};
struct OSamp { V v0, e1, e2, n; int sinst; unsigned prim; int gid; };
struct ONode { double lo[3], hi[3]; int left, right, first, count; };

struct Scene {
  std::vector<OTri> tris;
  std::vector<OQuad> quads;
  std::vector<OSInst> sinst;
  std::vector<OSamp> samp;
  std::vector<float> aprob;
  std::vector<int> aidx;
  std::vector<ONode> nodes;
  std::vector<int> order; /* primitive refs: >=0 tri, <0 ~quad */
  double area_rt = 0, area_proxy = 0;
  ssol_medium air;
  const ssol_sun* sun;
  V sun_dir;
  V basis[3];
  double buie[8];
  std::vector<double> wl, wpdf, wcdf;
  /* Shader values (reflectivity, roughness) per material at the sun
   * spectrum nodes: callbacks are host functions, evaluated once per solve
   * (the same wavelength-only rule as the device library) */
  std::map<const ssol_material*, std::vector<double>> shade_tab;
  std::vector<OTriAttr> tattr;
};

/* Same deterministic Vose construction as the device library */
void alias_table(const std::vector<double>& w, std::vector<float>& prob,
                 std::vector<int>& al)
{
  const size_t n = w.size();
  prob.assign(n, 1.0f); al.resize(n);
  double tot = 0;
  for(double x : w) tot += x;
  std::vector<double> p(n);
  std::vector<int> sm, lg;
  for(size_t i = 0; i < n; ++i) {
    al[i] = (int)i;
    p[i] = tot > 0 ? w[i] * (double)n / tot : 1.0;
    (p[i] < 1.0 ? sm : lg).push_back((int)i);
  }
  while(!sm.empty() && !lg.empty()) {
    const int s = sm.back(); sm.pop_back();
    const int l = lg.back(); lg.pop_back();
    prob[s] = (float)p[s]; al[s] = l;
    p[l] = (p[l] + p[s]) - 1.0;
    (p[l] < 1.0 ? sm : lg).push_back(l);
  }
}

void prim_box(const Scene& S, int ref, double lo[3], double hi[3])
{
  if(ref >= 0) {
    const OTri& t = S.tris[ref];
    const V p[3] = {t.v0, t.v1, t.v2};
    for(int c = 0; c < 3; ++c) {
      const double a = c == 0 ? p[0].x : c == 1 ? p[0].y : p[0].z;
      lo[c] = hi[c] = a;
      for(int k = 1; k < 3; ++k) {
        const double b = c == 0 ? p[k].x : c == 1 ? p[k].y : p[k].z;
        lo[c] = std::min(lo[c], b); hi[c] = std::max(hi[c], b);
      }
    }
  } else {
    const OQuad& q = S.quads[~ref];
    const ssol_shape* s = q.shape;
    double zl = 0, zh = 0;
    if(s->quad.type == SSOL_QUADRIC_HEMISPHERE) { zl = 0; zh = s->q[0]; }
    else if(s->quad.type != SSOL_QUADRIC_PLANE) {
      const double xm = (s->lo[0] <= 0 && s->hi[0] >= 0) ? 0
        : std::min(std::fabs(s->lo[0]), std::fabs(s->hi[0]));
      const double ym = (s->lo[1] <= 0 && s->hi[1] >= 0) ? 0
        : std::min(std::fabs(s->lo[1]), std::fabs(s->hi[1]));
      zl = qz(s->quad.type, s->q, xm, ym);
      zh = qz(s->quad.type, s->q, std::max(std::fabs(s->lo[0]), std::fabs(s->hi[0])),
              std::max(std::fabs(s->lo[1]), std::fabs(s->hi[1])));
      if(zl > zh) std::swap(zl, zh);
    }
    for(int c = 0; c < 3; ++c) { lo[c] = DBL_MAX; hi[c] = -DBL_MAX; }
    for(int k = 0; k < 8; ++k) {
      const V w = xpoint(q.l2w, v3((k & 1) ? s->hi[0] : s->lo[0],
                                   (k & 2) ? s->hi[1] : s->lo[1], (k & 4) ? zh : zl));
      const double a[3] = {w.x, w.y, w.z};
      for(int c = 0; c < 3; ++c) { lo[c] = std::min(lo[c], a[c]); hi[c] = std::max(hi[c], a[c]); }
    }
    for(int c = 0; c < 3; ++c) {
      const double pad = 1e-6 * (1 + std::fabs(lo[c]) + std::fabs(hi[c]));
      lo[c] -= pad; hi[c] += pad;
    }
  }
}

/* Median-split BVH (simple and adequate for a checker) */
int build_node(Scene& S, std::vector<int>& refs, int b, int e,
               std::vector<std::array<double,6>>& boxes, int depth)
{
  ONode n;
  for(int c = 0; c < 3; ++c) { n.lo[c] = DBL_MAX; n.hi[c] = -DBL_MAX; }
  for(int i = b; i < e; ++i)
    for(int c = 0; c < 3; ++c) {
      n.lo[c] = std::min(n.lo[c], boxes[i][c]);
      n.hi[c] = std::max(n.hi[c], boxes[i][3 + c]);
    }
  const int id = (int)S.nodes.size();
  S.nodes.push_back(n);
  if(e - b <= 4 || depth > 48) {
    S.nodes[id].left = S.nodes[id].right = -1;
    S.nodes[id].first = (int)S.order.size();
    S.nodes[id].count = e - b;
    for(int i = b; i < e; ++i) S.order.push_back(refs[i]);
    return id;
  }
  int axis = 0;
  double ext = -1;
  for(int c = 0; c < 3; ++c)
    if(n.hi[c] - n.lo[c] > ext) { ext = n.hi[c] - n.lo[c]; axis = c; }
  const int m = (b + e) / 2;
  std::vector<int> idx(e - b);
  for(int i = 0; i < e - b; ++i) idx[i] = b + i;
  std::nth_element(idx.begin(), idx.begin() + (m - b), idx.end(), [&](int x, int y) {
    return boxes[x][axis] + boxes[x][3 + axis] < boxes[y][axis] + boxes[y][3 + axis];
  });
  std::vector<int> r2(e - b);
  std::vector<std::array<double,6>> b2(e - b);
  for(int i = 0; i < e - b; ++i) { r2[i] = refs[idx[i]]; b2[i] = boxes[idx[i]]; }
  for(int i = 0; i < e - b; ++i) { refs[b + i] = r2[i]; boxes[b + i] = b2[i]; }
  const int l = build_node(S, refs, b, m, boxes, depth + 1);
  const int r = build_node(S, refs, m, e, boxes, depth + 1);
  S.nodes[id].left = l; S.nodes[id].right = r; S.nodes[id].count = 0;
  return id;
}

double buie_chi(double c)
{
  if(c > 0.145)
    return -0.04419909985804843 + c * (1.401323894233574 + c * (-0.3639746714505299
      + c * (-0.9579768560161194 + 1.1550475450828657 * c)));
  if(c > 0.035)
    return 0.022652077593662934 + c * (0.5252380349996234 + c * (2.5484334534423887
      - 0.8763755326550412 * c));
  return 0.004733749294807862 + c * (4.716738065192151 + c * (-463.506669149804
    + c * (24745.88727411664 + c * (-606122.7511711778 + 5521693.445014727 * c))));
}

void tabulate(Scene& S, const ssol_material* m);

/* Fragment of a mesh point (surface_fragment_setup, src/ssol_material.c:
 * 551-655): P, dir, Ng (unit, facing the incoming dir), uv and Ns
 * interpolated with the barycentric weights (1 - b1 - b2, b1, b2), Ns turned
 * toward -dir, dP/du and dP/dv of the triangle */
ssol_surface_fragment mesh_fragment(const OTriAttr& a, V P, V dir, V Ng, double b1,
                                    double b2)
{
  ssol_surface_fragment f = SSOL_SURFACE_FRAGMENT_NULL;
  const double b0 = 1 - b1 - b2;
  f.P[0] = P.x; f.P[1] = P.y; f.P[2] = P.z;
  f.dir[0] = dir.x; f.dir[1] = dir.y; f.dir[2] = dir.z;
  f.Ng[0] = Ng.x; f.Ng[1] = Ng.y; f.Ng[2] = Ng.z;
  V ns = Ng;
  if(a.has_n) {
    const V m = a.n[0] * b0 + a.n[1] * b1 + a.n[2] * b2;
    const double l = std::sqrt(dot(m, m));
    if(l > 0) {
      ns = m * (1 / l);
      if(dot(dir, ns) > 0) ns = -ns;
    }
  }
  f.Ns[0] = ns.x; f.Ns[1] = ns.y; f.Ns[2] = ns.z;
  f.uv[0] = a.uv[0][0] * b0 + a.uv[1][0] * b1 + a.uv[2][0] * b2;
  f.uv[1] = a.uv[0][1] * b0 + a.uv[1][1] * b1 + a.uv[2][1] * b2;
  f.dPdu[0] = a.dpdu.x; f.dPdu[1] = a.dpdu.y; f.dPdu[2] = a.dpdu.z;
  f.dPdv[0] = a.dpdv.x; f.dPdv[1] = a.dpdv.y; f.dPdv[2] = a.dpdv.z;
  return f;
}

/* Attributes of mesh triangle t of shape s under instance transform xf */
OTriAttr tri_attr(const ssol_shape* s, unsigned t, const Affine& xf)
{
  OTriAttr a;
  V p[3];
  for(int k = 0; k < 3; ++k) {
    const unsigned id = s->ids[t * 3 + k];
    p[k] = xpoint(xf, v3(s->pos[id * 3], s->pos[id * 3 + 1], s->pos[id * 3 + 2]));
    if(!s->uv.empty()) { a.uv[k][0] = s->uv[id * 2]; a.uv[k][1] = s->uv[id * 2 + 1]; }
    else { a.uv[k][0] = k == 0 ? 1 : 0; a.uv[k][1] = k == 1 ? 1 : 0; }
  }
  Affine inv;
  if(!s->nrm.empty() && inverse(xf, inv)) {
    a.has_n = true;
    /* src/ssol_material.c:632-646 turns the normal by the inverse transpose
     * only when none of the three linear columns, in FP32, equals the
     * identity's */
    bool any_id = false;
    for(int c = 0; c < 3; ++c) {
      bool eq = true;
      for(int r = 0; r < 3; ++r)
        eq = eq && (float)xf.m[3 * c + r] == (r == c ? 1.f : 0.f);
      any_id = any_id || eq;
    }
    for(int k = 0; k < 3; ++k) {
      const unsigned id = s->ids[t * 3 + k];
      const V n = v3(s->nrm[id * 3], s->nrm[id * 3 + 1], s->nrm[id * 3 + 2]);
      a.n[k] = any_id ? n : xvec_t(inv, n);
    }
  }
  const V e1 = p[1] - p[0], e2 = p[2] - p[0];
  const double du1 = a.uv[1][0] - a.uv[0][0], dv1 = a.uv[1][1] - a.uv[0][1];
  const double du2 = a.uv[2][0] - a.uv[0][0], dv2 = a.uv[2][1] - a.uv[0][1];
  const double det = du1 * dv2 - dv1 * du2;
  if(det == 0) {
    V n = cross(e2, e1);
    const double l = std::sqrt(dot(n, n));
    n = l > 0 ? n * (1 / l) : v3(0, 0, 1);
    onb(n, a.dpdu, a.dpdv);
  } else {
    a.dpdu = (e1 * dv2 - e2 * dv1) * (1 / det);
    a.dpdv = (e2 * du1 - e1 * du2) * (1 / det);
  }
  return a;
}

/* Whether a mirror or matte material gives other shader values at the
 * vertices of triangles t0 and t1 of a shape (seen from `side`) than at the
 * reference fragment of the per-material table: the same probe as the B200
 * library's, so that both evaluate the same materials per fragment */
bool varies_over(const ssol_material* m, const ssol_shape* s, const Affine& xf,
                 int side, double wl)
{
  if(m->type != SSOL_MATERIAL_MIRROR && m->type != SSOL_MATERIAL_MATTE) return false;
  ssol_surface_fragment ref = SSOL_SURFACE_FRAGMENT_NULL;
  ref.dir[2] = -1; ref.Ng[2] = 1; ref.Ns[2] = 1; ref.dPdu[0] = 1; ref.dPdv[1] = 1;
  double r0 = 0, g0 = 0;
  if(m->refl) m->refl(m->dev, m->buf, wl, &ref, &r0);
  if(m->rough) m->rough(m->dev, m->buf, wl, &ref, &g0);
  const unsigned nt = (unsigned)(s->ids.size() / 3);
  /* the vertices of up to 8 triangles spread over the mesh */
  const unsigned np = std::min(nt, 8u);
  std::vector<unsigned> probe;
  for(unsigned i = 0; i < np; ++i)
    probe.push_back(np > 1 ? (unsigned)((unsigned long long)i * (nt - 1) / (np - 1)) : 0);
  for(unsigned t : probe) {
    const OTriAttr a = tri_attr(s, t, xf);
    V p[3];
    for(int k = 0; k < 3; ++k) {
      const unsigned id = s->ids[t * 3 + k];
      p[k] = xpoint(xf, v3(s->pos[id * 3], s->pos[id * 3 + 1], s->pos[id * 3 + 2]));
    }
    V ng = cross(p[2] - p[0], p[1] - p[0]);
    const double l = std::sqrt(dot(ng, ng));
    ng = (l > 0 ? ng * (1 / l) : v3(0, 0, 1)) * (side == 0 ? 1.0 : -1.0);
    for(int k = 0; k < 3; ++k) {
      const double b1 = k == 1 ? 1 : 0, b2 = k == 2 ? 1 : 0;
      const ssol_surface_fragment f = mesh_fragment(a, p[k], -ng, ng, b1, b2);
      double r = 0, g = 0;
      if(m->refl) m->refl(m->dev, m->buf, wl, &f, &r);
      if(m->rough) m->rough(m->dev, m->buf, wl, &f, &g);
      if(r != r0 || g != g0) return true;
    }
  }
  return false;
}

res_T make_scene(ssol_scene* scn, Scene& S, bool need_sampled = true)
{
  if(!scn->sun || !scn->sun->spec || scn->sun->spec->wl.empty() || scn->sun->dni <= 0)
    return RES_BAD_ARG;
  S.sun = scn->sun;
  S.sun_dir = v3(scn->sun->dir[0], scn->sun->dir[1], scn->sun->dir[2]);
  onb(S.sun_dir, S.basis[0], S.basis[1]);
  S.basis[2] = S.sun_dir;
  S.air = SSOL_MEDIUM_VACUUM;
  if(scn->atm) S.air.extinction = scn->atm->ext;
  if(scn->sun->kind == 1 && !(scn->sun->param > 0)) return RES_BAD_ARG;
  if(scn->sun->kind == 2 && !(scn->sun->param > 0)) return RES_BAD_ARG;
  if(scn->sun->kind == 3) {
    const double csr = scn->sun->param;
    if(csr < 1e-6 || csr > 0.849) return RES_BAD_ARG;
    const double tSD = 0.00465, tCS = 0.0436, iA = 9.224724736098827E-6;
    const double chi = buie_chi(csr);
    const double k = 0.9 * std::log(13.5 * chi) * std::pow(chi, -0.3);
    const double gm = 2.2 * std::log(0.52 * chi) * std::pow(chi, 0.43) - 0.1;
    const double ek = std::exp(k) * std::pow(1000, gm);
    const double iB = ek / (gm + 2) * (std::pow(tCS, gm + 2) - std::pow(tSD, gm + 2));
    const double al = 1 / (iA + iB);
    auto pdf = [&](double t) {
      return al * (t < tSD ? std::cos(326 * t) / std::cos(308 * t) : ek * std::pow(t, gm))
           * std::sin(t);
    };
    const double h1 = 1.001 * pdf(0.0038915695846209047), h2 = pdf(tSD);
    const double d = tCS - tSD;
    const double b[8] = {tSD, d, gm, ek, al, h1, h2, tSD * h1 / (tSD * h1 + d * h2)};
    std::memcpy(S.buie, b, sizeof(b));
  }
  S.wl = scn->sun->spec->wl;
  S.wpdf = scn->sun->spec->val;
  S.wcdf.assign(S.wl.size(), 0);
  for(size_t i = 1; i < S.wl.size(); ++i)
    S.wcdf[i] = S.wcdf[i - 1] + 0.5 * (S.wpdf[i] + S.wpdf[i - 1]) * (S.wl[i] - S.wl[i - 1]);
  if(S.wl.size() > 1) {
    if(!(S.wcdf.back() > 0)) return RES_BAD_ARG;
    const double t = S.wcdf.back();
    for(double& c : S.wcdf) c /= t;
    S.wcdf.back() = 1;
  }
  std::vector<double> area;
  bool sampled = false;
  std::map<std::pair<const ssol_material*, const ssol_shape*>, bool> varies;
  for(ssol_instance* inst : scn->inst) {
    if(inst->sample) {
      sampled = true;
      S.area_rt += inst->obj->rt_area;
      S.area_proxy += inst->obj->samp_area;
    }
    for(const OShaded& sh : inst->obj->shaded) {
      if(!sh.shape->ready) continue;
      const int si = (int)S.sinst.size();
      OSInst o;
      o.inst = inst; o.shape = sh.shape; o.mtl[0] = sh.front; o.mtl[1] = sh.back;
      tabulate(S, sh.front);
      tabulate(S, sh.back);
      o.punched = sh.shape->punched; o.quad = -1;
      if(inst->per_prim && inst->mask && o.punched && !sh.shape->gexact)
        return RES_BAD_ARG;
      const ssol_shape* s = sh.shape;
      if(!s->punched) {
        const int first = (int)S.tris.size();
        for(size_t t = 0; t < s->ids.size() / 3; ++t) {
          float vf[3][3];
          for(int k = 0; k < 3; ++k) {
            const unsigned id = s->ids[t * 3 + k];
            const V w = xpoint(inst->xf, v3(s->pos[id*3], s->pos[id*3+1], s->pos[id*3+2]));
            vf[k][0] = (float)w.x; vf[k][1] = (float)w.y; vf[k][2] = (float)w.z;
          }
          const V p0 = v3(vf[0][0], vf[0][1], vf[0][2]);
          const V p1 = v3(vf[1][0], vf[1][1], vf[1][2]);
          const V p2 = v3(vf[2][0], vf[2][1], vf[2][2]);
          OTri tr = {p0, p1, p2, si, (unsigned)t, first + (int)t};
          const ssol_material* vary[2] = {nullptr, nullptr};
          for(int sd = 0; sd < 2; ++sd) {
            const ssol_material* m = sd == 0 ? sh.front : sh.back;
            const auto key = std::make_pair(m, (const ssol_shape*)s);
            auto f = varies.find(key);
            if(f == varies.end())
              f = varies.emplace(key, varies_over(m, s, inst->xf, sd, S.wl.front())
                                      || varies_over(m, s, inst->xf, sd, S.wl.back())).first;
            if(f->second) vary[sd] = m;
          }
          if(!s->nrm.empty() || vary[0] || vary[1]) {
            OTriAttr a = tri_attr(s, (unsigned)t, inst->xf);
            a.vary[0] = vary[0]; a.vary[1] = vary[1];
            tr.attr = (int)S.tattr.size();
            S.tattr.push_back(a);
          }
          S.tris.push_back(tr);
          if(inst->sample) {
            const V n = cross(p2 - p0, p1 - p0);
            const double len = std::sqrt(dot(n, n));
            const V nu = len > 0 ? n * (1 / len) : v3(0, 0, 0);
            const V nf = v3((float)nu.x, (float)nu.y, (float)nu.z);
            OSamp sp = {p0, p1 - p0, p2 - p0, nf, si, (unsigned)t, tr.gid};
            S.samp.push_back(sp);
            area.push_back(0.5 * len);
          }
        }
      } else {
        OQuad q;
        Affine qt; std::memcpy(qt.m, s->quad.transform, sizeof(qt.m));
        q.l2w = compose(inst->xf, qt);
        if(!inverse(q.l2w, q.w2l)) return RES_BAD_ARG;
        q.shape = s; q.sinst = si;
        o.quad = (int)S.quads.size();
        S.quads.push_back(q);
        if(inst->sample) {
          for(size_t t = 0; t < s->ids.size() / 3; ++t) {
            float vf[3][3];
            for(int k = 0; k < 3; ++k) {
              const unsigned id = s->ids[t * 3 + k];
              const V w = xpoint(q.l2w, v3((float)s->flat[id*2], (float)s->flat[id*2+1], 0));
              vf[k][0] = (float)w.x; vf[k][1] = (float)w.y; vf[k][2] = (float)w.z;
            }
            const V p0 = v3(vf[0][0], vf[0][1], vf[0][2]);
            const V e1 = v3(vf[1][0], vf[1][1], vf[1][2]) - p0;
            const V e2 = v3(vf[2][0], vf[2][1], vf[2][2]) - p0;
            const V n = cross(e2, e1);
            const double len = std::sqrt(dot(n, n));
            const V nu = len > 0 ? n * (1 / len) : v3(0, 0, 0);
            OSamp sp = {p0, e1, e2, v3((float)nu.x, (float)nu.y, (float)nu.z), si,
                        (unsigned)t, -1};
            S.samp.push_back(sp);
            area.push_back(0.5 * len);
          }
        }
      }
      S.sinst.push_back(o);
    }
  }
  if(need_sampled && (!sampled || S.samp.empty())) return RES_BAD_ARG;
  alias_table(area, S.aprob, S.aidx);
  std::vector<int> refs;
  std::vector<std::array<double,6>> boxes;
  for(size_t i = 0; i < S.tris.size(); ++i) refs.push_back((int)i);
  for(size_t i = 0; i < S.quads.size(); ++i) refs.push_back(~(int)i);
  for(int r : refs) {
    std::array<double,6> b;
    prim_box(S, r, b.data(), b.data() + 3);
    boxes.push_back(b);
  }
  build_node(S, refs, 0, (int)refs.size(), boxes, 0);
  return RES_OK;
}

/* Ray query with the reference hit filter (src/ssol_scene.c:439-535) */
struct Self { int gid; int sinst; int side; bool discard_virtual, reversed; };
struct OHit { double t; int sinst; unsigned prim; int gid; V n; bool found; double b1, b2; };

bool side_ok(const Scene& S, int si, int side, const Self& self)
{
  if(self.reversed) side = side == 1 ? 2 : 1;
  const OSInst& o = S.sinst[si];
  if(o.mtl[side - 1]->type == SSOL_MATERIAL_VIRTUAL) {
    if(self.discard_virtual) return false;
    if(!(o.inst->mask & side)) return false;
  }
  return true;
}

/* Watertight ray/triangle test (Woop, Benthin and Wald, "Watertight
 * Ray/Triangle Intersection", JCGT 2(1), 2013), which is what keeps the rays
 * through a shared edge or vertex (every ray through the focus of
 * src/test_ssol_solver4.c crosses the diagonal of its targets) from falling
 * between two triangles. The vertices are sheared into a frame where the ray
 * runs along +z; the 2D edge functions of an edge shared by two triangles are
 * then exact negations of each other (this file is compiled without FP
 * contraction). Ng = e2 x e1 is Star-3D's front face. */
struct OShear { int kx, ky, kz; double sx, sy, sz; };

OShear make_shear(V d)
{
  const double a[3] = {std::fabs(d.x), std::fabs(d.y), std::fabs(d.z)};
  const int kz = a[0] > a[1] ? (a[0] > a[2] ? 0 : 2) : (a[1] > a[2] ? 1 : 2);
  int kx = kz == 2 ? 0 : kz + 1, ky = kx == 2 ? 0 : kx + 1;
  const double dv[3] = {d.x, d.y, d.z};
  if(dv[kz] < 0) std::swap(kx, ky);
  return {kx, ky, kz, dv[kx] / dv[kz], dv[ky] / dv[kz], 1 / dv[kz]};
}

void hit_tri(const Scene& S, int i, V o, V d, const OShear& sh, double tmin,
             double eps, const Self& self, OHit& h)
{
  const OTri& T = S.tris[i];
  const V a = T.v0 - o, b = T.v1 - o, c = T.v2 - o;
  const double av[3] = {a.x, a.y, a.z}, bv[3] = {b.x, b.y, b.z};
  const double cv[3] = {c.x, c.y, c.z};
  const double ax = av[sh.kx] - sh.sx * av[sh.kz], ay = av[sh.ky] - sh.sy * av[sh.kz];
  const double bx = bv[sh.kx] - sh.sx * bv[sh.kz], by = bv[sh.ky] - sh.sy * bv[sh.kz];
  const double cx = cv[sh.kx] - sh.sx * cv[sh.kz], cy = cv[sh.ky] - sh.sy * cv[sh.kz];
  const double U = cx * by - cy * bx;
  const double Vv = ax * cy - ay * cx;
  const double W = bx * ay - by * ax;
  if((U < 0 || Vv < 0 || W < 0) && (U > 0 || Vv > 0 || W > 0)) return;
  if(U + Vv + W == 0) return;
  /* Distance from the plane of the triangle, dot(Ng, v0 - o) / dot(Ng, d):
   * the two triangles of a planar quad then give the same distance, so a
   * ray that passes through a virtual quad on its shared edge is not
   * counted twice (it continues from the hit with tmin = next(t)) */
  const V ng = cross(T.v2 - T.v0, T.v1 - T.v0);
  const double den = dot(ng, d);
  const double t = dot(ng, a) / den;
  if(!(t < h.t) || t <= eps || t <= tmin || T.gid == self.gid) return;
  const int side = den < 0 ? 1 : 2;
  if(!side_ok(S, T.sinst, side, self)) return;
  h.t = t; h.sinst = T.sinst; h.prim = T.prim; h.gid = T.gid;
  h.n = ng; h.found = true;
  h.b1 = Vv / (U + Vv + W); h.b2 = W / (U + Vv + W);
}

unsigned grid_prim(const ssol_shape* s, double x, double y)
{
  const double d = s->gdelta;
  long ix = (long)std::floor((x - s->lo[0]) / d), iy = (long)std::floor((y - s->lo[1]) / d);
  ix = std::min(std::max(ix, 0L), (long)s->gnx - 1);
  iy = std::min(std::max(iy, 0L), (long)s->gny - 1);
  const double x0 = s->lo[0] + ix * d, y0 = s->lo[1] + iy * d;
  const double x1 = std::min(x0 + d, s->hi[0]), y1 = std::min(y0 + d, s->hi[1]);
  const bool lower = (x - x0) * (y1 - y0) >= (y - y0) * (x1 - x0);
  return (unsigned)((ix * (long)s->gny + iy) * 2 + (lower ? 0 : 1));
}

void hit_quad(const Scene& S, int i, V o, V d, double tmin, const Self& self, OHit& h)
{
  const OQuad& Q = S.quads[i];
  const ssol_shape* s = Q.shape;
  const V ol = xpoint(Q.w2l, o), dl = xvec(Q.w2l, d);
  double a, b, c;
  qcoef(s->quad.type, s->q, ol, dl, a, b, c);
  double r[2];
  int n = 0;
  if(a == 0) { if(b != 0) { r[0] = -c / b; n = 1; } }
  else {
    const double delta = b * b - 4 * a * c;
    if(delta == 0) { r[0] = -b / (2 * a); n = 1; }
    else if(delta > 0) {
      const double sq = std::sqrt(delta);
      const double t1 = (-b - std::copysign(sq, b)) / (2 * a);
      const double t2 = t1 != 0 ? c / (a * t1) : -b / a;
      r[0] = std::min(t1, t2); r[1] = std::max(t1, t2); n = 2;
    }
  }
  for(int k = 0; k < n; ++k) {
    const double t = r[k];
    if(t <= tmin) continue;
    if(!(t < h.t)) break;
    const V pl = ol + dl * t;
    if(s->quad.type == SSOL_QUADRIC_HYPERBOL && !(pl.z + s->q[1] > 0)) continue;
    if(s->quad.type == SSOL_QUADRIC_HEMISPHERE && pl.z > s->q[0]) continue;
    if(!in_domain(s, pl.x, pl.y)) continue;
    const V nw = unit(xvec_t(Q.w2l, qgrad(s->quad.type, s->q, pl)));
    const int side = dot(d, nw) < 0 ? 1 : 2;
    if(Q.sinst == self.sinst && side != self.side) continue;
    if(!side_ok(S, Q.sinst, side, self)) continue;
    h.t = t; h.sinst = Q.sinst; h.gid = -1; h.n = nw; h.found = true;
    h.b1 = h.b2 = 0;
    h.prim = s->gexact ? grid_prim(s, pl.x, pl.y) : 0;
    break;
  }
}

bool box_hit(const ONode& n, V o, V inv, double tmin, double tmax)
{
  const double oo[3] = {o.x, o.y, o.z}, ii[3] = {inv.x, inv.y, inv.z};
  double t0 = tmin, t1 = tmax;
  for(int c = 0; c < 3; ++c) {
    double a = (n.lo[c] - oo[c]) * ii[c], b = (n.hi[c] - oo[c]) * ii[c];
    if(a > b) std::swap(a, b);
    if(a != a) a = -DBL_MAX; /* 0 * inf */
    if(b != b) b = DBL_MAX;
    t0 = std::max(t0, a); t1 = std::min(t1, b);
  }
  return t0 <= t1;
}

OHit trace(const Scene& S, V o, V d, double tmin, const Self& self, bool any)
{
  OHit h; h.t = DBL_MAX; h.found = false; h.gid = -1; h.prim = 0; h.sinst = -1;
  const V inv = v3(1 / d.x, 1 / d.y, 1 / d.z);
  const double am = std::max(std::fabs(o.x), std::max(std::fabs(o.y), std::fabs(o.z)));
  const double eps = 1e-6 * (1 + am);
  const OShear sh = make_shear(d);
  int stack[128]; int sp = 0;
  stack[sp++] = 0;
  while(sp) {
    const ONode& n = S.nodes[stack[--sp]];
    if(!box_hit(n, o, inv, tmin, h.t)) continue;
    if(n.left < 0) {
      for(int k = 0; k < n.count; ++k) {
        const int r = S.order[n.first + k];
        if(r >= 0) hit_tri(S, r, o, d, sh, tmin, eps, self, h);
        else hit_quad(S, ~r, o, d, tmin, self, h);
        if(any && h.found) return h;
      }
    } else {
      stack[sp++] = n.left; stack[sp++] = n.right;
    }
  }
  return h;
}

/* Per thread tallies (struct thread_context, src/ssol_solver.c:50-61) */
struct Ctx {
  McData g[6];
  std::map<const ssol_instance*, McRcv> rcv;
  std::map<const ssol_instance*, McSamp> samp;
  size_t nreal = 0;
};

void factor_rcv(McRcv& r, const ssol_instance* inst, size_t i, double f)
{
  for(int s = 0; s < 2; ++s) {
    if(!(inst->mask & (s == 0 ? 1 : 2))) continue;
    for(McData& d : r.side[s].q) d.factor(i, f);
    for(auto& sh : r.side[s].prims) for(auto& p : sh.second) for(McData& d : p.second)
      d.factor(i, f);
  }
}

/* apply_factor_mc (src/ssol_solver.c:805-871) */
void apply_factor(Ctx& c, size_t i, double f)
{
  for(McData& d : c.g) d.factor(i, f);
  for(auto& r : c.rcv) factor_rcv(r.second, r.first, i, f);
  for(auto& s : c.samp) {
    s.second.cos.factor(i, f);
    s.second.shadow.factor(i, f);
    for(auto& r : s.second.rcv) factor_rcv(r.second, r.first, i, f);
  }
}

double wl_sample(const Scene& S, double u)
{
  const size_t n = S.wl.size();
  if(n == 1) return S.wl[0];
  size_t lo = 0, hi = n - 1;
  while(hi - lo > 1) { const size_t m = (lo + hi) / 2; if(S.wcdf[m] <= u) lo = m; else hi = m; }
  const double mass = S.wcdf[lo + 1] - S.wcdf[lo];
  const double r = mass > 0 ? std::min(std::max((u - S.wcdf[lo]) / mass, 0.0), 1.0) : 0;
  const double a = S.wpdf[lo], b = S.wpdf[lo + 1];
  double t = r;
  if(a != b) {
    const double den = a + std::sqrt(a * a + r * (b * b - a * a));
    t = den > 0 ? r * (a + b) / den : r;
  }
  return S.wl[lo] + t * (S.wl[lo + 1] - S.wl[lo]);
}

V sun_dir(const Scene& S, const PathRng& rng, const Block& b)
{
  auto world = [&](double x, double y, double z) {
    return unit(S.basis[0] * x + S.basis[1] * y + S.basis[2] * z);
  };
  switch(S.sun->kind) {
    case 1: { /* pillbox (src/ssol_ranst_sun_dir.c:246-267) */
      const double smax = std::sin(S.sun->param);
      const double s2 = unif(b.x[0]) * (smax * smax);
      const double st = std::sqrt(s2), ct = std::sqrt(1 - s2);
      const double ph = 2 * M_PI * unif(b.x[1]);
      return world(std::cos(ph) * st, std::sin(ph) * st, ct);
    }
    case 2: { /* gaussian (src/ssol_ranst_sun_dir.c:272-295) */
      double st = S.sun->param * std::sqrt(-2 * std::log(1 - unif(b.x[0])));
      st = std::min(1.0, st);
      const double ct = std::sqrt(std::max(0.0, 1 - st * st));
      const double ph = 2 * M_PI * unif(b.x[1]);
      return world(std::cos(ph) * st, std::sin(ph) * st, ct);
    }
    case 3: { /* buie (src/ssol_ranst_sun_dir.c:177-241) */
      const double* B = S.buie;
      double th = 0;
      for(uint32_t k = 0; k < 64; ++k) {
        const Block r = rng.get(2 + k, DOM_PRIMARY);
        double val;
        if(unif(r.x[0]) < B[7]) { th = unif(r.x[1]) * B[0]; val = unif(r.x[2]) * B[5]; }
        else { th = B[0] + unif(r.x[1]) * B[1]; val = unif(r.x[2]) * B[6]; }
        const double phi = th < B[0] ? std::cos(326 * th) / std::cos(308 * th)
                                     : B[3] * std::pow(th, B[2]);
        if(val <= B[4] * phi * std::sin(th)) break;
      }
      const double ph = 2 * M_PI * unif(b.x[1]);
      return world(std::sin(th) * std::sin(ph), std::sin(th) * std::cos(ph), std::cos(th));
    }
    default: return S.sun_dir;
  }
}

double shader_eval(const ssol_material* m, ssol_shader_getter_T f, double wl)
{
  if(!f) return 0;
  ssol_surface_fragment fr = SSOL_SURFACE_FRAGMENT_NULL;
  fr.dir[2] = -1; fr.Ng[2] = 1; fr.Ns[2] = 1; fr.dPdu[0] = 1; fr.dPdv[1] = 1;
  double v = 0;
  f(m->dev, m->buf, wl, &fr, &v);
  return v;
}

void tabulate(Scene& S, const ssol_material* m)
{
  if(S.shade_tab.count(m)) return;
  std::vector<double> t;
  for(double w : S.wl) {
    t.push_back(shader_eval(m, m->refl, w));
    t.push_back(shader_eval(m, m->rough, w));
  }
  S.shade_tab.emplace(m, t);
}

/* which: 0 reflectivity, 1 roughness; linear in wavelength, clamped */
double shader(const Scene& S, const ssol_material* m, int which, double wl)
{
  const std::vector<double>& t = S.shade_tab.find(m)->second;
  const std::vector<double>& w = S.wl;
  const size_t i = (size_t)(std::lower_bound(w.begin(), w.end(), wl) - w.begin());
  if(i == w.size()) return t[2 * (w.size() - 1) + which];
  if(i == 0) return t[which];
  const double a = t[2 * (i - 1) + which], b = t[2 * i + which];
  return a + (wl - w[i - 1]) * (b - a) / (w[i] - w[i - 1]);
}

double fresnel(double ci, double ct, double ei, double et)
{
  const double rs = (ei * ci - et * ct) / (ei * ci + et * ct);
  const double rp = (et * ci - ei * ct) / (et * ci + ei * ct);
  return 0.5 * (rs * rs + rp * rp);
}

/* point_shade (src/ssol_solver.c:419-494); returns false on RES_BAD_OP */
bool shade(const Scene& S, const PathRng& rng, uint32_t j, const ssol_material* m,
           const ssol_medium& in, ssol_medium& out, double wl, V wo, V Ng,
           double& prop, V& dir, int& type, V N, const ssol_surface_fragment* frag)
{
  /* N: shading normal (the fragment's Ns), Ng: geometric normal; shaders
   * of a material that varies over its mesh are evaluated at the fragment */
  auto sv = [&](int which) {
    if(!frag) return shader(S, m, which, wl);
    double v = 0;
    ssol_shader_getter_T f = which == 0 ? m->refl : m->rough;
    if(f) f(m->dev, m->buf, wl, frag, &v);
    return v;
  };
  prop = 0; type = 0;
  ssol_medium_copy(&out, &in);
  if(m->type == SSOL_MATERIAL_DIELECTRIC && !media_ceq(in, m->out)) return false;
  const double ci = dot(wo, N);
  if(!(ci > 0)) return true;
  const Block r = rng.get(j, DOM_SCATTER);
  V b1, b2;
  switch(m->type) {
    case SSOL_MATERIAL_MIRROR: {
      const double R = sv(0), a = sv(1);
      type = 1;
      if(a == 0) { dir = N * (2 * ci) - wo; prop = R; }
      else {
        Block rr = r;
        bool ok = false;
        onb(N, b1, b2);
        for(uint32_t k = 0; k < 16 && !ok; ++k) {
          if(k) rr = rng.get((j << 6) | k, DOM_RETRY);
          const double u0 = unif(rr.x[0]);
          const double t2 = m->distrib == SSOL_MICROFACET_BECKMANN
            ? -a * a * std::log(1 - u0) : a * a * u0;
          const double ct = 1 / std::sqrt(1 + t2), st = std::sqrt(t2) * ct;
          const double ph = 2 * M_PI * unif(rr.x[1]);
          const V h = b1 * (std::cos(ph) * st) + b2 * (std::sin(ph) * st) + N * ct;
          const double wh = dot(wo, h);
          if(!(wh > 0)) continue;
          dir = h * (2 * wh) - wo;
          ok = dot(dir, N) > 0;
        }
        prop = ok ? R : 0;
      }
      break;
    }
    case SSOL_MATERIAL_MATTE: {
      const double u0 = unif(r.x[0]), rad = std::sqrt(u0);
      const double ph = 2 * M_PI * unif(r.x[1]);
      onb(N, b1, b2);
      dir = b1 * (rad * std::cos(ph)) + b2 * (rad * std::sin(ph)) + N * std::sqrt(1 - u0);
      prop = sv(0);
      type = 1;
      break;
    }
    case SSOL_MATERIAL_DIELECTRIC: {
      const double ei = data_value(m->out.refractive_index, wl);
      const double et = data_value(m->in.refractive_index, wl);
      const double eta = ei / et, s2 = eta * eta * (1 - ci * ci);
      double F = 1, ct = 0;
      if(s2 < 1) { ct = std::sqrt(1 - s2); F = fresnel(ci, ct, ei, et); }
      prop = 1;
      if(unif(r.x[0]) < F) { dir = N * (2 * ci) - wo; type = 1; }
      else {
        dir = unit(N * (eta * ci - ct) - wo * eta); type = 2;
        ssol_medium_copy(&out, &m->in); /* material_get_next_medium */
      }
      break;
    }
    case SSOL_MATERIAL_THIN_DIELECTRIC: {
      const double ei = data_value(m->out.refractive_index, wl);
      const double et = data_value(m->slab.refractive_index, wl);
      const double al = data_value(m->slab.extinction, wl);
      const double eta = ei / et, s2 = eta * eta * (1 - ci * ci);
      double Rt = 1, Tt = 0;
      if(s2 < 1) {
        const double ct = std::sqrt(1 - s2);
        const double F = fresnel(ci, ct, ei, et);
        const double tau = std::exp(-al * m->thickness / ct);
        const double den = 1 - F * F * tau * tau;
        Rt = F + (1 - F) * (1 - F) * F * tau * tau / den;
        Tt = (1 - F) * (1 - F) * tau / den;
      }
      prop = Rt + Tt;
      if(prop > 0 && unif(r.x[0]) * prop < Rt) { dir = N * (2 * ci) - wo; type = 1; }
      else { dir = -wo; type = 2; }
      break;
    }
    default: break;
  }
  const double c = dot(Ng, dir);
  if((c > 0 && type == 2) || (c < 0 && type == 1)) prop = 0;
  return true;
}

McRcv1& rcv_side(std::map<const ssol_instance*, McRcv>& m, const ssol_instance* i, int side)
{ return m[i].side[side == 1 ? 0 : 1]; }

/* Shading inputs of the point on triangle gid (or a quadric when gid < 0):
 * the shading normal, and the fragment when the side's material varies */
V shading_inputs(const Scene& S, int gid, int side, V pos, V dir, V N, double b1,
                 double b2, ssol_surface_fragment& frag, bool& use_frag)
{
  use_frag = false;
  if(gid < 0 || S.tris[gid].attr < 0) return N;
  const OTriAttr& a = S.tattr[S.tris[gid].attr];
  frag = mesh_fragment(a, pos, dir, N, b1, b2);
  use_frag = a.vary[side - 1] != nullptr;
  return v3(frag.Ns[0], frag.Ns[1], frag.Ns[2]);
}

/* One realisation (trace_radiative_path, src/ssol_solver.c:873-1127) */
/* Tracked-path lengths after the defaults (src/ssol_solver.c:1211-1220) */
struct TrackLen { double sun, inf; };

res_T realisation(const Scene& S, Ctx& ctx, size_t ireal, const PathRng& rng,
                  const TrackLen* track = nullptr, OPath* path = nullptr)
{
  bool hit_rcv = false;
  auto vtx = [&](V p, double w) {
    if(!path) return;
    ssol_path_vertex v;
    v.pos[0] = p.x; v.pos[1] = p.y; v.pos[2] = p.z; v.weight = w;
    path->v.push_back(v);
  };
  /* point_init */
  const Block r0 = rng.get(0, DOM_PRIMARY);
  int k = (int)(((uint64_t)(r0.x[0] >> 8) * (uint64_t)S.samp.size()) >> 24);
  if(!((float)unif(r0.x[1]) < S.aprob[k])) k = S.aidx[k];
  const OSamp& st = S.samp[k];
  const double sa = std::sqrt(unif(r0.x[2]));
  const double b2 = sa * unif(r0.x[3]), b1 = sa - b2;
  V pos = st.v0 + st.e1 * b1 + st.e2 * b2;
  double cb1 = b1, cb2 = b2; /* barycentric weights of the current point */
  const Block r1 = rng.get(1, DOM_PRIMARY);
  V dir = sun_dir(S, rng, r1);
  const double wl = wl_sample(S, unif(r1.x[2]));
  int si = st.sinst;
  unsigned prim = st.prim;
  int gid = st.gid;
  const OSInst* o = &S.sinst[si];
  V N = st.n;
  if(o->punched) {
    const OQuad& Q = S.quads[o->quad];
    V pl = xpoint(Q.w2l, pos);
    pl.z = qz(o->shape->quad.type, o->shape->q, pl.x, pl.y);
    N = unit(xvec_t(Q.w2l, qgrad(o->shape->quad.type, o->shape->q, pl)));
    pos = xpoint(Q.l2w, pl);
  }
  int side = 1;
  if(!(dot(N, dir) < 0)) { side = 2; N = -N; }
  const double ssc = dot(N, dir), ss0 = std::fabs(dot(S.sun_dir, N));
  const double s0s = dot(S.sun_dir, dir);
  const double spc = o->punched ? std::fabs(dot(st.n, N)) : 1.0;
  const double w0 = S.sun->dni * S.area_proxy * std::fabs(ssc / (spc * s0s));
  const double cosf = S.area_proxy / S.area_rt * ss0 / spc;
  McSamp& ms = ctx.samp[o->inst];
  ms.nb++;
  const ssol_instance* samp_inst = o->inst;
  const ssol_material* mtl = o->mtl[side - 1];
  ssol_medium in = SSOL_MEDIUM_VACUUM, out = SSOL_MEDIUM_VACUUM;
  if(mtl->type == SSOL_MATERIAL_DIELECTRIC || mtl->type == SSOL_MATERIAL_THIN_DIELECTRIC)
    ssol_medium_copy(&in, side == 1 ? &mtl->in : &mtl->out);
  else ssol_medium_copy(&in, &S.air);

  /* Tracked path: the sun end, then the sampled point (src/ssol_solver.c:909-922) */
  if(path) {
    if(track->sun > 0) vtx(pos - dir * track->sun, S.sun->dni);
    vtx(pos, w0);
  }
  Self self = {gid, si, side, true, true};
  OHit h = trace(S, pos, -dir, 0, self, true);
  int score = 0;
  res_T res = RES_OK;
  bool killed = false;
  if(h.found) {
    ms.shadow.add(ireal, w0);
    ctx.g[2].add(ireal, w0);
    if(path) path->type = SSOL_PATH_SHADOW;
  } else {
    double prev[3] = {w0, w0, w0}, inc[3], outw[3] = {0, 0, 0};
    double hit_t = 0, tmin = 0;
    V org = pos, rd = dir;
    unsigned depth = 0, interval = 64, j = 0, nr = 0;
    for(size_t seg = 0;; ++seg) {
      const bool in_atm = media_ceq(in, S.air);
      const bool is_rcv = (o->inst->mask & side) != 0;
      const bool is_virt = mtl->type == SSOL_MATERIAL_VIRTUAL;
      double trans = 1;
      if(hit_t > 0) {
        const double ke = data_value(in.extinction, wl);
        if(ke > 0) trans = std::exp(-ke * hit_t);
      }
      inc[0] = prev[0] * trans;
      inc[1] = in_atm ? prev[1] : prev[1] * trans;
      inc[2] = !in_atm ? prev[2] : prev[2] * trans;
      double kabs;
      if(is_virt) {
        kabs = 0;
        for(int c = 0; c < 3; ++c) outw[c] = inc[c];
        ssol_medium_copy(&out, &in);
      } else {
        double prop; V nd = dir; int type;
        ssol_surface_fragment frag;
        bool use_frag;
        const V Ns = shading_inputs(S, gid, side, pos, dir, N, cb1, cb2, frag, use_frag);
        if(!shade(S, rng, j++, mtl, in, out, wl, -dir, N, prop, nd, type, Ns,
                  use_frag ? &frag : nullptr)) {
          res = RES_BAD_OP; break;
        }
        kabs = 1 - prop;
        outw[0] = inc[0] * prop; outw[1] = inc[1] * prop;
        outw[2] = is_rcv ? inc[2] * prop : inc[2];
        if(type) dir = nd;
      }
      if(is_rcv) {
        hit_rcv = true;
        /* update_mc (src/ssol_solver.c:708-785) */
        ctx.g[1].add(ireal, inc[0] - outw[0]);
        const double w[10] = {inc[0], inc[1], inc[2], inc[2] - inc[0], inc[1] - inc[0],
          inc[0] * kabs, inc[1] * kabs, inc[2] * kabs, (inc[2] - inc[0]) * kabs,
          (inc[1] - inc[0]) * kabs};
        McRcv1& r1s = rcv_side(ctx.rcv, o->inst, side);
        McRcv1& r2s = rcv_side(ms.rcv, o->inst, side);
        for(int q = 0; q < 10; ++q) { r1s.q[q].add(ireal, w[q]); r2s.q[q].add(ireal, w[q]); }
        if(o->inst->per_prim) {
          std::vector<McData>& pd = r1s.prims[o->shape][prim];
          if(pd.empty()) pd.resize(10);
          for(int q = 0; q < 10; ++q) pd[q].add(ireal, w[q]);
        }
      } else {
        ctx.g[5].add(ireal, inc[0] * kabs);
      }
      const bool zero = outw[0] == 0;
      bool last = false;
      if(!zero) {
        if(is_virt) tmin = std::nextafter(hit_t, DBL_MAX);
        else { tmin = 0; org = pos; rd = dir; }
        Self s2 = {gid, si, side, false, false};
        h = trace(S, org, rd, tmin, s2, false);
        if(!h.found) {
          if(path && track->inf > 0) vtx(pos + rd * track->inf, outw[0]);
          last = true;
          if(!media_ceq(out, S.air)) { res = RES_BAD_OP; break; }
        }
      }
      if(zero || last || !is_virt) {
        const double ab = prev[0] - inc[0];
        ctx.g[in_atm ? 4 : 5].add(ireal, ab);
        if(zero || last) break;
        for(int c = 0; c < 3; ++c) prev[c] = outw[c];
      }
      depth += is_virt ? 0 : 1;
      if(depth > interval && depth % interval == 1) {
        const double p = unif(rng.get(nr++, DOM_ROULETTE).x[0]);
        if(p > 0.5) { ++score; interval = 16; }
        else { apply_factor(ctx, ireal, 0); killed = true; break; }
      }
      if(seg >= 1000000) { res = RES_BAD_OP; break; }
      /* point_update_from_hit */
      si = h.sinst; o = &S.sinst[si]; prim = h.prim; gid = h.gid;
      cb1 = h.b1; cb2 = h.b2;
      N = unit(h.n);
      pos = org + rd * h.t;
      vtx(pos, outw[0]);
      side = dot(rd, N) < 0 ? 1 : 2;
      if(side == 2) N = -N;
      mtl = o->mtl[side - 1];
      hit_t = h.t;
      ssol_medium_copy(&in, &out);
    }
    if(res == RES_OK && !killed) ctx.g[3].add(ireal, outw[0]);
    if(path) path->type = hit_rcv ? SSOL_PATH_SUCCESS : SSOL_PATH_MISSING;
  }
  if(path && res != RES_OK) path->type = SSOL_PATH_ERROR;
  if(path && killed) path->v.clear(), path->type = (ssol_path_type)-1;
  ssol_medium_clear(&in);
  ssol_medium_clear(&out);
  if(res != RES_OK) return res;
  if(killed) return RES_OK;
  ctx.samp[samp_inst].cos.add(ireal, cosf);
  ctx.g[0].add(ireal, cosf);
  if(score) apply_factor(ctx, ireal, (double)(1u << score));
  return RES_OK;
}

void merge_rcv(McRcv& dst, McRcv& src, const ssol_instance* inst)
{
  for(int s = 0; s < 2; ++s) {
    if(!(inst->mask & (s == 0 ? 1 : 2))) continue;
    for(int q = 0; q < 10; ++q) dst.side[s].q[q].accum(src.side[s].q[q]);
    for(auto& sh : src.side[s].prims)
      for(auto& p : sh.second) {
        std::vector<McData>& d = dst.side[s].prims[sh.first][p.first];
        if(d.empty()) d.resize(10);
        for(int q = 0; q < 10; ++q) d[q].accum(p.second[q]);
      }
  }
}

} /* namespace */

/* ssol_solve (src/ssol_solver.c:1132-1361) */
API res_T ssol_solve(ssol_scene* scn, const ssp_rng* rng, const size_t n,
                     const size_t max_failed, const ssol_path_tracker* tracker,
                     ssol_estimator** out)
{
  if(!scn || !rng || !n || !out) return RES_BAD_ARG;
  Scene S;
  res_T res = make_scene(scn, S);
  if(res != RES_OK) return res;
  const int nth = (int)scn->dev->nthreads;
  std::vector<Ctx> ctx(nth);
  std::atomic<size_t> nfail{0};
  std::atomic<int> stop{0};
  const int64_t N = (int64_t)n;
  /* Path tracking (src/ssol_solver.c:1211-1220): negative lengths default to
   * 0.75 x the largest extent of the scene's bounding box. The first
   * min(N, 2^20) realisations are tracked, in realisation order. */
  TrackLen tl = {0, 0};
  std::vector<OPath> paths;
  if(tracker) {
    double ext = 0;
    for(int c = 0; c < 3; ++c) ext = std::max(ext, S.nodes[0].hi[c] - S.nodes[0].lo[c]);
    ext *= 0.75;
    tl.sun = tracker->sun_ray_length < 0 ? ext : tracker->sun_ray_length;
    tl.inf = tracker->infinite_ray_length < 0 ? ext : tracker->infinite_ray_length;
    paths.resize((size_t)std::min<int64_t>(N, int64_t(1) << 20));
  }
  #pragma omp parallel for schedule(static) num_threads(nth)
  for(int64_t i = 0; i < N; ++i) {
    if(stop.load()) continue;
    Ctx& c = ctx[omp_get_thread_num()];
    PathRng pr = {rng->pos + (uint64_t)i, rng->seed};
    OPath* pp = (size_t)i < paths.size() ? &paths[(size_t)i] : nullptr;
    const res_T r = realisation(S, c, (size_t)i, pr, &tl, pp);
    if(r != RES_OK) {
      apply_factor(c, (size_t)i, 0);
      if(r == RES_BAD_OP) {
        if(++nfail >= max_failed) stop = 1;
      } else stop = 1;
      continue;
    }
    c.nreal++;
  }
  ssol_estimator* e = new ssol_estimator();
  e->dev = scn->dev; scn->dev->ref.get();
  e->nfail = nfail.load();
  for(ssol_instance* inst : scn->inst) {
    if(inst->mask) e->rcv[inst];
    if(inst->sample) e->samp[inst];
  }
  for(Ctx& c : ctx) {
    for(int q = 0; q < 6; ++q) e->g[q].accum(c.g[q]);
    e->nreal += c.nreal;
    for(auto& r : c.rcv) merge_rcv(e->rcv[r.first], r.second, r.first);
    for(auto& s : c.samp) {
      McSamp& d = e->samp[s.first];
      d.cos.accum(s.second.cos); d.shadow.accum(s.second.shadow);
      d.nb += s.second.nb;
      for(auto& r : s.second.rcv) merge_rcv(d.rcv[r.first], r.second, r.first);
    }
  }
  e->sampled_area = S.area_rt;
  for(OPath& p : paths)
    if((int)p.type >= 0 && !p.v.empty()) e->paths.push_back(std::move(p));
  e->rng = new ssp_rng();
  e->rng->type = rng->type; e->rng->seed = rng->seed; e->rng->pos = rng->pos + n;
  *out = e;
  if(e->nfail > 0 && e->nfail >= max_failed) return RES_BAD_OP;
  return RES_OK;
}

/* Oracle of the primal objective of the B200 library's ssol_solve_adjoint
 * (no reference counterpart; test infrastructure only): first-bounce paths
 * sampled on a mirror, not shadowed, reflected once (shade(), scatter event
 * 0) and reaching `receiver` first on a receiving side whose material is a
 * mirror or matte; weight w0 x reflectivity x exp(-k t) x (1 - receiver
 * reflectivity); absorbed = mean of w, flux_map = bilinear splat of w on the
 * nx x ny cell centres of [lower, upper] in the receiver's local frame,
 * divided by N and the cell area. */
API res_T ssol_oracle_first_bounce
  (ssol_scene* scn, const ssp_rng* rng, const size_t n, const ssol_instance* receiver,
   const double lower[2], const double upper[2], const unsigned nx, const unsigned ny,
   double* absorbed, double* absorbed_se, unsigned long long* hits, double* flux_map)
{
  if(!scn || !rng || !n || !receiver || !lower || !upper || !nx || !ny || !absorbed
  || !absorbed_se || !hits || !flux_map) return RES_BAD_ARG;
  Scene S;
  res_T res = make_scene(scn, S);
  if(res != RES_OK) return res;
  Affine rxf, rinv;
  rxf = receiver->xf;
  if(!inverse(rxf, rinv)) return RES_BAD_ARG;
  const double cw = (upper[0] - lower[0]) / nx, ch = (upper[1] - lower[1]) / ny;
  const int nth = (int)scn->dev->nthreads;
  std::vector<std::vector<double>> maps(nth, std::vector<double>((size_t)nx * ny, 0.0));
  std::vector<double> sw(nth, 0.0), sw2(nth, 0.0), sh(nth, 0.0);
  const int64_t N = (int64_t)n;
  #pragma omp parallel for schedule(static) num_threads(nth)
  for(int64_t i = 0; i < N; ++i) {
    const int th = omp_get_thread_num();
    const PathRng rg = {rng->pos + (uint64_t)i, rng->seed};
    const Block r0 = rg.get(0, DOM_PRIMARY);
    int k = (int)(((uint64_t)(r0.x[0] >> 8) * (uint64_t)S.samp.size()) >> 24);
    if(!((float)unif(r0.x[1]) < S.aprob[k])) k = S.aidx[k];
    const OSamp& st = S.samp[k];
    const double sa = std::sqrt(unif(r0.x[2]));
    const double b2 = sa * unif(r0.x[3]), b1 = sa - b2;
    V pos = st.v0 + st.e1 * b1 + st.e2 * b2;
    const Block r1 = rg.get(1, DOM_PRIMARY);
    const V dir = sun_dir(S, rg, r1);
    const double wl = wl_sample(S, unif(r1.x[2]));
    const OSInst* o = &S.sinst[st.sinst];
    V N = st.n;
    if(o->punched) {
      const OQuad& Q = S.quads[o->quad];
      V pl = xpoint(Q.w2l, pos);
      pl.z = qz(o->shape->quad.type, o->shape->q, pl.x, pl.y);
      N = unit(xvec_t(Q.w2l, qgrad(o->shape->quad.type, o->shape->q, pl)));
      pos = xpoint(Q.l2w, pl);
    }
    int side = 1;
    if(!(dot(N, dir) < 0)) { side = 2; N = -N; }
    const ssol_material* mtl = o->mtl[side - 1];
    if(mtl->type != SSOL_MATERIAL_MIRROR) continue;
    const double spc = o->punched ? std::fabs(dot(st.n, N)) : 1.0;
    double w = S.sun->dni * S.area_proxy
      * std::fabs(dot(N, dir) / (spc * dot(S.sun_dir, dir)));
    const Self self = {st.gid, st.sinst, side, true, true};
    if(trace(S, pos, -dir, 0, self, true).found) continue;
    ssol_medium in = S.air, out = S.air;
    double prop; V rd = dir; int type;
    ssol_surface_fragment frag;
    bool use_frag;
    const V Ns = shading_inputs(S, st.gid, side, pos, dir, N, b1, b2, frag, use_frag);
    if(!shade(S, rg, 0, mtl, in, out, wl, -dir, N, prop, rd, type, Ns,
              use_frag ? &frag : nullptr) || !(prop > 0)) continue;
    w *= prop;
    const Self s2 = {st.gid, st.sinst, side, false, false};
    const OHit h = trace(S, pos, rd, 0, s2, false);
    if(!h.found) continue;
    const OSInst& hs = S.sinst[h.sinst];
    if(hs.inst != receiver || hs.punched) continue;
    const int hside = dot(rd, h.n) < 0 ? 1 : 2;
    if(!(receiver->mask & hside)) continue;
    const ssol_material* hm = hs.mtl[hside - 1];
    if(hm->type != SSOL_MATERIAL_MIRROR && hm->type != SSOL_MATERIAL_MATTE) continue;
    const double kext = data_value(S.air.extinction, wl);
    if(kext > 0) w *= std::exp(-kext * h.t);
    w *= 1 - shader(S, hm, 0, wl);
    sw[th] += w; sw2[th] += w * w; sh[th] += 1;
    const V p = pos + rd * h.t;
    const V pl = xpoint(rinv, p);
    const double fx = (pl.x - lower[0]) / cw - 0.5, fy = (pl.y - lower[1]) / ch - 0.5;
    const int i0 = (int)std::floor(fx), j0 = (int)std::floor(fy);
    const double tx = fx - i0, ty = fy - j0;
    for(int dj = 0; dj < 2; ++dj)
      for(int di = 0; di < 2; ++di) {
        const int ci = i0 + di, cj = j0 + dj;
        if(ci < 0 || cj < 0 || ci >= (int)nx || cj >= (int)ny) continue;
        maps[th][(size_t)cj * nx + ci] += w * (di ? tx : 1 - tx) * (dj ? ty : 1 - ty);
      }
  }
  double a = 0, a2 = 0, hh = 0;
  for(int t = 0; t < nth; ++t) { a += sw[t]; a2 += sw2[t]; hh += sh[t]; }
  const double mean = a / (double)n;
  *absorbed = mean;
  *absorbed_se = std::sqrt(std::max(0.0, a2 / (double)n - mean * mean) / (double)n);
  *hits = (unsigned long long)hh;
  for(size_t c = 0; c < (size_t)nx * ny; ++c) {
    double v = 0;
    for(int t = 0; t < nth; ++t) v += maps[t][c];
    flux_map[c] = v / ((double)n * cw * ch);
  }
  return RES_OK;
}

/*******************************************************************************
 * Estimator read-out (src/ssol_estimator.c, src/ssol_mc_receiver.c)
 ******************************************************************************/
static ssol_mc_result res_of(McData d, double n)
{
  d.flush();
  ssol_mc_result r;
  if(n <= 0) { r.E = r.V = r.SE = 0; return r; }
  r.E = d.w / n;
  r.V = std::max(d.w2 / n - r.E * r.E, 0.0);
  r.SE = std::sqrt(r.V / n);
  return r;
}

API res_T ssol_estimator_ref_get(ssol_estimator* e)
{ if(!e) return RES_BAD_ARG; e->ref.get(); return RES_OK; }
API res_T ssol_estimator_ref_put(ssol_estimator* e)
{
  if(!e) return RES_BAD_ARG;
  if(e->ref.put()) {
    ssol_device* d = e->dev;
    if(e->rng) ssp_rng_ref_put(e->rng);
    delete e; ssol_device_ref_put(d);
  }
  return RES_OK;
}
API res_T ssol_estimator_get_mc_global(ssol_estimator* e, ssol_mc_global* g)
{
  if(!e || !g) return RES_BAD_ARG;
  ssol_mc_result* r = &g->cos_factor;
  for(int q = 0; q < 6; ++q) r[q] = res_of(e->g[q], (double)e->nreal);
  return RES_OK;
}
API res_T ssol_estimator_get_mc_receiver(ssol_estimator* e, const ssol_instance* i,
  const ssol_side_flag side, ssol_mc_receiver* rcv)
{
  if(!e || !i || !rcv || !(i->mask & (int)side)) return RES_BAD_ARG;
  std::memset(rcv, 0, sizeof(*rcv));
  auto it = e->rcv.find(i);
  if(it == e->rcv.end()) return RES_OK;
  McRcv1& s = it->second.side[side == SSOL_FRONT ? 0 : 1];
  ssol_mc_result* r = &rcv->incoming_flux;
  for(int q = 0; q < 10; ++q) r[q] = res_of(s.q[q], (double)e->nreal);
  rcv->mc__ = &s; rcv->N__ = e->nreal; rcv->instance__ = i;
  return RES_OK;
}
API res_T ssol_estimator_get_mc_sampled_x_receiver(ssol_estimator* e,
  const ssol_instance* si, const ssol_instance* ri, const ssol_side_flag side,
  ssol_mc_receiver* rcv)
{
  if(!e || !si || !ri || !rcv || (side != SSOL_FRONT && side != SSOL_BACK)
  || !si->sample || !(ri->mask & (int)side)) return RES_BAD_ARG;
  std::memset(rcv, 0, sizeof(*rcv));
  auto it = e->samp.find(si);
  if(it == e->samp.end()) return RES_BAD_ARG;
  auto jt = it->second.rcv.find(ri);
  if(jt == it->second.rcv.end()) return RES_OK;
  McRcv1& s = jt->second.side[side == SSOL_FRONT ? 0 : 1];
  ssol_mc_result* r = &rcv->incoming_flux;
  for(int q = 0; q < 10; ++q) r[q] = res_of(s.q[q], (double)e->nreal);
  rcv->mc__ = &s; rcv->N__ = it->second.nb;
  return RES_OK;
}
API res_T ssol_estimator_get_realisation_count(const ssol_estimator* e, size_t* c)
{ if(!e || !c) return RES_BAD_ARG; *c = e->nreal; return RES_OK; }
API res_T ssol_estimator_get_failed_count(const ssol_estimator* e, size_t* c)
{ if(!e || !c) return RES_BAD_ARG; *c = e->nfail; return RES_OK; }
API res_T ssol_estimator_get_sampled_area(const ssol_estimator* e, double* a)
{ if(!e || !a) return RES_BAD_ARG; *a = e->sampled_area; return RES_OK; }
API res_T ssol_estimator_get_sampled_count(const ssol_estimator* e, size_t* c)
{ if(!e || !c) return RES_BAD_ARG; *c = e->samp.size(); return RES_OK; }
API res_T ssol_estimator_get_mc_sampled(ssol_estimator* e, const ssol_instance* i,
                                        ssol_mc_sampled* s)
{
  if(!e || !i || !s) return RES_BAD_ARG;
  auto it = e->samp.find(i);
  if(it == e->samp.end()) return RES_BAD_ARG;
  s->nb_samples = it->second.nb;
  s->cos_factor = res_of(it->second.cos, (double)s->nb_samples);
  s->shadowed = res_of(it->second.shadow, (double)e->nreal);
  return RES_OK;
}
API res_T ssol_estimator_get_rng_state(const ssol_estimator* e, const ssp_rng** r)
{ if(!e || !r) return RES_BAD_ARG; *r = e->rng; return RES_OK; }
API res_T ssol_estimator_get_tracked_paths_count(const ssol_estimator* e, size_t* n)
{ if(!e || !n) return RES_BAD_ARG; *n = e->paths.size(); return RES_OK; }
/* src/ssol_estimator.c:280-322 */
API res_T ssol_estimator_get_tracked_path(const ssol_estimator* e, const size_t i,
                                          ssol_path* p)
{
  if(!e || i >= e->paths.size() || !p) return RES_BAD_ARG;
  p->path__ = &e->paths[i];
  return RES_OK;
}
API res_T ssol_path_get_vertices_count(const ssol_path* p, size_t* n)
{
  if(!p || !n) return RES_BAD_ARG;
  *n = static_cast<const OPath*>(p->path__)->v.size();
  return RES_OK;
}
API res_T ssol_path_get_vertex(const ssol_path* p, const size_t i, ssol_path_vertex* v)
{
  if(!p || !v) return RES_BAD_ARG;
  const OPath* o = static_cast<const OPath*>(p->path__);
  if(i >= o->v.size()) return RES_BAD_ARG;
  *v = o->v[i];
  return RES_OK;
}
API res_T ssol_path_get_type(const ssol_path* p, ssol_path_type* t)
{
  if(!p || !t) return RES_BAD_ARG;
  *t = static_cast<const OPath*>(p->path__)->type;
  return RES_OK;
}
API res_T ssol_mc_receiver_get_mc_shape(ssol_mc_receiver* rcv, const ssol_shape* s,
                                        ssol_mc_shape* mc)
{
  if(!rcv || !s || !mc || !rcv->instance__) return RES_BAD_ARG;
  bool has = false;
  for(const OShaded& x : rcv->instance__->obj->shaded) has = has || x.shape == s;
  if(!has) return RES_BAD_ARG;
  McRcv1* r = (McRcv1*)rcv->mc__;
  mc->N__ = rcv->N__;
  mc->mc__ = nullptr;
  if(r) { auto it = r->prims.find(s); if(it != r->prims.end()) mc->mc__ = &it->second; }
  mc->shape__ = s;
  return RES_OK;
}
API res_T ssol_mc_shape_get_mc_primitive(ssol_mc_shape* sh, const unsigned i,
                                         ssol_mc_primitive* p)
{
  if(!sh || !p || !sh->shape__) return RES_BAD_ARG;
  const ssol_shape* s = sh->shape__;
  if(i >= s->ids.size() / 3) return RES_BAD_ARG;
  std::memset(p, 0, sizeof(*p));
  auto* m = (std::map<unsigned, std::vector<McData>>*)sh->mc__;
  if(!m) return RES_OK;
  auto it = m->find(i);
  if(it == m->end()) return RES_OK;
  const V a = v3(s->pos[s->ids[i*3]*3], s->pos[s->ids[i*3]*3+1], s->pos[s->ids[i*3]*3+2]);
  const V b = v3(s->pos[s->ids[i*3+1]*3], s->pos[s->ids[i*3+1]*3+1], s->pos[s->ids[i*3+1]*3+2]);
  const V c = v3(s->pos[s->ids[i*3+2]*3], s->pos[s->ids[i*3+2]*3+1], s->pos[s->ids[i*3+2]*3+2]);
  const V n = cross(b - a, c - a);
  const double area = 0.5 * std::sqrt(dot(n, n));
  ssol_mc_result* r = &p->incoming_flux;
  for(int q = 0; q < 10; ++q) {
    r[q] = res_of(it->second[q], (double)sh->N__);
    r[q].E /= area; r[q].V /= area * area; r[q].SE /= area;
  }
  return RES_OK;
}

/*******************************************************************************
 * Camera, image and the preview renderers (src/ssol_camera.c,
 * src/ssol_image.c, src/ssol_draw.c, src/ssol_draw_draft.c,
 * src/ssol_draw_pt.c), with the same random streams as the B200 library:
 * draft sub-pixel offsets from Philox (i, 0, 0, 4) with key 0; path tracer
 * streams keyed by the seed with id = pixel x spp + sample (domains 5:
 * sub-pixel position, 6: wavelength of an attempt, 7: BSDF sample and 8:
 * roulette at event (attempt << 20) | bounce). Star-SF's rendering BSDFs
 * are restated as in the library (Lambertian, specular, dielectric and
 * thin-slab samplers, Cook-Torrance microfacet with V-cavity G and the
 * Walter et al. 2007 estimator weight).
 ******************************************************************************/
struct ssol_camera {
  Ref ref; ssol_device* dev;
  float x[3] = {0, 0, 0}, y[3] = {0, 0, 0}, z[3] = {0, 0, 0}, pos[3] = {0, 0, 0};
  float fov = 0, rcp_ratio = 1;
};
struct ssol_image {
  Ref ref; ssol_device* dev;
  std::vector<double> mem; size_t w = 0, h = 0;
  ssol_pixel_format fmt = SSOL_PIXEL_FORMATS_COUNT__;
};

namespace {

float f3norm(float o[3], const float v[3])
{
  const float l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  if(l == 0.f) return l;
  for(int c = 0; c < 3; ++c) o[c] = v[c] / l;
  return l;
}

void f3cross(float o[3], const float a[3], const float b[3])
{
  const float r[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2],
                      a[0] * b[1] - a[1] * b[0]};
  std::memcpy(o, r, sizeof(r));
}

/* camera_ray (src/ssol_camera.h:41-62), FP32 without contraction */
void cam_ray(const ssol_camera* c, float sx, float sy, float d[3])
{
  const float fx = sx * 2.f - 1.f, fy = sy * 2.f - 1.f;
  for(int k = 0; k < 3; ++k) d[k] = (c->x[k] * fx + c->y[k] * fy) + c->z[k];
  const float l = std::sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]);
  for(int k = 0; k < 3; ++k) d[k] = d[k] / l;
}

enum { DOM_DRAW_OFFSET = 4, DOM_DRAW_PIXEL = 5, DOM_DRAW_WL = 6, DOM_DRAW_BSDF = 7,
       DOM_DRAW_RR = 8 };
const int DRAW_MAX_BOUNCES = 1000, DRAW_MAX_FAILURES = 100;

/* Shading normal and fragment of a hit (src/ssol_material.c:551-655 with P
 * the hit point) */
V draw_normal(const Scene& S, const OHit& h, int side, V pos, V dir, V Ng,
              ssol_surface_fragment& frag, bool& use_frag)
{
  return shading_inputs(S, h.gid, side, pos, dir, Ng, h.b1, h.b2, frag, use_frag);
}

struct DBsdf { const ssol_material* m; double refl, rough; };

DBsdf draw_bsdf(const Scene& S, const ssol_material* m, double wl,
                const ssol_surface_fragment* frag)
{
  DBsdf f = {m, 0, 0};
  if(m->type != SSOL_MATERIAL_MIRROR && m->type != SSOL_MATERIAL_MATTE) return f;
  if(frag) {
    if(m->refl) m->refl(m->dev, m->buf, wl, frag, &f.refl);
    if(m->type == SSOL_MATERIAL_MIRROR && m->rough) m->rough(m->dev, m->buf, wl, frag, &f.rough);
  } else {
    f.refl = shader(S, m, 0, wl);
    if(m->type == SSOL_MATERIAL_MIRROR) f.rough = shader(S, m, 1, wl);
  }
  return f;
}

double mf_d(int distrib, double a, double nh)
{
  if(!(nh > 0)) return 0;
  const double c2 = nh * nh, t2 = (1 - c2) / c2, a2 = a * a;
  const double inv = 1 / (M_PI * a2 * c2 * c2);
  if(distrib == SSOL_MICROFACET_BECKMANN) return std::exp(-t2 / a2) * inv;
  return t2 <= a2 ? inv : 0;
}

double mf_g(double nh, double no, double ni, double oh)
{
  if(!(oh > 0)) return 0;
  return std::min(1.0, std::min(2 * nh * no / oh, 2 * nh * ni / oh));
}

double draw_eval(const DBsdf& f, V wo, V N, V wi)
{
  const double no = dot(wo, N), ni = dot(wi, N);
  if(!(no > 0) || !(ni > 0)) return 0;
  if(f.m->type == SSOL_MATERIAL_MATTE) return f.refl / M_PI;
  if(f.m->type == SSOL_MATERIAL_MIRROR && f.rough > 0) {
    const V h = unit(wo + wi);
    const double nh = dot(N, h), oh = dot(wo, h);
    return f.refl * mf_d(f.m->distrib, f.rough, nh) * mf_g(nh, no, ni, oh) / (4 * no * ni);
  }
  return 0;
}

/* Returns the weight; type 1 reflection, 2 transmission */
double draw_sample(const DBsdf& f, const Block& r, double wl, V wo, V N, V& wi, int& type,
                   bool& to_inside)
{
  const ssol_material* m = f.m;
  type = 0; to_inside = false; wi = N;
  const double ci = dot(wo, N);
  if(!(ci > 0)) return 0;
  V b1, b2;
  switch(m->type) {
    case SSOL_MATERIAL_MIRROR: {
      type = 1;
      if(f.rough == 0) { wi = N * (2 * ci) - wo; return f.refl; }
      const double a = f.rough, u0 = unif(r.x[0]);
      const double t2 = m->distrib == SSOL_MICROFACET_BECKMANN ? -a * a * std::log(1 - u0)
                                                               : a * a * u0;
      const double ct = 1 / std::sqrt(1 + t2), st = std::sqrt(t2) * ct;
      const double ph = 2 * M_PI * unif(r.x[1]);
      onb(N, b1, b2);
      const V h = b1 * (std::cos(ph) * st) + b2 * (std::sin(ph) * st) + N * ct;
      const double oh = dot(wo, h);
      wi = h * (2 * oh) - wo;
      const double ni = dot(wi, N);
      if(!(oh > 0) || !(ni > 0)) return 0;
      return f.refl * mf_g(ct, ci, ni, oh) * oh / (ci * ct);
    }
    case SSOL_MATERIAL_MATTE: {
      const double u0 = unif(r.x[0]), rad = std::sqrt(u0);
      const double ph = 2 * M_PI * unif(r.x[1]);
      onb(N, b1, b2);
      wi = b1 * (rad * std::cos(ph)) + b2 * (rad * std::sin(ph)) + N * std::sqrt(1 - u0);
      type = 1;
      return f.refl;
    }
    case SSOL_MATERIAL_DIELECTRIC: {
      const double ei = data_value(m->out.refractive_index, wl);
      const double et = data_value(m->in.refractive_index, wl);
      const double eta = ei / et, s2 = eta * eta * (1 - ci * ci);
      double F = 1, ct = 0;
      if(s2 < 1) { ct = std::sqrt(1 - s2); F = fresnel(ci, ct, ei, et); }
      if(unif(r.x[0]) < F) { wi = N * (2 * ci) - wo; type = 1; }
      else { wi = unit(N * (eta * ci - ct) - wo * eta); type = 2; to_inside = true; }
      return 1;
    }
    case SSOL_MATERIAL_THIN_DIELECTRIC: {
      const double ei = data_value(m->out.refractive_index, wl);
      const double et = data_value(m->slab.refractive_index, wl);
      const double al = data_value(m->slab.extinction, wl);
      const double eta = ei / et, s2 = eta * eta * (1 - ci * ci);
      double Rt = 1, Tt = 0;
      if(s2 < 1) {
        const double ct = std::sqrt(1 - s2), F = fresnel(ci, ct, ei, et);
        const double tau = std::exp(-al * m->thickness / ct);
        const double den = 1 - F * F * tau * tau;
        Rt = F + (1 - F) * (1 - F) * F * tau * tau / den;
        Tt = (1 - F) * (1 - F) * tau / den;
      }
      const double p = Rt + Tt;
      if(p > 0 && unif(r.x[0]) * p < Rt) { wi = N * (2 * ci) - wo; type = 1; }
      else { wi = -wo; type = 2; }
      return p;
    }
    default: return 0;
  }
}

/* Li of src/ssol_draw_pt.c:124-290; false on an inconsistent medium */
bool draw_li(const Scene& S, const PathRng& rng, uint32_t attempt, V org, V dir,
             V up, double& L)
{
  L = 0;
  double thr = 1;
  bool roulette = false;
  const double wl = wl_sample(S, unif(rng.get(attempt, DOM_DRAW_WL).x[0]));
  ssol_medium medium = S.air;
  Self self = {-1, -1, 0, true, false};
  const V to_sun = -S.sun_dir;
  for(int b = 0; b < DRAW_MAX_BOUNCES; ++b) {
    const OHit h = trace(S, org, dir, 0, self, false);
    if(!h.found) {
      if(dot(dir, up) > 0) L += thr * 1e-1;
      break;
    }
    const double kext = data_value(medium.extinction, wl);
    if(kext > 0) {
      thr *= std::exp(-kext * h.t);
      if(thr <= 0) break;
    }
    const V wo_in = unit(dir);
    V Ng = unit(h.n);
    int side = 1;
    if(!(dot(Ng, wo_in) < 0)) { side = 2; Ng = -Ng; }
    const V pos = org + dir * h.t;
    ssol_surface_fragment frag;
    bool use_frag = false;
    const V N = draw_normal(S, h, side, pos, wo_in, Ng, frag, use_frag);
    if(dot(N, wo_in) > 0) break;
    const ssol_material* m = S.sinst[h.sinst].mtl[side - 1];
    const DBsdf f = draw_bsdf(S, m, wl, use_frag ? &frag : nullptr);
    if(m->type == SSOL_MATERIAL_DIELECTRIC && !media_ceq(medium, m->out)) return false;
    self.gid = h.gid; self.sinst = h.sinst; self.side = side;
    org = pos;
    const V wo = -wo_in;
    const double c = dot(to_sun, N);
    if(c >= 0 && !(std::fabs(c) <= 1e-6)) {
      const double fv = draw_eval(f, wo, N, to_sun);
      if(fv > 0 && !trace(S, org, to_sun, 0, self, true).found) L += thr * fv * c;
    }
    const uint32_t ev = (attempt << 20) | (uint32_t)b;
    V wi;
    int type;
    bool inside;
    double w = draw_sample(f, rng.get(ev, DOM_DRAW_BSDF), wl, wo, N, wi, type, inside);
    const double cg = dot(Ng, wi);
    if((cg > 0 && type == 2) || (cg < 0 && type == 1)) w = 0;
    dir = wi;
    if(inside) ssol_medium_copy(&medium, &m->in);
    const double cn = std::fabs(dot(wi, N));
    if(!roulette) thr *= cn * w;
    else {
      if(unif(rng.get(ev, DOM_DRAW_RR).x[0]) >= w) break;
      thr *= cn;
    }
    if(thr <= 0) break;
    if(!roulette) roulette = thr < 0.1;
  }
  return true;
}

size_t pow2_up(size_t v) { size_t p = 1; while(p < v) p <<= 1; return p; }

uint32_t morton_even(uint32_t code)
{
  uint32_t x = code & 0x55555555u;
  x = (x | (x >> 1)) & 0x33333333u;
  x = (x | (x >> 2)) & 0x0F0F0F0Fu;
  x = (x | (x >> 4)) & 0x00FF00FFu;
  x = (x | (x >> 8)) & 0x0000FFFFu;
  return x;
}

/* Whole image, then the writer per 32 x 32 tile in Morton order */
res_T draw_image(ssol_scene* scn, ssol_camera* cam, size_t W, size_t H, size_t spp,
                 bool pt, const double* up, ssol_write_pixels_T writer, void* data)
{
  Scene S;
  const res_T r = make_scene(scn, S, false);
  if(r != RES_OK) return r;
  std::vector<double> img(W * H * 3);
  std::vector<float> off(spp * 2);
  for(size_t i = 0; i < spp; ++i) {
    const Block b = philox((uint32_t)i, (uint32_t)(i >> 32), 0, DOM_DRAW_OFFSET, 0, 0);
    off[2 * i] = (float)(b.x[0] >> 8) * (1.0f / 16777216.0f);
    off[2 * i + 1] = (float)(b.x[1] >> 8) * (1.0f / 16777216.0f);
  }
  const float pw = 1.f / (float)W, ph = 1.f / (float)H;
  const V cpos = v3(cam->pos[0], cam->pos[1], cam->pos[2]);
  const V vup = up ? v3((float)up[0], (float)up[1], (float)up[2]) : v3(0, 0, 0);
  #pragma omp parallel for schedule(dynamic, 64)
  for(long long p = 0; p < (long long)(W * H); ++p) {
    const size_t px = (size_t)p % W, py = (size_t)p / W;
    double sum = 0;
    bool failed = false;
    for(size_t s = 0; s < spp && !failed; ++s) {
      float sx, sy;
      PathRng rng = {(uint64_t)p * spp + s, 0};
      if(pt) {
        const Block j = rng.get(0, DOM_DRAW_PIXEL);
        sx = ((float)px + (float)(j.x[0] >> 8) * (1.0f / 16777216.0f)) * pw;
        sy = ((float)py + (float)(j.x[1] >> 8) * (1.0f / 16777216.0f)) * ph;
      } else {
        sx = ((float)px + off[2 * s]) * pw;
        sy = ((float)py + off[2 * s + 1]) * ph;
      }
      float df[3];
      cam_ray(cam, sx, sy, df);
      const V d = v3(df[0], df[1], df[2]);
      if(pt) {
        double L = 0;
        bool ok = false;
        for(uint32_t a = 0; a < (uint32_t)DRAW_MAX_FAILURES && !ok; ++a)
          ok = draw_li(S, rng, a, cpos, d, vup, L);
        if(!ok) failed = true;
        else sum += L;
      } else {
        const Self self = {-1, -1, 0, true, false};
        const OHit h = trace(S, cpos, d, 0, self, false);
        if(!h.found) continue;
        const V wi = unit(d);
        V N = unit(h.n);
        int side = 1;
        if(!(dot(N, wi) < 0)) { N = -N; side = 2; }
        ssol_surface_fragment frag;
        bool use_frag;
        N = draw_normal(S, h, side, cpos + d * h.t, wi, N, frag, use_frag);
        sum += std::max(dot(N, -wi), 0.0);
      }
    }
    double* o = &img[(size_t)p * 3];
    if(failed) { o[0] = 1; o[1] = 1; o[2] = 0; }
    else { const double v = sum / (double)spp; o[0] = v; o[1] = v; o[2] = v; }
  }
  const size_t T = 32, ntx = (W + T - 1) / T, nty = (H + T - 1) / T;
  size_t nt = pow2_up(std::max(ntx, nty));
  nt *= nt;
  std::vector<double> tile(T * T * 3);
  for(size_t code = 0; code < nt; ++code) {
    size_t org[2] = {morton_even((uint32_t)code), morton_even((uint32_t)(code >> 1))};
    if(org[0] >= ntx || org[1] >= nty) continue;
    org[0] *= T; org[1] *= T;
    const size_t sz[2] = {std::min(T, W - org[0]), std::min(T, H - org[1])};
    for(size_t y = 0; y < sz[1]; ++y)
      std::memcpy(&tile[y * sz[0] * 3], &img[((org[1] + y) * W + org[0]) * 3],
                  sz[0] * 3 * sizeof(double));
    const res_T wr = writer(data, org, sz, SSOL_PIXEL_DOUBLE3, tile.data());
    if(wr != RES_OK) return wr;
  }
  return RES_OK;
}

bool scene_ok(const ssol_scene* s)
{
  return s->sun && s->sun->spec && s->sun->dni > 0;
}

double map_addr(double a, ssol_address_mode mode)
{
  if(mode == SSOL_ADDRESS_CLAMP) return std::min(std::max(a, 0.0), std::nextafter(1.0, 0.0));
  double i, f = std::modf(a, &i);
  if(f < 0) f = 1.0 + f;
  return f < 1.0 ? f : std::nextafter(1.0, 0.0);
}

} /* namespace */

API res_T ssol_camera_create(ssol_device* d, ssol_camera** out)
{
  if(!d || !out) return RES_BAD_ARG;
  ssol_camera* c = new ssol_camera();
  c->dev = d; d->ref.get();
  c->rcp_ratio = 1.f; c->fov = (float)(M_PI / 2.0);
  const double p[3] = {0, 0, 0}, t[3] = {0, 0, -1}, u[3] = {0, 1, 0};
  ssol_camera_look_at(c, p, t, u);
  *out = c;
  return RES_OK;
}
API res_T ssol_camera_ref_get(ssol_camera* c) { if(!c) return RES_BAD_ARG; c->ref.get(); return RES_OK; }
API res_T ssol_camera_ref_put(ssol_camera* c)
{
  if(!c) return RES_BAD_ARG;
  if(c->ref.put()) { ssol_device* d = c->dev; delete c; ssol_device_ref_put(d); }
  return RES_OK;
}
API res_T ssol_camera_set_proj_ratio(ssol_camera* c, const double r)
{
  float y[3];
  if(!c || r <= 0 || f3norm(y, c->y) <= 0) return RES_BAD_ARG;
  c->rcp_ratio = (float)(1.0 / r);
  for(int k = 0; k < 3; ++k) c->y[k] = y[k] * c->rcp_ratio;
  return RES_OK;
}
API res_T ssol_camera_set_fov(ssol_camera* c, const double fov)
{
  float z[3];
  if(!c || (float)fov <= 0 || f3norm(z, c->z) <= 0) return RES_BAD_ARG;
  const float depth = (float)(1.0 / std::tan(fov * 0.5));
  for(int k = 0; k < 3; ++k) c->z[k] = z[k] * depth;
  c->fov = (float)fov;
  return RES_OK;
}
API res_T ssol_camera_look_at(ssol_camera* c, const double pos[3], const double tgt[3],
                              const double up[3])
{
  if(!c || !pos || !tgt || !up) return RES_BAD_ARG;
  float p[3], u[3], x[3], y[3], z[3], d[3];
  for(int k = 0; k < 3; ++k) {
    p[k] = (float)pos[k]; u[k] = (float)up[k];
    d[k] = (float)tgt[k] - p[k];
  }
  if(f3norm(z, d) <= 0) return RES_BAD_ARG;
  f3cross(d, z, u);
  if(f3norm(x, d) <= 0) return RES_BAD_ARG;
  f3cross(d, z, x);
  if(f3norm(y, d) <= 0) return RES_BAD_ARG;
  const float depth = (float)(1.0 / std::tan(c->fov * 0.5));
  for(int k = 0; k < 3; ++k) {
    c->x[k] = x[k]; c->y[k] = y[k] * c->rcp_ratio; c->z[k] = z[k] * depth; c->pos[k] = p[k];
  }
  return RES_OK;
}

API res_T ssol_image_create(ssol_device* d, ssol_image** out)
{
  if(!d || !out) return RES_BAD_ARG;
  ssol_image* i = new ssol_image();
  i->dev = d; d->ref.get();
  *out = i;
  return RES_OK;
}
API res_T ssol_image_ref_get(ssol_image* i) { if(!i) return RES_BAD_ARG; i->ref.get(); return RES_OK; }
API res_T ssol_image_ref_put(ssol_image* i)
{
  if(!i) return RES_BAD_ARG;
  if(i->ref.put()) { ssol_device* d = i->dev; delete i; ssol_device_ref_put(d); }
  return RES_OK;
}
API res_T ssol_image_setup(ssol_image* i, const size_t w, const size_t h,
                           const ssol_pixel_format f)
{
  if(!i || !w || !h || (unsigned)f >= SSOL_PIXEL_FORMATS_COUNT__) return RES_BAD_ARG;
  i->mem.assign(w * h * 3, 0.0);
  i->w = w; i->h = h; i->fmt = f;
  return RES_OK;
}
API res_T ssol_image_get_layout(const ssol_image* i, ssol_image_layout* l)
{
  if(!i || !l) return RES_BAD_ARG;
  l->row_pitch = i->w * sizeof(double[3]); l->offset = 0; l->size = i->w * i->h;
  l->width = i->w; l->height = i->h; l->pixel_format = i->fmt;
  return RES_OK;
}
API res_T ssol_image_map(const ssol_image* i, char** m)
{
  if(!i || !m) return RES_BAD_ARG;
  *m = (char*)i->mem.data();
  return RES_OK;
}
API res_T ssol_image_unmap(const ssol_image* i) { return i ? RES_OK : RES_BAD_ARG; }
API res_T ssol_image_sample(const ssol_image* i, const ssol_filter_mode filter,
                            const ssol_address_mode au, const ssol_address_mode av,
                            const double uv[2], void* val)
{
  if(!i || !uv || !val || i->fmt != SSOL_PIXEL_DOUBLE3 || i->mem.empty()) return RES_BAD_ARG;
  double* o = (double*)val;
  auto px = [&](size_t x, size_t y) { return &i->mem[(y * i->w + x) * 3]; };
  const double x0 = map_addr(uv[0], au) * (double)i->w, y0 = map_addr(uv[1], av) * (double)i->h;
  if(filter == SSOL_FILTER_NEAREST) {
    const double* z = px((size_t)x0, (size_t)y0);
    for(int k = 0; k < 3; ++k) o[k] = z[k];
    return RES_OK;
  }
  const double x1 = map_addr(uv[0] + 1.0 / (double)i->w, au) * (double)i->w;
  const double y1 = map_addr(uv[1] + 1.0 / (double)i->h, av) * (double)i->h;
  const double *a = px((size_t)x0, (size_t)y0), *b = px((size_t)x0, (size_t)y1);
  const double *c = px((size_t)x1, (size_t)y0), *e = px((size_t)x1, (size_t)y1);
  double ip;
  const double s = std::modf(x0, &ip), t = std::modf(y0, &ip);
  for(int k = 0; k < 3; ++k)
    o[k] = (1 - s) * ((1 - t) * a[k] + t * b[k]) + s * ((1 - t) * c[k] + t * e[k]);
  return RES_OK;
}
API res_T ssol_image_write(void* image, const size_t org[2], const size_t sz[2],
                           const ssol_pixel_format fmt, const void* pixels)
{
  ssol_image* i = (ssol_image*)image;
  if(!i || !org || !sz || !pixels || fmt != i->fmt || i->mem.empty()) return RES_BAD_ARG;
  if(org[0] + sz[0] > i->w || org[1] + sz[1] > i->h) return RES_BAD_ARG;
  const double* src = (const double*)pixels;
  for(size_t y = 0; y < sz[1]; ++y)
    std::memcpy(&i->mem[((org[1] + y) * i->w + org[0]) * 3], src + y * sz[0] * 3,
                sz[0] * 3 * sizeof(double));
  return RES_OK;
}

API res_T ssol_draw_draft(ssol_scene* scn, ssol_camera* cam, const size_t w, const size_t h,
                          const size_t spp, ssol_write_pixels_T writer, void* data)
{
  if(!scn || !spp || !scene_ok(scn)) return RES_BAD_ARG;
  if(!cam || !w || !h || !writer) return RES_BAD_ARG;
  return draw_image(scn, cam, w, h, spp, false, nullptr, writer, data);
}

API res_T ssol_draw_pt(ssol_scene* scn, ssol_camera* cam, const size_t w, const size_t h,
                       const size_t spp, const double up[3], ssol_write_pixels_T writer,
                       void* data)
{
  if(!scn || !up || !scene_ok(scn)) return RES_BAD_ARG;
  if(!cam || !w || !h || !spp || !writer) return RES_BAD_ARG;
  return draw_image(scn, cam, w, h, spp, true, up, writer, data);
}
