/*
 * kernels.cu - the sm_100a realisation loop of `ssol_solve`.
 *
 * One thread traces whole optical paths, persistent over a grid-stride range
 * of realisations. Per path it restates, on the flat device scene of
 * device_scene.h:
 *   point_init             src/ssol_solver.c:207-358
 *   trace_radiative_path   src/ssol_solver.c:873-1127
 *   point_update_from_hit  src/ssol_solver.c:360-411
 *   point_shade            src/ssol_solver.c:419-494
 *   update_mc              src/ssol_solver.c:708-785
 *   hit_filter_function    src/ssol_scene.c:439-535
 *   quadric intersection   src/ssol_shape.c:864-1244, 1408-1494
 *   sun direction samplers src/ssol_ranst_sun_dir.c:177-310
 * Tallies are FP64 (sum w, sum w^2) of each realisation's total, exactly the
 * deferred mc_data semantics of src/ssol_estimator_c.h:59-126: a path keeps
 * its per-receiver contributions in registers until it ends, applies the
 * Russian-roulette factor, then commits. Global quantities are reduced per
 * warp with __shfl_xor_sync and committed once per block; receiver-side sums
 * go through shared memory; sparse ones (per sampled instance, per primitive)
 * use FP64 atomics.
 *
 * Geometry, sampling and BSDFs run in the template type R (float for the
 * plain build, double for the all-FP64 build); quadric roots found in FP32 get
 * one FP64 Newton step.
 */
#include "device_scene.h"
#include "kernels.h"
#include "philox.h"

#include <cuda_runtime.h>
#include <float.h>
#include <math.h>

namespace ssolb {

/*******************************************************************************
 * Small vector helpers
 ******************************************************************************/
template<class R> struct V3 { R x, y, z; };

template<class R> __device__ __forceinline__ V3<R> mk(R x, R y, R z)
{ V3<R> v; v.x = x; v.y = y; v.z = z; return v; }
template<class R> __device__ __forceinline__ V3<R> ld3(const R* p)
{ return mk(p[0], p[1], p[2]); }
template<class R> __device__ __forceinline__ V3<R> operator+(V3<R> a, V3<R> b)
{ return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
template<class R> __device__ __forceinline__ V3<R> operator-(V3<R> a, V3<R> b)
{ return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
template<class R> __device__ __forceinline__ V3<R> operator-(V3<R> a)
{ return mk(-a.x, -a.y, -a.z); }
template<class R> __device__ __forceinline__ V3<R> operator*(V3<R> a, R s)
{ return mk(a.x * s, a.y * s, a.z * s); }
template<class R> __device__ __forceinline__ R dot(V3<R> a, V3<R> b)
{ return a.x * b.x + a.y * b.y + a.z * b.z; }
template<class R> __device__ __forceinline__ V3<R> cross(V3<R> a, V3<R> b)
{ return mk(a.y*b.z - a.z*b.y, a.z*b.x - a.x*b.z, a.x*b.y - a.y*b.x); }

__device__ __forceinline__ float rsq(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsq(double x) { return rsqrt(x); }
__device__ __forceinline__ float sq_rt(float x) { return sqrtf(x); }
__device__ __forceinline__ double sq_rt(double x) { return sqrt(x); }
__device__ __forceinline__ float lg(float x) { return logf(x); }
__device__ __forceinline__ double lg(double x) { return log(x); }
__device__ __forceinline__ float ex(float x) { return expf(x); }
__device__ __forceinline__ double ex(double x) { return exp(x); }
__device__ __forceinline__ float cpsgn(float a, float b) { return copysignf(a, b); }
__device__ __forceinline__ double cpsgn(double a, double b) { return copysign(a, b); }
__device__ __forceinline__ float nxt(float a) { return nextafterf(a, FLT_MAX); }
__device__ __forceinline__ double nxt(double a) { return nextafter(a, DBL_MAX); }
__device__ __forceinline__ void sincos2pi(float u, float* s, float* c)
{ sincospif(2.f * u, s, c); }
__device__ __forceinline__ void sincos2pi(double u, double* s, double* c)
{ sincospi(2.0 * u, s, c); }
__device__ __forceinline__ float cs(float x) { return cosf(x); }
__device__ __forceinline__ double cs(double x) { return cos(x); }
__device__ __forceinline__ float sn(float x) { return sinf(x); }
__device__ __forceinline__ double sn(double x) { return sin(x); }

template<class R> __device__ __forceinline__ V3<R> normalize(V3<R> v)
{ const R len = sq_rt(dot(v, v)); return len > R(0) ? v * (R(1) / len) : v; }

template<class R> __device__ __forceinline__ R uni(uint32_t x);
template<> __device__ __forceinline__ float uni<float>(uint32_t x)
{ return u01f(x); }
template<> __device__ __forceinline__ double uni<double>(uint32_t x)
{ return u01d(x); }

template<class R> __device__ __forceinline__ R rmax();
template<> __device__ __forceinline__ float rmax<float>() { return FLT_MAX; }
template<> __device__ __forceinline__ double rmax<double>() { return DBL_MAX; }

/* Orthonormal basis whose third axis is n (Duff et al., "Building an
 * Orthonormal Basis, Revisited", JCGT 2017) */
template<class R>
__device__ __forceinline__ void onb(V3<R> n, V3<R>& b1, V3<R>& b2)
{
  const R sgn = n.z >= R(0) ? R(1) : R(-1);
  const R a = R(-1) / (sgn + n.z);
  const R b = n.x * n.y * a;
  b1 = mk(R(1) + sgn * n.x * n.x * a, sgn * b, -sgn * n.x);
  b2 = mk(b, sgn + n.y * n.y * a, -n.y);
}

/* Per-realisation Philox block */
struct Rng {
  uint32_t i_lo, i_hi, k0, k1;
  __device__ __forceinline__ U32x4 get(uint32_t event, uint32_t domain) const
  { return philox4x32_10(i_lo, i_hi, event, domain, k0, k1); }
};

/*******************************************************************************
 * Scalar data and media
 ******************************************************************************/
/* Clamped linear interpolation (src/ssol_spectrum.c:57-89) */
__device__ __forceinline__ double interp_clamped
  (const double* w, const double* v, int n, double x)
{
  int lo = 0, hi = n; /* first index with w[i] >= x */
  while(lo < hi) {
    const int mid = (lo + hi) >> 1;
    if(w[mid] < x) lo = mid + 1; else hi = mid;
  }
  if(lo == n) return v[n - 1];
  if(lo == 0) return v[0];
  const double slope = (v[lo] - v[lo - 1]) / (w[lo] - w[lo - 1]);
  return v[lo - 1] + (x - w[lo - 1]) * slope;
}

template<class R>
__device__ __forceinline__ double data_value
  (const DScene<R>& S, const DData& d, double wl)
{
  if(d.spectrum < 0) return d.real;
  const DSpectrum sp = S.spectra[d.spectrum];
  return interp_clamped(S.spec_wl + sp.first, S.spec_val + sp.first,
                        sp.count, wl);
}

/* Shader value of a material at wavelength wl: index 0 reflectivity,
 * 1 roughness */
template<class R>
__device__ __forceinline__ R shader_value
  (const DScene<R>& S, const DMaterial& m, int which, double wl)
{
  const R* tab = S.shader_tab + m.table;
  const int n = S.shader_nodes;
  if(n == 1) return tab[which];
  const double* w = S.shader_wl;
  int lo = 0, hi = n;
  while(lo < hi) {
    const int mid = (lo + hi) >> 1;
    if(w[mid] < wl) lo = mid + 1; else hi = mid;
  }
  if(lo == n) return tab[2 * (n - 1) + which];
  if(lo == 0) return tab[which];
  const double a = tab[2 * (lo - 1) + which], b = tab[2 * lo + which];
  return (R)(a + (wl - w[lo - 1]) * (b - a) / (w[lo] - w[lo - 1]));
}

/*******************************************************************************
 * Sun: direction and wavelength (src/ssol_ranst_sun_dir.c:177-310,
 * src/ssol_ranst_sun_wl.c:84-105)
 ******************************************************************************/
template<class R>
__device__ __forceinline__ V3<R> sun_local_to_world(const DScene<R>& S, V3<R> p)
{
  const R* B = S.sun_basis;
  return normalize(mk(B[0] * p.x + B[3] * p.y + B[6] * p.z,
                      B[1] * p.x + B[4] * p.y + B[7] * p.z,
                      B[2] * p.x + B[5] * p.y + B[8] * p.z));
}

/* Buie zenith angle by rejection (src/ssol_ranst_sun_dir.c:177-195); the
 * draws of attempt k come from event 2 + k of the primary domain */
template<class R>
__device__ double buie_theta(const DScene<R>& S, const Rng& rng)
{
  const double thetaSD = S.buie[0], dCSSD = S.buie[1], gamma = S.buie[2];
  const double ek1000g = S.buie[3], alpha = S.buie[4];
  const double h1 = S.buie[5], h2 = S.buie[6], p1 = S.buie[7];
  double theta = 0;
  for(uint32_t k = 0; k < 64; ++k) {
    const U32x4 r = rng.get(2u + k, RNG_PRIMARY);
    double value;
    if(u01d(r.v[0]) < p1) {
      theta = u01d(r.v[1]) * thetaSD;
      value = u01d(r.v[2]) * h1;
    } else {
      theta = thetaSD + u01d(r.v[1]) * dCSSD;
      value = u01d(r.v[2]) * h2;
    }
    const double phi = theta < thetaSD
      ? cos(326 * theta) / cos(308 * theta)
      : ek1000g * pow(theta, gamma);
    if(value <= alpha * phi * sin(theta)) break;
  }
  return theta;
}

template<class R>
__device__ V3<R> sample_sun_dir(const DScene<R>& S, const Rng& rng, U32x4 r)
{
  switch(S.sun_type) {
    case SUN_PILLBOX: {
      const R sin2 = uni<R>(r.v[0]) * S.sun_param;
      const R st = sq_rt(sin2), ct = sq_rt(R(1) - sin2);
      R sp, cp; sincos2pi(uni<R>(r.v[1]), &sp, &cp);
      return sun_local_to_world(S, mk(cp * st, sp * st, ct));
    }
    case SUN_GAUSSIAN: {
      /* 1 - u keeps the log argument in (0, 1] */
      R st = S.sun_param * sq_rt(R(-2) * lg(R(1) - uni<R>(r.v[0])));
      st = st < R(1) ? st : R(1);
      const R ct = sq_rt(R(1) - st * st > R(0) ? R(1) - st * st : R(0));
      R sp, cp; sincos2pi(uni<R>(r.v[1]), &sp, &cp);
      return sun_local_to_world(S, mk(cp * st, sp * st, ct));
    }
    case SUN_BUIE: {
      const R theta = (R)buie_theta(S, rng);
      R sp, cp; sincos2pi(uni<R>(r.v[1]), &sp, &cp);
      const R st = sn(theta), ct = cs(theta);
      return sun_local_to_world(S, mk(st * sp, st * cp, ct));
    }
    default:
      return ld3(S.sun_dir);
  }
}

/* Piecewise linear density over the sun spectrum nodes: pick the interval by
 * its trapezoid mass, then invert the quadratic CDF inside it */
template<class R>
__device__ double sample_wavelength(const DScene<R>& S, double u)
{
  const int n = S.wl_count;
  if(n == 1) return S.wl_nodes[0];
  const double* cdf = S.wl_cdf;
  int lo = 0, hi = n - 1; /* interval j with cdf[j] <= u < cdf[j+1] */
  while(hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if(cdf[mid] <= u) lo = mid; else hi = mid;
  }
  const double mass = cdf[lo + 1] - cdf[lo];
  const double r = mass > 0 ? fmin(fmax((u - cdf[lo]) / mass, 0.0), 1.0) : 0;
  const double a = S.wl_pdf[lo], b = S.wl_pdf[lo + 1];
  double t;
  if(a == b) t = r;
  else {
    const double den = a + sqrt(a * a + r * (b * b - a * a));
    t = den > 0 ? r * (a + b) / den : r;
  }
  return S.wl_nodes[lo] + t * (S.wl_nodes[lo + 1] - S.wl_nodes[lo]);
}

/*******************************************************************************
 * Punched quadrics (src/ssol_shape.c:236-285, 864-1135, 1408-1494)
 ******************************************************************************/
template<class R>
__device__ __forceinline__ V3<R> xform_point(const R* M, V3<R> p)
{
  return mk(M[0] * p.x + M[1] * p.y + M[2] * p.z + M[3],
            M[4] * p.x + M[5] * p.y + M[6] * p.z + M[7],
            M[8] * p.x + M[9] * p.y + M[10] * p.z + M[11]);
}
template<class R>
__device__ __forceinline__ V3<R> xform_vec(const R* M, V3<R> v)
{
  return mk(M[0] * v.x + M[1] * v.y + M[2] * v.z,
            M[4] * v.x + M[5] * v.y + M[6] * v.z,
            M[8] * v.x + M[9] * v.y + M[10] * v.z);
}
/* Normal to world: transpose of the world->local linear part */
template<class R>
__device__ __forceinline__ V3<R> xform_normal(const R* W, V3<R> n)
{
  return mk(W[0] * n.x + W[4] * n.y + W[8] * n.z,
            W[1] * n.x + W[5] * n.y + W[9] * n.z,
            W[2] * n.x + W[6] * n.y + W[10] * n.z);
}

template<class R>
__device__ __forceinline__ R quadric_z(int type, const R* q, R x, R y)
{
  switch(type) {
    case QUAD_PARABOL: return (x * x + y * y) * q[1];
    case QUAD_PARABOL2F: return x * x * q[0] + y * y * q[1];
    case QUAD_HYPERBOL:
      return q[1] * sq_rt(R(1) + (x * x + y * y) * q[3]) - q[1];
    case QUAD_PCYLINDER: return y * y * q[1];
    case QUAD_HEMISPHERE: {
      const R z2 = q[1] - (x * x + y * y);
      return z2 > R(0) ? q[0] - sq_rt(z2) : q[0];
    }
    default: return R(0);
  }
}

template<class R>
__device__ __forceinline__ V3<R> quadric_grad(int type, const R* q, V3<R> p)
{
  switch(type) {
    case QUAD_PARABOL: return mk(-p.x, -p.y, R(2) * q[0]);
    case QUAD_PARABOL2F:
      return mk(-p.x * (R(4) * q[0]), -p.y * (R(4) * q[1]), R(2));
    case QUAD_HYPERBOL: return mk(p.x, p.y, -(p.z + q[1]) * q[2]);
    case QUAD_PCYLINDER: return mk(R(0), -p.y, R(2) * q[0]);
    case QUAD_HEMISPHERE: return mk(-p.x, -p.y, q[0] - p.z);
    default: return mk(R(0), R(0), R(1));
  }
}

/* Coefficients of a t^2 + b t + c = 0 for the local ray o + t d */
template<class T>
__device__ __forceinline__ void quadric_coefs
  (int type, const T* q, T ox, T oy, T oz, T dx, T dy, T dz,
   T& a, T& b, T& c)
{
  switch(type) {
    case QUAD_PLANE: a = T(0); b = dz; c = oz; break;
    case QUAD_PARABOL: {
      const T f4 = T(4) * q[0];
      a = dx * dx + dy * dy;
      b = T(2) * (ox * dx + oy * dy) - f4 * dz;
      c = ox * ox + oy * oy - f4 * oz;
      break;
    }
    case QUAD_PARABOL2F:
      a = dx * dx * q[0] + dy * dy * q[1];
      b = T(2) * (ox * dx * q[0] + oy * dy * q[1]) - dz;
      c = ox * ox * q[0] + oy * oy * q[1] - oz;
      break;
    case QUAD_HYPERBOL: {
      const T b2 = q[1] * q[1];
      const T b2a2 = b2 * q[3];
      const T zz = oz + q[1];
      a = b2a2 * (dx * dx + dy * dy) - dz * dz;
      b = T(2) * (b2a2 * (ox * dx + oy * dy) - zz * dz);
      c = b2a2 * (ox * ox + oy * oy) + b2 - zz * zz;
      break;
    }
    case QUAD_PCYLINDER: {
      const T f4 = T(4) * q[0];
      a = dy * dy;
      b = T(2) * oy * dy - f4 * dz;
      c = oy * oy - f4 * oz;
      break;
    }
    case QUAD_HEMISPHERE: {
      const T z0 = -q[0];
      a = dx * dx + dy * dy + dz * dz;
      b = T(2) * (ox * dx + oy * dy + oz * dz + z0 * dz);
      c = ox * ox + oy * oy + oz * oz - q[1] + T(2) * z0 * oz + z0 * z0;
      break;
    }
    default: a = b = c = T(0); break;
  }
}

/* Roots in ascending order; stable form of src/ssol_shape.c:864-896 */
template<class R>
__device__ __forceinline__ int solve_quadratic(R a, R b, R c, R t[2])
{
  if(a == R(0)) {
    if(b == R(0)) return 0;
    t[0] = -c / b;
    return 1;
  }
  const R delta = b * b - R(4) * a * c;
  if(delta < R(0)) return 0;
  if(delta == R(0)) { t[0] = -b / (R(2) * a); return 1; }
  const R s = sq_rt(delta);
  const R t1 = (-b - cpsgn(s, b)) / (R(2) * a);
  const R t2 = t1 != R(0) ? c / (a * t1) : -b / a;
  t[0] = t1 < t2 ? t1 : t2;
  t[1] = t1 < t2 ? t2 : t1;
  return 2;
}

/* One FP64 Newton step on the root of the FP32 solve */
__device__ __forceinline__ float refine_root
  (int type, const float* q, float ox, float oy, float oz,
   float dx, float dy, float dz, float t)
{
  double qd[4] = {q[0], q[1], q[2], q[3]};
  double a, b, c;
  quadric_coefs<double>(type, qd, ox, oy, oz, dx, dy, dz, a, b, c);
  const double td = t;
  const double f = (a * td + b) * td + c;
  const double df = 2.0 * a * td + b;
  return df != 0.0 ? (float)(td - f / df) : t;
}
__device__ __forceinline__ double refine_root
  (int, const double*, double, double, double, double, double, double,
   double t)
{ return t; }

template<class R>
__device__ bool in_carvings(const DScene<R>& S, const DQuadric<R>& Q, R x, R y)
{
  if(Q.type == QUAD_HEMISPHERE && x * x + y * y > Q.param[2]) return false;
  if(x < Q.carve_lo[0] || x > Q.carve_hi[0]
  || y < Q.carve_lo[1] || y > Q.carve_hi[1]) {
    if(Q.type != QUAD_HEMISPHERE || Q.carve_count) return false;
  }
  for(int k = 0; k < Q.carve_count; ++k) {
    const DCarving C = S.carvings[Q.carve_first + k];
    const R* v = S.carve_verts + 2 * C.first;
    bool in = false;
    for(int i = 0, j = C.count - 1; i < C.count; j = i++) {
      const R xi = v[2 * i], yi = v[2 * i + 1];
      const R xj = v[2 * j], yj = v[2 * j + 1];
      if(((yi > y) != (yj > y)) && (x < (xj - xi) * (y - yi) / (yj - yi) + xi))
        in = !in;
    }
    if(C.op == 0 ? !in : in) return false;
  }
  return true;
}

/*******************************************************************************
 * Ray casting with the reference hit filter (src/ssol_scene.c:439-535)
 ******************************************************************************/
struct SelfInfo {
  int gid; /* triangle the ray leaves, -1 if none */
  int sinst; /* shaded instance the ray leaves */
  int side; /* its side (SSOL_FRONT=1 / SSOL_BACK=2) */
  bool discard_virtual;
  bool reversed;
};

template<class R> struct Hit {
  R t;
  int sinst;
  int prim; /* triangle id in its shape (meshes) */
  int gid; /* global triangle id, -1 for quadrics */
  V3<R> n; /* world normal (unnormalised for triangles) */
};

struct Counters {
  uint32_t rays, nodes, tris, quads;
};

template<class R>
__device__ __forceinline__ bool side_passes
  (const DScene<R>& S, int sinst, int side, const SelfInfo& self)
{
  if(self.reversed) side = side == 1 ? 2 : 1;
  const DShadedInst& si = S.sinsts[sinst];
  if(si.virtual_mask & (side == 1 ? 1 : 2)) {
    if(self.discard_virtual) return false;
    if(!(si.receiver_mask & side)) return false;
  }
  return true;
}

/* Mesh rule: reject t <= eps, t <= tmin and the starting triangle */
template<class R>
__device__ __forceinline__ void test_triangle
  (const DScene<R>& S, int idx, V3<R> o, V3<R> d, R tmin, R eps,
   const SelfInfo& self, Hit<R>& best, bool& found)
{
  const DTri<R> T = S.tris[idx];
  const V3<R> e1 = ld3(T.e1), e2 = ld3(T.e2);
  const V3<R> p = cross(d, e2);
  const R det = dot(e1, p);
  if(det == R(0)) return;
  const R inv = R(1) / det;
  const V3<R> s = o - ld3(T.v0);
  const R u = dot(s, p) * inv;
  if(u < R(0) || u > R(1)) return;
  const V3<R> qv = cross(s, e1);
  const R v = dot(d, qv) * inv;
  if(v < R(0) || u + v > R(1)) return;
  const R t = dot(e2, qv) * inv;
  if(!(t < best.t) || t <= eps || t <= tmin || T.gid == self.gid) return;
  /* Ng = e2 x e1, so dot(Ng, d) = det */
  const int side = det < R(0) ? 1 : 2;
  if(!side_passes(S, T.sinst, side, self)) return;
  best.t = t;
  best.sinst = T.sinst;
  best.prim = T.prim;
  best.gid = T.gid;
  best.n = cross(e2, e1);
  found = true;
}

/* Triangle of the RT tessellation grid that contains local (x, y): cell
 * (ix, iy) holds triangles 2 (ix ny + iy) (below its diagonal) and + 1;
 * only used when no carving cut the grid */
template<class R>
__device__ __forceinline__ int quad_grid_prim(const DQuadric<R>& Q, R x, R y)
{
  if(Q.grid_n[0] <= 0 || Q.grid_n[1] <= 0 || !(Q.grid_delta > R(0))) return 0;
  const R d = Q.grid_delta;
  int ix = (int)floor((x - Q.carve_lo[0]) / d);
  int iy = (int)floor((y - Q.carve_lo[1]) / d);
  ix = min(max(ix, 0), Q.grid_n[0] - 1);
  iy = min(max(iy, 0), Q.grid_n[1] - 1);
  const R x0 = Q.carve_lo[0] + (R)ix * d, y0 = Q.carve_lo[1] + (R)iy * d;
  const R x1 = fmin(x0 + d, Q.carve_hi[0]), y1 = fmin(y0 + d, Q.carve_hi[1]);
  const bool lower = (x - x0) * (y1 - y0) >= (y - y0) * (x1 - x0);
  return (ix * Q.grid_n[1] + iy) * 2 + (lower ? 0 : 1);
}

/* Punched rule: analytic roots inside the carved domain, not below tmin, and
 * not the opposite side of the shape the ray leaves */
template<class R>
__device__ __forceinline__ void test_quadric
  (const DScene<R>& S, int idx, V3<R> o, V3<R> d, R tmin,
   const SelfInfo& self, Hit<R>& best, bool& found)
{
  const DQuadric<R>& Q = S.quads[idx];
  const V3<R> ol = xform_point(Q.w2l, o);
  const V3<R> dl = xform_vec(Q.w2l, d);
  R a, b, c;
  quadric_coefs<R>(Q.type, Q.param, ol.x, ol.y, ol.z, dl.x, dl.y, dl.z,
                   a, b, c);
  R roots[2];
  const int n = solve_quadratic(a, b, c, roots);
  for(int k = 0; k < n; ++k) {
    const R t = refine_root(Q.type, Q.param, ol.x, ol.y, ol.z,
                            dl.x, dl.y, dl.z, roots[k]);
    if(t <= tmin) continue;
    if(!(t < best.t)) break;
    const V3<R> pl = ol + dl * t;
    if(Q.type == QUAD_HYPERBOL && !(pl.z + Q.param[1] > R(0))) continue;
    if(Q.type == QUAD_HEMISPHERE && pl.z > Q.param[0]) continue;
    if(!in_carvings(S, Q, pl.x, pl.y)) continue;
    const V3<R> nw = normalize(xform_normal(Q.w2l, quadric_grad(Q.type,
                                                                 Q.param, pl)));
    const int side = dot(d, nw) < R(0) ? 1 : 2;
    if(Q.sinst == self.sinst && side != self.side) continue;
    if(!side_passes(S, Q.sinst, side, self)) continue;
    best.t = t;
    best.sinst = Q.sinst;
    best.prim = quad_grid_prim(Q, pl.x, pl.y);
    best.gid = -1;
    best.n = nw;
    found = true;
    break;
  }
}

template<class R>
__device__ __forceinline__ bool slab
  (const R* lo, const R* hi, V3<R> inv, V3<R> oinv, R tmin, R tmax, R& tent)
{
  const R tx0 = lo[0] * inv.x - oinv.x, tx1 = hi[0] * inv.x - oinv.x;
  const R ty0 = lo[1] * inv.y - oinv.y, ty1 = hi[1] * inv.y - oinv.y;
  const R tz0 = lo[2] * inv.z - oinv.z, tz1 = hi[2] * inv.z - oinv.z;
  const R t0 = fmax(fmax(fmin(tx0, tx1), fmin(ty0, ty1)),
                    fmax(fmin(tz0, tz1), tmin));
  const R t1 = fmin(fmin(fmax(tx0, tx1), fmax(ty0, ty1)),
                    fmin(fmax(tz0, tz1), tmax));
  tent = t0;
  return t0 <= t1;
}

constexpr int STACK_SIZE = 64;

/* Closest accepted hit (ANY == false) or any accepted hit (ANY == true) */
template<class R, bool ANY>
__device__ bool trace_ray
  (const DScene<R>& S, V3<R> o, V3<R> d, R tmin, const SelfInfo& self,
   Hit<R>& best, Counters& cnt)
{
  ++cnt.rays;
  /* A zero direction component would make lo * inv - o * inv an inf - inf
   * NaN for boxes the ray runs parallel to; clamp it to +-2^-64 so that the
   * FMA form of the slab test stays finite (Aila and Laine, HPG 2009) */
  const R tiny = R(5.42101086242752217e-20);
  const V3<R> inv = mk(R(1) / (fabs(d.x) > tiny ? d.x : cpsgn(tiny, d.x)),
                       R(1) / (fabs(d.y) > tiny ? d.y : cpsgn(tiny, d.y)),
                       R(1) / (fabs(d.z) > tiny ? d.z : cpsgn(tiny, d.z)));
  const V3<R> oinv = mk(o.x * inv.x, o.y * inv.y, o.z * inv.z);
  /* Self-hit epsilon of the mesh rule: the reference's 1e-6, scaled by the
   * magnitude of the origin so that it stays above the FP32 resolution */
  const R amax = fmax(fmax(fabs(o.x), fabs(o.y)), fabs(o.z));
  const R eps = R(1e-6) * (R(1) + amax);
  best.t = rmax<R>();
  bool found = false;
  int stack[STACK_SIZE];
  int sp = 0;
  int node = 0;
  for(;;) {
    const DNode<R> N = S.nodes[node];
    ++cnt.nodes;
    R te[2];
    bool h[2];
    h[0] = slab(N.lo[0], N.hi[0], inv, oinv, tmin, best.t, te[0])
        && N.count[0] >= 0;
    h[1] = slab(N.lo[1], N.hi[1], inv, oinv, tmin, best.t, te[1])
        && N.count[1] >= 0;
    int next[2];
    int nnext = 0;
    for(int k = 0; k < 2; ++k) {
      if(!h[k]) continue;
      if(N.count[k] > 0) {
        for(int p = 0; p < N.count[k]; ++p) {
          const uint32_t ref = S.primrefs[N.child[k] + p];
          if(primref_kind(ref) == PRIM_TRIANGLE) {
            ++cnt.tris;
            test_triangle(S, (int)primref_index(ref), o, d, tmin, eps, self,
                          best, found);
          } else {
            ++cnt.quads;
            test_quadric(S, (int)primref_index(ref), o, d, tmin, self,
                         best, found);
          }
          if(ANY && found) return true;
        }
      } else {
        next[nnext++] = k;
      }
    }
    if(nnext == 2) {
      const int nearer = te[0] <= te[1] ? 0 : 1;
      if(sp < STACK_SIZE) stack[sp++] = N.child[1 - nearer];
      node = N.child[nearer];
    } else if(nnext == 1) {
      node = N.child[next[0]];
    } else {
      if(sp == 0) break;
      node = stack[--sp];
    }
  }
  return found;
}

/*******************************************************************************
 * BSDF sampling (Star-SF restated from published optics)
 ******************************************************************************/
enum { BXDF_REFLECTION = 1, BXDF_TRANSMISSION = 2 };

/* Unpolarised Fresnel reflectance at a dielectric interface */
template<class R>
__device__ __forceinline__ R fresnel(R cos_i, R cos_t, R eta_i, R eta_t)
{
  const R rs = (eta_i * cos_i - eta_t * cos_t) / (eta_i * cos_i + eta_t * cos_t);
  const R rp = (eta_t * cos_i - eta_i * cos_t) / (eta_t * cos_i + eta_i * cos_t);
  return R(0.5) * (rs * rs + rp * rp);
}

template<class R>
__device__ __forceinline__ V3<R> local_to(V3<R> n, R x, R y, R z)
{
  V3<R> b1, b2;
  onb(n, b1, b2);
  return b1 * x + b2 * y + n * z;
}

/* Returns false on an inconsistent medium (RES_BAD_OP) */
template<class R>
__device__ bool shade
  (const DScene<R>& S, const Rng& rng, uint32_t scatter, int mtl_idx,
   int medium, double wl, V3<R> wo, V3<R> N, R& prop, V3<R>& out,
   int& type, int& next_medium)
{
  const DMaterial m = S.mtls[mtl_idx];
  prop = R(0);
  type = 0;
  next_medium = medium;
  /* src/ssol_material.c:97-101 */
  if(m.type == MTL_DIELECTRIC && medium != m.out_medium) return false;
  const R cos_i = dot(wo, N);
  if(!(cos_i > R(0))) return true;
  const U32x4 r = rng.get(scatter, RNG_SCATTER);
  switch(m.type) {
    case MTL_MIRROR: {
      const R refl = shader_value(S, m, 0, wl);
      const R rough = shader_value(S, m, 1, wl);
      type = BXDF_REFLECTION;
      if(rough == R(0)) {
        out = N * (R(2) * cos_i) - wo;
        prop = refl;
      } else {
        /* Microfacet normal drawn around N (Beckmann: tan^2 = -a^2 ln(1-u);
         * pillbox: tan^2 = a^2 u), mirrored about; re-drawn while the
         * reflection falls below the surface */
        U32x4 rr = r;
        bool ok = false;
        for(uint32_t k = 0; k < 16 && !ok; ++k) {
          if(k) rr = rng.get((scatter << 6) | k, RNG_RETRY);
          const R u0 = uni<R>(rr.v[0]);
          const R tan2 = m.distrib == DISTRIB_BECKMANN
            ? -rough * rough * lg(R(1) - u0)
            : rough * rough * u0;
          const R ct = rsq(R(1) + tan2);
          const R st = sq_rt(tan2) * ct;
          R sp, cp; sincos2pi(uni<R>(rr.v[1]), &sp, &cp);
          const V3<R> h = local_to(N, cp * st, sp * st, ct);
          const R wh = dot(wo, h);
          if(!(wh > R(0))) continue;
          out = h * (R(2) * wh) - wo;
          ok = dot(out, N) > R(0);
        }
        prop = ok ? refl : R(0);
      }
      break;
    }
    case MTL_MATTE: {
      /* Cosine weighted hemisphere */
      const R u0 = uni<R>(r.v[0]);
      const R rad = sq_rt(u0);
      R sp, cp; sincos2pi(uni<R>(r.v[1]), &sp, &cp);
      out = local_to(N, rad * cp, rad * sp, sq_rt(R(1) - u0));
      prop = shader_value(S, m, 0, wl);
      type = BXDF_REFLECTION;
      break;
    }
    case MTL_DIELECTRIC: {
      const R eta_i = (R)data_value(S, S.media[m.out_medium].refractive_index, wl);
      const R eta_t = (R)data_value(S, S.media[m.in_medium].refractive_index, wl);
      const R eta = eta_i / eta_t;
      const R sin2_t = eta * eta * (R(1) - cos_i * cos_i);
      R F = R(1), cos_t = R(0);
      if(sin2_t < R(1)) {
        cos_t = sq_rt(R(1) - sin2_t);
        F = fresnel(cos_i, cos_t, eta_i, eta_t);
      }
      prop = R(1);
      if(uni<R>(r.v[0]) < F) {
        out = N * (R(2) * cos_i) - wo;
        type = BXDF_REFLECTION;
      } else {
        out = normalize(N * (eta * cos_i - cos_t) - wo * eta);
        type = BXDF_TRANSMISSION;
        next_medium = m.in_medium;
      }
      break;
    }
    case MTL_THIN_DIELECTRIC: {
      const R eta_i = (R)data_value(S, S.media[m.out_medium].refractive_index, wl);
      const R eta_t = (R)data_value(S, S.media[m.slab_medium].refractive_index, wl);
      const R alpha = (R)data_value(S, S.media[m.slab_medium].extinction, wl);
      const R eta = eta_i / eta_t;
      const R sin2_t = eta * eta * (R(1) - cos_i * cos_i);
      R Rt = R(1), Tt = R(0);
      if(sin2_t < R(1)) {
        const R cos_t = sq_rt(R(1) - sin2_t);
        const R F = fresnel(cos_i, cos_t, eta_i, eta_t);
        const R tau = ex(-alpha * (R)m.thickness / cos_t);
        const R den = R(1) - F * F * tau * tau;
        Rt = F + (R(1) - F) * (R(1) - F) * F * tau * tau / den;
        Tt = (R(1) - F) * (R(1) - F) * tau / den;
      }
      prop = Rt + Tt;
      if(prop > R(0) && uni<R>(r.v[0]) * prop < Rt) {
        out = N * (R(2) * cos_i) - wo;
        type = BXDF_REFLECTION;
      } else {
        out = -wo;
        type = BXDF_TRANSMISSION;
      }
      break;
    }
    default: break;
  }
  /* Wrong hemisphere for the sampled component (src/ssol_solver.c:468-475) */
  const R cos_out = dot(N, out);
  if((cos_out > R(0) && (type & BXDF_TRANSMISSION))
  || (cos_out < R(0) && (type & BXDF_REFLECTION)))
    prop = R(0);
  return true;
}

/*******************************************************************************
 * Per path tallies
 ******************************************************************************/
constexpr int MAX_RCV_ENTRIES = 4;
constexpr int MAX_PRIM_ENTRIES = 4;

struct PathTally {
  int nrcv, nprim;
  int rcv_slot[MAX_RCV_ENTRIES];
  double rcv[MAX_RCV_ENTRIES][6];
  int prim_slot[MAX_PRIM_ENTRIES];
  double prim[MAX_PRIM_ENTRIES][6];
  bool overflow;

  __device__ void add(int rslot, int pslot, const double v[6])
  {
    int k = 0;
    while(k < nrcv && rcv_slot[k] != rslot) ++k;
    if(k == nrcv) {
      if(nrcv == MAX_RCV_ENTRIES) { overflow = true; return; }
      rcv_slot[nrcv] = rslot;
      for(int q = 0; q < 6; ++q) rcv[nrcv][q] = 0;
      ++nrcv;
    }
    for(int q = 0; q < 6; ++q) rcv[k][q] += v[q];
    if(pslot < 0) return;
    k = 0;
    while(k < nprim && prim_slot[k] != pslot) ++k;
    if(k == nprim) {
      if(nprim == MAX_PRIM_ENTRIES) { overflow = true; return; }
      prim_slot[nprim] = pslot;
      for(int q = 0; q < 6; ++q) prim[nprim][q] = 0;
      ++nprim;
    }
    for(int q = 0; q < 6; ++q) prim[k][q] += v[q];
  }
};

/* 10 receiver quantities from the 6 accumulated ones, in MC_RECEIVER_DATA
 * order (src/ssol_solver.c:735-755) */
__device__ __forceinline__ void expand10(const double v[6], double f,
                                         double out[NRCV_Q])
{
  out[0] = f * v[0];
  out[1] = f * v[1];
  out[2] = f * v[2];
  out[3] = f * (v[2] - v[0]);
  out[4] = f * (v[1] - v[0]);
  out[5] = f * v[3];
  out[6] = f * v[4];
  out[7] = f * v[5];
  out[8] = f * (v[5] - v[3]);
  out[9] = f * (v[4] - v[3]);
}

__device__ __forceinline__ void red_add(double* p, double v)
{
  if(v != 0.0) atomicAdd(p, v);
}

/*******************************************************************************
 * The realisation (src/ssol_solver.c:873-1127)
 ******************************************************************************/
enum PathStatus { PATH_OK = 0, PATH_KILLED = 1, PATH_FAILED = 2 };

template<class R> struct ThreadAcc {
  double sum[NGLOBAL];
  double sq[NGLOBAL];
};

template<class R>
__device__ void trace_realisation
  (const DScene<R>& S, const DTallies& T, const Rng& rng,
   ThreadAcc<R>& acc, double* smem_rcv, Counters& cnt, uint32_t& bounces,
   unsigned long long max_segments)
{
  /* ---- point_init (src/ssol_solver.c:207-358) ---- */
  const U32x4 r0 = rng.get(0u, RNG_PRIMARY);
  /* bucket = floor(u * n) computed exactly on the 24-bit integer draw */
  int k = (int)(((unsigned long long)(r0.v[0] >> 8)
                 * (unsigned long long)S.nsamp) >> 24);
  if(!(uni<float>(r0.v[1]) < S.alias_prob[k])) k = S.alias_idx[k];
  const DSampTri<R> st = S.samp[k];
  const R sa = sq_rt(uni<R>(r0.v[2]));
  const R b2 = sa * uni<R>(r0.v[3]);
  const R b1 = sa - b2;
  V3<R> pos = ld3(st.v0) + ld3(st.e1) * b1 + ld3(st.e2) * b2;
  const V3<R> nproxy = ld3(st.n);

  const U32x4 r1 = rng.get(1u, RNG_PRIMARY);
  V3<R> dir = sample_sun_dir(S, rng, r1);
  const double wl = sample_wavelength(S, u01d(r1.v[2]));

  int sinst = st.sinst;
  DShadedInst si = S.sinsts[sinst];
  int prim = st.prim;
  int gid = st.gid;
  V3<R> N = nproxy;
  if(si.is_punched) {
    /* punched_shape_project_point (src/ssol_shape.c:1408-1447) */
    const DQuadric<R>& Q = S.quads[si.quadric];
    V3<R> pl = xform_point(Q.w2l, pos);
    pl.z = quadric_z(Q.type, Q.param, pl.x, pl.y);
    N = normalize(xform_normal(Q.w2l, quadric_grad(Q.type, Q.param, pl)));
    pos = xform_point(Q.l2w, pl);
  }
  int side = 1;
  if(dot(N, dir) >= R(0)) { side = 2; N = -N; }

  const V3<R> sun0 = ld3(S.sun_dir);
  const R surface_sun_cos = dot(N, dir);
  const R surface_sun0_cos = fabs(dot(sun0, N));
  const R sun0_sun_cos = dot(sun0, dir);
  const R surface_proxy_cos = si.is_punched ? fabs(dot(nproxy, N)) : R(1);
  const R cos_ratio = fabs(surface_sun_cos / (surface_proxy_cos * sun0_sun_cos));
  const double w0 = S.dni * S.area_proxy * (double)cos_ratio;
  const double cos_factor = S.area_proxy / S.area_rt
    * (double)surface_sun0_cos / (double)surface_proxy_cos;
  const int samp_idx = si.sampled;

  int mtl = si.mtl[side - 1];
  const int mtype0 = S.mtls[mtl].type;
  int medium = S.air_medium;
  if(mtype0 == MTL_DIELECTRIC || mtype0 == MTL_THIN_DIELECTRIC) {
    medium = side == 1 ? S.mtls[mtl].in_medium : S.mtls[mtl].out_medium;
  }

  double g[NGLOBAL] = {0, 0, 0, 0, 0, 0};
  double samp_shadow = 0;
  PathTally pt;
  pt.nrcv = pt.nprim = 0;
  pt.overflow = false;
  int status = PATH_OK;
  int score = 0;

  /* Shadow ray toward the sun (src/ssol_solver.c:320-352) */
  SelfInfo self;
  self.gid = gid;
  self.sinst = sinst;
  self.side = side;
  self.discard_virtual = true;
  self.reversed = true;
  Hit<R> h;
  const bool occluded = trace_ray<R, true>(S, pos, -dir, R(0), self, h, cnt);

  if(occluded) {
    g[G_SHADOW] = w0;
    samp_shadow = w0;
  } else {
    double prev[3] = {w0, w0, w0};
    double inc[3], out[3];
    R hit_t = R(0);
    R tmin = R(0);
    V3<R> org = pos, rd = dir;
    uint32_t depth = 0, roulette_interval = 64;
    uint32_t scatter = 0, nroulette = 0;
    unsigned long long segments = 0;
    for(;;) {
      const bool in_atm = medium == S.air_medium;
      const bool hit_receiver = (si.receiver_mask & side) != 0;
      const bool hit_virtual = (si.virtual_mask & side) != 0;
      double trans = 1;
      if(hit_t > R(0)) {
        const double kext = data_value(S, S.media[medium].extinction, wl);
        if(kext > 0) trans = (double)ex((R)(-kext * (double)hit_t));
      }
      inc[0] = prev[0] * trans;
      inc[1] = in_atm ? prev[1] : prev[1] * trans;
      inc[2] = !in_atm ? prev[2] : prev[2] * trans;

      double kabs;
      int out_medium = medium;
      if(hit_virtual) {
        kabs = 0;
        out[0] = inc[0]; out[1] = inc[1]; out[2] = inc[2];
      } else {
        R prop;
        V3<R> ndir;
        int type;
        ++bounces;
        if(!shade(S, rng, scatter++, mtl, medium, wl, -dir, N, prop, ndir,
                  type, out_medium)) {
          status = PATH_FAILED;
          break;
        }
        const double p = (double)prop;
        kabs = 1.0 - p;
        out[0] = inc[0] * p;
        out[1] = inc[1] * p;
        out[2] = hit_receiver ? inc[2] * p : inc[2];
        if(type) dir = ndir;
      }

      if(hit_receiver) {
        const int si_side = side - 1;
        const double v[6] = {inc[0], inc[1], inc[2],
                             inc[0] * kabs, inc[1] * kabs, inc[2] * kabs};
        const int pslot = si.prim_base[si_side] >= 0
          ? si.prim_base[si_side] + prim : -1;
        pt.add(si.rcv_slot[si_side], pslot, v);
        g[G_ABS_RCV] += inc[0] - out[0];
      } else {
        g[G_OTHER] += inc[0] * kabs;
      }

      const bool weight_zero = out[0] == 0.0;
      bool last = false;
      if(!weight_zero) {
        if(hit_virtual) {
          tmin = nxt(hit_t);
        } else {
          tmin = R(0);
          org = pos;
          rd = dir;
        }
        self.gid = gid;
        self.sinst = sinst;
        self.side = side;
        self.discard_virtual = false;
        self.reversed = false;
        if(!trace_ray<R, false>(S, org, rd, tmin, self, h, cnt)) {
          last = true;
          if(out_medium != S.air_medium) { status = PATH_FAILED; break; }
        }
      }
      if(weight_zero || last || !hit_virtual) {
        const double absorbed = prev[0] - inc[0];
        if(in_atm) g[G_ATM] += absorbed; else g[G_OTHER] += absorbed;
        if(weight_zero || last) break;
        prev[0] = out[0]; prev[1] = out[1]; prev[2] = out[2];
      }
      depth += hit_virtual ? 0u : 1u;
      if(depth > roulette_interval && depth % roulette_interval == 1) {
        const double p = u01d(rng.get(nroulette++, RNG_ROULETTE).v[0]);
        if(p > 0.5) {
          ++score;
          roulette_interval = 16;
        } else {
          status = PATH_KILLED;
          break;
        }
      }
      if(++segments >= max_segments) { status = PATH_FAILED; break; }

      /* point_update_from_hit (src/ssol_solver.c:360-411) */
      sinst = h.sinst;
      si = S.sinsts[sinst];
      prim = h.prim;
      gid = h.gid;
      N = normalize(h.n);
      pos = org + rd * h.t;
      side = dot(rd, N) < R(0) ? 1 : 2;
      if(side == 2) N = -N;
      mtl = si.mtl[side - 1];
      hit_t = h.t;
      medium = out_medium;
    }
    if(status == PATH_OK) g[G_MISSING] += out[0];
  }
  if(status == PATH_OK) g[G_COS] += cos_factor;
  if(pt.overflow) status = PATH_FAILED;

  /* ---- commit ---- */
  atomicAdd(&T.nb_samples[samp_idx], 1ull);
  if(status == PATH_FAILED) {
    atomicAdd(&T.counters[0], 1ull);
    if(pt.overflow) atomicAdd(&T.counters[2], 1ull);
    return;
  }
  if(status == PATH_KILLED) {
    atomicAdd(&T.counters[1], 1ull);
    return;
  }
  const double f = (double)(1ull << score);
  for(int q = 0; q < NGLOBAL; ++q) {
    const double w = f * g[q];
    acc.sum[q] += w;
    acc.sq[q] += w * w;
  }
  {
    const double wc = f * cos_factor, ws = f * samp_shadow;
    double* sp = T.samp + (size_t)samp_idx * 4;
    red_add(sp + 0, wc);
    red_add(sp + 1, wc * wc);
    red_add(sp + 2, ws);
    red_add(sp + 3, ws * ws);
  }
  for(int e = 0; e < pt.nrcv; ++e) {
    double v10[NRCV_Q];
    expand10(pt.rcv[e], f, v10);
    const int r = pt.rcv_slot[e];
    double* dst = smem_rcv ? smem_rcv + (size_t)r * NRCV_Q * 2
                           : T.rcv + (size_t)r * NRCV_Q * 2;
    double* dsr = T.samp_rcv + ((size_t)samp_idx * S.nrcv + r) * NRCV_Q * 2;
    for(int q = 0; q < NRCV_Q; ++q) {
      red_add(dst + 2 * q, v10[q]);
      red_add(dst + 2 * q + 1, v10[q] * v10[q]);
      red_add(dsr + 2 * q, v10[q]);
      red_add(dsr + 2 * q + 1, v10[q] * v10[q]);
    }
  }
  for(int e = 0; e < pt.nprim; ++e) {
    double v10[NRCV_Q];
    expand10(pt.prim[e], f, v10);
    double* dst = T.prim + (size_t)pt.prim_slot[e] * NRCV_Q * 2;
    for(int q = 0; q < NRCV_Q; ++q) {
      red_add(dst + 2 * q, v10[q]);
      red_add(dst + 2 * q + 1, v10[q] * v10[q]);
    }
  }
}

/*******************************************************************************
 * Kernel
 ******************************************************************************/
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
  for(int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v)
{
#pragma unroll
  for(int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

constexpr int SMEM_RCV_MAX = 16;

template<class R>
__global__ void __launch_bounds__(256)
realisation_kernel
  (const DScene<R> S, const DTallies T, uint64_t seed, uint64_t first,
   uint64_t count, unsigned long long max_segments)
{
  extern __shared__ double smem[];
  __shared__ double red[32][2 * NGLOBAL];
  const bool use_smem = S.nrcv <= SMEM_RCV_MAX;
  double* smem_rcv = use_smem ? smem : nullptr;
  if(use_smem) {
    for(int i = threadIdx.x; i < S.nrcv * NRCV_Q * 2; i += blockDim.x)
      smem_rcv[i] = 0;
  }
  __syncthreads();

  ThreadAcc<R> acc;
  for(int q = 0; q < NGLOBAL; ++q) acc.sum[q] = acc.sq[q] = 0;
  Counters cnt = {0, 0, 0, 0};
  uint32_t bounces = 0, paths = 0;

  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  Rng rng;
  rng.k0 = (uint32_t)seed;
  rng.k1 = (uint32_t)(seed >> 32);
  for(uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
      i += stride) {
    const uint64_t id = first + i;
    rng.i_lo = (uint32_t)id;
    rng.i_hi = (uint32_t)(id >> 32);
    trace_realisation(S, T, rng, acc, smem_rcv, cnt, bounces, max_segments);
    ++paths;
  }

  /* Warp then block reduction of the global sums, one commit per block */
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for(int q = 0; q < NGLOBAL; ++q) {
    const double s = warp_sum(acc.sum[q]);
    const double s2 = warp_sum(acc.sq[q]);
    if(lane == 0) { red[warp][2 * q] = s; red[warp][2 * q + 1] = s2; }
  }
  unsigned long long c[6] = {cnt.rays, cnt.nodes, cnt.tris, cnt.quads,
                             bounces, paths};
  for(int q = 0; q < 6; ++q) c[q] = warp_sum_u64(c[q]);
  if(lane == 0) {
    unsigned long long* st = &T.stats->rays;
    for(int q = 0; q < 6; ++q) if(c[q]) atomicAdd(st + q, c[q]);
  }
  __syncthreads();
  if(threadIdx.x < 2 * NGLOBAL) {
    double v = 0;
    for(int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[w][threadIdx.x];
    red_add(T.global + threadIdx.x, v);
  }
  if(use_smem) {
    for(int i = threadIdx.x; i < S.nrcv * NRCV_Q * 2; i += blockDim.x)
      red_add(T.rcv + i, smem_rcv[i]);
  }
}

/*******************************************************************************
 * Host launchers
 ******************************************************************************/
template<class R>
static int launch_impl
  (const DScene<R>& S, const DTallies& T, uint64_t seed, uint64_t first,
   uint64_t count, const LaunchConfig& cfg, void* stream)
{
  int dev = 0;
  cudaGetDevice(&dev);
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int block = cfg.block_size > 0 ? cfg.block_size : 256;
  const size_t smem = S.nrcv <= SMEM_RCV_MAX
    ? (size_t)S.nrcv * NRCV_Q * 2 * sizeof(double) : 0;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor
    (&per_sm, realisation_kernel<R>, block, smem);
  if(per_sm < 1) per_sm = 1;
  uint64_t blocks = cfg.grid_blocks > 0
    ? (uint64_t)cfg.grid_blocks
    : (uint64_t)nsm * (uint64_t)per_sm * (uint64_t)(cfg.waves > 0 ? cfg.waves : 1);
  const uint64_t needed = (count + block - 1) / block;
  if(blocks > needed) blocks = needed;
  if(blocks < 1) blocks = 1;
  realisation_kernel<R><<<(unsigned)blocks, block, smem,
                          (cudaStream_t)stream>>>
    (S, T, seed, first, count, cfg.max_segments);
  return (int)cudaGetLastError();
}

int launch_realisations_f32
  (const DScene<float>& S, const DTallies& T, uint64_t seed, uint64_t first,
   uint64_t count, const LaunchConfig& cfg, void* stream)
{ return launch_impl<float>(S, T, seed, first, count, cfg, stream); }

int launch_realisations_f64
  (const DScene<double>& S, const DTallies& T, uint64_t seed, uint64_t first,
   uint64_t count, const LaunchConfig& cfg, void* stream)
{ return launch_impl<double>(S, T, seed, first, count, cfg, stream); }

} /* namespace ssolb */
