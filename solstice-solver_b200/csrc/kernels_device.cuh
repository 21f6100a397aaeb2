/*
 * kernels_device.cuh - device code of the sm_100a realisation loop of
 * `ssol_solve`, and the templates of its host launchers. Included by the
 * kernels_*.cu translation units, each of which instantiates some of the
 * launchers, so that they compile in parallel.
 *
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
#ifndef SSOL_B200_KERNELS_DEVICE_CUH
#define SSOL_B200_KERNELS_DEVICE_CUH

#include "device_scene.h"
#include "kernels.h"
#include "philox.h"

#include <cuda_runtime.h>
#include <float.h>
#include <math.h>

#include <atomic>
#include <mutex>
#include <numeric>

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
__device__ __forceinline__ R shader_lerp
  (const DScene<R>& S, const R* tab, int which, double wl)
{
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

template<class R>
__device__ __forceinline__ R shader_value
  (const DScene<R>& S, const DMaterial& m, int which, double wl)
{ return shader_lerp(S, S.shader_tab + m.table, which, wl); }

/* Shader value baked at the vertices of a triangle side (offset `bake` in
 * bake_tab), interpolated in wavelength then with the barycentric weights
 * (1 - b1 - b2, b1, b2) of the point */
template<class R>
__device__ __forceinline__ R baked_value
  (const DScene<R>& S, int bake, int which, double wl, R b1, R b2)
{
  const R* tab = S.bake_tab + bake;
  const int stride = 2 * S.shader_nodes;
  const R v0 = shader_lerp(S, tab, which, wl);
  const R v1 = shader_lerp(S, tab + stride, which, wl);
  const R v2 = shader_lerp(S, tab + 2 * stride, which, wl);
  return v0 * (R(1) - b1 - b2) + v1 * b1 + v2 * b2;
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
__device__ __noinline__ double buie_theta(const DScene<R>& S, const Rng rng)
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

/* Front normal (local frame, unnormalised) at pl of the general form in
 * DQuadric::gen */
template<class R>
__device__ __forceinline__ V3<R> quadric_general_normal(const DQuadric<R>& Q, V3<R> pl)
{
  const R sg = (R)Q.gen[6];
  return mk(sg * R(2) * (R)Q.gen[0] * pl.x, sg * R(2) * (R)Q.gen[1] * pl.y,
            sg * (R(2) * (R)Q.gen[2] * (pl.z - (R)Q.gen[3]) + (R)Q.gen[4]));
}

/* Height of the surface above local (x, y): the linear case, or the
 * root on the side gen[7] of z0 (upper sheet of the hyperboloid, lower
 * hemisphere); src/ssol_shape.c:236-285 */
template<class R>
__device__ __forceinline__ R quadric_general_z(const DQuadric<R>& Q, R x, R y)
{
  const R kz = (R)Q.gen[2];
  const R rest = (R)Q.gen[0] * x * x + (R)Q.gen[1] * y * y + (R)Q.gen[5];
  if(kz == R(0)) return -rest / (R)Q.gen[4];
  const R w = -rest / kz;
  return (R)Q.gen[3] + (R)Q.gen[7] * sq_rt(w > R(0) ? w : R(0));
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

/* One FP64 Newton step of F(o + t d) on the FP32 root, general form */
__device__ __forceinline__ float refine_root_general
  (const double* g, V3<float> o, V3<float> d, float t)
{
  const double ox = o.x, oy = o.y, dx = d.x, dy = d.y, dz = d.z;
  const double zz = (double)o.z - g[3];
  const double a = g[0] * dx * dx + g[1] * dy * dy + g[2] * dz * dz;
  const double b = 2.0 * (g[0] * ox * dx + g[1] * oy * dy + g[2] * zz * dz) + g[4] * dz;
  const double c = g[0] * ox * ox + g[1] * oy * oy + g[2] * zz * zz + g[4] * (double)o.z
                 + g[5];
  const double td = t;
  const double f = (a * td + b) * td + c;
  const double df = 2.0 * a * td + b;
  return df != 0.0 ? (float)(td - f / df) : t;
}
__device__ __forceinline__ double refine_root_general
  (const double*, V3<double>, V3<double>, double t)
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
  const DShadedInst si = ldg_record(S.sinsts + sinst);
  if(si.virtual_mask & (side == 1 ? 1 : 2)) {
    if(self.discard_virtual) return false;
    if(!(si.receiver_mask & side)) return false;
  }
  return true;
}

/* Products and differences rounded on their own (no FMA contraction): the
 * edge functions of the watertight test must be exact negations on an edge
 * shared by two triangles */
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

/* Per-ray shear of the watertight ray/triangle test (Woop, Benthin and Wald,
 * "Watertight Ray/Triangle Intersection", JCGT 2(1), 2013): rows that map a
 * vertex relative to the origin into a frame where the ray runs along +z,
 * x' = v[kx] - Sx v[kz], y' = v[ky] - Sy v[kz], z' = Sz v[kz], with kz the
 * dominant axis of the direction and kx, ky swapped when d[kz] < 0 so that
 * the winding is kept. Applying the rows is deterministic per vertex, which
 * is all watertightness needs. */
template<class R> struct Shear { V3<R> rx, ry, rz; };

template<class R>
__device__ __forceinline__ Shear<R> make_shear(V3<R> d)
{
  const R ax = fabs(d.x), ay = fabs(d.y), az = fabs(d.z);
  const int kz = ax > ay ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
  int kx = kz == 2 ? 0 : kz + 1;
  int ky = kx == 2 ? 0 : kx + 1;
  const R dz = kz == 0 ? d.x : kz == 1 ? d.y : d.z;
  if(dz < R(0)) { const int t = kx; kx = ky; ky = t; }
  const R dx = kx == 0 ? d.x : kx == 1 ? d.y : d.z;
  const R dy = ky == 0 ? d.x : ky == 1 ? d.y : d.z;
  const R sx = dx / dz, sy = dy / dz, sz = R(1) / dz;
  Shear<R> s;
  s.rx = mk(kx == 0 ? R(1) : kz == 0 ? -sx : R(0),
            kx == 1 ? R(1) : kz == 1 ? -sx : R(0),
            kx == 2 ? R(1) : kz == 2 ? -sx : R(0));
  s.ry = mk(ky == 0 ? R(1) : kz == 0 ? -sy : R(0),
            ky == 1 ? R(1) : kz == 1 ? -sy : R(0),
            ky == 2 ? R(1) : kz == 2 ? -sy : R(0));
  s.rz = mk(kz == 0 ? sz : R(0), kz == 1 ? sz : R(0), kz == 2 ? sz : R(0));
  return s;
}

template<class R>
__device__ __forceinline__ R shear_row(V3<R> r, V3<R> a)
{
  return fma(r.z, a.z, fma(r.y, a.y, mul_rn(r.x, a.x)));
}

/* A 16-byte aligned record through the read-only data path, 16 bytes at a
 * time */
template<class T>
__device__ __forceinline__ T ldg_record(const T* p)
{
  static_assert(sizeof(T) % 16 == 0 && alignof(T) >= 16, "16-byte records only");
  union { T t; int4 w[sizeof(T) / 16]; } u;
#pragma unroll
  for(int i = 0; i < (int)(sizeof(T) / 16); ++i)
    u.w[i] = __ldg(reinterpret_cast<const int4*>(p) + i);
  return u.t;
}

/* A triangle through the read-only data path: three 16-byte loads in FP32 */
__device__ __forceinline__ DTri<float> load_tri(const DTri<float>* p)
{
  const float4* q = reinterpret_cast<const float4*>(p);
  const float4 a = __ldg(q), b = __ldg(q + 1);
  const int4 c = __ldg(reinterpret_cast<const int4*>(q + 2));
  DTri<float> t;
  t.v0[0] = a.x; t.v0[1] = a.y; t.v0[2] = a.z;
  t.v1[0] = a.w; t.v1[1] = b.x; t.v1[2] = b.y;
  t.v2[0] = b.z; t.v2[1] = b.w; t.v2[2] = __int_as_float(c.x);
  t.sinst = c.y; t.prim = c.z; t.gid = c.w;
  return t;
}
__device__ __forceinline__ DTri<double> load_tri(const DTri<double>* p) { return *p; }

/* A BVH node through the read-only data path: four 16-byte loads in FP32 */
__device__ __forceinline__ DNode<float> load_node(const DNode<float>* p)
{
  const float4* q = reinterpret_cast<const float4*>(p);
  const float4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
  const int4 d = __ldg(reinterpret_cast<const int4*>(q + 3));
  DNode<float> n;
  n.lo[0][0] = a.x; n.lo[0][1] = a.y; n.lo[0][2] = a.z;
  n.lo[1][0] = a.w; n.lo[1][1] = b.x; n.lo[1][2] = b.y;
  n.hi[0][0] = b.z; n.hi[0][1] = b.w; n.hi[0][2] = c.x;
  n.hi[1][0] = c.y; n.hi[1][1] = c.z; n.hi[1][2] = c.w;
  n.child[0] = d.x; n.child[1] = d.y; n.count[0] = d.z; n.count[1] = d.w;
  return n;
}
__device__ __forceinline__ DNode<double> load_node(const DNode<double>* p) { return *p; }

/* Mesh rule: reject t <= eps, t <= tmin and the starting triangle.
 * Inclusion by the watertight edge functions, so that no ray is lost between
 * two triangles; distance from the triangle's plane, dot(Ng, v0 - o) /
 * dot(Ng, d), so that the two triangles of a planar quad give the same t and
 * a ray crossing a virtual quad on its diagonal is not counted twice.
 * Ng = e2 x e1 is Star-3D's front face. */
template<class R>
__device__ __forceinline__ void test_triangle
  (const DScene<R>& S, int idx, V3<R> o, V3<R> d, const Shear<R>& sh, R tmin,
   R eps, const SelfInfo& self, Hit<R>& best, bool& found)
{
  const DTri<R> T = load_tri(S.tris + idx);
  const V3<R> p0 = ld3(T.v0), p1 = ld3(T.v1), p2 = ld3(T.v2);
  const V3<R> a = p0 - o, b = p1 - o, c = p2 - o;
  const R ax = shear_row(sh.rx, a), ay = shear_row(sh.ry, a);
  const R bx = shear_row(sh.rx, b), by = shear_row(sh.ry, b);
  const R cx = shear_row(sh.rx, c), cy = shear_row(sh.ry, c);
  const R u = sub_rn(mul_rn(cx, by), mul_rn(cy, bx));
  const R v = sub_rn(mul_rn(ax, cy), mul_rn(ay, cx));
  const R w = sub_rn(mul_rn(bx, ay), mul_rn(by, ax));
  if((u < R(0) || v < R(0) || w < R(0)) && (u > R(0) || v > R(0) || w > R(0)))
    return;
  if(u + v + w == R(0)) return;
  const V3<R> ng = cross(p2 - p0, p1 - p0);
  const R den = dot(ng, d);
  const R t = dot(ng, a) / den;
  if(!(t < best.t) || t <= eps || t <= tmin || T.gid == self.gid) return;
  const int side = den < R(0) ? 1 : 2;
  if(!side_passes(S, T.sinst, side, self)) return;
  best.t = t;
  best.sinst = T.sinst;
  best.prim = T.prim;
  best.gid = T.gid;
  best.n = ng;
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
  /* One code path for every kind: the general form of DQuadric::gen */
  const R kx = (R)Q.gen[0], ky = (R)Q.gen[1], kz = (R)Q.gen[2], z0 = (R)Q.gen[3];
  const R lz = (R)Q.gen[4], m = (R)Q.gen[5];
  const R zz = ol.z - z0;
  const R a = kx * dl.x * dl.x + ky * dl.y * dl.y + kz * dl.z * dl.z;
  const R b = R(2) * (kx * ol.x * dl.x + ky * ol.y * dl.y + kz * zz * dl.z) + lz * dl.z;
  const R c = kx * ol.x * ol.x + ky * ol.y * ol.y + kz * zz * zz + lz * ol.z + m;
  R roots[2];
  const int n = solve_quadratic(a, b, c, roots);
  /* Not unrolled: one inlined copy of the refinement, carving and normal
   * code for both roots */
#pragma unroll 1
  for(int k = 0; k < n; ++k) {
    const R t = refine_root_general(Q.gen, ol, dl, k == 0 ? roots[0] : roots[1]);
    if(t <= tmin) continue;
    if(!(t < best.t)) break;
    const V3<R> pl = ol + dl * t;
    if(Q.type == QUAD_HYPERBOL && !(pl.z + Q.param[1] > R(0))) continue;
    if(Q.type == QUAD_HEMISPHERE && pl.z > Q.param[0]) continue;
    if(!in_carvings(S, Q, pl.x, pl.y)) continue;
    const V3<R> nw = normalize(xform_normal(Q.w2l, quadric_general_normal(Q, pl)));
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

/* The builder bounds the BVH depth to 30, so a traversal never holds more
 * than 30 deferred nodes. The first SMEM_STACK entries live in shared
 * memory; the rare deeper ones in a per-thread array (local memory), which
 * leaves shared memory to the L1 cache that holds the BVH. With 5 entries
 * three blocks of 256 threads of the realisation kernel (53.4 KB each, plus
 * the 1 KB the SM reserves per block) fit the 164 KB shared-memory
 * configuration of the SM, which leaves 92 KB of L1 instead of 60: field
 * 535 -> 550 Mpaths/s (8 entries needed the 196 KB configuration). */
constexpr int STACK_SIZE = 32;
constexpr int SMEM_STACK = 5;

/* Closest accepted hit, or the first accepted hit when `any` (shadow rays).
 * Deferred node i < SMEM_STACK of this thread is stack[i * stride] in shared
 * memory, deeper ones go to `spill`. */
template<class R, int FEAT = FEAT_ALL>
__device__ bool trace_ray
  (const DScene<R>& S, V3<R> o, V3<R> d, R tmin, const SelfInfo& self,
   bool any, Hit<R>& best, Counters& cnt, int* stack, int stride)
{
  if(!(FEAT & FEAT_NOCOUNT)) ++cnt.rays;
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
  const Shear<R> sh = make_shear(d);
  best.t = rmax<R>();
  bool found = false;
  int spill[STACK_SIZE - SMEM_STACK];
  int sp = 0;
  int node = 0;
  for(;;) {
    const DNode<R> N = load_node(S.nodes + node);
    if(!(FEAT & FEAT_NOCOUNT)) ++cnt.nodes;
    R te[2];
    bool h[2];
    h[0] = slab(N.lo[0], N.hi[0], inv, oinv, tmin, best.t, te[0])
        && N.count[0] >= 0;
    h[1] = slab(N.lo[1], N.hi[1], inv, oinv, tmin, best.t, te[1])
        && N.count[1] >= 0;
    /* The hit leaves, slot 0 then slot 1, through one loop so that the
     * primitive tests are inlined once (a loop over k would be unrolled
     * and hold two copies of each) */
    unsigned leaves = (h[0] && N.count[0] > 0 ? 1u : 0u) | (h[1] && N.count[1] > 0 ? 2u : 0u);
    while(leaves) {
      const bool k1 = (leaves & 1u) == 0u;
      leaves &= leaves - 1u;
      const int lc = k1 ? N.count[1] : N.count[0];
      const int first = k1 ? N.child[1] : N.child[0];
      for(int p = 0; p < lc; ++p) {
        const uint32_t ref = lc == 1 ? (uint32_t)first : S.primrefs[first + p];
        if(!(FEAT & FEAT_QUADRIC) || primref_kind(ref) == PRIM_TRIANGLE) {
          if(!(FEAT & FEAT_NOCOUNT)) ++cnt.tris;
          test_triangle(S, (int)primref_index(ref), o, d, sh, tmin, eps,
                        self, best, found);
        } else {
          if(!(FEAT & FEAT_NOCOUNT)) ++cnt.quads;
          test_quadric(S, (int)primref_index(ref), o, d, tmin, self,
                       best, found);
        }
        if(any && found) return true;
      }
    }
    const bool in0 = h[0] && N.count[0] == 0, in1 = h[1] && N.count[1] == 0;
    if(in0 && in1) {
      const bool first0 = te[0] <= te[1];
      const int far = first0 ? N.child[1] : N.child[0];
      if(sp < SMEM_STACK) stack[(sp++) * stride] = far;
      else if(sp < STACK_SIZE) spill[(sp++) - SMEM_STACK] = far;
      node = first0 ? N.child[0] : N.child[1];
    } else if(in0 || in1) {
      node = in0 ? N.child[0] : N.child[1];
    } else {
      if(sp == 0) break;
      --sp;
      node = sp < SMEM_STACK ? stack[sp * stride] : spill[sp - SMEM_STACK];
    }
  }
  return found;
}

/* Per-thread FP64 path sums kept in shared memory (column `tid`, stride
 * blockDim): the first receiver entry's 6 values, the 3 global quantities
 * accumulated along the path and the cosine factor */
enum : int { PS_V0 = 0, PS_ABS = 6, PS_ATM = 7, PS_OTHER = 8, PS_COS = 9,
             PS_UV = 10, PS_COUNT = 11 };

/* Barycentric weights (b1, b2) of vertices 1 and 2 of triangle gid at the
 * point x of its plane */
template<class R>
__device__ __forceinline__ float2 tri_uv(const DScene<R>& S, int gid, V3<R> x)
{
  const DTri<R>& T = S.tris[gid];
  const V3<R> a = ld3(T.v0);
  const V3<R> e1 = ld3(T.v1) - a, e2 = ld3(T.v2) - a, q = x - a;
  const R d11 = dot(e1, e1), d12 = dot(e1, e2), d22 = dot(e2, e2);
  const R q1 = dot(q, e1), q2 = dot(q, e2);
  const R den = d11 * d22 - d12 * d12;
  if(!(den != R(0))) return make_float2(0.f, 0.f);
  return make_float2((float)((d22 * q1 - d12 * q2) / den),
                     (float)((d11 * q2 - d12 * q1) / den));
}

/* Barycentric weights (b1, b2) of the current point, kept as two floats in
 * the PS_UV slot when the scene has shading attributes */
__device__ __forceinline__ void put_uv(double* ps, int stride, float b1, float b2)
{
  float2* q = reinterpret_cast<float2*>(ps + PS_UV * stride);
  *q = make_float2(b1, b2);
}
__device__ __forceinline__ float2 get_uv(const double* ps, int stride)
{
  return *reinterpret_cast<const float2*>(ps + PS_UV * stride);
}

/*******************************************************************************
 * BSDF sampling (Star-SF's BSDFs restated from published optics: Fresnel
 * equations, Walter et al. 2007 microfacet sampling, thin-slab series)
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

/* One BSDF sample: the propagated fraction, the outgoing direction, the
 * sampled component (BXDF_*, 0 if none) and the medium beyond, through
 * references; false on an inconsistent medium (RES_BAD_OP). Out of line, to
 * keep the hot loop short. (Returning these as a struct by value measured
 * slower: 354 against 486 Mpaths/s on the field.) */
template<class R, int FEAT = FEAT_ALL>
__device__ __noinline__ bool shade
  (const DScene<R>& S, const Rng& rng, uint32_t scatter, int mtl_idx,
   int medium, double wl, V3<R> wo, V3<R> Ng, R& prop, V3<R>& out,
   int& type, int& next_medium, int gid, int side, const double* ps, int stride)
{
  const DMaterial m = S.mtls[mtl_idx];
  prop = R(0);
  type = 0;
  next_medium = medium;
  /* src/ssol_material.c:97-101 */
  if((FEAT & FEAT_DIELECTRIC) && m.type == MTL_DIELECTRIC && medium != m.out_medium)
    return false;
  /* Shading normal: the interpolated vertex normal turned toward the
   * incoming side, else Ng (src/ssol_material.c:630-654); shader values
   * baked per vertex where the material varies over the mesh */
  V3<R> N = Ng;
  int bake = -1;
  R b1 = R(0), b2 = R(0);
  if((FEAT & FEAT_ATTRIBUTES) && S.tshade && gid >= 0) {
    const float2 uv = get_uv(ps, stride);
    b1 = (R)uv.x;
    b2 = (R)uv.y;
    const DTriShade<R>& ts = S.tshade[gid];
    bake = ts.bake[side - 1];
    if(!isnan(ts.n[0])) {
      const V3<R> ns = ld3(ts.n) * (R(1) - b1 - b2) + ld3(ts.n + 3) * b1
                     + ld3(ts.n + 6) * b2;
      const R l2 = dot(ns, ns);
      if(l2 > R(0)) {
        N = ns * rsq(l2);
        if(dot(N, wo) < R(0)) N = -N;
      }
    }
  }
  const R cos_i = dot(wo, N);
  if(!(cos_i > R(0))) return true;
  const U32x4 r = rng.get(scatter, RNG_SCATTER);
  switch(m.type) {
    case MTL_MIRROR: {
      const R refl = bake >= 0 ? baked_value(S, bake, 0, wl, b1, b2)
                               : shader_value(S, m, 0, wl);
      const R rough = bake >= 0 ? baked_value(S, bake, 1, wl, b1, b2)
                                : shader_value(S, m, 1, wl);
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
#pragma unroll 1
        for(uint32_t k = 0; k < 16; ++k) {
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
          if(ok) break;
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
      prop = bake >= 0 ? baked_value(S, bake, 0, wl, b1, b2) : shader_value(S, m, 0, wl);
      type = BXDF_REFLECTION;
      break;
    }
    case MTL_DIELECTRIC: {
      if(!(FEAT & FEAT_DIELECTRIC)) break;
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
      if(!(FEAT & FEAT_DIELECTRIC)) break;
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
  /* Wrong hemisphere for the sampled component, against the geometric
   * normal (src/ssol_solver.c:468-475) */
  const R cos_out = dot(Ng, out);
  if((cos_out > R(0) && (type & BXDF_TRANSMISSION))
  || (cos_out < R(0) && (type & BXDF_REFLECTION)))
    prop = R(0);
  return true;
}

/*******************************************************************************
 * Realisation state machine
 *
 * Each warp iteration casts exactly one ray per active lane, from a single
 * call site: the shadow ray of a new path (any hit) or the next segment of a
 * path (closest hit). Around it, lanes regenerate (fetch a new realisation
 * through a warp-aggregated atomic counter), interact with the surface they
 * reached, or commit a finished path. Lanes never wait for the longest path
 * of their warp, and lanes in different phases still trace together.
 ******************************************************************************/
enum : int { PH_NONE = 0, PH_SHADOW = 1, PH_BOUNCE = 2 };
enum : int {
  END_NONE = 0, END_SHADOW, END_MISS, END_ZERO, END_KILL, END_FAIL
};

/* Extra (receiver side, primitive) entries of one path beyond the first,
 * kept in local memory: only paths reaching several receivers touch them */
constexpr int MAX_EXTRA = 7;

__device__ __forceinline__ void red_add(double* p, double v)
{
  if(v != 0.0) atomicAdd(p, v);
}
/* The same into device memory, as a reduction (no value comes back): an
 * atomicAdd through a pointer that may address shared memory is a generic
 * atomic whose sector returns to L1 */
__device__ __forceinline__ void red_add_global(double* p, double v)
{
  if(v != 0.0)
    asm volatile("red.global.add.f64 [%0], %1;"
                 :: "l"(__cvta_generic_to_global(p)), "d"(v) : "memory");
}
__device__ __forceinline__ void red_add_shared(double* p, double v)
{
  if(v != 0.0)
    asm volatile("red.shared.add.f64 [%0], %1;"
                 :: "r"((unsigned)__cvta_generic_to_shared(p)), "d"(v) : "memory");
}
__device__ __forceinline__ void red_inc_global(unsigned long long* p)
{
  asm volatile("red.global.add.u64 [%0], 1;"
               :: "l"(__cvta_generic_to_global(p)) : "memory");
}

/* (w, w^2) of the 10 receiver quantities of one path, from its 6
 * accumulated values (MC_RECEIVER_DATA order, src/ssol_solver.c:735-755:
 * incoming, incoming if no atmosphere loss, if no field loss, lost in the
 * field, lost in the atmosphere, then the same 5 absorbed), added to dst. The values travel as scalars, so that
 * none of them goes through local memory. */
template<bool GLOBAL>
static __device__ __noinline__ void commit10
  (double* dst, double v0, double v1, double v2, double v3, double v4, double v5,
   double f)
{
  const double q[NRCV_Q] = {f * v0, f * v1, f * v2, f * (v2 - v0), f * (v1 - v0),
                            f * v3, f * v4, f * v5, f * (v5 - v3), f * (v4 - v3)};
#pragma unroll
  for(int k = 0; k < NRCV_Q; ++k) {
    if(GLOBAL) {
      red_add_global(dst + 2 * k, q[k]);
      red_add_global(dst + 2 * k + 1, q[k] * q[k]);
    } else {
      red_add(dst + 2 * k, q[k]);
      red_add(dst + 2 * k + 1, q[k] * q[k]);
    }
  }
}
/* GLOBAL: dst is device memory (else shared or device memory) */
template<bool GLOBAL>
__device__ __forceinline__ void commit10(double* dst, const double v[6], double f)
{
  commit10<GLOBAL>(dst, v[0], v[1], v[2], v[3], v[4], v[5], f);
}

/* dst: shared memory when `shared`, else device memory */
static __device__ __noinline__ void flush_racc(double* dst, const double* racc, bool shared)
{
  if(shared) {
#pragma unroll 1
    for(int k = 0; k < 2 * NRCV_Q; ++k) red_add_shared(dst + k, racc[k]);
  } else {
#pragma unroll 1
    for(int k = 0; k < 2 * NRCV_Q; ++k) red_add_global(dst + k, racc[k]);
  }
}

template<class R> struct PathState {
  int phase;
  int samp;
  int tslot; /* tracked path slot, -1 if not tracked */
  uint32_t tseq; /* vertices recorded so far */
  /* current point / ray: the point is org (+ rd t after a hit) */
  int sinst, side, prim, gid, medium, out_medium;
  V3<R> N, org, rd;
  R tmin, hit_t;
  double wl;
  /* weights (FP64) */
  double prev[3];
  double inc0;
  bool virt;
  /* counters */
  uint32_t depth, interval, scatter, nroul, segments;
  int score;
  /* receiver entries: the first one's values live in shared memory */
  int nent;
  int r0, p0;
  bool overflow;
};

/* Sampled proxy primitive of a primary draw: Vose alias table, bucket =
 * floor(u * n) computed exactly on the 24-bit integer draw */
template<class R>
__device__ __forceinline__ int sample_prim(const DScene<R>& S, const U32x4& r0)
{
  int k = (int)(((unsigned long long)(r0.v[0] >> 8)
                 * (unsigned long long)S.nsamp) >> 24);
  if(!(uni<float>(r0.v[1]) < S.alias_prob[k])) k = S.alias_idx[k];
  return k;
}

/* point_init (src/ssol_solver.c:207-352) up to the shadow ray; `draw` is the
 * realisation's primary draw when the caller already has it */
template<class R, int FEAT = FEAT_ALL>
__device__ __forceinline__ void init_path
  (const DScene<R>& S, const Rng& rng, PathState<R>& p, double* ps, int stride,
   const U32x4* draw = nullptr)
{
  const U32x4 r0 = draw ? *draw : rng.get(0u, RNG_PRIMARY);
  const int k = sample_prim(S, r0);
  const DSampTri<R> st = S.samp[k];
  const R sa = sq_rt(uni<R>(r0.v[2]));
  const R b2 = sa * uni<R>(r0.v[3]);
  const R b1 = sa - b2;
  V3<R> pos = ld3(st.v0) + ld3(st.e1) * b1 + ld3(st.e2) * b2;
  const V3<R> nproxy = ld3(st.n);
  if((FEAT & FEAT_ATTRIBUTES) && S.tshade) put_uv(ps, stride, (float)b1, (float)b2);

  const U32x4 r1 = rng.get(1u, RNG_PRIMARY);
  const V3<R> dir = sample_sun_dir(S, rng, r1);
  p.wl = sample_wavelength(S, u01d(r1.v[2]));

  const DShadedInst si = S.sinsts[st.sinst];
  V3<R> N = nproxy;
  if((FEAT & FEAT_QUADRIC) && si.is_punched) {
    /* punched_shape_project_point (src/ssol_shape.c:1408-1447) */
    const DQuadric<R>& Q = S.quads[si.quadric];
    V3<R> pl = xform_point(Q.w2l, pos);
    pl.z = quadric_general_z(Q, pl.x, pl.y);
    N = normalize(xform_normal(Q.w2l, quadric_general_normal(Q, pl)));
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
  ps[PS_COS * stride] = S.area_proxy / S.area_rt
    * (double)surface_sun0_cos / (double)surface_proxy_cos;
  ps[PS_ABS * stride] = ps[PS_ATM * stride] = ps[PS_OTHER * stride] = 0;
  p.samp = si.sampled;

  const DMaterial m = S.mtls[si.mtl[side - 1]];
  p.medium = S.air_medium;
  if((FEAT & FEAT_DIELECTRIC)
  && (m.type == MTL_DIELECTRIC || m.type == MTL_THIN_DIELECTRIC))
    p.medium = side == 1 ? m.in_medium : m.out_medium;

  p.sinst = st.sinst;
  p.side = side;
  p.prim = st.prim;
  p.gid = st.gid;
  p.N = N;
  p.hit_t = R(0);
  p.prev[0] = p.prev[1] = p.prev[2] = w0;
  p.inc0 = 0;
  p.virt = false;
  p.depth = p.scatter = p.nroul = p.segments = 0;
  p.interval = 64;
  p.score = 0;
  p.nent = 0;
  p.overflow = false;
  /* Shadow ray toward the sun (src/ssol_solver.c:320-352) */
  p.org = pos;
  p.rd = -dir;
  p.tmin = R(0);
  p.phase = PH_SHADOW;
}

template<class R>
__device__ __forceinline__ void add_entry
  (PathState<R>& p, int rslot, int pslot, const double v[6], double* ps,
   int stride, int* xr, int* xp, double (*xv)[6])
{
  if(p.nent == 0) {
    p.nent = 1;
    p.r0 = rslot;
    p.p0 = pslot;
    for(int q = 0; q < 6; ++q) ps[(PS_V0 + q) * stride] = v[q];
    return;
  }
  if(p.r0 == rslot && p.p0 == pslot) {
    for(int q = 0; q < 6; ++q) ps[(PS_V0 + q) * stride] += v[q];
    return;
  }
  for(int e = 0; e < p.nent - 1; ++e) {
    if(xr[e] == rslot && xp[e] == pslot) {
      for(int q = 0; q < 6; ++q) xv[e][q] += v[q];
      return;
    }
  }
  if(p.nent - 1 >= MAX_EXTRA) { p.overflow = true; return; }
  const int e = p.nent - 1;
  xr[e] = rslot;
  xp[e] = pslot;
  for(int q = 0; q < 6; ++q) xv[e][q] = v[q];
  ++p.nent;
}

/* One surface interaction (src/ssol_solver.c:939-1011): extinction of the
 * incoming segment, virtual pass-through or BSDF sample, receiver tallies,
 * then either the next ray or the end of the path */
template<class R, int FEAT = FEAT_ALL>
__device__ int interact
  (const DScene<R>& S, const Rng& rng, PathState<R>& p, V3<R> pos, V3<R> dir,
   uint32_t& bounces, unsigned long long max_segments, double* ps, int stride,
   int* xr, int* xp, double (*xv)[6])
{
  const DShadedInst si = S.sinsts[p.sinst];
  const bool in_atm = p.medium == S.air_medium;
  const bool hit_receiver = (si.receiver_mask & p.side) != 0;
  const bool hit_virtual = (si.virtual_mask & p.side) != 0;
  double trans = 1;
  if(p.hit_t > R(0)) {
    const double kext = data_value(S, S.media[p.medium].extinction, p.wl);
    if(kext > 0) trans = (double)ex((R)(-kext * (double)p.hit_t));
  }
  const double inc0 = p.prev[0] * trans;
  const double inc1 = in_atm ? p.prev[1] : p.prev[1] * trans;
  const double inc2 = !in_atm ? p.prev[2] : p.prev[2] * trans;
  double out0, out1, out2, kabs;
  int out_medium = p.medium;
  if(hit_virtual) {
    kabs = 0;
    out0 = inc0; out1 = inc1; out2 = inc2;
  } else {
    ++bounces;
    R prop;
    V3<R> ndir;
    int type;
    if(!shade<R, FEAT>(S, rng, p.scatter++, si.mtl[p.side - 1], p.medium, p.wl, -dir,
              p.N, prop, ndir, type, out_medium, p.gid, p.side, ps, stride))
      return END_FAIL;
    const double pr = (double)prop;
    kabs = 1.0 - pr;
    out0 = inc0 * pr;
    out1 = inc1 * pr;
    out2 = hit_receiver ? inc2 * pr : inc2;
    if(type) dir = ndir;
  }
  if(hit_receiver) {
    const int s = p.side - 1;
    const double v[6] = {inc0, inc1, inc2, inc0 * kabs, inc1 * kabs, inc2 * kabs};
    const int pslot = si.prim_base[s] >= 0 ? si.prim_base[s] + p.prim : -1;
    add_entry(p, si.rcv_slot[s], pslot, v, ps, stride, xr, xp, xv);
    ps[PS_ABS * stride] += inc0 - out0;
  } else {
    ps[PS_OTHER * stride] += inc0 * kabs;
  }
  /* Loss along the incoming segment, accounted at non-virtual points or at
   * the end of the path (src/ssol_solver.c:1036-1054) */
  const double seg_loss = p.prev[0] - inc0;
  if(out0 == 0.0 || !hit_virtual)
    ps[(in_atm ? PS_ATM : PS_OTHER) * stride] += seg_loss;
  if(out0 == 0.0) return END_ZERO;
  if(!hit_virtual) {
    p.prev[0] = out0; p.prev[1] = out1; p.prev[2] = out2;
    p.org = pos;
    p.rd = dir;
    p.tmin = R(0);
  } else {
    /* Virtual: pursue the same ray beyond the hit (src/ssol_solver.c:988-995) */
    p.inc0 = inc0;
    p.tmin = nxt(p.hit_t);
  }
  p.virt = hit_virtual;
  p.out_medium = out_medium;
  if(++p.segments >= max_segments) return END_FAIL;
  p.phase = PH_BOUNCE;
  return END_NONE;
}

/* What commit_path_pe reads of a finished path */
struct PathEnd {
  int end; /* END_* */
  int samp, score, nent, r0, p0;
  bool overflow;
  double w_end; /* weight shadowed (END_SHADOW) or missing (END_MISS) */
};

template<class R>
__device__ __forceinline__ PathEnd path_end(const PathState<R>& p, int end)
{
  PathEnd e;
  e.end = p.overflow ? END_FAIL : end;
  e.samp = p.samp;
  e.score = p.score;
  e.nent = p.nent;
  e.r0 = p.r0;
  e.p0 = p.p0;
  e.overflow = p.overflow;
  e.w_end = end == END_MISS && p.virt ? p.inc0 : p.prev[0];
  return e;
}

/* Commit a finished path: FP64 (w, w^2) of its totals, x 2^score for
 * roulette survivors (src/ssol_solver.c:1087-1108). Returns the receiver
 * side of the thread's running sums `racc` after the commit. */
template<class R>
__device__ __noinline__ int commit_path_pe
  (const DScene<R>& S, const DTallies& T, const PathEnd& pe, double* acc,
   double* ps, int stride, double* smem_rcv, const int* xr, const int* xp,
   const double (*xv)[6], double* racc, int racc_slot, const DControl* ctl)
{
  const int end = pe.end;
  red_inc_global(&T.nb_samples[pe.samp]);
  if(end == END_FAIL) {
    /* The failure that reaches the limit stops the launch's work fetch
     * (src/ssol_solver.c:1240-1245) */
    const unsigned long long nf = atomicAdd(&T.counters[0], 1ull) + 1ull;
    if(ctl && ctl->stop && nf >= ctl->max_failed) atomicExch(ctl->stop, 1ull);
    if(pe.overflow) atomicAdd(&T.counters[2], 1ull);
    return racc_slot;
  }
  if(end == END_KILL) {
    atomicAdd(&T.counters[1], 1ull);
    return racc_slot;
  }
  const double f = (double)(1ull << pe.score);
  const double g[NGLOBAL] = {
    ps[PS_COS * stride], ps[PS_ABS * stride],
    end == END_SHADOW ? pe.w_end : 0.0,
    end == END_MISS ? pe.w_end : 0.0,
    ps[PS_ATM * stride], ps[PS_OTHER * stride]};
  if(acc) {
#pragma unroll
    for(int q = 0; q < NGLOBAL; ++q) {
      const double w = f * g[q];
      acc[(2 * q) * stride] += w;
      acc[(2 * q + 1) * stride] += w * w;
    }
  }
  {
    const double wc = f * g[G_COS], ws = f * g[G_SHADOW];
    double* sp = T.samp + (size_t)pe.samp * 4;
    red_add_global(sp + 0, wc);
    red_add_global(sp + 1, wc * wc);
    red_add_global(sp + 2, ws);
    red_add_global(sp + 3, ws * ws);
  }
  if(pe.nent == 0) return racc_slot;
  double* rbase = smem_rcv ? smem_rcv : T.rcv;
  if(pe.nent == 1) {
    const double a0 = ps[(PS_V0 + 0) * stride], a1 = ps[(PS_V0 + 1) * stride];
    const double a2 = ps[(PS_V0 + 2) * stride], a3 = ps[(PS_V0 + 3) * stride];
    const double a4 = ps[(PS_V0 + 4) * stride], a5 = ps[(PS_V0 + 5) * stride];
    if(racc) {
      /* The thread's running sums of one receiver side, flushed when the
       * side changes: no atomics while its paths keep reaching it */
      if(racc_slot != pe.r0) {
        if(racc_slot >= 0)
          flush_racc(rbase + (size_t)racc_slot * NRCV_Q * 2, racc, smem_rcv != nullptr);
        racc_slot = pe.r0;
#pragma unroll
        for(int k = 0; k < 2 * NRCV_Q; ++k) racc[k] = 0.0;
      }
      const double q[NRCV_Q] = {f * a0, f * a1, f * a2, f * (a2 - a0), f * (a1 - a0),
                                f * a3, f * a4, f * a5, f * (a5 - a3), f * (a4 - a3)};
#pragma unroll
      for(int k = 0; k < NRCV_Q; ++k) {
        racc[2 * k] += q[k];
        racc[2 * k + 1] += q[k] * q[k];
      }
    } else {
      commit10<false>(rbase + (size_t)pe.r0 * NRCV_Q * 2, a0, a1, a2, a3, a4, a5, f);
    }
    commit10<true>(T.samp_rcv + ((size_t)pe.samp * S.nrcv + pe.r0) * NRCV_Q * 2,
                   a0, a1, a2, a3, a4, a5, f);
    if(pe.p0 >= 0)
      commit10<true>(T.prim + (size_t)pe.p0 * NRCV_Q * 2, a0, a1, a2, a3, a4, a5, f);
    return racc_slot;
  }
  double v0[6];
  for(int q = 0; q < 6; ++q) v0[q] = ps[(PS_V0 + q) * stride];
  /* Several entries: sum per receiver side and per primitive before
   * squaring (deferred mc_data semantics) */
  const int n = pe.nent;
  for(int e = 0; e < n; ++e) {
    const int re = e == 0 ? pe.r0 : xr[e - 1];
    bool seen = false;
    for(int k = 0; k < e && !seen; ++k) seen = (k == 0 ? pe.r0 : xr[k - 1]) == re;
    if(!seen) {
      double v[6] = {0, 0, 0, 0, 0, 0};
      for(int k = e; k < n; ++k) {
        if((k == 0 ? pe.r0 : xr[k - 1]) != re) continue;
        for(int q = 0; q < 6; ++q) v[q] += k == 0 ? v0[q] : xv[k - 1][q];
      }
      commit10<false>(rbase + (size_t)re * NRCV_Q * 2, v, f);
      commit10<true>(T.samp_rcv + ((size_t)pe.samp * S.nrcv + re) * NRCV_Q * 2, v, f);
    }
    const int prim = e == 0 ? pe.p0 : xp[e - 1];
    if(prim >= 0) {
      /* (receiver side, primitive) keys are unique among the entries */
      commit10<true>(T.prim + (size_t)prim * NRCV_Q * 2, e == 0 ? v0 : xv[e - 1], f);
    }
  }
  return racc_slot;
}

/* commit_path_pe on a path state; two out-of-line levels, as measured
 * fastest (with the path end passed by value, 354 against 486 Mpaths/s) */
template<class R>
__device__ __noinline__ int commit_path
  (const DScene<R>& S, const DTallies& T, const PathState<R>& p, int end, double* acc,
   double* ps, int stride, double* smem_rcv, const int* xr, const int* xp,
   const double (*xv)[6], double* racc, int racc_slot, const DControl* ctl)
{
  const PathEnd pe = path_end(p, end);
  return commit_path_pe(S, T, pe, acc, ps, stride, smem_rcv, xr, xp, xv, racc, racc_slot, ctl);
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
constexpr int MAX_BLOCK = 256;
/* SMs per item group of the batched kernel's work order: small items
 * (fewer than BATCH_LARGE_ITEM realisations on average) by groups of 8 SMs,
 * larger ones by 16. Measured on 256 field items (Mpaths/s, groups of 8 /
 * 16 / 37 SMs): 1e5 each 437 / 420 / 345, 1e6 each 482 / 489 / 485. */
constexpr int BATCH_GROUP_SMALL = 8, BATCH_GROUP_LARGE = 16;
constexpr unsigned long long BATCH_LARGE_ITEM = 400000;
/* Coherent order (see presort_count) */
constexpr int SORT_MAX_BINS = 12288; /* shared-memory histogram of primitives */
constexpr uint64_t SORT_CHUNK = 1ull << 24; /* realisations per sorted chunk */
/* Smaller launches keep the id order: there the warps get few segments each
 * (the last ones leave lanes idle) and the presort does not pay. On the field
 * (Mpaths/s, sorted against id order): 1e6 paths 596 / 597, 4e6 615 / 632,
 * 8e6 652 / 637, 1.6e7 675 / 640 */
constexpr uint64_t SORT_MIN = 6000000;
constexpr uint32_t SORT_SEG = SORT_SEGMENT; /* sorted realisations per warp segment */

/* Append one vertex of a tracked path (src/ssol_solver.c:909-922, 1014-1019,
 * 1080-1083: the sun end, the sampled point, every hit and the end at
 * infinity, each with the flux carried to it) */
template<class R>
__device__ __forceinline__ void track_vertex
  (const DTrack& tr, PathState<R>& p, V3<R> x, double w)
{
  const unsigned long long k = atomicAdd(tr.nverts, 1ull);
  if(k < tr.cap) {
    TrackVertex& v = tr.verts[k];
    v.slot = (uint32_t)p.tslot;
    v.seq = p.tseq;
    v.pos[0] = (double)x.x;
    v.pos[1] = (double)x.y;
    v.pos[2] = (double)x.z;
    v.weight = w;
  }
  ++p.tseq;
}

template<class R, int MINB, bool TRACK, int FEAT>
__global__ void __launch_bounds__(MAX_BLOCK, MINB)
realisation_kernel
  (const DScene<R> S, const DTallies T,
   uint64_t seed, uint64_t first, uint64_t count, unsigned long long max_segments,
   unsigned long long* next_path, const DTrack tr,
   const uint4* sorted_draw, const uint32_t* sorted_off, uint32_t seg_mul,
   const DControl ctl)
{
  /* Shared memory: per-thread FP64 global sums [12][blockDim], per-thread
   * path sums [10][blockDim], the receiver-side sums, the first traversal
   * stack entries [8][blockDim]; shared memory left unused goes to the L1
   * cache */
  extern __shared__ double smem[];
  __shared__ double red[MAX_BLOCK / 32][2 * NGLOBAL];
  const int bd = blockDim.x, tid = threadIdx.x;
  const unsigned lane = tid & 31u;
  const bool use_smem_rcv = S.nrcv <= SMEM_RCV_MAX;
  double* acc = smem + tid;
  double* ps = smem + 2 * NGLOBAL * bd + tid;
  double* smem_rcv = use_smem_rcv ? smem + (2 * NGLOBAL + PS_COUNT) * bd : nullptr;
  const int rcv_doubles = use_smem_rcv ? S.nrcv * NRCV_Q * 2 : 0;
  int* stack = reinterpret_cast<int*>(smem + (2 * NGLOBAL + PS_COUNT) * bd
                                      + rcv_doubles) + tid;
  for(int q = 0; q < 2 * NGLOBAL; ++q) acc[q * bd] = 0;
  for(int i = tid; i < rcv_doubles; i += bd) smem_rcv[i] = 0;
  __syncthreads();

  Rng rng;
  rng.k0 = (uint32_t)seed;
  rng.k1 = (uint32_t)(seed >> 32);
  PathState<R> p;
  p.phase = PH_NONE;
  bool done = false;
  Counters cnt = {0, 0, 0, 0};
  uint32_t bounces = 0, npaths = 0;
  int xr[MAX_EXTRA], xp[MAX_EXTRA];
  double xv[MAX_EXTRA][6];
  double racc[2 * NRCV_Q];
  int racc_slot = -1;

  /* Coherent order: the warp's current segment [seg_cur, seg_end) of the
   * sorted realisations */
  uint32_t seg_cur = 0, seg_end = 0;
  const uint32_t nseg = (uint32_t)((count + SORT_SEG - 1) / SORT_SEG);
  const bool polled = ctl.stop || ctl.abort;
  uint32_t fetches = 0;

  for(;;) {
    /* Regeneration: idle lanes take the next realisations */
    const unsigned need = __ballot_sync(0xffffffffu, p.phase == PH_NONE && !done);
    bool start = false;
    uint64_t off = 0;
    U32x4 r0;
    /* Early stop: every 8th fetch of the warp reads the stop and abort
     * words (one L2 sector); a halted warp takes no new realisation and ends
     * once its paths in flight end */
    bool halt = false;
    if(need && polled && (fetches++ & 7u) == 0u) {
      const int leader = __ffs(need) - 1;
      int h = 0;
      if((int)lane == leader) {
        if(ctl.stop && *(volatile const unsigned long long*)ctl.stop) h = 1;
        if(ctl.abort && *(volatile const unsigned long long*)ctl.abort) h = 1;
      }
      halt = __shfl_sync(0xffffffffu, h, leader) != 0;
    }
    if(halt) {
      if(p.phase == PH_NONE) done = true;
    } else if(need && sorted_off) {
      /* Segments of SORT_SEG sorted realisations (one or two primitives) go
       * to warps whole, in a strided order, so that a warp's lanes start on
       * the same heliostat while the warps of the GPU spread over the field */
      const int leader = __ffs(need) - 1;
      const unsigned rank = __popc(need & ((1u << lane) - 1u));
      const unsigned c = __popc(need);
      const unsigned avail = seg_end - seg_cur;
      uint32_t idx = 0;
      bool got = rank < avail, exhausted = false;
      if(got) idx = seg_cur + rank;
      if(c > avail) {
        unsigned long long sg = 0;
        if((int)lane == leader) sg = atomicAdd(next_path, 1ull);
        sg = __shfl_sync(0xffffffffu, sg, leader);
        if(sg < nseg) {
          const uint32_t s0 = (uint32_t)((sg * seg_mul) % nseg) * SORT_SEG;
          const uint32_t s1 = (uint32_t)min((uint64_t)s0 + SORT_SEG, count);
          if(!got && rank - avail < s1 - s0) {
            idx = s0 + (rank - avail);
            got = true;
          }
          seg_cur = s0 + min(c - avail, s1 - s0);
          seg_end = s1;
        } else {
          seg_cur = seg_end;
          exhausted = true;
        }
      } else {
        seg_cur += c;
      }
      if(p.phase == PH_NONE && !done) {
        if(got) {
          start = true;
          /* read once: streaming loads, evicted from L2 first */
          off = __ldcs(&sorted_off[idx]);
          const uint4 d = __ldcs(&sorted_draw[idx]);
          r0 = {{d.x, d.y, d.z, d.w}};
        } else if(exhausted) {
          done = true;
        }
      }
    } else if(need) {
      const int leader = __ffs(need) - 1;
      unsigned long long base = 0;
      if((int)lane == leader)
        base = atomicAdd(next_path, (unsigned long long)__popc(need));
      base = __shfl_sync(0xffffffffu, base, leader);
      if(p.phase == PH_NONE && !done) {
        const unsigned long long idx = base + __popc(need & ((1u << lane) - 1u));
        if(idx >= count) {
          done = true;
        } else {
          start = true;
          off = idx;
        }
      }
    }
    /* One init_path for both orders, so that a realisation computes the same
     * bits whichever order it runs in */
    if(start) {
      const uint64_t id = first + off;
      rng.i_lo = (uint32_t)id;
      rng.i_hi = (uint32_t)(id >> 32);
      if(!sorted_off) r0 = rng.get(0u, RNG_PRIMARY);
      init_path<R, FEAT>(S, rng, p, ps, bd, &r0);
      ++npaths;
      if(TRACK) {
        p.tslot = off < tr.npaths ? (int)off : -1;
        p.tseq = 0;
        if(p.tslot >= 0) {
          if(tr.sun_len > 0)
            track_vertex(tr, p, p.org + p.rd * (R)tr.sun_len, S.dni);
          track_vertex(tr, p, p.org, p.prev[0]);
        }
      }
    }
    if(!__any_sync(0xffffffffu, p.phase != PH_NONE)) break;

    /* One ray per active lane */
    Hit<R> h;
    bool found = false;
    if(p.phase != PH_NONE) {
      const bool shadow = p.phase == PH_SHADOW;
      SelfInfo self;
      self.gid = p.gid;
      self.sinst = p.sinst;
      self.side = p.side;
      self.discard_virtual = shadow;
      self.reversed = shadow;
      found = trace_ray<R, FEAT>(S, p.org, p.rd, p.tmin, self, shadow, h, cnt, stack, bd);
    }

    int end = END_NONE;
    bool do_interact = false;
    V3<R> pos = p.org, dir = -p.rd;
    if(p.phase == PH_SHADOW) {
      if(found) end = END_SHADOW;
      else {
        /* The path starts at the sampled point along the sun direction; a
         * virtual sampled surface pursues that ray (src/ssol_solver.c:
         * 988-995), not the shadow ray */
        p.rd = dir;
        do_interact = true;
      }
    } else if(p.phase == PH_BOUNCE) {
      if(!found) {
        if(TRACK && p.tslot >= 0 && tr.inf_len > 0) {
          const V3<R> last = p.virt ? p.org + p.rd * p.hit_t : p.org;
          track_vertex(tr, p, last + p.rd * (R)tr.inf_len, p.virt ? p.inc0 : p.prev[0]);
        }
        /* Last segment: the medium the ray leaves into must be the air
         * (src/ssol_solver.c:1012-1032) */
        if(p.out_medium != S.air_medium) {
          end = END_FAIL;
        } else {
          if(p.virt) {
            const double loss = p.prev[0] - p.inc0;
            ps[(p.medium == S.air_medium ? PS_ATM : PS_OTHER) * bd] += loss;
          }
          end = END_MISS;
        }
      } else {
        /* Russian roulette on deep paths (src/ssol_solver.c:1056-1075) */
        p.depth += p.virt ? 0u : 1u;
        if(p.depth > p.interval && p.depth % p.interval == 1) {
          const double u = u01d(rng.get(p.nroul++, RNG_ROULETTE).v[0]);
          if(u > 0.5) {
            ++p.score;
            p.interval = 16;
          } else {
            end = END_KILL;
          }
        }
        if(end == END_NONE) {
          /* point_update_from_hit (src/ssol_solver.c:360-411) */
          p.sinst = h.sinst;
          p.prim = h.prim;
          p.gid = h.gid;
          dir = p.rd;
          p.N = normalize(h.n);
          pos = p.org + p.rd * h.t;
          if((FEAT & FEAT_ATTRIBUTES) && S.tshade && h.gid >= 0) {
            const float2 uv = tri_uv(S, h.gid, pos);
            put_uv(ps, bd, uv.x, uv.y);
          }
          if(TRACK && p.tslot >= 0)
            track_vertex(tr, p, pos, p.virt ? p.inc0 : p.prev[0]);
          p.side = dot(p.rd, p.N) < R(0) ? 1 : 2;
          if(p.side == 2) p.N = -p.N;
          p.hit_t = h.t;
          p.medium = p.out_medium;
          do_interact = true;
        }
      }
    }
    if(do_interact)
      end = interact<R, FEAT>(S, rng, p, pos, dir, bounces, max_segments, ps, bd, xr, xp, xv);
    if(end != END_NONE) {
      if(TRACK && p.tslot >= 0 && end != END_KILL) {
        /* src/ssol_solver.c:931, 1092-1094, 1122-1125; killed paths are not
         * registered (1111) */
        tr.path_type[p.tslot] = end == END_SHADOW ? 1
          : (end == END_FAIL || p.overflow) ? 3 : (p.nent > 0 ? 2 : 0);
        tr.path_nv[p.tslot] = (int32_t)p.tseq;
      }
      racc_slot = commit_path(S, T, p, end, acc, ps, bd, smem_rcv, xr, xp, xv,
                              racc, racc_slot, &ctl);
      p.phase = PH_NONE;
    }
  }

  if(racc_slot >= 0)
    flush_racc((use_smem_rcv ? smem_rcv : T.rcv) + (size_t)racc_slot * NRCV_Q * 2, racc,
               use_smem_rcv);

  /* Warp then block reduction of the global sums, one commit per block */
  const int warp = tid >> 5;
  for(int q = 0; q < 2 * NGLOBAL; ++q) {
    const double s = warp_sum(acc[q * bd]);
    if(lane == 0) red[warp][q] = s;
  }
  unsigned long long c[6] = {cnt.rays, cnt.nodes, cnt.tris, cnt.quads,
                             bounces, npaths};
  for(int q = 0; q < 6; ++q) c[q] = warp_sum_u64(c[q]);
  if(lane == 0) {
    unsigned long long* st = &T.stats->rays;
    for(int q = 0; q < 6; ++q) if(c[q]) atomicAdd(st + q, c[q]);
  }
  __syncthreads();
  if(tid < 2 * NGLOBAL) {
    double v = 0;
    for(int w = 0; w < (bd >> 5); ++w) v += red[w][tid];
    red_add_global(T.global + tid, v);
  }
  for(int i = tid; i < rcv_doubles; i += bd) red_add_global(T.rcv + i, smem_rcv[i]);
}

/* Batched form: several scenes (e.g. one re-aimed field per sun position)
 * and their realisation budgets in one persistent launch. Global work index
 * g maps to item it = max{i : prefix[i] <= g} and to realisation
 * firsts[it] + g - prefix[it] of that item's streams. Every item has its own
 * tallies; the per-thread FP64 global sums are flushed when a thread moves
 * to another item. The launch's total is prefix[nitems], read from device
 * memory so that a captured CUDA graph replays with new budgets. */
template<class R, int MINB, int FEAT>
__global__ void __launch_bounds__(MAX_BLOCK, MINB)
batch_kernel
  (const DScene<R>* __restrict__ scenes, const DTallies* __restrict__ tallies,
   const unsigned long long* __restrict__ prefix,
   const unsigned long long* __restrict__ firsts, int nitems, uint64_t seed,
   unsigned long long max_segments, unsigned long long* next_items,
   DStats* stats, int rcvd, const uint32_t* __restrict__ sorted_off,
   const uint4* __restrict__ sorted_draw, const uint32_t* __restrict__ seg_mul)
{
  extern __shared__ double smem[];
  const int bd = blockDim.x, tid = threadIdx.x;
  const unsigned lane = tid & 31u;
  double* acc = smem + tid;
  double* ps = smem + 2 * NGLOBAL * bd + tid;
  int* stack = reinterpret_cast<int*>(smem + (2 * NGLOBAL + PS_COUNT) * bd) + tid;
  for(int q = 0; q < 2 * NGLOBAL; ++q) acc[q * bd] = 0;
  int acc_item = -1;
  /* Global and receiver sums: every path adds to the same few addresses of
   * its item, so they are gathered per warp in two shared-memory slots
   * tagged with an item (the warp's current item and the previous one, for
   * the paths still running across an item boundary) and flushed to the
   * item's tallies when the warp moves on: one device atomic per warp and
   * address for each item instead of one per thread. A slot holds the
   * 2 x NGLOBAL global sums, then `rcvd` receiver sums. Tags change only
   * where the warp is converged. */
  const int ss = 2 * NGLOBAL + rcvd;
  double* wslots = reinterpret_cast<double*>(
    reinterpret_cast<int*>(smem + (2 * NGLOBAL + PS_COUNT) * bd) + SMEM_STACK * bd)
    + (size_t)(tid >> 5) * 2 * ss;
  for(int i = (int)lane; i < 2 * ss; i += 32) wslots[i] = 0;
  /* Copies of the two tagged items' scene records, so that lanes on those
   * items read their scene from shared memory instead of device memory */
  DScene<R>* wscene = reinterpret_cast<DScene<R>*>(
    reinterpret_cast<double*>(reinterpret_cast<int*>(smem + (2 * NGLOBAL + PS_COUNT) * bd)
                              + SMEM_STACK * bd) + (size_t)(bd >> 5) * 2 * ss)
    + (size_t)(tid >> 5) * 2;
  __syncwarp();
  int stag[2] = {-1, -1};
  int cur = 0;
  auto scene_of = [&](int item) -> const DScene<R>& {
    return item == stag[cur] ? wscene[cur] : item == stag[cur ^ 1] ? wscene[cur ^ 1]
                                                                   : scenes[item];
  };

  /* Work: every item has its own counter (next_items). The SMs form groups
   * of group_sms; group g works through its own items g, g + G, g + 2G, ...
   * in turn, then through the next groups' lists, taking its realisations
   * from the first item of the sequence with work left. The warps of an SM
   * thus stay long on one item (its scene arrays stay warm in L1 and the
   * item tags rarely change), and only about G items are open at a time
   * (their arrays and tallies stay in L2). Positions q of the sequence map
   * to items (q % L) x G + q / L, L = ceil(nitems / G); those past the last
   * item are skipped. Measured on 256 field items: with one counter over
   * all items (every warp moved to the next item at the same time, its
   * arrays cold for all of them) 1e5 realisations per item ran at 199
   * Mpaths/s; with every SM starting on its own item 416, and 1e6 per item
   * 436 (about 150 items open). */
  const unsigned long long total = prefix[nitems];
  unsigned smid, nsmid;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
  asm volatile("mov.u32 %0, %%nsmid;" : "=r"(nsmid));
  const unsigned group_sms = total < BATCH_LARGE_ITEM * (unsigned long long)nitems
                            ? BATCH_GROUP_SMALL : BATCH_GROUP_LARGE;
  const int ngroups = min(nitems, max(1, (int)(nsmid / group_sms)));
  const int seq_len = (nitems + ngroups - 1) / ngroups;
  const int npos = ngroups * seq_len;
  int wq = (int)(min(smid, nsmid - 1) * (unsigned)ngroups / nsmid) * seq_len;
  int wit = 0;
  Rng rng;
  rng.k0 = (uint32_t)seed;
  rng.k1 = (uint32_t)(seed >> 32);
  PathState<R> p;
  p.phase = PH_NONE;
  int it = 0;
  bool done = total == 0;
  Counters cnt = {0, 0, 0, 0};
  uint32_t bounces = 0, npaths = 0;
  int xr[MAX_EXTRA], xp[MAX_EXTRA];
  double xv[MAX_EXTRA][6];
  /* Running sums of one (item, receiver side), as in realisation_kernel;
   * flushed into the item's warp slot (or its tallies) when either changes */
  double racc[2 * NRCV_Q];
  int racc_slot = -1, racc_item = -1;
  auto racc_flush = [&]() {
    if(racc_slot < 0) return;
    const bool in_slot = rcvd && (racc_item == stag[cur] || racc_item == stag[cur ^ 1]);
    double* dst = rcvd && racc_item == stag[cur] ? wslots + cur * ss + 2 * NGLOBAL
      : rcvd && racc_item == stag[cur ^ 1] ? wslots + (cur ^ 1) * ss + 2 * NGLOBAL
      : tallies[racc_item].rcv;
    flush_racc(dst + (size_t)racc_slot * NRCV_Q * 2, racc, in_slot);
    racc_slot = -1;
  };

  for(;;) {
    const unsigned need = __ballot_sync(0xffffffffu, p.phase == PH_NONE && !done);
    if(need) {
      const int leader = __ffs(need) - 1;
      unsigned long long base = 0;
      int item = wit, got = 0, q = wq;
      if((int)lane == leader) {
        /* The warp's position, or the next ones in turn, until an item has
         * work */
        for(int k = 0; k < npos; ++k) {
          item = (q % seq_len) * ngroups + q / seq_len;
          if(item < nitems) {
            const unsigned long long budget = prefix[item + 1] - prefix[item];
            if(*(volatile const unsigned long long*)(next_items + item) < budget) {
              base = atomicAdd(next_items + item, (unsigned long long)__popc(need));
              if(base < budget) { got = 1; break; }
            }
          }
          q = q + 1 == npos ? 0 : q + 1;
        }
      }
      got = __shfl_sync(0xffffffffu, got, leader);
      item = __shfl_sync(0xffffffffu, item, leader);
      q = __shfl_sync(0xffffffffu, q, leader);
      base = __shfl_sync(0xffffffffu, base, leader);
      if(got) { wit = item; wq = q; }
      if(p.phase == PH_NONE && !done) {
        const unsigned long long g = base + __popc(need & ((1u << lane) - 1u));
        if(!got) {
          done = true;
        } else if(g < prefix[item + 1] - prefix[item]) {
          /* lanes past the item's end take work at the next fetch */
          it = item;
          if(it != acc_item) {
            if(acc_item >= 0) {
              double* sl = acc_item == stag[cur] ? wslots + cur * ss
                : acc_item == stag[cur ^ 1] ? wslots + (cur ^ 1) * ss : nullptr;
              for(int q = 0; q < 2 * NGLOBAL; ++q) {
                const double v = acc[q * bd];
                if(v != 0.0) {
                  if(sl) atomicAdd(sl + q, v);
                  else red_add(tallies[acc_item].global + q, v);
                }
                acc[q * bd] = 0;
              }
            }
            acc_item = it;
          }
          /* Coherent order: the item's full warp segments of SORT_SEG
           * sorted realisations in a strided order (so that the warps of an
           * item group spread over its primitives), the ragged last one
           * last; each record gives the realisation and its primary draw */
          uint64_t off = g;
          U32x4 r0;
          if(sorted_off) {
            const unsigned long long nfull = (prefix[it + 1] - prefix[it]) / SORT_SEG;
            unsigned long long sg = g / SORT_SEG;
            if(sg < nfull)
              sg = nfull < 65536ull
                ? (unsigned long long)((uint32_t)sg * seg_mul[it] % (uint32_t)nfull)
                : sg * seg_mul[it] % nfull;
            const unsigned long long rec = prefix[it] + sg * SORT_SEG + g % SORT_SEG;
            off = __ldcs(&sorted_off[rec]);
            const uint4 d = __ldcs(&sorted_draw[rec]);
            r0 = {{d.x, d.y, d.z, d.w}};
          }
          const uint64_t id = firsts[it] + off;
          rng.i_lo = (uint32_t)id;
          rng.i_hi = (uint32_t)(id >> 32);
          if(!sorted_off) r0 = rng.get(0u, RNG_PRIMARY);
          init_path<R, FEAT>(scene_of(it), rng, p, ps, bd, &r0);
          ++npaths;
        }
      }
      {
        /* Converged: the item fetched becomes the current slot */
        const int newest = got ? wit : -1;
        if(newest >= 0 && newest != stag[cur]) {
          const int prv = cur ^ 1;
          double* sl = wslots + prv * ss;
          __syncwarp();
          if(stag[prv] >= 0) {
            if((int)lane < 2 * NGLOBAL) red_add(tallies[stag[prv]].global + lane, sl[lane]);
            double* dst = tallies[stag[prv]].rcv;
            const int nd = rcvd ? scenes[stag[prv]].nrcv * NRCV_Q * 2 : 0;
            for(int i = (int)lane; i < nd; i += 32) red_add(dst + i, sl[2 * NGLOBAL + i]);
          }
          /* The lanes clear other entries than they flushed: every read of
           * the slot before any clear */
          __syncwarp();
          for(int i = (int)lane; i < ss; i += 32) sl[i] = 0;
          {
            const int* src = reinterpret_cast<const int*>(scenes + newest);
            int* dst = reinterpret_cast<int*>(wscene + prv);
            constexpr int words = (int)(sizeof(DScene<R>) / sizeof(int));
            for(int i = (int)lane; i < words; i += 32) dst[i] = src[i];
          }
          __syncwarp();
          stag[prv] = newest;
          cur = prv;
        }
      }
    }
    if(!__any_sync(0xffffffffu, p.phase != PH_NONE)) break;

    const DScene<R>& S = scene_of(it);
    Hit<R> h;
    bool found = false;
    if(p.phase != PH_NONE) {
      const bool shadow = p.phase == PH_SHADOW;
      SelfInfo self;
      self.gid = p.gid;
      self.sinst = p.sinst;
      self.side = p.side;
      self.discard_virtual = shadow;
      self.reversed = shadow;
      found = trace_ray<R, FEAT>(S, p.org, p.rd, p.tmin, self, shadow, h, cnt, stack, bd);
    }

    int end = END_NONE;
    bool do_interact = false;
    V3<R> pos = p.org, dir = -p.rd;
    if(p.phase == PH_SHADOW) {
      if(found) end = END_SHADOW;
      else {
        /* The path starts at the sampled point along the sun direction; a
         * virtual sampled surface pursues that ray (src/ssol_solver.c:
         * 988-995), not the shadow ray */
        p.rd = dir;
        do_interact = true;
      }
    } else if(p.phase == PH_BOUNCE) {
      if(!found) {
        if(p.out_medium != S.air_medium) {
          end = END_FAIL;
        } else {
          if(p.virt) {
            const double loss = p.prev[0] - p.inc0;
            ps[(p.medium == S.air_medium ? PS_ATM : PS_OTHER) * bd] += loss;
          }
          end = END_MISS;
        }
      } else {
        p.depth += p.virt ? 0u : 1u;
        if(p.depth > p.interval && p.depth % p.interval == 1) {
          const double u = u01d(rng.get(p.nroul++, RNG_ROULETTE).v[0]);
          if(u > 0.5) {
            ++p.score;
            p.interval = 16;
          } else {
            end = END_KILL;
          }
        }
        if(end == END_NONE) {
          p.sinst = h.sinst;
          p.prim = h.prim;
          p.gid = h.gid;
          dir = p.rd;
          p.N = normalize(h.n);
          pos = p.org + p.rd * h.t;
          if((FEAT & FEAT_ATTRIBUTES) && S.tshade && h.gid >= 0) {
            const float2 uv = tri_uv(S, h.gid, pos);
            put_uv(ps, bd, uv.x, uv.y);
          }
          p.side = dot(p.rd, p.N) < R(0) ? 1 : 2;
          if(p.side == 2) p.N = -p.N;
          p.hit_t = h.t;
          p.medium = p.out_medium;
          do_interact = true;
        }
      }
    }
    if(do_interact)
      end = interact<R, FEAT>(S, rng, p, pos, dir, bounces, max_segments, ps, bd, xr, xp, xv);
    if(end != END_NONE) {
      double* rb = nullptr;
      if(rcvd) {
        if(it == stag[cur]) rb = wslots + cur * ss + 2 * NGLOBAL;
        else if(it == stag[cur ^ 1]) rb = wslots + (cur ^ 1) * ss + 2 * NGLOBAL;
      }
      if(racc_item != it) racc_flush();
      racc_item = it;
      racc_slot = commit_path(S, tallies[it], p, end, acc, ps, bd, rb, xr, xp, xv,
                              racc, racc_slot, (const DControl*)nullptr);
      p.phase = PH_NONE;
    }
  }

  racc_flush();
  if(acc_item >= 0) {
    double* sl = acc_item == stag[cur] ? wslots + cur * ss
      : acc_item == stag[cur ^ 1] ? wslots + (cur ^ 1) * ss : nullptr;
    for(int q = 0; q < 2 * NGLOBAL; ++q) {
      const double v = acc[q * bd];
      if(v == 0.0) continue;
      if(sl) atomicAdd(sl + q, v);
      else red_add(tallies[acc_item].global + q, v);
    }
  }
  __syncwarp();
  for(int k = 0; k < 2; ++k) {
    if(stag[k] < 0) continue;
    if((int)lane < 2 * NGLOBAL)
      red_add(tallies[stag[k]].global + lane, wslots[k * ss + lane]);
    double* dst = tallies[stag[k]].rcv;
    const int nd = rcvd ? scenes[stag[k]].nrcv * NRCV_Q * 2 : 0;
    for(int i = (int)lane; i < nd; i += 32)
      red_add(dst + i, wslots[k * ss + 2 * NGLOBAL + i]);
  }
  unsigned long long c[6] = {cnt.rays, cnt.nodes, cnt.tris, cnt.quads,
                             bounces, npaths};
  for(int q = 0; q < 6; ++q) c[q] = warp_sum_u64(c[q]);
  if(lane == 0) {
    unsigned long long* st = &stats->rays;
    for(int q = 0; q < 6; ++q) if(c[q]) atomicAdd(st + q, c[q]);
  }
}

/*******************************************************************************
 * Coherent order. The realisations of a launch, chunk by chunk, are sorted by
 * the primitive their primary draw samples (a counting sort), so that the
 * lanes of a warp start on the same or neighbouring heliostats and trace
 * nearly parallel shadow and reflected rays. Every realisation is traced once
 * with its own stream; only the order, and so the order of the FP64 sums,
 * changes. The primary draw travels with the sorted offset so that init_path
 * does not draw it again.
 ******************************************************************************/

/* Sampled primitive of realisation first + j, counted per block in shared
 * memory */
template<class R>
__global__ void __launch_bounds__(256) presort_count
  (const DScene<R> S, uint64_t seed, uint64_t first, uint32_t n, uint32_t* hist)
{
  __shared__ uint32_t h[SORT_MAX_BINS];
  for(int i = threadIdx.x; i < S.nsamp; i += blockDim.x) h[i] = 0;
  __syncthreads();
  Rng rng;
  rng.k0 = (uint32_t)seed;
  rng.k1 = (uint32_t)(seed >> 32);
  for(uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n;
      j += gridDim.x * blockDim.x) {
    const uint64_t id = first + j;
    rng.i_lo = (uint32_t)id;
    rng.i_hi = (uint32_t)(id >> 32);
    atomicAdd(&h[sample_prim(S, rng.get(0u, RNG_PRIMARY))], 1u);
  }
  __syncthreads();
  for(int i = threadIdx.x; i < S.nsamp; i += blockDim.x)
    if(h[i]) atomicAdd(&hist[i], h[i]);
}

/* Exclusive prefix sum of the nb histogram bins, one block of 1024 threads */
static __global__ void __launch_bounds__(1024) presort_scan
  (const uint32_t* hist, uint32_t* off, int nb)
{
  __shared__ uint32_t part[1024];
  const int t = threadIdx.x;
  const int per = (nb + 1023) / 1024;
  const int b0 = min(t * per, nb), b1 = min(b0 + per, nb);
  uint32_t sum = 0;
  for(int i = b0; i < b1; ++i) sum += hist[i];
  part[t] = sum;
  __syncthreads();
  for(int d = 1; d < 1024; d <<= 1) {
    const uint32_t v = t >= d ? part[t - d] : 0u;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  uint32_t run = t ? part[t - 1] : 0u;
  for(int i = b0; i < b1; ++i) {
    off[i] = run;
    run += hist[i];
  }
}

/* Each realisation to the next free place of its primitive's range. A block
 * ranks a tile of SCATTER_PER x 256 realisations in shared memory, reserves
 * one range per primitive of the tile with a single global atomic, then
 * writes: one global atomic per (tile, primitive) instead of one per
 * realisation */
constexpr int SCATTER_PER = 16;

template<class R>
__global__ void __launch_bounds__(256) presort_scatter
  (const DScene<R> S, uint64_t seed, uint64_t first, uint32_t n, uint32_t* off,
   uint4* out_draws, uint32_t* out_off)
{
  __shared__ uint32_t cnt[SORT_MAX_BINS];
  const int nb = S.nsamp;
  const uint32_t tile = 256u * SCATTER_PER;
  Rng rng;
  rng.k0 = (uint32_t)seed;
  rng.k1 = (uint32_t)(seed >> 32);
  for(uint32_t t0 = blockIdx.x * tile; t0 < n; t0 += gridDim.x * tile) {
    for(int i = threadIdx.x; i < nb; i += 256) cnt[i] = 0;
    __syncthreads();
    uint32_t k[SCATTER_PER], rank[SCATTER_PER];
#pragma unroll
    for(int e = 0; e < SCATTER_PER; ++e) {
      const uint32_t j = t0 + e * 256u + threadIdx.x;
      k[e] = 0u;
      rank[e] = 0u;
      if(j < n) {
        const uint64_t id = first + j;
        rng.i_lo = (uint32_t)id;
        rng.i_hi = (uint32_t)(id >> 32);
        k[e] = (uint32_t)sample_prim(S, rng.get(0u, RNG_PRIMARY));
        rank[e] = atomicAdd(&cnt[k[e]], 1u);
      }
    }
    __syncthreads();
    for(int i = threadIdx.x; i < nb; i += 256)
      if(cnt[i]) cnt[i] = atomicAdd(&off[i], cnt[i]);
    __syncthreads();
    /* The draws again rather than kept: 16 more registers per realisation
     * of the tile, or 20 B of scratch per realisation */
#pragma unroll
    for(int e = 0; e < SCATTER_PER; ++e) {
      const uint32_t j = t0 + e * 256u + threadIdx.x;
      if(j < n) {
        const uint32_t pos = cnt[k[e]] + rank[e];
        const uint64_t id = first + j;
        rng.i_lo = (uint32_t)id;
        rng.i_hi = (uint32_t)(id >> 32);
        const U32x4 r0 = rng.get(0u, RNG_PRIMARY);
        out_draws[pos] = make_uint4(r0.v[0], r0.v[1], r0.v[2], r0.v[3]);
        out_off[pos] = j;
      }
    }
    __syncthreads();
  }
}

/* Coherent order of a batched launch. Every size comes from the launch's
 * device arrays (prefix: the budgets' inclusive prefix, prefix[nitems] the
 * total), so that a captured graph serves any budgets. Item of realisation
 * j: prefix[item] <= j < prefix[item + 1]. */
__device__ __forceinline__ int batch_item_of
  (const unsigned long long* prefix, int nitems, unsigned long long j, int hint)
{
  if(prefix[hint] <= j && j < prefix[hint + 1]) return hint;
  int lo = 0, hi = nitems;
  while(hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if(prefix[mid] <= j) lo = mid; else hi = mid;
  }
  return lo;
}

/* Sampled primitive of every realisation of the launch, counted in one
 * histogram whose bins run item by item (bin_base) */
template<class R>
__global__ void __launch_bounds__(256) batch_presort_count
  (const DScene<R>* scenes, const unsigned long long* prefix,
   const unsigned long long* firsts, int nitems, uint64_t seed,
   const uint32_t* bin_base, uint32_t* hist)
{
  const unsigned long long total = prefix[nitems];
  Rng rng;
  rng.k0 = (uint32_t)seed;
  rng.k1 = (uint32_t)(seed >> 32);
  int item = 0;
  for(unsigned long long j = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
      j < total; j += (unsigned long long)gridDim.x * blockDim.x) {
    item = batch_item_of(prefix, nitems, j, item);
    const uint64_t id = firsts[item] + (j - prefix[item]);
    rng.i_lo = (uint32_t)id;
    rng.i_hi = (uint32_t)(id >> 32);
    const int k = sample_prim(scenes[item], rng.get(0u, RNG_PRIMARY));
    atomicAdd(&hist[bin_base[item] + (uint32_t)k], 1u);
  }
}

/* Each realisation to the next free place of its (item, primitive) range,
 * with its offset in the item and its primary draw (drawn again: the
 * scratch keeps only the sorted records, 20 B per realisation) */
template<class R>
__global__ void __launch_bounds__(256) batch_presort_scatter
  (const DScene<R>* scenes, const unsigned long long* prefix,
   const unsigned long long* firsts, int nitems, uint64_t seed,
   const uint32_t* bin_base, uint32_t* bin_off, uint32_t* sorted_off,
   uint4* sorted_draw)
{
  const unsigned long long total = prefix[nitems];
  Rng rng;
  rng.k0 = (uint32_t)seed;
  rng.k1 = (uint32_t)(seed >> 32);
  int item = 0;
  for(unsigned long long j = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
      j < total; j += (unsigned long long)gridDim.x * blockDim.x) {
    item = batch_item_of(prefix, nitems, j, item);
    const uint64_t id = firsts[item] + (j - prefix[item]);
    rng.i_lo = (uint32_t)id;
    rng.i_hi = (uint32_t)(id >> 32);
    const U32x4 r0 = rng.get(0u, RNG_PRIMARY);
    const int k = sample_prim(scenes[item], r0);
    const uint32_t pos = atomicAdd(&bin_off[bin_base[item] + (uint32_t)k], 1u);
    sorted_off[pos] = (uint32_t)(j - prefix[item]);
    sorted_draw[pos] = make_uint4(r0.v[0], r0.v[1], r0.v[2], r0.v[3]);
  }
}

/* Per-device pool of the sort's scratch (kernels_plain.cu) */
cudaMemPool_t sort_pool(int dev);

static size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

/*******************************************************************************
 * Host launchers
 ******************************************************************************/

/* The dynamic shared-memory limit of a kernel is an attribute of one
 * device's context: raise it once per (kernel, device). `Tag` tells the
 * kernels apart (one set of flags per template instance). */
template<class Tag, class K>
static void raise_smem_limit(K kernel, int dev)
{
  static std::atomic<unsigned long long> done_mask{0};
  const unsigned long long bit = dev >= 0 && dev < 64 ? 1ull << dev : 0ull;
  if(bit && (done_mask.load(std::memory_order_acquire) & bit)) return;
  if(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          160 * 1024) == cudaSuccess && bit)
    done_mask.fetch_or(bit, std::memory_order_acq_rel);
}
template<class R, int MINB, bool TRACK, int FEAT> struct RealisationTag {};
template<class R, int MINB, int FEAT> struct BatchTag {};

template<class R, int MINB, bool TRACK, int FEAT>
static int launch_variant
  (const DScene<R>& S, const DTallies& T, uint64_t seed, uint64_t first,
   uint64_t count, const LaunchConfig& cfg, void* stream, const DTrack& tr)
{
  int dev = 0;
  cudaGetDevice(&dev);
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int block = cfg.block_size > 0 ? cfg.block_size : MAX_BLOCK;
  if(block > MAX_BLOCK || block % 32) return (int)cudaErrorInvalidValue;
  const int rcv_doubles = S.nrcv <= SMEM_RCV_MAX ? S.nrcv * NRCV_Q * 2 : 0;
  const size_t smem = (size_t)((2 * NGLOBAL + PS_COUNT) * block + rcv_doubles)
                      * sizeof(double)
                    + (size_t)SMEM_STACK * block * sizeof(int);
  raise_smem_limit<RealisationTag<R, MINB, TRACK, FEAT>>(realisation_kernel<R, MINB, TRACK, FEAT>, dev);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor
    (&per_sm, realisation_kernel<R, MINB, TRACK, FEAT>, block, smem);
  if(per_sm < 1) per_sm = 1;
  uint64_t blocks = cfg.grid_blocks > 0
    ? (uint64_t)cfg.grid_blocks
    : (uint64_t)nsm * (uint64_t)per_sm * (uint64_t)(cfg.waves > 0 ? cfg.waves : 1);
  const uint64_t needed = (count + block - 1) / block;
  if(blocks > needed) blocks = needed;
  if(blocks < 1) blocks = 1;
  const cudaStream_t st = (cudaStream_t)stream;
  const bool sort = !TRACK && cfg.coherent && count >= SORT_MIN && S.nsamp > 1
                 && S.nsamp <= SORT_MAX_BINS;
  DControl ctl;
  ctl.max_failed = cfg.max_failed;
  ctl.stop = cfg.max_failed != ~0ull ? T.counters + 4 : nullptr;
  ctl.abort = cfg.abortable ? T.counters + 5 : nullptr;
  if(!sort) {
    /* Work counter of this launch: counters[3] */
    cudaMemsetAsync(T.counters + 3, 0, sizeof(unsigned long long), st);
    realisation_kernel<R, MINB, TRACK, FEAT><<<(unsigned)blocks, block, smem, st>>>
      (S, T, seed, first, count, cfg.max_segments, T.counters + 3, tr, nullptr,
       nullptr, 1u, ctl);
    return (int)cudaGetLastError();
  }
  const uint64_t chunk = count < SORT_CHUNK ? count : SORT_CHUNK;
  const size_t o_sdraws = 0;
  const size_t o_soff = o_sdraws + align256(chunk * sizeof(uint4));
  const size_t o_hist = o_soff + align256(chunk * sizeof(uint32_t));
  const size_t o_off = o_hist + align256((size_t)S.nsamp * sizeof(uint32_t));
  const size_t bytes = o_off + align256((size_t)S.nsamp * sizeof(uint32_t));
  cudaMemPool_t pool = sort_pool(dev);
  unsigned char* buf = nullptr;
  if(!pool || cudaMallocFromPoolAsync((void**)&buf, bytes, pool, st) != cudaSuccess)
    return (int)cudaErrorMemoryAllocation;
  uint4* sdraws = (uint4*)(buf + o_sdraws);
  uint32_t* soff = (uint32_t*)(buf + o_soff);
  uint32_t* hist = (uint32_t*)(buf + o_hist);
  uint32_t* off = (uint32_t*)(buf + o_off);
  const unsigned sort_blocks = (unsigned)nsm * 8u;
  for(uint64_t c0 = 0; c0 < count; c0 += chunk) {
    const uint32_t n = (uint32_t)(count - c0 < chunk ? count - c0 : chunk);
    cudaMemsetAsync(hist, 0, (size_t)S.nsamp * sizeof(uint32_t), st);
    presort_count<R><<<sort_blocks, 256, 0, st>>>(S, seed, first + c0, n, hist);
    presort_scan<<<1, 1024, 0, st>>>(hist, off, S.nsamp);
    presort_scatter<R><<<sort_blocks, 256, 0, st>>>(S, seed, first + c0, n, off, sdraws,
                                                    soff);
    uint64_t nb = (n + block - 1) / block;
    if(nb > blocks) nb = blocks;
    /* Segment s of the launch is segment (s x mul) mod nseg of the sorted
     * order, mul coprime with nseg and near nseg / golden ratio */
    const uint32_t nseg = (uint32_t)((n + SORT_SEG - 1) / SORT_SEG);
    uint32_t mul = (uint32_t)(0.6180339887 * nseg) | 1u;
    while(nseg > 1 && std::gcd(mul, nseg) != 1u) mul += 2;
    if(nseg <= 1) mul = 1;
    cudaMemsetAsync(T.counters + 3, 0, sizeof(unsigned long long), st);
    realisation_kernel<R, MINB, TRACK, FEAT><<<(unsigned)nb, block, smem, st>>>
      (S, T, seed, first + c0, n, cfg.max_segments, T.counters + 3, tr, sdraws, soff,
       mul, ctl);
  }
  cudaFreeAsync(buf, st);
  return (int)cudaGetLastError();
}

/* Feature variants of the FP32 kernel: meshes with mirror and matte
 * materials only, quadrics and dielectrics, or everything (vertex
 * attributes); the all-FP64 build, for precision checks, has the last one */
template<class R, int MINB, int NC>
static int launch_features
  (const DScene<R>& S, const DTallies& T, uint64_t seed, uint64_t first,
   uint64_t count, const LaunchConfig& cfg, void* stream)
{
  const DTrack none = {};
  if constexpr(sizeof(R) == sizeof(float)) {
    if(cfg.features == 0)
      return launch_variant<R, MINB, false, NC>(S, T, seed, first, count, cfg, stream, none);
    if(!(cfg.features & FEAT_ATTRIBUTES))
      return launch_variant<R, MINB, false, FEAT_QUADRIC | FEAT_DIELECTRIC | NC>
        (S, T, seed, first, count, cfg, stream, none);
  }
  return launch_variant<R, MINB, false, FEAT_ALL | NC>(S, T, seed, first, count, cfg, stream,
                                                       none);
}

/* Register budget variants: at least MINB blocks of 256 threads per SM; NC
 * is FEAT_NOCOUNT for the variants without work counters (path tracking
 * always counts) */
template<class R, int NC = 0>
static int launch_impl
  (const DScene<R>& S, const DTallies& T, uint64_t seed, uint64_t first,
   uint64_t count, const LaunchConfig& cfg, void* stream, const DTrack* track)
{
  if(track)
    return launch_variant<R, 2, true, FEAT_ALL>(S, T, seed, first, count, cfg, stream, *track);
  switch(cfg.min_blocks) {
    case 1: return launch_features<R, 1, NC>(S, T, seed, first, count, cfg, stream);
    case 3: return launch_features<R, 3, NC>(S, T, seed, first, count, cfg, stream);
    default: return launch_features<R, 2, NC>(S, T, seed, first, count, cfg, stream);
  }
}

template<class R, int MINB, int FEAT>
static int launch_batch_variant(const BatchLaunch<R>& b, const LaunchConfig& cfg,
                                void* stream)
{
  int dev = 0;
  cudaGetDevice(&dev);
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int block = cfg.block_size > 0 ? cfg.block_size : MAX_BLOCK;
  if(block > MAX_BLOCK || block % 32) return (int)cudaErrorInvalidValue;
  const size_t smem = (size_t)((2 * NGLOBAL + PS_COUNT) * block) * sizeof(double)
                    + (size_t)SMEM_STACK * block * sizeof(int)
                    + (size_t)(block / 32) * 2 * (2 * NGLOBAL + cfg.rcv_doubles) * sizeof(double)
                    + (size_t)(block / 32) * 2 * sizeof(DScene<R>);
  raise_smem_limit<BatchTag<R, MINB, FEAT>>(batch_kernel<R, MINB, FEAT>, dev);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor
    (&per_sm, batch_kernel<R, MINB, FEAT>, block, smem);
  if(per_sm < 1) per_sm = 1;
  const uint64_t blocks = cfg.grid_blocks > 0
    ? (uint64_t)cfg.grid_blocks
    : (uint64_t)nsm * (uint64_t)per_sm * (uint64_t)(cfg.waves > 0 ? cfg.waves : 1);
  const cudaStream_t st = (cudaStream_t)stream;
  const BatchOrder& o = b.order;
  if(o.sorted_off) {
    const unsigned sort_blocks = (unsigned)nsm * 8u;
    cudaMemsetAsync(o.hist, 0, (size_t)o.nbins * sizeof(uint32_t), st);
    batch_presort_count<R><<<sort_blocks, 256, 0, st>>>
      (b.scenes, b.prefix, b.firsts, b.nitems, b.seed, o.bin_base, o.hist);
    presort_scan<<<1, 1024, 0, st>>>(o.hist, o.bin_off, (int)o.nbins);
    batch_presort_scatter<R><<<sort_blocks, 256, 0, st>>>
      (b.scenes, b.prefix, b.firsts, b.nitems, b.seed, o.bin_base, o.bin_off,
       o.sorted_off, reinterpret_cast<uint4*>(o.sorted_draw));
  }
  cudaMemsetAsync(b.next_items, 0, (size_t)b.nitems * sizeof(unsigned long long), st);
  batch_kernel<R, MINB, FEAT><<<(unsigned)blocks, block, smem, st>>>
    (b.scenes, b.tallies, b.prefix, b.firsts, b.nitems, b.seed, cfg.max_segments,
     b.next_items, b.stats, cfg.rcv_doubles, o.sorted_off,
     reinterpret_cast<const uint4*>(o.sorted_draw), o.seg_mul);
  return (int)cudaGetLastError();
}

/* NC is FEAT_NOCOUNT for the variants without work counters */
template<class R, int NC = 0>
static int launch_batch_impl(const BatchLaunch<R>& b, const LaunchConfig& cfg,
                             void* stream)
{
  /* FP32 batches of meshes with mirror and matte materials only get the
   * smaller variant */
  if(sizeof(R) == sizeof(float) && cfg.features == 0) {
    switch(cfg.min_blocks) {
      case 1: return launch_batch_variant<R, 1, NC>(b, cfg, stream);
      case 3: return launch_batch_variant<R, 3, NC>(b, cfg, stream);
      default: return launch_batch_variant<R, 2, NC>(b, cfg, stream);
    }
  }
  switch(cfg.min_blocks) {
    case 1: return launch_batch_variant<R, 1, FEAT_ALL | NC>(b, cfg, stream);
    case 3: return launch_batch_variant<R, 3, FEAT_ALL | NC>(b, cfg, stream);
    default: return launch_batch_variant<R, 2, FEAT_ALL | NC>(b, cfg, stream);
  }
}

} /* namespace ssolb */

#endif /* SSOL_B200_KERNELS_DEVICE_CUH */
