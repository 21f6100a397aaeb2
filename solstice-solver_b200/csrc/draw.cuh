/*
 * draw.cuh - the preview renderers behind ssol_draw_draft and ssol_draw_pt
 * (src/ssol_draw.c, src/ssol_draw_draft.c, src/ssol_draw_pt.c) as CUDA
 * kernels that write a device image: width x height pixels of 3 doubles,
 * row after row. Included by kernels_aux.cu, whose ray casting (trace_ray with
 * the hit filter's "discard virtual materials" mode), Philox streams,
 * wavelength sampler, media and shader tables they share.
 *
 * One thread per pixel; a block of 256 threads covers a 16 x 16 tile and
 * each warp an 8 x 4 sub-tile, so that the camera rays of a warp are close
 * together. Each thread loops over its samples and writes its pixel once.
 *
 * Star-SF's BSDFs used for rendering (src/ssol_material.c:151-225 with
 * rendering = 1) are restated from published optics: Lambertian
 * (rho / pi, Malley cosine sampling), specular reflection, the same
 * dielectric and thin-slab samplers as the solver, and for rough mirrors a
 * Cook-Torrance microfacet BRDF F D G / (4 cos_o cos_i) with Beckmann or
 * pillbox D, V-cavity G, microfacet normals drawn from D(h) cos(h) and the
 * estimator weight F G (wo.h) / ((wo.N) (h.N)) of Walter et al. 2007.
 */

/* No bound in the reference: a path between two perfect mirrors at normal
 * incidence keeps its throughput forever. */
constexpr int DRAW_MAX_BOUNCES = 1000;
/* src/ssol_draw_pt.c:334-348 */
constexpr int DRAW_MAX_FAILURES = 100;

/* Pixel of thread `tid` in block `blk` (16 x 16 tiles, 8 x 4 per warp) */
__device__ __forceinline__ void draw_pixel_of(int blk, int tid, int width,
                                              int& px, int& py)
{
  const int ntx = (width + 15) >> 4;
  const int tx = blk % ntx, ty = blk / ntx;
  const int warp = tid >> 5, lane = tid & 31;
  px = (tx << 4) + ((warp & 1) << 3) + (lane & 7);
  py = (ty << 4) + ((warp >> 1) << 2) + (lane >> 3);
}

/* camera_ray (src/ssol_camera.h:41-62) in FP32 with every product and sum
 * rounded on its own, so that the host restatement gets the same rays */
__device__ __forceinline__ void camera_ray(const DrawArgs& A, float sx, float sy,
                                           float d[3])
{
  const float fx = __fsub_rn(__fmul_rn(sx, 2.f), 1.f);
  const float fy = __fsub_rn(__fmul_rn(sy, 2.f), 1.f);
  for(int c = 0; c < 3; ++c)
    d[c] = __fadd_rn(__fadd_rn(__fmul_rn(A.cam_x[c], fx), __fmul_rn(A.cam_y[c], fy)),
                     A.cam_z[c]);
  const float l2 = __fadd_rn(__fadd_rn(__fmul_rn(d[0], d[0]), __fmul_rn(d[1], d[1])),
                             __fmul_rn(d[2], d[2]));
  const float len = __fsqrt_rn(l2);
  for(int c = 0; c < 3; ++c) d[c] = __fdiv_rn(d[c], len);
}

/* Shading normal of a hit (surface_fragment_setup, src/ssol_material.c:
 * 630-654): the interpolated vertex normal turned toward -dir, else N */
template<class R>
__device__ __forceinline__ V3<R> draw_shading_normal
  (const DScene<R>& S, int gid, V3<R> pos, V3<R> dir, V3<R> N, R& b1, R& b2)
{
  b1 = b2 = R(0);
  if(!S.tshade || gid < 0) return N;
  const float2 uv = tri_uv(S, gid, pos);
  b1 = (R)uv.x;
  b2 = (R)uv.y;
  const DTriShade<R>& ts = S.tshade[gid];
  if(isnan(ts.n[0])) return N;
  const V3<R> ns = ld3(ts.n) * (R(1) - b1 - b2) + ld3(ts.n + 3) * b1
                 + ld3(ts.n + 6) * b2;
  const R l2 = dot(ns, ns);
  if(!(l2 > R(0))) return N;
  V3<R> out = ns * rsq(l2);
  if(dot(dir, out) > R(0)) out = -out;
  return out;
}

/* Sum of the per-thread counters of the warp into the launch counters */
__device__ __forceinline__ void draw_flush(unsigned long long* ctr, const uint32_t v[6])
{
  for(int k = 0; k < 6; ++k) {
    const unsigned s = __reduce_add_sync(0xffffffffu, v[k]);
    if((threadIdx.x & 31) == 0 && s) atomicAdd(ctr + k, (unsigned long long)s);
  }
}

/* ssol_draw_draft: Li and draw_pixel of src/ssol_draw_draft.c:37-142 */
template<class R>
__global__ void __launch_bounds__(256) draft_kernel(const DScene<R> S, const DrawArgs A)
{
  extern __shared__ int draw_stack[];
  int px, py;
  draw_pixel_of(blockIdx.x, threadIdx.x, A.width, px, py);
  const bool valid = px < A.width && py < A.height;
  Counters cnt = {0, 0, 0, 0};
  if(valid) {
    const SelfInfo self = {-1, -1, 0, true, false};
    double sum = 0;
    for(int i = 0; i < A.spp; ++i) {
      const float sx = __fmul_rn(__fadd_rn((float)px, A.offsets[2 * i]), A.pix_w);
      const float sy = __fmul_rn(__fadd_rn((float)py, A.offsets[2 * i + 1]), A.pix_h);
      float df[3];
      camera_ray(A, sx, sy, df);
      const V3<R> o = mk((R)A.cam_pos[0], (R)A.cam_pos[1], (R)A.cam_pos[2]);
      const V3<R> d = mk((R)df[0], (R)df[1], (R)df[2]);
      Hit<R> h;
      if(!trace_ray(S, o, d, R(0), self, false, h, cnt, draw_stack + threadIdx.x,
                    (int)blockDim.x))
        continue;
      const V3<R> wi = normalize(d);
      V3<R> N = normalize(h.n);
      if(!(dot(N, wi) < R(0))) N = -N;
      R b1, b2;
      N = draw_shading_normal(S, h.gid, o + d * h.t, wi, N, b1, b2);
      const double c = (double)dot(N, -wi);
      sum += c > 0.0 ? c : 0.0;
    }
    const double v = sum / (double)A.spp;
    double* out = A.pixels + ((size_t)py * (size_t)A.width + (size_t)px) * 3;
    out[0] = v; out[1] = v; out[2] = v;
  }
  const uint32_t c6[6] = {cnt.rays, cnt.nodes, cnt.tris, cnt.quads, 0u,
                          valid ? (uint32_t)A.spp : 0u};
  draw_flush(A.counters, c6);
}

/* Rendering BSDF of material m at a point: shader values (baked per vertex
 * where they vary over the mesh) */
template<class R>
struct DrawBsdf {
  DMaterial m;
  R refl, rough;
};

template<class R>
__device__ __forceinline__ DrawBsdf<R> draw_bsdf
  (const DScene<R>& S, int mtl, int bake, double wl, R b1, R b2)
{
  DrawBsdf<R> f;
  f.m = S.mtls[mtl];
  f.refl = R(0);
  f.rough = R(0);
  if(f.m.type == MTL_MIRROR || f.m.type == MTL_MATTE) {
    f.refl = bake >= 0 ? baked_value(S, bake, 0, wl, b1, b2) : shader_value(S, f.m, 0, wl);
    if(f.m.type == MTL_MIRROR)
      f.rough = bake >= 0 ? baked_value(S, bake, 1, wl, b1, b2) : shader_value(S, f.m, 1, wl);
  }
  return f;
}

/* Microfacet distribution D(h) for cos(h, N) = nh */
template<class R>
__device__ __forceinline__ R microfacet_d(int distrib, R a, R nh)
{
  if(!(nh > R(0))) return R(0);
  const R c2 = nh * nh;
  const R tan2 = (R(1) - c2) / c2;
  const R a2 = a * a;
  const R inv = R(1) / (R(3.14159265358979323846) * a2 * c2 * c2);
  if(distrib == DISTRIB_BECKMANN) return ex(-tan2 / a2) * inv;
  return tan2 <= a2 ? inv : R(0);
}

/* V-cavity masking-shadowing of Cook and Torrance */
template<class R>
__device__ __forceinline__ R microfacet_g(R nh, R no, R ni, R oh)
{
  if(!(oh > R(0))) return R(0);
  const R g = fmin(R(2) * nh * no / oh, R(2) * nh * ni / oh);
  return fmin(R(1), g);
}

/* ssf_bsdf_eval: BRDF value for wo, wi (both pointing away), 0 for the
 * specular components */
template<class R>
__device__ __forceinline__ R draw_bsdf_eval(const DrawBsdf<R>& f, V3<R> wo, V3<R> N, V3<R> wi)
{
  const R no = dot(wo, N), ni = dot(wi, N);
  if(!(no > R(0)) || !(ni > R(0))) return R(0);
  if(f.m.type == MTL_MATTE) return f.refl * R(0.31830988618379067154);
  if(f.m.type == MTL_MIRROR && f.rough > R(0)) {
    const V3<R> h = normalize(wo + wi);
    const R nh = dot(N, h), oh = dot(wo, h);
    const R D = microfacet_d(f.m.distrib, f.rough, nh);
    const R G = microfacet_g(nh, no, ni, oh);
    return f.refl * D * G / (R(4) * no * ni);
  }
  return R(0);
}

/* ssf_bsdf_sample: direction wi and weight R (src/ssol_draw_pt.c:257-264);
 * next_medium follows material_get_next_medium on a transmission */
template<class R>
__device__ __forceinline__ R draw_bsdf_sample
  (const DScene<R>& S, const DrawBsdf<R>& f, const U32x4& r, int medium, double wl,
   V3<R> wo, V3<R> N, V3<R>& wi, int& type, int& next_medium)
{
  const DMaterial& m = f.m;
  type = 0;
  next_medium = medium;
  const R ci = dot(wo, N);
  wi = N;
  if(!(ci > R(0))) return R(0);
  switch(m.type) {
    case MTL_MIRROR: {
      type = BXDF_REFLECTION;
      if(f.rough == R(0)) {
        wi = N * (R(2) * ci) - wo;
        return f.refl;
      }
      const R a = f.rough;
      const R u0 = uni<R>(r.v[0]);
      const R tan2 = m.distrib == DISTRIB_BECKMANN ? -a * a * lg(R(1) - u0) : a * a * u0;
      const R ct = rsq(R(1) + tan2);
      const R st = sq_rt(tan2) * ct;
      R sp, cp; sincos2pi(uni<R>(r.v[1]), &sp, &cp);
      const V3<R> h = local_to(N, cp * st, sp * st, ct);
      const R oh = dot(wo, h);
      wi = h * (R(2) * oh) - wo;
      const R ni = dot(wi, N);
      if(!(oh > R(0)) || !(ni > R(0))) return R(0);
      const R G = microfacet_g(ct, ci, ni, oh);
      return f.refl * G * oh / (ci * ct);
    }
    case MTL_MATTE: {
      const R u0 = uni<R>(r.v[0]);
      const R rad = sq_rt(u0);
      R sp, cp; sincos2pi(uni<R>(r.v[1]), &sp, &cp);
      wi = local_to(N, rad * cp, rad * sp, sq_rt(R(1) - u0));
      type = BXDF_REFLECTION;
      return f.refl;
    }
    case MTL_DIELECTRIC: {
      const R eta_i = (R)data_value(S, S.media[m.out_medium].refractive_index, wl);
      const R eta_t = (R)data_value(S, S.media[m.in_medium].refractive_index, wl);
      const R eta = eta_i / eta_t;
      const R sin2_t = eta * eta * (R(1) - ci * ci);
      R F = R(1), cos_t = R(0);
      if(sin2_t < R(1)) {
        cos_t = sq_rt(R(1) - sin2_t);
        F = fresnel(ci, cos_t, eta_i, eta_t);
      }
      if(uni<R>(r.v[0]) < F) {
        wi = N * (R(2) * ci) - wo;
        type = BXDF_REFLECTION;
      } else {
        wi = normalize(N * (eta * ci - cos_t) - wo * eta);
        type = BXDF_TRANSMISSION;
        next_medium = m.in_medium;
      }
      return R(1);
    }
    case MTL_THIN_DIELECTRIC: {
      const R eta_i = (R)data_value(S, S.media[m.out_medium].refractive_index, wl);
      const R eta_t = (R)data_value(S, S.media[m.slab_medium].refractive_index, wl);
      const R alpha = (R)data_value(S, S.media[m.slab_medium].extinction, wl);
      const R eta = eta_i / eta_t;
      const R sin2_t = eta * eta * (R(1) - ci * ci);
      R Rt = R(1), Tt = R(0);
      if(sin2_t < R(1)) {
        const R cos_t = sq_rt(R(1) - sin2_t);
        const R F = fresnel(ci, cos_t, eta_i, eta_t);
        const R tau = ex(-alpha * (R)m.thickness / cos_t);
        const R den = R(1) - F * F * tau * tau;
        Rt = F + (R(1) - F) * (R(1) - F) * F * tau * tau / den;
        Tt = (R(1) - F) * (R(1) - F) * tau / den;
      }
      const R p = Rt + Tt;
      if(p > R(0) && uni<R>(r.v[0]) * p < Rt) {
        wi = N * (R(2) * ci) - wo;
        type = BXDF_REFLECTION;
      } else {
        wi = -wo;
        type = BXDF_TRANSMISSION;
      }
      return p;
    }
    default: return R(0);
  }
}

/* Li of src/ssol_draw_pt.c:124-290 for one attempt. Returns false on an
 * inconsistent medium (RES_BAD_OP), which the caller retries. */
template<class R>
__device__ __noinline__ bool draw_radiance
  (const DScene<R>& S, const DrawArgs& A, const Rng& rng, uint32_t attempt,
   V3<R> org, V3<R> dir, double& L, Counters& cnt, uint32_t& bounces,
   int* stack, int stride)
{
  L = 0;
  double thr = 1;
  bool roulette = false;
  const double wl = sample_wavelength(S, u01d(rng.get(attempt, RNG_DRAW_WL).v[0]));
  int medium = S.air_medium;
  SelfInfo self = {-1, -1, 0, true, false};
  const V3<R> up = mk((R)A.up[0], (R)A.up[1], (R)A.up[2]);
  const V3<R> to_sun = -ld3(S.sun_dir);
  for(int b = 0; b < DRAW_MAX_BOUNCES; ++b) {
    Hit<R> h;
    if(!trace_ray(S, org, dir, R(0), self, false, h, cnt, stack, stride)) {
      if(dot(dir, up) > R(0)) L += thr * 1e-1;
      break;
    }
    const double kext = data_value(S, S.media[medium].extinction, wl);
    if(kext > 0) {
      thr *= exp(-kext * (double)h.t);
      if(thr <= 0) break;
    }
    const V3<R> wo_in = normalize(dir);
    V3<R> Ng = normalize(h.n);
    int side = 1;
    if(!(dot(Ng, wo_in) < R(0))) { side = 2; Ng = -Ng; }
    const V3<R> pos = org + dir * h.t;
    R b1, b2;
    const V3<R> N = draw_shading_normal(S, h.gid, pos, wo_in, Ng, b1, b2);
    if(dot(N, wo_in) > R(0)) break;
    const DShadedInst& si = S.sinsts[h.sinst];
    const int bake = S.tshade && h.gid >= 0 ? S.tshade[h.gid].bake[side - 1] : -1;
    const DrawBsdf<R> f = draw_bsdf(S, si.mtl[side - 1], bake, wl, b1, b2);
    /* src/ssol_material.c:97-101 */
    if(f.m.type == MTL_DIELECTRIC && medium != f.m.out_medium) return false;
    ++bounces;
    self.gid = h.gid;
    self.sinst = h.sinst;
    self.side = side;
    org = pos;
    const V3<R> wo = -wo_in;
    /* sun_lighting (src/ssol_draw_pt.c:92-121) */
    {
      const R c = dot(to_sun, N);
      if(c >= R(0) && !(fabs(c) <= R(1e-6))) {
        const R fv = draw_bsdf_eval(f, wo, N, to_sun);
        if(fv > R(0)) {
          Hit<R> hs;
          if(!trace_ray(S, org, to_sun, R(0), self, true, hs, cnt, stack, stride))
            L += thr * (double)(fv * c);
        }
      }
    }
    const uint32_t ev = (attempt << 20) | (uint32_t)b;
    V3<R> wi;
    int type, next_medium;
    R w = draw_bsdf_sample(S, f, rng.get(ev, RNG_DRAW_BSDF), medium, wl, wo, N, wi,
                           type, next_medium);
    /* Wrong hemisphere for the sampled component, against Ng */
    const R cg = dot(Ng, wi);
    if((cg > R(0) && (type & BXDF_TRANSMISSION)) || (cg < R(0) && (type & BXDF_REFLECTION)))
      w = R(0);
    dir = wi;
    if(type & BXDF_TRANSMISSION) medium = next_medium;
    const double cn = fabs((double)dot(wi, N));
    if(!roulette) {
      thr *= cn * (double)w;
    } else {
      if(u01d(rng.get(ev, RNG_DRAW_RR).v[0]) >= (double)w) break;
      thr *= cn;
    }
    if(thr <= 0) break;
    if(!roulette) roulette = thr < 0.1;
  }
  return true;
}

/* ssol_draw_pt: draw_pixel of src/ssol_draw_pt.c:292-350 */
template<class R>
__global__ void __launch_bounds__(256) pt_kernel(const DScene<R> S, const DrawArgs A)
{
  extern __shared__ int draw_stack[];
  int px, py;
  draw_pixel_of(blockIdx.x, threadIdx.x, A.width, px, py);
  const bool valid = px < A.width && py < A.height;
  Counters cnt = {0, 0, 0, 0};
  uint32_t bounces = 0;
  if(valid) {
    Rng rng;
    rng.k0 = (uint32_t)A.seed;
    rng.k1 = (uint32_t)(A.seed >> 32);
    const uint64_t pix = (uint64_t)py * (uint64_t)A.width + (uint64_t)px;
    double sum = 0;
    bool failed = false;
    for(int s = 0; s < A.spp && !failed; ++s) {
      const uint64_t id = pix * (uint64_t)A.spp + (uint64_t)s;
      rng.i_lo = (uint32_t)id;
      rng.i_hi = (uint32_t)(id >> 32);
      const U32x4 j = rng.get(0u, RNG_DRAW_PIXEL);
      const float sx = __fmul_rn(__fadd_rn((float)px, u01f(j.v[0])), A.pix_w);
      const float sy = __fmul_rn(__fadd_rn((float)py, u01f(j.v[1])), A.pix_h);
      float df[3];
      camera_ray(A, sx, sy, df);
      const V3<R> o = mk((R)A.cam_pos[0], (R)A.cam_pos[1], (R)A.cam_pos[2]);
      const V3<R> d = mk((R)df[0], (R)df[1], (R)df[2]);
      double L = 0;
      bool ok = false;
      for(uint32_t a = 0; a < (uint32_t)DRAW_MAX_FAILURES && !ok; ++a)
        ok = draw_radiance(S, A, rng, a, o, d, L, cnt, bounces,
                           draw_stack + threadIdx.x, (int)blockDim.x);
      if(!ok) failed = true;
      else sum += L;
    }
    double* out = A.pixels + (pix * 3);
    if(failed) {
      out[0] = 1; out[1] = 1; out[2] = 0;
    } else {
      const double v = sum / (double)A.spp;
      out[0] = v; out[1] = v; out[2] = v;
    }
  }
  const uint32_t c6[6] = {cnt.rays, cnt.nodes, cnt.tris, cnt.quads, bounces,
                          valid ? (uint32_t)A.spp : 0u};
  draw_flush(A.counters, c6);
}

template<class R>
static int launch_draw(const DScene<R>& S, const DrawArgs& A, bool pt, void* stream)
{
  if(A.width <= 0 || A.height <= 0 || A.spp <= 0) return (int)cudaErrorInvalidValue;
  const long long ntx = (A.width + 15) / 16, nty = (A.height + 15) / 16;
  if(ntx * nty > 0x7fffffffLL) return (int)cudaErrorInvalidValue;
  const dim3 grid((unsigned)(ntx * nty));
  const size_t smem = (size_t)SMEM_STACK * 256 * sizeof(int);
  if(pt) pt_kernel<R><<<grid, 256, smem, (cudaStream_t)stream>>>(S, A);
  else draft_kernel<R><<<grid, 256, smem, (cudaStream_t)stream>>>(S, A);
  return (int)cudaGetLastError();
}

int launch_draft_f32(const DScene<float>& S, const DrawArgs& A, void* stream)
{ return launch_draw<float>(S, A, false, stream); }
int launch_draft_f64(const DScene<double>& S, const DrawArgs& A, void* stream)
{ return launch_draw<double>(S, A, false, stream); }
int launch_pt_f32(const DScene<float>& S, const DrawArgs& A, void* stream)
{ return launch_draw<float>(S, A, true, stream); }
int launch_pt_f64(const DScene<double>& S, const DrawArgs& A, void* stream)
{ return launch_draw<double>(S, A, true, stream); }
