/*
 * adjoint.cuh - ssol_solve_adjoint: gradients of a receiver flux objective
 * with respect to the aim angles of heliostats (no counterpart in the
 * reference). Included by kernels_aux.cu inside namespace ssolb, where the
 * sampling, tracing and shading helpers live.
 *
 * Objective. Only first-bounce paths count: a realisation sampled on a
 * mirror (src/ssol_solver.c:207-352 for the primary sample), not shadowed,
 * reflected once (src/ssol_material.c:186-218) and reaching the front of the
 * receiver instance first. Its weight there, after the atmosphere and the
 * receiver's absorptivity (1 - reflectivity of its mirror or matte
 * material), is w. The objectives are
 *   J_abs   = (1/N) sum w                     (absorbed power, W)
 *   J_spill = sum_c (M_c - T)^2,  M_c = (1/(N A_c)) sum w K_c(u, v)
 * with (u, v) the hit in the receiver's local frame and K_c the bilinear
 * (tent) weight of cell c, so that the map moves smoothly with the spot.
 *
 * Parameters. Each listed heliostat instance turns by theta_x about its own
 * local x axis and theta_y about its local y axis, through its translation.
 * At theta = 0 the sampled point and normal move as d/dtheta_k p = e_k x
 * (p - c), d/dtheta_k N = e_k x N: the sample is reparameterised with the
 * heliostat (its barycentrics, sun direction and microfacet draws are kept),
 * and every quantity downstream is carried as a dual number with the two
 * tangents, from the cosine weight through the microfacet normal (built on
 * the rotated basis of N), the reflected direction, the distance to the
 * receiver plane, the extinction and the hit's cell weights. Changes of the
 * discrete outcome (shadowing, blocking, the receiver's edges) are not
 * differentiated: these edge terms are the bias the finite-difference
 * harness reports.
 *
 * Two passes over the same Philox keys (replay): pass 0 tallies the map and
 * J_abs, pass 1 recomputes every path of a listed heliostat with tangents
 * and accumulates dJ_abs and 2 (M_c - T) dM_c per heliostat.
 */

/* Dual number with two tangents */
struct Dd { double v, a, b; };

__device__ __forceinline__ Dd dd(double v) { Dd r = {v, 0.0, 0.0}; return r; }
__device__ __forceinline__ Dd operator+(Dd x, Dd y)
{ Dd r = {x.v + y.v, x.a + y.a, x.b + y.b}; return r; }
__device__ __forceinline__ Dd operator-(Dd x, Dd y)
{ Dd r = {x.v - y.v, x.a - y.a, x.b - y.b}; return r; }
__device__ __forceinline__ Dd operator-(Dd x) { Dd r = {-x.v, -x.a, -x.b}; return r; }
__device__ __forceinline__ Dd operator*(Dd x, Dd y)
{ Dd r = {x.v * y.v, x.a * y.v + x.v * y.a, x.b * y.v + x.v * y.b}; return r; }
__device__ __forceinline__ Dd operator*(Dd x, double k)
{ Dd r = {x.v * k, x.a * k, x.b * k}; return r; }
__device__ __forceinline__ Dd operator*(double k, Dd x) { return x * k; }
__device__ __forceinline__ Dd operator+(Dd x, double k) { Dd r = {x.v + k, x.a, x.b}; return r; }
__device__ __forceinline__ Dd operator-(Dd x, double k) { Dd r = {x.v - k, x.a, x.b}; return r; }
__device__ __forceinline__ Dd operator/(Dd x, Dd y)
{
  const double q = x.v / y.v;
  Dd r = {q, (x.a - q * y.a) / y.v, (x.b - q * y.b) / y.v};
  return r;
}
__device__ __forceinline__ Dd dexp(Dd x)
{ const double e = exp(x.v); Dd r = {e, x.a * e, x.b * e}; return r; }
__device__ __forceinline__ Dd dabs(Dd x) { return x.v < 0.0 ? -x : x; }

struct DV { Dd x, y, z; };

__device__ __forceinline__ DV dv(V3<double> v)
{ DV r = {dd(v.x), dd(v.y), dd(v.z)}; return r; }
__device__ __forceinline__ DV operator+(DV p, DV q)
{ DV r = {p.x + q.x, p.y + q.y, p.z + q.z}; return r; }
__device__ __forceinline__ DV operator-(DV p, V3<double> q)
{ DV r = {p.x - q.x, p.y - q.y, p.z - q.z}; return r; }
__device__ __forceinline__ DV operator*(DV p, Dd k)
{ DV r = {p.x * k, p.y * k, p.z * k}; return r; }
__device__ __forceinline__ DV operator*(DV p, double k)
{ DV r = {p.x * k, p.y * k, p.z * k}; return r; }
__device__ __forceinline__ Dd ddot(DV p, DV q) { return p.x * q.x + p.y * q.y + p.z * q.z; }
__device__ __forceinline__ Dd ddot(DV p, V3<double> q)
{ return p.x * q.x + p.y * q.y + p.z * q.z; }

template<class R> __device__ __forceinline__ V3<double> vd(V3<R> v)
{ return mk((double)v.x, (double)v.y, (double)v.z); }

/* The Duff et al. basis of onb() on a dual normal: the sign is taken from
 * the value, so the tangents follow the same branch as the primal */
__device__ __forceinline__ void donb(const DV& n, DV& b1, DV& b2)
{
  const double sgn = n.z.v >= 0.0 ? 1.0 : -1.0;
  const Dd a = dd(-1.0) / (n.z + sgn);
  const Dd b = n.x * n.y * a;
  b1.x = dd(1.0) + n.x * n.x * a * sgn;
  b1.y = b * sgn;
  b1.z = -(n.x * sgn);
  b2.x = b;
  b2.y = n.y * n.y * a + sgn;
  b2.z = -n.y;
}

/* Tangents of a point or vector turned with a heliostat about the axes e_x,
 * e_y through c (c = 0 for directions) */
__device__ __forceinline__ DV with_tangents(V3<double> v, V3<double> ex, V3<double> ey)
{
  const V3<double> ta = cross(ex, v), tb = cross(ey, v);
  DV r;
  r.x.v = v.x; r.x.a = ta.x; r.x.b = tb.x;
  r.y.v = v.y; r.y.a = ta.y; r.y.b = tb.y;
  r.z.v = v.z; r.z.a = ta.z; r.z.b = tb.z;
  return r;
}

/* Two blocks per SM (128 registers): one block of 256 threads left 8 warps
 * per SM to hide the BVH loads; with two the kernel runs 1.56x faster
 * despite its spills (field, 5e7 paths: 187.5 -> 292.8 Mpaths/s) */
template<class R, int PASS>
__global__ void __launch_bounds__(MAX_BLOCK, 2)
adjoint_kernel(const DScene<R> S, const AdjointArgs A, uint64_t seed, uint64_t first,
               uint64_t count)
{
  __shared__ int stack_sm[SMEM_STACK * MAX_BLOCK];
  int* stack = stack_sm + threadIdx.x;
  const int stride = blockDim.x;
  Counters cnt = {0, 0, 0, 0};
  Rng rng;
  rng.k0 = (uint32_t)seed;
  rng.k1 = (uint32_t)(seed >> 32);
  double s_w = 0.0, s_w2 = 0.0, s_hit = 0.0;
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x;
  for(uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += step) {
    const uint64_t id = first + i;
    rng.i_lo = (uint32_t)id;
    rng.i_hi = (uint32_t)(id >> 32);

    /* Primary sample: the draws and arithmetic of init_path */
    const U32x4 r0 = rng.get(0u, RNG_PRIMARY);
    int k = (int)(((unsigned long long)(r0.v[0] >> 8)
                   * (unsigned long long)S.nsamp) >> 24);
    if(!(uni<float>(r0.v[1]) < S.alias_prob[k])) k = S.alias_idx[k];
    const DSampTri<R> st = S.samp[k];
    const DShadedInst si = S.sinsts[st.sinst];
    const int slot = A.inst_slot[si.instance];
    if(PASS == 1 && slot < 0) continue;
    const R sa = sq_rt(uni<R>(r0.v[2]));
    const R b2 = sa * uni<R>(r0.v[3]);
    const R b1 = sa - b2;
    V3<R> pos = ld3(st.v0) + ld3(st.e1) * b1 + ld3(st.e2) * b2;
    const V3<R> nproxy = ld3(st.n);
    const U32x4 r1 = rng.get(1u, RNG_PRIMARY);
    const V3<R> dir = sample_sun_dir(S, rng, r1);
    const double wl = sample_wavelength(S, u01d(r1.v[2]));
    V3<R> N = nproxy;
    if(si.is_punched) {
      const DQuadric<R>& Q = S.quads[si.quadric];
      V3<R> pl = xform_point(Q.w2l, pos);
      pl.z = quadric_general_z(Q, pl.x, pl.y);
      N = normalize(xform_normal(Q.w2l, quadric_general_normal(Q, pl)));
      pos = xform_point(Q.l2w, pl);
    }
    int side = 1;
    if(dot(N, dir) >= R(0)) { side = 2; N = -N; }
    const DMaterial m = S.mtls[si.mtl[side - 1]];
    if(m.type != MTL_MIRROR) continue;
    /* Shading normal and baked shader values at the sampled point, as in
     * shade() */
    V3<R> Ns = N;
    int bake = -1;
    if(S.tshade && st.gid >= 0) {
      const DTriShade<R>& ts = S.tshade[st.gid];
      bake = ts.bake[side - 1];
      if(!isnan(ts.n[0])) {
        const V3<R> v = ld3(ts.n) * (R(1) - b1 - b2) + ld3(ts.n + 3) * b1
                      + ld3(ts.n + 6) * b2;
        const R l2 = dot(v, v);
        if(l2 > R(0)) {
          Ns = v * rsq(l2);
          if(dot(Ns, -dir) < R(0)) Ns = -Ns;
        }
      }
    }
    if(!(dot(-dir, Ns) > R(0))) continue;

    /* Point and normals with their tangents (zero for other instances) */
    DV x = dv(vd(pos)), n = dv(vd(N)), ns = dv(vd(Ns));
    if(slot >= 0) {
      const double* ax = A.axes + 9 * slot;
      const V3<double> c = mk(ax[0], ax[1], ax[2]);
      const V3<double> ex = mk(ax[3], ax[4], ax[5]);
      const V3<double> ey = mk(ax[6], ax[7], ax[8]);
      x = with_tangents(vd(pos) - c, ex, ey);
      x.x.v += c.x; x.y.v += c.y; x.z.v += c.z;
      n = with_tangents(vd(N), ex, ey);
      ns = with_tangents(vd(Ns), ex, ey);
    }
    const V3<double> sdir = vd(dir);
    const V3<R> sun0 = ld3(S.sun_dir);
    const R proxy_cos = si.is_punched ? fabs(dot(nproxy, N)) : R(1);
    const double den = (double)proxy_cos * (double)dot(sun0, dir);
    Dd w = dabs(ddot(n, sdir) * (1.0 / den)) * (S.dni * S.area_proxy);

    /* Shadow ray toward the sun */
    Hit<R> h;
    SelfInfo self;
    self.gid = st.gid;
    self.sinst = st.sinst;
    self.side = side;
    self.discard_virtual = true;
    self.reversed = true;
    if(trace_ray(S, pos, -dir, R(0), self, true, h, cnt, stack, stride)) continue;

    /* Mirror reflection with the draws of shade() (scatter event 0) */
    const R refl = bake >= 0 ? baked_value(S, bake, 0, wl, b1, b2)
                             : shader_value(S, m, 0, wl);
    const R rough = bake >= 0 ? baked_value(S, bake, 1, wl, b1, b2)
                              : shader_value(S, m, 1, wl);
    const V3<double> wo = -sdir;
    DV out;
    if(rough == R(0)) {
      out = ns * (2.0 * ddot(ns, wo));
      out.x = out.x - wo.x; out.y = out.y - wo.y; out.z = out.z - wo.z;
    } else {
      bool ok = false;
      U32x4 rr = rng.get(0u, RNG_SCATTER);
      for(uint32_t kk = 0; kk < 16 && !ok; ++kk) {
        if(kk) rr = rng.get(kk, RNG_RETRY);
        const R u0 = uni<R>(rr.v[0]);
        const R tan2 = m.distrib == DISTRIB_BECKMANN
          ? -rough * rough * lg(R(1) - u0)
          : rough * rough * u0;
        const R ct = rsq(R(1) + tan2);
        const R stn = sq_rt(tan2) * ct;
        R sp, cp; sincos2pi(uni<R>(rr.v[1]), &sp, &cp);
        DV e1, e2;
        donb(ns, e1, e2);
        const DV hh = e1 * (double)(cp * stn) + e2 * (double)(sp * stn) + ns * (double)ct;
        const Dd wh = ddot(hh, wo);
        if(!(wh.v > 0.0)) continue;
        out = hh * (2.0 * wh);
        out.x = out.x - wo.x; out.y = out.y - wo.y; out.z = out.z - wo.z;
        ok = ddot(out, ns).v > 0.0;
      }
      if(!ok) continue;
    }
    if(ddot(out, n).v < 0.0) continue;
    w = w * (double)refl;

    /* First hit along the reflected ray: the receiver's front, or nothing */
    const V3<R> rd = mk((R)out.x.v, (R)out.y.v, (R)out.z.v);
    self.discard_virtual = false;
    self.reversed = false;
    const bool found = trace_ray(S, pos, rd, R(0), self, false, h, cnt, stack, stride);
    bool on_rcv = false;
    int hside = 1;
    if(found) {
      const DShadedInst hs = S.sinsts[h.sinst];
      hside = dot(rd, h.n) < R(0) ? 1 : 2;
      on_rcv = hs.instance == A.rcv_instance && !hs.is_punched && (hs.receiver_mask & hside);
      if(on_rcv) {
        const DMaterial hm = S.mtls[hs.mtl[hside - 1]];
        on_rcv = hm.type == MTL_MIRROR || hm.type == MTL_MATTE;
      }
    }
    /* Pass 1 also follows rays that cross the receiver's plane just outside
     * it, unblocked: the ramp that smooths the receiver's boundary gives
     * them the derivative of the hits that would enter it */
    Dd tpl = dd(0.0);
    bool edge_only = false;
    if(!on_rcv) {
      if(PASS == 0) continue;
      const Dd zx = x.x * A.w2l[8] + x.y * A.w2l[9] + x.z * A.w2l[10] + A.w2l[11];
      const Dd zo = out.x * A.w2l[8] + out.y * A.w2l[9] + out.z * A.w2l[10];
      /* crossing toward the receiving side: from +z for the front */
      if(A.rcv_side == 1 ? !(zx.v > 0.0 && zo.v < 0.0) : !(zx.v < 0.0 && zo.v > 0.0))
        continue;
      tpl = -zx / zo;
      if(found && (double)h.t < tpl.v) continue; /* blocked before the plane */
      edge_only = true;
    }
    double kabs;
    Dd t;
    if(!edge_only) {
      const DShadedInst hs = S.sinsts[h.sinst];
      const DMaterial hm = S.mtls[hs.mtl[hside - 1]];
      const int hbake = S.tshade ? S.tshade[h.gid].bake[hside - 1] : -1;
      float2 huv = make_float2(0.f, 0.f);
      if(hbake >= 0) huv = tri_uv(S, h.gid, pos + rd * h.t);
      kabs = 1.0 - (double)(hbake >= 0
        ? baked_value(S, hbake, 0, wl, (R)huv.x, (R)huv.y) : shader_value(S, hm, 0, wl));
      /* Distance to the hit triangle's plane, with tangents */
      const DTri<R>& T = S.tris[h.gid];
      const V3<double> ng = vd(h.n);
      t = (dd(dot(ng, vd(ld3(T.v0)))) - ddot(x, ng)) / ddot(out, ng);
    } else {
      kabs = 1.0 - (double)shader_value(S, S.mtls[A.rcv_mtl], 0, wl);
      t = tpl;
    }
    const DV p = x + out * t;
    const double kext = data_value(S, S.media[S.air_medium].extinction, wl);
    if(kext > 0.0) w = w * dexp(t * (-kext));
    w = w * kabs;

    const Dd u = p.x * A.w2l[0] + p.y * A.w2l[1] + p.z * A.w2l[2] + A.w2l[3];
    const Dd v = p.x * A.w2l[4] + p.y * A.w2l[5] + p.z * A.w2l[6] + A.w2l[7];
    if(PASS == 0) {
      s_w += w.v;
      s_w2 += w.v * w.v;
      s_hit += 1.0;
    } else {
      /* Smoothed receiver: a ramp of width `edge` across each side of the
       * map's rectangle, 1 inside, 0 outside; on the hits of the receiver
       * away from its boundary it is 1 with no tangent */
      auto ramp = [&](Dd q, double lo, double hi) -> Dd {
        const Dd d = q.v - lo < hi - q.v ? q - lo : dd(hi) - q;
        const Dd r = d * (1.0 / A.edge) + 0.5;
        return r.v >= 1.0 ? dd(1.0) : r.v <= 0.0 ? dd(0.0) : r;
      };
      const Dd sm = ramp(u, A.lower[0], A.upper[0]) * ramp(v, A.lower[1], A.upper[1]);
      if(edge_only && !(sm.v > 0.0)) continue;
      w = w * sm;
      red_add_global(A.grad_abs + 2 * slot, w.a * A.inv_n);
      red_add_global(A.grad_abs + 2 * slot + 1, w.b * A.inv_n);
    }
    /* Bilinear splat on the cell centres */
    const Dd fx = (u - A.lower[0]) * A.inv_cell[0] - 0.5;
    const Dd fy = (v - A.lower[1]) * A.inv_cell[1] - 0.5;
    const int i0 = (int)floor(fx.v), j0 = (int)floor(fy.v);
    const Dd tx = fx - (double)i0, ty = fy - (double)j0;
    double ga = 0.0, gb = 0.0;
    for(int dj = 0; dj < 2; ++dj) {
      const int cj = j0 + dj;
      if(cj < 0 || cj >= A.ny) continue;
      const Dd ky = dj ? ty : dd(1.0) - ty;
      for(int di = 0; di < 2; ++di) {
        const int ci = i0 + di;
        if(ci < 0 || ci >= A.nx) continue;
        const Dd kx = di ? tx : dd(1.0) - tx;
        const Dd c = w * (kx * ky);
        const int cell = cj * A.nx + ci;
        if(PASS == 0) {
          red_add_global(A.map + cell, c.v);
        } else {
          const double r = 2.0 * (A.map[cell] * A.map_scale - A.target);
          ga += r * c.a;
          gb += r * c.b;
        }
      }
    }
    if(PASS == 1) {
      red_add_global(A.grad_spill + 2 * slot, ga * A.map_scale);
      red_add_global(A.grad_spill + 2 * slot + 1, gb * A.map_scale);
    }
  }
  if(PASS == 0) {
    for(int o = 16; o > 0; o >>= 1) {
      s_w += __shfl_down_sync(0xffffffffu, s_w, o);
      s_w2 += __shfl_down_sync(0xffffffffu, s_w2, o);
      s_hit += __shfl_down_sync(0xffffffffu, s_hit, o);
    }
    if((threadIdx.x & 31u) == 0) {
      red_add_global(A.sums + 0, s_w);
      red_add_global(A.sums + 1, s_w2);
      red_add_global(A.sums + 2, s_hit);
    }
  }
  unsigned long long c4[4] = {cnt.rays, cnt.nodes, cnt.tris, cnt.quads};
  for(int q = 0; q < 4; ++q) c4[q] = warp_sum_u64(c4[q]);
  if((threadIdx.x & 31u) == 0)
    for(int q = 0; q < 4; ++q) if(c4[q]) atomicAdd(A.counters + q, c4[q]);
}

template<class R>
static int launch_adjoint_impl
  (const DScene<R>& S, const AdjointArgs& A, uint64_t seed, uint64_t first,
   uint64_t count, int pass, void* stream)
{
  int dev = 0;
  cudaGetDevice(&dev);
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  int per_sm = 0;
  if(pass == 0)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adjoint_kernel<R, 0>,
                                                  MAX_BLOCK, 0);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adjoint_kernel<R, 1>,
                                                  MAX_BLOCK, 0);
  if(per_sm < 1) per_sm = 1;
  uint64_t blocks = (uint64_t)nsm * (uint64_t)per_sm * 4;
  const uint64_t needed = (count + MAX_BLOCK - 1) / MAX_BLOCK;
  if(blocks > needed) blocks = needed;
  if(blocks < 1) blocks = 1;
  const cudaStream_t s = (cudaStream_t)stream;
  if(pass == 0)
    adjoint_kernel<R, 0><<<(unsigned)blocks, MAX_BLOCK, 0, s>>>(S, A, seed, first, count);
  else
    adjoint_kernel<R, 1><<<(unsigned)blocks, MAX_BLOCK, 0, s>>>(S, A, seed, first, count);
  return (int)cudaGetLastError();
}

int launch_adjoint_f32
  (const DScene<float>& S, const AdjointArgs& A, uint64_t seed, uint64_t first,
   uint64_t count, int pass, void* stream)
{ return launch_adjoint_impl<float>(S, A, seed, first, count, pass, stream); }

int launch_adjoint_f64
  (const DScene<double>& S, const AdjointArgs& A, uint64_t seed, uint64_t first,
   uint64_t count, int pass, void* stream)
{ return launch_adjoint_impl<double>(S, A, seed, first, count, pass, stream); }
