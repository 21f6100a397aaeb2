/*
 * estimator.cpp - ssol_estimator_* read-out: E = sum(w) / N,
 * V = max(sum(w^2) / N - E^2, 0), SE = sqrt(V / N)
 * (src/ssol_estimator.c:112-322, src/ssol_mc_receiver.c:32-173).
 */
#include "objects.h"

#include <cmath>
#include <cstring>

static ssol_mc_result mc_result(const double w[2], double n)
{
  ssol_mc_result r;
  if(n <= 0) { r.E = r.V = r.SE = 0; return r; }
  r.E = w[0] / n;
  r.V = w[1] / n - r.E * r.E;
  r.V = r.V > 0 ? r.V : 0;
  r.SE = std::sqrt(r.V / n);
  return r;
}

/* Field order of struct ssol_mc_receiver / ssol_mc_primitive equals the
 * tally order (incoming x5, absorbed x5) */
static void fill_rcv(ssol_mc_result* out, const double q[10][2], double n)
{
  for(int i = 0; i < 10; ++i) out[i] = mc_result(q[i], n);
}

extern "C" res_T ssol_estimator_ref_get(ssol_estimator* e)
{
  if(!e) return RES_BAD_ARG;
  e->ref.get();
  return RES_OK;
}

extern "C" res_T ssol_estimator_ref_put(ssol_estimator* e)
{
  if(!e) return RES_BAD_ARG;
  if(e->ref.put()) {
    ssol_device* dev = e->dev;
    if(e->rng) ssp_rng_ref_put(e->rng);
    delete e;
    if(dev) ssol_device_ref_put(dev);
  }
  return RES_OK;
}

extern "C" res_T ssol_estimator_get_mc_global
  (ssol_estimator* e, ssol_mc_global* g)
{
  if(!e || !g) return RES_BAD_ARG;
  const double n = (double)e->realisation_count;
  g->cos_factor = mc_result(e->global[0], n);
  g->absorbed_by_receivers = mc_result(e->global[1], n);
  g->shadowed = mc_result(e->global[2], n);
  g->missing = mc_result(e->global[3], n);
  g->extinguished_by_atmosphere = mc_result(e->global[4], n);
  g->other_absorbed = mc_result(e->global[5], n);
  return RES_OK;
}

extern "C" res_T ssol_estimator_get_mc_receiver
  (ssol_estimator* e, const ssol_instance* inst, const enum ssol_side_flag side,
   ssol_mc_receiver* rcv)
{
  if(!e || !inst || !rcv || !(inst->receiver_mask & (int)side))
    return RES_BAD_ARG;
  std::memset(rcv, 0, sizeof(*rcv));
  auto it = e->receivers.find(inst);
  if(it == e->receivers.end()) return RES_OK;
  const RcvSums& s = it->second.side[side == SSOL_FRONT ? 0 : 1];
  fill_rcv(&rcv->incoming_flux, s.q, (double)e->realisation_count);
  rcv->mc__ = (void*)&s;
  rcv->N__ = e->realisation_count;
  rcv->instance__ = inst;
  return RES_OK;
}

extern "C" res_T ssol_estimator_get_mc_sampled_x_receiver
  (ssol_estimator* e, const ssol_instance* samp, const ssol_instance* recv,
   const enum ssol_side_flag side, ssol_mc_receiver* rcv)
{
  if(!e || !samp || !recv || !rcv
  || (side != SSOL_BACK && side != SSOL_FRONT)
  || !samp->sample || !(recv->receiver_mask & (int)side))
    return RES_BAD_ARG;
  std::memset(rcv, 0, sizeof(*rcv));
  auto it = e->sampled.find(samp);
  if(it == e->sampled.end()) return RES_BAD_ARG;
  auto jt = it->second.by_receiver.find(recv);
  if(jt == it->second.by_receiver.end()) return RES_OK;
  const RcvSums& s = jt->second.side[side == SSOL_FRONT ? 0 : 1];
  fill_rcv(&rcv->incoming_flux, s.q, (double)e->realisation_count);
  rcv->mc__ = (void*)&s;
  rcv->N__ = it->second.nb_samples;
  return RES_OK;
}

extern "C" res_T ssol_estimator_get_realisation_count
  (const ssol_estimator* e, size_t* count)
{
  if(!e || !count) return RES_BAD_ARG;
  *count = e->realisation_count;
  return RES_OK;
}

extern "C" res_T ssol_estimator_get_failed_count
  (const ssol_estimator* e, size_t* count)
{
  if(!e || !count) return RES_BAD_ARG;
  *count = e->failed_count;
  return RES_OK;
}

extern "C" res_T ssol_estimator_get_sampled_area
  (const ssol_estimator* e, double* area)
{
  if(!e || !area) return RES_BAD_ARG;
  *area = e->sampled_area;
  return RES_OK;
}

extern "C" res_T ssol_estimator_get_sampled_count
  (const ssol_estimator* e, size_t* count)
{
  if(!e || !count) return RES_BAD_ARG;
  *count = e->sampled.size();
  return RES_OK;
}

extern "C" res_T ssol_estimator_get_mc_sampled
  (ssol_estimator* e, const ssol_instance* samp, ssol_mc_sampled* out)
{
  if(!e || !samp || !out) return RES_BAD_ARG;
  auto it = e->sampled.find(samp);
  if(it == e->sampled.end()) return RES_BAD_ARG;
  out->nb_samples = it->second.nb_samples;
  out->cos_factor = mc_result(it->second.cos, (double)out->nb_samples);
  out->shadowed = mc_result(it->second.shadow, (double)e->realisation_count);
  return RES_OK;
}

extern "C" res_T ssol_estimator_get_rng_state
  (const ssol_estimator* e, const ssp_rng** rng)
{
  if(!e || !rng) return RES_BAD_ARG;
  *rng = e->rng;
  return RES_OK;
}

extern "C" res_T ssol_estimator_get_tracked_paths_count
  (const ssol_estimator* e, size_t* n)
{
  if(!e || !n) return RES_BAD_ARG;
  *n = e->paths.size();
  return RES_OK;
}

extern "C" res_T ssol_estimator_get_tracked_path
  (const ssol_estimator* e, const size_t i, ssol_path* path)
{
  if(!e || i >= e->paths.size() || !path) return RES_BAD_ARG;
  path->path__ = &e->paths[i];
  return RES_OK;
}

extern "C" res_T ssol_path_get_vertices_count
  (const ssol_path* path, size_t* n)
{
  if(!path || !n) return RES_BAD_ARG;
  *n = static_cast<const TrackedPath*>(path->path__)->vertices.size();
  return RES_OK;
}

extern "C" res_T ssol_path_get_vertex
  (const ssol_path* path, const size_t i, ssol_path_vertex* v)
{
  if(!path || !v) return RES_BAD_ARG;
  const TrackedPath* p = static_cast<const TrackedPath*>(path->path__);
  if(i >= p->vertices.size()) return RES_BAD_ARG;
  *v = p->vertices[i];
  return RES_OK;
}

extern "C" res_T ssol_path_get_type
  (const ssol_path* path, enum ssol_path_type* type)
{
  if(!path || !type) return RES_BAD_ARG;
  *type = static_cast<const TrackedPath*>(path->path__)->type;
  return RES_OK;
}

extern "C" res_T ssol_mc_receiver_get_mc_shape
  (ssol_mc_receiver* rcv, const ssol_shape* shape, ssol_mc_shape* mc)
{
  if(!rcv || !shape || !mc) return RES_BAD_ARG;
  if(!rcv->instance__
  || !ssolb_object_has_shape(rcv->instance__->object, shape))
    return RES_BAD_ARG;
  const RcvSums* s = static_cast<const RcvSums*>(rcv->mc__);
  mc->N__ = rcv->N__;
  mc->mc__ = nullptr;
  if(s) {
    auto it = s->prims.find(shape);
    if(it != s->prims.end()) mc->mc__ = (void*)&it->second;
  }
  mc->shape__ = shape;
  return RES_OK;
}

/* Per-primitive values are divided by the RT triangle area
 * (src/ssol_mc_receiver.c:121-166) */
extern "C" res_T ssol_mc_shape_get_mc_primitive
  (ssol_mc_shape* shape, const unsigned i, ssol_mc_primitive* prim)
{
  if(!shape || !prim || !shape->shape__) return RES_BAD_ARG;
  const ssol_shape* s = shape->shape__;
  const size_t ntris = s->ids.size() / 3;
  if(i >= ntris) return RES_BAD_ARG;
  std::memset(prim, 0, sizeof(*prim));
  const std::vector<double>* v =
    static_cast<const std::vector<double>*>(shape->mc__);
  if(!v) return RES_OK;
  double p[3][3];
  for(int k = 0; k < 3; ++k)
    for(int c = 0; c < 3; ++c) p[k][c] = s->pos[(size_t)s->ids[i * 3 + k] * 3 + c];
  const double e0[3] = {p[1][0]-p[0][0], p[1][1]-p[0][1], p[1][2]-p[0][2]};
  const double e1[3] = {p[2][0]-p[0][0], p[2][1]-p[0][1], p[2][2]-p[0][2]};
  const double n[3] = {e0[1]*e1[2] - e0[2]*e1[1], e0[2]*e1[0] - e0[0]*e1[2],
                       e0[0]*e1[1] - e0[1]*e1[0]};
  const double area = 0.5 * std::sqrt(n[0]*n[0] + n[1]*n[1] + n[2]*n[2]);
  const double* q = v->data() + (size_t)i * 20;
  bool any = false;
  for(int k = 0; k < 20; ++k) any = any || q[k] != 0;
  if(!any) return RES_OK;
  ssol_mc_result* r = &prim->incoming_flux;
  for(int k = 0; k < 10; ++k) {
    r[k] = mc_result(q + 2 * k, (double)shape->N__);
    r[k].E /= area;
    r[k].V /= area * area;
    r[k].SE /= area;
  }
  return RES_OK;
}
