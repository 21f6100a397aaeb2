/*
 * objects.cpp - ssol_* setup API: device, spectrum, data, shapes, materials,
 * objects, instances, sun, atmosphere, scene and parameter buffers.
 *
 * Argument checks and reference-count ownership follow the reference
 * (src/ssol_device.c, src/ssol_spectrum.c, src/ssol_data.c,
 * src/ssol_shape.c:1525-1769, src/ssol_material.c:379-535,
 * src/ssol_object.c, src/ssol_instance.c, src/ssol_sun.c,
 * src/ssol_atmosphere.c, src/ssol_scene.c:46-330,
 * src/ssol_param_buffer.c).
 */
#include "objects.h"
#include "tessellate.h"
#include "../../include/ssol_b200.h"

#include <cmath>
#include <cstdarg>
#include <cfloat>
#include <cstring>
#include <limits>

/*******************************************************************************
 * Shared helpers
 ******************************************************************************/
uint32_t ssolb_next_uid()
{
  static std::atomic<uint32_t> next{1};
  return next.fetch_add(1);
}

void ssol_device::log_error(const char* fmt, ...) const
{
  if(!verbose) return;
  va_list ap;
  va_start(ap, fmt);
  fprintf(stderr, "ssol-b200 error: ");
  vfprintf(stderr, fmt, ap);
  va_end(ap);
}

void ssol_device::log_warning(const char* fmt, ...) const
{
  if(!verbose) return;
  va_list ap;
  va_start(ap, fmt);
  fprintf(stderr, "ssol-b200 warning: ");
  vfprintf(stderr, fmt, ap);
  va_end(ap);
}

/* 64-bit FNV-1a over a byte range (Fowler/Noll/Vo); used as the spectrum
 * checksum that decides medium equality (src/ssol_spectrum.c:199-200,
 * src/ssol_material.c:42-66) */
static uint64_t fnv1a64(const void* data, size_t n)
{
  const unsigned char* p = static_cast<const unsigned char*>(data);
  uint64_t h = 0xcbf29ce484222325ull;
  for(size_t i = 0; i < n; ++i) {
    h ^= p[i];
    h *= 0x100000001b3ull;
  }
  return h;
}

bool ssolb_data_ceq(const ssol_data& a, const ssol_data& b)
{
  if(a.type != b.type) return false;
  if(a.type == SSOL_DATA_REAL) return a.value.real == b.value.real;
  return a.value.spectrum->checksum[0] == b.value.spectrum->checksum[0]
      && a.value.spectrum->checksum[1] == b.value.spectrum->checksum[1];
}

bool ssolb_media_ceq(const ssol_medium& a, const ssol_medium& b)
{
  return ssolb_data_ceq(a.refractive_index, b.refractive_index)
      && ssolb_data_ceq(a.extinction, b.extinction);
}

/* Linear interpolation clamped at both ends (src/ssol_spectrum.c:57-89) */
double ssolb_spectrum_interpolate(const ssol_spectrum* s, double wl)
{
  const std::vector<double>& w = s->wavelengths;
  const std::vector<double>& v = s->intensities;
  const size_t n = w.size();
  size_t lo = 0, hi = n; /* first index with w[i] >= wl */
  while(lo < hi) {
    const size_t mid = (lo + hi) / 2;
    if(w[mid] < wl) lo = mid + 1; else hi = mid;
  }
  if(lo == n) return v[n - 1];
  if(lo == 0) return v[0];
  const double slope = (v[lo] - v[lo - 1]) / (w[lo] - w[lo - 1]);
  return v[lo - 1] + (wl - w[lo - 1]) * slope;
}

void ssolb_d33_invtrans(double out[9], const double m[9]);

bool ssolb_object_has_shape(const ssol_object* obj, const ssol_shape* s)
{
  for(const ShadedShape& ss : obj->shaded) if(ss.shape == s) return true;
  return false;
}

static bool spectrum_check_data
  (const ssol_spectrum* s, double lower, double upper)
{
  if(!s || s->intensities.empty()) return false;
  if(s->intensities.size() != s->wavelengths.size()) return false;
  double current = 0;
  for(size_t i = 0; i < s->intensities.size(); ++i) {
    const double wl = s->wavelengths[i], d = s->intensities[i];
    if(d < lower || d > upper || wl <= 0 || wl <= current) return false;
    current = wl;
  }
  return true;
}

/* check_medium (src/ssol_material.c:300-335) */
static bool check_medium(const ssol_medium* m)
{
  if(!m) return false;
  if(m->extinction.type == SSOL_DATA_REAL) {
    if(m->extinction.value.real < 0) return false;
  } else if(m->extinction.type == SSOL_DATA_SPECTRUM) {
    if(!spectrum_check_data(m->extinction.value.spectrum, 0, DBL_MAX))
      return false;
  } else return false;
  if(m->refractive_index.type == SSOL_DATA_REAL) {
    if(m->refractive_index.value.real <= 0) return false;
  } else if(m->refractive_index.type == SSOL_DATA_SPECTRUM) {
    if(!spectrum_check_data
       (m->refractive_index.value.spectrum, DBL_EPSILON, DBL_MAX))
      return false;
  } else return false;
  return true;
}

/*******************************************************************************
 * Device
 ******************************************************************************/
extern "C" res_T ssol_device_create
  (struct logger* logger, struct mem_allocator* allocator,
   const unsigned nthreads_hint, const int verbose, ssol_device** out)
{
  (void)logger, (void)allocator;
  if(nthreads_hint == 0 || !out) return RES_BAD_ARG;
  ssol_device* dev = new (std::nothrow) ssol_device();
  if(!dev) return RES_MEM_ERR;
  dev->verbose = verbose;
  *out = dev;
  return RES_OK;
}

void ssolb_device_release_gpu(ssol_device* dev); /* solve.cpp */

extern "C" res_T ssol_device_ref_get(ssol_device* dev)
{
  if(!dev) return RES_BAD_ARG;
  dev->ref.get();
  return RES_OK;
}

extern "C" res_T ssol_device_ref_put(ssol_device* dev)
{
  if(!dev) return RES_BAD_ARG;
  if(dev->ref.put()) {
    ssolb_device_release_gpu(dev);
    delete dev;
  }
  return RES_OK;
}

/*******************************************************************************
 * Spectrum and data
 ******************************************************************************/
extern "C" res_T ssol_spectrum_create(ssol_device* dev, ssol_spectrum** out)
{
  if(!dev || !out) return RES_BAD_ARG;
  ssol_spectrum* s = new (std::nothrow) ssol_spectrum();
  if(!s) return RES_MEM_ERR;
  ssol_device_ref_get(dev);
  s->dev = dev;
  *out = s;
  return RES_OK;
}

extern "C" res_T ssol_spectrum_ref_get(ssol_spectrum* s)
{
  if(!s) return RES_BAD_ARG;
  s->ref.get();
  return RES_OK;
}

extern "C" res_T ssol_spectrum_ref_put(ssol_spectrum* s)
{
  if(!s) return RES_BAD_ARG;
  if(s->ref.put()) {
    ssol_device* dev = s->dev;
    delete s;
    ssol_device_ref_put(dev);
  }
  return RES_OK;
}

/* src/ssol_spectrum.c:166-213 */
extern "C" res_T ssol_spectrum_setup
  (ssol_spectrum* s,
   void (*get)(const size_t, double*, double*, void*),
   const size_t n, void* ctx)
{
  if(!s || !n || !get) return RES_BAD_ARG;
  std::vector<double> wl(n), val(n);
  double current = 0;
  for(size_t i = 0; i < n; ++i) {
    get(i, &wl[i], &val[i], ctx);
    if(wl[i] <= current || val[i] < 0) {
      s->wavelengths.clear();
      s->intensities.clear();
      s->checksum[0] = s->checksum[1] = 0;
      return RES_BAD_ARG;
    }
    current = wl[i];
  }
  s->wavelengths = std::move(wl);
  s->intensities = std::move(val);
  s->checksum[0] = fnv1a64(s->wavelengths.data(), n * sizeof(double));
  s->checksum[1] = fnv1a64(s->intensities.data(), n * sizeof(double));
  return RES_OK;
}

extern "C" ssol_data* ssol_data_clear(ssol_data* data)
{
  if(data->type != SSOL_DATA_SPECTRUM) return data;
  ssol_spectrum_ref_put(data->value.spectrum);
  *data = SSOL_DATA_NULL;
  return data;
}

extern "C" ssol_data* ssol_data_set_real(ssol_data* data, const double real)
{
  ssol_data_clear(data);
  data->type = SSOL_DATA_REAL;
  data->value.real = real;
  return data;
}

extern "C" ssol_data* ssol_data_set_spectrum(ssol_data* data, ssol_spectrum* s)
{
  if(data->type == SSOL_DATA_SPECTRUM && data->value.spectrum == s)
    return data;
  ssol_data_clear(data);
  data->type = SSOL_DATA_SPECTRUM;
  data->value.spectrum = s;
  ssol_spectrum_ref_get(s);
  return data;
}

extern "C" ssol_data* ssol_data_copy(ssol_data* dst, const ssol_data* src)
{
  if(dst == src) return dst;
  if(src->type == SSOL_DATA_SPECTRUM) {
    ssol_data_set_spectrum(dst, src->value.spectrum);
  } else {
    ssol_data_set_real(dst, src->value.real);
  }
  return dst;
}

extern "C" double ssol_data_get_value(const ssol_data* data, const double wl)
{
  if(data->type == SSOL_DATA_REAL) return data->value.real;
  return ssolb_spectrum_interpolate(data->value.spectrum, wl);
}

/*******************************************************************************
 * Shapes
 ******************************************************************************/
static res_T shape_create(ssol_device* dev, ssol_shape** out, ShapeKind k)
{
  if(!dev || !out) return RES_BAD_ARG;
  ssol_shape* s = new (std::nothrow) ssol_shape();
  if(!s) return RES_MEM_ERR;
  ssol_device_ref_get(dev);
  s->dev = dev;
  s->kind = k;
  s->uid = ssolb_next_uid();
  *out = s;
  return RES_OK;
}

extern "C" res_T ssol_shape_create_mesh(ssol_device* dev, ssol_shape** out)
{ return shape_create(dev, out, SHAPE_MESH); }

extern "C" res_T ssol_shape_create_punched_surface
  (ssol_device* dev, ssol_shape** out)
{ return shape_create(dev, out, SHAPE_PUNCHED); }

extern "C" res_T ssol_shape_ref_get(ssol_shape* s)
{
  if(!s) return RES_BAD_ARG;
  s->ref.get();
  return RES_OK;
}

extern "C" res_T ssol_shape_ref_put(ssol_shape* s)
{
  if(!s) return RES_BAD_ARG;
  if(s->ref.put()) {
    ssol_device* dev = s->dev;
    delete s;
    ssol_device_ref_put(dev);
  }
  return RES_OK;
}

extern "C" res_T ssol_shape_get_vertices_count
  (const ssol_shape* s, unsigned* n)
{
  if(!s || !n) return RES_BAD_ARG;
  *n = (unsigned)(s->pos.size() / 3);
  return RES_OK;
}

extern "C" res_T ssol_shape_get_triangles_count
  (const ssol_shape* s, unsigned* n)
{
  if(!s || !n) return RES_BAD_ARG;
  *n = (unsigned)(s->ids.size() / 3);
  return RES_OK;
}

extern "C" res_T ssol_shape_get_triangle_indices
  (const ssol_shape* s, const unsigned itri, unsigned ids[3])
{
  if(!s || !ids || itri >= s->ids.size() / 3)
    return RES_BAD_ARG;
  for(int i = 0; i < 3; ++i) ids[i] = s->ids[(size_t)itri * 3 + i];
  return RES_OK;
}

/* Raw attribute fetch: missing components default to 1
 * (src/ssol_shape.c:1496-1522); positions of punched surfaces are already in
 * object space in `pos` */
extern "C" res_T ssol_shape_get_vertex_attrib
  (const ssol_shape* s, const unsigned iv,
   const enum ssol_attrib_usage usage, double value[])
{
  if(!s || (unsigned)usage >= SSOL_ATTRIBS_COUNT__ || !value)
    return RES_BAD_ARG;
  const size_t nverts = s->pos.size() / 3;
  if(iv >= nverts) return RES_BAD_ARG;
  value[0] = value[1] = value[2] = 1;
  switch(usage) {
    case SSOL_POSITION:
      for(int i = 0; i < 3; ++i) value[i] = s->pos[(size_t)iv * 3 + i];
      break;
    case SSOL_NORMAL:
      if(s->nrm.empty()) return RES_BAD_ARG;
      for(int i = 0; i < 3; ++i) value[i] = s->nrm[(size_t)iv * 3 + i];
      break;
    case SSOL_TEXCOORD:
      if(s->uv.empty()) return RES_BAD_ARG;
      for(int i = 0; i < 2; ++i) value[i] = s->uv[(size_t)iv * 2 + i];
      break;
    default: return RES_BAD_ARG;
  }
  /* Like the reference (src/ssol_shape.c:1584-1593), punched positions and
   * normals get the quadric transform applied on top of the stored vertex,
   * which is already in object space; the two agree for identity quadric
   * transforms */
  if(s->kind == SHAPE_PUNCHED && usage != SSOL_TEXCOORD) {
    const double* T = s->quadric.transform;
    double tmp[3];
    if(usage == SSOL_POSITION) {
      for(int c = 0; c < 3; ++c)
        tmp[c] = T[c] * value[0] + T[3 + c] * value[1] + T[6 + c] * value[2]
               + T[9 + c];
    } else {
      double R[9];
      ssolb_d33_invtrans(R, T);
      for(int c = 0; c < 3; ++c)
        tmp[c] = R[c] * value[0] + R[3 + c] * value[1] + R[6 + c] * value[2];
    }
    for(int c = 0; c < 3; ++c) value[c] = tmp[c];
  }
  return RES_OK;
}

/* Sum of triangle areas from float positions (src/ssol_shape.c:654-689) */
static double mesh_area(const std::vector<float>& pos,
                        const std::vector<uint32_t>& ids)
{
  double area = 0;
  for(size_t t = 0; t + 2 < ids.size(); t += 3) {
    double v[3][3];
    for(int k = 0; k < 3; ++k)
      for(int c = 0; c < 3; ++c) v[k][c] = pos[(size_t)ids[t + k] * 3 + c];
    const double e0[3] = {v[1][0]-v[0][0], v[1][1]-v[0][1], v[1][2]-v[0][2]};
    const double e1[3] = {v[2][0]-v[0][0], v[2][1]-v[0][1], v[2][2]-v[0][2]};
    const double n[3] = {e0[1]*e1[2] - e0[2]*e1[1],
                         e0[2]*e1[0] - e0[0]*e1[2],
                         e0[0]*e1[1] - e0[1]*e1[0]};
    area += std::sqrt(n[0]*n[0] + n[1]*n[1] + n[2]*n[2]);
  }
  return area * 0.5;
}

/* src/ssol_shape.c:1701-1769 */
extern "C" res_T ssol_mesh_setup
  (ssol_shape* s, const unsigned ntris,
   void (*get_indices)(const unsigned, unsigned[3], void*),
   const unsigned nverts, const ssol_vertex_data attribs[],
   const unsigned nattribs, void* data)
{
  if(!s || !s->dev || s->kind != SHAPE_MESH || !get_indices || !ntris
  || !nverts || !attribs || !nattribs)
    return RES_BAD_ARG;
  if(nattribs > SSOL_ATTRIBS_COUNT__) return RES_MEM_ERR;

  const ssol_vertex_data* apos = nullptr;
  const ssol_vertex_data* anrm = nullptr;
  const ssol_vertex_data* auv = nullptr;
  for(unsigned i = 0; i < nattribs; ++i) {
    switch(attribs[i].usage) {
      case SSOL_POSITION: apos = &attribs[i]; break;
      case SSOL_NORMAL: anrm = &attribs[i]; break;
      case SSOL_TEXCOORD: auv = &attribs[i]; break;
      default: return RES_BAD_ARG;
    }
    if(!attribs[i].get) return RES_BAD_ARG;
  }
  if(!apos) return RES_BAD_ARG;

  std::vector<uint32_t> ids((size_t)ntris * 3);
  for(unsigned t = 0; t < ntris; ++t) {
    unsigned tri[3];
    get_indices(t, tri, data);
    for(int k = 0; k < 3; ++k) {
      if(tri[k] >= nverts) return RES_BAD_ARG;
      ids[(size_t)t * 3 + k] = tri[k];
    }
  }
  std::vector<float> pos((size_t)nverts * 3), nrm, uv;
  for(unsigned v = 0; v < nverts; ++v) apos->get(v, &pos[(size_t)v * 3], data);
  if(anrm) {
    nrm.resize((size_t)nverts * 3);
    for(unsigned v = 0; v < nverts; ++v)
      anrm->get(v, &nrm[(size_t)v * 3], data);
  }
  if(auv) {
    uv.resize((size_t)nverts * 2);
    for(unsigned v = 0; v < nverts; ++v) auv->get(v, &uv[(size_t)v * 2], data);
  }
  s->pos = std::move(pos);
  s->nrm = std::move(nrm);
  s->uv = std::move(uv);
  s->ids = std::move(ids);
  s->rt_area = mesh_area(s->pos, s->ids);
  s->samp_area = s->rt_area;
  s->ready = true;
  return RES_OK;
}

/* check_quadric / check_punched_surface (src/ssol_shape.c:63-136) */
static bool check_quadric(const ssol_quadric* q)
{
  if(!q) return false;
  switch(q->type) {
    case SSOL_QUADRIC_PLANE: return true;
    case SSOL_QUADRIC_PARABOL: return q->data.parabol.focal > 0;
    case SSOL_QUADRIC_PARABOL2F:
      return q->data.parabol2f.focal_x > 0 && q->data.parabol2f.focal_y > 0;
    case SSOL_QUADRIC_HYPERBOL:
      return q->data.hyperbol.img_focal > 0 && q->data.hyperbol.real_focal > 0;
    case SSOL_QUADRIC_PARABOLIC_CYLINDER:
      return q->data.parabolic_cylinder.focal > 0;
    case SSOL_QUADRIC_HEMISPHERE: return q->data.hemisphere.radius > 0;
    default: return false;
  }
}

static bool check_punched_surface(const ssol_punched_surface* p)
{
  if(!p || !p->quadric) return false;
  if(p->nb_carvings == 0 && p->quadric->type != SSOL_QUADRIC_HEMISPHERE)
    return false;
  if(p->nb_carvings && !p->carvings) return false;
  if(!check_quadric(p->quadric)) return false;
  for(size_t i = 0; i < p->nb_carvings; ++i) {
    const ssol_carving& c = p->carvings[i];
    if(!c.get || c.nb_vertices == 0) return false;
    if((unsigned)c.operation >= SSOL_CLIPPING_OPS_COUNT__) return false;
  }
  return true;
}

/* src/ssol_shape.c:1611-1699 */
extern "C" res_T ssol_punched_surface_setup
  (ssol_shape* s, const ssol_punched_surface* p)
{
  if(!s || !s->dev || s->kind != SHAPE_PUNCHED || !check_punched_surface(p))
    return RES_BAD_ARG;

  PunchedInput in;
  in.quadric = *p->quadric;
  for(size_t i = 0; i < p->nb_carvings; ++i) {
    Carving c;
    c.op = p->carvings[i].operation;
    c.xy.resize(p->carvings[i].nb_vertices * 2);
    for(size_t v = 0; v < p->carvings[i].nb_vertices; ++v)
      p->carvings[i].get(v, &c.xy[v * 2], p->carvings[i].context);
    in.carvings.push_back(std::move(c));
  }
  PunchedMesh out;
  const res_T res = ssolb_tessellate_punched(in, out);
  if(res != RES_OK) {
    s->dev->log_error("%s: invalid punched surface.\n", __func__);
    return res;
  }
  s->quadric = in.quadric;
  s->carvings = std::move(in.carvings);
  for(int i = 0; i < 4; ++i) s->qparam[i] = out.qparam[i];
  s->carve_lo[0] = out.lower[0]; s->carve_lo[1] = out.lower[1];
  s->carve_hi[0] = out.upper[0]; s->carve_hi[1] = out.upper[1];
  s->hemi_radius = out.hemi_radius;
  s->grid_n[0] = out.grid_n[0];
  s->grid_n[1] = out.grid_n[1];
  s->grid_delta = out.grid_delta;
  s->grid_exact = out.grid_exact;
  s->pos = std::move(out.rt_pos);
  s->ids = std::move(out.ids);
  s->nrm.clear();
  s->uv = std::move(out.uv);
  s->samp_xy = std::move(out.flat_xy);
  s->samp_ids = s->ids;
  s->rt_area = mesh_area(s->pos, s->ids);
  s->samp_area = mesh_area(out.samp_pos, s->samp_ids);
  s->ready = true;
  return RES_OK;
}

/*******************************************************************************
 * Materials
 ******************************************************************************/
static res_T material_create
  (ssol_device* dev, ssol_material** out, ssol_material_type type)
{
  if(!dev || !out || (unsigned)type >= SSOL_MATERIAL_TYPES_COUNT__)
    return RES_BAD_ARG;
  ssol_material* m = new (std::nothrow) ssol_material();
  if(!m) return RES_MEM_ERR;
  ssol_device_ref_get(dev);
  m->dev = dev;
  m->type = type;
  *out = m;
  return RES_OK;
}

extern "C" res_T ssol_material_create_dielectric
  (ssol_device* dev, ssol_material** out)
{ return material_create(dev, out, SSOL_MATERIAL_DIELECTRIC); }
extern "C" res_T ssol_material_create_mirror
  (ssol_device* dev, ssol_material** out)
{ return material_create(dev, out, SSOL_MATERIAL_MIRROR); }
extern "C" res_T ssol_material_create_matte
  (ssol_device* dev, ssol_material** out)
{ return material_create(dev, out, SSOL_MATERIAL_MATTE); }
extern "C" res_T ssol_material_create_virtual
  (ssol_device* dev, ssol_material** out)
{ return material_create(dev, out, SSOL_MATERIAL_VIRTUAL); }
extern "C" res_T ssol_material_create_thin_dielectric
  (ssol_device* dev, ssol_material** out)
{ return material_create(dev, out, SSOL_MATERIAL_THIN_DIELECTRIC); }

extern "C" res_T ssol_material_get_type
  (const ssol_material* m, enum ssol_material_type* type)
{
  if(!m || !type) return RES_BAD_ARG;
  *type = m->type;
  return RES_OK;
}

extern "C" res_T ssol_material_ref_get(ssol_material* m)
{
  if(!m) return RES_BAD_ARG;
  m->ref.get();
  return RES_OK;
}

extern "C" res_T ssol_material_ref_put(ssol_material* m)
{
  if(!m) return RES_BAD_ARG;
  if(m->ref.put()) {
    ssol_device* dev = m->dev;
    if(m->buf) ssol_param_buffer_ref_put(m->buf);
    ssol_medium_clear(&m->slab_medium);
    ssol_medium_clear(&m->in_medium);
    ssol_medium_clear(&m->out_medium);
    delete m;
    ssol_device_ref_put(dev);
  }
  return RES_OK;
}

extern "C" res_T ssol_material_set_param_buffer
  (ssol_material* m, ssol_param_buffer* buf)
{
  if(!m || !buf) return RES_BAD_ARG;
  ssol_param_buffer_ref_get(buf);
  if(m->buf) ssol_param_buffer_ref_put(m->buf);
  m->buf = buf;
  return RES_OK;
}

extern "C" res_T ssol_dielectric_setup
  (ssol_material* m, const ssol_dielectric_shader* shader,
   const ssol_medium* outside, const ssol_medium* inside)
{
  if(!m || m->type != SSOL_MATERIAL_DIELECTRIC || !shader || !shader->normal
  || !check_medium(outside) || !check_medium(inside))
    return RES_BAD_ARG;
  ssol_medium_copy(&m->out_medium, outside);
  ssol_medium_copy(&m->in_medium, inside);
  m->normal = shader->normal;
  return RES_OK;
}

extern "C" res_T ssol_mirror_setup
  (ssol_material* m, const ssol_mirror_shader* shader,
   const enum ssol_microfacet_distribution distrib)
{
  if(!m || m->type != SSOL_MATERIAL_MIRROR || !shader || !shader->normal
  || !shader->reflectivity || !shader->roughness
  || (unsigned)distrib >= SSOL_MICROFACET_DISTRIBUTIONS_COUNT__)
    return RES_BAD_ARG;
  m->normal = shader->normal;
  m->reflectivity = shader->reflectivity;
  m->roughness = shader->roughness;
  m->distrib = distrib;
  return RES_OK;
}

extern "C" res_T ssol_matte_setup
  (ssol_material* m, const ssol_matte_shader* shader)
{
  if(!m || m->type != SSOL_MATERIAL_MATTE || !shader || !shader->normal
  || !shader->reflectivity)
    return RES_BAD_ARG;
  m->normal = shader->normal;
  m->reflectivity = shader->reflectivity;
  return RES_OK;
}

extern "C" res_T ssol_thin_dielectric_setup
  (ssol_material* m, const ssol_thin_dielectric_shader* shader,
   const ssol_medium* outside, const ssol_medium* slab,
   const double thickness)
{
  if(!m || m->type != SSOL_MATERIAL_THIN_DIELECTRIC || !shader
  || !shader->normal || !check_medium(outside) || !check_medium(slab)
  || thickness < 0)
    return RES_BAD_ARG;
  ssol_medium_copy(&m->slab_medium, slab);
  m->thickness = thickness;
  ssol_medium_copy(&m->out_medium, outside);
  ssol_medium_copy(&m->in_medium, outside);
  m->normal = shader->normal;
  return RES_OK;
}

/*******************************************************************************
 * Param buffer (src/ssol_param_buffer.c)
 ******************************************************************************/
extern "C" res_T ssol_param_buffer_create
  (ssol_device* dev, const size_t capacity, ssol_param_buffer** out)
{
  if(!dev || !capacity || !out) return RES_BAD_ARG;
  ssol_param_buffer* b = new (std::nothrow) ssol_param_buffer();
  if(!b) return RES_MEM_ERR;
  b->mem.resize(capacity + 64);
  b->capacity = capacity;
  ssol_device_ref_get(dev);
  b->dev = dev;
  *out = b;
  return RES_OK;
}

extern "C" res_T ssol_param_buffer_ref_get(ssol_param_buffer* b)
{
  if(!b) return RES_BAD_ARG;
  b->ref.get();
  return RES_OK;
}

extern "C" res_T ssol_param_buffer_clear(ssol_param_buffer* b)
{
  if(!b) return RES_BAD_ARG;
  for(auto& r : b->releases) if(r.second) r.second(r.first);
  b->releases.clear();
  b->used = 0;
  b->first = SIZE_MAX;
  return RES_OK;
}

extern "C" res_T ssol_param_buffer_ref_put(ssol_param_buffer* b)
{
  if(!b) return RES_BAD_ARG;
  if(b->ref.put()) {
    ssol_device* dev = b->dev;
    ssol_param_buffer_clear(b);
    delete b;
    ssol_device_ref_put(dev);
  }
  return RES_OK;
}

static unsigned char* pool_base(ssol_param_buffer* b)
{
  uintptr_t p = reinterpret_cast<uintptr_t>(b->mem.data());
  p = (p + 63) & ~uintptr_t(63);
  return reinterpret_cast<unsigned char*>(p);
}

extern "C" void* ssol_param_buffer_allocate
  (ssol_param_buffer* b, const size_t size, const size_t align,
   void (*release)(void*))
{
  if(!b || !size || !align || (align & (align - 1)) || align > 64)
    return nullptr;
  const size_t offset = (b->used + align - 1) & ~(align - 1);
  if(offset + size > b->capacity) return nullptr;
  void* mem = pool_base(b) + offset;
  b->releases.emplace_back(mem, release);
  b->used = offset + size;
  return mem;
}

extern "C" void* ssol_param_buffer_get(ssol_param_buffer* b)
{
  if(!b) return nullptr;
  return b->used ? pool_base(b) : nullptr;
}

/*******************************************************************************
 * Native shaders for properties that do not vary (include/ssol_b200.h)
 ******************************************************************************/
extern "C" void ssol_b200_shader_param0
  (ssol_device*, ssol_param_buffer* buf, const double, const ssol_surface_fragment*,
   double* val)
{
  const double* p = static_cast<const double*>(ssol_param_buffer_get(buf));
  *val = p ? p[0] : 0.0;
}

extern "C" void ssol_b200_shader_param1
  (ssol_device*, ssol_param_buffer* buf, const double, const ssol_surface_fragment*,
   double* val)
{
  const double* p = static_cast<const double*>(ssol_param_buffer_get(buf));
  *val = p ? p[1] : 0.0;
}

extern "C" void ssol_b200_shader_Ns
  (ssol_device*, ssol_param_buffer*, const double, const ssol_surface_fragment* frag,
   double* val)
{
  val[0] = frag->Ns[0];
  val[1] = frag->Ns[1];
  val[2] = frag->Ns[2];
}

/*******************************************************************************
 * Object and instance
 ******************************************************************************/
extern "C" res_T ssol_object_create(ssol_device* dev, ssol_object** out)
{
  if(!dev || !out) return RES_BAD_ARG;
  ssol_object* o = new (std::nothrow) ssol_object();
  if(!o) return RES_MEM_ERR;
  ssol_device_ref_get(dev);
  o->dev = dev;
  *out = o;
  return RES_OK;
}

extern "C" res_T ssol_object_ref_get(ssol_object* o)
{
  if(!o) return RES_BAD_ARG;
  o->ref.get();
  return RES_OK;
}

extern "C" res_T ssol_object_clear(ssol_object* o)
{
  if(!o) return RES_BAD_ARG;
  for(ShadedShape& s : o->shaded) {
    ssol_shape_ref_put(s.shape);
    ssol_material_ref_put(s.front);
    ssol_material_ref_put(s.back);
  }
  o->shaded.clear();
  o->rt_area = o->samp_area = 0;
  return RES_OK;
}

extern "C" res_T ssol_object_ref_put(ssol_object* o)
{
  if(!o) return RES_BAD_ARG;
  if(o->ref.put()) {
    ssol_device* dev = o->dev;
    ssol_object_clear(o);
    delete o;
    ssol_device_ref_put(dev);
  }
  return RES_OK;
}

/* src/ssol_object.c:111-198: a shape is added once; later adds only warn */
extern "C" res_T ssol_object_add_shaded_shape
  (ssol_object* o, ssol_shape* shape, ssol_material* front,
   ssol_material* back)
{
  if(!o || !shape || !front || !back) return RES_BAD_ARG;
  if(ssolb_object_has_shape(o, shape)) {
    o->dev->log_warning("%s: the object already own the shape.\n", __func__);
    return RES_OK;
  }
  ssol_shape_ref_get(shape);
  ssol_material_ref_get(front);
  ssol_material_ref_get(back);
  o->shaded.push_back({shape, front, back});
  o->rt_area += shape->rt_area;
  o->samp_area += shape->samp_area;
  return RES_OK;
}

extern "C" res_T ssol_object_get_area(const ssol_object* o, double* area)
{
  if(!o || !area) return RES_BAD_ARG;
  *area = o->rt_area;
  return RES_OK;
}

extern "C" res_T ssol_object_instantiate(ssol_object* o, ssol_instance** out)
{
  if(!o || !out) return RES_BAD_ARG;
  ssol_instance* inst = new (std::nothrow) ssol_instance();
  if(!inst) return RES_MEM_ERR;
  ssol_device_ref_get(o->dev);
  ssol_object_ref_get(o);
  inst->dev = o->dev;
  inst->object = o;
  inst->uid = ssolb_next_uid();
  *out = inst;
  return RES_OK;
}

extern "C" res_T ssol_instance_ref_get(ssol_instance* i)
{
  if(!i) return RES_BAD_ARG;
  i->ref.get();
  return RES_OK;
}

extern "C" res_T ssol_instance_ref_put(ssol_instance* i)
{
  if(!i) return RES_BAD_ARG;
  if(i->ref.put()) {
    ssol_device* dev = i->dev;
    ssol_object_ref_put(i->object);
    delete i;
    ssol_device_ref_put(dev);
  }
  return RES_OK;
}

extern "C" res_T ssol_instance_set_transform
  (ssol_instance* i, const double transform[12])
{
  if(!i || !transform) return RES_BAD_ARG;
  for(int k = 0; k < 12; ++k) i->transform[k] = transform[k];
  return RES_OK;
}

extern "C" res_T ssol_instance_set_receiver
  (ssol_instance* i, const int mask, const int per_primitive)
{
  if(!i) return RES_BAD_ARG;
  i->receiver_mask = mask;
  i->per_primitive = per_primitive;
  return RES_OK;
}

extern "C" res_T ssol_instance_is_receiver
  (ssol_instance* i, int* mask, int* per_primitive)
{
  if(!i || !mask || !per_primitive) return RES_BAD_ARG;
  *mask = i->receiver_mask;
  *per_primitive = i->per_primitive;
  return RES_OK;
}

extern "C" res_T ssol_instance_sample(ssol_instance* i, const int sample)
{
  if(!i) return RES_BAD_ARG;
  i->sample = sample;
  return RES_OK;
}

extern "C" res_T ssol_instance_get_id(const ssol_instance* i, uint32_t* id)
{
  if(!i || !id) return RES_BAD_ARG;
  *id = i->uid;
  return RES_OK;
}

/* The area of the instantiated object, untransformed
 * (src/ssol_instance.c:91, 222-230) */
extern "C" res_T ssol_instance_get_area(const ssol_instance* i, double* area)
{
  if(!i || !area) return RES_BAD_ARG;
  *area = i->object->rt_area;
  return RES_OK;
}

extern "C" res_T ssol_instance_get_shaded_shapes_count
  (const ssol_instance* i, size_t* n)
{
  if(!i || !n) return RES_BAD_ARG;
  *n = i->object->shaded.size();
  return RES_OK;
}

void ssolb_d33_invtrans(double out[9], const double m[9])
{
  /* Column major: m[c*3 + r]. inverse transpose = cofactor / det */
  const double a = m[0], b = m[3], c = m[6];
  const double d = m[1], e = m[4], f = m[7];
  const double g = m[2], h = m[5], k = m[8];
  const double A = e*k - f*h, B = -(d*k - f*g), C = d*h - e*g;
  const double D = -(b*k - c*h), E = a*k - c*g, F = -(a*h - b*g);
  const double G = b*f - c*e, H = -(a*f - c*d), K = a*e - b*d;
  const double det = a*A + b*B + c*C;
  const double inv = det != 0 ? 1.0 / det : 0.0;
  /* cofactor matrix (row major) is [[A,B,C],[D,E,F],[G,H,K]]; the inverse
   * transpose equals cofactor / det; store it column major */
  out[0] = A*inv; out[3] = B*inv; out[6] = C*inv;
  out[1] = D*inv; out[4] = E*inv; out[7] = F*inv;
  out[2] = G*inv; out[5] = H*inv; out[8] = K*inv;
}

extern "C" res_T ssol_instance_get_shaded_shape
  (const ssol_instance* i, const size_t k,
   ssol_instantiated_shaded_shape* out)
{
  if(!i || !out || k >= i->object->shaded.size()) return RES_BAD_ARG;
  const ShadedShape& s = i->object->shaded[k];
  out->shape = s.shape;
  out->mtl_front = s.front;
  out->mtl_back = s.back;
  for(int c = 0; c < 9; ++c) out->R__[c] = i->transform[c];
  for(int c = 0; c < 3; ++c) out->T__[c] = i->transform[9 + c];
  ssolb_d33_invtrans(out->R_invtrans__, out->R__);
  return RES_OK;
}

extern "C" res_T ssol_instantiated_shaded_shape_get_vertex_attrib
  (const ssol_instantiated_shaded_shape* s, const unsigned iv,
   const enum ssol_attrib_usage usage, double value[])
{
  if(!s || (unsigned)usage >= SSOL_ATTRIBS_COUNT__ || !value)
    return RES_BAD_ARG;
  const res_T r = ssol_shape_get_vertex_attrib(s->shape, iv, usage, value);
  if(r != RES_OK) return r;
  double tmp[3];
  if(usage == SSOL_NORMAL) {
    for(int c = 0; c < 3; ++c)
      tmp[c] = s->R_invtrans__[c] * value[0] + s->R_invtrans__[3 + c] * value[1]
             + s->R_invtrans__[6 + c] * value[2];
    for(int c = 0; c < 3; ++c) value[c] = tmp[c];
  } else if(usage == SSOL_POSITION) {
    for(int c = 0; c < 3; ++c)
      tmp[c] = s->R__[c] * value[0] + s->R__[3 + c] * value[1]
             + s->R__[6 + c] * value[2] + s->T__[c];
    for(int c = 0; c < 3; ++c) value[c] = tmp[c];
  }
  return RES_OK;
}

/*******************************************************************************
 * Sun (src/ssol_sun.c)
 ******************************************************************************/
static res_T sun_create(ssol_device* dev, ssol_sun** out, SunKind k)
{
  if(!dev || !out) return RES_BAD_ARG;
  ssol_sun* s = new (std::nothrow) ssol_sun();
  if(!s) return RES_MEM_ERR;
  ssol_device_ref_get(dev);
  s->dev = dev;
  s->kind = k;
  *out = s;
  return RES_OK;
}

extern "C" res_T ssol_sun_create_directional(ssol_device* d, ssol_sun** o)
{ return sun_create(d, o, SUNK_DIRECTIONAL); }
extern "C" res_T ssol_sun_create_pillbox(ssol_device* d, ssol_sun** o)
{ return sun_create(d, o, SUNK_PILLBOX); }
extern "C" res_T ssol_sun_create_gaussian(ssol_device* d, ssol_sun** o)
{ return sun_create(d, o, SUNK_GAUSSIAN); }
extern "C" res_T ssol_sun_create_buie(ssol_device* d, ssol_sun** o)
{ return sun_create(d, o, SUNK_BUIE); }

extern "C" res_T ssol_sun_ref_get(ssol_sun* s)
{
  if(!s) return RES_BAD_ARG;
  s->ref.get();
  return RES_OK;
}

extern "C" res_T ssol_sun_ref_put(ssol_sun* s)
{
  if(!s) return RES_BAD_ARG;
  if(s->ref.put()) {
    ssol_device* dev = s->dev;
    if(s->spectrum) ssol_spectrum_ref_put(s->spectrum);
    delete s;
    ssol_device_ref_put(dev);
  }
  return RES_OK;
}

extern "C" res_T ssol_sun_set_direction(ssol_sun* s, const double d[3])
{
  if(!s || !d) return RES_BAD_ARG;
  const double len = std::sqrt(d[0]*d[0] + d[1]*d[1] + d[2]*d[2]);
  if(len == 0) return RES_BAD_ARG;
  for(int i = 0; i < 3; ++i) s->direction[i] = d[i] / len;
  return RES_OK;
}

extern "C" res_T ssol_sun_get_direction(const ssol_sun* s, double d[3])
{
  if(!s || !d) return RES_BAD_ARG;
  for(int i = 0; i < 3; ++i) d[i] = s->direction[i];
  return RES_OK;
}

extern "C" res_T ssol_sun_set_dni(ssol_sun* s, const double dni)
{
  if(!s || dni <= 0) return RES_BAD_ARG;
  s->dni = dni;
  return RES_OK;
}

extern "C" res_T ssol_sun_get_dni(const ssol_sun* s, double* dni)
{
  if(!s || !dni) return RES_BAD_ARG;
  *dni = s->dni;
  return RES_OK;
}

extern "C" res_T ssol_sun_set_spectrum(ssol_sun* s, ssol_spectrum* spec)
{
  if(!s || !spec) return RES_BAD_ARG;
  if(spec == s->spectrum) return RES_OK;
  ssol_spectrum_ref_get(spec);
  if(s->spectrum) ssol_spectrum_ref_put(s->spectrum);
  s->spectrum = spec;
  return RES_OK;
}

extern "C" res_T ssol_sun_pillbox_set_half_angle(ssol_sun* s, const double a)
{
  if(!s || a <= 0 || a > M_PI * 0.5 || s->kind != SUNK_PILLBOX)
    return RES_BAD_ARG;
  s->half_angle = a;
  return RES_OK;
}

extern "C" res_T ssol_sun_gaussian_set_std_dev(ssol_sun* s, const double sd)
{
  if(!s || sd <= 0 || s->kind != SUNK_GAUSSIAN) return RES_BAD_ARG;
  s->std_dev = sd;
  return RES_OK;
}

extern "C" res_T ssol_sun_set_buie_param(ssol_sun* s, const double csr)
{
  if(!s || csr <= 0 || csr >= 1 || s->kind != SUNK_BUIE) return RES_BAD_ARG;
  s->csr = csr;
  return RES_OK;
}

/*******************************************************************************
 * Atmosphere (src/ssol_atmosphere.c)
 ******************************************************************************/
extern "C" res_T ssol_atmosphere_create(ssol_device* dev, ssol_atmosphere** o)
{
  if(!dev || !o) return RES_BAD_ARG;
  ssol_atmosphere* a = new (std::nothrow) ssol_atmosphere();
  if(!a) return RES_MEM_ERR;
  ssol_device_ref_get(dev);
  a->dev = dev;
  *o = a;
  return RES_OK;
}

extern "C" res_T ssol_atmosphere_ref_get(ssol_atmosphere* a)
{
  if(!a) return RES_BAD_ARG;
  a->ref.get();
  return RES_OK;
}

extern "C" res_T ssol_atmosphere_ref_put(ssol_atmosphere* a)
{
  if(!a) return RES_BAD_ARG;
  if(a->ref.put()) {
    ssol_device* dev = a->dev;
    ssol_data_clear(&a->extinction);
    delete a;
    ssol_device_ref_put(dev);
  }
  return RES_OK;
}

/* Extinction must lie in [0, 1] (src/ssol_atmosphere.c:42-62) */
extern "C" res_T ssol_atmosphere_set_extinction
  (ssol_atmosphere* a, ssol_data* ext)
{
  if(!a || !ext) return RES_BAD_ARG;
  if(ext->type == SSOL_DATA_REAL) {
    if(ext->value.real < 0 || ext->value.real > 1) return RES_BAD_ARG;
  } else if(ext->type == SSOL_DATA_SPECTRUM) {
    if(!spectrum_check_data(ext->value.spectrum, 0, 1)) return RES_BAD_ARG;
  } else return RES_BAD_ARG;
  ssol_data_copy(&a->extinction, ext);
  return RES_OK;
}

/*******************************************************************************
 * Scene (src/ssol_scene.c:46-330)
 ******************************************************************************/
extern "C" res_T ssol_scene_create(ssol_device* dev, ssol_scene** out)
{
  if(!dev || !out) return RES_BAD_ARG;
  ssol_scene* s = new (std::nothrow) ssol_scene();
  if(!s) return RES_MEM_ERR;
  ssol_device_ref_get(dev);
  s->dev = dev;
  *out = s;
  return RES_OK;
}

extern "C" res_T ssol_scene_ref_get(ssol_scene* s)
{
  if(!s) return RES_BAD_ARG;
  s->ref.get();
  return RES_OK;
}

extern "C" res_T ssol_scene_detach_sun(ssol_scene* s, ssol_sun* sun)
{
  if(!s || !sun || !s->sun || sun->attached != s) return RES_BAD_ARG;
  sun->attached = nullptr;
  s->sun = nullptr;
  ssol_sun_ref_put(sun);
  return RES_OK;
}

extern "C" res_T ssol_scene_detach_atmosphere
  (ssol_scene* s, ssol_atmosphere* a)
{
  if(!s || !a || !s->atmosphere || a->attached != s) return RES_BAD_ARG;
  a->attached = nullptr;
  s->atmosphere = nullptr;
  ssol_atmosphere_ref_put(a);
  return RES_OK;
}

extern "C" res_T ssol_scene_clear(ssol_scene* s)
{
  if(!s) return RES_BAD_ARG;
  for(ssol_instance* i : s->instances) ssol_instance_ref_put(i);
  s->instances.clear();
  if(s->sun) ssol_scene_detach_sun(s, s->sun);
  if(s->atmosphere) ssol_scene_detach_atmosphere(s, s->atmosphere);
  return RES_OK;
}

extern "C" res_T ssol_scene_ref_put(ssol_scene* s)
{
  if(!s) return RES_BAD_ARG;
  if(s->ref.put()) {
    ssol_device* dev = s->dev;
    ssol_scene_clear(s);
    delete s;
    ssol_device_ref_put(dev);
  }
  return RES_OK;
}

extern "C" res_T ssol_scene_attach_instance(ssol_scene* s, ssol_instance* i)
{
  if(!s || !i) return RES_BAD_ARG;
  for(ssol_instance* x : s->instances) if(x == i) return RES_OK;
  ssol_instance_ref_get(i);
  s->instances.push_back(i);
  return RES_OK;
}

extern "C" res_T ssol_scene_detach_instance(ssol_scene* s, ssol_instance* i)
{
  if(!s || !i) return RES_BAD_ARG;
  for(size_t k = 0; k < s->instances.size(); ++k) {
    if(s->instances[k] == i) {
      s->instances.erase(s->instances.begin() + (long)k);
      ssol_instance_ref_put(i);
      return RES_OK;
    }
  }
  return RES_BAD_ARG;
}

extern "C" res_T ssol_scene_attach_sun(ssol_scene* s, ssol_sun* sun)
{
  if(!s || !sun) return RES_BAD_ARG;
  if(sun->attached || s->sun) {
    if(sun->attached != s || s->sun != sun) return RES_BAD_ARG;
    return RES_OK;
  }
  ssol_sun_ref_get(sun);
  s->sun = sun;
  sun->attached = s;
  return RES_OK;
}

extern "C" res_T ssol_scene_attach_atmosphere
  (ssol_scene* s, ssol_atmosphere* a)
{
  if(!s || !a) return RES_BAD_ARG;
  if(a->attached || s->atmosphere) {
    if(a->attached != s || s->atmosphere != a) return RES_BAD_ARG;
    return RES_OK;
  }
  ssol_atmosphere_ref_get(a);
  s->atmosphere = a;
  a->attached = s;
  return RES_OK;
}

extern "C" res_T ssol_scene_for_each_instance
  (ssol_scene* s, res_T (*func)(ssol_instance*, void*), void* ctx)
{
  if(!s || !func) return RES_BAD_ARG;
  for(ssol_instance* i : s->instances) {
    const res_T r = func(i, ctx);
    if(r != RES_OK) return r;
  }
  return RES_OK;
}

/* World AABB of every instantiated triangle (RT representation) */
extern "C" res_T ssol_scene_compute_aabb
  (const ssol_scene* s, float lower[3], float upper[3])
{
  if(!s || !lower || !upper) return RES_BAD_ARG;
  for(int c = 0; c < 3; ++c) {
    lower[c] = std::numeric_limits<float>::max();
    upper[c] = -std::numeric_limits<float>::max();
  }
  for(const ssol_instance* i : s->instances) {
    const double* T = i->transform;
    for(const ShadedShape& ss : i->object->shaded) {
      const std::vector<float>& p = ss.shape->pos;
      for(size_t v = 0; v + 2 < p.size(); v += 3) {
        for(int c = 0; c < 3; ++c) {
          const double w = T[c] * p[v] + T[3 + c] * p[v + 1]
                         + T[6 + c] * p[v + 2] + T[9 + c];
          lower[c] = std::fmin(lower[c], (float)w);
          upper[c] = std::fmax(upper[c], (float)w);
        }
      }
    }
  }
  return RES_OK;
}
