/*
 * render.cpp - camera, image and the preview renderers ssol_draw_draft /
 * ssol_draw_pt (src/ssol_camera.c, src/ssol_image.c, src/ssol_draw.c,
 * src/ssol_draw_draft.c, src/ssol_draw_pt.c).
 *
 * The renderers snapshot the scene to the device (snapshot.h), render the
 * whole image there (draw.cuh, one thread per pixel) into a device buffer,
 * and, for the ssol.h entry points, copy it back once and hand it to the
 * writer in 32 x 32 tiles visited in Morton order, each tile's pixels row
 * after row, as the reference's draw loop does (src/ssol_draw.c:94-169).
 * The reference calls the writer from its OpenMP threads; here one host
 * thread calls it, tile after tile.
 */
#include "kernels.h"
#include "objects.h"
#include "philox.h"
#include "snapshot.h"

#include <cuda_runtime_api.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

using namespace ssolb;

/*******************************************************************************
 * Camera (src/ssol_camera.c, src/ssol_camera.h): FP32 basis
 ******************************************************************************/
struct ssol_camera {
  RefCount ref;
  ssol_device* dev = nullptr;
  float axis_x[3] = {0, 0, 0};
  float axis_y[3] = {0, 0, 0};
  float axis_z[3] = {0, 0, 0};
  float position[3] = {0, 0, 0};
  float fov_x = 0;
  float rcp_proj_ratio = 1;
};

/* f3_normalize: returns the length, 0 leaves v as it is */
static float f3_normalize(float out[3], const float v[3])
{
  const float len = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  if(len == 0.f) return len;
  for(int c = 0; c < 3; ++c) out[c] = v[c] / len;
  return len;
}

static void f3_cross(float out[3], const float a[3], const float b[3])
{
  const float r[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2],
                      a[0] * b[1] - a[1] * b[0]};
  for(int c = 0; c < 3; ++c) out[c] = r[c];
}

extern "C" res_T ssol_camera_create(ssol_device* dev, ssol_camera** out)
{
  if(!dev || !out) return RES_BAD_ARG;
  ssol_camera* cam = new (std::nothrow) ssol_camera();
  if(!cam) return RES_MEM_ERR;
  ssol_device_ref_get(dev);
  cam->dev = dev;
  cam->rcp_proj_ratio = 1.f;
  cam->fov_x = (float)(M_PI / 2.0);
  const double pos[3] = {0, 0, 0}, tgt[3] = {0, 0, -1}, up[3] = {0, 1, 0};
  ssol_camera_look_at(cam, pos, tgt, up);
  *out = cam;
  return RES_OK;
}

extern "C" res_T ssol_camera_ref_get(ssol_camera* cam)
{
  if(!cam) return RES_BAD_ARG;
  cam->ref.get();
  return RES_OK;
}

extern "C" res_T ssol_camera_ref_put(ssol_camera* cam)
{
  if(!cam) return RES_BAD_ARG;
  if(cam->ref.put()) {
    ssol_device* dev = cam->dev;
    delete cam;
    ssol_device_ref_put(dev);
  }
  return RES_OK;
}

extern "C" res_T ssol_camera_set_proj_ratio(ssol_camera* cam, const double ratio)
{
  float y[3];
  if(!cam || ratio <= 0) return RES_BAD_ARG;
  if(f3_normalize(y, cam->axis_y) <= 0) return RES_BAD_ARG;
  cam->rcp_proj_ratio = (float)(1.0 / ratio);
  for(int c = 0; c < 3; ++c) cam->axis_y[c] = y[c] * cam->rcp_proj_ratio;
  return RES_OK;
}

extern "C" res_T ssol_camera_set_fov(ssol_camera* cam, const double fov_x)
{
  float z[3];
  if(!cam || (float)fov_x <= 0) return RES_BAD_ARG;
  if(f3_normalize(z, cam->axis_z) <= 0) return RES_BAD_ARG;
  const float depth = (float)(1.0 / std::tan(fov_x * 0.5));
  for(int c = 0; c < 3; ++c) cam->axis_z[c] = z[c] * depth;
  cam->fov_x = (float)fov_x;
  return RES_OK;
}

extern "C" res_T ssol_camera_look_at
  (ssol_camera* cam, const double pos[3], const double tgt[3], const double up[3])
{
  if(!cam || !pos || !tgt || !up) return RES_BAD_ARG;
  float p[3], t[3], u[3], x[3], y[3], z[3], d[3];
  for(int c = 0; c < 3; ++c) {
    p[c] = (float)pos[c];
    t[c] = (float)tgt[c];
    u[c] = (float)up[c];
    d[c] = t[c] - p[c];
  }
  if(f3_normalize(z, d) <= 0) return RES_BAD_ARG;
  f3_cross(d, z, u);
  if(f3_normalize(x, d) <= 0) return RES_BAD_ARG;
  f3_cross(d, z, x);
  if(f3_normalize(y, d) <= 0) return RES_BAD_ARG;
  const float depth = (float)(1.0 / std::tan(cam->fov_x * 0.5));
  for(int c = 0; c < 3; ++c) {
    cam->axis_x[c] = x[c];
    cam->axis_y[c] = y[c] * cam->rcp_proj_ratio;
    cam->axis_z[c] = z[c] * depth;
    cam->position[c] = p[c];
  }
  return RES_OK;
}

/*******************************************************************************
 * Image (src/ssol_image.c): host memory, 16-byte aligned rows
 ******************************************************************************/
struct ssol_image {
  RefCount ref;
  ssol_device* dev = nullptr;
  char* mem = nullptr;
  size_t pitch = 0;
  size_t size[2] = {0, 0};
  ssol_pixel_format format = SSOL_PIXEL_FORMATS_COUNT__;
};

extern "C" res_T ssol_image_create(ssol_device* dev, ssol_image** out)
{
  if(!dev || !out) return RES_BAD_ARG;
  ssol_image* img = new (std::nothrow) ssol_image();
  if(!img) return RES_MEM_ERR;
  ssol_device_ref_get(dev);
  img->dev = dev;
  *out = img;
  return RES_OK;
}

extern "C" res_T ssol_image_ref_get(ssol_image* img)
{
  if(!img) return RES_BAD_ARG;
  img->ref.get();
  return RES_OK;
}

extern "C" res_T ssol_image_ref_put(ssol_image* img)
{
  if(!img) return RES_BAD_ARG;
  if(img->ref.put()) {
    ssol_device* dev = img->dev;
    std::free(img->mem);
    delete img;
    ssol_device_ref_put(dev);
  }
  return RES_OK;
}

extern "C" res_T ssol_image_setup
  (ssol_image* img, const size_t width, const size_t height,
   const ssol_pixel_format fmt)
{
  if(!img || width == 0 || height == 0 || (unsigned)fmt >= SSOL_PIXEL_FORMATS_COUNT__)
    return RES_BAD_ARG;
  const size_t pitch = width * ssol_sizeof_pixel_format(fmt);
  if(height > SIZE_MAX / pitch) return RES_MEM_ERR;
  const size_t bytes = ((pitch * height) + 15) & ~size_t(15);
  void* mem = std::aligned_alloc(16, bytes);
  if(!mem) return RES_MEM_ERR;
  std::free(img->mem);
  img->mem = (char*)mem;
  img->pitch = pitch;
  img->size[0] = width;
  img->size[1] = height;
  img->format = fmt;
  return RES_OK;
}

/* `size` is width x height as in src/ssol_image.c:152 */
extern "C" res_T ssol_image_get_layout(const ssol_image* img, ssol_image_layout* layout)
{
  if(!img || !layout) return RES_BAD_ARG;
  layout->row_pitch = img->pitch;
  layout->offset = 0;
  layout->size = img->size[0] * img->size[1];
  layout->width = img->size[0];
  layout->height = img->size[1];
  layout->pixel_format = img->format;
  return RES_OK;
}

extern "C" res_T ssol_image_map(const ssol_image* img, char** mem)
{
  if(!img || !mem) return RES_BAD_ARG;
  *mem = img->mem;
  return RES_OK;
}

extern "C" res_T ssol_image_unmap(const ssol_image* img)
{
  return img ? RES_OK : RES_BAD_ARG;
}

/* map_address (src/ssol_image.c:32-47) */
static double map_address(const double a, const ssol_address_mode mode)
{
  if(mode == SSOL_ADDRESS_CLAMP) return std::min(std::max(a, 0.0), std::nextafter(1.0, 0.0));
  double i;
  double f = std::modf(a, &i);
  if(f < 0) f = 1.0 + f;
  /* 1 + f rounds to 1 for |f| < 2^-53: keep the address inside the image */
  return f < 1.0 ? f : std::nextafter(1.0, 0.0);
}

static const double* image_pixel(const ssol_image* img, size_t x, size_t y)
{
  return (const double*)(img->mem + y * img->pitch + x * sizeof(double[3]));
}

extern "C" res_T ssol_image_sample
  (const ssol_image* img, const ssol_filter_mode filter,
   const ssol_address_mode address_u, const ssol_address_mode address_v,
   const double uv[2], void* val)
{
  if(!img || !uv || !val) return RES_BAD_ARG;
  if(img->format != SSOL_PIXEL_DOUBLE3 || !img->mem) return RES_BAD_ARG;
  if((unsigned)address_u > SSOL_ADDRESS_REPEAT || (unsigned)address_v > SSOL_ADDRESS_REPEAT)
    return RES_BAD_ARG;
  double* pix = (double*)val;
  const double x0 = map_address(uv[0], address_u) * (double)img->size[0];
  const double y0 = map_address(uv[1], address_v) * (double)img->size[1];
  if(filter == SSOL_FILTER_NEAREST) {
    const double* z = image_pixel(img, (size_t)x0, (size_t)y0);
    for(int c = 0; c < 3; ++c) pix[c] = z[c];
    return RES_OK;
  }
  if(filter != SSOL_FILTER_LINEAR) return RES_BAD_ARG;
  const double x1 = map_address(uv[0] + 1.0 / (double)img->size[0], address_u)
                  * (double)img->size[0];
  const double y1 = map_address(uv[1] + 1.0 / (double)img->size[1], address_v)
                  * (double)img->size[1];
  const double* z00 = image_pixel(img, (size_t)x0, (size_t)y0);
  const double* z01 = image_pixel(img, (size_t)x0, (size_t)y1);
  const double* z10 = image_pixel(img, (size_t)x1, (size_t)y0);
  const double* z11 = image_pixel(img, (size_t)x1, (size_t)y1);
  double i;
  const double s = std::modf(x0, &i), t = std::modf(y0, &i);
  for(int c = 0; c < 3; ++c)
    pix[c] = (1 - s) * ((1 - t) * z00[c] + t * z01[c]) + s * ((1 - t) * z10[c] + t * z11[c]);
  return RES_OK;
}

extern "C" res_T ssol_image_write
  (void* image, const size_t origin[2], const size_t size[2],
   const ssol_pixel_format fmt, const void* pixels)
{
  ssol_image* img = (ssol_image*)image;
  if(!img || !origin || !size || !pixels) return RES_BAD_ARG;
  if(fmt != img->format || !img->mem) return RES_BAD_ARG;
  if(origin[0] + size[0] > img->size[0] || origin[1] + size[1] > img->size[1])
    return RES_BAD_ARG;
  const size_t bpp = ssol_sizeof_pixel_format(img->format);
  const size_t src_pitch = size[0] * bpp;
  const char* src = (const char*)pixels;
  for(size_t y = origin[1]; y < origin[1] + size[1]; ++y) {
    std::memcpy(img->mem + y * img->pitch + origin[0] * bpp, src, src_pitch);
    src += src_pitch;
  }
  return RES_OK;
}

/*******************************************************************************
 * Renderers
 ******************************************************************************/
namespace {

constexpr int TILE_SIZE = 32; /* src/ssol_draw.c:27 */

size_t round_up_pow2(size_t v)
{
  size_t p = 1;
  while(p < v) p <<= 1;
  return p;
}

/* morton2D_decode (src/ssol_draw.c:34-43): even bits of `code` */
uint32_t morton_even(uint32_t code)
{
  uint32_t x = code & 0x55555555u;
  x = (x | (x >> 1)) & 0x33333333u;
  x = (x | (x >> 2)) & 0x0F0F0F0Fu;
  x = (x | (x >> 4)) & 0x00FF00FFu;
  x = (x | (x >> 8)) & 0x0000FFFFu;
  return x;
}

/* The draft's sub-pixel offsets, one pair per sample, the same for every
 * pixel (src/ssol_draw_draft.c:164-170): Philox block (i, 0, 0,
 * RNG_DRAW_OFFSET) with key 0, two 24-bit uniforms */
std::vector<float> draft_offsets(size_t spp)
{
  std::vector<float> off(spp * 2);
  for(size_t i = 0; i < spp; ++i) {
    const U32x4 r = philox4x32_10((uint32_t)i, (uint32_t)(i >> 32), 0u,
                                  RNG_DRAW_OFFSET, 0u, 0u);
    off[2 * i] = u01f(r.v[0]);
    off[2 * i + 1] = u01f(r.v[1]);
  }
  return off;
}

struct DrawJob {
  bool pt;
  size_t width, height, spp;
  double up[3];
  uint64_t seed;
};

/* Render into device memory: into `d_pixels` (width x height x 3 doubles)
 * when given, else into a device block of the library that is then copied
 * to `host` */
res_T render_device
  (ssol_scene* scn, ssol_camera* cam, const DrawJob& job,
   const ssol_b200_options* options, double* d_pixels, std::vector<double>* host,
   ssol_b200_stats* stats)
{
  if(job.width > 0x7fffffff || job.height > 0x7fffffff || job.spp > 0x7fffffff)
    return RES_BAD_ARG;
  const size_t npix = job.width * job.height;
  if(npix / job.width != job.height || npix > SIZE_MAX / (3 * sizeof(double)))
    return RES_BAD_ARG;
  const size_t img_bytes = npix * 3 * sizeof(double);
  DeviceSnapshot snap;
  res_T res = ssolb_snapshot_create(scn, options, snap);
  if(res != RES_OK) return res;
  ssol_device* dev = scn->dev;
  const cudaStream_t s = (cudaStream_t)dev->stream;

  /* Scratch: 6 counters, then the draft offsets */
  const std::vector<float> off = job.pt ? std::vector<float>() : draft_offsets(job.spp);
  const size_t scratch = 64 + off.size() * sizeof(float);
  void* d_scratch = nullptr;
  void* d_img = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if(ssolb_dev_alloc(dev, &d_scratch, scratch) != cudaSuccess) {
    d_scratch = nullptr;
    res = RES_MEM_ERR;
  }
  if(res == RES_OK && !d_pixels) {
    if(ssolb_dev_alloc(dev, &d_img, img_bytes) != cudaSuccess) {
      d_img = nullptr;
      res = RES_MEM_ERR;
    }
    d_pixels = (double*)d_img;
  }
  if(res == RES_OK && (cudaMemsetAsync(d_scratch, 0, 64, s) != cudaSuccess
     || (!off.empty() && cudaMemcpyAsync((char*)d_scratch + 64, off.data(),
                                         off.size() * sizeof(float),
                                         cudaMemcpyHostToDevice, s) != cudaSuccess)))
    res = RES_UNKNOWN_ERR;
  if(res == RES_OK) {
    DrawArgs A;
    for(int c = 0; c < 3; ++c) {
      A.cam_x[c] = cam->axis_x[c];
      A.cam_y[c] = cam->axis_y[c];
      A.cam_z[c] = cam->axis_z[c];
      A.cam_pos[c] = cam->position[c];
      A.up[c] = (float)job.up[c];
    }
    A.pix_w = 1.f / (float)job.width;
    A.pix_h = 1.f / (float)job.height;
    A.width = (int)job.width;
    A.height = (int)job.height;
    A.spp = (int)job.spp;
    A.offsets = job.pt ? nullptr : (const float*)((char*)d_scratch + 64);
    A.seed = job.seed;
    A.pixels = d_pixels;
    A.counters = (unsigned long long*)d_scratch;
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    cudaEventRecord(ev0, s);
    int err;
    if(snap.precision == SSOL_B200_FP32)
      err = job.pt ? launch_pt_f32(snap.s32, A, s) : launch_draft_f32(snap.s32, A, s);
    else
      err = job.pt ? launch_pt_f64(snap.s64, A, s) : launch_draft_f64(snap.s64, A, s);
    cudaEventRecord(ev1, s);
    if(err != 0) {
      dev->log_error("draw kernel launch failed: %s\n",
                     cudaGetErrorString((cudaError_t)err));
      res = RES_UNKNOWN_ERR;
    }
  }
  unsigned long long ctr[6] = {0, 0, 0, 0, 0, 0};
  if(res == RES_OK) {
    if(host) {
      try {
        host->resize(npix * 3);
      } catch(...) {
        res = RES_MEM_ERR;
      }
    }
    if(res == RES_OK
    && ((host && cudaMemcpyAsync(host->data(), d_pixels, img_bytes,
                                 cudaMemcpyDeviceToHost, s) != cudaSuccess)
        || cudaMemcpyAsync(ctr, d_scratch, sizeof(ctr), cudaMemcpyDeviceToHost, s)
           != cudaSuccess
        || cudaStreamSynchronize(s) != cudaSuccess)) {
      dev->log_error("draw kernel failed: %s\n", cudaGetErrorString(cudaGetLastError()));
      res = RES_UNKNOWN_ERR;
    }
  }
  if(res == RES_OK && stats) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0, ev1);
    *stats = ssol_b200_stats();
    stats->kernel_ms = ms;
    stats->rays = ctr[0];
    stats->node_visits = ctr[1];
    stats->triangle_tests = ctr[2];
    stats->quadric_tests = ctr[3];
    stats->bounces = ctr[4];
    stats->paths = ctr[5];
    stats->scene_bytes = snap.bytes;
    stats->tally_bytes = host ? img_bytes : 0;
  }
  if(ev0) cudaEventDestroy(ev0);
  if(ev1) cudaEventDestroy(ev1);
  ssolb_dev_free(dev, d_img, img_bytes);
  ssolb_dev_free(dev, d_scratch, scratch);
  ssolb_snapshot_release(dev, snap);
  return res;
}

/* draw (src/ssol_draw.c:97-169) on a device-rendered image */
res_T render_to_writer
  (ssol_scene* scn, ssol_camera* cam, const DrawJob& job,
   ssol_write_pixels_T writer, void* writer_data)
{
  std::vector<double> host;
  const res_T res = render_device(scn, cam, job, nullptr, nullptr, &host, nullptr);
  if(res != RES_OK) return res;

  const size_t ntx = (job.width + TILE_SIZE - 1) / TILE_SIZE;
  const size_t nty = (job.height + TILE_SIZE - 1) / TILE_SIZE;
  size_t ntiles = round_up_pow2(std::max(ntx, nty));
  ntiles *= ntiles;
  std::vector<double> tile((size_t)TILE_SIZE * TILE_SIZE * 3);
  for(size_t code = 0; code < ntiles; ++code) {
    size_t org[2], sz[2];
    org[0] = morton_even((uint32_t)code);
    if(org[0] >= ntx) continue;
    org[1] = morton_even((uint32_t)(code >> 1));
    if(org[1] >= nty) continue;
    org[0] *= TILE_SIZE;
    org[1] *= TILE_SIZE;
    sz[0] = std::min<size_t>(TILE_SIZE, job.width - org[0]);
    sz[1] = std::min<size_t>(TILE_SIZE, job.height - org[1]);
    for(size_t y = 0; y < sz[1]; ++y)
      std::memcpy(tile.data() + y * sz[0] * 3,
                  host.data() + ((org[1] + y) * job.width + org[0]) * 3,
                  sz[0] * 3 * sizeof(double));
    const res_T r = writer(writer_data, org, sz, SSOL_PIXEL_DOUBLE3, tile.data());
    if(r != RES_OK) return r;
  }
  return RES_OK;
}

} /* namespace */

/* src/ssol_draw_draft.c:147-188 then src/ssol_draw.c:108-109: a missing
 * scene or spp fails first, then the scene check, then the other
 * arguments */
extern "C" res_T ssol_draw_draft
  (ssol_scene* scn, ssol_camera* cam, const size_t width, const size_t height,
   const size_t spp, ssol_write_pixels_T writer, void* writer_data)
{
  if(!scn || !spp) return RES_BAD_ARG;
  if(!scn->sun || !scn->sun->spectrum || scn->sun->dni <= 0) return RES_BAD_ARG;
  if(!cam || !width || !height || !writer) return RES_BAD_ARG;
  DrawJob job = {false, width, height, spp, {0, 0, 0}, 0};
  return render_to_writer(scn, cam, job, writer, writer_data);
}

/* src/ssol_draw_pt.c:355-403: the renderer keys its own random streams
 * (seed 0 here) */
extern "C" res_T ssol_draw_pt
  (ssol_scene* scn, ssol_camera* cam, const size_t width, const size_t height,
   const size_t spp, const double up[3], ssol_write_pixels_T writer,
   void* writer_data)
{
  if(!scn || !up) return RES_BAD_ARG;
  if(!scn->sun || !scn->sun->spectrum || scn->sun->dni <= 0) return RES_BAD_ARG;
  if(!cam || !width || !height || !spp || !writer) return RES_BAD_ARG;
  DrawJob job = {true, width, height, spp, {up[0], up[1], up[2]}, 0};
  return render_to_writer(scn, cam, job, writer, writer_data);
}

extern "C" res_T ssol_b200_draw_draft_device
  (ssol_scene* scn, ssol_camera* cam, const size_t width, const size_t height,
   const size_t spp, const ssol_b200_options* options, double* device_pixels,
   ssol_b200_stats* stats)
{
  if(!scn || !cam || !width || !height || !spp || !device_pixels) return RES_BAD_ARG;
  DrawJob job = {false, width, height, spp, {0, 0, 0}, 0};
  return render_device(scn, cam, job, options, device_pixels, nullptr, stats);
}

extern "C" res_T ssol_b200_draw_pt_device
  (ssol_scene* scn, ssol_camera* cam, const size_t width, const size_t height,
   const size_t spp, const double up[3], const uint64_t seed,
   const ssol_b200_options* options, double* device_pixels, ssol_b200_stats* stats)
{
  if(!scn || !cam || !up || !width || !height || !spp || !device_pixels)
    return RES_BAD_ARG;
  DrawJob job = {true, width, height, spp, {up[0], up[1], up[2]}, seed};
  return render_device(scn, cam, job, options, device_pixels, nullptr, stats);
}
