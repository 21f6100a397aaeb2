/*
 * solve_mirror.c - a C caller of the ssol API, written the way the
 * reference's own tests and callers are (include only ssol.h and ssp.h,
 * link one library), to show the B200 library as a drop-in at the C ABI.
 *
 * Scene: one 10 x 10 m horizontal mirror (reflectivity 0.9) at the origin,
 * a 4 x 4 m receiver 50 m along the reflected ray facing the mirror
 * (specular 0.05, front side receiver, not sampled), pillbox sun of
 * 4.65 mrad, DNI 1000, from (0, -cos45, sin45). Solves N realisations with
 * a Philox stream seeded by SEED and prints, one per line,
 * "name E SE" for the global estimates and the receiver's incoming and
 * absorbed flux.
 *
 * Usage: solve_mirror N SEED
 */
#include "ssol.h"
#include "ssp.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>

static const unsigned square_ids[6] = {0, 2, 1, 2, 0, 3};

struct square { float half; };

static void get_ids(const unsigned itri, unsigned ids[3], void* ctx)
{
  (void)ctx;
  ids[0] = square_ids[itri * 3 + 0];
  ids[1] = square_ids[itri * 3 + 1];
  ids[2] = square_ids[itri * 3 + 2];
}

static void get_pos(const unsigned ivert, float pos[], void* ctx)
{
  const float h = ((const struct square*)ctx)->half;
  static const float sx[4] = {-1, 1, 1, -1}, sy[4] = {-1, -1, 1, 1};
  pos[0] = sx[ivert] * h;
  pos[1] = sy[ivert] * h;
  pos[2] = 0;
}

static void get_normal(struct ssol_device* dev, struct ssol_param_buffer* buf,
                       const double wl, const struct ssol_surface_fragment* frag,
                       double* val)
{
  (void)dev, (void)buf, (void)wl;
  val[0] = frag->Ns[0];
  val[1] = frag->Ns[1];
  val[2] = frag->Ns[2];
}

static void get_refl_09(struct ssol_device* dev, struct ssol_param_buffer* buf,
                        const double wl, const struct ssol_surface_fragment* frag,
                        double* val)
{
  (void)dev, (void)buf, (void)wl, (void)frag;
  *val = 0.9;
}

static void get_refl_005(struct ssol_device* dev, struct ssol_param_buffer* buf,
                         const double wl, const struct ssol_surface_fragment* frag,
                         double* val)
{
  (void)dev, (void)buf, (void)wl, (void)frag;
  *val = 0.05;
}

static void get_zero(struct ssol_device* dev, struct ssol_param_buffer* buf,
                     const double wl, const struct ssol_surface_fragment* frag,
                     double* val)
{
  (void)dev, (void)buf, (void)wl, (void)frag;
  *val = 0;
}

static void get_wlen(const size_t i, double* wlen, double* data, void* ctx)
{
  static const double w[3] = {1, 2, 3}, v[3] = {1, 0.8, 1};
  (void)ctx;
  *wlen = w[i];
  *data = v[i];
}

#define CHECK(call) do { res_T r_ = (call); if(r_ != RES_OK) { \
  fprintf(stderr, "%s failed: %d\n", #call, r_); return 1; } } while(0)

static int make_square(struct ssol_device* dev, float half, struct ssol_shape** shape)
{
  static struct square sq[2];
  static int n = 0;
  struct ssol_vertex_data attr;
  struct square* s = &sq[n++ % 2];
  s->half = half;
  attr.usage = SSOL_POSITION;
  attr.get = get_pos;
  CHECK(ssol_shape_create_mesh(dev, shape));
  CHECK(ssol_mesh_setup(*shape, 2, get_ids, 4, &attr, 1, s));
  return 0;
}

static void print_result(const char* name, const struct ssol_mc_result* r)
{
  printf("%s %.17g %.17g\n", name, r->E, r->SE);
}

int main(int argc, char** argv)
{
  struct ssol_device* dev = NULL;
  struct ssol_scene* scn = NULL;
  struct ssol_shape *mirror_shape = NULL, *rcv_shape = NULL;
  struct ssol_material *mirror = NULL, *rcv_mtl = NULL;
  struct ssol_object *mirror_obj = NULL, *rcv_obj = NULL;
  struct ssol_instance *heliostat = NULL, *receiver = NULL;
  struct ssol_sun* sun = NULL;
  struct ssol_spectrum* spectrum = NULL;
  struct ssp_rng* rng = NULL;
  struct ssol_estimator* est = NULL;
  struct ssol_mirror_shader shader = SSOL_MIRROR_SHADER_NULL;
  struct ssol_mc_global glob;
  struct ssol_mc_receiver rcv;
  const double c = sqrt(0.5); /* cos 45 deg */
  const double r[3] = {0, c, c};
  double T[12];
  double sun_dir[3];
  size_t n;
  unsigned long long seed;
  int k;

  if(argc != 3) {
    fprintf(stderr, "usage: %s N SEED\n", argv[0]);
    return 2;
  }
  n = (size_t)strtoull(argv[1], NULL, 10);
  seed = strtoull(argv[2], NULL, 10);

  CHECK(ssol_device_create(NULL, NULL, SSOL_NTHREADS_DEFAULT, 0, &dev));
  CHECK(ssol_scene_create(dev, &scn));

  if(make_square(dev, 5.f, &mirror_shape) || make_square(dev, 2.f, &rcv_shape)) return 1;
  CHECK(ssol_material_create_mirror(dev, &mirror));
  shader.normal = get_normal;
  shader.reflectivity = get_refl_09;
  shader.roughness = get_zero;
  CHECK(ssol_mirror_setup(mirror, &shader, SSOL_MICROFACET_BECKMANN));
  CHECK(ssol_material_create_mirror(dev, &rcv_mtl));
  shader.reflectivity = get_refl_005;
  CHECK(ssol_mirror_setup(rcv_mtl, &shader, SSOL_MICROFACET_BECKMANN));

  CHECK(ssol_object_create(dev, &mirror_obj));
  CHECK(ssol_object_add_shaded_shape(mirror_obj, mirror_shape, mirror, mirror));
  CHECK(ssol_object_instantiate(mirror_obj, &heliostat));
  CHECK(ssol_scene_attach_instance(scn, heliostat));

  /* Receiver frame: local +z toward the mirror (-r), x = up x z with
   * up = (1, 0, 0), y = z x x; 3x4 column-major with the translation 50 r */
  {
    const double z[3] = {-r[0], -r[1], -r[2]};
    const double up[3] = {1, 0, 0};
    double x[3] = {up[1] * z[2] - up[2] * z[1], up[2] * z[0] - up[0] * z[2],
                   up[0] * z[1] - up[1] * z[0]};
    const double lx = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    double y[3];
    for(k = 0; k < 3; ++k) x[k] /= lx;
    y[0] = z[1] * x[2] - z[2] * x[1];
    y[1] = z[2] * x[0] - z[0] * x[2];
    y[2] = z[0] * x[1] - z[1] * x[0];
    for(k = 0; k < 3; ++k) {
      T[k] = x[k];
      T[3 + k] = y[k];
      T[6 + k] = z[k];
      T[9 + k] = 50 * r[k];
    }
  }
  CHECK(ssol_object_create(dev, &rcv_obj));
  CHECK(ssol_object_add_shaded_shape(rcv_obj, rcv_shape, rcv_mtl, rcv_mtl));
  CHECK(ssol_object_instantiate(rcv_obj, &receiver));
  CHECK(ssol_instance_set_transform(receiver, T));
  CHECK(ssol_instance_set_receiver(receiver, SSOL_FRONT, 0));
  CHECK(ssol_instance_sample(receiver, 0));
  CHECK(ssol_scene_attach_instance(scn, receiver));

  CHECK(ssol_spectrum_create(dev, &spectrum));
  CHECK(ssol_spectrum_setup(spectrum, get_wlen, 3, NULL));
  CHECK(ssol_sun_create_pillbox(dev, &sun));
  sun_dir[0] = 0;
  sun_dir[1] = c;
  sun_dir[2] = -c;
  CHECK(ssol_sun_set_direction(sun, sun_dir));
  CHECK(ssol_sun_set_dni(sun, 1000));
  CHECK(ssol_sun_set_spectrum(sun, spectrum));
  CHECK(ssol_sun_pillbox_set_half_angle(sun, 4.65e-3));
  CHECK(ssol_scene_attach_sun(scn, sun));

  CHECK(ssp_rng_create(NULL, SSP_RNG_THREEFRY, &rng));
  CHECK(ssp_rng_set(rng, seed));
  CHECK(ssol_solve(scn, rng, n, 0, NULL, &est));

  CHECK(ssol_estimator_get_mc_global(est, &glob));
  print_result("cos_factor", &glob.cos_factor);
  print_result("absorbed_by_receivers", &glob.absorbed_by_receivers);
  print_result("shadowed", &glob.shadowed);
  print_result("missing", &glob.missing);
  CHECK(ssol_estimator_get_mc_receiver(est, receiver, SSOL_FRONT, &rcv));
  print_result("incoming_flux", &rcv.incoming_flux);
  print_result("absorbed_flux", &rcv.absorbed_flux);

  ssol_estimator_ref_put(est);
  ssp_rng_ref_put(rng);
  ssol_instance_ref_put(heliostat);
  ssol_instance_ref_put(receiver);
  ssol_object_ref_put(mirror_obj);
  ssol_object_ref_put(rcv_obj);
  ssol_material_ref_put(mirror);
  ssol_material_ref_put(rcv_mtl);
  ssol_shape_ref_put(mirror_shape);
  ssol_shape_ref_put(rcv_shape);
  ssol_sun_ref_put(sun);
  ssol_spectrum_ref_put(spectrum);
  ssol_scene_ref_put(scn);
  ssol_device_ref_put(dev);
  return 0;
}
