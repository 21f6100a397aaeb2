/*
 * ssol.h - public C API of the B200 solar-flux Monte Carlo solver.
 *
 * Drop-in replacement for the `ssol_*` API of Solstice-Solver 0.9
 * (reference: src/ssol.h). Function names, enumerations, their value order
 * and the public structure layouts follow src/ssol.h so that an application
 * written against the reference compiles unchanged. Everything in here is
 * plain C: no CUDA or C++ type crosses this boundary.
 *
 * What differs from the reference:
 *  - `res_T` and its codes are defined here (the reference takes them from
 *    RSys, which is not part of the reference tree); source compatibility is
 *    the target, not binary compatibility with RSys-built callers.
 *  - `struct ssp_rng` is the counter-based Philox shim declared in ssp.h.
 *  - Shader callbacks are evaluated on the host when `ssol_solve` snapshots
 *    the scene: per material at the sun-spectrum wavelength nodes, and, for
 *    mirror and matte shaders that vary over a mesh, at every vertex of that
 *    mesh; the device interpolates in wavelength and with the barycentric
 *    weights of the hit. Normal shaders are taken to return Ns.
 *  - `ssol_draw_draft` / `ssol_draw_pt` (src/ssol.h:1225-1244) render the
 *    whole image on the GPU into a device buffer, copy it back once and then
 *    hand it to the writer tile by tile (32 x 32, Morton order of tiles, one
 *    thread), as the reference's draw loop does; include/ssol_b200.h adds
 *    entry points that leave the image in device memory.
 */
#ifndef SSOL_H
#define SSOL_H

#include <stddef.h>
#include <stdint.h>

#if defined(SSOL_SHARED_BUILD)
  #define SSOL_API extern __attribute__((visibility("default")))
#else
  #define SSOL_API extern
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Result codes. The reference gets them from RSys (rsys/rsys.h). */
#ifndef SSOL_RES_T_DEFINED
#define SSOL_RES_T_DEFINED
typedef int res_T;
#define RES_OK 0
#define RES_BAD_ARG 1
#define RES_MEM_ERR 2
#define RES_IO_ERR 3
#define RES_UNKNOWN_ERR 4
#define RES_BAD_OP 5
#define RES_EOF 6
#endif

/* "Use as many threads as there are cores" (src/ssol.h:42). Kept for source
 * compatibility; the solve itself runs on the GPU. */
#define SSOL_NTHREADS_DEFAULT (~0u)

struct logger;
struct mem_allocator;
struct ssp_rng;

struct ssol_atmosphere;
struct ssol_camera;
struct ssol_device;
struct ssol_image;
struct ssol_material;
struct ssol_object;
struct ssol_instance;
struct ssol_param_buffer;
struct ssol_scene;
struct ssol_shape;
struct ssol_spectrum;
struct ssol_sun;
struct ssol_estimator;

/* src/ssol.h:64-68 */
enum ssol_side_flag {
  SSOL_FRONT = 1 << 0,
  SSOL_BACK = 1 << 1,
  SSOL_INVALID_SIDE = 1 << 2
};

/* src/ssol.h:70-75 */
enum ssol_path_type {
  SSOL_PATH_MISSING,
  SSOL_PATH_SHADOW,
  SSOL_PATH_SUCCESS,
  SSOL_PATH_ERROR
};

/* src/ssol.h:77-84 */
enum ssol_material_type {
  SSOL_MATERIAL_DIELECTRIC,
  SSOL_MATERIAL_MATTE,
  SSOL_MATERIAL_MIRROR,
  SSOL_MATERIAL_THIN_DIELECTRIC,
  SSOL_MATERIAL_VIRTUAL,
  SSOL_MATERIAL_TYPES_COUNT__
};

/* src/ssol.h:86-90 */
enum ssol_microfacet_distribution {
  SSOL_MICROFACET_BECKMANN,
  SSOL_MICROFACET_PILLBOX,
  SSOL_MICROFACET_DISTRIBUTIONS_COUNT__
};

/* src/ssol.h:92-96 */
enum ssol_clipping_op {
  SSOL_AND,
  SSOL_SUB,
  SSOL_CLIPPING_OPS_COUNT__
};

/* src/ssol.h:98-111 */
enum ssol_pixel_format {
  SSOL_PIXEL_DOUBLE3,
  SSOL_PIXEL_FORMATS_COUNT__
};

enum ssol_filter_mode {
  SSOL_FILTER_LINEAR,
  SSOL_FILTER_NEAREST
};

enum ssol_address_mode {
  SSOL_ADDRESS_CLAMP,
  SSOL_ADDRESS_REPEAT
};

/* src/ssol.h:113-121 */
enum ssol_quadric_type {
  SSOL_QUADRIC_PLANE,
  SSOL_QUADRIC_PARABOL,
  SSOL_QUADRIC_PARABOL2F,
  SSOL_QUADRIC_HYPERBOL,
  SSOL_QUADRIC_PARABOLIC_CYLINDER,
  SSOL_QUADRIC_HEMISPHERE,
  SSOL_QUADRIC_TYPE_COUNT__
};

/* src/ssol.h:124-129 */
enum ssol_attrib_usage {
  SSOL_POSITION,
  SSOL_NORMAL,
  SSOL_TEXCOORD,
  SSOL_ATTRIBS_COUNT__
};

/* src/ssol.h:131-134 */
enum ssol_data_type {
  SSOL_DATA_REAL,
  SSOL_DATA_SPECTRUM
};

/* Per-vertex attribute callback (src/ssol.h:137-145). */
struct ssol_vertex_data {
  enum ssol_attrib_usage usage;
  void (*get)(const unsigned ivert, float value[], void* ctx);
};
#define SSOL_VERTEX_DATA_NULL__ { SSOL_ATTRIBS_COUNT__, NULL }
static const struct ssol_vertex_data SSOL_VERTEX_DATA_NULL =
  SSOL_VERTEX_DATA_NULL__;

/* Layout of an image's pixels (src/ssol.h:160-171) */
struct ssol_image_layout {
  size_t row_pitch; /* bytes between two consecutive rows */
  size_t offset; /* byte offset of the first pixel */
  size_t size; /* overall size of the image buffer */
  size_t width, height; /* pixels in X and Y */
  enum ssol_pixel_format pixel_format;
};
#define SSOL_IMAGE_LAYOUT_NULL__ { 0, 0, 0, 0, 0, SSOL_PIXEL_FORMATS_COUNT__ }
static const struct ssol_image_layout SSOL_IMAGE_LAYOUT_NULL =
  SSOL_IMAGE_LAYOUT_NULL__;

/* Quadrics, all in their local frame (src/ssol.h:172-246). */
struct ssol_quadric_plane { char dummy; }; /* z = 0 */
#define SSOL_QUADRIC_PLANE_DEFAULT__ { 0 }
static const struct ssol_quadric_plane SSOL_QUADRIC_PLANE_DEFAULT =
  SSOL_QUADRIC_PLANE_DEFAULT__;

struct ssol_quadric_parabol { double focal; }; /* x^2 + y^2 = 4 f z */
#define SSOL_QUADRIC_PARABOL_NULL__ { -1.0 }
static const struct ssol_quadric_parabol SSOL_QUADRIC_PARABOL_NULL =
  SSOL_QUADRIC_PARABOL_NULL__;

/* x^2/(4 fx) + y^2/(4 fy) = z */
struct ssol_quadric_parabol2f { double focal_x; double focal_y; };
#define SSOL_QUADRIC_PARABOL2F_NULL__ { -1.0, -1.0 }
static const struct ssol_quadric_parabol2f SSOL_QUADRIC_PARABOL2F_NULL =
  SSOL_QUADRIC_PARABOL2F_NULL__;

/* Hyperboloid of two sheets, upper sheet, vertex at the origin; its foci are
 * at z = -img_focal and z = real_focal (see src/ssol.h:193-198). */
struct ssol_quadric_hyperbol { double img_focal, real_focal; };
#define SSOL_QUADRIC_HYPERBOL_NULL__ { -1.0 , -1.0 }
static const struct ssol_quadric_hyperbol SSOL_QUADRIC_HYPERBOL_NULL =
  SSOL_QUADRIC_HYPERBOL_NULL__;

struct ssol_quadric_parabolic_cylinder { double focal; }; /* y^2 = 4 f z */
#define SSOL_QUADRIC_PARABOLIC_CYLINDER_NULL__ { -1.0 }
static const struct ssol_quadric_parabolic_cylinder
SSOL_QUADRIC_PARABOLIC_CYLINDER_NULL = SSOL_QUADRIC_PARABOLIC_CYLINDER_NULL__;

/* x^2 + y^2 + (z - r)^2 = r^2, z <= r */
struct ssol_quadric_hemisphere { double radius; };
#define SSOL_QUADRIC_HEMISPHERE_NULL__ { -1.0 }
static const struct ssol_quadric_hemisphere SSOL_QUADRIC_HEMISPHERE_NULL =
  SSOL_QUADRIC_HEMISPHERE_NULL__;

/* src/ssol.h:221-236 */
struct ssol_quadric {
  enum ssol_quadric_type type;
  union {
    struct ssol_quadric_plane plane;
    struct ssol_quadric_parabol parabol;
    struct ssol_quadric_parabol2f parabol2f;
    struct ssol_quadric_hyperbol hyperbol;
    struct ssol_quadric_parabolic_cylinder parabolic_cylinder;
    struct ssol_quadric_hemisphere hemisphere;
  } data;
  double transform[12]; /* 3x4 column major, quadric -> object space */
  size_t slices_count_hint; /* SIZE_MAX <=> default discretisation */
};
#define SSOL_QUADRIC_DEFAULT__ {                                               \
  SSOL_QUADRIC_PLANE,                                                          \
  {SSOL_QUADRIC_PLANE_DEFAULT__},                                              \
  {1,0,0, 0,1,0, 0,0,1, 0,0,0},                                                \
  SIZE_MAX                                                                     \
}
static const struct ssol_quadric SSOL_QUADRIC_DEFAULT = SSOL_QUADRIC_DEFAULT__;

/* 2D polygon clipping the quadric domain in its local xy plane
 * (src/ssol.h:248-257). */
struct ssol_carving {
  void (*get)(const size_t ivert, double position[2], void* ctx);
  size_t nb_vertices;
  enum ssol_clipping_op operation;
  void* context;
};
#define SSOL_CARVING_NULL__ { NULL, 0, SSOL_CLIPPING_OPS_COUNT__, NULL }
static const struct ssol_carving SSOL_CARVING_NULL = SSOL_CARVING_NULL__;

/* src/ssol.h:259-266 */
struct ssol_punched_surface {
  struct ssol_quadric* quadric;
  struct ssol_carving* carvings;
  size_t nb_carvings;
};
#define SSOL_PUNCHED_SURFACE_NULL__ { NULL, NULL, 0 }
static const struct ssol_punched_surface SSOL_PUNCHED_SURFACE_NULL =
  SSOL_PUNCHED_SURFACE_NULL__;

/* Real or spectrum valued scalar (src/ssol.h:268-276). */
struct ssol_data {
  enum ssol_data_type type;
  union {
    double real;
    struct ssol_spectrum* spectrum;
  } value;
};
#define SSOL_DATA_NULL__ {SSOL_DATA_REAL, {0.0}}
static const struct ssol_data SSOL_DATA_NULL = SSOL_DATA_NULL__;

/* src/ssol.h:278-284 */
struct ssol_medium {
  struct ssol_data extinction;
  struct ssol_data refractive_index;
};
#define SSOL_MEDIUM_VACUUM__ {{SSOL_DATA_REAL, {0}}, {SSOL_DATA_REAL, {1}}}
static const struct ssol_medium SSOL_MEDIUM_VACUUM = SSOL_MEDIUM_VACUUM__;

/* src/ssol.h:286-298 */
struct ssol_surface_fragment {
  double dir[3];
  double P[3];
  double Ng[3];
  double Ns[3];
  double uv[2];
  double dPdu[3];
  double dPdv[3];
};
#define SSOL_SURFACE_FRAGMENT_NULL__ \
  {{0,0,0}, {0,0,0}, {0,0,0}, {0,0,0}, {0,0}, {0,0,0}, {0,0,0}}
static const struct ssol_surface_fragment SSOL_SURFACE_FRAGMENT_NULL =
  SSOL_SURFACE_FRAGMENT_NULL__;

/* Material parameter callback (src/ssol.h:301-307). */
typedef void
(*ssol_shader_getter_T)
  (struct ssol_device* dev,
   struct ssol_param_buffer* buf,
   const double wavelength,
   const struct ssol_surface_fragment* fragment,
   double* val);

struct ssol_dielectric_shader { ssol_shader_getter_T normal; };
#define SSOL_DIELECTRIC_SHADER_NULL__ { NULL }
static const struct ssol_dielectric_shader SSOL_DIELECTRIC_SHADER_NULL =
  SSOL_DIELECTRIC_SHADER_NULL__;

struct ssol_mirror_shader {
  ssol_shader_getter_T normal;
  ssol_shader_getter_T reflectivity;
  ssol_shader_getter_T roughness;
};
#define SSOL_MIRROR_SHADER_NULL__ { NULL, NULL, NULL }
static const struct ssol_mirror_shader SSOL_MIRROR_SHADER_NULL =
  SSOL_MIRROR_SHADER_NULL__;

struct ssol_matte_shader {
  ssol_shader_getter_T normal;
  ssol_shader_getter_T reflectivity;
};
#define SSOL_MATTE_SHADER_NULL__ { NULL, NULL }
static const struct ssol_matte_shader SSOL_MATTE_SHADER_NULL =
  SSOL_MATTE_SHADER_NULL__;

struct ssol_thin_dielectric_shader { ssol_shader_getter_T normal; };
#define SSOL_THIN_DIELECTRIC_SHADER_NULL__ { NULL }
static const struct ssol_thin_dielectric_shader
SSOL_THIN_DIELECTRIC_SHADER_NULL = SSOL_THIN_DIELECTRIC_SHADER_NULL__;

/* src/ssol.h:342-355 */
struct ssol_instantiated_shaded_shape {
  struct ssol_shape* shape;
  struct ssol_material* mtl_front;
  struct ssol_material* mtl_back;
  double R__[9];
  double T__[3];
  double R_invtrans__[9];
};
#define SSOL_INSTANTIATED_SHADED_SHAPE_NULL__ { 0 }
static const struct ssol_instantiated_shaded_shape
SSOL_INSTANTIATED_SHADED_SHAPE_NULL = SSOL_INSTANTIATED_SHADED_SHAPE_NULL__;

/* src/ssol.h:357-366 */
struct ssol_path_tracker {
  double sun_ray_length;
  double infinite_ray_length;
};
#define SSOL_PATH_TRACKER_DEFAULT__ {-1, -1}
static const struct ssol_path_tracker SSOL_PATH_TRACKER_DEFAULT =
  SSOL_PATH_TRACKER_DEFAULT__;

struct ssol_path { const void* path__; };

struct ssol_path_vertex {
  double pos[3];
  double weight;
};

/* Expectation, variance and standard error of an estimate
 * (src/ssol.h:380-386). */
struct ssol_mc_result {
  double E;
  double V;
  double SE;
};
#define SSOL_MC_RESULT_NULL__ {0, 0, 0}
static const struct ssol_mc_result SSOL_MC_RESULT_NULL = SSOL_MC_RESULT_NULL__;

/* src/ssol.h:388-405 */
struct ssol_mc_global {
  struct ssol_mc_result cos_factor;
  struct ssol_mc_result absorbed_by_receivers;
  struct ssol_mc_result shadowed;
  struct ssol_mc_result missing;
  struct ssol_mc_result extinguished_by_atmosphere;
  struct ssol_mc_result other_absorbed;
};
#define SSOL_MC_GLOBAL_NULL__ {                                                \
  SSOL_MC_RESULT_NULL__, SSOL_MC_RESULT_NULL__, SSOL_MC_RESULT_NULL__,         \
  SSOL_MC_RESULT_NULL__, SSOL_MC_RESULT_NULL__, SSOL_MC_RESULT_NULL__ }
static const struct ssol_mc_global SSOL_MC_GLOBAL_NULL = SSOL_MC_GLOBAL_NULL__;

/* src/ssol.h:407-438 */
struct ssol_mc_receiver {
  struct ssol_mc_result incoming_flux;
  struct ssol_mc_result incoming_if_no_atm_loss;
  struct ssol_mc_result incoming_if_no_field_loss;
  struct ssol_mc_result incoming_lost_in_field;
  struct ssol_mc_result incoming_lost_in_atmosphere;
  struct ssol_mc_result absorbed_flux;
  struct ssol_mc_result absorbed_if_no_atm_loss;
  struct ssol_mc_result absorbed_if_no_field_loss;
  struct ssol_mc_result absorbed_lost_in_field;
  struct ssol_mc_result absorbed_lost_in_atmosphere;
  /* Internal data */
  size_t N__;
  void* mc__;
  const struct ssol_instance* instance__;
};
#define SSOL_MC_RECEIVER_NULL__ {                                              \
  SSOL_MC_RESULT_NULL__, SSOL_MC_RESULT_NULL__, SSOL_MC_RESULT_NULL__,         \
  SSOL_MC_RESULT_NULL__, SSOL_MC_RESULT_NULL__, SSOL_MC_RESULT_NULL__,         \
  SSOL_MC_RESULT_NULL__, SSOL_MC_RESULT_NULL__, SSOL_MC_RESULT_NULL__,         \
  SSOL_MC_RESULT_NULL__, 0, NULL, NULL }
static const struct ssol_mc_receiver SSOL_MC_RECEIVER_NULL =
  SSOL_MC_RECEIVER_NULL__;

/* src/ssol.h:454-461 */
struct ssol_mc_shape {
  size_t N__;
  void* mc__;
  const struct ssol_shape* shape__;
};
#define SSOL_MC_SHAPE_NULL__ { 0, NULL, NULL }
static const struct ssol_mc_shape SSOL_MC_SHAPE_NULL = SSOL_MC_SHAPE_NULL__;

/* src/ssol.h:463-467 */
struct ssol_mc_sampled {
  struct ssol_mc_result cos_factor;
  struct ssol_mc_result shadowed;
  size_t nb_samples;
};

/* Same quantities as ssol_mc_receiver, per unit area (src/ssol.h:469-480). */
struct ssol_mc_primitive {
  struct ssol_mc_result incoming_flux;
  struct ssol_mc_result incoming_if_no_atm_loss;
  struct ssol_mc_result incoming_if_no_field_loss;
  struct ssol_mc_result incoming_lost_in_field;
  struct ssol_mc_result incoming_lost_in_atmosphere;
  struct ssol_mc_result absorbed_flux;
  struct ssol_mc_result absorbed_if_no_atm_loss;
  struct ssol_mc_result absorbed_if_no_field_loss;
  struct ssol_mc_result absorbed_lost_in_field;
  struct ssol_mc_result absorbed_lost_in_atmosphere;
};
#define SSOL_MC_PRIMITIVE_NULL__ {                                             \
  SSOL_MC_RESULT_NULL__, SSOL_MC_RESULT_NULL__, SSOL_MC_RESULT_NULL__,         \
  SSOL_MC_RESULT_NULL__, SSOL_MC_RESULT_NULL__, SSOL_MC_RESULT_NULL__,         \
  SSOL_MC_RESULT_NULL__, SSOL_MC_RESULT_NULL__, SSOL_MC_RESULT_NULL__,         \
  SSOL_MC_RESULT_NULL__ }
static const struct ssol_mc_primitive SSOL_MC_PRIMITIVE_NULL =
  SSOL_MC_PRIMITIVE_NULL__;

/* Pixel sink of the draw functions (src/ssol.h:495-501): `pixels` holds
 * size[0] x size[1] pixels of format `fmt`, row after row, for the tile whose
 * first pixel is `origin` */
typedef res_T
(*ssol_write_pixels_T)
  (void* context,
   const size_t origin[2],
   const size_t size[2],
   const enum ssol_pixel_format fmt,
   const void* pixels);

/* src/ssol.h:503-510; 0 for a format that does not exist (the reference
 * aborts) */
static inline size_t
ssol_sizeof_pixel_format(const enum ssol_pixel_format format)
{
  return format == SSOL_PIXEL_DOUBLE3 ? sizeof(double[3]) : 0;
}

/*
 * Every object is reference counted: `*_create` hands the caller one
 * reference; `*_ref_put` releases it and the object is destroyed when the
 * count reaches zero (src/ssol.h:512-519).
 */

/* Device: src/ssol.h:527-541 (src/ssol_device.c:68-129). The B200 device
 * binds the current CUDA device and owns one CUDA stream. */
SSOL_API res_T ssol_device_create
  (struct logger* logger, struct mem_allocator* allocator,
   const unsigned nthreads_hint, const int verbose, struct ssol_device** dev);
SSOL_API res_T ssol_device_ref_get(struct ssol_device* dev);
SSOL_API res_T ssol_device_ref_put(struct ssol_device* dev);

/* Scene: src/ssol.h:637-691 (src/ssol_scene.c). */
SSOL_API res_T ssol_scene_create
  (struct ssol_device* dev, struct ssol_scene** scn);
SSOL_API res_T ssol_scene_ref_get(struct ssol_scene* scn);
SSOL_API res_T ssol_scene_ref_put(struct ssol_scene* scn);
SSOL_API res_T ssol_scene_attach_instance
  (struct ssol_scene* scn, struct ssol_instance* instance);
SSOL_API res_T ssol_scene_detach_instance
  (struct ssol_scene* scn, struct ssol_instance* instance);
SSOL_API res_T ssol_scene_compute_aabb
  (const struct ssol_scene* scn, float lower[3], float upper[3]);
SSOL_API res_T ssol_scene_clear(struct ssol_scene* scn);
SSOL_API res_T ssol_scene_attach_sun
  (struct ssol_scene* scn, struct ssol_sun* sun);
SSOL_API res_T ssol_scene_detach_sun
  (struct ssol_scene* scn, struct ssol_sun* sun);
SSOL_API res_T ssol_scene_attach_atmosphere
  (struct ssol_scene* scn, struct ssol_atmosphere* atm);
SSOL_API res_T ssol_scene_detach_atmosphere
  (struct ssol_scene* scn, struct ssol_atmosphere* atm);
SSOL_API res_T ssol_scene_for_each_instance
  (struct ssol_scene* scn,
   res_T (*func)(struct ssol_instance* instance, void* ctx),
   void* ctx);

/* Shapes: src/ssol.h:697-761 (src/ssol_shape.c:1525-1769). */
SSOL_API res_T ssol_shape_create_mesh
  (struct ssol_device* dev, struct ssol_shape** shape);
SSOL_API res_T ssol_shape_create_punched_surface
  (struct ssol_device* dev, struct ssol_shape** shape);
SSOL_API res_T ssol_shape_ref_get(struct ssol_shape* shape);
SSOL_API res_T ssol_shape_ref_put(struct ssol_shape* shape);
SSOL_API res_T ssol_shape_get_vertices_count
  (const struct ssol_shape* shape, unsigned* nverts);
SSOL_API res_T ssol_shape_get_vertex_attrib
  (const struct ssol_shape* shape, const unsigned ivert,
   const enum ssol_attrib_usage usage, double value[]);
SSOL_API res_T ssol_shape_get_triangles_count
  (const struct ssol_shape* shape, unsigned* ntris);
SSOL_API res_T ssol_shape_get_triangle_indices
  (const struct ssol_shape* shape, const unsigned itri, unsigned ids[3]);
SSOL_API res_T ssol_punched_surface_setup
  (struct ssol_shape* shape,
   const struct ssol_punched_surface* punched_surface);
SSOL_API res_T ssol_mesh_setup
  (struct ssol_shape* shape,
   const unsigned ntris,
   void (*get_indices)(const unsigned itri, unsigned ids[3], void* ctx),
   const unsigned nverts,
   const struct ssol_vertex_data attribs[],
   const unsigned nattribs,
   void* data);

/* Materials: src/ssol.h:767-834 (src/ssol_material.c:379-535). */
SSOL_API res_T ssol_material_create_dielectric
  (struct ssol_device* dev, struct ssol_material** mtl);
SSOL_API res_T ssol_material_create_mirror
  (struct ssol_device* dev, struct ssol_material** mtl);
SSOL_API res_T ssol_material_create_matte
  (struct ssol_device* dev, struct ssol_material** mtl);
SSOL_API res_T ssol_material_create_virtual
  (struct ssol_device* dev, struct ssol_material** mtl);
SSOL_API res_T ssol_material_create_thin_dielectric
  (struct ssol_device* dev, struct ssol_material** mtl);
SSOL_API res_T ssol_material_get_type
  (const struct ssol_material* mtl, enum ssol_material_type* type);
SSOL_API res_T ssol_material_ref_get(struct ssol_material* mtl);
SSOL_API res_T ssol_material_ref_put(struct ssol_material* mtl);
SSOL_API res_T ssol_material_set_param_buffer
  (struct ssol_material* mtl, struct ssol_param_buffer* buf);
SSOL_API res_T ssol_dielectric_setup
  (struct ssol_material* mtl, const struct ssol_dielectric_shader* shader,
   const struct ssol_medium* outside_medium,
   const struct ssol_medium* inside_medium);
SSOL_API res_T ssol_mirror_setup
  (struct ssol_material* mtl, const struct ssol_mirror_shader* shader,
   const enum ssol_microfacet_distribution distrib);
SSOL_API res_T ssol_matte_setup
  (struct ssol_material* mtl, const struct ssol_matte_shader* shader);
SSOL_API res_T ssol_thin_dielectric_setup
  (struct ssol_material* mtl,
   const struct ssol_thin_dielectric_shader* shader,
   const struct ssol_medium* outside_medium,
   const struct ssol_medium* slab_medium,
   const double thickness);

/* Objects: src/ssol.h:839-870 (src/ssol_object.c). */
SSOL_API res_T ssol_object_create
  (struct ssol_device* dev, struct ssol_object** obj);
SSOL_API res_T ssol_object_ref_get(struct ssol_object* obj);
SSOL_API res_T ssol_object_ref_put(struct ssol_object* obj);
SSOL_API res_T ssol_object_add_shaded_shape
  (struct ssol_object* object, struct ssol_shape* shape,
   struct ssol_material* mtl_front, struct ssol_material* mtl_back);
SSOL_API res_T ssol_object_clear(struct ssol_object* object);
SSOL_API res_T ssol_object_get_area
  (const struct ssol_object* object, double* area);

/* Instances: src/ssol.h:875-942 (src/ssol_instance.c). */
SSOL_API res_T ssol_object_instantiate
  (struct ssol_object* object, struct ssol_instance** instance);
SSOL_API res_T ssol_instance_ref_get(struct ssol_instance* instance);
SSOL_API res_T ssol_instance_ref_put(struct ssol_instance* instance);
SSOL_API res_T ssol_instance_set_transform
  (struct ssol_instance* instance, const double transform[12]);
SSOL_API res_T ssol_instance_set_receiver
  (struct ssol_instance* instance, const int mask, const int per_primitive);
SSOL_API res_T ssol_instance_is_receiver
  (struct ssol_instance* instance, int* mask, int* per_primitive);
SSOL_API res_T ssol_instance_sample
  (struct ssol_instance* instance, const int sample);
SSOL_API res_T ssol_instance_get_id
  (const struct ssol_instance* instance, uint32_t* id);
SSOL_API res_T ssol_instance_get_area
  (const struct ssol_instance* instance, double* area);
SSOL_API res_T ssol_instance_get_shaded_shapes_count
  (const struct ssol_instance* instance, size_t* nshaded_shapes);
SSOL_API res_T ssol_instance_get_shaded_shape
  (const struct ssol_instance* instance, const size_t ishaded_shape,
   struct ssol_instantiated_shaded_shape* shaded_shape_instance);
SSOL_API res_T ssol_instantiated_shaded_shape_get_vertex_attrib
  (const struct ssol_instantiated_shaded_shape* sshape, const unsigned ivert,
   const enum ssol_attrib_usage usage, double value[]);

/* Parameter buffer handed to shader callbacks: src/ssol.h:947-977
 * (src/ssol_param_buffer.c). Host memory only. */
SSOL_API res_T ssol_param_buffer_create
  (struct ssol_device* dev, const size_t capacity,
   struct ssol_param_buffer** buf);
SSOL_API res_T ssol_param_buffer_ref_get(struct ssol_param_buffer* buf);
SSOL_API res_T ssol_param_buffer_ref_put(struct ssol_param_buffer* buf);
SSOL_API void* ssol_param_buffer_allocate
  (struct ssol_param_buffer* buf, const size_t size, const size_t alignment,
   void (*release)(void*));
SSOL_API void* ssol_param_buffer_get(struct ssol_param_buffer* buf);
SSOL_API res_T ssol_param_buffer_clear(struct ssol_param_buffer* buf);

/* Spectrum: src/ssol.h:982-1000 (src/ssol_spectrum.c:123-213). */
SSOL_API res_T ssol_spectrum_create
  (struct ssol_device* dev, struct ssol_spectrum** spectrum);
SSOL_API res_T ssol_spectrum_ref_get(struct ssol_spectrum* spectrum);
SSOL_API res_T ssol_spectrum_ref_put(struct ssol_spectrum* spectrum);
SSOL_API res_T ssol_spectrum_setup
  (struct ssol_spectrum* spectrum,
   void (*get)(const size_t iwlen, double* wlen, double* data, void* ctx),
   const size_t nwlens, void* ctx);

/* Sun: src/ssol.h:1007-1080 (src/ssol_sun.c). */
SSOL_API res_T ssol_sun_create_directional
  (struct ssol_device* dev, struct ssol_sun** sun);
SSOL_API res_T ssol_sun_create_pillbox
  (struct ssol_device* dev, struct ssol_sun** sun);
SSOL_API res_T ssol_sun_create_gaussian
  (struct ssol_device* dev, struct ssol_sun** sun);
SSOL_API res_T ssol_sun_create_buie
  (struct ssol_device* dev, struct ssol_sun** sun);
SSOL_API res_T ssol_sun_ref_get(struct ssol_sun* sun);
SSOL_API res_T ssol_sun_ref_put(struct ssol_sun* sun);
SSOL_API res_T ssol_sun_set_direction
  (struct ssol_sun* sun, const double direction[3]);
SSOL_API res_T ssol_sun_get_direction
  (const struct ssol_sun* sun, double direction[3]);
SSOL_API res_T ssol_sun_set_dni(struct ssol_sun* sun, const double dni);
SSOL_API res_T ssol_sun_get_dni(const struct ssol_sun* sun, double* dni);
SSOL_API res_T ssol_sun_set_spectrum
  (struct ssol_sun* sun, struct ssol_spectrum* spectrum);
SSOL_API res_T ssol_sun_pillbox_set_half_angle
  (struct ssol_sun* sun, const double half_angle);
SSOL_API res_T ssol_sun_gaussian_set_std_dev
  (struct ssol_sun* sun, const double std_dev);
SSOL_API res_T ssol_sun_set_buie_param
  (struct ssol_sun* sun, const double param);

/* Atmosphere: src/ssol.h:1086-1102 (src/ssol_atmosphere.c). */
SSOL_API res_T ssol_atmosphere_create
  (struct ssol_device* dev, struct ssol_atmosphere** atmosphere);
SSOL_API res_T ssol_atmosphere_ref_get(struct ssol_atmosphere* atmosphere);
SSOL_API res_T ssol_atmosphere_ref_put(struct ssol_atmosphere* atmosphere);
SSOL_API res_T ssol_atmosphere_set_extinction
  (struct ssol_atmosphere* atmosphere, struct ssol_data* extinction);

/* Estimator: src/ssol.h:1107-1211 (src/ssol_estimator.c,
 * src/ssol_mc_receiver.c). */
SSOL_API res_T ssol_estimator_ref_get(struct ssol_estimator* estimator);
SSOL_API res_T ssol_estimator_ref_put(struct ssol_estimator* estimator);
SSOL_API res_T ssol_estimator_get_mc_global
  (struct ssol_estimator* estimator, struct ssol_mc_global* mc_global);
SSOL_API res_T ssol_estimator_get_mc_sampled_x_receiver
  (struct ssol_estimator* estimator,
   const struct ssol_instance* prim_instance,
   const struct ssol_instance* recv_instance,
   const enum ssol_side_flag side,
   struct ssol_mc_receiver* rcv);
SSOL_API res_T ssol_estimator_get_realisation_count
  (const struct ssol_estimator* estimator, size_t* count);
SSOL_API res_T ssol_estimator_get_failed_count
  (const struct ssol_estimator* estimator, size_t* count);
SSOL_API res_T ssol_estimator_get_sampled_area
  (const struct ssol_estimator* estimator, double* area);
SSOL_API res_T ssol_estimator_get_sampled_count
  (const struct ssol_estimator* estimator, size_t* count);
SSOL_API res_T ssol_estimator_get_mc_sampled
  (struct ssol_estimator* estimator,
   const struct ssol_instance* samp_instance,
   struct ssol_mc_sampled* sampled);
SSOL_API res_T ssol_estimator_get_rng_state
  (const struct ssol_estimator* estimator, const struct ssp_rng** rng_state);
SSOL_API res_T ssol_estimator_get_tracked_paths_count
  (const struct ssol_estimator* estimator, size_t* npaths);
SSOL_API res_T ssol_estimator_get_tracked_path
  (const struct ssol_estimator* estimator, const size_t ipath,
   struct ssol_path* path);
SSOL_API res_T ssol_path_get_vertices_count
  (const struct ssol_path* path, size_t* nvertices);
SSOL_API res_T ssol_path_get_vertex
  (const struct ssol_path* path, const size_t ivertex,
   struct ssol_path_vertex* vertex);
SSOL_API res_T ssol_path_get_type
  (const struct ssol_path* path, enum ssol_path_type* type);
SSOL_API res_T ssol_estimator_get_mc_receiver
  (struct ssol_estimator* estimator, const struct ssol_instance* instance,
   const enum ssol_side_flag side, struct ssol_mc_receiver* rcv);
SSOL_API res_T ssol_mc_receiver_get_mc_shape
  (struct ssol_mc_receiver* rcv, const struct ssol_shape* shape,
   struct ssol_mc_shape* mc);
SSOL_API res_T ssol_mc_shape_get_mc_primitive
  (struct ssol_mc_shape* shape, const unsigned i,
   struct ssol_mc_primitive* prim);

/* The hot entry point: trace `realisations_count` independent optical paths
 * and return their estimator (src/ssol.h:1216-1223,
 * src/ssol_solver.c:1132-1361). Synchronous: on return the GPU work is done
 * and the estimator is in host memory. */
SSOL_API res_T ssol_solve
  (struct ssol_scene* scn,
   const struct ssp_rng* rng,
   const size_t realisations_count,
   const size_t max_failed_count,
   const struct ssol_path_tracker* tracker,
   struct ssol_estimator** estimator);

/* Preview renderers: src/ssol.h:1225-1244 (src/ssol_draw.c,
 * src/ssol_draw_draft.c, src/ssol_draw_pt.c). Both render with the scene's
 * sun, need its spectrum and DNI (RES_BAD_ARG otherwise) and ignore virtual
 * materials.
 *  - ssol_draw_draft: per pixel, the mean over `spp` sub-pixel positions
 *    (the same `spp` offsets for every pixel) of max(0, cos(N, -dir)) at
 *    the first surface the camera ray reaches, N its shading normal;
 *  - ssol_draw_pt: path tracing with the sun as a directional light (shadow
 *    ray toward -sun direction), a sky of radiance 0.1 above `up`, the
 *    materials' BSDFs and Russian roulette once the throughput drops below
 *    0.1. */
SSOL_API res_T ssol_draw_draft
  (struct ssol_scene* scn,
   struct ssol_camera* cam,
   const size_t width,
   const size_t height,
   const size_t spp,
   ssol_write_pixels_T writer,
   void* writer_data);

SSOL_API res_T ssol_draw_pt
  (struct ssol_scene* scn,
   struct ssol_camera* cam,
   const size_t width,
   const size_t height,
   const size_t spp,
   const double up[3],
   ssol_write_pixels_T writer,
   void* writer_data);

/* Camera: src/ssol.h:543-575 (src/ssol_camera.c). A pinhole camera; its
 * basis is kept in single precision as in the reference. Defaults: at the
 * origin looking toward -z with +y up, horizontal field of view pi/2,
 * width/height ratio 1. */
SSOL_API res_T ssol_camera_create
  (struct ssol_device* dev, struct ssol_camera** cam);
SSOL_API res_T ssol_camera_ref_get(struct ssol_camera* cam);
SSOL_API res_T ssol_camera_ref_put(struct ssol_camera* cam);
SSOL_API res_T ssol_camera_set_proj_ratio
  (struct ssol_camera* cam, const double proj_ratio); /* width / height */
SSOL_API res_T ssol_camera_set_fov /* horizontal field of view, radians */
  (struct ssol_camera* cam, const double fov);
SSOL_API res_T ssol_camera_look_at
  (struct ssol_camera* cam,
   const double position[3],
   const double target[3],
   const double up[3]);

/* Image: src/ssol.h:577-632 (src/ssol_image.c). Host memory, rows of
 * width x pixel size bytes. */
SSOL_API res_T ssol_image_create
  (struct ssol_device* dev, struct ssol_image** image);
SSOL_API res_T ssol_image_ref_get(struct ssol_image* image);
SSOL_API res_T ssol_image_ref_put(struct ssol_image* image);
SSOL_API res_T ssol_image_setup
  (struct ssol_image* image,
   const size_t width,
   const size_t height,
   const enum ssol_pixel_format format);
SSOL_API res_T ssol_image_get_layout
  (const struct ssol_image* image, struct ssol_image_layout* layout);
SSOL_API res_T ssol_image_map
  (const struct ssol_image* image, char** memory);
SSOL_API res_T ssol_image_unmap(const struct ssol_image* image);
SSOL_API res_T ssol_image_sample
  (const struct ssol_image* image,
   const enum ssol_filter_mode filter,
   const enum ssol_address_mode address_u,
   const enum ssol_address_mode address_v,
   const double uv[2],
   void* val);
/* Writer that copies the tile into an ssol_image (`image`) */
SSOL_API res_T ssol_image_write
  (void* image,
   const size_t origin[2],
   const size_t size[2],
   const enum ssol_pixel_format fmt,
   const void* pixels);

/* Data helpers: src/ssol.h:1249-1273 (src/ssol_data.c). */
SSOL_API struct ssol_data* ssol_data_set_real
  (struct ssol_data* data, const double real);
SSOL_API struct ssol_data* ssol_data_set_spectrum
  (struct ssol_data* data, struct ssol_spectrum* spectrum);
SSOL_API struct ssol_data* ssol_data_clear(struct ssol_data* data);
SSOL_API struct ssol_data* ssol_data_copy
  (struct ssol_data* dst, const struct ssol_data* src);
SSOL_API double ssol_data_get_value
  (const struct ssol_data* data, const double wavelength);

static inline struct ssol_medium*
ssol_medium_clear(struct ssol_medium* medium)
{
  ssol_data_clear(&medium->extinction);
  ssol_data_clear(&medium->refractive_index);
  return medium;
}

static inline struct ssol_medium*
ssol_medium_copy(struct ssol_medium* dst, const struct ssol_medium* src)
{
  ssol_data_copy(&dst->extinction, &src->extinction);
  ssol_data_copy(&dst->refractive_index, &src->refractive_index);
  return dst;
}

#ifdef __cplusplus
}
#endif

#endif /* SSOL_H */
