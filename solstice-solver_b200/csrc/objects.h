/*
 * objects.h - host-side object model behind the ssol_* setup API.
 *
 * Each opaque handle of ssol.h is a C++ struct here. They hold host copies of
 * what the caller described (meshes, quadrics, carvings, materials, the sun);
 * nothing touches the GPU until `ssol_solve` flattens the scene
 * (flatten.cpp) and uploads it (solve.cpp).
 */
#ifndef SSOL_B200_OBJECTS_H
#define SSOL_B200_OBJECTS_H

#define SSOL_SHARED_BUILD
#include "../../include/ssol.h"
#include "../../include/ssp.h"

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <map>
#include <memory>
#include <string>
#include <vector>

/* Intrusive reference counter; `release` runs when it drops to zero */
struct RefCount {
  std::atomic<int> n{1};
  void get() { n.fetch_add(1, std::memory_order_relaxed); }
  bool put() { return n.fetch_sub(1, std::memory_order_acq_rel) == 1; }
};

struct ssol_device {
  RefCount ref;
  int verbose = 0;
  int cuda_device = -1; /* bound lazily on the first solve */
  void* stream = nullptr; /* cudaStream_t, created lazily */
  void* mem_cache = nullptr; /* device blocks kept for reuse (solve.cpp) */
  void log_error(const char* fmt, ...) const;
  void log_warning(const char* fmt, ...) const;
};

struct ssol_spectrum {
  RefCount ref;
  ssol_device* dev = nullptr;
  std::vector<double> wavelengths;
  std::vector<double> intensities;
  uint64_t checksum[2] = {0, 0};
};

enum ShapeKind { SHAPE_MESH = 0, SHAPE_PUNCHED = 1 };

struct Carving {
  int op; /* SSOL_AND / SSOL_SUB */
  std::vector<double> xy; /* 2 * nverts */
};

struct ssol_shape {
  RefCount ref;
  ssol_device* dev = nullptr;
  ShapeKind kind = SHAPE_MESH;
  uint32_t uid = 0;
  bool ready = false;

  /* Triangulated representation in shape space: for meshes the user mesh,
   * for punched surfaces the RT tessellation of the carved quadric */
  std::vector<float> pos; /* 3 * nverts */
  std::vector<float> nrm; /* 3 * nverts (optional) */
  std::vector<float> uv; /* 2 * nverts (optional) */
  std::vector<uint32_t> ids; /* 3 * ntris */
  double rt_area = 0;
  double samp_area = 0;

  /* Punched surface only */
  ssol_quadric quadric{};
  double qparam[4] = {0, 0, 0, 0}; /* kind specific, see flatten.cpp */
  std::vector<Carving> carvings;
  double carve_lo[2] = {0, 0}, carve_hi[2] = {0, 0};
  double hemi_radius = 0; /* disk radius for hemispheres */
  size_t grid_n[2] = {0, 0};
  double grid_delta = 0;
  bool grid_exact = false;
  /* flat sampling proxy (quadric local xy, z = 0) */
  std::vector<double> samp_xy; /* 2 * nverts */
  std::vector<uint32_t> samp_ids; /* 3 * ntris */
};

struct ssol_param_buffer {
  RefCount ref;
  ssol_device* dev = nullptr;
  std::vector<unsigned char> mem;
  size_t capacity = 0, used = 0, first = SIZE_MAX;
  std::vector<std::pair<void*, void (*)(void*)>> releases;
};

struct ssol_material {
  RefCount ref;
  ssol_device* dev = nullptr;
  ssol_material_type type = SSOL_MATERIAL_VIRTUAL;
  ssol_shader_getter_T normal = nullptr;
  ssol_shader_getter_T reflectivity = nullptr;
  ssol_shader_getter_T roughness = nullptr;
  ssol_microfacet_distribution distrib = SSOL_MICROFACET_BECKMANN;
  ssol_medium out_medium = SSOL_MEDIUM_VACUUM__;
  ssol_medium in_medium = SSOL_MEDIUM_VACUUM__;
  ssol_medium slab_medium = SSOL_MEDIUM_VACUUM__;
  double thickness = 0;
  ssol_param_buffer* buf = nullptr;
};

struct ShadedShape {
  ssol_shape* shape;
  ssol_material* front;
  ssol_material* back;
};

struct ssol_object {
  RefCount ref;
  ssol_device* dev = nullptr;
  std::vector<ShadedShape> shaded;
  double rt_area = 0, samp_area = 0;
};

struct ssol_instance {
  RefCount ref;
  ssol_device* dev = nullptr;
  ssol_object* object = nullptr;
  uint32_t uid = 0;
  double transform[12] = {1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0};
  int receiver_mask = 0;
  int per_primitive = 0;
  int sample = 1;
};

enum SunKind { SUNK_DIRECTIONAL, SUNK_PILLBOX, SUNK_GAUSSIAN, SUNK_BUIE };

struct ssol_sun {
  RefCount ref;
  ssol_device* dev = nullptr;
  SunKind kind = SUNK_DIRECTIONAL;
  double direction[3] = {0, 0, 0};
  double dni = 0;
  ssol_spectrum* spectrum = nullptr;
  double half_angle = 0;
  double std_dev = 0;
  double csr = 0;
  ssol_scene* attached = nullptr;
};

struct ssol_atmosphere {
  RefCount ref;
  ssol_device* dev = nullptr;
  ssol_data extinction = SSOL_DATA_NULL__;
  ssol_scene* attached = nullptr;
};

struct ssol_scene {
  RefCount ref;
  ssol_device* dev = nullptr;
  std::vector<ssol_instance*> instances; /* attach order */
  ssol_sun* sun = nullptr;
  ssol_atmosphere* atmosphere = nullptr;
};

/* Per side receiver estimate: 10 quantities x (sum w, sum w^2) */
struct RcvSums {
  double q[10][2] = {};
  /* per shape: ntris x 10 x 2, only for per-primitive receivers */
  std::map<const ssol_shape*, std::vector<double>> prims;
};

struct RcvEntry {
  const ssol_instance* inst = nullptr;
  RcvSums side[2]; /* [0] front, [1] back */
};

struct SampEntry {
  double cos[2] = {0, 0};
  double shadow[2] = {0, 0};
  size_t nb_samples = 0;
  std::map<const ssol_instance*, RcvEntry> by_receiver;
};

struct TrackedPath {
  ssol_path_type type = SSOL_PATH_MISSING;
  std::vector<ssol_path_vertex> vertices;
};

/* The mc_data of ssol_mc_receiver points at one of these */
struct McRcvHandle {
  const RcvSums* sums;
};

struct ssol_estimator {
  RefCount ref;
  ssol_device* dev = nullptr;
  size_t realisation_count = 0;
  size_t failed_count = 0;
  double global[6][2] = {};
  double sampled_area = 0;
  std::map<const ssol_instance*, RcvEntry> receivers;
  std::map<const ssol_instance*, SampEntry> sampled;
  std::vector<TrackedPath> paths;
  ssp_rng* rng = nullptr;
  /* B200 extras: last launch timing and counters */
  double kernel_ms = 0;
  unsigned long long stats[6] = {};
  unsigned long long killed = 0;
  unsigned long long scene_bytes = 0, tally_bytes = 0;
  unsigned long long bvh_nodes = 0, bvh_depth = 0, bvh_device = 0;
};

/* Shared helpers (objects.cpp) */
uint32_t ssolb_next_uid();
bool ssolb_data_ceq(const ssol_data& a, const ssol_data& b);
bool ssolb_media_ceq(const ssol_medium& a, const ssol_medium& b);
double ssolb_spectrum_interpolate(const ssol_spectrum* s, double wl);
bool ssolb_object_has_shape(const ssol_object* obj, const ssol_shape* s);

/* ssp_rng state (rng.cpp) */
struct ssp_rng {
  RefCount ref;
  ssp_rng_type type = SSP_RNG_THREEFRY;
  uint64_t seed = 0;
  uint64_t position = 0;
};
res_T ssolb_rng_clone_advanced
  (const ssp_rng* src, uint64_t advance, ssp_rng** out);

#endif /* SSOL_B200_OBJECTS_H */
