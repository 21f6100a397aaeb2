/*
 * snapshot.h - a scene snapshot resident in device memory, for the
 * renderers (render.cpp). solve.cpp builds it with the same flattening,
 * index validation and device memory cache as a solve.
 */
#ifndef SSOL_B200_SNAPSHOT_H
#define SSOL_B200_SNAPSHOT_H

#include "device_scene.h"
#include "objects.h"

#define SSOL_SHARED_BUILD
#include "../../include/ssol_b200.h"

#include <cuda_runtime_api.h>

struct DeviceSnapshot {
  void* d_scene = nullptr;
  size_t alloc = 0; /* bytes of the device block */
  size_t bytes = 0; /* host -> device bytes */
  int precision = SSOL_B200_FP32;
  ssolb::DScene<float> s32{};
  ssolb::DScene<double> s64{};
};

/* Flatten `scn` in the precision and BVH leaf size of `options` (NULL =>
 * defaults; the launch shape fields are ignored), check it and upload it on
 * the device's stream. Needs the sun, its spectrum and DNI (RES_BAD_ARG),
 * not a sampled instance. */
res_T ssolb_snapshot_create
  (ssol_scene* scn, const ssol_b200_options* options, DeviceSnapshot& out);
void ssolb_snapshot_release(ssol_device* dev, DeviceSnapshot& s);

/* Device blocks through the per-device cache of solve.cpp */
cudaError_t ssolb_dev_alloc(ssol_device* dev, void** p, size_t bytes);
void ssolb_dev_free(ssol_device* dev, void* p, size_t bytes);

#endif /* SSOL_B200_SNAPSHOT_H */
