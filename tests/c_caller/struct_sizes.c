/*
 * struct_sizes.c - sizes and field offsets of the structs the Python binding
 * mirrors (include/ssol_b200.h), printed as "name value" lines, and the
 * default options, so that a test can hold the ctypes layouts to the C ones.
 */
#include <stddef.h>
#include <stdio.h>

#include "ssol_b200.h"

int main(void)
{
  const struct ssol_b200_options d = SSOL_B200_OPTIONS_DEFAULT;
  printf("options.size %zu\n", sizeof(struct ssol_b200_options));
  printf("options.bvh_builder %zu\n", offsetof(struct ssol_b200_options, bvh_builder));
  printf("options.count_work %zu\n", offsetof(struct ssol_b200_options, count_work));
  printf("stats.size %zu\n", sizeof(struct ssol_b200_stats));
  printf("stats.bvh_device %zu\n", offsetof(struct ssol_b200_stats, bvh_device));
  printf("default.precision %d\n", (int)d.precision);
  printf("default.block_size %d\n", d.block_size);
  printf("default.waves %d\n", d.waves);
  printf("default.bvh_builder %d\n", (int)d.bvh_builder);
  printf("default.count_work %d\n", d.count_work);
  printf("builder.auto %d\n", (int)SSOL_B200_BVH_AUTO);
  printf("builder.sah %d\n", (int)SSOL_B200_BVH_SAH);
  printf("builder.lbvh %d\n", (int)SSOL_B200_BVH_LBVH);
  return 0;
}
