// Scene-preparation C API of mutracer_b200 (host memory only).  Produces the
// flattened buffer bundle that mt_context_commit_bundle and the mtc_* entry
// points consume, from seeded synthetic generators.
#pragma once
#include <stdint.h>
#include "../../include/mutracer_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mtp_scene_info {
  uint64_t triangles, unique_triangles;
  uint32_t instances, blases, tlas_vec4, _pad;
  uint64_t bvh_vec4, vertices;
  float world_bounds[6];
  float _pad2[2];
} mtp_scene_info_t;

void *mtp_scene_make(const char *kind, uint32_t width, uint32_t height, uint64_t seed, const uint32_t *params,
                     uint32_t nparams);
void mtp_scene_free(void *scene);
int mtp_scene_bundle(void *scene, mt_scene_bundle *out);
int mtp_scene_info(void *scene, mtp_scene_info_t *info);
int mtp_scene_set_uniform(void *scene, const mtc_trace_uniform *u, const mtc_camera_uniform *cam, uint32_t flags);
int mtp_scene_refit_inputs(void *scene, double *transforms, float *localBounds, int32_t *blasOffsets,
                           int32_t *blasLayouts, int32_t *vertexOffsets, int32_t *materials, float *colors);
int mtp_scene_set_transforms(void *scene, const double *transforms, uint32_t count);
int mtp_scene_refit_host(void *scene);
/* Re-encodes the scene's BLASes in layout code 0 (BVH2) or 2 (BVH_GPU). */
int mtp_scene_set_blas_layout(void *scene, uint32_t layout);
// Source mesh `mesh` of the scene (the input of its BLAS) and where that BLAS
// lies in the scene's bvh buffer (vec4 units).  NULL positions/indices query
// the counts only.
int mtp_scene_mesh(void *scene, uint32_t mesh, float *positions, uint32_t *indices, uint32_t *vertexCount,
                   uint32_t *triangleCount, uint32_t *blasOffset, uint32_t *blasVec4, uint32_t *bins);
int mtp_build_binned_sah(const float *aabbs, uint32_t count, int bins, uint32_t *nodeCount, float *bounds,
                         uint32_t *leftFirst, uint32_t *primCount, uint32_t *primIndices);
int mtp_build_blas(const float *positions, uint32_t vertexCount, const uint32_t *indices, uint32_t triCount, int bins,
                   float *out, uint64_t capacity, uint64_t *vec4Count, uint32_t *maxDepth);
// Host refitBLAS (bvhAccel.ts:800-870) of a layout-0 BLAS buffer in place.
int mtp_refit_blas(float *bvh, uint64_t vec4Count, const float *positions, uint32_t vertexCount, double *area);
int mtp_energy_lut(float *out);
// Light-selection table of `n` weighted choices (source type 2 = analytic,
// source index = position): 4 words per choice, the PMFs and the total.
int mtp_light_alias_table(const double *weights, uint32_t n, uint32_t *words, float *pmfs, double *total);
// Sampling power of one analytic light (type MTC_LIGHT_*).
double mtp_light_power(int type, const float *color, float intensity, float area, float radius);
/* CameraUniform of a perspective look-at camera for a width x height image
 * (the generators' own camera construction). */
int mtp_camera_look_at(uint32_t width, uint32_t height, const double *eye, const double *target, const double *up,
                       double fov_y_deg, mtc_camera_uniform *out);
/* Decodes a scene descriptor v8 (the input of mt_context_commit) into a host
 * scene (free with mtp_scene_free); NULL with *status and a message when the
 * descriptor is rejected.  The same decoding mt_context_commit runs. */
void *mtp_descriptor_decode(const uint8_t *bytes, size_t length, int32_t *status, char *error, size_t capacity);
int mtp_env_distribution(const float *image, uint32_t width, uint32_t height, float *distribution, double *power);

#ifdef __cplusplus
}
#endif
