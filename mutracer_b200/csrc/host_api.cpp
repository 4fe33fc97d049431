// Host C entry points of the scene producers (mtp_*), used by the Python
// package, the benchmark and the tests to create seeded synthetic workloads
// in the reference's flattened buffer formats.
#include <cstring>
#include <string>

#include "mtp_api.h"
#include "scene_prep.h"

using namespace mtp;

extern "C" {

void *mtp_scene_make(const char *kind, uint32_t width, uint32_t height, uint64_t seed, const uint32_t *params,
                     uint32_t nparams) {
  if (!kind || width == 0 || height == 0) return nullptr;
  auto *s = new SceneHost();
  auto param = [&](uint32_t i, uint32_t dflt) { return i < nparams && params ? params[i] : dflt; };
  try {
    std::string k(kind);
    if (k == "cornell") makeCornell(*s, width, height, seed);
    else if (k == "instanced_spheres")
      makeInstancedSpheres(*s, width, height, seed, param(0, 256), param(1, 16), param(2, 28), param(3, 2048),
                           param(4, 4));
    else if (k == "glass_spheres") makeGlassSpheres(*s, width, height, seed, param(0, 32));
    else { delete s; return nullptr; }
  } catch (...) {
    delete s;
    return nullptr;
  }
  return s;
}

int mtp_camera_look_at(uint32_t width, uint32_t height, const double *eye, const double *target, const double *up,
                       double fov_y_deg, mtc_camera_uniform *out) {
  if (!eye || !target || !up || !out || width == 0 || height == 0 || !(fov_y_deg > 0.0 && fov_y_deg < 180.0))
    return MT_ERROR_INVALID_ARGUMENT;
  SceneHost s;
  s.width = width;
  s.height = height;
  CameraDesc c{{eye[0], eye[1], eye[2]}, {target[0], target[1], target[2]}, {up[0], up[1], up[2]}, fov_y_deg};
  setCamera(s, c);
  *out = s.camera;
  return MT_OK;
}

int mtp_scene_set_blas_layout(void *scene, uint32_t layout) {
  if (!scene || (layout != 0 && layout != 2)) return MT_ERROR_INVALID_ARGUMENT;
  try {
    setBlasLayout(*static_cast<SceneHost *>(scene), layout);
  } catch (...) {
    return MT_ERROR_INVALID_ARGUMENT;
  }
  return MT_OK;
}

void mtp_scene_free(void *scene) { delete static_cast<SceneHost *>(scene); }

int mtp_scene_bundle(void *scene, mt_scene_bundle *b) {
  if (!scene || !b) return MT_ERROR_INVALID_ARGUMENT;
  SceneHost &s = *static_cast<SceneHost *>(scene);
  std::memset(b, 0, sizeof(*b));
  b->struct_size = sizeof(mt_scene_bundle);
  b->width = s.width;
  b->height = s.height;
  b->flags = s.flags;
  b->bvh = s.bvh.data();
  b->bvh_vec4_count = s.bvh.size() / 4;
  b->instances = s.instances.data();
  b->instance_count = uint32_t(s.instances.size() / 40);
  b->material_count = uint32_t(s.materials.size() / (MTC_MATERIAL_VEC4_ROWS * 4));
  b->attributes = s.attributes.data();
  b->attribute_words = s.attributes.size();
  b->vertex_layout = s.layout;
  b->materials = s.materials.data();
  b->env_map = s.env.image.empty() ? nullptr : s.env.image.data();
  b->env_width = s.env.width;
  b->env_height = s.env.height;
  b->env_distribution = s.env.image.empty() ? nullptr : s.env.distribution.data();
  b->light_sampling = s.lightSampling.data();
  b->light_sampling_texels = uint32_t(s.lightSampling.size() / 4);
  b->lights_count = uint32_t(s.lights.size() / 24);
  b->energy_lut = s.lut.data();
  b->analytic_lights = s.lights.empty() ? nullptr : s.lights.data();
  b->tlas_stack_size = s.tlasStack;
  b->blas_stack_size = s.blasStack;
  b->camera = s.camera;
  b->uniform = s.uniform;
  b->maps = s.maps.empty() ? nullptr : s.maps.data();
  b->map_count = uint32_t(s.maps.size() / (MTC_MAP_VEC4_ROWS * 4));
  b->map_texels = s.mapTexels.empty() ? nullptr : s.mapTexels.data();
  b->map_texel_count = s.mapTexels.size() / 4;
  b->triangle_materials = s.triangleMaterials.empty() ? nullptr : s.triangleMaterials.data();
  return MT_OK;
}

int mtp_scene_info(void *scene, mtp_scene_info_t *info) {
  if (!scene || !info) return MT_ERROR_INVALID_ARGUMENT;
  SceneHost &s = *static_cast<SceneHost *>(scene);
  std::memset(info, 0, sizeof(*info));
  info->triangles = s.triangleCount;
  info->unique_triangles = s.uniqueTriangleCount;
  info->instances = uint32_t(s.sourceInstances.size());
  info->blases = uint32_t(s.blases.size());
  info->tlas_vec4 = s.tlasVec4;
  info->bvh_vec4 = uint64_t(s.bvh.size() / 4);
  info->vertices = uint64_t(s.attributes.size() / std::max(1u, s.layout.stride));
  for (int k = 0; k < 6; k++) {
    float lo = k < 3 ? s.bvh[k] : s.bvh[4 + (k - 3)];
    info->world_bounds[k] = lo;
  }
  return MT_OK;
}

int mtp_scene_set_uniform(void *scene, const mtc_trace_uniform *u, const mtc_camera_uniform *cam, uint32_t flags) {
  if (!scene) return MT_ERROR_INVALID_ARGUMENT;
  SceneHost &s = *static_cast<SceneHost *>(scene);
  if (u) s.uniform = *u;
  if (cam) s.camera = *cam;
  s.flags = flags;
  return MT_OK;
}

// Per-source-instance refit inputs (same order as the TLAS leaf source index).
int mtp_scene_refit_inputs(void *scene, double *transforms, float *localBounds, int32_t *blasOffsets,
                           int32_t *blasLayouts, int32_t *vertexOffsets, int32_t *materials, float *colors) {
  if (!scene) return MT_ERROR_INVALID_ARGUMENT;
  SceneHost &s = *static_cast<SceneHost *>(scene);
  for (size_t i = 0; i < s.sourceInstances.size(); i++) {
    const Instance &ins = s.sourceInstances[i];
    if (transforms) std::memcpy(transforms + i * 16, ins.transform, sizeof(ins.transform));
    if (localBounds) std::memcpy(localBounds + i * 6, s.blases[ins.blasIndex].localBounds, 24);
    if (blasOffsets) blasOffsets[i] = int32_t(s.blasOffsets[ins.blasIndex]);
    if (blasLayouts) blasLayouts[i] = int32_t(s.blasLayout);
    if (vertexOffsets) vertexOffsets[i] = int32_t(s.vertexOffsets[ins.blasIndex]);
    if (materials) materials[i] = ins.material;
    if (colors) std::memcpy(colors + i * 3, ins.color, 12);
  }
  return MT_OK;
}

// Replace source-instance transforms (column-major f64) before a host refit.
int mtp_scene_set_transforms(void *scene, const double *transforms, uint32_t count) {
  if (!scene || !transforms) return MT_ERROR_INVALID_ARGUMENT;
  SceneHost &s = *static_cast<SceneHost *>(scene);
  if (count != s.sourceInstances.size()) return MT_ERROR_INVALID_ARGUMENT;
  for (uint32_t i = 0; i < count; i++) std::memcpy(s.sourceInstances[i].transform, transforms + size_t(i) * 16, 128);
  return MT_OK;
}

// Full host refit of the scene's own TLAS and records (bvhAccel.ts:579-740).
int mtp_scene_refit_host(void *scene) {
  if (!scene) return MT_ERROR_INVALID_ARGUMENT;
  SceneHost &s = *static_cast<SceneHost *>(scene);
  refitTlasHost(s.bvh.data(), s.instances.data(), s.sourceInstances, s.blases, s.blasOffsets, s.vertexOffsets,
                s.blasLayout);
  return MT_OK;
}

int mtp_build_binned_sah(const float *aabbs, uint32_t count, int bins, uint32_t *nodeCount, float *bounds,
                         uint32_t *leftFirst, uint32_t *primCount, uint32_t *primIndices) {
  if ((!aabbs && count) || !nodeCount || bins < 2) return MT_ERROR_INVALID_ARGUMENT;
  BinnedBvh b = buildBinnedSahBvh(aabbs, count, bins);
  *nodeCount = b.nodeCount;
  if (bounds) std::memcpy(bounds, b.bounds.data(), size_t(b.nodeCount) * 24);
  if (leftFirst) std::memcpy(leftFirst, b.leftFirst.data(), size_t(b.nodeCount) * 4);
  if (primCount) std::memcpy(primCount, b.primCount.data(), size_t(b.nodeCount) * 4);
  if (primIndices) std::memcpy(primIndices, b.primIndices.data(), size_t(count) * 4);
  return MT_OK;
}

// buildBLAS into a caller buffer of `capacity` vec4 words; reports the size.
int mtp_build_blas(const float *positions, uint32_t vertexCount, const uint32_t *indices, uint32_t triCount, int bins,
                   float *out, uint64_t capacity, uint64_t *vec4Count, uint32_t *maxDepth) {
  if (!positions || !indices || !vec4Count) return MT_ERROR_INVALID_ARGUMENT;
  std::vector<float> p(positions, positions + size_t(vertexCount) * 3);
  std::vector<uint32_t> ix(indices, indices + size_t(triCount) * 3);
  Blas b = buildBlas(p, ix, bins);
  *vec4Count = b.buffer.size() / 4;
  if (maxDepth) *maxDepth = b.maxDepth;
  if (!out) return MT_OK;
  if (capacity < *vec4Count) return MT_ERROR_BUFFER_TOO_SMALL;
  std::memcpy(out, b.buffer.data(), b.buffer.size() * 4);
  return MT_OK;
}

int mtp_scene_mesh(void *scene, uint32_t mesh, float *positions, uint32_t *indices, uint32_t *vertexCount,
                   uint32_t *triangleCount, uint32_t *blasOffset, uint32_t *blasVec4, uint32_t *bins) {
  if (!scene) return MT_ERROR_INVALID_ARGUMENT;
  SceneHost &s = *static_cast<SceneHost *>(scene);
  if (mesh >= s.sourceIndices.size()) return MT_ERROR_INVALID_ARGUMENT;
  const std::vector<float> &p = s.sourcePositions[mesh];
  const std::vector<uint32_t> &ix = s.sourceIndices[mesh];
  if (vertexCount) *vertexCount = uint32_t(p.size() / 3);
  if (triangleCount) *triangleCount = uint32_t(ix.size() / 3);
  if (blasOffset) *blasOffset = s.tlasVec4 + s.blasOffsets[mesh];
  if (blasVec4) *blasVec4 = uint32_t(s.blases[mesh].buffer.size() / 4);
  if (bins) *bins = s.blasBins;
  if (positions) std::memcpy(positions, p.data(), p.size() * 4);
  if (indices) std::memcpy(indices, ix.data(), ix.size() * 4);
  return MT_OK;
}

int mtp_refit_blas(float *bvh, uint64_t vec4Count, const float *positions, uint32_t vertexCount, double *area) {
  if (!bvh || vec4Count < 2 || (vertexCount && !positions)) return MT_ERROR_INVALID_ARGUMENT;
  try {
    double a = refitBlasHost(bvh, size_t(vec4Count), positions, vertexCount);
    if (area) *area = a;
  } catch (const std::exception &) {
    return MT_ERROR_INVALID_ARGUMENT;
  }
  return MT_OK;
}

int mtp_light_alias_table(const double *weights, uint32_t n, uint32_t *words, float *pmfs, double *total) {
  if (!weights || !words || !n) return MT_ERROR_INVALID_ARGUMENT;
  std::vector<int> types(n, MTC_CHOICE_ANALYTIC), indices(n);
  for (uint32_t i = 0; i < n; i++) indices[i] = int(i);
  AliasTable t = buildAlias(types, indices, std::vector<double>(weights, weights + n));
  std::memcpy(words, t.words.data(), std::min<size_t>(t.words.size(), size_t(n) * 4) * 4);
  if (pmfs) for (uint32_t i = 0; i < n && i < t.pmfs.size(); i++) pmfs[i] = t.pmfs[i];
  if (total) *total = t.total;
  return MT_OK;
}

double mtp_light_power(int type, const float *color, float intensity, float area, float radius) {
  LightDesc L;
  L.type = type;
  for (int c = 0; c < 3; c++) L.color[c] = color ? color[c] : 1.0f;
  L.intensity = intensity;
  L.area = area;
  L.radius = radius;
  return lightPower(L);
}

int mtp_energy_lut(float *out) {
  if (!out) return MT_ERROR_INVALID_ARGUMENT;
  std::vector<float> lut;
  buildEnergyLut(lut);
  std::memcpy(out, lut.data(), lut.size() * 4);
  return MT_OK;
}

int mtp_env_distribution(const float *image, uint32_t width, uint32_t height, float *distribution, double *power) {
  if (!image || !width || !height || !distribution) return MT_ERROR_INVALID_ARGUMENT;
  Environment env;
  env.width = width;
  env.height = height;
  env.image.assign(image, image + size_t(width) * height * 4);
  buildEnvDistribution(env);
  std::memcpy(distribution, env.distribution.data(), env.distribution.size() * 4);
  if (power) *power = env.power;
  return MT_OK;
}

}  // extern "C"
