// Host-side producers of the flattened buffers the megakernel consumes:
// binned-SAH BVH2 (src/renderer/binnedSahBvh.ts), BLAS/TLAS packing and
// instance records (src/renderer/bvhAccel.ts), analytic-light packing and
// Walker alias table (src/renderer/wgpuSceneUniform.ts,
// src/renderer/lightSampling.ts), the environment CDF
// (src/renderer/envMapDistribution.ts), the 26-row material layout
// (src/renderer/materialLayoutSchema.ts), plus the seeded synthetic scene
// generators used by the benchmark and tests.
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include "../../include/mutracer_b200.h"

namespace mtp {

struct BinnedBvh {
  uint32_t nodeCount = 0;
  std::vector<float> bounds;        // 6 per node
  std::vector<uint32_t> leftFirst;  // interior: left child; leaf: first prim slot
  std::vector<uint32_t> primCount;  // 0 for interior nodes
  std::vector<uint32_t> primIndices;
};
BinnedBvh buildBinnedSahBvh(const float *aabbs, uint32_t count, int bins);

struct Bvh2Layout {
  std::vector<uint32_t> order, offsets;
  uint32_t vec4Count = 0, maxDepth = 0, maxLeafPrimitives = 0;
};
Bvh2Layout layoutBvh2(const BinnedBvh &bvh);

struct Blas {
  std::vector<float> buffer;  // vec4 words (floats; ints bit-cast)
  uint32_t maxDepth = 0;
  uint32_t vertexCount = 0;
  float localBounds[6] = {0, 0, 0, 0, 0, 0};
};
// positions: f32 xyz per vertex; indices: 3 per triangle.
Blas buildBlas(const std::vector<float> &positions, const std::vector<uint32_t> &indices, int bins);

struct Instance {
  uint32_t blasIndex = 0;
  double transform[16];  // column-major local-to-world
  int32_t material = 0;  // packed (index << 8) | 255
  float color[3] = {1, 1, 1};
};

struct Tlas {
  std::vector<float> buffer;     // TLAS vec4 words
  std::vector<float> instances;  // 40 floats per instance record, leaf order
  uint32_t maxDepth = 0;
};
void computeInstanceBounds(const Instance &ins, const float local[6], float out[6]);
Tlas buildTlas(const std::vector<Instance> &instances, const std::vector<Blas> &blases,
               const std::vector<uint32_t> &blasOffsets, const std::vector<uint32_t> &vertexOffsets, int bins);
void writeInstanceRecord(float *record, const Instance &ins, uint32_t blasOffset, uint32_t vertexOffset,
                         uint32_t blasLayout = 0);
bool invert4(const double *a, double *out);

// Full TLAS refit on the host (bvhAccel.ts:579-740 without a dirty set);
// the oracle of the device refit kernel.
void refitTlasHost(float *tlas, float *records, const std::vector<Instance> &instances,
                   const std::vector<Blas> &blases, const std::vector<uint32_t> &blasOffsets,
                   const std::vector<uint32_t> &vertexOffsets, uint32_t blasLayout = 0);

// Texture slots of a material (MATERIAL_TEXTURE_NAMES, materialTextureNames.ts:3-8).
enum MapSlot {
  kMapBase, kMapAlpha, kMapNormal, kMapEmissive, kMapMetallicRoughness, kMapRoughness, kMapMetalness,
  kMapTransmission, kMapThinFilm, kMapDisplacement, kMapCoatWeight, kMapCoatRoughness, kMapFuzzColor,
  kMapFuzzRoughness, kMapSpecularWeight, kMapSpecularColor, kMapAnisotropy, kMapCoatNormal, kMapSlots
};

struct MaterialDesc {
  float baseColor[3] = {0.8f, 0.8f, 0.8f};
  float baseWeight = 1.0f, baseMetalness = 0.0f, diffuseRoughness = 0.0f;
  float specularWeight = 1.0f, specularRoughness = 0.3f, specularIor = 1.5f, specularAnisotropy = 0.0f;
  float specularColor[3] = {1, 1, 1};
  float transmissionWeight = 0.0f, transmissionColor[3] = {1, 1, 1};
  float dispersionScale = 0.0f, abbe = 20.0f;
  float coatWeight = 0.0f, coatColor[3] = {1, 1, 1}, coatRoughness = 0.0f, coatIor = 1.6f, coatDarkening = 1.0f;
  float fuzzWeight = 0.0f, fuzzColor[3] = {1, 1, 1}, fuzzRoughness = 0.5f;
  float subsurfaceWeight = 0.0f, subsurfaceColor[3] = {0.8f, 0.8f, 0.8f};
  float thinFilmWeight = 0.0f, thinFilmThickness = 0.5f, thinFilmIor = 1.4f;
  float emission[3] = {0, 0, 0};
  float mediumExtinction[3] = {0, 0, 0}, mediumScattering[3] = {0, 0, 0}, mediumAnisotropy = 0.0f;
  bool thin = false, doubleSided = false;
  int type = 0;
  // Material maps: indices into SceneHost::maps (-1 none) per slot, in the
  // reference's slot order (materialTextureNames.ts).
  int maps[kMapSlots] = {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1};
  float normalScale[2] = {1, 1};
  float uvScale[2] = {1, 1};     // uvProjectionScale: multiplies the interpolated UV
  int uvProjection = 0;          // uvProjectionConstants: 0 none, 1 spherical, 2 cylindrical, 3 triplanar
  int mapAlphaUsage = 0;         // mapAlphaUsageConstants: 0 opaque, 2 alpha, 3 transmission
  float thinFilmThicknessMinimum = 0.0f;
  int thinFilmMapChannel = 0;    // r, g, b, a
  float opacity = 1.0f, alphaCutoff = 0.0f;
  int alphaMode = 0;             // materialAlphaModeConstants: 0 opaque, 1 mask, 2 blend
};
void packMaterial(const MaterialDesc &m, float rows[MTC_MATERIAL_VEC4_ROWS * 4]);

struct LightDesc {
  int type = MTC_LIGHT_RECT;
  float position[3] = {0, 0, 0};
  float color[3] = {1, 1, 1};
  float intensity = 1.0f;
  float u[3] = {1, 0, 0}, v[3] = {0, 0, 1};  // rect: full edge vectors; disk: frame * radius
  float radius = 0.0f, spread = 1.0f, area = 1.0f;
  float frameX[3] = {1, 0, 0};
  // Rows packed by the caller (every analytic type, wgpuSceneUniform.ts:70-152)
  // and their selection power; assembleScene then only writes the PMF word.
  bool packed = false;
  float rows[24] = {};
  double power = 0.0;
};

// estimateAnalyticLightPower (lightSampling.ts): luminance x intensity x
// emitting area x pi (4 pi for delta emitters).
double lightPower(const LightDesc &L);
// buildLightAliasTable (lightSampling.ts:172-212): 16-byte texels
// (probability f32, alias i32, source type, source index), f32 PMFs, total.
struct AliasTable {
  std::vector<uint32_t> words;  // 4 per choice
  std::vector<float> pmfs;
  double total = 0.0;
};
AliasTable buildAlias(const std::vector<int> &types, const std::vector<int> &indices, const std::vector<double> &weights);

// Environment: RGBA32F image + RG32F distribution + power estimate.
struct Environment {
  uint32_t width = 0, height = 0;
  std::vector<float> image, distribution;
  double power = 0.0;
};
void buildEnvDistribution(Environment &env);
void makeAnalyticSky(Environment &env, uint32_t width, uint32_t height, uint64_t seed);

// Energy-compensation tables in the 32 x 2177 layout of
// decodeOpenPbrEnergyLut.ts, tabulated by this build's own quadrature.
void buildEnergyLut(std::vector<float> &lut);

// One emissive triangle of the light-sampling table (lightSampling.ts
// collectEmissiveTriangles :237-321, packEmissiveTriangles :329-348): world
// corners (f32), area and sampling luminance (float64), material index.
struct EmissiveTriangle {
  float p[9];
  float uv[6] = {0, 0, 0, 0, 0, 0};   // corner UVs
  float uv1[6] = {0, 0, 0, 0, 0, 0};  // corner secondary UVs (the primary ones without a secondary set)
  double area = 0.0, luminance = 0.0;
  int32_t material = 0;
};

struct SceneHost {
  uint32_t width = 0, height = 0, flags = 0;
  // Emissive triangles sampled by next-event estimation; assembleScene packs
  // them ahead of the light choices (sceneAssembly.ts:42-84).
  std::vector<EmissiveTriangle> emissive;
  std::vector<float> bvh;            // TLAS then BLASes
  std::vector<float> instances;      // 40 floats per record
  std::vector<uint32_t> attributes;  // compact vertex words
  mtc_vertex_layout layout{4, 3, 0, 0};
  std::vector<float> materials;
  std::vector<float> lights;         // 24 floats per light
  std::vector<uint32_t> triangleMaterials;  // material + 1 per bvh vec4, or empty
  std::vector<std::vector<int32_t>> sourceVertexMaterials;  // per BLAS (MeshData::vertexMaterials)
  std::vector<float> maps;           // MTC_MAP_VEC4_ROWS * 4 floats per map
  std::vector<float> mapTexels;      // RGBA f32 per texel, maps back to back
  std::vector<float> lightSampling;  // RGBA32F texels
  std::vector<float> lut;
  Environment env;
  uint32_t tlasStack = 1, blasStack = 1, tlasVec4 = 0;
  mtc_camera_uniform camera{};
  mtc_trace_uniform uniform{};
  // Source data kept for refit and tests.
  std::vector<Blas> blases;
  std::vector<Instance> sourceInstances;
  std::vector<uint32_t> blasOffsets, vertexOffsets;
  std::vector<std::vector<float>> sourcePositions;     // per BLAS: xyz f32 per vertex
  std::vector<std::vector<uint32_t>> sourceIndices;    // per BLAS: 3 per triangle
  uint32_t blasBins = 8;
  uint32_t blasLayout = 0;  // BLAS layout code of every instance (0 BVH2, 2 BVH_GPU)
  uint64_t triangleCount = 0, uniqueTriangleCount = 0;
  std::string name;
};

// Re-encodes every BLAS of an assembled scene in the given layout code
// (0: BVH2 of bvhAccel.ts:248-275; 2: the two-children-per-node BVH_GPU
// layout that intersect.wgsl.ts:453-497 traverses) and rewrites the TLAS leaf
// records and instance records that point at them.  Same tree, same child
// order: a ray visits the same nodes in the same order in either layout.
void setBlasLayout(SceneHost &s, uint32_t layout);
// A layout-0 BLAS buffer (vec4 words, offsets relative to its start) in the
// BVH_GPU layout: 4 vec4 per node, (left min, left index) (left max, right
// index) (right min, leaf count) (right max, first record), node k at vec4
// 4k, leaf primitive records after the nodes.
std::vector<float> blasToGpuLayout(const std::vector<float> &bvh2);
// packTriangleMaterials (compactVertices.ts:93-102) over every BLAS of `s`:
// for each vec4 of a BLAS whose first word, read as a vertex index, lies
// inside the BLAS's vertices, that vertex's material + 1 (the triangle
// records; other vec4s are never read).  Empty when no BLAS has per-vertex
// materials.
void buildTrianglePlane(SceneHost &s);
// refitBLAS (bvhAccel.ts:800-870) on a layout-0 BLAS in place; returns the
// summed node surface area in post order.  Throws on offsets that leave the
// buffer or break the depth-first order.
double refitBlasHost(float *bvh, size_t vec4, const float *positions, uint32_t vertexCount);

struct CameraDesc {
  double eye[3], target[3], up[3];
  double fovYDeg;
  double aperture = 0.0, focus = 1.0;
};
void setCamera(SceneHost &s, const CameraDesc &c);
void defaultUniform(SceneHost &s, uint32_t bounces, uint32_t candidates, uint32_t seed, int pattern);

// Assemble buffers from meshes, instances, materials and lights.
struct MeshData {
  std::vector<float> positions, normals;
  std::vector<uint32_t> indices;
  std::vector<float> uvs;  // 2 per vertex, or empty (zero UVs when another mesh has some)
  std::vector<float> uv1s;  // secondary set, 2 per vertex, or empty (the primary set stands in)
  std::vector<float> colors;  // 3 per vertex, or empty (white when another mesh has some)
  // Global material index per vertex (a triangle takes its first vertex's),
  // or empty: every triangle uses its instance's material.
  std::vector<int32_t> vertexMaterials;
};
void assembleScene(SceneHost &s, const std::vector<MeshData> &meshes, const std::vector<Instance> &instances,
                   const std::vector<MaterialDesc> &materials, const std::vector<LightDesc> &lights, int blasBins,
                   int tlasBins, bool normalFloat);

// Scene descriptor v8 (mt_context_commit's input) decoded into `s`: MT_OK,
// or the status of a rejected descriptor with `message` naming the problem.
int32_t decodeSceneDescriptor(const uint8_t *bytes, size_t length, SceneHost &s, std::string &message);

// Synthetic workloads.
void makeCornell(SceneHost &s, uint32_t width, uint32_t height, uint64_t seed);
void makeInstancedSpheres(SceneHost &s, uint32_t width, uint32_t height, uint64_t seed, uint32_t instances,
                          uint32_t baseMeshes, uint32_t frequency, uint32_t envWidth, uint32_t rectLights);
void makeGlassSpheres(SceneHost &s, uint32_t width, uint32_t height, uint64_t seed, uint32_t spheres);

}  // namespace mtp
