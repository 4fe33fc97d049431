// Test infrastructure only (the checker, never the product).
//
// CPU restatement of MuTracer's WGSL path-tracing megakernel.  Each function
// cites the reference file:line it follows; paths are relative to the
// reference project root.  Compiled with g++ -O2 -ffp-contract=off so every
// f32 product and sum is rounded as the WGSL source states it.
#pragma once
#include "om.h"
#include "../include/mutracer_b200.h"

namespace oracle {
using namespace om;

// Per-ray traversal counters used for the algorithmic-bytes figure.
struct Traffic {
  uint64_t box_tests = 0, prim_records = 0, tri_tests = 0, instance_visits = 0,
           material_fetches = 0, paths = 0, extension_rays = 0, shadow_rays = 0;
  void add(const Traffic &o) {
    box_tests += o.box_tests; prim_records += o.prim_records; tri_tests += o.tri_tests;
    instance_visits += o.instance_visits; material_fetches += o.material_fetches;
    paths += o.paths; extension_rays += o.extension_rays; shadow_rays += o.shadow_rays;
  }
};

// Host view over the bind groups (same layout as mtc_scene_view).
struct Scene {
  const V4 *bvh = nullptr;
  const V4 *ins = nullptr;
  const u32 *attr = nullptr;
  const V4 *mats = nullptr;
  const V4 *env = nullptr;
  const float *envDist = nullptr;  // RG32F
  u32 envW = 0, envH = 0;
  const V4 *lightData = nullptr;
  const float *lut = nullptr;
  const V4 *lights = nullptr;
  // Material maps: MTC_MAP_VEC4_ROWS vec4 per map, texels RGBA f32.
  const V4 *maps = nullptr, *mapTexels = nullptr;
  u32 mapCount = 0, mapTexelCount = 0;
  const u32 *triMats = nullptr;  // triangle material plane (material + 1 per bvh vec4), or null
  u32 matCount = 0;
  mtc_vertex_layout vl{};
  u32 flags = 0;
  u32 tlasStack = 64, blasStack = 64;
  const mtc_trace_uniform *u = nullptr;
  const mtc_camera_uniform *cam = nullptr;
  bool feature(u32 bit) const { return (u->scene_feature_flags & bit) != 0; }
  bool useEnvmap() const { return feature(MTC_FEATURE_USE_ENVMAP) && env != nullptr; }
};

struct Ray { V3 o, d; };

struct SurfaceInteraction {
  V3 position{}; bool albedoSampled = false;
  V3 normal{}, vertexNormal{}, shadowOffset{}, faceNormal{}; bool hit = false;
  V3 tangent{}, directionTangent{}, directionBitangent{}, geometryTangent{}, geometryBitangent{};
  V2 uv{}, uv1{}; V3 vertexColor{};
  i32 triangleIndex = 0, instanceIndex = 0, materialIndex = 0; V2 barycentrics{};
  float wavelength = 0; i32 spectralChannel = 0;
  i32 mediumType = 0; V3 mediumExtinction{}, mediumScattering{}; float mediumAnisotropy = 0;
};

struct FirstHit { bool hit; i32 instance, record; float t; V3 bary; };

// Sampler state of sobol.wgsl.ts:18-22 and rand.wgsl.ts:6-23.
struct Sampler {
  u32 px = 0, py = 0, width = 0, index = 0, bounce = 0, hashed = 0, seed = 0, logspp = 0;
  int pattern = 0;
  u32 s0[4] = {0, 0, 0, 0};
  V2 structured(u32 dim);
  float s1(u32 dim);
  V2 s2(u32 dim);
  float hashedSample(u32 slot);
  float lightCandidateRandom(u32 salt);
  float rnd();
  u32 bounceDim(u32 slot) const { return 3u + 8u + bounce * 64u + slot; }
  u32 lightDim(u32 candidate, u32 slot) const;
};

// Sampler primitives (sobol.wgsl.ts:23-71), exported for the golden tests.
u32 sampleHash(u32 x);
u32 sampleSeed(u32 a, u32 b);
u32 lkPermute(u32 v, u32 seed);
u32 reverseBits(u32 x);
u32 owen(u32 x, u32 seed);
u32 sobolD1(u32 v);
u32 zSobolIndex(u32 morton, u32 dim, u32 logSPP);
u32 morton2(u32 x, u32 y);

// sampleMap (materialBuffer.wgsl.ts:335-367): bilinear footprint of texel
// wrapped(uv * scale + offset) * size - 0.5 with repeat or clamped texel
// coordinates; zero for an index or texel range outside the scene's maps.
V4 sampleMap(const Scene &s, i32 idx, V2 uv);
// A material's map index names a map of this scene (an index past the map
// table, like -1, means no map).
bool mapValid(const Scene &s, float index);
// decodeMapColor (materialBuffer.wgsl.ts:270-278).
V3 decodeMapColor(const Scene &s, i32 idx, V3 c);

// Traversal (intersect.wgsl.ts:213-629, 660-684, 696-740, 829-879).
FirstHit querySceneSoftware(const Scene &s, const Ray &r, Traffic *tr);
bool intersectScene(const Scene &s, const Ray &r, SurfaceInteraction &si, int bounces,
                    bool doubleSided, Traffic *tr);
// With a sampler, scenes with alpha (MTC_SCENE_HAS_ALPHA) test each
// candidate's coverage (intersectionAlphaPasses), drawing from it.
bool intersectSceneShadow(const Scene &s, const Ray &r, float lightDistance, i32 tri, i32 ins,
                          Traffic *tr, Sampler *smp = nullptr);

// One path sample for pixel (x, y): rayTrace.compute.ts:1157-1263.
void tracePixel(const Scene &s, u32 x, u32 y, V4 *outColor, V4 *outNormal, V4 *outAlbedo,
                V4 *outCatcher, Traffic *tr);

}  // namespace oracle
