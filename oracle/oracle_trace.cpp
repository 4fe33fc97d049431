// Test infrastructure only (the checker, never the product).
//
// Sampler and two-level traversal of the CPU oracle.
#include "oracle_core.h"

namespace oracle {

// ---------------------------------------------------------------- sampler
// src/renderer/wgsl/chunks/sobol.wgsl.ts:23-26
u32 sampleHash(u32 x) {
  x ^= x >> 16; x *= 0x7feb352du;
  x ^= x >> 15; x *= 0x846ca68bu;
  return x ^ (x >> 16);
}
// sobol.wgsl.ts:28-30
u32 sampleSeed(u32 a, u32 b) { return sampleHash(a ^ sampleHash(b + 0x9e3779b9u)); }
// sobol.wgsl.ts:31-36 (Laine-Karras style permutation)
u32 lkPermute(u32 v, u32 seed) {
  u32 x = v + seed;
  x ^= x * 0x6c50b47cu; x ^= x * 0xb82f1e52u;
  x ^= x * 0xc7afe638u; x ^= x * 0x8d22f6e6u;
  return x;
}
u32 reverseBits(u32 x) {
  x = ((x & 0x55555555u) << 1) | ((x >> 1) & 0x55555555u);
  x = ((x & 0x33333333u) << 2) | ((x >> 2) & 0x33333333u);
  x = ((x & 0x0f0f0f0fu) << 4) | ((x >> 4) & 0x0f0f0f0fu);
  x = ((x & 0x00ff00ffu) << 8) | ((x >> 8) & 0x00ff00ffu);
  return (x << 16) | (x >> 16);
}
// sobol.wgsl.ts:37-39
u32 owen(u32 x, u32 seed) { return reverseBits(lkPermute(reverseBits(x), seed)); }
// sobol.wgsl.ts:41-45 with the steps of src/renderer/sampling.ts:31-34
u32 sobolD1(u32 v) {
  u32 r = reverseBits(v);
  r ^= (r << 1) & 0xaaaaaaaau;
  r ^= (r << 2) & 0xccccccccu;
  r ^= (r << 4) & 0xf0f0f0f0u;
  r ^= (r << 8) & 0xff00ff00u;
  r ^= (r << 16) & 0xffff0000u;
  return r;
}
// sobol.wgsl.ts:52-58
u32 morton2(u32 x, u32 y) {
  u32 vx = x & 255u, vy = y & 255u;
  vx = (vx | (vx << 4)) & 0x0f0fu; vy = (vy | (vy << 4)) & 0x0f0fu;
  vx = (vx | (vx << 2)) & 0x3333u; vy = (vy | (vy << 2)) & 0x3333u;
  vx = (vx | (vx << 1)) & 0x5555u; vy = (vy | (vy << 1)) & 0x5555u;
  return vx | (vy << 1);
}
// pbrt-v4 ZSobol digit permutations (src/renderer/sampling.ts:16-21).
static const uint8_t kZPerm[24][4] = {
  {0,1,2,3},{0,1,3,2},{0,2,1,3},{0,2,3,1},{0,3,2,1},{0,3,1,2},
  {1,0,2,3},{1,0,3,2},{1,2,0,3},{1,2,3,0},{1,3,2,0},{1,3,0,2},
  {2,1,0,3},{2,1,3,0},{2,0,1,3},{2,0,3,1},{2,3,0,1},{2,3,1,0},
  {3,1,2,0},{3,1,0,2},{3,2,1,0},{3,2,0,1},{3,0,2,1},{3,0,1,2}};
static u32 zPerm(u32 p) {
  u32 v = 0;
  for (int i = 0; i < 4; i++) v |= u32(kZPerm[p][i]) << (2 * i);
  return v;
}
// sobol.wgsl.ts:66-83
u32 zSobolIndex(u32 morton, u32 dim, u32 logSPP) {
  u32 odd = logSPP & 1u;
  u32 digits = 8u + ((logSPP + 1u) >> 1);
  u32 result = 0;
  for (int digit = int(digits) - 1; digit >= int(odd); digit--) {
    u32 shift = 2u * u32(digit) - odd;
    u32 higher = 0;
    if (shift < 30u) higher = morton >> (shift + 2u);
    u32 perm = (sampleHash(higher ^ (0x55555555u * dim)) >> 24) % 24u;
    u32 d = (morton >> shift) & 3u;
    result |= ((zPerm(perm) >> (2u * d)) & 3u) << shift;
  }
  if (odd != 0u) result |= (morton & 1u) ^ (sampleHash((morton >> 1) ^ (0x55555555u * dim)) & 1u);
  return result;
}
// sobol.wgsl.ts:98-133 (prepareStructuredSample + structuredSample, no cache)
V2 Sampler::structured(u32 dim) {
  u32 pixelID = px + py * width;
  u32 sd = sampleSeed(sampleSeed(pixelID, dim), seed);
  u32 idx = index;
  if (pattern == 1) {
    u32 log = logspp;
    if (idx == 0u) log = 0u; else idx -= 1u;
    u32 block = idx >> log;
    u32 mask = (1u << log) - 1u;
    u32 morton = (morton2(px, py) << log) | (idx & mask);
    idx = zSobolIndex(morton, dim, log);
    sd = sampleSeed(sampleSeed(dim, seed), sampleSeed(px >> 8, py >> 8));
    if (index != 0u) block += 1u;
    sd = sampleSeed(sd, block);
  }
  u32 i = owen(idx, sampleSeed(sd, 0u));
  u32 x = reverseBits(lkPermute(i, sampleSeed(sd, 1u)));
  u32 y = owen(sobolD1(i), sampleSeed(sd, 2u));
  float fx = float(x >> 8) * (1.0f / 16777216.0f);
  float fy = float(y >> 8) * (1.0f / 16777216.0f);
  return {EPS + 0.999f * fx, EPS + 0.999f * fy};
}
// rand.wgsl.ts:12-23
float Sampler::rnd() {
  for (int k = 0; k < 4; k++) s0[k] = s0[k] * 1664525u + 1013904223u;
  s0[0] += s0[1] * s0[3]; s0[1] += s0[2] * s0[0]; s0[2] += s0[0] * s0[1]; s0[3] += s0[1] * s0[2];
  for (int k = 0; k < 4; k++) s0[k] = s0[k] ^ (s0[k] >> 16);
  s0[0] += s0[1] * s0[3]; s0[1] += s0[2] * s0[0]; s0[2] += s0[0] * s0[1]; s0[3] += s0[1] * s0[2];
  return float(s0[0]) / float(0xffffffffu);
}
// sobol.wgsl.ts:134-145
float Sampler::s1(u32 dim) {
  if (pattern == 2) return EPS + 0.999f * rnd();
  return structured(dim).x;
}
V2 Sampler::s2(u32 dim) {
  if (pattern == 2) { float a = s1(dim); float b = s1(dim); return {a, b}; }
  return structured(dim);
}
// sobol.wgsl.ts:147-157
float Sampler::hashedSample(u32 slot) {
  u32 dim = sampleSeed(sampleSeed(bounce, slot), hashed) | 0x80000000u;
  hashed += 1u;
  if (pattern == 2) return EPS + 0.999f * rnd();
  u32 pixelID = px + py * width;
  u32 sd = sampleSeed(sampleSeed(pixelID, dim), seed);
  u32 i = owen(index, sampleSeed(sd, 0u));
  u32 x = reverseBits(lkPermute(i, sampleSeed(sd, 1u)));
  return EPS + 0.999f * (float(x >> 8) * (1.0f / 16777216.0f));
}
// rayTrace.compute.ts:251-262
float Sampler::lightCandidateRandom(u32 salt) {
  if (pattern == 2) (void)rnd();
  u32 pixelID = px + py * width;
  u32 key = sampleSeed(sampleSeed(pixelID, index), seed);
  u32 dimension = sampleSeed(bounce, salt) ^ 0xa511e9b3u;
  return float(sampleHash(key ^ dimension) >> 8) * (1.0f / 16777216.0f);
}
// sobol.wgsl.ts:88-94
u32 Sampler::lightDim(u32 candidate, u32 slot) const {
  if (candidate == 0u) {
    if (slot == 2u) return bounceDim(8u);
    return bounceDim(slot);
  }
  return bounceDim(9u + (candidate - 1u) * 3u + slot);
}

// -------------------------------------------------------------- traversal
// intersect.wgsl.ts:1500-1521
static inline V3 traversalInverse(V3 d) { return {1.0f / d.x, 1.0f / d.y, 1.0f / d.z}; }
static inline float intersectBox(V3 o, V3 bmin, V3 bmax, V3 invD, float tMax) {
  V3 tBot = (bmin - o) * invD;
  V3 tTop = (bmax - o) * invD;
  V3 tNear = vmin(tBot, tTop);
  V3 tFar = vmax(tBot, tTop);
  float t0 = fmaxf(tNear.x, fmaxf(tNear.y, tNear.z));
  float t1 = fminf(tFar.x, fminf(tFar.y, tFar.z));
  if (t0 > t1 || t0 > tMax) return -1.0f;
  return t0 > 0.0f ? t0 : t1;
}
// intersect.wgsl.ts:1523-1537
static inline int maxDimension(V3 v) {
  if (v.x > v.y) return v.x > v.z ? 0 : 2;
  return v.y > v.z ? 1 : 2;
}
static inline V3 getShear(V3 d, int maxDim) {
  if (maxDim == 0) return {-d.y / d.x, -d.z / d.x, 1.0f / d.x};
  if (maxDim == 1) return {-d.z / d.y, -d.x / d.y, 1.0f / d.y};
  return {-d.x / d.z, -d.y / d.z, 1.0f / d.z};
}
struct TriHit { float t; V3 bary; };
// intersect.wgsl.ts:1430-1493 (pbrt-v3 watertight test, DEPTH_QUERY_MODE off)
static inline TriHit intersectTriangle(V3 o, V3 p0, V3 p1, V3 p2, int maxDim, V3 shear, float tMax) {
  TriHit ti{0.0f, {0, 0, 0}};
  V3 p0t = p0 - o, p1t = p1 - o, p2t = p2 - o;
  if (maxDim == 0) {
    p0t = {p0t.y, p0t.z, p0t.x}; p1t = {p1t.y, p1t.z, p1t.x}; p2t = {p2t.y, p2t.z, p2t.x};
  } else if (maxDim == 1) {
    p0t = {p0t.z, p0t.x, p0t.y}; p1t = {p1t.z, p1t.x, p1t.y}; p2t = {p2t.z, p2t.x, p2t.y};
  }
  p0t.x = p0t.x + shear.x * p0t.z; p0t.y = p0t.y + shear.y * p0t.z;
  p1t.x = p1t.x + shear.x * p1t.z; p1t.y = p1t.y + shear.y * p1t.z;
  p2t.x = p2t.x + shear.x * p2t.z; p2t.y = p2t.y + shear.y * p2t.z;
  V3 e = {p1t.x * p2t.y - p1t.y * p2t.x, p2t.x * p0t.y - p2t.y * p0t.x, p0t.x * p1t.y - p0t.y * p1t.x};
  bool anyNeg = e.x < 0.0f || e.y < 0.0f || e.z < 0.0f;
  bool anyPos = e.x > 0.0f || e.y > 0.0f || e.z > 0.0f;
  if (anyNeg && anyPos) return ti;
  float det = e.x + e.y + e.z;
  p0t.z *= shear.z; p1t.z *= shear.z; p2t.z *= shear.z;
  float tScaled = e.x * p0t.z + e.y * p1t.z + e.z * p2t.z;
  if (std::fabs(tScaled) > std::fabs(tMax * det)) return ti;
  float invDet = 1.0f / det;
  ti.t = tScaled * invDet;
  ti.bary = e * invDet;
  return ti;
}

// ------------------------------------------------------------ material maps
// wrapMapCoordinate (materialBuffer.wgsl.ts:316-320): 0 repeat, 1 clamp,
// 2 mirrored repeat.
static float wrapMapCoordinate(float v, float mode) {
  if (mode < 0.5f) return v - std::floor(v);
  if (mode < 1.5f) return clampf(v, 0.0f, 1.0f);
  return 1.0f - std::fabs(1.0f - (v - 2.0f * std::floor(v * 0.5f)));
}

// sampleMap + loadMapTexel (materialBuffer.wgsl.ts:335-378).  The shader
// filters footprints that stay inside the image in hardware and the repeat
// footprints that cross its edge by hand; both are the bilinear mix of the
// four texels around wrapped * size - 0.5 with clamped (or, for repeat,
// modular) texel coordinates, which is what this evaluates everywhere.
V4 sampleMap(const Scene &s, i32 idx, V2 uv) {
  if (idx < 0 || u32(idx) >= s.mapCount) return {0, 0, 0, 0};
  const V4 *mi = s.maps + size_t(idx) * MTC_MAP_VEC4_ROWS;
  const i32 w = asi(mi[0].x), h = asi(mi[0].y);
  const u32 first = asu(mi[0].z);
  if (w < 1 || h < 1 || uint64_t(first) + uint64_t(w) * uint64_t(h) > s.mapTexelCount) return {0, 0, 0, 0};
  const V4 t = mi[1], modes = mi[2];
  const float tx = wrapMapCoordinate(uv.x * t.x + t.z, modes.z) * float(w) - 0.5f;
  const float ty = wrapMapCoordinate(uv.y * t.y + t.w, modes.w) * float(h) - 0.5f;
  const float fx = std::floor(tx), fy = std::floor(ty), wx = tx - fx, wy = ty - fy;
  // Finite coordinates wrap into [-1, size - 1]; the clamp only pins NaN.
  const i32 bx = i32(fminf(fmaxf(fx, -1.0f), float(w))), by = i32(fminf(fmaxf(fy, -1.0f), float(h)));
  auto load = [&](i32 x, i32 y) {
    i32 px = std::min(std::max(x, 0), w - 1), py = std::min(std::max(y, 0), h - 1);
    if (modes.z < 0.5f) px = ((x % w) + w) % w;
    if (modes.w < 0.5f) py = ((y % h) + h) % h;
    return s.mapTexels[first + size_t(py) * size_t(w) + size_t(px)];
  };
  auto mix = [](V4 a, V4 b, float k) {
    return V4{a.x * (1.0f - k) + b.x * k, a.y * (1.0f - k) + b.y * k, a.z * (1.0f - k) + b.z * k,
              a.w * (1.0f - k) + b.w * k};
  };
  return mix(mix(load(bx, by), load(bx + 1, by), wx), mix(load(bx, by + 1), load(bx + 1, by + 1), wx), wy);
}

bool mapValid(const Scene &s, float index) { return index >= 0.0f && index < float(s.mapCount); }

// sRGBToLinear / decodeMapColor (materialBuffer.wgsl.ts:266-278).
static float srgbToLinear(float c) {
  return c < 0.04045f ? c * 0.0773993808f : std::pow(c * 0.9478672986f + 0.0521327014f, 2.4f);
}
V3 decodeMapColor(const Scene &s, i32 idx, V3 c) {
  if (idx < 0 || u32(idx) >= s.mapCount) return c;
  if (i32(std::nearbyint(s.maps[size_t(idx) * MTC_MAP_VEC4_ROWS + 2].y)) % 2 == 1) return c;
  return {srgbToLinear(c.x), srgbToLinear(c.y), srgbToLinear(c.z)};
}

// getMatNormal (materialBuffer.wgsl.ts:377-418), local space.
static V3 getMatNormal(const Scene &s, i32 materialIndex, V2 uv, V3 normal, V3 dp1, V3 dp2, V2 duv1, V2 duv2) {
  const V4 *d = s.mats + size_t(materialIndex) * MTC_MATERIAL_VEC4_ROWS;
  if (!mapValid(s, d[1].y)) return normal;
  const i32 idx = i32(d[1].y);
  V3 dp2perp = cross(dp2, normal), dp1perp = cross(normal, dp1);
  V3 dpdu = dp2perp * duv1.x + dp1perp * duv2.x;
  V3 dpdv = dp2perp * duv1.y + dp1perp * duv2.y;
  float g2 = fmaxf(dot(dpdu, dpdu), dot(dpdv, dpdv));
  if (g2 > 1e-12f) {
    float invmax = 1.0f / std::sqrt(g2);
    dpdu = dpdu * invmax;
    dpdv = dpdv * invmax;
  } else {
    V3 axis = std::fabs(normal.z) < 0.999f ? V3{0, 0, 1} : V3{0, 1, 0};
    dpdu = normalize(cross(axis, normal));
    dpdv = cross(normal, dpdu);
  }
  V4 t = sampleMap(s, idx, uv);
  V3 n = {2.0f * t.x - 1.0f, 2.0f * t.y - 1.0f, 2.0f * t.z - 1.0f};
  n = normalize(V3{n.x * d[1].z, n.y * d[1].w, n.z});
  return normalize(dpdu * n.x + dpdv * n.y + normal * n.z);
}

// vertexColor (vertexAttributes.wgsl.ts:38-43): f32x3, or unpack4x8unorm of
// one RGBA8 word; white without color words.
static inline V3 vertexColor(const Scene &s, i32 i) {
  if (!s.vl.color_offset) return v3(1.0f);
  const u32 *w = s.attr + size_t(i) * s.vl.stride + s.vl.color_offset;
  if (s.vl.color_float) return {asf(w[0]), asf(w[1]), asf(w[2])};
  return {float(w[0] & 255u) / 255.0f, float((w[0] >> 8) & 255u) / 255.0f, float((w[0] >> 16) & 255u) / 255.0f};
}

static inline V2 vertexUv(const Scene &s, i32 i) {
  if (!s.vl.uv_offset) return {0, 0};
  const u32 *w = s.attr + size_t(i) * s.vl.stride + s.vl.uv_offset;
  return {asf(w[0]), asf(w[1])};
}

static inline V3 vertexPosition(const Scene &s, i32 i) {
  const u32 *w = s.attr + size_t(i) * s.vl.stride;
  return {asf(w[0]), asf(w[1]), asf(w[2])};
}
// vertexAttributes.wgsl.ts:14-28 (octDirection + vertexNormal)
static inline V3 vertexNormal(const Scene &s, i32 i) {
  const u32 *w = s.attr + size_t(i) * s.vl.stride + s.vl.normal_offset;
  if (s.vl.normal_float) return {asf(w[0]), asf(w[1]), asf(w[2])};
  u32 word = w[0];
  i32 a = i32(word << 16) >> 16;
  i32 b = i32(word) >> 16;
  if (a == -32768 && b == -32768) return v3(0.0f);
  V3 v = {float(a) / 32767.0f, float(b) / 32767.0f, 0.0f};
  v.z = 1.0f - std::fabs(v.x) - std::fabs(v.y);
  if (v.z < 0.0f) {
    float nx = (1.0f - std::fabs(v.y)) * (v.x >= 0.0f ? 1.0f : -1.0f);
    float ny = (1.0f - std::fabs(v.x)) * (v.y >= 0.0f ? 1.0f : -1.0f);
    v.x = nx; v.y = ny;
  }
  return normalize(v);
}
static inline float materialDoubleSided(const Scene &s, i32 materialIndex) {
  return s.mats[size_t(materialIndex) * MTC_MATERIAL_VEC4_ROWS + 23].z;
}
static inline i32 unpackMaterialIndex(i32 v) { return v >> 8; }

// Traversal state shared by the closest-hit, shadow and first-hit queries:
// getBVHTraverseCode, intersect.wgsl.ts:213-629 (BVH2 layout code 0).
struct TraversalHit {
  bool isHit = false;
  float tMax;
  V3 hitPosition{}, hitNormal{}, hitBary{};
  i32 triangleIndex = -1, insIdx = -1;
  i32 idx[3] = {0, 0, 0};
  V3 tri[3];
};

enum class Mode { Closest, Shadow };

// intersectionAlphaPasses (intersectionAlpha.wgsl.ts:14-90): whether a
// shadow candidate on a triangle of `materialIndex` (vertex indices `index`,
// barycentrics `bary`) occludes.
// projectUV (uvProjection.wgsl.ts): 1 spherical, 2 cylindrical, 3 triplanar.
static V2 projectUV(i32 type, V3 pos, V3 normal) {
  if (type == 3) {
    const V3 a = {std::fabs(normal.x), std::fabs(normal.y), std::fabs(normal.z)};
    if (a.x > a.y && a.x > a.z) return {pos.y, pos.z};
    if (a.y > a.x && a.y > a.z) return {pos.x, pos.z};
    return {pos.x, pos.y};
  }
  if (type == 1) {
    const V3 n = normalize(pos);
    return {std::atan2(n.x, n.z) / (2.0f * PI) + 0.5f, 1.0f - std::acos(n.y) / PI};
  }
  if (type == 2) return {std::atan2(pos.z, pos.x) / (2.0f * PI) + 0.5f, pos.y};
  return {0.0f, 0.0f};
}

// triangleMaterial (vertexAttributes.wgsl.ts:51-56): the plane's material of
// the triangle record, else the instance's (`fallback`).
static i32 triangleMaterial(const Scene &s, i32 fallback, i32 record) {
  if (!s.triMats) return fallback;
  const u32 m = s.triMats[record];
  return m && m - 1u < s.matCount ? i32(m - 1u) : fallback;
}

static bool intersectionAlphaPasses(const Scene &s, i32 initialMaterialIndex, i32 record, const i32 index[3], V3 bary,
                                    V3 hitPosition, V3 hitNormal, Sampler &smp) {
  const i32 materialIndex = triangleMaterial(s, initialMaterialIndex, record);
  const V4 *ma = s.mats + size_t(materialIndex) * MTC_MATERIAL_VEC4_ROWS;
  float alpha = ma[9].x;
  auto surfaceUv = [&]() {
    V2 uv0 = vertexUv(s, index[0]), uv1 = vertexUv(s, index[1]), uv2 = vertexUv(s, index[2]);
    V2 uv = {bary.x * uv0.x + bary.y * uv1.x + bary.z * uv2.x, bary.x * uv0.y + bary.y * uv1.y + bary.z * uv2.y};
    const i32 projection = i32(ma[7].x);
    if (projection > 0) uv = projectUV(projection, hitPosition, hitNormal);
    uv = {uv.x * ma[7].z, uv.y * ma[7].w};
    if (projection == 3) uv = {uv.x - std::floor(uv.x), uv.y - std::floor(uv.y)};
    return uv;
  };
  if (ma[5].w == 2.0f && mapValid(s, ma[2].z)) alpha *= sampleMap(s, i32(ma[2].z), surfaceUv()).w;
  if (mapValid(s, ma[22].z)) alpha *= sampleMap(s, i32(ma[22].z), surfaceUv()).y;
  const i32 alphaMode = i32(ma[23].w);
  if (alphaMode == 0) alpha = 1.0f;
  else if (alphaMode == 1) alpha = alpha >= ma[22].w ? 1.0f : 0.0f;
  if (alphaMode == 2) return smp.hashedSample(1u) <= alpha;
  return alpha >= 1.0f;
}

// Returns true when a shadow query found an occluder.  `alphaSmp`: the
// shadow hook's coverage test (intersect.wgsl.ts:846-866).
static bool traverse(const Scene &s, const Ray &ray, int bounces, bool doubleSided, i32 currentTri,
                     i32 currentIns, Mode mode, TraversalHit &h, Traffic *tr, Sampler *alphaSmp = nullptr) {
  const float shadowRayTMax = h.tMax;
  i32 tlasStack[MTC_MAX_STACK];
  i32 blasStack[MTC_MAX_STACK];
  int tlasTop = -1;
  V3 o = ray.o, d = ray.d;
  V3 invD = traversalInverse(d);
  if (tr) tr->box_tests++;
  if (intersectBox(o, xyz(s.bvh[0]), xyz(s.bvh[1]), invD, h.tMax) > 0.0f) {
    tlasTop = 0;
    tlasStack[0] = 0;
  }
  const i32 bufferOff = s.u->blas_offset;
  while (tlasTop >= 0) {
    i32 tlasNode = tlasStack[tlasTop--];
    o = ray.o; d = ray.d; invD = traversalInverse(d);
    V4 r1 = s.bvh[tlasNode];
    i32 ptr = asi(r1.w);
    if (ptr >= 0) {
      i32 left = tlasNode + 2, right = ptr;
      float d0 = intersectBox(o, xyz(s.bvh[left]), xyz(s.bvh[left + 1]), invD, h.tMax);
      float d1 = intersectBox(o, xyz(s.bvh[right]), xyz(s.bvh[right + 1]), invD, h.tMax);
      if (tr) tr->box_tests += 2;
      if (d0 > d1) {
        if (d0 > 0.0f && tlasTop + 1 < MTC_MAX_STACK) tlasStack[++tlasTop] = left;
        if (d1 > 0.0f && tlasTop + 1 < MTC_MAX_STACK) tlasStack[++tlasTop] = right;
      } else {
        if (d1 > 0.0f && tlasTop + 1 < MTC_MAX_STACK) tlasStack[++tlasTop] = right;
        if (d0 > 0.0f && tlasTop + 1 < MTC_MAX_STACK) tlasStack[++tlasTop] = left;
      }
      continue;
    }
    i32 tlasCount = -ptr;
    for (i32 io = tlasCount - 1; io >= 0; io--) {
      V4 rec = s.bvh[tlasNode + 2 + io];
      i32 insIdx = asi(rec.x);
      i32 blasRoot = asi(rec.y);
      const V4 *insv = s.ins + size_t(insIdx) * MTC_INSTANCE_VEC4_STRIDE;
      V4 insData = insv[0];
      if (tr) tr->instance_visits++;
      o = mat4_mul(insv + 1, ray.o, 1.0f);
      d = mat4_mul(insv + 1, ray.d, 0.0f);
      invD = traversalInverse(d);
      int maxDim = maxDimension(vabs(d));
      V3 shear = getShear(d, maxDim);
      u32 encoded = asu(insData.x);
      u32 layout = encoded >> 30;
      i32 blasOffset = i32(encoded & 0x3fffffffu);
      i32 vertexOffset = asi(insData.y);
      // BVH2 (code 0) and BVH_GPU (code 2) BLASes are consumed; the TinyBVH
      // bvh4 and cwbvh layouts (codes 1 and 3) are not.
      if (layout != 0u && layout != 2u) continue;
      int blasTop = 0;
      blasStack[0] = blasRoot;
      while (blasTop >= 0) {
        i32 node = blasStack[blasTop--];
        i32 i = node + bufferOff;
        i32 primitiveCount = 0, primitiveOffset = 0;
        i32 left = 0, right = 0;
        float d0 = 0.0f, d1 = 0.0f;
        bool interior;
        if (layout == 2u) {
          // intersect.wgsl.ts:453-497: both child boxes live in the node.
          V4 g0 = s.bvh[i], g1 = s.bvh[i + 1], g2 = s.bvh[i + 2], g3 = s.bvh[i + 3];
          primitiveCount = i32(asu(g2.w));
          interior = primitiveCount <= 0;
          if (!interior) {
            primitiveOffset = bufferOff + blasOffset + i32(asu(g3.w));
          } else {
            left = blasOffset + i32(asu(g0.w) * 4u);
            right = blasOffset + i32(asu(g1.w) * 4u);
            d0 = intersectBox(o, xyz(g0), xyz(g1), invD, h.tMax);
            d1 = intersectBox(o, xyz(g2), xyz(g3), invD, h.tMax);
          }
        } else {
          V4 n1 = s.bvh[i];
          i32 p = asi(n1.w);
          interior = p >= 0;
          if (interior) {
            left = node + 2;
            right = p + blasOffset;
            d0 = intersectBox(o, xyz(s.bvh[left + bufferOff]), xyz(s.bvh[left + 1 + bufferOff]), invD, h.tMax);
            d1 = intersectBox(o, xyz(s.bvh[right + bufferOff]), xyz(s.bvh[right + 1 + bufferOff]), invD, h.tMax);
          } else {
            primitiveCount = -p;
            primitiveOffset = i + 2;
          }
        }
        if (interior) {
          if (tr) tr->box_tests += 2;
          if (d0 > d1) {
            if (d0 > 0.0f && blasTop + 1 < MTC_MAX_STACK) blasStack[++blasTop] = left;
            if (d1 > 0.0f && blasTop + 1 < MTC_MAX_STACK) blasStack[++blasTop] = right;
          } else {
            if (d1 > 0.0f && blasTop + 1 < MTC_MAX_STACK) blasStack[++blasTop] = right;
            if (d0 > 0.0f && blasTop + 1 < MTC_MAX_STACK) blasStack[++blasTop] = left;
          }
          continue;
        }
        for (i32 k = 0; k < primitiveCount; k++) {
          i32 triangleIndex = primitiveOffset + k;
          if (bounces > 0 && triangleIndex == currentTri && insIdx == currentIns) continue;
          V4 r3 = s.bvh[triangleIndex];
          if (tr) { tr->prim_records++; tr->tri_tests++; }
          i32 i0 = asi(r3.x) + vertexOffset, i1 = asi(r3.y) + vertexOffset, i2 = asi(r3.z) + vertexOffset;
          V3 p0 = vertexPosition(s, i0), p1 = vertexPosition(s, i1), p2 = vertexPosition(s, i2);
          TriHit hit = intersectTriangle(o, p0, p1, p2, maxDim, shear, h.tMax);
          if (!(hit.t > 0.0f)) continue;
          V3 e1 = p1 - p0, e2 = p2 - p0;
          V3 candidateNormal = normalize(cross(e1, e2));
          i32 sideMaterial = unpackMaterialIndex(asi(insData.z));
          bool matDoubleSided = materialDoubleSided(s, sideMaterial) > 0.5f;
          if (!doubleSided && !matDoubleSided && dot(candidateNormal, d) > 0.0f) continue;
          h.hitNormal = candidateNormal;
          h.tMax = hit.t;
          h.isHit = true;
          h.hitPosition = o + d * h.tMax;
          h.hitBary = hit.bary;
          if (mode == Mode::Shadow) {
            const i32 index[3] = {i0, i1, i2};
            if (alphaSmp && !intersectionAlphaPasses(s, sideMaterial, triangleIndex, index, hit.bary, h.hitPosition,
                                                     candidateNormal, *alphaSmp)) {
              h.tMax = shadowRayTMax;  // not occluded: never traverse beyond the light
              continue;
            }
            return true;
          }
          h.triangleIndex = triangleIndex;
          h.insIdx = insIdx;
          h.idx[0] = i0; h.idx[1] = i1; h.idx[2] = i2;
          h.tri[0] = p0; h.tri[1] = p1; h.tri[2] = p2;
        }
      }
    }
  }
  return false;
}

// intersect.wgsl.ts:665-684
FirstHit querySceneSoftware(const Scene &s, const Ray &r, Traffic *tr) {
  FirstHit res{false, -1, -1, RAY_MAX_DISTANCE, {0, 0, 0}};
  if (s.u->is_empty > 0) return res;
  TraversalHit h;
  h.tMax = RAY_MAX_DISTANCE;
  traverse(s, r, 0, false, -1, -1, Mode::Closest, h, tr);
  if (h.isHit) {
    res.hit = true; res.instance = h.insIdx; res.record = h.triangleIndex;
    res.t = h.tMax; res.bary = h.hitBary;
  }
  return res;
}

// intersect.wgsl.ts:1058-1087 anisotropy_axes
static void anisotropyAxes(V3 normal, V3 dp1, V3 dp2, V2 duv1, V2 duv2, V4 input, V3 &outT, V3 &outB) {
  float determinant = duv1.x * duv2.y - duv1.y * duv2.x;
  V3 t = {input.x, input.y, input.z};
  V3 b = v3(0.0f);
  float sign = std::fabs(input.w) > 1.5f ? 0.0f : input.w;
  if (std::fabs(determinant) > 1e-12f) {
    V3 dt = (dp1 * duv2.y - dp2 * duv1.y) / determinant;
    V3 db = (dp2 * duv1.x - dp1 * duv2.x) / determinant;
    if (dot(t, t) < 1e-8f) t = dt;
    if (sign == 0.0f) sign = dot(cross(normal, dt), db) < 0.0f ? -1.0f : 1.0f;
  }
  t = t - normal * dot(normal, t);
  if (dot(t, t) < 1e-8f) {
    float signZ = normal.z >= 0.0f ? 1.0f : -1.0f;
    float factor = -1.0f / (signZ + normal.z);
    float xy = normal.x * normal.y * factor;
    t = {1.0f + signZ * normal.x * normal.x * factor, signZ * xy, -signZ * normal.x};
    b = {xy, signZ + normal.y * normal.y * factor, -normal.y};
  } else {
    t = normalize(t);
    b = normalize(cross(normal, t));
  }
  outT = t;
  outB = b * (sign < 0.0f ? -1.0f : 1.0f);
}

// fetchAttributes (intersect.wgsl.ts:1233-1419) for compact vertices without
// UV/color/tangent words, followed by completeSurfaceInteraction's transforms
// (intersect.wgsl.ts:1539-1601).
static void completeSurfaceInteraction(const Scene &s, SurfaceInteraction &si, const TraversalHit &h) {
  si.instanceIndex = h.insIdx;
  si.barycentrics = {h.hitBary.x, h.hitBary.y};
  si.normal = h.hitNormal;
  si.position = h.hitPosition;
  const V4 *insv = s.ins + size_t(h.insIdx) * MTC_INSTANCE_VEC4_STRIDE;
  si.materialIndex = unpackMaterialIndex(asi(insv[0].z));
  si.hit = true;
  V3 bary = h.hitBary;
  si.vertexColor = v3(1.0f);
  if (s.vl.color_offset)
    si.vertexColor = vertexColor(s, h.idx[0]) * bary.x + vertexColor(s, h.idx[1]) * bary.y +
                     vertexColor(s, h.idx[2]) * bary.z;
  V3 n0 = vertexNormal(s, h.idx[0]), n1 = vertexNormal(s, h.idx[1]), n2 = vertexNormal(s, h.idx[2]);
  V3 normal = normalize(n0 * bary.x + n1 * bary.y + n2 * bary.z);
  const V2 uv0 = vertexUv(s, h.idx[0]), uv1 = vertexUv(s, h.idx[1]), uv2 = vertexUv(s, h.idx[2]);
  // uvScale comes from the instance's material (fetchAttributes' `material`),
  // read before the triangle's own material is resolved.
  const V4 *im = s.mats + size_t(si.materialIndex) * MTC_MATERIAL_VEC4_ROWS;
  si.materialIndex = triangleMaterial(s, si.materialIndex, h.triangleIndex);
  const V4 *dm = s.mats + size_t(si.materialIndex) * MTC_MATERIAL_VEC4_ROWS;
  V2 uv = {bary.x * uv0.x + bary.y * uv1.x + bary.z * uv2.x, bary.x * uv0.y + bary.y * uv1.y + bary.z * uv2.y};
  // vertexUv1 reads UV1_OFF, which aliases UV_OFF without secondary words
  V2 secondary = uv;
  if (s.vl.uv1_offset) {
    auto vuv1 = [&](i32 i) {
      const u32 *w = s.attr + size_t(i) * s.vl.stride + s.vl.uv1_offset;
      return V2{asf(w[0]), asf(w[1])};
    };
    const V2 a = vuv1(h.idx[0]), b = vuv1(h.idx[1]), c = vuv1(h.idx[2]);
    secondary = {bary.x * a.x + bary.y * b.x + bary.z * c.x, bary.x * a.y + bary.y * b.y + bary.z * c.y};
  }
  const i32 projection = i32(im[7].x);  // intersect.wgsl.ts:1311-1322, local position and normal
  if (projection > 0) {
    uv = projectUV(projection, si.position, normal);
    secondary = uv;
  }
  uv = {uv.x * im[7].z, uv.y * im[7].w};
  secondary = {secondary.x * im[7].z, secondary.y * im[7].w};
  if (projection == 3) uv = {uv.x - std::floor(uv.x), uv.y - std::floor(uv.y)};
  const V2 duv1 = {uv0.x - uv2.x, uv0.y - uv2.y}, duv2 = {uv1.x - uv2.x, uv1.y - uv2.y};
  if (dm[24].x >= 0.0f || dm[24].y != 0.0f || dm[25].x != 0.0f) {
    V3 dp1 = h.tri[0] - h.tri[2];
    V3 dp2 = h.tri[1] - h.tri[2];
    V3 gt, gb;
    anisotropyAxes(normal, dp1, dp2, duv1, duv2, {0, 0, 0, 0}, gt, gb);
    si.geometryTangent = gt; si.geometryBitangent = gb;
    si.directionTangent = gt; si.directionBitangent = gb;
  }
  si.normal = normal;
  si.vertexNormal = normal;
  // Cycles shadow-terminator offset (intersect.wgsl.ts:1376-1407).
  {
    const V3 &p0 = h.tri[0], &p1 = h.tri[1], &p2 = h.tri[2];
    V3 geometricNormal = normalize(cross(p1 - p0, p2 - p0));
    V3 smoothNormal = n0 * bary.x + n1 * bary.y + n2 * bary.z;
    float a = dot(n2 - n0, p0 - p2);
    float b = dot(n2 - n1, p1 - p2);
    float c = dot(n1 - n0, p1 - p0);
    float hh = a * bary.x * (bary.x - 1.0f) + (a + b + c) * bary.x * bary.y + b * bary.y * (bary.y - 1.0f);
    if (dot(smoothNormal, geometricNormal) > 0.0f) {
      float h0 = fmaxf(fmaxf(dot(p1 - p0, n0), dot(p2 - p0, n0)), 0.0f);
      float h1 = fmaxf(fmaxf(dot(p0 - p1, n1), dot(p2 - p1, n1)), 0.0f);
      float h2 = fmaxf(fmaxf(dot(p0 - p2, n2), dot(p1 - p2, n2)), 0.0f);
      h0 = fmaxf(dot(p0 - si.position, n0) + h0, 0.0f);
      h1 = fmaxf(dot(p1 - si.position, n1) + h1, 0.0f);
      h2 = fmaxf(dot(p2 - si.position, n2) + h2, 0.0f);
      hh = fmaxf(fminf(fminf(h0, h1), h2), hh * 0.5f);
    } else {
      float h0 = fmaxf(fmaxf(dot(p0 - p1, n0), dot(p0 - p2, n0)), 0.0f);
      float h1 = fmaxf(fmaxf(dot(p1 - p0, n1), dot(p1 - p2, n1)), 0.0f);
      float h2 = fmaxf(fmaxf(dot(p2 - p0, n2), dot(p2 - p1, n2)), 0.0f);
      h0 = fmaxf(dot(si.position - p0, n0) + h0, 0.0f);
      h1 = fmaxf(dot(si.position - p1, n1) + h1, 0.0f);
      h2 = fmaxf(dot(si.position - p2, n2) + h2, 0.0f);
      hh = fminf(-fminf(fminf(h0, h1), h2), hh * 0.5f);
    }
    si.shadowOffset = smoothNormal * hh;
  }
  si.uv = uv;
  si.uv1 = secondary;
  si.normal = getMatNormal(s, si.materialIndex, uv, normal, h.tri[0] - h.tri[2], h.tri[1] - h.tri[2], duv1, duv2);
  const V4 *w2l = insv + 1;
  const V4 *l2w = insv + 5;
  auto nt = [&](V3 v) { return V3{dot(xyz(w2l[0]), v), dot(xyz(w2l[1]), v), dot(xyz(w2l[2]), v)}; };
  si.faceNormal = normalize(nt(h.hitNormal));
  si.vertexNormal = normalize(nt(si.vertexNormal));
  si.normal = normalize(nt(si.normal));
  si.directionTangent = mat4_mul(l2w, si.directionTangent, 0.0f);
  si.directionBitangent = mat4_mul(l2w, si.directionBitangent, 0.0f);
  si.geometryTangent = mat4_mul(l2w, si.geometryTangent, 0.0f);
  si.geometryBitangent = mat4_mul(l2w, si.geometryBitangent, 0.0f);
  si.shadowOffset = mat4_mul(l2w, si.shadowOffset, 0.0f);
  si.position = mat4_mul(l2w, si.position, 1.0f);
}

// intersect.wgsl.ts:696-740 intersectScene
bool intersectScene(const Scene &s, const Ray &r, SurfaceInteraction &si, int bounces, bool doubleSided,
                    Traffic *tr) {
  si.hit = false;
  if (s.u->is_empty > 0) return false;
  if (tr) tr->extension_rays++;
  TraversalHit h;
  h.tMax = RAY_MAX_DISTANCE;
  traverse(s, r, bounces, doubleSided, si.triangleIndex, si.instanceIndex, Mode::Closest, h, tr);
  if (h.isHit) {
    si.triangleIndex = h.triangleIndex;
    completeSurfaceInteraction(s, si, h);
  }
  return si.hit;
}

// intersect.wgsl.ts:829-879 intersectSceneShadow
bool intersectSceneShadow(const Scene &s, const Ray &r, float lightDistance, i32 tri, i32 ins, Traffic *tr,
                          Sampler *smp) {
  if (s.u->is_empty > 0) return false;
  if (tr) tr->shadow_rays++;
  TraversalHit h;
  h.tMax = fminf(fmaxf(lightDistance, 0.0f), RAY_MAX_DISTANCE);
  return traverse(s, r, 1, true, tri, ins, Mode::Shadow, h, tr, (s.flags & MTC_SCENE_HAS_ALPHA) ? smp : nullptr);
}

}  // namespace oracle
