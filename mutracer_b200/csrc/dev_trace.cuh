// Device sampler (Owen-scrambled Sobol, ZSobol, PCG4D) and two-level BVH2
// traversal with the watertight FP32 triangle test.
#pragma once
#include "../../include/mutracer_b200.h"
#include "dev_math.cuh"

namespace mt {

// Device copy of the bind groups; all pointers are device pointers.
struct DevScene {
  const float4 *bvh;
  const float4 *ins;
  const uint32_t *attr;
  const float4 *mats;
  const float4 *env;
  const float2 *envDist;
  const float4 *lightData;
  const float *lut;
  const float4 *lights;
  uint32_t envW, envH;
  uint32_t vstride, vnormalOff, vnormalFloat;
  uint32_t flags;
  uint32_t insCount, matCount;
  const float4 *maps;       // MTC_MAP_VEC4_ROWS per material map
  const float4 *mapTexels;  // RGBA per texel
  uint32_t mapCount, mapTexelCount;
  uint32_t vuvOff;          // word offset of the f32 UV pair (0: no UVs)
  uint32_t vcolorOff, vcolorFloat;  // vertex color word(s) (0: white), f32x3 or RGBA8
  uint32_t vuv1Off;         // secondary UV pair (0: the primary pair)
  const uint32_t *triMats;  // material + 1 per bvh vec4 (null: instance materials only)
};

// One render job: scene, uniforms, outputs (the plain kernel takes one as a
// __grid_constant__ parameter; the batched kernel reads a table of them).
struct JobData {
  DevScene s;
  mtc_trace_uniform u;
  mtc_camera_uniform cam;
  float4 *outColor, *outNormal, *outAlbedo, *outCatcher;
  uint32_t samples;
  uint32_t width, height;
  uint32_t tilesX, tilesY;
  uint32_t firstItem;  // first global work item of this job (batched kernel)
  uint32_t items;      // tiles * samples
  uint32_t _pad;
};

struct Counters {
  uint32_t ext = 0, shadow = 0;
};

// ------------------------------------------------------------------ sampler
// sobol.wgsl.ts:23-45
MTD uint32_t sampleHash(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352du;
  x ^= x >> 15; x *= 0x846ca68bu;
  return x ^ (x >> 16);
}
MTD uint32_t sampleSeed(uint32_t a, uint32_t b) { return sampleHash(a ^ sampleHash(b + 0x9e3779b9u)); }
MTD uint32_t lkPermute(uint32_t v, uint32_t seed) {
  uint32_t x = v + seed;
  x ^= x * 0x6c50b47cu; x ^= x * 0xb82f1e52u;
  x ^= x * 0xc7afe638u; x ^= x * 0x8d22f6e6u;
  return x;
}
MTD uint32_t owen(uint32_t x, uint32_t seed) { return __brev(lkPermute(__brev(x), seed)); }
MTD uint32_t sobolD1(uint32_t v) {
  uint32_t r = __brev(v);
  r ^= (r << 1) & 0xaaaaaaaau;
  r ^= (r << 2) & 0xccccccccu;
  r ^= (r << 4) & 0xf0f0f0f0u;
  r ^= (r << 8) & 0xff00ff00u;
  r ^= (r << 16) & 0xffff0000u;
  return r;
}
MTD uint32_t morton2(uint32_t x, uint32_t y) {
  uint32_t vx = x & 255u, vy = y & 255u;
  vx = (vx | (vx << 4)) & 0x0f0fu; vy = (vy | (vy << 4)) & 0x0f0fu;
  vx = (vx | (vx << 2)) & 0x3333u; vy = (vy | (vy << 2)) & 0x3333u;
  vx = (vx | (vx << 1)) & 0x5555u; vy = (vy | (vy << 1)) & 0x5555u;
  return vx | (vy << 1);
}
// Packed pbrt-v4 ZSobol digit permutations (src/renderer/sampling.ts:23-28).
__device__ __constant__ static const uint32_t kZPermWords[6] = {
    0x78d8b4e4u, 0xb1e19c6cu, 0x8d2d39c9u, 0x72d236c6u, 0x87271e4eu, 0x93634b1bu};
MTD uint32_t zSobolPermutation(uint32_t perm) {
  return (kZPermWords[perm >> 2] >> ((perm & 3u) * 8u)) & 255u;
}
MTD uint32_t zSobolIndex(uint32_t morton, uint32_t dim, uint32_t logSPP) {
  uint32_t odd = logSPP & 1u;
  uint32_t digits = 8u + ((logSPP + 1u) >> 1);
  uint32_t result = 0;
  for (int digit = int(digits) - 1; digit >= int(odd); digit--) {
    uint32_t shift = 2u * uint32_t(digit) - odd;
    uint32_t higher = shift < 30u ? morton >> (shift + 2u) : 0u;
    uint32_t perm = (sampleHash(higher ^ (0x55555555u * dim)) >> 24) % 24u;
    uint32_t d = (morton >> shift) & 3u;
    result |= ((zSobolPermutation(perm) >> (2u * d)) & 3u) << shift;
  }
  if (odd != 0u) result |= (morton & 1u) ^ (sampleHash((morton >> 1) ^ (0x55555555u * dim)) & 1u);
  return result;
}

struct Sampler {
  uint32_t px, py, width, index, bounce, hashed, seed, logspp;
  int pattern;
  uint4 s0;
  MTD V2 structured(uint32_t dim) const {
    uint32_t pixelID = px + py * width;
    uint32_t sd = sampleSeed(sampleSeed(pixelID, dim), seed);
    uint32_t idx = index;
    if (pattern == 1) {
      uint32_t lg = logspp;
      if (idx == 0u) lg = 0u; else idx -= 1u;
      uint32_t block = idx >> lg;
      uint32_t mask = (1u << lg) - 1u;
      uint32_t morton = (morton2(px, py) << lg) | (idx & mask);
      idx = zSobolIndex(morton, dim, lg);
      sd = sampleSeed(sampleSeed(dim, seed), sampleSeed(px >> 8, py >> 8));
      if (index != 0u) block += 1u;
      sd = sampleSeed(sd, block);
    }
    uint32_t i = owen(idx, sampleSeed(sd, 0u));
    uint32_t x = __brev(lkPermute(i, sampleSeed(sd, 1u)));
    uint32_t y = owen(sobolD1(i), sampleSeed(sd, 2u));
    float fx = float(x >> 8) * (1.0f / 16777216.0f);
    float fy = float(y >> 8) * (1.0f / 16777216.0f);
    return {EPS + 0.999f * fx, EPS + 0.999f * fy};
  }
  MTD float rnd() {
    s0.x = s0.x * 1664525u + 1013904223u; s0.y = s0.y * 1664525u + 1013904223u;
    s0.z = s0.z * 1664525u + 1013904223u; s0.w = s0.w * 1664525u + 1013904223u;
    s0.x += s0.y * s0.w; s0.y += s0.z * s0.x; s0.z += s0.x * s0.y; s0.w += s0.y * s0.z;
    s0.x ^= s0.x >> 16; s0.y ^= s0.y >> 16; s0.z ^= s0.z >> 16; s0.w ^= s0.w >> 16;
    s0.x += s0.y * s0.w; s0.y += s0.z * s0.x; s0.z += s0.x * s0.y; s0.w += s0.y * s0.z;
    return float(s0.x) / float(0xffffffffu);
  }
  MTD float s1(uint32_t dim) {
    if (pattern == 2) return EPS + 0.999f * rnd();
    return structured(dim).x;
  }
  MTD V2 s2(uint32_t dim) {
    if (pattern == 2) { float a = s1(dim); float b = s1(dim); return {a, b}; }
    return structured(dim);
  }
  MTD float hashedSample(uint32_t slot) {
    uint32_t dim = sampleSeed(sampleSeed(bounce, slot), hashed) | 0x80000000u;
    hashed += 1u;
    if (pattern == 2) return EPS + 0.999f * rnd();
    uint32_t pixelID = px + py * width;
    uint32_t sd = sampleSeed(sampleSeed(pixelID, dim), seed);
    uint32_t i = owen(index, sampleSeed(sd, 0u));
    uint32_t x = __brev(lkPermute(i, sampleSeed(sd, 1u)));
    return EPS + 0.999f * (float(x >> 8) * (1.0f / 16777216.0f));
  }
  MTD float lightCandidateRandom(uint32_t salt) {
    if (pattern == 2) (void)rnd();
    uint32_t pixelID = px + py * width;
    uint32_t key = sampleSeed(sampleSeed(pixelID, index), seed);
    uint32_t dimension = sampleSeed(bounce, salt) ^ 0xa511e9b3u;
    return float(sampleHash(key ^ dimension) >> 8) * (1.0f / 16777216.0f);
  }
  MTD uint32_t bounceDim(uint32_t slot) const { return 3u + 8u + bounce * 64u + slot; }
  MTD uint32_t lightDim(uint32_t c, uint32_t slot) const {
    if (c == 0u) return slot == 2u ? bounceDim(8u) : bounceDim(slot);
    return bounceDim(9u + (c - 1u) * 3u + slot);
  }
};

// ---------------------------------------------------------------- traversal
// intersect.wgsl.ts:1500-1521 (every operation rounded, fminf/fmaxf)
MTD V3 traversalInverse(V3 d) { return {__frcp_rn(d.x), __frcp_rn(d.y), __frcp_rn(d.z)}; }
MTD float intersectBox(V3 o, V3 bmin, V3 bmax, V3 invD, float tMax) {
  V3 tBot = xmul3(xsub3(bmin, o), invD);
  V3 tTop = xmul3(xsub3(bmax, o), invD);
  float t0 = fmaxf(fminf(tBot.x, tTop.x), fmaxf(fminf(tBot.y, tTop.y), fminf(tBot.z, tTop.z)));
  float t1 = fminf(fmaxf(tBot.x, tTop.x), fminf(fmaxf(tBot.y, tTop.y), fmaxf(tBot.z, tTop.z)));
  if (t0 > t1 || t0 > tMax) return -1.0f;
  return t0 > 0.0f ? t0 : t1;
}
MTD int maxDimension(V3 v) {
  if (v.x > v.y) return v.x > v.z ? 0 : 2;
  return v.y > v.z ? 1 : 2;
}
MTD V3 getShear(V3 d, int maxDim) {
  if (maxDim == 0) return {xd(-d.y, d.x), xd(-d.z, d.x), __frcp_rn(d.x)};
  if (maxDim == 1) return {xd(-d.z, d.y), xd(-d.x, d.y), __frcp_rn(d.y)};
  return {xd(-d.x, d.z), xd(-d.y, d.z), __frcp_rn(d.z)};
}
// intersect.wgsl.ts:1430-1493; returns t (0 for a miss) and barycentrics.
MTD float intersectTriangle(V3 o, V3 p0, V3 p1, V3 p2, int maxDim, V3 shear, float tMax, V3 &bary) {
  V3 a = xsub3(p0, o), b = xsub3(p1, o), c = xsub3(p2, o);
  if (maxDim == 0) { a = {a.y, a.z, a.x}; b = {b.y, b.z, b.x}; c = {c.y, c.z, c.x}; }
  else if (maxDim == 1) { a = {a.z, a.x, a.y}; b = {b.z, b.x, b.y}; c = {c.z, c.x, c.y}; }
  a.x = xa(a.x, xm(shear.x, a.z)); a.y = xa(a.y, xm(shear.y, a.z));
  b.x = xa(b.x, xm(shear.x, b.z)); b.y = xa(b.y, xm(shear.y, b.z));
  c.x = xa(c.x, xm(shear.x, c.z)); c.y = xa(c.y, xm(shear.y, c.z));
  V3 e = {xs(xm(b.x, c.y), xm(b.y, c.x)), xs(xm(c.x, a.y), xm(c.y, a.x)), xs(xm(a.x, b.y), xm(a.y, b.x))};
  bool anyNeg = e.x < 0.0f || e.y < 0.0f || e.z < 0.0f;
  bool anyPos = e.x > 0.0f || e.y > 0.0f || e.z > 0.0f;
  if (anyNeg && anyPos) return 0.0f;
  float det = xa(xa(e.x, e.y), e.z);
  float az = xm(a.z, shear.z), bz = xm(b.z, shear.z), cz = xm(c.z, shear.z);
  float tScaled = xa(xa(xm(e.x, az), xm(e.y, bz)), xm(e.z, cz));
  if (fabsf(tScaled) > fabsf(xm(tMax, det))) return 0.0f;
  float invDet = __frcp_rn(det);
  bary = {xm(e.x, invDet), xm(e.y, invDet), xm(e.z, invDet)};
  return xm(tScaled, invDet);
}

MTD V3 vertexPosition(const DevScene &s, int32_t i) {
  const uint32_t *w = s.attr + size_t(i) * s.vstride;
  if (s.vstride == 4) {
    float4 q = __ldg(reinterpret_cast<const float4 *>(w));
    return {q.x, q.y, q.z};
  }
  return {asf(__ldg(w)), asf(__ldg(w + 1)), asf(__ldg(w + 2))};
}
// vertexAttributes.wgsl.ts:14-28
MTD V3 vertexNormal(const DevScene &s, int32_t i) {
  const uint32_t *w = s.attr + size_t(i) * s.vstride + s.vnormalOff;
  if (s.vnormalFloat) return {asf(__ldg(w)), asf(__ldg(w + 1)), asf(__ldg(w + 2))};
  uint32_t word = __ldg(w);
  int32_t a = int32_t(word << 16) >> 16;
  int32_t b = int32_t(word) >> 16;
  if (a == -32768 && b == -32768) return v3(0.0f);
  V3 v = {float(a) / 32767.0f, float(b) / 32767.0f, 0.0f};
  v.z = 1.0f - fabsf(v.x) - fabsf(v.y);
  if (v.z < 0.0f) {
    float nx = (1.0f - fabsf(v.y)) * (v.x >= 0.0f ? 1.0f : -1.0f);
    float ny = (1.0f - fabsf(v.x)) * (v.y >= 0.0f ? 1.0f : -1.0f);
    v.x = nx; v.y = ny;
  }
  return normalize(v);
}

// ------------------------------------------------------------ material maps
// materialBuffer.wgsl.ts:316-378 wrapMapCoordinate / sampleMap / loadMapTexel
// with independent textures.  The shader filters footprints inside the image
// in hardware and repeat footprints that cross its edge by hand; both are the
// bilinear mix of the four texels around wrapped * size - 0.5 with clamped
// (repeat: modular) texel coordinates, evaluated here in software for every
// footprint.  Rounded operations throughout (no contraction), so a lookup is
// bit-identical to the CPU restatement.
MTD float wrapMapCoordinate(float v, float mode) {
  if (mode < 0.5f) return __fsub_rn(v, floorf(v));
  if (mode < 1.5f) return clampf(v, 0.0f, 1.0f);
  const float m = __fsub_rn(v, __fmul_rn(2.0f, floorf(__fmul_rn(v, 0.5f))));
  return __fsub_rn(1.0f, fabsf(__fsub_rn(1.0f, m)));
}
static __device__ __noinline__ float4 sampleMap(const DevScene &s, int idx, V2 uv) {
  if (idx < 0 || uint32_t(idx) >= s.mapCount) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const float4 *mi = s.maps + size_t(idx) * MTC_MAP_VEC4_ROWS;
  const float4 a = ld4(mi), t = ld4(mi + 1), modes = ld4(mi + 2);
  const int w = asi(a.x), h = asi(a.y);
  const uint32_t first = asu(a.z);
  if (w < 1 || h < 1 || uint64_t(first) + uint64_t(w) * uint64_t(h) > s.mapTexelCount)
    return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const float tx = __fsub_rn(__fmul_rn(wrapMapCoordinate(__fadd_rn(__fmul_rn(uv.x, t.x), t.z), modes.z), float(w)), 0.5f);
  const float ty = __fsub_rn(__fmul_rn(wrapMapCoordinate(__fadd_rn(__fmul_rn(uv.y, t.y), t.w), modes.w), float(h)), 0.5f);
  const float fx = floorf(tx), fy = floorf(ty), wx = __fsub_rn(tx, fx), wy = __fsub_rn(ty, fy);
  // Finite coordinates wrap into [-1, size - 1]; the clamp only pins NaN.
  const int bx = int(fminf(fmaxf(fx, -1.0f), float(w))), by = int(fminf(fmaxf(fy, -1.0f), float(h)));
  auto load = [&](int x, int y) {
    int px = modes.z < 0.5f ? ((x % w) + w) % w : min(max(x, 0), w - 1);
    int py = modes.w < 0.5f ? ((y % h) + h) % h : min(max(y, 0), h - 1);
    return ld4(s.mapTexels + first + size_t(py) * size_t(w) + size_t(px));
  };
  const float4 t00 = load(bx, by), t10 = load(bx + 1, by), t01 = load(bx, by + 1), t11 = load(bx + 1, by + 1);
  auto mix1 = [](float p, float q, float k) { return __fadd_rn(__fmul_rn(p, __fsub_rn(1.0f, k)), __fmul_rn(q, k)); };
  auto mix4 = [&](float4 p, float4 q, float k) {
    return make_float4(mix1(p.x, q.x, k), mix1(p.y, q.y, k), mix1(p.z, q.z, k), mix1(p.w, q.w, k));
  };
  return mix4(mix4(t00, t10, wx), mix4(t01, t11, wx), wy);
}
// projectUV (uvProjection.wgsl.ts): procedural UVs from a local-space
// position and normal; 1 spherical, 2 cylindrical, 3 triplanar.
MTD V2 projectUV(int type, V3 pos, V3 normal) {
  if (type == 3) {
    const V3 a = {fabsf(normal.x), fabsf(normal.y), fabsf(normal.z)};
    if (a.x > a.y && a.x > a.z) return {pos.y, pos.z};
    if (a.y > a.x && a.y > a.z) return {pos.x, pos.z};
    return {pos.x, pos.y};
  }
  if (type == 1) {
    const V3 n = normalize(pos);
    return {atan2f(n.x, n.z) / (2.0f * PI) + 0.5f, 1.0f - acosf(n.y) / PI};
  }
  if (type == 2) return {atan2f(pos.z, pos.x) / (2.0f * PI) + 0.5f, pos.y};
  return {0.0f, 0.0f};
}

// A material's map index names a map of this scene (an index past the map
// table, like -1, means no map).
MTD bool mapValid(const DevScene &s, float index) { return index >= 0.0f && index < float(s.mapCount); }

// intersectionAlphaPasses (intersectionAlpha.wgsl.ts:14-90): whether a shadow
// ray's candidate hit on a triangle of `material` occludes.  Coverage is the
// material's alpha times the base color's alpha (map alpha usage "alpha") and
// the alpha map's g at the hit's UV, then resolved by the alpha mode: opaque
// occludes, mask compares with the cutoff, blend draws hashedSample(1).
static __device__ __noinline__ bool alphaPasses(const DevScene &s, int32_t material, int32_t record, int32_t i0,
                                                int32_t i1, int32_t i2, V3 bary, V3 hitPosition, V3 hitNormal,
                                                Sampler &smp) {
  if (s.triMats) {  // triangleMaterial (vertexAttributes.wgsl.ts:51-56)
    const uint32_t m = __ldg(s.triMats + record);
    if (m && m - 1u < s.matCount) material = int32_t(m - 1u);
  }
  const float4 *d = s.mats + size_t(material) * MTC_MATERIAL_VEC4_ROWS;
  const float4 r2 = ld4(d + 2), r5 = ld4(d + 5), r22 = ld4(d + 22);
  float alpha = ld4(d + 9).x;
  const bool baseAlpha = r5.w == 2.0f && mapValid(s, r2.z), alphaMap = mapValid(s, r22.z);
  if (baseAlpha || alphaMap) {
    V2 uv0 = {0.0f, 0.0f}, uv1 = uv0, uv2 = uv0;
    if (s.vuvOff) {
      auto vuv = [&](int32_t i) {
        const uint32_t *w = s.attr + size_t(i) * s.vstride + s.vuvOff;
        return V2{asf(__ldg(w)), asf(__ldg(w + 1))};
      };
      uv0 = vuv(i0); uv1 = vuv(i1); uv2 = vuv(i2);
    }
    const float4 r7 = ld4(d + 7);
    const int projection = int(r7.x);
    V2 uv = {bary.x * uv0.x + bary.y * uv1.x + bary.z * uv2.x, bary.x * uv0.y + bary.y * uv1.y + bary.z * uv2.y};
    if (projection > 0) uv = projectUV(projection, hitPosition, hitNormal);
    uv = {uv.x * r7.z, uv.y * r7.w};
    if (projection == 3) uv = {uv.x - floorf(uv.x), uv.y - floorf(uv.y)};
    if (baseAlpha) alpha *= sampleMap(s, int(r2.z), uv).w;
    if (alphaMap) alpha *= sampleMap(s, int(r22.z), uv).y;
  }
  const int mode = int(ld4(d + 23).w);
  if (mode == 0) alpha = 1.0f;
  else if (mode == 1) alpha = alpha >= r22.w ? 1.0f : 0.0f;
  if (mode == 2) return smp.hashedSample(1u) <= alpha;
  return alpha >= 1.0f;
}

struct TraversalHit {
  float tMax;
  V3 hitNormal, hitBary;
  int32_t triangleIndex, insIdx;
};

// Levels of the near path taken in one interior visit beyond the first.
#ifndef MT_FUSED_LEVELS
#define MT_FUSED_LEVELS 1
#endif

// The interior visit of getBVHTraverseCode at either level (intersect.wgsl.ts
// :265-300, :439-624 for BVH2): box-test both children (boxes given), push
// the nearer last (the `>` rule).  The node the reference pops next is the
// child pushed last; when that child is an interior node (its header word
// came with its box) its children are tested in the same visit instead of
// going through the stack, for up to MT_FUSED_LEVELS more levels.  Nothing in
// between could change tMax, so the boxes tested, their order and the stack
// contents are those of one level per visit.  `base` is where node indices
// start in the buffer (the BLAS base), `rightOffset` what a right pointer is
// relative to (the BLAS offset; 0 in the TLAS).
MTD void visitInterior(const float4 *bvh, int32_t base, int32_t rightOffset, bool fusable, V3 ro, V3 invDir,
                       float tMax, int32_t left, int32_t right, float4 lmin, float4 lmax, float4 rmin, float4 rmax,
                       int32_t *stack, int &top) {
  for (int level = 0;; level++) {
    const float d0 = intersectBox(ro, xyz(lmin), xyz(lmax), invDir, tMax);
    const float d1 = intersectBox(ro, xyz(rmin), xyz(rmax), invDir, tMax);
    int32_t first = right, second = left;
    float df = d1, ds = d0;
    float firstPtr = rmin.w, secondPtr = lmin.w;
    if (d0 > d1) {
      first = left; second = right;
      df = d0; ds = d1;
      firstPtr = lmin.w; secondPtr = rmin.w;
    }
    const bool pushFirst = df > 0.0f && top + 1 < MTC_MAX_STACK;
    const bool pushSecond = ds > 0.0f && top + (pushFirst ? 2 : 1) < MTC_MAX_STACK;
    // The node popped next: the second child if pushed, else the first.
    const int32_t next = pushSecond ? second : first;
    const int32_t nextPtr = asi(pushSecond ? secondPtr : firstPtr);
    const bool fuse = fusable && level < MT_FUSED_LEVELS && (pushFirst || pushSecond) && nextPtr >= 0;
    if (pushFirst && !(fuse && !pushSecond)) stack[++top] = first;
    if (pushSecond && !fuse) stack[++top] = second;
    if (!fuse) return;
    left = next + 2;
    right = nextPtr + rightOffset;
    lmin = ld4(bvh + left + base);
    lmax = ld4(bvh + left + 1 + base);
    rmin = ld4(bvh + right + base);
    rmax = ld4(bvh + right + 1 + base);
  }
}

// getBVHTraverseCode, intersect.wgsl.ts:213-629 for the BVH2 layout.  With
// `shadow` the first accepted hit ends the query (returns true).
//
// kGpuLayout mirrors the reference's blasLayoutMask specialisation
// (getBVHTraverseCode's layout branches are compiled only for the layouts a
// scene uses): without it only BVH2 (layout 0) BLASes are traversed and the
// BVH_GPU (layout 2) code is not compiled in.
//
// A shadow query with kAlpha tests each candidate hit's coverage
// (alphaPasses, drawing from `alphaSmp`): a hit that does not occlude
// restores the query's tMax and traversal goes on (intersect.wgsl.ts
// :846-866).  Without kAlpha the test is not compiled in.
template <bool shadow, bool kGpuLayout, bool kAlpha = false>
__device__ __noinline__ bool traverse(const DevScene &s, int32_t blasBase, V3 rayO, V3 rayD, int bounces,
                                      bool doubleSided, int32_t currentTri, int32_t currentIns, TraversalHit &h,
                                      Sampler *alphaSmp = nullptr) {
  const float tMaxInit = h.tMax;
  int32_t tlasStack[MTC_MAX_STACK];
  int32_t blasStack[MTC_MAX_STACK];
  int tlasTop = -1;
  const float4 *bvh = s.bvh;
  V3 invD = traversalInverse(rayD);
  if (intersectBox(rayO, xyz(ld4(bvh)), xyz(ld4(bvh + 1)), invD, h.tMax) > 0.0f) {
    tlasTop = 0;
    tlasStack[0] = 0;
  }
  while (tlasTop >= 0) {
    int32_t tlasNode = tlasStack[tlasTop--];
    float4 r1 = ld4(bvh + tlasNode);
    int32_t ptr = asi(r1.w);
    if (ptr >= 0) {
      int32_t left = tlasNode + 2, right = ptr;
      visitInterior(bvh, 0, 0, true, rayO, invD, h.tMax, left, right, ld4(bvh + left), ld4(bvh + left + 1),
                    ld4(bvh + right), ld4(bvh + right + 1), tlasStack, tlasTop);
      continue;
    }
    int32_t tlasCount = -ptr;
    for (int32_t io = tlasCount - 1; io >= 0; io--) {
      float4 rec = ld4(bvh + tlasNode + 2 + io);
      int32_t insIdx = asi(rec.x);
      int32_t blasRoot = asi(rec.y);
      const float4 *insv = s.ins + size_t(insIdx) * MTC_INSTANCE_VEC4_STRIDE;
      float4 insData = ld4(insv);
      float4 c0 = ld4(insv + 1), c1 = ld4(insv + 2), c2 = ld4(insv + 3), c3 = ld4(insv + 4);
      V3 o = xmat4(c0, c1, c2, c3, rayO, 1.0f);
      V3 d = xmat4(c0, c1, c2, c3, rayD, 0.0f);
      V3 linvD = traversalInverse(d);
      int maxDim = maxDimension(vabs(d));
      V3 shear = getShear(d, maxDim);
      uint32_t encoded = asu(insData.x);
      const uint32_t layout = encoded >> 30;
      if (layout != 0u && !(kGpuLayout && layout == 2u)) continue;  // TinyBVH bvh4 / cwbvh are not consumed
      int32_t blasOffset = int32_t(encoded & 0x3fffffffu);
      int32_t vertexOffset = asi(insData.y);
      int32_t sideMaterial = asi(insData.z) >> 8;
      int blasTop = 0;
      blasStack[0] = blasRoot;
      while (blasTop >= 0) {
        int32_t node = blasStack[blasTop--];
        int32_t i = node + blasBase;
        int32_t p, left, right;
        float d0 = 0.0f, d1 = 0.0f;
        if (kGpuLayout && layout == 2u) {
          // BVH_GPU node (intersect.wgsl.ts:453-497): both child boxes inline.
          float4 g0 = ld4(bvh + i), g1 = ld4(bvh + i + 1), g2 = ld4(bvh + i + 2), g3 = ld4(bvh + i + 3);
          int32_t count = int32_t(asu(g2.w));
          p = count > 0 ? -count : 0;
          left = blasOffset + int32_t(asu(g0.w) * 4u);
          right = blasOffset + int32_t(asu(g1.w) * 4u);
          if (p >= 0) {
            d0 = intersectBox(o, xyz(g0), xyz(g1), linvD, h.tMax);
            d1 = intersectBox(o, xyz(g2), xyz(g3), linvD, h.tMax);
          } else {
            i = blasBase + blasOffset + int32_t(asu(g3.w)) - 2;  // records at i + 2
          }
        } else {
          float4 n1 = ld4(bvh + i);
          p = asi(n1.w);
          left = node + 2;
          right = p + blasOffset;
          if (p >= 0) {
            visitInterior(bvh, blasBase, blasOffset, true, o, linvD, h.tMax, left, right, ld4(bvh + left + blasBase),
                          ld4(bvh + left + 1 + blasBase), ld4(bvh + right + blasBase),
                          ld4(bvh + right + 1 + blasBase), blasStack, blasTop);
            continue;
          }
        }
        if (p >= 0) {
          if (d0 > d1) {
            if (d0 > 0.0f && blasTop + 1 < MTC_MAX_STACK) blasStack[++blasTop] = left;
            if (d1 > 0.0f && blasTop + 1 < MTC_MAX_STACK) blasStack[++blasTop] = right;
          } else {
            if (d1 > 0.0f && blasTop + 1 < MTC_MAX_STACK) blasStack[++blasTop] = right;
            if (d0 > 0.0f && blasTop + 1 < MTC_MAX_STACK) blasStack[++blasTop] = left;
          }
          continue;
        }
        int32_t primitiveCount = -p;
        int32_t primitiveOffset = i + 2;
        for (int32_t k = 0; k < primitiveCount; k++) {
          int32_t triangleIndex = primitiveOffset + k;
          if (bounces > 0 && triangleIndex == currentTri && insIdx == currentIns) continue;
          float4 r3 = ld4(bvh + triangleIndex);
          V3 p0 = vertexPosition(s, asi(r3.x) + vertexOffset);
          V3 p1 = vertexPosition(s, asi(r3.y) + vertexOffset);
          V3 p2 = vertexPosition(s, asi(r3.z) + vertexOffset);
          V3 bary;
          float t = intersectTriangle(o, p0, p1, p2, maxDim, shear, h.tMax, bary);
          if (!(t > 0.0f)) continue;
          V3 candidateNormal = xnormalize(xcross(xsub3(p1, p0), xsub3(p2, p0)));
          if (!doubleSided) {
            bool matDoubleSided = __ldg(&s.mats[size_t(sideMaterial) * MTC_MATERIAL_VEC4_ROWS + 23].z) > 0.5f;
            if (!matDoubleSided && xdot(candidateNormal, d) > 0.0f) continue;
          }
          h.hitNormal = candidateNormal;
          h.tMax = t;
          h.hitBary = bary;
          if (shadow) {
            if (kAlpha && !alphaPasses(s, sideMaterial, triangleIndex, asi(r3.x) + vertexOffset,
                                       asi(r3.y) + vertexOffset, asi(r3.z) + vertexOffset, bary, o + d * t,
                                       candidateNormal, *alphaSmp)) {
              h.tMax = tMaxInit;
              continue;
            }
            return true;
          }
          h.triangleIndex = triangleIndex;
          h.insIdx = insIdx;
        }
      }
    }
  }
  return false;
}

// getBVHTraverseCode (intersect.wgsl.ts:213-629) as a restartable state
// machine, for kernels that keep a queue of rays and give a lane a new ray as
// soon as its current one has finished.  Each step() does exactly one of:
// one node (a BLAS node of the current instance, or a TLAS node when no
// instance is open: interior nodes of both levels run the same code, so lanes
// at different levels stay together), or entering the next instance of the
// current TLAS leaf.  Visit order, box tests, the `>` tie rule and the
// self-hit and backface rules are those of traverse(), so the hits are
// bit-identical to it.
constexpr int kTraversalStackEntries = 2 * MTC_MAX_STACK;

template <bool shadow, bool kGpuLayout, bool kAlpha = false>
struct RayTraversal {
  const float4 *bvh, *ins, *mats;
  const uint32_t *attr;
  uint32_t vstride;
  int32_t blasBase;
  V3 rayO, rayD, invD;
  int bounces;
  bool doubleSided;
  int32_t currentTri, currentIns;
  // TLAS entries at [0, MTC_MAX_STACK), the current instance's BLAS entries
  // at [MTC_MAX_STACK, 2 * MTC_MAX_STACK): two stacks of the reference's
  // depth, addressed through one array of kTraversalStackEntries so TLAS and
  // BLAS node visits share one code path.  The array belongs to the caller
  // (a local array of the kernel): a dynamically indexed array inside this
  // object would keep the whole object, ray and hit included, in local
  // memory.
  int32_t *stack;
  int tlasTop, blasTop;
  int32_t leafNode, io;
  V3 o, d, linvD, shear;
  int maxDim;
  int32_t blasOffset, vertexOffset, sideMaterial, insIdx;
  uint32_t blasLayout;
  bool found;
  TraversalHit h;
  // Shadow queries of scenes with alpha: the scene and the path's sampler
  // for alphaPasses, and the query's tMax to restore after a hit that does
  // not occlude.  Null otherwise.
  const DevScene *alphaScene;
  Sampler *alphaSmp;
  float tMaxInit;

  MTD V3 position(int32_t i) const {
    const uint32_t *w = attr + size_t(i) * vstride;
    if (vstride == 4) {
      float4 q = __ldg(reinterpret_cast<const float4 *>(w));
      return {q.x, q.y, q.z};
    }
    return {asf(__ldg(w)), asf(__ldg(w + 1)), asf(__ldg(w + 2))};
  }

  // Starts a query; returns false when the root box is missed (nothing to do).
  MTD bool begin(const DevScene &s, int32_t base, V3 ro, V3 rd, int b, bool ds, int32_t ct, int32_t ci, float tMax) {
    bvh = s.bvh; ins = s.ins; mats = s.mats; attr = s.attr; vstride = s.vstride; blasBase = base;
    rayO = ro; rayD = rd; bounces = b; doubleSided = ds; currentTri = ct; currentIns = ci;
    if (kAlpha) {
      alphaScene = nullptr;
      alphaSmp = nullptr;
      tMaxInit = tMax;
    }
    h.tMax = tMax;
    h.triangleIndex = -1;
    h.insIdx = -1;
    h.hitBary = v3(0.0f);
    h.hitNormal = v3(0.0f);
    found = false;
    tlasTop = -1;
    blasTop = -1;
    io = -1;
    leafNode = 0;
    insIdx = -1;
    blasOffset = 0;
    blasLayout = 0;
    invD = traversalInverse(rd);
    if (intersectBox(rayO, xyz(ld4(bvh)), xyz(ld4(bvh + 1)), invD, h.tMax) > 0.0f) {
      tlasTop = 0;
      stack[0] = 0;
      return true;
    }
    return false;
  }

  // One traversal step; returns true when the query has finished.
  MTD bool step() {
    const bool blas = blasTop >= 0;
    if (!blas) {
      if (io >= 0) return enterInstance();
      if (tlasTop < 0) return true;
    }
    // Pop one node of the current level.
    int top = blas ? blasTop : tlasTop;
    const int stackBase = blas ? MTC_MAX_STACK : 0;
    int32_t node = stack[stackBase + top];
    top--;
    const int32_t base = blas ? blasBase : 0;
    // Decode the node: BVH2 (TLAS, BLAS layout 0) keeps each child's box in
    // the child; BVH_GPU (BLAS layout 2, intersect.wgsl.ts:453-497) keeps both
    // child boxes in the node itself.
    bool interior;
    int32_t left = 0, right = 0, primitiveCount = 0, primitiveOffset = 0;
    float4 lmin, lmax, rmin, rmax;
    if (kGpuLayout && blas && blasLayout == 2u) {
      lmin = ld4(bvh + node + base);
      lmax = ld4(bvh + node + base + 1);
      rmin = ld4(bvh + node + base + 2);
      rmax = ld4(bvh + node + base + 3);
      int32_t count = int32_t(asu(rmin.w));
      interior = count <= 0;
      left = blasOffset + int32_t(asu(lmin.w) * 4u);
      right = blasOffset + int32_t(asu(lmax.w) * 4u);
      primitiveCount = count;
      primitiveOffset = base + blasOffset + int32_t(asu(rmax.w));
    } else {
      int32_t p = asi(ld4(bvh + node + base).w);
      interior = p >= 0;
      left = node + 2;
      right = blas ? p + blasOffset : p;
      primitiveCount = -p;
      primitiveOffset = node + base + 2;
      if (interior) {
        lmin = ld4(bvh + left + base);
        lmax = ld4(bvh + left + 1 + base);
        rmin = ld4(bvh + right + base);
        rmax = ld4(bvh + right + 1 + base);
      }
    }
    if (interior) {
      // Interior node at either level (one code path for both).
      visitInterior(bvh, base, blas ? blasOffset : 0, !(kGpuLayout && blas && blasLayout == 2u), blas ? o : rayO,
                    blas ? linvD : invD, h.tMax, left, right, lmin, lmax, rmin, rmax, stack + stackBase, top);
      if (blas) blasTop = top; else tlasTop = top;
      return false;
    }
    if (blas) blasTop = top; else tlasTop = top;
    if (!blas) {
      leafNode = node;
      io = primitiveCount - 1;
      return false;
    }
    for (int32_t k = 0; k < primitiveCount; k++) {
      int32_t triangleIndex = primitiveOffset + k;
      if (bounces > 0 && triangleIndex == currentTri && insIdx == currentIns) continue;
      float4 r3 = ld4(bvh + triangleIndex);
      V3 p0 = position(asi(r3.x) + vertexOffset);
      V3 p1 = position(asi(r3.y) + vertexOffset);
      V3 p2 = position(asi(r3.z) + vertexOffset);
      V3 bary;
      float t = intersectTriangle(o, p0, p1, p2, maxDim, shear, h.tMax, bary);
      if (!(t > 0.0f)) continue;
      V3 candidateNormal = xnormalize(xcross(xsub3(p1, p0), xsub3(p2, p0)));
      if (!doubleSided) {
        bool matDoubleSided = __ldg(&mats[size_t(sideMaterial) * MTC_MATERIAL_VEC4_ROWS + 23].z) > 0.5f;
        if (!matDoubleSided && xdot(candidateNormal, d) > 0.0f) continue;
      }
      h.hitNormal = candidateNormal;
      h.tMax = t;
      h.hitBary = bary;
      if (shadow) {
        if (kAlpha && alphaSmp &&
            !alphaPasses(*alphaScene, sideMaterial, triangleIndex, asi(r3.x) + vertexOffset,
                         asi(r3.y) + vertexOffset, asi(r3.z) + vertexOffset, bary, o + d * t, candidateNormal,
                         *alphaSmp)) {
          h.tMax = tMaxInit;
          continue;
        }
        found = true;
        return true;
      }
      h.triangleIndex = triangleIndex;
      h.insIdx = insIdx;
    }
    return false;
  }

  // Next instance entry of the current TLAS leaf (descending, as the WGSL's
  // leaf loop): the ray in instance space and its watertight-test shear.
  MTD bool enterInstance() {
    float4 rec = ld4(bvh + leafNode + 2 + io);
    io--;
    insIdx = asi(rec.x);
    int32_t blasRoot = asi(rec.y);
    const float4 *insv = ins + size_t(insIdx) * MTC_INSTANCE_VEC4_STRIDE;
    float4 insData = ld4(insv);
    uint32_t encoded = asu(insData.x);
    blasLayout = encoded >> 30;
    if (blasLayout != 0u && !(kGpuLayout && blasLayout == 2u)) return false;  // TinyBVH bvh4 / cwbvh are not consumed
    float4 c0 = ld4(insv + 1), c1 = ld4(insv + 2), c2 = ld4(insv + 3), c3 = ld4(insv + 4);
    o = xmat4(c0, c1, c2, c3, rayO, 1.0f);
    d = xmat4(c0, c1, c2, c3, rayD, 0.0f);
    linvD = traversalInverse(d);
    maxDim = maxDimension(vabs(d));
    shear = getShear(d, maxDim);
    blasOffset = int32_t(encoded & 0x3fffffffu);
    vertexOffset = asi(insData.y);
    sideMaterial = asi(insData.z) >> 8;
    blasTop = 0;
    stack[MTC_MAX_STACK] = blasRoot;
    return false;
  }
};

}  // namespace mt
