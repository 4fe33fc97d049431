// Device lights, environment, material resolve, next-event estimation with
// RIS + MIS, and the RGB integrator of the megakernel.  Function-by-function
// restatement of rayTrace.compute.ts, sampleMaterial.wgsl.ts,
// sampleLight.wgsl.ts, envMap.wgsl.ts, background.wgsl.ts and
// materialBuffer.wgsl.ts (paths relative to src/renderer/wgsl/).
#pragma once
#include "dev_bsdf.cuh"
#include "dev_trace.cuh"
#include "spectrum_cdf.h"

namespace mt {

MTD V3 kLuminance() { return {0.2126f, 0.7152f, 0.0722f}; }
MTD bool feature(const JobData &J, uint32_t bit) { return (J.u.scene_feature_flags & bit) != 0u; }
MTD bool useEnvmap(const JobData &J) { return feature(J, MTC_FEATURE_USE_ENVMAP) && J.s.env != nullptr; }
MTD bool isSpectral(const JobData &J) { return (J.s.flags & MTC_SCENE_SPECTRAL) != 0u; }

struct Ray { V3 o, d; };

// ------------------------------------------------------------ environment
// envMap.wgsl.ts:10-31
MTD float4 textureLinear(const float4 *tex, uint32_t w, uint32_t h, V2 uv) {
  float ux = uv.x * float(w) - 0.5f, uy = uv.y * float(h) - 0.5f;
  float fx = floorf(ux), fy = floorf(uy);
  float tx = ux - fx, ty = uy - fy;
  int ix = int(fx), iy = int(fy);
  int x0 = min(max(ix, 0), int(w) - 1), x1 = min(max(ix + 1, 0), int(w) - 1);
  int y0 = min(max(iy, 0), int(h) - 1), y1 = min(max(iy + 1, 0), int(h) - 1);
  float4 s1 = ld4(tex + size_t(y0) * w + x0), s2 = ld4(tex + size_t(y0) * w + x1);
  float4 s3 = ld4(tex + size_t(y1) * w + x0), s4 = ld4(tex + size_t(y1) * w + x1);
  auto mix4 = [](float4 a, float4 b, float t) {
    return make_float4(a.x * (1.0f - t) + b.x * t, a.y * (1.0f - t) + b.y * t, a.z * (1.0f - t) + b.z * t,
                       a.w * (1.0f - t) + b.w * t);
  };
  return mix4(mix4(s1, s2, tx), mix4(s3, s4, tx), ty);
}
// envMap.wgsl.ts:33-49
MTD V2 cartesianToEquirect(V3 p) {
  float phi = atan2f(-p.z, -p.x);
  if (phi < 0.0f) phi += TWOPI;
  float theta = acosf(clampf(p.y, -1.0f, 1.0f));
  return {phi * 0.5f * INVPI, theta * INVPI};
}
MTD V3 envRotCol(const JobData &J, int c) {
  const float *m = J.u.environment_rotation;
  return {m[c * 4 + 0], m[c * 4 + 1], m[c * 4 + 2]};
}
MTD V2 environmentUv(const JobData &J, V3 d) {
  return cartesianToEquirect({dot(envRotCol(J, 0), d), dot(envRotCol(J, 1), d), dot(envRotCol(J, 2), d)});
}
MTD float2 distAt(const JobData &J, int x, int y) { return __ldg(J.s.envDist + size_t(y) * (J.s.envW + 2) + x); }
// envMap.wgsl.ts:51-99
MTD float getEnvmapV(const JobData &J, float u, int &vOffset, V2 &pdf) {
  int left = 0, right = int(J.s.envH) + 1;
  while (left < right) {
    int mid = (left + right) >> 1;
    if (distAt(J, 0, mid).x <= u) left = mid + 1; else right = mid;
  }
  vOffset = left - 1;
  float2 s0 = distAt(J, 0, vOffset), s1 = distAt(J, 0, vOffset + 1);
  pdf.y = s0.y;
  return (float(vOffset) + (u - s0.x) / (s1.x - s0.x)) / float(J.s.envH);
}
MTD float getEnvmapU(const JobData &J, float u, int vOffset, V2 &pdf) {
  int left = 0, right = int(J.s.envW) + 1;
  while (left < right) {
    int mid = (left + right) >> 1;
    if (distAt(J, 1 + mid, vOffset).x <= u) left = mid + 1; else right = mid;
  }
  int uOffset = left - 1;
  float2 s0 = distAt(J, 1 + uOffset, vOffset), s1 = distAt(J, 1 + uOffset + 1, vOffset);
  pdf.x = s0.y;
  return (float(uOffset) + (u - s0.x) / (s1.x - s0.x)) / float(J.s.envW);
}
// envMap.wgsl.ts:103-141
MTD float envMapSolidAnglePdf(V2 partial, float v) {
  if (!(v > 0.0f && v < 1.0f)) return 0.0f;
  float sinTheta = sinf(fminf(v, 1.0f - v) * PI);
  return partial.x * partial.y * INVPI2 / (2.0f * sinTheta);
}
MTD V3 sampleEnvmap(const JobData &J, V2 rnd, V2 &uv, float &pdf) {
  V2 partial = {0.0f, 0.0f};
  int vOffset;
  uv.y = getEnvmapV(J, rnd.x, vOffset, partial);
  uv.x = getEnvmapU(J, rnd.y, vOffset, partial);
  float phi = uv.x * TWOPI, theta = uv.y * PI;
  float st, ct, sp, cp;
  sincosf(theta, &st, &ct);
  sincosf(phi, &sp, &cp);
  V3 dir = {-st * cp, ct, -st * sp};
  pdf = envMapSolidAnglePdf(partial, uv.y);
  return envRotCol(J, 0) * dir.x + envRotCol(J, 1) * dir.y + envRotCol(J, 2) * dir.z;
}
MTD float envMapPdf(const JobData &J, V2 uv) {
  int x = int(uv.x * float(J.s.envW)), y = int(uv.y * float(J.s.envH));
  x = min(max(x, 0), int(J.s.envW) - 1);
  y = min(max(y, 0), int(J.s.envH) - 1);
  return envMapSolidAnglePdf({distAt(J, 1 + x, y).y, distAt(J, 0, y).y}, uv.y);
}
// background.wgsl.ts:84-99 (no background map)
MTD float4 sampleSceneBackground(const JobData &J, V3 d) {
  if (J.u.background_flags & MTC_BACKGROUND_COLOR) {
    const float *c = J.u.background_color;
    return make_float4(c[0], c[1], c[2], c[3]);
  }
  if (useEnvmap(J)) return textureLinear(J.s.env, J.s.envW, J.s.envH, environmentUv(J, d));
  return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}
MTD V3 spectralFilter(V3 rgb, int channel) {
  if (channel == 0) return rgb;
  V3 f = v3(0.0f);
  setcomp(f, channel - 1, comp(rgb, channel - 1));
  return f;
}

// spectrum.ts:62-88: inverse CDFs of continuous wavelength sampling, one per
// RGB channel and one for r+g+b (generated by gen_spectrum_cdf.py).
static __constant__ float c_spectrumCdf[MT_SPECTRUM_CDF_SIZE] = {MT_SPECTRUM_CDF_VALUES};

// spectrum.ts:133-141 spectrumSample + spectrumIorWavelength: the refracting
// wavelength of a camera path that carries RGB channel `channel`.
MTD float spectrumCameraWavelength(uint32_t channel, float u) {
  const float *cdf = c_spectrumCdf + channel * (MT_SPECTRUM_BINS + 1);
  uint32_t low = 0, high = MT_SPECTRUM_BINS;
  while (high - low > 1u) {
    uint32_t middle = (low + high) >> 1;
    if (cdf[middle] <= u) low = middle; else high = middle;
  }
  float mass = cdf[low + 1] - cdf[low];
  float wavelength = 400.0f + 5.0f * (float(low) + (u - cdf[low]) / mass);
  if (wavelength >= 500.0f) return wavelength;
  return 500.0f - 25.0f * (1.0f - expf((wavelength - 500.0f) / 25.0f));
}

// sRGBToLinear / decodeMapColor (materialBuffer.wgsl.ts:258-265).
MTD float srgbToLinear(float c) {
  return c < 0.04045f ? c * 0.0773993808f : powf(c * 0.9478672986f + 0.0521327014f, 2.4f);
}
MTD V3 decodeMapColor(const DevScene &s, int idx, V3 c) {
  if (idx < 0 || uint32_t(idx) >= s.mapCount) return c;
  const float linear = ld4(s.maps + size_t(idx) * MTC_MAP_VEC4_ROWS + 2).y;
  if (int(rintf(linear)) % 2 == 1) return c;
  return {srgbToLinear(c.x), srgbToLinear(c.y), srgbToLinear(c.z)};
}

MTD V3 mulv(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }


// getMaterialEmission (materialBuffer.wgsl.ts:381-403): the packed emission
// times the sRGB-decoded emissive map and, for standard materials, the coat
// weight map's single coat passage.  `uv` is the caller's (the surface's
// scaled UV, or a light sample's unscaled one).
// getMapUvSet (materialBuffer.wgsl.ts:329-331): a map on UV set 1 samples the
// secondary coordinates.
MTD V2 mapUvSet(const DevScene &s, int idx, V2 uv, V2 uv1) {
  return ld4(s.maps + size_t(idx) * MTC_MAP_VEC4_ROWS + 2).x > 0.5f ? uv1 : uv;
}
static __device__ __noinline__ V3 materialEmission(const DevScene &s, const float4 *d, V2 uv, V2 uv1) {
  const float4 r3 = ld4(d + 3);
  V3 emission = xyz(r3);
  const int emissive = int(r3.w), coatWeightMap = int(ld4(d + 6).x);
  if (mapValid(s, r3.w)) {
    const float4 t = sampleMap(s, emissive, mapUvSet(s, emissive, uv, uv1));
    emission = mulv(emission, decodeMapColor(s, emissive, {t.x, t.y, t.z}));
  }
  if (mapValid(s, ld4(d + 6).x) && ld4(d).w == 0.0f) {
    const float4 r16 = ld4(d + 16);
    const float w = clampf(r16.w, 0.0f, 1.0f) * sampleMap(s, coatWeightMap, mapUvSet(s, coatWeightMap, uv, uv1)).x;
    const V3 c = {sqrtf(fmaxf(r16.x, 0.0f)), sqrtf(fmaxf(r16.y, 0.0f)), sqrtf(fmaxf(r16.z, 0.0f))};
    emission = mulv(emission, V3{(1.0f - w) + c.x * w, (1.0f - w) + c.y * w, (1.0f - w) + c.z * w});
  }
  return emission;
}
// Any texture slot getMaterial samples (emissive, base color, alpha,
// transmission, metallic-roughness, roughness, metalness, thin film, coat
// weight, coat roughness, fuzz color, fuzz roughness, specular weight,
// specular color).
MTD bool materialHasMaps(float4 r2, float4 r3, float4 r6, float4 r9, float4 r18, float4 r19, float4 r21,
                         float4 r22) {
  return fmaxf(fmaxf(fmaxf(r2.z, r2.w), fmaxf(r3.w, r6.x)), fmaxf(fmaxf(r6.y, r6.w), fmaxf(r9.y, r9.w))) >= 0.0f ||
         fmaxf(fmaxf(r18.w, r19.w), fmaxf(fmaxf(r21.w, r22.x), fmaxf(r22.y, r22.z))) >= 0.0f;
}
// The texture block of getMaterial (materialBuffer.wgsl.ts:79-139, slots of
// materialTextureSlots.ts), in the reference's order; the alpha-mode
// resolution that sits between the alpha and transmission maps touches only
// alpha, so the caller resolves it after this.  Out of line: only materials
// with maps call it.
static __device__ __noinline__ void applyMaterialMaps(const DevScene &s, const float4 *d, V2 uv, V2 uv1,
                                                      Material &m) {
  m.emission = materialEmission(s, d, uv, uv1);
  const float4 r2 = ld4(d + 2), r5 = ld4(d + 5), r6 = ld4(d + 6), r9 = ld4(d + 9), r22 = ld4(d + 22);
  auto slot = [&](float index, float4 &t) {
    if (!mapValid(s, index)) return false;
    t = sampleMap(s, int(index), mapUvSet(s, int(index), uv, uv1));
    return true;
  };
  float4 t;
  if (slot(r2.z, t)) {
    m.baseColor = mulv(m.baseColor, decodeMapColor(s, int(r2.z), {t.x, t.y, t.z}));
    // mapAlphaUsageConstants (materialConstants.ts:2): 3 transmission, 2 alpha
    if (r5.w == 3.0f) m.transmissionWeight = 1.0f - t.w;
    else if (r5.w == 2.0f) m.alpha *= t.w;
  }
  if (slot(r22.z, t)) m.alpha *= t.y;
  if (slot(r9.w, t)) m.transmissionWeight *= t.x;
  if (slot(r2.w, t)) {
    m.baseMetalness *= t.z;
    m.specularRoughness *= t.y;
  }
  if (slot(r22.x, t)) m.specularRoughness *= t.y;
  if (slot(r22.y, t)) m.baseMetalness *= t.z;
  if (slot(r9.y, t)) {
    // thinFilmTextureSample (materialTextureSlots.ts:214-228)
    const float4 r25 = ld4(d + 25);
    if (r25.z == 0.0f && r25.w == 0.0f) {
      m.thinFilmThickness *= t.x;
    } else {
      const int channel = int(r25.w);
      const float k = channel == 0 ? t.x : channel == 1 ? t.y : channel == 2 ? t.z : t.w;
      m.thinFilmThickness = (r25.z * (1.0f - k) + r5.z * k) * 1000.0f;
    }
  }
  if (slot(r6.x, t)) m.coatWeight *= t.x;
  if (slot(r6.y, t)) m.coatRoughness *= t.y;
  if (slot(r6.w, t)) m.fuzzColor = mulv(m.fuzzColor, decodeMapColor(s, int(r6.w), {t.x, t.y, t.z}));
  if (slot(ld4(d + 18).w, t)) m.fuzzRoughness *= t.w;
  if (slot(ld4(d + 19).w, t)) m.specularWeight *= t.w;
  if (slot(ld4(d + 21).w, t)) m.specularColor = mulv(m.specularColor, decodeMapColor(s, int(ld4(d + 21).w), {t.x, t.y, t.z}));
}

// ------------------------------------------------------------------ lights
struct Light {
  V3 position; float litType; V3 emission; float area; V3 u; float radiusOrSpread; V3 v; float textureIndex;
  float selectionPmf;
};
MTD Light loadLight(const JobData &J, int i) {
  const float4 *L = J.s.lights + size_t(i) * MTC_LIGHT_VEC4_ROWS;
  float4 a = ld4(L), b = ld4(L + 1), c = ld4(L + 2), d = ld4(L + 3), e = ld4(L + 4);
  return {xyz(a), a.w, xyz(b), b.w, xyz(c), c.w, xyz(d), d.w, e.x};
}
struct LightSample {
  V3 normal, emission, direction;
  float dist, pdf, selectionPmf;
  bool isDelta;
  uint32_t sourceType, sourceIndex;
};
MTD LightSample zeroLightSample() {
  LightSample ls;
  ls.normal = v3(0.0f); ls.emission = v3(0.0f); ls.direction = v3(0.0f);
  ls.dist = 0.0f; ls.pdf = 0.0f; ls.selectionPmf = 0.0f; ls.isDelta = false; ls.sourceType = 0; ls.sourceIndex = 0;
  return ls;
}
// intersect.wgsl.ts:894-949
MTD float intersectSphere(float rad, V3 pos, const Ray &r) {
  V3 op = pos - r.o;
  float b = dot(op, r.d);
  float det = b * b - dot(op, op) + rad * rad;
  if (det < 0.0f) return INF;
  det = sqrtf(det);
  float t1 = b - det;
  if (t1 > 0.001f) return t1;
  float t2 = b + det;
  if (t2 > 0.001f) return t2;
  return INF;
}
MTD float intersectRect(V3 pos, V3 u, V3 v, V3 n, const Ray &r) {
  float dt = dot(r.d, n);
  float t = (dot(n, pos) - dot(n, r.o)) / dt;
  if (t > EPS) {
    V3 p = r.o + r.d * t;
    V3 vi = p - pos;
    float a1 = dot(u / dot(u, u), vi);
    if (a1 >= 0.0f && a1 <= 1.0f) {
      float a2 = dot(v / dot(v, v), vi);
      if (a2 >= 0.0f && a2 <= 1.0f) return t;
    }
  }
  return INF;
}
MTD float sphereSolidAnglePdf(V3 origin, V3 center, float radius) {
  float cd = distance(origin, center);
  if (cd <= radius) return INV4PI;
  float s2 = fminf(1.0f, radius * radius / (cd * cd));
  float ct = sqrtf(fmaxf(0.0f, 1.0f - s2));
  return 1.0f / fmaxf(TWOPI * (s2 / (1.0f + ct)), 1e-8f);
}
MTD float spotEmissionMultiplier(const Light &L, V3 lightToSurface) {
  float cosTheta = dot(normalize(L.u), lightToSurface);
  float cone = cosTheta >= L.v.x ? 1.0f : 0.0f;
  if (L.v.y > L.v.x + 1e-6f) cone = smoothstepf(L.v.x, L.v.y, cosTheta);
  return cone;
}
// intersect.wgsl.ts:976-1131
MTD float intersectLight(const Ray &r, const Light &L, LightSample &ls) {
  float d = INF;
  ls.direction = r.d; ls.normal = -r.d; ls.dist = INF; ls.pdf = 0.0f; ls.emission = v3(0.0f); ls.isDelta = false;
  V3 u = L.u, v = L.v;
  int type = int(L.litType);
  if (type == MTC_LIGHT_RECT) {
    V3 pos = L.position - u * 0.5f - v * 0.5f;
    V3 normal = normalize(cross(u, v));
    if (dot(normal, r.d) > 0.0f) return INF;
    d = intersectRect(pos, u, v, normal, r);
    if (d < 0.0f) d = INF;
    else {
      float cosTheta = dot(-r.d, normal);
      if (cosTheta >= cosf(L.radiusOrSpread * PI / 2.0f)) {
        ls.direction = r.d; ls.normal = normal; ls.dist = d;
        ls.pdf = (d * d) / (L.area * cosTheta);
        ls.emission = L.emission; ls.isDelta = false;
      } else d = INF;
    }
  } else if (type == MTC_LIGHT_DISK) {
    V3 normal = normalize(cross(u, v));
    if (dot(normal, r.d) >= 0.0f) return INF;
    d = dot(L.position - r.o, normal) / dot(normal, r.d);
    V3 hit = r.o + r.d * d - L.position;
    float radius = fmaxf(length(u), 1e-8f);
    if (d <= EPS || dot(hit, hit) > radius * radius) return INF;
    float cosine = dot(-r.d, normal);
    ls.direction = r.d; ls.normal = normal; ls.dist = d;
    ls.pdf = d * d / fmaxf(L.area * cosine, 1e-8f);
    ls.emission = L.emission;
  } else if (type == MTC_LIGHT_CYLINDER) {
    V3 axis = normalize(u);
    float halfLength = 0.5f * length(u);
    V3 oc = r.o - L.position;
    V3 rd = r.d - axis * dot(r.d, axis);
    V3 od = oc - axis * dot(oc, axis);
    float a = dot(rd, rd), b = dot(od, rd), c = dot(od, od) - L.radiusOrSpread * L.radiusOrSpread;
    float disc = b * b - a * c;
    if (a <= 1e-12f || disc < 0.0f) return INF;
    float root = sqrtf(disc);
    float nearT = (-b - root) / a, farT = (-b + root) / a;
    d = nearT > EPS ? nearT : farT;
    float axial = dot(oc + r.d * d, axis);
    if (d <= EPS || fabsf(axial) > halfLength) return INF;
    V3 normal = normalize(r.o + r.d * d - L.position - axis * axial);
    float cosine = dot(-r.d, normal);
    if (cosine <= 0.0f) return INF;
    ls.direction = r.d; ls.normal = normal; ls.dist = d;
    ls.pdf = d * d / fmaxf(L.area * cosine, 1e-8f);
    ls.emission = L.emission;
  } else if (type == MTC_LIGHT_SPHERE || type == MTC_LIGHT_SPOT) {
    if (L.radiusOrSpread <= 0.0f) {
      V3 toPoint = L.position - r.o;
      float proj = dot(toPoint, r.d);
      V3 perp = toPoint - r.d * proj;
      if (proj <= EPS || dot(perp, perp) > 1e-8f) return INF;
      d = proj;
      ls.direction = r.d; ls.normal = -r.d; ls.dist = d; ls.pdf = 1.0f; ls.isDelta = true;
    } else {
      d = intersectSphere(L.radiusOrSpread, L.position, r);
      ls.isDelta = false;
      if (type == MTC_LIGHT_SPHERE && d > 0.0f && d != INF) {
        ls.direction = r.d; ls.dist = d;
        ls.normal = normalize(r.o + r.d * d - L.position);
        ls.pdf = sphereSolidAnglePdf(r.o, L.position, L.radiusOrSpread);
      }
    }
    if (type == MTC_LIGHT_SPHERE) {
      if (d < 0.0f) d = INF;
      else {
        ls.direction = r.d; ls.dist = d;
        ls.emission = L.radiusOrSpread <= 0.0f ? L.emission / fmaxf(d * d, 1e-8f) : L.emission;
      }
    } else if (d != INF) {
      V3 hitPt = r.o + r.d * d;
      float mult = spotEmissionMultiplier(L, normalize(r.o - hitPt));
      if (mult <= 0.0f) return INF;
      if (L.radiusOrSpread > 0.0f) {
        ls.direction = r.d; ls.dist = d;
        ls.normal = normalize(r.o + r.d * d - L.position);
        ls.pdf = sphereSolidAnglePdf(r.o, L.position, L.radiusOrSpread);
      }
      ls.emission = L.emission * mult * (L.radiusOrSpread <= 0.0f ? 1.0f / fmaxf(d * d, 1e-8f) : 1.0f);
    }
  } else {
    d = INF;
  }
  return d;
}
// sampleLight.wgsl.ts:10-87
MTD void lightSampleSphere(const Light &L, V3 p, V2 rnd, LightSample &ls) {
  V3 co = L.position - p;
  float cd = length(co);
  if (L.radiusOrSpread <= 0.0f) {
    if (cd <= 1e-6f) {
      ls.direction = {0, 0, 1}; ls.normal = {0, 0, -1}; ls.dist = 0; ls.pdf = 1; ls.emission = v3(0.0f); ls.isDelta = true;
      return;
    }
    ls.direction = co / cd; ls.normal = -ls.direction; ls.dist = cd; ls.pdf = 1.0f;
    ls.emission = L.emission / fmaxf(cd * cd, 1e-8f); ls.isDelta = true;
    return;
  }
  float radius = fmaxf(L.radiusOrSpread, 1e-6f);
  ls.isDelta = false;
  V3 sd;
  if (cd <= radius) {
    float z = 1.0f - 2.0f * rnd.x;
    float radial = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    float sa, ca;
    sincosf(TWOPI * rnd.y, &sa, &ca);
    sd = {radial * ca, radial * sa, z};
    ls.pdf = INV4PI;
  } else {
    V3 axis = co / cd;
    float s2 = fminf(1.0f, radius * radius / (cd * cd));
    float ctm = sqrtf(fmaxf(0.0f, 1.0f - s2));
    float omctm = s2 / (1.0f + ctm);
    float omct = rnd.x * omctm;
    float ct = 1.0f - omct;
    float st = sqrtf(fmaxf(0.0f, omct * (2.0f - omct)));
    float sa, ca;
    sincosf(TWOPI * rnd.y, &sa, &ca);
    V3 t, b;
    orthonormalBasis(axis, t, b);
    sd = axis * ct + t * (st * ca) + b * (st * sa);
    ls.pdf = 1.0f / fmaxf(TWOPI * omctm, 1e-8f);
  }
  float cp = dot(sd, co);
  float disc = cp * cp - dot(co, co) + radius * radius;
  float nearT = cp - sqrtf(fmaxf(0.0f, disc));
  float farT = cp + sqrtf(fmaxf(0.0f, disc));
  ls.dist = nearT > 1e-6f ? nearT : farT;
  ls.direction = sd;
  ls.normal = normalize(p + sd * ls.dist - L.position);
  ls.emission = L.emission;
}
// sampleLight.wgsl.ts:108-161 (no light texture)
MTD void lightSampleRect(const Light &L, V3 p, V2 rnd, LightSample &ls) {
  V3 normal = normalize(cross(L.u, L.v));
  V3 lowerLeft = L.position - (L.u + L.v) * 0.5f;
  float spread = clampf(L.radiusOrSpread, 0.0f, 1.0f);
  if (spread <= 0.001f) {
    float pd = dot(normal, p - L.position);
    V3 rel = p - normal * pd - lowerLeft;
    float w = length(L.u), h = length(L.v);
    V2 uv = {dot(rel, L.u / w) / w, dot(rel, L.v / h) / h};
    if (pd <= 0.0f || uv.x < 0.0f || uv.y < 0.0f || uv.x > 1.0f || uv.y > 1.0f) {
      ls.emission = v3(0.0f); ls.pdf = 0.0f; return;
    }
    ls.direction = -normal; ls.dist = pd; ls.normal = normal; ls.emission = L.emission; ls.pdf = 1.0f; ls.isDelta = true;
    return;
  }
  V3 sp = lowerLeft + L.u * rnd.x + L.v * rnd.y;
  V3 off = sp - p;
  float d2 = dot(off, off);
  ls.dist = sqrtf(d2);
  ls.direction = off / ls.dist;
  ls.normal = normal;
  float ec = dot(-ls.direction, normal);
  if (ec <= 0.0f || ec < cosf(0.5f * PI * spread)) { ls.emission = v3(0.0f); ls.pdf = 0.0f; return; }
  ls.emission = L.emission;
  ls.pdf = d2 / fmaxf(L.area * ec, 1e-8f);
}
// sampleLight.wgsl.ts:163-195
MTD void lightSampleDiskOrCylinder(const Light &L, V3 p, V2 rnd, LightSample &ls, bool cylinder) {
  V3 sp, normal;
  if (!cylinder) {
    float r = sqrtf(rnd.x);
    float sa, ca;
    sincosf(TWOPI * rnd.y, &sa, &ca);
    sp = L.position + L.u * (r * ca) + L.v * (r * sa);
    normal = normalize(cross(L.u, L.v));
  } else {
    V3 axis = normalize(L.u), r0 = normalize(L.v);
    V3 r1 = normalize(cross(axis, r0));
    float sa, ca;
    sincosf(TWOPI * rnd.y, &sa, &ca);
    normal = r0 * ca + r1 * sa;
    sp = L.position + L.u * (rnd.x - 0.5f) + normal * L.radiusOrSpread;
  }
  V3 off = sp - p;
  float d2 = dot(off, off);
  ls.dist = sqrtf(d2);
  ls.direction = off / fmaxf(ls.dist, 1e-8f);
  ls.normal = normal;
  float ec = dot(-ls.direction, normal);
  if (ec <= 0.0f) { ls.emission = v3(0.0f); ls.pdf = 0.0f; return; }
  ls.emission = L.emission;
  ls.pdf = d2 / fmaxf(L.area * ec, 1e-8f);
}
// sampleLight.wgsl.ts:197-244
MTD void sampleAnalyticLight(const Light &L, V3 p, V2 rnd, LightSample &ls) {
  int type = int(L.litType);
  if (type == MTC_LIGHT_RECT) { lightSampleRect(L, p, rnd, ls); return; }
  if (type == MTC_LIGHT_SPHERE) { lightSampleSphere(L, p, rnd, ls); return; }
  if (type == MTC_LIGHT_SPOT) {
    lightSampleSphere(L, p, rnd, ls);
    V3 surf = p + ls.direction * ls.dist;
    ls.emission *= spotEmissionMultiplier(L, normalize(p - surf));
    return;
  }
  if (type == MTC_LIGHT_DIRECTIONAL) {
    ls.direction = normalize(-L.u); ls.normal = -ls.direction; ls.emission = L.emission;
    ls.dist = INF; ls.pdf = 1.0f; ls.isDelta = true;
    return;
  }
  if (type == MTC_LIGHT_DISK) { lightSampleDiskOrCylinder(L, p, rnd, ls, false); return; }
  if (type == MTC_LIGHT_CYLINDER) lightSampleDiskOrCylinder(L, p, rnd, ls, true);
}
// sampleLight.wgsl.ts:319-357
MTD void sampleEmissiveTriangle(const JobData &J, int index, V3 p, V2 rnd, LightSample &ls) {
  const float4 *t = J.s.lightData + size_t(index) * 6;
  float4 a = ld4(t), b = ld4(t + 1), c = ld4(t + 2);
  V3 p0 = xyz(a), p1 = xyz(b), p2 = xyz(c);
  float su = sqrtf(rnd.x);
  V3 bc = {1.0f - su, su * (1.0f - rnd.y), su * rnd.y};
  V3 lp = p0 * bc.x + p1 * bc.y + p2 * bc.z;
  V3 normal = normalize(cross(p1 - p0, p2 - p0));
  ls.direction = lp - p;
  ls.dist = length(ls.direction);
  if (ls.dist <= EPS) { ls.emission = v3(0.0f); ls.pdf = 0.0f; return; }
  ls.direction /= ls.dist;
  ls.normal = normal;
  float cl = dot(normal, -ls.direction);
  if (cl <= 0.0f) { ls.emission = v3(0.0f); ls.pdf = 0.0f; return; }
  // getMaterialEmission at the sampled point's unscaled UV (sampleLight.wgsl.ts:356-358)
  const float4 *md = J.s.mats + size_t(int(c.w)) * MTC_MATERIAL_VEC4_ROWS;
  const float4 r3 = ld4(md + 3);
  if (mapValid(J.s, r3.w) || mapValid(J.s, ld4(md + 6).x)) {
    const float4 d3 = ld4(t + 3), d4 = ld4(t + 4), d5 = ld4(t + 5);  // uv0 uv1 | uv2 uv1_0 | uv1_1 uv1_2
    ls.emission = materialEmission(J.s, md, V2{bc.x * d3.x + bc.y * d3.z + bc.z * d4.x, bc.x * d3.y + bc.y * d3.w + bc.z * d4.y},
                                   V2{bc.x * d4.z + bc.y * d5.x + bc.z * d5.z, bc.x * d4.w + bc.y * d5.y + bc.z * d5.w});
  } else {
    ls.emission = xyz(r3);
  }
  ls.selectionPmf = a.w;
  ls.pdf = a.w * (ls.dist * ls.dist) / fmaxf(b.w * cl, 1e-8f);
}
// sampleLight.wgsl.ts:359-420 sampleLightChoiceTable
MTD void sampleLightChoiceTable(const JobData &J, V3 p, V3 rnd, LightSample &ls) {
  ls.emission = v3(0.0f); ls.pdf = 0.0f; ls.selectionPmf = 0.0f; ls.dist = INF; ls.isDelta = false;
  ls.sourceType = 0; ls.sourceIndex = 0xffffffffu;
  int count = J.u.light_choice_count;
  if (count <= 0) return;
  float scaled = rnd.z * float(count);
  int column = min(int(scaled), count - 1);
  float4 cc = ld4(J.s.lightData + J.u.light_choice_texel_offset + column);
  int selected = fractf(scaled) < cc.x ? column : asi(cc.y);
  float4 ch = ld4(J.s.lightData + J.u.light_choice_texel_offset + selected);
  int type = asi(ch.z), src = asi(ch.w);
  if (useEnvmap(J) && type == MTC_CHOICE_ENVIRONMENT) {
    ls.sourceType = 0; ls.sourceIndex = uint32_t(src);
    V2 uv;
    float pdf;
    ls.direction = sampleEnvmap(J, {rnd.x, rnd.y}, uv, pdf);
    ls.pdf = pdf;
    ls.emission = xyz(textureLinear(J.s.env, J.s.envW, J.s.envH, uv));
    ls.dist = INF;
    ls.selectionPmf = J.u.env_light_pmf;
    ls.pdf *= J.u.env_light_pmf;
  } else if (type == MTC_CHOICE_ANALYTIC) {
    ls.sourceType = 2; ls.sourceIndex = uint32_t(src);
    Light L = loadLight(J, src);
    sampleAnalyticLight(L, p, {rnd.x, rnd.y}, ls);
    ls.selectionPmf = L.selectionPmf;
    ls.pdf *= L.selectionPmf;
  } else if (type == MTC_CHOICE_EMISSIVE_TRIANGLE) {
    ls.sourceType = 1; ls.sourceIndex = uint32_t(src);
    sampleEmissiveTriangle(J, src, p, {rnd.x, rnd.y}, ls);
  }
}

// --------------------------------------------------------------- material
// materialBuffer.wgsl.ts:170-257 getMaterial with its texture block
MTD void getMaterial(const JobData &J, int materialIndex, int instanceIndex, V2 uv, V2 uv1, V3 vertexColor,
                     Material &m) {
  // A miss keeps the previous hit's indices (zero before the first hit);
  // clamp so an empty or single-material scene never reads past its buffers.
  if (materialIndex < 0 || uint32_t(materialIndex) >= J.s.matCount) materialIndex = 0;
  if (uint32_t(max(instanceIndex, 0)) >= J.s.insCount) instanceIndex = -1;
  const float4 *d = J.s.mats + size_t(materialIndex) * MTC_MATERIAL_VEC4_ROWS;
  float4 r0 = ld4(d), r1 = ld4(d + 1), r2 = ld4(d + 2), r3 = ld4(d + 3), r4 = ld4(d + 4), r5 = ld4(d + 5);
  float4 r9 = ld4(d + 9), r10 = ld4(d + 10), r11 = ld4(d + 11), r12 = ld4(d + 12), r14 = ld4(d + 14);
  float4 r15 = ld4(d + 15), r16 = ld4(d + 16), r17 = ld4(d + 17), r18 = ld4(d + 18), r20 = ld4(d + 20);
  float4 r21 = ld4(d + 21), r22 = ld4(d + 22), r23 = ld4(d + 23), r24 = ld4(d + 24), r25 = ld4(d + 25);
  float4 r6 = ld4(d + 6), r19 = ld4(d + 19);
  m.baseColor = xyz(r0);
  m.materialType = int(r0.w);
  m.specularRoughness = r1.x;
  m.baseMetalness = r2.x;
  m.specularAnisotropy = clampf(r2.y, 0.0f, 1.0f);
  m.emission = xyz(r3);
  m.inside = false;
  m.specularIor = r4.x;
  m.transmissionWeight = r4.y;
  m.thinWalled = r4.w > 0.5f;
  m.bevel = r5.x;
  m.transmissionDispersionScale = r5.y;
  m.dispersionAbbeNumber = fmaxf(r18.y, 1e-6f);
  m.mediumExtinction = vmax(xyz(r20), v3(0.0f));
  m.mediumScattering = vmax(xyz(r21), v3(0.0f));
  m.mediumAnisotropy = clampf(r20.w, -1.0f, 1.0f);
  m.mediumType = maxc(m.mediumExtinction) > 0.0f ? 1 : 0;
  m.alpha = r9.x;
  m.alphaMode = int(r23.w);
  m.thinFilmThickness = r5.z * 1000.0f;
  m.thinFilmIor = r9.z;
  m.thinFilmWeight = feature(J, MTC_FEATURE_HAS_THIN_FILM) ? clampf(r18.x, 0.0f, 1.0f) : 0.0f;
  m.baseWeight = clampf(r10.x, 0.0f, 1.0f);
  m.diffuseRoughness = clampf(r10.y, 0.0f, 1.0f);
  m.specularWeight = fmaxf(r10.z, 0.0f);
  m.specularColor = vmax(xyz(r11), v3(0.0f));
  m.subsurfaceWeight = feature(J, MTC_FEATURE_HAS_SUBSURFACE) ? clampf(r10.w, 0.0f, 1.0f) : 0.0f;
  m.subsurfaceColor = vmax(xyz(r14), v3(0.0f));
  m.transmissionColor = vmax(xyz(r12), v3(0.0f));
  m.fuzzWeight = feature(J, MTC_FEATURE_HAS_FUZZ) ? clampf(r11.w, 0.0f, 1.0f) : 0.0f;
  m.fuzzColor = vmax(xyz(r15), v3(0.0f));
  m.fuzzRoughness = clampf(r15.w, 0.0f, 1.0f);
  m.coatWeight = feature(J, MTC_FEATURE_HAS_COAT) ? clampf(r16.w, 0.0f, 1.0f) : 0.0f;
  m.coatColor = vmax(xyz(r16), v3(0.0f));
  m.coatRoughness = clampf(r17.x, ROUGHNESS_MIN, 1.0f);
  m.coatAnisotropy = clampf(r17.y, 0.0f, 1.0f);
  m.coatIor = fmaxf(r17.z, 1.0f);
  m.coatDarkening = clampf(r17.w, 0.0f, 1.0f);
  if (materialHasMaps(r2, r3, r6, r9, r18, r19, r21, r22)) applyMaterialMaps(J.s, d, uv, uv1, m);
  if (m.alphaMode == 0) m.alpha = 1.0f;
  else if (m.alphaMode == 1) m.alpha = m.alpha >= r22.w ? 1.0f : 0.0f;
  m.anisotropyDirection = {1.0f, 0.0f};
  m.anisotropyDirectionEnabled = r24.y != 0.0f;
  m.coatAnisotropyRotation = r25.x;
  if (r25.y > 0.5f && m.specularAnisotropy > 0.0f) {
    float roughness = clampf(m.specularRoughness, 0.0f, 1.0f), strength = m.specularAnisotropy;
    float u = roughness * roughness;
    float a = u + (1.0f - u) * strength * strength;
    if (a == 0.0f) { m.specularRoughness = 0.0f; m.specularAnisotropy = 0.0f; }
    else {
      m.specularRoughness = powf((a * a + u * u) * 0.5f, 0.25f);
      m.specularAnisotropy = clampf(1.0f - u / a, 0.0f, 1.0f);
    }
  }
  if (m.anisotropyDirectionEnabled) {
    float st, ct;
    sincosf(r24.y, &st, &ct);
    V2 dd = m.anisotropyDirection;
    m.anisotropyDirection = {ct * dd.x - st * dd.y, st * dd.x + ct * dd.y};
  }
  if (m.coatWeight > 0.0f && m.coatRoughness > 0.0f) {
    float br2 = m.specularRoughness * m.specularRoughness;
    float cr2 = m.coatRoughness * m.coatRoughness;
    m.specularRoughness = mixf(m.specularRoughness, powf(fminf(1.0f, br2 * br2 + 2.0f * cr2 * cr2), 0.25f), m.coatWeight);
  }
  V3 color = v3(1.0f);
  if (instanceIndex >= 0) color = xyz(ld4(J.s.ins + size_t(instanceIndex) * MTC_INSTANCE_VEC4_STRIDE + 9));
  color = mulv(color, vertexColor);  // getInstanceColor(instanceIndex) * vertexColor
  m.baseColor *= color;
  if (m.materialType == 2) m.emission *= color;
  m.specularRoughness = clampf(m.specularRoughness, ROUGHNESS_MIN, 1.0f);
  m.baseMetalness = clampf(m.baseMetalness, 0.0f, 1.0f);
  V2 a = roughnessToAlpha(m.specularRoughness, m.specularAnisotropy);
  m.alphaX = a.x;
  m.alphaY = a.y;
  m.directionTangent = v3(0.0f); m.directionBitangent = v3(0.0f);
  m.geometryTangent = v3(0.0f); m.geometryBitangent = v3(0.0f);
  m.relativeIor = 0.0f;
}

// ------------------------------------------------------------- surface hit
struct SurfaceInteraction {
  V3 position; bool albedoSampled;
  V3 normal, vertexNormal, shadowOffset, faceNormal; bool hit;
  int32_t triangleIndex, instanceIndex, materialIndex;
  float wavelength; int32_t spectralChannel;
  int32_t mediumType; V3 mediumExtinction, mediumScattering; float mediumAnisotropy;
};

// getMatNormal (materialBuffer.wgsl.ts:377-418): the tangent frame from the
// triangle's position and UV differences (co-tangent construction), or a
// fixed-axis frame when the UVs have no gradient; the map's xy scaled by the
// material's normalMapScale.  Local space.  Out of line: only materials with
// a normal map call it.
static __device__ __noinline__ V3 applyNormalMap(const DevScene &s, int idx, float2 scale, V2 uv, V3 normal, V3 dp1,
                                                 V3 dp2, V2 duv1, V2 duv2) {
  V3 dp2perp = cross(dp2, normal), dp1perp = cross(normal, dp1);
  V3 dpdu = dp2perp * duv1.x + dp1perp * duv2.x;
  V3 dpdv = dp2perp * duv1.y + dp1perp * duv2.y;
  float g2 = fmaxf(dot(dpdu, dpdu), dot(dpdv, dpdv));
  if (g2 > 1e-12f) {
    float invmax = rsqrtf(g2);
    dpdu = dpdu * invmax;
    dpdv = dpdv * invmax;
  } else {
    V3 axis = fabsf(normal.z) < 0.999f ? V3{0.0f, 0.0f, 1.0f} : V3{0.0f, 1.0f, 0.0f};
    dpdu = normalize(cross(axis, normal));
    dpdv = cross(normal, dpdu);
  }
  float4 t = sampleMap(s, idx, uv);
  V3 n = {2.0f * t.x - 1.0f, 2.0f * t.y - 1.0f, 2.0f * t.z - 1.0f};
  n = normalize(V3{n.x * scale.x, n.y * scale.y, n.z});
  return normalize(dpdu * n.x + dpdv * n.y + normal * n.z);
}

// fetchAttributes + completeSurfaceInteraction (intersect.wgsl.ts:1233-1419,
// 1539-1601) for compact vertices with an optional primary UV pair (no
// tangent words, no UV projection).
// The surface's texture coordinates and vertex color, which only the
// material fetch reads.  They live beside the path sample (SpectralState)
// rather than in its SurfaceInteraction, so the wavefront's per-step copy of
// a slot's path sample stays as small as before textures.
struct SurfaceTexcoords {
  V2 uv;           // primary UV times the material's uvScale (0 without UVs)
  V2 uv1;          // secondary UV times uvScale (the primary set without UV1 words)
  V3 vertexColor;  // interpolated vertex color (white without colors)
};

// The attribute half of fetchAttributes (intersect.wgsl.ts:1250-1322,
// 1408-1418) that only scenes with UVs, vertex colors, maps or UV projections
// need: interpolated (or projected) UV sets times the instance material's
// `r7` uvScale, the vertex color, and the normal map of `material`, whose
// bent local normal goes to `mapped` (returns whether one applied).  Out of
// line, so scenes without such data keep a lean surface completion.
static __device__ __noinline__ bool surfaceTexcoords(const DevScene &s, int32_t material, float4 r7, int32_t i0,
                                                     int32_t i1, int32_t i2, V3 bary, V3 position, V3 normal,
                                                     V3 p0, V3 p1, V3 p2, SurfaceTexcoords &tex, V3 &mapped) {
  V2 uv0 = {0.0f, 0.0f}, uv1 = uv0, uv2 = uv0;
  if (s.vuvOff) {
    auto vuv = [&](int32_t i) {
      const uint32_t *w = s.attr + size_t(i) * s.vstride + s.vuvOff;
      return V2{asf(__ldg(w)), asf(__ldg(w + 1))};
    };
    uv0 = vuv(i0); uv1 = vuv(i1); uv2 = vuv(i2);
  }
  tex.vertexColor = v3(1.0f);
  if (s.vcolorOff) {
    // vertexColor (vertexAttributes.wgsl.ts:38-43): f32x3, or unpack4x8unorm
    auto vcol = [&](int32_t i) {
      const uint32_t *w = s.attr + size_t(i) * s.vstride + s.vcolorOff;
      if (s.vcolorFloat) return V3{asf(__ldg(w)), asf(__ldg(w + 1)), asf(__ldg(w + 2))};
      const uint32_t c = __ldg(w);
      return V3{float(c & 255u) / 255.0f, float((c >> 8) & 255u) / 255.0f, float((c >> 16) & 255u) / 255.0f};
    };
    const V3 c0 = vcol(i0), c1 = vcol(i1), c2 = vcol(i2);
    tex.vertexColor = c0 * bary.x + c1 * bary.y + c2 * bary.z;
  }
  // UV projection (intersect.wgsl.ts:1311-1322) from the local position and
  // normal; triplanar UVs repeat.
  const int projection = int(r7.x);
  V2 uv = {bary.x * uv0.x + bary.y * uv1.x + bary.z * uv2.x, bary.x * uv0.y + bary.y * uv1.y + bary.z * uv2.y};
  // vertexUv1 reads UV1_OFF, which aliases UV_OFF without secondary words
  V2 second = uv;
  if (s.vuv1Off) {
    auto vuv1 = [&](int32_t i) {
      const uint32_t *w = s.attr + size_t(i) * s.vstride + s.vuv1Off;
      return V2{asf(__ldg(w)), asf(__ldg(w + 1))};
    };
    const V2 a = vuv1(i0), b = vuv1(i1), c = vuv1(i2);
    second = {bary.x * a.x + bary.y * b.x + bary.z * c.x, bary.x * a.y + bary.y * b.y + bary.z * c.y};
  }
  if (projection > 0) {
    uv = projectUV(projection, position, normal);
    second = uv;
  }
  tex.uv = {uv.x * r7.z, uv.y * r7.w};
  tex.uv1 = {second.x * r7.z, second.y * r7.w};
  if (projection == 3) tex.uv = {tex.uv.x - floorf(tex.uv.x), tex.uv.y - floorf(tex.uv.y)};
  const float4 r1 = ld4(s.mats + size_t(material) * MTC_MATERIAL_VEC4_ROWS + 1);
  if (!mapValid(s, r1.y)) return false;
  mapped = applyNormalMap(s, int(r1.y), make_float2(r1.z, r1.w), tex.uv, normal, p0 - p2, p1 - p2,
                          V2{uv0.x - uv2.x, uv0.y - uv2.y}, V2{uv1.x - uv2.x, uv1.y - uv2.y});
  return true;
}

MTD void completeSurfaceInteraction(const JobData &J, SurfaceInteraction &si, SurfaceTexcoords &tex,
                                    const TraversalHit &h, V3 rayO, V3 rayD) {
  const DevScene &s = J.s;
  const float4 *insv = s.ins + size_t(h.insIdx) * MTC_INSTANCE_VEC4_STRIDE;
  float4 insData = ld4(insv);
  float4 w0 = ld4(insv + 1), w1 = ld4(insv + 2), w2 = ld4(insv + 3), w3 = ld4(insv + 4);
  float4 l0 = ld4(insv + 5), l1 = ld4(insv + 6), l2 = ld4(insv + 7), l3 = ld4(insv + 8);
  V3 o = xmat4(w0, w1, w2, w3, rayO, 1.0f);
  V3 d = xmat4(w0, w1, w2, w3, rayD, 0.0f);
  V3 position = o + d * h.tMax;
  si.instanceIndex = h.insIdx;
  si.materialIndex = asi(insData.z) >> 8;
  si.hit = true;
  int32_t vertexOffset = asi(insData.y);
  float4 rec = ld4(s.bvh + h.triangleIndex);
  int32_t i0 = asi(rec.x) + vertexOffset, i1 = asi(rec.y) + vertexOffset, i2 = asi(rec.z) + vertexOffset;
  V3 p0 = vertexPosition(s, i0), p1 = vertexPosition(s, i1), p2 = vertexPosition(s, i2);
  V3 n0 = vertexNormal(s, i0), n1 = vertexNormal(s, i1), n2 = vertexNormal(s, i2);
  V3 bary = h.hitBary;
  V3 smoothNormal = n0 * bary.x + n1 * bary.y + n2 * bary.z;
  V3 normal = normalize(smoothNormal);
  // Cycles shadow-terminator offset (intersect.wgsl.ts:1376-1407).
  V3 geometricNormal = normalize(cross(p1 - p0, p2 - p0));
  float a = dot(n2 - n0, p0 - p2);
  float b = dot(n2 - n1, p1 - p2);
  float c = dot(n1 - n0, p1 - p0);
  float hh = a * bary.x * (bary.x - 1.0f) + (a + b + c) * bary.x * bary.y + b * bary.y * (bary.y - 1.0f);
  if (dot(smoothNormal, geometricNormal) > 0.0f) {
    float h0 = fmaxf(fmaxf(dot(p1 - p0, n0), dot(p2 - p0, n0)), 0.0f);
    float h1 = fmaxf(fmaxf(dot(p0 - p1, n1), dot(p2 - p1, n1)), 0.0f);
    float h2 = fmaxf(fmaxf(dot(p0 - p2, n2), dot(p1 - p2, n2)), 0.0f);
    h0 = fmaxf(dot(p0 - position, n0) + h0, 0.0f);
    h1 = fmaxf(dot(p1 - position, n1) + h1, 0.0f);
    h2 = fmaxf(dot(p2 - position, n2) + h2, 0.0f);
    hh = fmaxf(fminf(fminf(h0, h1), h2), hh * 0.5f);
  } else {
    float h0 = fmaxf(fmaxf(dot(p0 - p1, n0), dot(p0 - p2, n0)), 0.0f);
    float h1 = fmaxf(fmaxf(dot(p1 - p0, n1), dot(p1 - p2, n1)), 0.0f);
    float h2 = fmaxf(fmaxf(dot(p2 - p0, n2), dot(p2 - p1, n2)), 0.0f);
    h0 = fmaxf(dot(position - p0, n0) + h0, 0.0f);
    h1 = fmaxf(dot(position - p1, n1) + h1, 0.0f);
    h2 = fmaxf(dot(position - p2, n2) + h2, 0.0f);
    hh = fminf(-fminf(fminf(h0, h1), h2), hh * 0.5f);
  }
  V3 shadowOffset = smoothNormal * hh;
  // UVs (intersect.wgsl.ts:1274-1319, 1408-1418): interpolated, times the
  // instance material's uvScale; a normal map bends the shading normal.
  // fetchAttributes reads uvScale and the UV projection from the instance's
  // material, then resolves the triangle's own (resolveSurfaceMaterialIndex).
  const float4 r7 = ld4(s.mats + size_t(si.materialIndex) * MTC_MATERIAL_VEC4_ROWS + 7);
  if (s.triMats) {
    const uint32_t tm = __ldg(s.triMats + h.triangleIndex);
    if (tm && tm - 1u < s.matCount) si.materialIndex = int32_t(tm - 1u);
  }
  V3 mapped = normal;
  bool normalMapped = false;
  // Only maps and vertex colors read `tex`; without them it keeps the
  // sample's initial zero UVs and white.
  if (s.vuvOff | s.vuv1Off | s.vcolorOff | s.mapCount || r7.x > 0.0f)
    normalMapped = surfaceTexcoords(s, si.materialIndex, r7, i0, i1, i2, bary, position, normal, p0, p1, p2, tex, mapped);
  auto nt = [&](V3 v) { return V3{dot(xyz(w0), v), dot(xyz(w1), v), dot(xyz(w2), v)}; };
  si.faceNormal = normalize(nt(h.hitNormal));
  si.vertexNormal = normalize(nt(normal));
  si.normal = normalMapped ? normalize(nt(mapped)) : si.vertexNormal;
  si.shadowOffset = mat4v(l0, l1, l2, l3, shadowOffset, 0.0f);
  si.position = mat4v(l0, l1, l2, l3, position, 1.0f);
}

// intersect.wgsl.ts:829-879; scenes with alpha test each candidate's
// coverage with the path's sampler.
template <bool kGpuLayout>
MTD bool intersectSceneShadow(const JobData &J, const Ray &r, float lightDistance, int32_t tri, int32_t ins,
                              Counters &cnt, Sampler &smp) {
  if (J.u.is_empty > 0) return false;
  cnt.shadow++;
  TraversalHit h;
  h.tMax = fminf(fmaxf(lightDistance, 0.0f), RAY_MAX_DISTANCE);
  if (J.s.flags & MTC_SCENE_HAS_ALPHA)
    return traverse<true, kGpuLayout, true>(J.s, J.u.blas_offset, r.o, r.d, 1, true, tri, ins, h, &smp);
  return traverse<true, kGpuLayout>(J.s, J.u.blas_offset, r.o, r.d, 1, true, tri, ins, h);
}

// ------------------------------------------------------------- integrator
struct Path {
  bool scatteringMediumEntered;
  Ray ray;
  V3 li; float alpha; V3 beta;
  bool fromEye, abort;
  float scatteringPdf; bool scatteringIsDelta, isNextRefraction;
};
struct Aux { V3 albedo; V3 normal; bool isBlank; };

// The NEE shadow ray selected at a vertex, traced after shading returns
// (outside the shading code's branches, and out of its register pressure).
struct ShadowQuery {
  Ray ray;
  float maxDistance;
  int32_t triangleIndex, instanceIndex;
  V3 contribution;  // added to the path radiance when unoccluded
  bool valid;
};

struct Ctx {
  const JobData &J;
  Sampler smp;
  BsdfContext bc;
  Counters cnt;
  ShadowQuery shadow;
  MTD uint32_t candidateCount() const { return uint32_t(max(J.u.direct_light_candidates, 1)); }
};

// rayTrace.compute.ts:264-284
MTD float neeMISWeight(const Ctx &c, float lightPdf, float scatteringPdf) {
  uint32_t n = c.candidateCount();
  if (n <= 1u) return powerHeuristic(lightPdf, scatteringPdf);
  float w = float(n) * lightPdf;
  return w / fmaxf(w + scatteringPdf, 1e-20f);
}
MTD float bsdfMISWeight(const Ctx &c, float scatteringPdf, float lightPdf) {
  uint32_t n = c.candidateCount();
  if (n <= 1u) return powerHeuristic(scatteringPdf, lightPdf);
  float w = float(n) * lightPdf;
  return scatteringPdf / fmaxf(scatteringPdf + w, 1e-20f);
}
// common.wgsl.ts:14-20
MTD V3 offsetSurfaceRay(V3 p, V3 gn, V3 dir) {
  V3 n = dot(gn, dir) >= 0.0f ? gn : -gn;
  V3 r;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    float pc = comp(p, k), nc = comp(n, k);
    int io = int(256.0f * nc);
    int sh = __float_as_int(pc) + (pc < 0.0f ? -io : io);
    setcomp(r, k, fabsf(pc) < 1.0f / 32.0f ? pc + nc / 65536.0f : __int_as_float(sh));
  }
  return r;
}
// rayTrace.compute.ts:592-600
MTD Ray initCameraRay(const JobData &J, V2 coord) {
  const float *m = J.cam.view_projection_inv;
  float x = coord.x * 2.0f - 1.0f, y = coord.y * 2.0f - 1.0f;
  float ox = m[0] * x + m[4] * y + m[8] * -1.0f + m[12];
  float oy = m[1] * x + m[5] * y + m[9] * -1.0f + m[13];
  float oz = m[2] * x + m[6] * y + m[10] * -1.0f + m[14];
  float ow = m[3] * x + m[7] * y + m[11] * -1.0f + m[15];
  float cx = m[0] * x + m[4] * y + m[8] + m[12];
  float cy = m[1] * x + m[5] * y + m[9] + m[13];
  float cz = m[2] * x + m[6] * y + m[10] + m[14];
  float cw = m[3] * x + m[7] * y + m[11] + m[15];
  Ray r;
  r.o = {ox / ow, oy / ow, oz / ow};
  r.d = normalize(V3{cx * ow - ox * cw, cy * ow - oy * cw, cz * ow - oz * cw});
  return r;
}
MTD V3 cameraEye(const JobData &J) { return {J.cam.view_inv[12], J.cam.view_inv[13], J.cam.view_inv[14]}; }

struct ShadowWork {
  Ray ray; float maxDistance; int32_t triangleIndex; V3 contribution;
  float risTarget, lightSelectionPmf; bool valid;
};
// sampleMaterial.wgsl.ts:32-151
MTD bool finishDirectLight(Ctx &c, const SurfaceInteraction &si, Path &path, V3 ffnormal, bool isSurface,
                           const LightSample &ls, V3 f, float scatteringPdf, ShadowWork &w) {
  w.valid = false; w.lightSelectionPmf = 0.0f; w.risTarget = 0.0f;
  V3 Li = ls.emission;
  V3 lightDir = ls.direction;
  float lightPdf = ls.pdf, lsp = ls.selectionPmf;
  float cosThetaL = dot(ffnormal, lightDir);
  if (lightPdf <= 0.0f || lsp <= 0.0f || maxc(Li) <= 0.0f) return false;
  if (scatteringPdf <= 0.0f || maxc(f) <= 0.0f) return false;
  V3 shadowOrigin = si.position + lightDir * EPS;
  if (isSurface) {
    shadowOrigin = offsetSurfaceRay(si.position, si.faceNormal, lightDir);
    const float cutoff = 0.1f;
    float nl = dot(si.normal, lightDir);
    V3 gn = nl < 0.0f ? -si.faceNormal : si.faceNormal;
    nl = fabsf(nl);
    float gl = dot(gn, lightDir);
    float off = nl < cutoff ? clampf(2.0f - (gl + nl) / cutoff, 0.0f, 1.0f) : clampf(1.0f - gl / cutoff, 0.0f, 1.0f);
    shadowOrigin += si.shadowOffset * off;
  }
  V3 visDir = lightDir;
  float visDist = ls.dist - EPS;
  if (ls.sourceType == 1u) {
    V3 to = si.position + ls.direction * ls.dist + ls.normal * EPS - shadowOrigin;
    visDist = length(to);
    visDir = normalize(to);
  }
  if (isSurface && cosThetaL < 0.0f && ls.sourceType == 0u) {
    float4 bg = sampleSceneBackground(c.J, visDir);
    Li = V3{bg.x, bg.y, bg.z} * bg.w;
  }
  // Spectral scenes use channel-independent RIS (WGPURayTracePass.ts:1349,
  // sampleMaterial.wgsl.ts:119-140): with three wavelengths the radiance is
  // filtered after the target, and each RGB component weighs 1/3.
  const bool spectral = isSpectral(c.J);
  const bool threeWavelengths = spectral && c.J.u.dispersion_wavelengths != 1;
  if (spectral && !threeWavelengths) Li = spectralFilter(Li, si.spectralChannel);
  float mis = ls.isDelta ? 1.0f : neeMISWeight(c, lightPdf, scatteringPdf);
  if (mis > 0.0f) {
    V3 un = Li * f / lightPdf * path.beta;
    const V3 targetWeights = threeWavelengths ? v3(1.0f / 3.0f) : kLuminance();
    w.risTarget = fmaxf(dot(vmax(un * lsp, v3(0.0f)), targetWeights), 0.0f);
    w.ray = {shadowOrigin, visDir};
    w.maxDistance = visDist;
    w.triangleIndex = si.triangleIndex;
    w.contribution = un * mis;
    if (threeWavelengths) w.contribution = spectralFilter(w.contribution, si.spectralChannel);
    w.lightSelectionPmf = lsp;
    w.valid = true;
    return true;
  }
  return false;
}

struct Scattering { V3 direction, response; float pdf; bool transmission; };

MTD bool isDiscrete(const Prepared &p) {
  return !p.mat->thinWalled && fabsf(p.relativeIor - 1.0f) <= 1e-6f &&
         p.probabilities[LOBE_TRANSMISSION] >= 1.0f - 1e-6f;
}

// sampleMaterial.wgsl.ts:160-277
MTD Scattering sampleScattering(Ctx &c, SurfaceInteraction &si, const Material &ma, const Prepared &prepared,
                                Path &path, V3 ffnormal, bool isSurface) {
  uint32_t count = c.candidateCount();
  ShadowWork selected;
  selected.valid = false;
  float selectedTarget = 0.0f, scalarWeightSum = 0.0f;
  Scattering result = {v3(0.0f), v3(0.0f), 0.0f, false};
  for (uint32_t event = 0; event <= count; event++) {
    bool continuation = event == count;
    LightSample ls = zeroLightSample();
    V3 lightDir = v3(0.0f);
    float scatteringPdf = 0.0f;
    V3 response = v3(0.0f);
    bool discrete = false;
    if (continuation) {
      float ucw = 1.0f;
      bool valid = selected.valid;
      if (count > 1u) {
        valid = valid && selectedTarget > 0.0f;
        if (valid) ucw = selected.lightSelectionPmf * scalarWeightSum / (float(count) * selectedTarget);
      }
      // The shadow ray is traced after shading returns (resolveShadow); no
      // other radiance is added to the path between here and there, so the
      // sum is formed in the same order.
      if (valid) {
        c.shadow.ray = selected.ray;
        c.shadow.maxDistance = selected.maxDistance;
        c.shadow.triangleIndex = selected.triangleIndex;
        c.shadow.instanceIndex = si.instanceIndex;
        c.shadow.contribution = selected.contribution * ucw;
        c.shadow.valid = true;
      }
      if (!isSurface) {
        result.direction = henyeyGreenstein(-path.ray.d, si.mediumAnisotropy, c.smp.s2(c.smp.bounceDim(6)));
        result.pdf = henyeyGreensteinPhase(dot(result.direction, -path.ray.d), si.mediumAnisotropy);
        return result;
      }
      V2 dr = c.smp.s2(c.smp.bounceDim(3));
      float lobe = c.smp.s1(c.smp.bounceDim(2));
      discrete = isDiscrete(prepared);
      if (discrete) {
        lightDir = toWorld(prepared.basis, -prepared.viewLocal);
        response = transmissionTint(c.bc, *prepared.mat) * coatBaseScale(c.bc, prepared, -prepared.viewLocal.z);
        scatteringPdf = 1.0f;
        result.transmission = true;
      } else {
        bool transmission = false;
        if (!sampleDirection(c.bc, prepared, {dr.x, dr.y, lobe}, lightDir, transmission)) return result;
        result.transmission = transmission;
      }
    } else {
      V2 lr = c.smp.s2(c.smp.lightDim(event, 1u));
      float lz = c.smp.s1(c.smp.lightDim(event, 0u));
      V3 rnd = {lr.x, lr.y, (lz + float(min(event, count - 1u))) / float(max(count, 1u))};
      sampleLightChoiceTable(c.J, si.position, rnd, ls);
      lightDir = ls.direction;
      if (ls.pdf <= 0.0f || ls.selectionPmf <= 0.0f || maxc(ls.emission) <= 0.0f) continue;
      float cosThetaL = dot(ffnormal, lightDir);
      if (isSurface && cosThetaL <= 0.0f && ma.transmissionWeight <= 0.0f && ma.subsurfaceWeight <= 0.0f) continue;
    }
    if (!discrete) {
      if (isSurface) response = evalPrepared(c.bc, prepared, lightDir, scatteringPdf);
      else {
        scatteringPdf = henyeyGreensteinPhase(dot(-path.ray.d, lightDir), si.mediumAnisotropy);
        response = v3(scatteringPdf);
      }
    }
    if (continuation) {
      result.direction = lightDir; result.response = response; result.pdf = scatteringPdf;
      return result;
    }
    ShadowWork cand;
    if (!finishDirectLight(c, si, path, ffnormal, isSurface, ls, response, scatteringPdf, cand)) continue;
    if (count == 1u) { selected = cand; continue; }
    float sw = cand.risTarget / fmaxf(cand.lightSelectionPmf, 1e-20f);
    if (!(sw > 0.0f) || sw != sw) continue;
    scalarWeightSum += sw;
    if (!selected.valid || c.smp.lightCandidateRandom(event) * scalarWeightSum <= sw) {
      selected = cand;
      selectedTarget = cand.risTarget;
    }
  }
  return result;
}

// sampleMaterial.wgsl.ts:279-303
MTD float emissiveHitMisWeight(Ctx &c, const SurfaceInteraction &si, const Path &path, float4 row0, float4 row3,
                               float doubleSided) {
  float cosLight = dot(si.faceNormal, -path.ray.d);
  if (cosLight <= 0.0f && doubleSided < 0.5f) return 0.0f;
  if (path.fromEye || c.J.u.light_weight_total <= 0.0f || int(row0.w) == 2) return 1.0f;
  float lum = dot(xyz(row3), kLuminance());
  if (lum <= 0.0f || cosLight <= 0.0f) return 1.0f;
  float hd = distance(si.position, path.ray.o);
  float lightPdf = lum / c.J.u.light_weight_total * hd * hd / fmaxf(cosLight, 1e-8f);
  return bsdfMISWeight(c, path.scatteringPdf, lightPdf);
}

// sampleMaterial.wgsl.ts:316-508
MTD void sampleMaterial(Ctx &c, SurfaceInteraction &si, Material &ma, Path &path) {
  const bool hasMedium = (c.J.s.flags & MTC_SCENE_HAS_MEDIUM) != 0u;
  float ndv1 = -dot(si.faceNormal, path.ray.d);
  float ndv2 = -dot(si.normal, path.ray.d);
  if ((ma.transmissionWeight > 0.0f || ma.subsurfaceWeight > 0.0f) && ma.thinWalled) {
    if (ndv1 < 0.0f) { si.faceNormal = -si.faceNormal; ndv1 = -ndv1; }
    if (ndv2 < 0.0f) { si.normal = -si.normal; ndv2 = -ndv2; }
  }
  bool useFaceN = ndv1 >= 0.0f && ndv2 < 0.0f;
  float ndv = useFaceN ? ndv1 : ndv2;
  V3 N = useFaceN ? si.faceNormal : si.normal;
  ma.inside = ndv <= 0.0f && !ma.thinWalled;
  ma.relativeIor = ndv > 0.0f ? 1.0f / ma.specularIor : ma.specularIor;
  V3 ffnormal = ndv >= 0.0f ? N : -N;
  path.scatteringIsDelta = false;
  bool mediumSampled = false, crossedBoundary = false;
  if (hasMedium) {
    float d = distance(si.position, path.ray.o);
    V3 segmentOrigin = path.ray.o;
    V3 ext = si.mediumExtinction;
    V3 scat = vmin(si.mediumScattering, ext);
    float majorant = maxc(ext);
    if (si.mediumType > 0 && majorant > 0.0f) {
      int ch = min(int(c.smp.s1(c.smp.bounceDim(4)) * 3.0f), 2);
      float ce = comp(ext, ch);
      float sd = ce > 0.0f ? fminf(-logf(fmaxf(c.smp.s1(c.smp.bounceDim(5)), 1e-7f)) / ce, d) : d;
      mediumSampled = sd < d;
      V3 T = {expf(-ext.x * sd), expf(-ext.y * sd), expf(-ext.z * sd)};
      V3 density = mediumSampled ? ext * T : T;
      float mp = fmaxf((density.x + density.y + density.z) / 3.0f, 1e-8f);
      if (mediumSampled) {
        path.beta *= T * scat / mp;
        if (path.beta.x == 0.0f && path.beta.y == 0.0f && path.beta.z == 0.0f) { path.abort = true; return; }
        path.ray.o = segmentOrigin + path.ray.d * sd;
        si.position = path.ray.o;
        si.triangleIndex = -1;
        si.instanceIndex = -1;
      } else {
        path.beta *= T / mp;
        if (path.beta.x == 0.0f && path.beta.y == 0.0f && path.beta.z == 0.0f) { path.abort = true; return; }
      }
    }
  }
  if (!mediumSampled) {
    int mi = uint32_t(si.materialIndex) < c.J.s.matCount ? si.materialIndex : 0;
    const float4 *md = c.J.s.mats + size_t(mi) * MTC_MATERIAL_VEC4_ROWS;
    V3 se = ma.emission;
    if (se.x != 0.0f || se.y != 0.0f || se.z != 0.0f) {
      if (isSpectral(c.J)) se = spectralFilter(se, si.spectralChannel);
      float w = emissiveHitMisWeight(c, si, path, ld4(md), ld4(md + 3), ld4(md + 23).z);
      path.li += se * w * path.beta;
    }
  }
  if (ma.materialType == 2) { path.abort = true; return; }
  Prepared prepared;
  if (!mediumSampled) prepared = prepare(c.bc, v3(0.0f), ma, -path.ray.d, ffnormal);
  else { prepared = Prepared{}; prepared.mat = &ma; }
  Scattering sc = sampleScattering(c, si, ma, prepared, path, ffnormal, !mediumSampled);
  V3 scatterDir = sc.direction;
  float scatteringPdf = sc.pdf;
  if (!mediumSampled) {
    V3 f = sc.response;
    bool nextRefraction = sc.transmission;
    bool finite = f.x == f.x && f.y == f.y && f.z == f.z && fabsf(f.x) < 3.402823e38f &&
                  fabsf(f.y) < 3.402823e38f && fabsf(f.z) < 3.402823e38f;
    if (!(scatteringPdf > 0.0f) || !finite || dot(scatterDir, scatterDir) < 0.5f) {
      path.scatteringPdf = 0.0f;
      path.abort = true;
      return;
    }
    path.scatteringIsDelta = isDiscrete(prepared);
    path.beta *= f / scatteringPdf;
    if (path.beta.x == 0.0f && path.beta.y == 0.0f && path.beta.z == 0.0f) { path.abort = true; return; }
    crossedBoundary = nextRefraction && !ma.thinWalled;
    path.isNextRefraction = nextRefraction;
    path.ray.o = si.position + scatterDir * EPS;
  }
  path.scatteringPdf = scatteringPdf;
  path.ray.d = scatterDir;
  if (mediumSampled) path.isNextRefraction = false;
  path.fromEye = false;
  if (hasMedium && !mediumSampled && crossedBoundary && ma.mediumType > 0) {
    if (ndv1 >= 0.0f) {
      si.mediumType = ma.mediumType;
      si.mediumExtinction = ma.mediumExtinction;
      si.mediumScattering = ma.mediumScattering;
      path.scatteringMediumEntered = path.scatteringMediumEntered || ma.mediumScattering.x > 0.0f ||
                                     ma.mediumScattering.y > 0.0f || ma.mediumScattering.z > 0.0f;
      si.mediumAnisotropy = ma.mediumAnisotropy;
    } else {
      si.mediumType = 0;
      si.mediumExtinction = v3(0.0f);
      si.mediumScattering = v3(0.0f);
      si.mediumAnisotropy = 0.0f;
    }
  }
}

// rayTrace.compute.ts:341-512 shadeVertex (no shadow catcher, no bevel)
MTD void shadeVertex(Ctx &c, V2 uv, Path &path, int &depth, SurfaceInteraction &si, Material &ma, Aux &aux,
                     bool &sampleIgnored) {
  sampleIgnored = false;
  c.smp.bounce = uint32_t(max(depth, 0));
  int matType = ma.materialType;
  const mtc_trace_uniform &u = c.J.u;
  if (!si.hit) {
    float4 bg = sampleSceneBackground(c.J, path.ray.d);
    if (isSpectral(c.J)) {
      V3 f = spectralFilter({bg.x, bg.y, bg.z}, si.spectralChannel);
      bg = make_float4(f.x, f.y, f.z, bg.w);
    }
    if (path.fromEye) {
      path.li = path.beta * V3{bg.x, bg.y, bg.z} * bg.w;
      path.alpha = bg.w;
      aux.isBlank = bg.w < 0.001f || ((u.background_flags & MTC_BACKGROUND_COLOR) && !(u.background_flags & MTC_BACKGROUND_MAP));
    } else {
      Ray cam = initCameraRay(c.J, uv);
      bool towardsCam = dot(cam.d, path.ray.d) > 0.0f;
      if (u.transmissive_output_alpha_min < 1.0f) {
        if (towardsCam) path.alpha = fmaxf(path.alpha, bg.w); else path.alpha = 1.0f;
      }
      if (!useEnvmap(c.J) && towardsCam)
        path.li += path.beta * bsdfMISWeight(c, path.scatteringPdf, 1.0f) * V3{bg.x, bg.y, bg.z};
    }
    path.abort = true;
    return;
  }
  if (matType == 0 || matType == 2) {
    float alpha = clampf(ma.alpha, 0.0f, 1.0f);
    if (alpha < 1.0f) {
      if (alpha <= 0.0f || c.smp.hashedSample(3u) > alpha) sampleIgnored = true;
    }
    if (!sampleIgnored && u.transmissive_output_alpha_min < 1.0f) {
      float oa = fmaxf(1.0f - ma.transmissionWeight, 1.0f - powf(1.0f - u.transmissive_output_alpha_min, float(depth)));
      path.alpha = fmaxf(oa, path.alpha);
    }
    if (!sampleIgnored) sampleMaterial(c, si, ma, path);
    else path.ray.o = si.position + path.ray.d * EPS;
  }
  if (!si.albedoSampled && !sampleIgnored) {
    if (matType == 0 || matType == 2) {
      if (!(ma.transmissionWeight > 0.5f || (ma.specularRoughness <= 0.02f && ma.baseMetalness > 0.98f))) {
        aux.albedo = ma.baseColor;
        aux.normal = dot(si.normal, si.position - cameraEye(c.J)) > 0.0f ? -si.normal : si.normal;
        si.albedoSampled = true;
      }
      if (depth > 4) si.albedoSampled = true;
    }
  }
  if (depth >= (path.scatteringMediumEntered ? 12 : 2) && !sampleIgnored) {
    float q = fmaxf(0.0f, 1.0f - maxc(path.beta));
    if (c.smp.s1(c.smp.bounceDim(7)) < q) { path.alpha = 1.0f; path.abort = true; }
    else path.beta /= 1.0f - q;
  }
}

// rayTrace.compute.ts:514-589 completeVertex
MTD void completeVertex(Ctx &c, Path &path, int &depth, SurfaceInteraction &si, Material &ma, bool sampleIgnored) {
  const bool spectral = isSpectral(c.J);
  if (spectral && ma.transmissionWeight > 0.001f)
    ma.specularIor = cauchyIor(si.wavelength, ma.specularIor, ma.transmissionDispersionScale, ma.dispersionAbbeNumber);
  if (sampleIgnored) return;
  bool isAlphaOccluded = ma.alpha >= 1.0f ? (c.smp.hashed += 1u, true) : c.smp.hashedSample(3u) < ma.alpha;
  for (int i = 0; i < c.J.u.lights_count; i++) {
    Light L = loadLight(c.J, i);
    LightSample ls = zeroLightSample();
    float d = intersectLight(path.ray, L, ls);
    ls.pdf *= L.selectionPmf;
    bool occluded = si.hit && d > distance(si.position, path.ray.o);
    if (d != INF && !(occluded && isAlphaOccluded)) {
      float mis = bsdfMISWeight(c, path.scatteringPdf, ls.pdf);
      if (spectral) ls.emission = spectralFilter(ls.emission, si.spectralChannel);
      path.li += path.beta * ls.emission * mis;
      path.alpha = 1.0f;
      path.abort = true;
    }
  }
  if (useEnvmap(c.J) && !(si.hit && isAlphaOccluded)) {
    if (path.isNextRefraction) {
      float4 bg = sampleSceneBackground(c.J, path.ray.d);
      V3 rgb = {bg.x, bg.y, bg.z};
      if (spectral) rgb = spectralFilter(rgb, si.spectralChannel);
      float w = path.scatteringIsDelta ? 1.0f
                : bsdfMISWeight(c, path.scatteringPdf, envMapPdf(c.J, environmentUv(c.J, path.ray.d)) * c.J.u.env_light_pmf);
      path.li += path.beta * rgb * (w * bg.w);
      path.alpha = fmaxf(path.alpha, bg.w);
      path.abort = true;
      return;
    }
    V2 euv = environmentUv(c.J, path.ray.d);
    V3 emission = xyz(textureLinear(c.J.s.env, c.J.s.envW, c.J.s.envH, euv));
    float mis = bsdfMISWeight(c, path.scatteringPdf, envMapPdf(c.J, euv) * c.J.u.env_light_pmf);
    if (spectral) emission = spectralFilter(emission, si.spectralChannel);
    if (!(c.J.u.background_flags & MTC_BACKGROUND_COLOR)) path.alpha = 1.0f;
    path.li += path.beta * emission * mis;
    path.abort = true;
  }
  depth = depth + 1;
}

// One path sample in flight: the locals of the RGB integrator
// (rayTrace.compute.ts:891-946) kept across events, so that a thread can
// advance its path one event at a time and start its pixel's next sample as
// soon as the current one ends, without waiting for the other lanes.
struct PathSample {
  SurfaceInteraction si;
  Path path;
  Aux aux;
  V2 coord;
  int depth, event;
  bool sampleIgnored, isNotTransparent;
};

// Locals of the spectral integrator (rayTrace.compute.ts:947-1057) that live
// across its three wavelength paths: the primary vertex they share, the
// sampler state each restarts from, and the running sums.  The alpha-split
// RGB integrator (:815-890) keeps its primary vertex, guides and camera ray
// in the same fields, plus the coverage split and the back path's result.
struct SpectralState {
  SurfaceInteraction primarySi;
  Aux primaryAux;        // the integrator's outAux: primary-hit guides
  Ray cameraRay;
  uint4 savedS0;
  uint32_t savedHashed;
  float wavelengthSample;
  int wavelengthIndex, heroWavelengthIndex;
  bool primaryReady, dispersivePrimary, allBlank;
  V3 color, guideAlbedo, guideNormal;
  float alpha;
  // alpha split: coverage of the primary hit, whether it was split, whether
  // the front path runs (frontPending: its first step reuses the primary
  // vertex without a query), and the back path's (li, alpha) and guides
  float coverage;
  bool split, front, frontPending;
  float4 back;
  Aux backAux;
  // Texture coordinates of the current surface (kept from the last hit on a
  // miss, like the rest of the surface interaction) and of the primary one.
  SurfaceTexcoords tex, primaryTex;
  // Shared spectral prefix (spectralPrefix.wgsl.ts): whether the current
  // wavelength path still runs in RGB (spActive), whether the first one forked
  // (spForkCall == 0), the channel and wavelength it forks to, and the loop
  // state at the fork vertex (the flatPrefix checkpoint of
  // rayTrace.compute.ts:145-148; the material is refetched from the surface).
  bool spActive, spForked;
  int spChannel;
  float spWavelength;
  Path forkPath;
  SurfaceInteraction forkSi;
  SurfaceTexcoords forkTex;
  Aux forkAux;
  int forkDepth, forkEvent;
  bool forkIgnored, forkOpaque;
  uint4 forkS0;
  uint32_t forkHashed, forkBounce;
};

// spDisperses (spectralPrefix.wgsl.ts:29-31).
MTD bool spDisperses(const Material &ma) {
  return ma.transmissionDispersionScale > 0.0f && ma.specularIor != 1.0f;
}

// The alpha-split integrator runs for RGB scenes with a non-opaque material.
MTD bool alphaSplit(const JobData &J) { return (J.s.flags & MTC_SCENE_HAS_ALPHA) && !isSpectral(J); }

// rayTrace.compute.ts:1157-1208 main up to the integrator call: sampler
// state for (x, y, outNormal.a + sampleSequenceOffset), Sobol jitter, camera
// ray and thin lens, then integrator() locals (:891-905).  Out of line, like
// shadeStep and endSample, so every kernel runs one compiled copy.
static __device__ __noinline__ void beginSample(Ctx &c, uint32_t x, uint32_t y, PathSample &ps, SpectralState &sp) {
  const JobData &J = c.J;
  const mtc_trace_uniform &u = J.u;
  uint32_t W = J.width;
  uint32_t idx = x + y * W;
  float count = J.outNormal[idx].w;
  V2 outputSize = {u.output_size[0], u.output_size[1]};
  V2 uv = {(float(x) + 0.5f) / outputSize.x, (float(y) + 0.5f) / outputSize.y};
  c.smp.px = x; c.smp.py = y; c.smp.width = W;
  c.smp.index = uint32_t(count) + u.sample_sequence_offset;
  c.smp.bounce = 0; c.smp.hashed = 0;
  c.smp.seed = u.sequence_seed; c.smp.logspp = u.zsobol_log_spp;
  c.smp.pattern = int((J.s.flags & MTC_SCENE_PATTERN_MASK) >> MTC_SCENE_PATTERN_SHIFT);
  V2 jitter = {u.jitter[0], u.jitter[1]};
  if (c.smp.pattern == 0 || c.smp.pattern == 1) {
    V2 j = c.smp.s2(0u);
    jitter = {(j.x - 0.5f) / outputSize.x, (j.y - 0.5f) / outputSize.y};
  }
  c.smp.s0 = make_uint4(x, y, c.smp.index ^ sampleHash(u.sequence_seed), x + y);
  V2 coord = {uv.x + jitter.x, uv.y + jitter.y};
  Ray cam = initCameraRay(J, coord);
  if (J.cam.aperture_radius > 0.0f) {
    const float *vi = J.cam.view_inv;
    V3 eye = cameraEye(J);
    V3 forward = -normalize(V3{vi[8], vi[9], vi[10]});
    V3 focus = eye + cam.d * (J.cam.focus_distance / dot(cam.d, forward));
    V2 ip = c.smp.s2(1u);
    V2 pp = {2.0f * ip.x - 1.0f, 2.0f * ip.y - 1.0f};
    bool greater = fabsf(pp.x) > fabsf(pp.y);
    float r = greater ? pp.x : pp.y;
    float theta = greater ? 0.25f * PI * pp.y / pp.x : PI * (0.5f - 0.25f * pp.x / pp.y);
    float st, ct;
    sincosf(theta, &st, &ct);
    float lx = J.cam.aperture_radius * r * ct, ly = J.cam.aperture_radius * r * st;
    V3 origin = {vi[0] * lx + vi[4] * ly + vi[12], vi[1] * lx + vi[5] * ly + vi[13], vi[2] * lx + vi[6] * ly + vi[14]};
    cam = {origin, normalize(focus - origin)};
  }
  ps.coord = coord;
  ps.aux = {v3(0.0f), v3(0.0f), false};
  SurfaceInteraction &si = ps.si;
  si.albedoSampled = false; si.hit = false; si.triangleIndex = 0; si.instanceIndex = 0; si.materialIndex = 0;
  si.wavelength = 0.0f; si.spectralChannel = 0; si.mediumType = 0; si.mediumExtinction = v3(0.0f);
  si.mediumScattering = v3(0.0f); si.mediumAnisotropy = 0.0f;
  si.position = v3(0.0f); si.normal = v3(0.0f); si.vertexNormal = v3(0.0f); si.shadowOffset = v3(0.0f);
  sp.tex = {v2(0.0f, 0.0f), v2(0.0f, 0.0f), v3(1.0f)};
  si.faceNormal = v3(0.0f);
  Path &path = ps.path;
  path.scatteringMediumEntered = false;
  path.ray = cam;
  path.li = v3(0.0f);
  path.alpha = u.transmissive_output_alpha_min < 1.0f ? 0.0f : 1.0f;
  path.beta = v3(1.0f);
  path.fromEye = true;
  path.abort = false;
  path.scatteringPdf = 0.0f;
  path.scatteringIsDelta = false;
  path.isNextRefraction = false;
  ps.depth = 0;
  ps.event = 0;
  ps.sampleIgnored = false;
  ps.isNotTransparent = false;
  if (alphaSplit(J)) {
    sp.primaryReady = false;
    sp.cameraRay = cam;
    sp.coverage = 1.0f;
    sp.split = false;
    sp.front = false;
    sp.frontPending = false;
  }
  if (isSpectral(J)) {
    sp.primaryReady = false;
    sp.spActive = false;
    sp.spForked = false;
    sp.primaryAux = {v3(0.0f), v3(0.0f), false};
    sp.cameraRay = cam;
    sp.wavelengthIndex = 0;
    sp.heroWavelengthIndex = 0;
    sp.dispersivePrimary = false;
    sp.allBlank = true;
    sp.color = v3(0.0f);
    sp.guideAlbedo = v3(0.0f);
    sp.guideNormal = v3(0.0f);
    sp.alpha = 0.0f;
  }
}

// The traversal half of intersectScene (intersect.wgsl.ts:696-740) for the
// path's current event: the closest hit of its extension ray.
// A spectral wavelength path after the first starts from the shared primary
// vertex and traces nothing at its event 0 (rayTrace.compute.ts:978).
MTD bool reusesPrimary(const JobData &J, const PathSample &ps, bool primaryReady) {
  return isSpectral(J) && ps.event == 0 && primaryReady;
}

template <bool kGpuLayout>
MTD void traceExtension(const JobData &J, const PathSample &ps, TraversalHit &h, Counters &cnt) {
  h.tMax = RAY_MAX_DISTANCE;
  h.triangleIndex = -1;
  h.insIdx = -1;
  if (J.u.is_empty > 0) return;
  cnt.ext++;
  traverse<false, kGpuLayout>(J.s, J.u.blas_offset, ps.path.ray.o, ps.path.ray.d, ps.depth, ps.event != 0,
                              ps.si.triangleIndex,
                  ps.si.instanceIndex, h);
}

// The rest of one iteration of the integrator's event loop
// (rayTrace.compute.ts:906-944) once the extension ray's closest hit `h` is
// known: surface interaction, material, primary guides or completeVertex,
// shadeVertex.  Returns true when the path has ended.  Out of line so that
// the megakernel and the wavefront shading kernel run one compiled copy.
static __device__ __noinline__ bool shadeStep(Ctx &c, PathSample &ps, SpectralState &sp, const TraversalHit &h) {
  Path &path = ps.path;
  SurfaceInteraction &si = ps.si;
  const int bounceLimit = max(c.J.u.bounces, 0);
  const int eventLimit = min(bounceLimit * 3, 20);
  const int event = ps.event;
  si.hit = false;
  if (h.insIdx >= 0) {
    si.triangleIndex = h.triangleIndex;
    completeSurfaceInteraction(c.J, si, sp.tex, h, path.ray.o, path.ray.d);
  }
  Material ma;
  getMaterial(c.J, si.materialIndex, si.instanceIndex, sp.tex.uv, sp.tex.uv1, sp.tex.vertexColor, ma);
  if (event == 0) {
    if (si.hit && (ma.materialType == 0 || ma.materialType == 2)) {
      ps.aux.albedo = ma.transmissionWeight > 0.5f ? v3(1.0f) : ma.baseColor;
      ps.aux.normal = dot(si.normal, si.position - cameraEye(c.J)) > 0.0f ? -si.normal : si.normal;
      si.albedoSampled = ma.transmissionWeight > 0.5f;
    }
    ps.isNotTransparent = ma.transmissionWeight < 0.001f && ma.subsurfaceWeight < 0.001f && ma.alpha > 0.99f;
  } else {
    completeVertex(c, path, ps.depth, si, ma, ps.sampleIgnored);
  }
  if (ps.isNotTransparent && event > bounceLimit) path.abort = true;
  if (path.abort || event >= eventLimit) return true;
  shadeVertex(c, ps.coord, path, ps.depth, si, ma, ps.aux, ps.sampleIgnored);
  if (path.abort) return true;
  ps.event = event + 1;
  return false;
}

// One iteration of the alpha-split RGB integrator (rayTrace.compute.ts
// :815-890) once its query (if any) is answered.  The primary hit keeps the
// guides; if it is a standard or unlit surface with coverage below 1 the
// sample splits: the back path continues through it first (event 0 again,
// from just behind the surface), then the front path restarts at the primary
// vertex with full coverage, and finishAlphaSplit mixes the two by the
// coverage.  Returns true when the current path has ended.
static __device__ __noinline__ bool shadeStepAlpha(Ctx &c, PathSample &ps, SpectralState &sp, const TraversalHit &h) {
  Path &path = ps.path;
  SurfaceInteraction &si = ps.si;
  const int bounceLimit = max(c.J.u.bounces, 0);
  const int eventLimit = min(bounceLimit * 3, 20);
  const int event = ps.event;
  Material ma;
  if (sp.frontPending) {
    sp.frontPending = false;
    si = sp.primarySi;
    sp.tex = sp.primaryTex;
    getMaterial(c.J, si.materialIndex, si.instanceIndex, sp.tex.uv, sp.tex.uv1, sp.tex.vertexColor, ma);
    ma.alpha = 1.0f;
  } else {
    si.hit = false;
    if (h.insIdx >= 0) {
      si.triangleIndex = h.triangleIndex;
      completeSurfaceInteraction(c.J, si, sp.tex, h, path.ray.o, path.ray.d);
    }
    getMaterial(c.J, si.materialIndex, si.instanceIndex, sp.tex.uv, sp.tex.uv1, sp.tex.vertexColor, ma);
  }
  if (!sp.primaryReady) {
    if (si.hit && (ma.materialType == 0 || ma.materialType == 2)) {
      ps.aux.albedo = ma.transmissionWeight > 0.5f ? v3(1.0f) : ma.baseColor;
      ps.aux.normal = dot(si.normal, si.position - cameraEye(c.J)) > 0.0f ? -si.normal : si.normal;
      si.albedoSampled = ma.transmissionWeight > 0.5f;
    }
    sp.primarySi = si;
    sp.primaryTex = sp.tex;
    sp.primaryAux = ps.aux;
    sp.primaryReady = true;
    sp.coverage = clampf(ma.alpha, 0.0f, 1.0f);
    sp.split = si.hit && (ma.materialType == 0 || ma.materialType == 2) && sp.coverage < 1.0f;
    if (sp.split) {
      path.ray.o = si.position + sp.cameraRay.d * (EPS * 0.02f);
      si.albedoSampled = false;
      return false;
    }
  } else if (event == 0 && !sp.front && sp.split) {
    if (si.hit && ma.materialType == 0) {
      ps.aux.albedo = ma.transmissionWeight > 0.5f ? v3(1.0f) : ma.baseColor;
      ps.aux.normal = dot(si.normal, si.position - cameraEye(c.J)) > 0.0f ? -si.normal : si.normal;
      si.albedoSampled = ma.transmissionWeight > 0.5f;
    }
  }
  if (event == 0) {
    ps.isNotTransparent = ma.transmissionWeight < 0.001f && ma.subsurfaceWeight < 0.001f && ma.alpha > 0.99f;
  } else {
    completeVertex(c, path, ps.depth, si, ma, ps.sampleIgnored);
  }
  if (ps.isNotTransparent && event > bounceLimit) path.abort = true;
  if (!path.abort && event < eventLimit) shadeVertex(c, ps.coord, path, ps.depth, si, ma, ps.aux, ps.sampleIgnored);
  if (path.abort || event >= eventLimit) return true;
  ps.event = event + 1;
  return false;
}

// End of an alpha-split path, after its last shadow ray (rayTrace.compute.ts
// :870-888): true when the sample is complete (unsplit, zero coverage, or the
// front path done: radiance, alpha and guides mixed by the coverage);
// otherwise the back path's result is kept and the front path starts.
MTD bool finishAlphaSplit(const JobData &J, PathSample &ps, SpectralState &sp) {
  if (!sp.split || sp.coverage <= 0.0f) return true;
  const float k = sp.coverage;
  auto mix3 = [k](V3 a, V3 b) { return V3{a.x * (1.0f - k) + b.x * k, a.y * (1.0f - k) + b.y * k, a.z * (1.0f - k) + b.z * k}; };
  if (sp.front) {
    Aux &a = ps.aux;
    const Aux &b = sp.backAux;
    a.albedo = mix3(b.albedo, a.albedo);
    const V3 n = mix3(b.normal, a.normal);
    a.normal = dot(n, n) > 1e-12f ? normalize(n) : v3(0.0f);
    a.isBlank = b.isBlank && a.isBlank;
    ps.path.li = mix3(xyz(sp.back), ps.path.li);
    ps.path.alpha = sp.back.w * (1.0f - k) + ps.path.alpha * k;
    return true;
  }
  sp.back = make_float4(ps.path.li.x, ps.path.li.y, ps.path.li.z, ps.path.alpha);
  sp.backAux = ps.aux;
  sp.front = true;
  sp.frontPending = true;
  ps.event = 0;
  ps.depth = 0;
  ps.sampleIgnored = false;
  ps.aux = sp.primaryAux;
  Path &path = ps.path;
  path.scatteringMediumEntered = false;
  path.ray = sp.cameraRay;
  path.li = v3(0.0f);
  path.alpha = J.u.transmissive_output_alpha_min < 1.0f ? 0.0f : 1.0f;
  path.beta = v3(1.0f);
  path.fromEye = true;
  path.abort = false;
  path.scatteringPdf = 0.0f;
  path.scatteringIsDelta = false;
  path.isNextRefraction = false;
  return false;
}

// One step of the spectral integrator (rayTrace.compute.ts:947-1057) after
// its extension ray (if any) has been traced: at event 0 the first wavelength
// path resolves and keeps the primary vertex, and every wavelength path
// restarts there with its own wavelength, Cauchy IOR and the sampler state
// saved after the wavelength draw.  With three wavelengths the path prefix is
// shared (unless MTC_SCENE_SPECTRAL_INDEPENDENT): the first wavelength path
// runs in RGB until its first dispersive transmissive vertex past the primary
// one, saves its state there and forks; the later wavelength paths resume at
// that vertex instead of the camera (:1001-1019).  Returns true when the
// current wavelength path has ended (finishWavelength then decides whether
// the sample has).
static __device__ __noinline__ bool shadeStepSpectral(Ctx &c, PathSample &ps, SpectralState &sp,
                                                      const TraversalHit &h) {
  Path &path = ps.path;
  SurfaceInteraction &si = ps.si;
  const mtc_trace_uniform &u = c.J.u;
  const int bounceLimit = max(u.bounces, 0);
  const int eventLimit = min(bounceLimit * 3, 20);
  int event = ps.event;
  const bool singleWavelength = u.dispersion_wavelengths == 1;
  const bool spEnabled = !singleWavelength && !(c.J.s.flags & MTC_SCENE_SPECTRAL_INDEPENDENT);
  auto spFork = [&]() {  // spectralPrefix.wgsl.ts:32-36
    sp.spActive = false;
    path.li = spectralFilter(path.li, sp.spChannel);
    si.spectralChannel = sp.spChannel;
    si.wavelength = sp.spWavelength;
  };
  Material ma;
  if (!reusesPrimary(c.J, ps, sp.primaryReady)) {
    si.hit = false;
    if (h.insIdx >= 0) {
      si.triangleIndex = h.triangleIndex;
      completeSurfaceInteraction(c.J, si, sp.tex, h, path.ray.o, path.ray.d);
    }
    getMaterial(c.J, si.materialIndex, si.instanceIndex, sp.tex.uv, sp.tex.uv1, sp.tex.vertexColor, ma);
  } else {
    // The primary material is a pure function of the primary vertex.
    getMaterial(c.J, sp.primarySi.materialIndex, sp.primarySi.instanceIndex, sp.primaryTex.uv, sp.primaryTex.uv1,
                sp.primaryTex.vertexColor, ma);
  }
  if (event == 0) {
    if (!sp.primaryReady) {
      if (si.hit && (ma.materialType == 0 || ma.materialType == 2)) {
        sp.primaryAux.albedo = ma.transmissionWeight > 0.5f ? v3(1.0f) : ma.baseColor;
        sp.primaryAux.normal = dot(si.normal, si.position - cameraEye(c.J)) > 0.0f ? -si.normal : si.normal;
        si.albedoSampled = ma.transmissionWeight > 0.5f;
      }
      sp.primarySi = si;
      sp.primaryTex = sp.tex;
      sp.primaryReady = true;
      sp.dispersivePrimary = si.hit && ma.transmissionWeight > 0.001f && ma.transmissionDispersionScale > 0.001f;
      sp.wavelengthSample = c.smp.s1(2u);  // CAMERA_WAVELENGTH, sobol.wgsl.ts:5
      if (singleWavelength) {
        sp.heroWavelengthIndex = min(int(floorf(sp.wavelengthSample * 3.0f)), 2);
        float w3 = sp.wavelengthSample * 3.0f;
        sp.wavelengthSample = w3 - floorf(w3);
      }
      sp.savedS0 = c.smp.s0;
      sp.savedHashed = c.smp.hashed;
    }
    si = sp.primarySi;
    ps.aux = sp.primaryAux;
    if (!singleWavelength) {
      c.smp.s0 = sp.savedS0;
      c.smp.hashed = sp.savedHashed;
      c.smp.bounce = 0;
      ps.aux.isBlank = false;
    }
    si.wavelength = 0.0f;
    si.spectralChannel = 0;
    if (!singleWavelength || sp.dispersivePrimary) {
      int channel = singleWavelength ? sp.heroWavelengthIndex : sp.wavelengthIndex;
      si.spectralChannel = channel + 1;
      si.wavelength = spectrumCameraWavelength(uint32_t(channel), sp.wavelengthSample);
      // spBegin (spectralPrefix.wgsl.ts:22-27)
      sp.spChannel = channel + 1;
      sp.spWavelength = si.wavelength;
      sp.spActive = spEnabled && !spDisperses(ma);
      if (sp.spActive) si.spectralChannel = 0;
      ma.specularIor = cauchyIor(si.wavelength, ma.specularIor, ma.transmissionDispersionScale,
                                 ma.dispersionAbbeNumber);
    }
    path.scatteringMediumEntered = false;
    path.ray = sp.cameraRay;
    path.li = v3(0.0f);
    path.alpha = u.transmissive_output_alpha_min < 1.0f ? 0.0f : 1.0f;
    path.beta = v3(1.0f);
    path.fromEye = true;
    path.abort = false;
    path.scatteringPdf = 0.0f;
    path.scatteringIsDelta = false;
    path.isNextRefraction = false;
    ps.depth = 0;
    ps.sampleIgnored = false;
    ps.isNotTransparent = ma.transmissionWeight < 0.001f && ma.subsurfaceWeight < 0.001f && ma.alpha > 0.99f;
    if (sp.spActive && sp.wavelengthIndex > 0 && sp.spForked) {
      // Resume at the first wavelength path's fork vertex (:1010-1013).
      path = sp.forkPath;
      si = sp.forkSi;
      sp.tex = sp.forkTex;
      ps.aux = sp.forkAux;
      ps.depth = sp.forkDepth;
      event = sp.forkEvent;
      ps.sampleIgnored = sp.forkIgnored;
      ps.isNotTransparent = sp.forkOpaque;
      c.smp.s0 = sp.forkS0;
      c.smp.hashed = sp.forkHashed;
      c.smp.bounce = sp.forkBounce;
      getMaterial(c.J, si.materialIndex, si.instanceIndex, sp.tex.uv, sp.tex.uv1, sp.tex.vertexColor, ma);
      spFork();
    }
  }
  if (event > 0 && !path.abort) {
    if (sp.spActive && ma.transmissionWeight > 0.001f && spDisperses(ma)) {
      // The first dispersive transmission of the RGB prefix (:1015-1019).
      sp.forkPath = path;
      sp.forkSi = si;
      sp.forkTex = sp.tex;
      sp.forkAux = ps.aux;
      sp.forkDepth = ps.depth;
      sp.forkEvent = event;
      sp.forkIgnored = ps.sampleIgnored;
      sp.forkOpaque = ps.isNotTransparent;
      sp.forkS0 = c.smp.s0;
      sp.forkHashed = c.smp.hashed;
      sp.forkBounce = c.smp.bounce;
      sp.spForked = true;
      spFork();
    }
    completeVertex(c, path, ps.depth, si, ma, ps.sampleIgnored);
  }
  if (ps.isNotTransparent && event > bounceLimit) path.abort = true;
  if (!path.abort && event < eventLimit) shadeVertex(c, ps.coord, path, ps.depth, si, ma, ps.aux, ps.sampleIgnored);
  if (path.abort || event >= eventLimit) return true;
  ps.event = event + 1;
  return false;
}

// End of a spectral wavelength path, after its last NEE shadow ray has been
// resolved (rayTrace.compute.ts:1036-1053).  Returns true when the sample is
// complete; its radiance, alpha and guides are then in ps.path / ps.aux for
// endSample.  Otherwise the next wavelength path starts at event 0.
MTD bool finishWavelength(const JobData &J, PathSample &ps, SpectralState &sp) {
  if (J.u.dispersion_wavelengths == 1) {
    float scale = sp.dispersivePrimary ? 3.0f : 1.0f;
    ps.path.li = ps.path.li * scale;
    return true;
  }
  if (sp.spActive) {
    // The shared prefix never forked: its RGB path is the whole sample, with
    // the guides of three identical wavelength paths (:1035-1041).
    const V3 a = ps.aux.albedo, n = ps.aux.normal;
    ps.aux.albedo = (a + a + a) / 3.0f;
    ps.aux.normal = (n + n + n) / 3.0f;
    return true;
  }
  sp.color += ps.path.li;
  sp.alpha = fmaxf(sp.alpha, ps.path.alpha);
  sp.guideAlbedo += ps.aux.albedo;
  sp.guideNormal += ps.aux.normal;
  sp.allBlank = sp.allBlank && ps.aux.isBlank;
  sp.wavelengthIndex++;
  if (sp.wavelengthIndex >= 3) {
    ps.path.li = sp.color;
    ps.path.alpha = sp.alpha;
    ps.aux.albedo = sp.guideAlbedo / 3.0f;
    ps.aux.normal = sp.guideNormal / 3.0f;
    ps.aux.isBlank = sp.allBlank;
    return true;
  }
  ps.event = 0;
  return false;
}

// One iteration of the integrator's event loop: true when the path (the
// current wavelength path of a spectral sample) has ended.
template <bool kGpuLayout>
MTD bool stepPath(Ctx &c, PathSample &ps, SpectralState &sp) {
  TraversalHit h;
  h.tMax = RAY_MAX_DISTANCE;
  h.triangleIndex = -1;
  h.insIdx = -1;
  const bool spectral = isSpectral(c.J), split = alphaSplit(c.J);
  const bool reuse = spectral ? reusesPrimary(c.J, ps, sp.primaryReady) : split && sp.frontPending;
  if (!reuse) traceExtension<kGpuLayout>(c.J, ps, h, c.cnt);
  return spectral ? shadeStepSpectral(c, ps, sp, h) : split ? shadeStepAlpha(c, ps, sp, h) : shadeStep(c, ps, sp, h);
}

// The deferred NEE visibility test of sampleScattering (sampleMaterial.wgsl.ts
// :238-245): unoccluded -> the selected candidate's contribution.
template <bool kGpuLayout>
MTD void resolveShadow(Ctx &c, PathSample &ps) {
  if (!c.shadow.valid) return;
  c.shadow.valid = false;
  if (!intersectSceneShadow<kGpuLayout>(c.J, c.shadow.ray, c.shadow.maxDistance, c.shadow.triangleIndex,
                                        c.shadow.instanceIndex, c.cnt, c.smp))
    ps.path.li += c.shadow.contribution;
}

// rayTrace.compute.ts:1209-1262: clamp, NaN guard and accumulation of the
// finished sample into the job's outputs.
static __device__ __noinline__ void endSample(const JobData &J, uint32_t idx, const PathSample &ps) {
  const mtc_trace_uniform &u = J.u;
  float4 li = make_float4(ps.path.li.x, ps.path.li.y, ps.path.li.z, ps.path.alpha);
  const Aux &aux = ps.aux;
  if (u.clamping > 0.0f) {
    float cl = u.clamping;
    li = make_float4(clampf(li.x, -cl, cl), clampf(li.y, -cl, cl), clampf(li.z, -cl, cl), li.w);
  }
  if (!(li.x < INF && li.x > -EPS)) li = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
  float4 col = J.outColor[idx];
  J.outColor[idx] = make_float4(col.x + li.x, col.y + li.y, col.z + li.z, col.w + li.w);
  float4 alb = J.outAlbedo[idx];
  J.outAlbedo[idx] = make_float4(alb.x + aux.albedo.x, alb.y + aux.albedo.y, alb.z + aux.albedo.z,
                                 alb.w + (aux.isBlank ? 0.0f : 1.0f));
  float lum = dot(V3{li.x, li.y, li.z}, kLuminance());
  float4 nrm = J.outNormal[idx];
  if (u.variance_moments != 0) J.outNormal[idx] = make_float4(nrm.x + lum * lum, nrm.y, nrm.z, nrm.w + 1.0f);
  else J.outNormal[idx] = make_float4(nrm.x + aux.normal.x, nrm.y + aux.normal.y, nrm.z + aux.normal.z, nrm.w + 1.0f);
  float4 *mom = J.outCatcher + size_t(idx) * 3 + 2;
  float4 m = *mom;
  *mom = make_float4(m.x + lum, m.y + lum * lum, m.z, m.w);
}

// `samples` consecutive progressive passes of pixel (x, y), in order, each
// accumulated before the next begins (the same sums as `samples` separate
// dispatches).  The thread runs its own sample sequence in one event loop,
// so a lane whose path ended early starts its next sample while the warp's
// longer paths are still tracing.  Kept out of line so that every kernel that
// traces pixels (plain, batched, allocation-free batched) calls the same
// out-of-line function, compiled once per translation unit from this one
// source, instead of an inlined copy shaped by its caller: inlined copies could
// contract multiply-adds differently, and a job's image must be bit-identical
// alone and in a batch.
template <bool kGpuLayout>
static __device__ __noinline__ void tracePixelSamples(const JobData &J, uint32_t x, uint32_t y, uint32_t samples,
                                                      Counters &cnt) {
  Ctx c{J, Sampler(), BsdfContext{J.s.lut, (J.s.flags & MTC_SCENE_HAS_MEDIUM) != 0u, feature(J, MTC_FEATURE_HAS_THIN_FILM)},
        Counters(), ShadowQuery()};
  c.shadow.valid = false;
  const uint32_t idx = x + y * J.width;
  PathSample ps;
  SpectralState sp;
  const bool spectral = isSpectral(J), split = alphaSplit(J);
  uint32_t left = samples;
  bool active = left > 0u;
  if (active) beginSample(c, x, y, ps, sp);
  // No warp vote here: the traversal and shading are latency-bound, and
  // lanes left free to diverge give the scheduler more independent loads in
  // flight than a warp forced back together at every event.
  while (active) {
    bool ended = stepPath<kGpuLayout>(c, ps, sp);
    resolveShadow<kGpuLayout>(c, ps);
    if (ended && spectral) ended = finishWavelength(J, ps, sp);
    else if (ended && split) ended = finishAlphaSplit(J, ps, sp);
    if (ended) {
      endSample(J, idx, ps);
      if (--left == 0u) active = false;
      else beginSample(c, x, y, ps, sp);
    }
  }
  cnt.ext += c.cnt.ext;
  cnt.shadow += c.cnt.shadow;
}

}  // namespace mt
