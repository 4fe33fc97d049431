// Test infrastructure only (the checker, never the product).
//
// Lights, environment, material resolve, next-event estimation and the RGB
// integrator of the CPU oracle.
#include <cstdio>
#include <cstdlib>

#include "oracle_bsdf.h"

namespace oracle {

static const V3 kLuminance = {0.2126f, 0.7152f, 0.0722f};

// ------------------------------------------------------------ environment
// envMap.wgsl.ts:10-31 textureLinear on an RGBA32F image
static V4 textureLinear(const V4 *tex, u32 w, u32 h, V2 uv) {
  float ux = uv.x * float(w) - 0.5f, uy = uv.y * float(h) - 0.5f;
  float fx = std::floor(ux), fy = std::floor(uy);
  float tx = ux - fx, ty = uy - fy;
  i32 ix = i32(fx), iy = i32(fy);
  auto at = [&](i32 x, i32 y) {
    x = std::min(std::max(x, 0), i32(w) - 1);
    y = std::min(std::max(y, 0), i32(h) - 1);
    return tex[size_t(y) * w + x];
  };
  V4 s1 = at(ix, iy), s2 = at(ix + 1, iy), s3 = at(ix, iy + 1), s4 = at(ix + 1, iy + 1);
  auto mix4 = [](V4 a, V4 b, float t) {
    return V4{a.x * (1.0f - t) + b.x * t, a.y * (1.0f - t) + b.y * t, a.z * (1.0f - t) + b.z * t,
              a.w * (1.0f - t) + b.w * t};
  };
  return mix4(mix4(s1, s2, tx), mix4(s3, s4, tx), ty);
}
// envMap.wgsl.ts:33-41
V2 cartesianToEquirect(V3 p) {
  float phi = std::atan2(-p.z, -p.x);
  if (phi < 0.0f) phi += TWOPI;
  float theta = std::acos(clampf(p.y, -1.0f, 1.0f));
  return {phi * 0.5f * INVPI, theta * INVPI};
}
// envMap.wgsl.ts:43-49
static V3 envRotCol(const Scene &s, int c) {
  const float *m = s.u->environment_rotation;
  return {m[c * 4 + 0], m[c * 4 + 1], m[c * 4 + 2]};
}
static V2 environmentUv(const Scene &s, V3 d) {
  return cartesianToEquirect({dot(envRotCol(s, 0), d), dot(envRotCol(s, 1), d), dot(envRotCol(s, 2), d)});
}
static inline V2 distAt(const Scene &s, i32 x, i32 y) {
  const float *p = s.envDist + (size_t(y) * (s.envW + 2) + x) * 2;
  return {p[0], p[1]};
}
// envMap.wgsl.ts:51-75
static float getEnvmapV(const Scene &s, float u, i32 &vOffset, V2 &pdf) {
  i32 left = 0, right = i32(s.envH) + 1;
  while (left < right) {
    i32 mid = (left + right) >> 1;
    if (distAt(s, 0, mid).x <= u) left = mid + 1; else right = mid;
  }
  vOffset = left - 1;
  V2 s0 = distAt(s, 0, vOffset), s1 = distAt(s, 0, vOffset + 1);
  pdf.y = s0.y;
  return (float(vOffset) + (u - s0.x) / (s1.x - s0.x)) / float(s.envH);
}
// envMap.wgsl.ts:77-99
static float getEnvmapU(const Scene &s, float u, i32 vOffset, V2 &pdf) {
  i32 left = 0, right = i32(s.envW) + 1;
  while (left < right) {
    i32 mid = (left + right) >> 1;
    if (distAt(s, 1 + mid, vOffset).x <= u) left = mid + 1; else right = mid;
  }
  i32 uOffset = left - 1;
  V2 s0 = distAt(s, 1 + uOffset, vOffset), s1 = distAt(s, 1 + uOffset + 1, vOffset);
  pdf.x = s0.y;
  return (float(uOffset) + (u - s0.x) / (s1.x - s0.x)) / float(s.envW);
}
// envMap.wgsl.ts:103-107
static float envMapSolidAnglePdf(V2 partial, float v) {
  if (!(v > 0.0f && v < 1.0f)) return 0.0f;
  float sinTheta = std::sin(fminf(v, 1.0f - v) * PI);
  return partial.x * partial.y * INVPI2 / (2.0f * sinTheta);
}
// envMap.wgsl.ts:110-130
V3 sampleEnvmap(const Scene &s, V2 rnd, V2 &uv, float &pdf) {
  V2 partial{0, 0};
  i32 vOffset;
  uv.y = getEnvmapV(s, rnd.x, vOffset, partial);
  uv.x = getEnvmapU(s, rnd.y, vOffset, partial);
  float phi = uv.x * TWOPI, theta = uv.y * PI;
  float ct = std::cos(theta), st = std::sin(theta), cp = std::cos(phi), sp = std::sin(phi);
  V3 dir = {-st * cp, ct, -st * sp};
  pdf = envMapSolidAnglePdf(partial, uv.y);
  return envRotCol(s, 0) * dir.x + envRotCol(s, 1) * dir.y + envRotCol(s, 2) * dir.z;
}
// envMap.wgsl.ts:132-141
float envMapPdf(const Scene &s, V2 uv) {
  i32 x = i32(uv.x * float(s.envW)), y = i32(uv.y * float(s.envH));
  x = std::min(std::max(x, 0), i32(s.envW) - 1);
  y = std::min(std::max(y, 0), i32(s.envH) - 1);
  float px = distAt(s, 1 + x, y).y, py = distAt(s, 0, y).y;
  return envMapSolidAnglePdf({px, py}, uv.y);
}
// background.wgsl.ts:84-99 (no background map)
static V4 sampleSceneBackground(const Scene &s, const Ray &r) {
  if (s.u->background_flags & MTC_BACKGROUND_COLOR) {
    const float *c = s.u->background_color;
    return {c[0], c[1], c[2], c[3]};
  }
  if (s.useEnvmap()) return textureLinear(s.env, s.envW, s.envH, environmentUv(s, r.d));
  return {0, 0, 0, 0};
}
static V3 spectralFilter(V3 rgb, i32 channel) {
  if (channel == 0) return rgb;
  V3 f = v3(0.0f);
  setcomp(f, channel - 1, comp(rgb, channel - 1));
  return f;
}

// --------------------------------------------------------------- spectrum
// spectrum.ts:10-88: continuous wavelength sampling.  The inverse-CDF tables
// are built in float64 exactly as the reference's module builds them when it
// loads (Wyman-Sloan-Shirley CIE lobes -> linear sRGB, clamp, per-channel
// scale rounded to 6 decimals, 60 bins x 20 midpoint substeps, every CDF value
// rounded to 7 decimals), then read as f32 like the WGSL literals.
namespace {
struct SpectrumTables {
  float cdf[4 * 61];
  double scale[3];
  static void unnormalized(double wl, double rgb[3]) {
    static const double lobes[3][3][4] = {
        {{1.056, 599.8, 37.9, 31.0}, {0.362, 442.0, 16.0, 26.7}, {-0.065, 501.1, 20.4, 26.2}},
        {{0.821, 568.8, 46.9, 40.5}, {0.286, 530.9, 16.3, 31.1}, {0, 0, 0, 0}},
        {{1.217, 437.0, 11.8, 36.0}, {0.681, 459.0, 26.0, 13.8}, {0, 0, 0, 0}}};
    static const int counts[3] = {3, 2, 2};
    static const double m[3][3] = {{3.2406, -1.5372, -0.4986}, {-0.9689, 1.8758, 0.0415}, {0.0557, -0.204, 1.057}};
    double xyz[3];
    for (int c = 0; c < 3; c++) {
      double sum = 0;
      for (int l = 0; l < counts[c]; l++) {
        const double *L = lobes[c][l];
        double t = (wl - L[1]) / (wl < L[1] ? L[2] : L[3]);
        sum += L[0] * std::exp(-0.5 * t * t);
      }
      xyz[c] = sum;
    }
    for (int r = 0; r < 3; r++) rgb[r] = std::max(0.0, m[r][0] * xyz[0] + m[r][1] * xyz[1] + m[r][2] * xyz[2]);
  }
  static double rounded(double v, int digits) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.*f", digits, v);
    return std::strtod(buf, nullptr);
  }
  SpectrumTables() {
    const int steps = 3000;
    double sum[3] = {0, 0, 0};
    for (int i = 0; i < steps; i++) {
      double rgb[3];
      unnormalized(400.0 + (300.0 * (i + 0.5)) / steps, rgb);
      for (int c = 0; c < 3; c++) sum[c] += rgb[c] / steps;
    }
    for (int c = 0; c < 3; c++) scale[c] = rounded(1.0 / sum[c], 6);
    for (int d = 0; d <= 3; d++) {
      double cdf[61];
      cdf[0] = 0;
      for (int b = 0; b < 60; b++) {
        double mass = 0;
        for (int i = 0; i < 20; i++) {
          double rgb[3];
          unnormalized(400.0 + (b + (i + 0.5) / 20) * 5.0, rgb);
          for (int c = 0; c < 3; c++) rgb[c] *= scale[c];
          mass += d == 3 ? rgb[0] + rgb[1] + rgb[2] : rgb[d];
        }
        cdf[b + 1] = cdf[b] + mass;
      }
      for (int b = 0; b <= 60; b++) {
        char buf[64];
        std::snprintf(buf, sizeof buf, "%.7f", cdf[b] / cdf[60]);
        this->cdf[d * 61 + b] = std::strtof(buf, nullptr);
      }
    }
  }
};
const SpectrumTables &spectrumTables() {
  static const SpectrumTables t;
  return t;
}
}  // namespace

// spectrum.ts:133-141 spectrumSample + spectrumIorWavelength: the refracting
// wavelength of a camera path that carries one RGB channel.
static float spectrumCameraWavelength(u32 channel, float u) {
  const float *cdf = spectrumTables().cdf + channel * 61u;
  u32 low = 0, high = 60;
  while (high - low > 1u) {
    u32 middle = (low + high) / 2u;
    if (cdf[middle] <= u) low = middle; else high = middle;
  }
  float mass = cdf[low + 1] - cdf[low];
  float wavelength = 400.0f + 5.0f * (float(low) + (u - cdf[low]) / mass);
  if (wavelength >= 500.0f) return wavelength;
  return 500.0f - 25.0f * (1.0f - std::exp((wavelength - 500.0f) / 25.0f));
}

// ------------------------------------------------------------------ lights
struct Light {
  V3 position; float litType; V3 emission; float area; V3 u; float radiusOrSpread; V3 v; float textureIndex;
  float selectionPmf; V3 iesReference;
};
static Light loadLight(const Scene &s, i32 i) {
  const V4 *L = s.lights + size_t(i) * MTC_LIGHT_VEC4_ROWS;
  return {xyz(L[0]), L[0].w, xyz(L[1]), L[1].w, xyz(L[2]), L[2].w, xyz(L[3]), L[3].w, L[4].x, xyz(L[5])};
}
struct LightSample {
  V3 normal{}, emission{}, direction{};
  float dist = 0, pdf = 0, selectionPmf = 0;
  bool isDelta = false;
  u32 sourceType = 0, sourceIndex = 0;
};
// intersect.wgsl.ts:894-919
static float intersectSphere(float rad, V3 pos, const Ray &r) {
  V3 op = pos - r.o;
  const float eps = 0.001f;
  float b = dot(op, r.d);
  float det = b * b - dot(op, op) + rad * rad;
  if (det < 0.0f) return INF;
  det = std::sqrt(det);
  float t1 = b - det;
  if (t1 > eps) return t1;
  float t2 = b + det;
  if (t2 > eps) return t2;
  return INF;
}
// intersect.wgsl.ts:921-939
static float intersectRect(V3 pos, V3 u, V3 v, V3 n, const Ray &r) {
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
// intersect.wgsl.ts:941-949
static float sphereSolidAnglePdf(V3 origin, V3 center, float radius) {
  float cd = distance(origin, center);
  if (cd <= radius) return INV4PI;
  float s2 = fminf(1.0f, radius * radius / (cd * cd));
  float ct = std::sqrt(fmaxf(0.0f, 1.0f - s2));
  float omc = s2 / (1.0f + ct);
  return 1.0f / fmaxf(TWOPI * omc, 1e-8f);
}
// rayTraceCore.wgsl.ts:362-375 (no IES texture)
static float spotEmissionMultiplier(const Light &L, V3 lightToSurface) {
  V3 axis = normalize(L.u);
  float cosTheta = dot(axis, lightToSurface);
  float cone = cosTheta >= L.v.x ? 1.0f : 0.0f;
  if (L.v.y > L.v.x + 1e-6f) cone = smoothstepf(L.v.x, L.v.y, cosTheta);
  return cone;
}
// intersect.wgsl.ts:976-1131
static float intersectLight(const Ray &r, const Light &L, LightSample &ls) {
  float d = INF;
  ls.direction = r.d; ls.normal = -r.d; ls.dist = INF; ls.pdf = 0.0f; ls.emission = v3(0.0f); ls.isDelta = false;
  V3 u = L.u, v = L.v;
  i32 type = i32(L.litType);
  if (type == MTC_LIGHT_RECT) {
    V3 pos = L.position - u * 0.5f - v * 0.5f;
    V3 normal = normalize(cross(u, v));
    if (dot(normal, r.d) > 0.0f) return INF;
    d = intersectRect(pos, u, v, normal, r);
    if (d < 0.0f) d = INF;
    else {
      float cosTheta = dot(-r.d, normal);
      if (cosTheta >= std::cos(L.radiusOrSpread * PI / 2.0f)) {
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
    float root = std::sqrt(disc);
    float nearT = (-b - root) / a, farT = (-b + root) / a;
    d = nearT > EPS ? nearT : farT;
    float axial = dot(oc + r.d * d, axis);
    if (d <= EPS || std::fabs(axial) > halfLength) return INF;
    V3 hit = r.o + r.d * d;
    V3 normal = normalize(hit - L.position - axis * axial);
    float cosine = dot(-r.d, normal);
    if (cosine <= 0.0f) return INF;
    ls.direction = r.d; ls.normal = normal; ls.dist = d;
    ls.pdf = d * d / fmaxf(L.area * cosine, 1e-8f);
    ls.emission = L.emission;
  } else if (type == MTC_LIGHT_SPHERE) {
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
      if (d > 0.0f && d != INF) {
        ls.direction = r.d; ls.dist = d;
        ls.normal = normalize(r.o + r.d * d - L.position);
        ls.pdf = sphereSolidAnglePdf(r.o, L.position, L.radiusOrSpread);
      }
    }
    if (d < 0.0f) d = INF;
    else {
      ls.direction = r.d; ls.dist = d;
      ls.emission = L.radiusOrSpread <= 0.0f ? L.emission / fmaxf(d * d, 1e-8f) : L.emission;
    }
  } else if (type == MTC_LIGHT_SPOT) {
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
    }
    if (d != INF) {
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
static void lightSampleSphere(const Light &L, V3 p, V2 rnd, LightSample &ls) {
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
    float radial = std::sqrt(fmaxf(0.0f, 1.0f - z * z));
    float az = TWOPI * rnd.y;
    sd = {radial * std::cos(az), radial * std::sin(az), z};
    ls.pdf = INV4PI;
  } else {
    V3 axis = co / cd;
    float s2 = fminf(1.0f, radius * radius / (cd * cd));
    float ctm = std::sqrt(fmaxf(0.0f, 1.0f - s2));
    float omctm = s2 / (1.0f + ctm);
    float omct = rnd.x * omctm;
    float ct = 1.0f - omct;
    float st = std::sqrt(fmaxf(0.0f, omct * (2.0f - omct)));
    float az = TWOPI * rnd.y;
    V3 t, b;
    orthonormalBasis(axis, t, b);
    sd = axis * ct + t * (st * std::cos(az)) + b * (st * std::sin(az));
    ls.pdf = 1.0f / fmaxf(TWOPI * omctm, 1e-8f);
  }
  float cp = dot(sd, co);
  float co2 = dot(co, co);
  float disc = cp * cp - co2 + radius * radius;
  float nearT = cp - std::sqrt(fmaxf(0.0f, disc));
  float farT = cp + std::sqrt(fmaxf(0.0f, disc));
  ls.dist = nearT > 1e-6f ? nearT : farT;
  ls.direction = sd;
  V3 lp = p + sd * ls.dist;
  ls.normal = normalize(lp - L.position);
  ls.emission = L.emission;
}
// sampleLight.wgsl.ts:108-161 (no light texture)
static void lightSampleRect(const Light &L, V3 p, V2 rnd, LightSample &ls) {
  V3 normal = normalize(cross(L.u, L.v));
  V3 lowerLeft = L.position - (L.u + L.v) * 0.5f;
  float spread = clampf(L.radiusOrSpread, 0.0f, 1.0f);
  if (spread <= 0.001f) {
    float pd = dot(normal, p - L.position);
    V3 sp = p - normal * pd;
    V3 rel = sp - lowerLeft;
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
  ls.dist = std::sqrt(d2);
  ls.direction = off / ls.dist;
  ls.normal = normal;
  float ec = dot(-ls.direction, normal);
  float sc = std::cos(0.5f * PI * spread);
  if (ec <= 0.0f || ec < sc) { ls.emission = v3(0.0f); ls.pdf = 0.0f; return; }
  ls.emission = L.emission;
  ls.pdf = d2 / fmaxf(L.area * ec, 1e-8f);
}
// sampleLight.wgsl.ts:163-177
static void lightSampleDisk(const Light &L, V3 p, V2 rnd, LightSample &ls) {
  float r = std::sqrt(rnd.x);
  float phi = TWOPI * rnd.y;
  V3 sp = L.position + L.u * (r * std::cos(phi)) + L.v * (r * std::sin(phi));
  V3 normal = normalize(cross(L.u, L.v));
  V3 off = sp - p;
  float d2 = dot(off, off);
  ls.dist = std::sqrt(d2);
  ls.direction = off / fmaxf(ls.dist, 1e-8f);
  ls.normal = normal;
  float ec = dot(-ls.direction, normal);
  if (ec <= 0.0f) { ls.emission = v3(0.0f); ls.pdf = 0.0f; return; }
  ls.emission = L.emission;
  ls.pdf = d2 / fmaxf(L.area * ec, 1e-8f);
}
// sampleLight.wgsl.ts:179-195
static void lightSampleCylinder(const Light &L, V3 p, V2 rnd, LightSample &ls) {
  V3 axis = normalize(L.u);
  V3 r0 = normalize(L.v);
  V3 r1 = normalize(cross(axis, r0));
  float phi = TWOPI * rnd.y;
  V3 normal = r0 * std::cos(phi) + r1 * std::sin(phi);
  V3 sp = L.position + L.u * (rnd.x - 0.5f) + normal * L.radiusOrSpread;
  V3 off = sp - p;
  float d2 = dot(off, off);
  ls.dist = std::sqrt(d2);
  ls.direction = off / fmaxf(ls.dist, 1e-8f);
  ls.normal = normal;
  float ec = dot(-ls.direction, normal);
  if (ec <= 0.0f) { ls.emission = v3(0.0f); ls.pdf = 0.0f; return; }
  ls.emission = L.emission;
  ls.pdf = d2 / fmaxf(L.area * ec, 1e-8f);
}
// sampleLight.wgsl.ts:197-244
static void sampleAnalyticLight(const Light &L, V3 p, V2 rnd, LightSample &ls) {
  i32 type = i32(L.litType);
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
  if (type == MTC_LIGHT_DISK) { lightSampleDisk(L, p, rnd, ls); return; }
  if (type == MTC_LIGHT_CYLINDER) lightSampleCylinder(L, p, rnd, ls);
}
// sampleLight.wgsl.ts:319-357 (material emission without maps)
// getMaterialEmission (materialBuffer.wgsl.ts:381-403).
// getMapUvSet (materialBuffer.wgsl.ts:329-331).
static V2 getMapUvSet(const Scene &s, i32 idx, V2 uv, V2 uv1) {
  return s.maps[size_t(idx) * MTC_MAP_VEC4_ROWS + 2].x > 0.5f ? uv1 : uv;
}

V3 getMaterialEmission(const Scene &s, i32 materialIndex, V2 uv, V2 uv1) {
  const V4 *d = s.mats + size_t(materialIndex) * MTC_MATERIAL_VEC4_ROWS;
  V3 emission = xyz(d[3]);
  const i32 emissiveMapIndex = i32(d[3].w);
  if (mapValid(s, d[3].w)) {
    V4 t = sampleMap(s, emissiveMapIndex, getMapUvSet(s, emissiveMapIndex, uv, uv1));
    emission = emission * decodeMapColor(s, emissiveMapIndex, {t.x, t.y, t.z});
  }
  if (d[0].w == 0.0f) {
    const i32 coatWeightMapIndex = i32(d[6].x);
    if (mapValid(s, d[6].x)) {
      const float coatWeight = clampf(d[16].w, 0.0f, 1.0f) * sampleMap(s, coatWeightMapIndex, getMapUvSet(s, coatWeightMapIndex, uv, uv1)).x;
      const V3 c = {std::sqrt(fmaxf(d[16].x, 0.0f)), std::sqrt(fmaxf(d[16].y, 0.0f)), std::sqrt(fmaxf(d[16].z, 0.0f))};
      emission = emission * V3{1.0f * (1.0f - coatWeight) + c.x * coatWeight, 1.0f * (1.0f - coatWeight) + c.y * coatWeight,
                               1.0f * (1.0f - coatWeight) + c.z * coatWeight};
    }
  }
  return emission;
}

static void sampleEmissiveTriangle(const Scene &s, i32 index, V3 p, V2 rnd, LightSample &ls) {
  const V4 *t = s.lightData + size_t(index) * 6;
  V3 p0 = xyz(t[0]), p1 = xyz(t[1]), p2 = xyz(t[2]);
  float selectionPmf = t[0].w, area = t[1].w;
  i32 materialIndex = i32(t[2].w);
  float su = std::sqrt(rnd.x);
  V3 b = {1.0f - su, su * (1.0f - rnd.y), su * rnd.y};
  V3 lp = p0 * b.x + p1 * b.y + p2 * b.z;
  V3 normal = normalize(cross(p1 - p0, p2 - p0));
  ls.direction = lp - p;
  ls.dist = length(ls.direction);
  if (ls.dist <= EPS) { ls.emission = v3(0.0f); ls.pdf = 0.0f; return; }
  ls.direction /= ls.dist;
  ls.normal = normal;
  float cl = dot(normal, -ls.direction);
  if (cl <= 0.0f) { ls.emission = v3(0.0f); ls.pdf = 0.0f; return; }
  // getMaterialEmission at the unscaled barycentric UV (sampleLight.wgsl.ts:331-358)
  V2 uv = {b.x * t[3].x + b.y * t[3].z + b.z * t[4].x, b.x * t[3].y + b.y * t[3].w + b.z * t[4].y};
  V2 uv1 = {b.x * t[4].z + b.y * t[5].x + b.z * t[5].z, b.x * t[4].w + b.y * t[5].y + b.z * t[5].w};
  ls.emission = getMaterialEmission(s, materialIndex, uv, uv1);
  ls.selectionPmf = selectionPmf;
  ls.pdf = selectionPmf * (ls.dist * ls.dist) / fmaxf(area * cl, 1e-8f);
}
// sampleLight.wgsl.ts:359-420 sampleLightChoiceTable (table offset 0, scale 1)
static void sampleLightChoiceTable(const Scene &s, V3 p, V3 rnd, LightSample &ls) {
  ls.emission = v3(0.0f); ls.pdf = 0.0f; ls.selectionPmf = 0.0f; ls.dist = INF; ls.isDelta = false;
  ls.sourceType = 0; ls.sourceIndex = 0xffffffffu;
  i32 count = s.u->light_choice_count;
  if (count <= 0) return;
  float scaled = rnd.z * float(count);
  i32 column = std::min(i32(scaled), count - 1);
  V4 cc = s.lightData[s.u->light_choice_texel_offset + column];
  i32 selected = fractf(scaled) < cc.x ? column : asi(cc.y);
  V4 ch = s.lightData[s.u->light_choice_texel_offset + selected];
  i32 type = asi(ch.z), src = asi(ch.w);
  if (s.useEnvmap() && type == MTC_CHOICE_ENVIRONMENT) {
    ls.sourceType = 0; ls.sourceIndex = u32(src);
    V2 uv;
    float pdf;
    ls.direction = sampleEnvmap(s, {rnd.x, rnd.y}, uv, pdf);
    ls.pdf = pdf;
    ls.emission = xyz(textureLinear(s.env, s.envW, s.envH, uv));
    ls.dist = INF;
    ls.selectionPmf = s.u->env_light_pmf;
    ls.pdf *= s.u->env_light_pmf;
  } else if (type == MTC_CHOICE_ANALYTIC) {
    ls.sourceType = 2; ls.sourceIndex = u32(src);
    Light L = loadLight(s, src);
    sampleAnalyticLight(L, p, {rnd.x, rnd.y}, ls);
    ls.selectionPmf = L.selectionPmf;
    ls.pdf *= L.selectionPmf;
  } else if (type == MTC_CHOICE_EMISSIVE_TRIANGLE) {
    ls.sourceType = 1; ls.sourceIndex = u32(src);
    sampleEmissiveTriangle(s, src, p, {rnd.x, rnd.y}, ls);
  }
}

// --------------------------------------------------------------- material
// materialBuffer.wgsl.ts:170-257 getMaterial with its texture block
// (:79-139 and the slots of materialTextureSlots.ts)
Material getMaterial(const Scene &s, i32 materialIndex, i32 instanceIndex, V2 uv, V2 uv1, V3 vertexColor) {
  const V4 *d = s.mats + size_t(materialIndex) * MTC_MATERIAL_VEC4_ROWS;
  Material m;
  m.baseColor = xyz(d[0]);
  m.materialType = i32(d[0].w);
  m.specularRoughness = d[1].x;
  m.baseMetalness = d[2].x;
  m.specularAnisotropy = clampf(d[2].y, 0.0f, 1.0f);
  m.emission = getMaterialEmission(s, materialIndex, uv, uv1);
  m.inside = false;
  m.specularIor = d[4].x;
  m.transmissionWeight = d[4].y;
  m.thinWalled = d[4].w > 0.5f;
  m.bevel = d[5].x;
  m.transmissionDispersionScale = d[5].y;
  m.dispersionAbbeNumber = fmaxf(d[18].y, 1e-6f);
  m.mediumExtinction = vmax(xyz(d[20]), v3(0.0f));
  m.mediumScattering = vmax(xyz(d[21]), v3(0.0f));
  m.mediumAnisotropy = clampf(d[20].w, -1.0f, 1.0f);
  m.mediumType = maxc(m.mediumExtinction) > 0.0f ? 1 : 0;
  m.alpha = d[9].x;
  m.alphaMode = i32(d[23].w);
  m.thinFilmThickness = d[5].z * 1000.0f;
  m.thinFilmIor = d[9].z;
  m.thinFilmWeight = s.feature(MTC_FEATURE_HAS_THIN_FILM) ? clampf(d[18].x, 0.0f, 1.0f) : 0.0f;
  m.baseWeight = clampf(d[10].x, 0.0f, 1.0f);
  m.diffuseRoughness = clampf(d[10].y, 0.0f, 1.0f);
  m.specularWeight = fmaxf(d[10].z, 0.0f);
  m.specularColor = vmax(xyz(d[11]), v3(0.0f));
  m.subsurfaceWeight = s.feature(MTC_FEATURE_HAS_SUBSURFACE) ? clampf(d[10].w, 0.0f, 1.0f) : 0.0f;
  m.subsurfaceColor = vmax(xyz(d[14]), v3(0.0f));
  m.transmissionColor = vmax(xyz(d[12]), v3(0.0f));
  m.fuzzWeight = s.feature(MTC_FEATURE_HAS_FUZZ) ? clampf(d[11].w, 0.0f, 1.0f) : 0.0f;
  m.fuzzColor = vmax(xyz(d[15]), v3(0.0f));
  m.fuzzRoughness = clampf(d[15].w, 0.0f, 1.0f);
  m.coatWeight = s.feature(MTC_FEATURE_HAS_COAT) ? clampf(d[16].w, 0.0f, 1.0f) : 0.0f;
  m.coatColor = vmax(xyz(d[16]), v3(0.0f));
  m.coatRoughness = clampf(d[17].x, ROUGHNESS_MIN, 1.0f);
  m.coatAnisotropy = clampf(d[17].y, 0.0f, 1.0f);
  m.coatIor = fmaxf(d[17].z, 1.0f);
  m.coatDarkening = clampf(d[17].w, 0.0f, 1.0f);
  const i32 diffuseMapIndex = i32(d[2].z);
  if (mapValid(s, d[2].z)) {
    V4 t = sampleMap(s, diffuseMapIndex, getMapUvSet(s, diffuseMapIndex, uv, uv1));
    m.baseColor = m.baseColor * decodeMapColor(s, diffuseMapIndex, {t.x, t.y, t.z});
    // mapAlphaUsageConstants (materialConstants.ts:2): 3 transmission, 2 alpha
    if (d[5].w == 3.0f) m.transmissionWeight = 1.0f - t.w;
    else if (d[5].w == 2.0f) m.alpha *= t.w;
  }
  // simpleTextureSample (materialTextureSlots.ts:184-212): factor *= channel
  auto simple = [&](float index, float &target, int channel) {
    if (!mapValid(s, index)) return;
    const i32 idx = i32(index);
    V4 t = sampleMap(s, idx, getMapUvSet(s, idx, uv, uv1));
    target *= channel == 0 ? t.x : channel == 1 ? t.y : channel == 2 ? t.z : t.w;
  };
  simple(d[22].z, m.alpha, 1);  // alphaMap: g
  // alpha mode resolution (materialBuffer.wgsl.ts:65-73)
  if (m.alphaMode == 0) m.alpha = 1.0f;
  else if (m.alphaMode == 1) m.alpha = m.alpha >= d[22].w ? 1.0f : 0.0f;
  simple(d[9].w, m.transmissionWeight, 0);  // transmissionMap: r
  const i32 mrtMapIndex = i32(d[2].w);
  if (mapValid(s, d[2].w)) {
    V4 t = sampleMap(s, mrtMapIndex, getMapUvSet(s, mrtMapIndex, uv, uv1));
    m.baseMetalness *= t.z;
    m.specularRoughness *= t.y;
  }
  simple(d[22].x, m.specularRoughness, 1);  // roughnessMap: g
  simple(d[22].y, m.baseMetalness, 2);      // metalnessMap: b
  const i32 thinFilmMapIndex = i32(d[9].y);
  if (mapValid(s, d[9].y)) {
    // thinFilmTextureSample (materialTextureSlots.ts:214-228)
    V4 t = sampleMap(s, thinFilmMapIndex, getMapUvSet(s, thinFilmMapIndex, uv, uv1));
    if (d[25].z == 0.0f && d[25].w == 0.0f) {
      m.thinFilmThickness *= t.x;
    } else {
      const i32 channel = i32(d[25].w);
      const float k = channel == 0 ? t.x : channel == 1 ? t.y : channel == 2 ? t.z : t.w;
      m.thinFilmThickness = (d[25].z * (1.0f - k) + d[5].z * k) * 1000.0f;
    }
  }
  simple(d[6].x, m.coatWeight, 0);      // coatWeightMap: r
  simple(d[6].y, m.coatRoughness, 1);   // coatRoughnessMap: g
  const i32 fuzzColorMapIndex = i32(d[6].w);
  if (mapValid(s, d[6].w)) {
    V4 t = sampleMap(s, fuzzColorMapIndex, getMapUvSet(s, fuzzColorMapIndex, uv, uv1));
    m.fuzzColor = m.fuzzColor * decodeMapColor(s, fuzzColorMapIndex, {t.x, t.y, t.z});
  }
  simple(d[18].w, m.fuzzRoughness, 3);  // fuzzRoughnessMap: a
  simple(d[19].w, m.specularWeight, 3); // specularWeightMap: a
  const i32 specularColorMapIndex = i32(d[21].w);
  if (mapValid(s, d[21].w)) {
    V4 t = sampleMap(s, specularColorMapIndex, getMapUvSet(s, specularColorMapIndex, uv, uv1));
    m.specularColor = m.specularColor * decodeMapColor(s, specularColorMapIndex, {t.x, t.y, t.z});
  }
  m.anisotropyDirection = {1.0f, 0.0f};
  m.anisotropyDirectionEnabled = d[24].y != 0.0f;
  m.coatAnisotropyRotation = d[25].x;
  if (d[25].y > 0.5f && m.specularAnisotropy > 0.0f) {
    // gltf_anisotropy_to_openpbr (materialBuffer.wgsl.ts:260-266)
    float roughness = clampf(m.specularRoughness, 0.0f, 1.0f), strength = m.specularAnisotropy;
    float u = roughness * roughness;
    float a = u + (1.0f - u) * strength * strength;
    if (a == 0.0f) { m.specularRoughness = 0.0f; m.specularAnisotropy = 0.0f; }
    else {
      m.specularRoughness = std::pow((a * a + u * u) * 0.5f, 0.25f);
      m.specularAnisotropy = clampf(1.0f - u / a, 0.0f, 1.0f);
    }
  }
  if (m.anisotropyDirectionEnabled) {
    float theta = d[24].y;
    V2 dd = m.anisotropyDirection;
    m.anisotropyDirection = {std::cos(theta) * dd.x - std::sin(theta) * dd.y, std::sin(theta) * dd.x + std::cos(theta) * dd.y};
  }
  if (m.coatWeight > 0.0f && m.coatRoughness > 0.0f) {
    float br2 = m.specularRoughness * m.specularRoughness;
    float cr2 = m.coatRoughness * m.coatRoughness;
    m.specularRoughness = mixf(m.specularRoughness, std::pow(fminf(1.0f, br2 * br2 + 2.0f * cr2 * cr2), 0.25f), m.coatWeight);
  }
  V3 color = v3(1.0f);
  if (instanceIndex >= 0) color = xyz(s.ins[size_t(instanceIndex) * MTC_INSTANCE_VEC4_STRIDE + 9]);
  color = color * vertexColor;  // getInstanceColor(instanceIndex) * vertexColor
  m.baseColor *= color;
  if (m.materialType == 2) m.emission *= color;
  m.specularRoughness = clampf(m.specularRoughness, ROUGHNESS_MIN, 1.0f);
  m.baseMetalness = clampf(m.baseMetalness, 0.0f, 1.0f);
  V2 a = roughnessToAlpha(m.specularRoughness, m.specularAnisotropy);
  m.alphaX = a.x;
  m.alphaY = a.y;
  return m;
}

// ------------------------------------------------------------- integrator
struct Path {
  bool scatteringMediumEntered = false;
  Ray ray{};
  V3 li{}; float alpha = 0; V3 beta{};
  bool fromEye = false, abort = false;
  float scatteringPdf = 0; bool scatteringIsDelta = false, isNextRefraction = false;
};
struct Aux { V3 albedo{}; bool isShadowCatcher = false; V3 normal{}; bool isBlank = false; };

struct Ctx {
  const Scene &s;
  Sampler smp;
  BsdfContext bc;
  Traffic *tr;
  u32 candidateCount() const { return u32(std::max(s.u->direct_light_candidates, 1)); }
};

// rayTrace.compute.ts:264-284
static float neeMISWeight(const Ctx &c, float lightPdf, float scatteringPdf) {
  u32 n = c.candidateCount();
  if (n <= 1u) return powerHeuristic(lightPdf, scatteringPdf);
  float w = float(n) * lightPdf;
  return w / fmaxf(w + scatteringPdf, 1e-20f);
}
static float bsdfMISWeight(const Ctx &c, float scatteringPdf, float lightPdf) {
  u32 n = c.candidateCount();
  if (n <= 1u) return powerHeuristic(scatteringPdf, lightPdf);
  float w = float(n) * lightPdf;
  return scatteringPdf / fmaxf(scatteringPdf + w, 1e-20f);
}
// common.wgsl.ts:14-20
static V3 offsetSurfaceRay(V3 p, V3 gn, V3 dir) {
  V3 n = dot(gn, dir) >= 0.0f ? gn : -gn;
  V3 r;
  for (int k = 0; k < 3; k++) {
    float pc = comp(p, k), nc = comp(n, k);
    i32 io = i32(256.0f * nc);
    i32 bits = asi(pc);
    i32 sh = bits + (pc < 0.0f ? -io : io);
    float shifted;
    std::memcpy(&shifted, &sh, 4);
    setcomp(r, k, std::fabs(pc) < 1.0f / 32.0f ? pc + nc / 65536.0f : shifted);
  }
  return r;
}
static V3 initCameraRayDir(const Scene &s, V2 coord, V3 &origin) {
  const float *m = s.cam->view_projection_inv;
  V4 o = mat4_mul4(m, {coord.x * 2.0f - 1.0f, coord.y * 2.0f - 1.0f, -1.0f, 1.0f});
  V4 c = mat4_mul4(m, {coord.x * 2.0f - 1.0f, coord.y * 2.0f - 1.0f, 1.0f, 1.0f});
  origin = {o.x / o.w, o.y / o.w, o.z / o.w};
  V3 cd = {c.x * o.w - o.x * c.w, c.y * o.w - o.y * c.w, c.z * o.w - o.z * c.w};
  return normalize(cd);
}
// rayTrace.compute.ts:592-600 initCameraRay
static Ray initCameraRay(const Scene &s, V2 coord) {
  Ray r;
  r.d = initCameraRayDir(s, coord, r.o);
  return r;
}
static V3 cameraEye(const Scene &s) {
  const float *v = s.cam->view_inv;
  return {v[12], v[13], v[14]};
}

struct ShadowWork {
  Ray ray{}; float maxDistance = 0; i32 triangleIndex = 0; V3 contribution{};
  float risTarget = 0, lightSelectionPmf = 0; bool valid = false;
};
// sampleMaterial.wgsl.ts:32-151 finishDirectLight
static bool finishDirectLight(Ctx &c, SurfaceInteraction &si, const Material &ma, Path &path, V3 ffnormal,
                              bool isSurface, const LightSample &ls, V3 f, float scatteringPdf, ShadowWork &w) {
  w.valid = false; w.lightSelectionPmf = 0.0f; w.risTarget = 0.0f;
  (void)ma;
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
    nl = std::fabs(nl);
    float gl = dot(gn, lightDir);
    float off = nl < cutoff ? clampf(2.0f - (gl + nl) / cutoff, 0.0f, 1.0f) : clampf(1.0f - gl / cutoff, 0.0f, 1.0f);
    shadowOrigin += si.shadowOffset * off;
  }
  V3 visDir = lightDir;
  float visDist = ls.dist - EPS;
  if (ls.sourceType == 1u) {
    V3 end = si.position + ls.direction * ls.dist;
    V3 offEnd = end + ls.normal * EPS;
    V3 to = offEnd - shadowOrigin;
    visDist = length(to);
    visDir = normalize(to);
  }
  Ray lightRay{shadowOrigin, visDir};
  if (isSurface && cosThetaL < 0.0f && ls.sourceType == 0u) {
    V4 bg = sampleSceneBackground(c.s, lightRay);
    Li = V3{bg.x, bg.y, bg.z} * bg.w;
  }
  // Spectral scenes use channel-independent RIS (WGPURayTracePass.ts:1349,
  // sampleMaterial.wgsl.ts:119-140): with three wavelengths the radiance is
  // filtered after the target, and each RGB component weighs 1/3.
  const bool spectral = (c.s.flags & MTC_SCENE_SPECTRAL) != 0;
  const bool threeWavelengths = spectral && c.s.u->dispersion_wavelengths != 1;
  if (spectral && !threeWavelengths) Li = spectralFilter(Li, si.spectralChannel);
  float mis = ls.isDelta ? 1.0f : neeMISWeight(c, lightPdf, scatteringPdf);
  if (mis > 0.0f) {
    V3 un = Li * f / lightPdf * path.beta;
    const V3 targetWeights = threeWavelengths ? v3(1.0f / 3.0f) : kLuminance;
    w.risTarget = fmaxf(dot(vmax(un * lsp, v3(0.0f)), targetWeights), 0.0f);
    w.ray = lightRay;
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

struct Scattering { V3 direction{}, response{}; float pdf = 0; bool transmission = false; };

static bool isDiscrete(const Prepared &p) {
  return !p.material.thinWalled && std::fabs(p.material.relativeIor - 1.0f) <= 1e-6f &&
         p.probabilities[LOBE_TRANSMISSION] >= 1.0f - 1e-6f;
}

// sampleMaterial.wgsl.ts:160-277 sampleScattering
static Scattering sampleScattering(Ctx &c, SurfaceInteraction &si, const Material &ma, const Prepared &prepared,
                                   Path &path, V3 ffnormal, bool isSurface) {
  u32 count = c.candidateCount();
  ShadowWork selected;
  float selectedTarget = 0.0f, scalarWeightSum = 0.0f;
  Scattering result;
  for (u32 event = 0; event <= count; event++) {
    bool continuation = event == count;
    LightSample ls;
    V3 lightDir{};
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
      if (valid && !intersectSceneShadow(c.s, selected.ray, selected.maxDistance, selected.triangleIndex,
                                         si.instanceIndex, c.tr, &c.smp))
        path.li += selected.contribution * ucw;
      if (!isSurface) {
        result.direction = henyeyGreenstein(-path.ray.d, si.mediumAnisotropy, c.smp.s2(c.smp.bounceDim(6)));
        result.pdf = henyeyGreensteinPhase(dot(result.direction, -path.ray.d), si.mediumAnisotropy);
        return result;
      }
      V2 dr = c.smp.s2(c.smp.bounceDim(3));
      float lobe = c.smp.s1(c.smp.bounceDim(2));
      V3 matRnd = {dr.x, dr.y, lobe};
      discrete = isDiscrete(prepared);
      if (discrete) {
        lightDir = toWorld(prepared.basis, -prepared.viewLocal);
        response = transmissionTint(c.bc, prepared.material) * coatBaseScale(c.bc, prepared, -prepared.viewLocal.z);
        scatteringPdf = 1.0f;
        result.transmission = true;
      } else {
        bool transmission = false;
        if (!sampleDirection(c.bc, prepared, matRnd, lightDir, transmission)) return result;
        result.transmission = transmission;
      }
    } else {
      V2 lr = c.smp.s2(c.smp.lightDim(event, 1u));
      float lz = c.smp.s1(c.smp.lightDim(event, 0u));
      V3 rnd = {lr.x, lr.y, (lz + float(std::min(event, count - 1u))) / float(std::max(count, 1u))};
      sampleLightChoiceTable(c.s, si.position, rnd, ls);
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
    if (!finishDirectLight(c, si, ma, path, ffnormal, isSurface, ls, response, scatteringPdf, cand)) continue;
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
static float emissiveHitMisWeight(Ctx &c, SurfaceInteraction &si, Path &path) {
  const V4 *md = c.s.mats + size_t(si.materialIndex) * MTC_MATERIAL_VEC4_ROWS;
  float cosLight = dot(si.faceNormal, -path.ray.d);
  if (cosLight <= 0.0f && md[23].z < 0.5f) return 0.0f;
  if (path.fromEye || c.s.u->light_weight_total <= 0.0f || i32(md[0].w) == 2) return 1.0f;
  float lum = dot(xyz(md[3]), kLuminance);
  if (lum <= 0.0f || cosLight <= 0.0f) return 1.0f;
  float hd = distance(si.position, path.ray.o);
  float lightPdf = lum / c.s.u->light_weight_total * hd * hd / fmaxf(cosLight, 1e-8f);
  return bsdfMISWeight(c, path.scatteringPdf, lightPdf);
}

// sampleMaterial.wgsl.ts:316-508 SampleMaterial
static void sampleMaterial(Ctx &c, SurfaceInteraction &si, Material &ma, Path &path) {
  const bool hasMedium = (c.s.flags & MTC_SCENE_HAS_MEDIUM) != 0;
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
      i32 ch = std::min(i32(c.smp.s1(c.smp.bounceDim(4)) * 3.0f), 2);
      float ce = comp(ext, ch);
      float sd = ce > 0.0f ? fminf(-std::log(fmaxf(c.smp.s1(c.smp.bounceDim(5)), 1e-7f)) / ce, d) : d;
      mediumSampled = sd < d;
      V3 T = {std::exp(-ext.x * sd), std::exp(-ext.y * sd), std::exp(-ext.z * sd)};
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
    V3 se = ma.emission;
    if (c.s.flags & MTC_SCENE_SPECTRAL) se = spectralFilter(se, si.spectralChannel);
    path.li += se * emissiveHitMisWeight(c, si, path) * path.beta;
  }
  if (ma.materialType == 2) { path.abort = true; return; }
  Prepared prepared;
  if (!mediumSampled) {
    ma.directionTangent = si.directionTangent;
    ma.directionBitangent = si.directionBitangent;
    ma.geometryTangent = si.geometryTangent;
    ma.geometryBitangent = si.geometryBitangent;
    prepared = prepare(c.bc, si.tangent, ma, -path.ray.d, ffnormal);
  }
  Scattering sc = sampleScattering(c, si, ma, prepared, path, ffnormal, !mediumSampled);
  V3 scatterDir = sc.direction;
  float scatteringPdf = sc.pdf;
  if (!mediumSampled) {
    V3 f = sc.response;
    bool nextRefraction = sc.transmission;
    bool finite = f.x == f.x && f.y == f.y && f.z == f.z && std::fabs(f.x) < 3.402823e38f &&
                  std::fabs(f.y) < 3.402823e38f && std::fabs(f.z) < 3.402823e38f;
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
      path.scatteringMediumEntered = path.scatteringMediumEntered ||
          ma.mediumScattering.x > 0.0f || ma.mediumScattering.y > 0.0f || ma.mediumScattering.z > 0.0f;
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
static void shadeVertex(Ctx &c, V2 uv, Path &path, int &depth, SurfaceInteraction &si, Material &ma, Aux &aux,
                        bool &sampleIgnored) {
  sampleIgnored = false;
  c.smp.bounce = u32(std::max(depth, 0));
  i32 matType = ma.materialType;
  const mtc_trace_uniform &u = *c.s.u;
  if (!si.hit) {
    V4 bg = sampleSceneBackground(c.s, path.ray);
    if (c.s.flags & MTC_SCENE_SPECTRAL) {
      V3 f = spectralFilter({bg.x, bg.y, bg.z}, si.spectralChannel);
      bg = {f.x, f.y, f.z, bg.w};
    }
    if (path.fromEye) {
      path.li = path.beta * V3{bg.x, bg.y, bg.z} * bg.w;
      path.alpha = bg.w;
      aux.isBlank = bg.w < 0.001f || ((u.background_flags & MTC_BACKGROUND_COLOR) && !(u.background_flags & MTC_BACKGROUND_MAP));
    } else {
      Ray cam = initCameraRay(c.s, uv);
      bool towardsCam = dot(cam.d, path.ray.d) > 0.0f;
      if (u.transmissive_output_alpha_min < 1.0f) {
        if (towardsCam) path.alpha = fmaxf(path.alpha, bg.w); else path.alpha = 1.0f;
      }
      if (!c.s.useEnvmap()) {
        if (towardsCam) path.li += path.beta * (bsdfMISWeight(c, path.scatteringPdf, 1.0f)) * V3{bg.x, bg.y, bg.z};
      }
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
      float oa = fmaxf(1.0f - ma.transmissionWeight, 1.0f - std::pow(1.0f - u.transmissive_output_alpha_min, float(depth)));
      path.alpha = fmaxf(oa, path.alpha);
    }
    if (!sampleIgnored) sampleMaterial(c, si, ma, path);
    else path.ray.o = si.position + path.ray.d * EPS;
  }
  if (!si.albedoSampled && !sampleIgnored) {
    if (matType == 0 || matType == 2) {
      if (!(ma.transmissionWeight > 0.5f || (ma.specularRoughness <= 0.02f && ma.baseMetalness > 0.98f))) {
        aux.albedo = ma.baseColor;
        aux.normal = dot(si.normal, si.position - cameraEye(c.s)) > 0.0f ? -si.normal : si.normal;
        si.albedoSampled = true;
      }
      if (depth > 4) si.albedoSampled = true;
    }
  }
  // Russian roulette, RR_MAX = 12 (wgpuMaterialConstants.ts:67-69)
  if (depth >= (path.scatteringMediumEntered ? 12 : 2) && !sampleIgnored) {
    float mc = maxc(path.beta);
    float q = fmaxf(0.0f, 1.0f - mc);
    if (c.smp.s1(c.smp.bounceDim(7)) < q) { path.alpha = 1.0f; path.abort = true; }
    else path.beta /= 1.0f - q;
  }
}

// rayTrace.compute.ts:514-589 completeVertex
static void completeVertex(Ctx &c, Path &path, int &depth, SurfaceInteraction &si, Material &ma, bool sampleIgnored) {
  const bool spectral = (c.s.flags & MTC_SCENE_SPECTRAL) != 0;
  if (spectral && ma.transmissionWeight > 0.001f)
    ma.specularIor = cauchyIor(si.wavelength, ma.specularIor, ma.transmissionDispersionScale, ma.dispersionAbbeNumber);
  if (sampleIgnored) return;
  bool isAlphaOccluded = c.smp.hashedSample(3u) < ma.alpha;
  for (i32 i = 0; i < c.s.u->lights_count; i++) {
    Light L = loadLight(c.s, i);
    LightSample ls;
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
  if (c.s.useEnvmap()) {
    if (!(si.hit && isAlphaOccluded)) {
      if (path.isNextRefraction) {
        V4 bg = sampleSceneBackground(c.s, path.ray);
        if (spectral) { V3 f = spectralFilter({bg.x, bg.y, bg.z}, si.spectralChannel); bg = {f.x, f.y, f.z, bg.w}; }
        float w = path.scatteringIsDelta ? 1.0f
                  : bsdfMISWeight(c, path.scatteringPdf, envMapPdf(c.s, environmentUv(c.s, path.ray.d)) * c.s.u->env_light_pmf);
        path.li += path.beta * V3{bg.x, bg.y, bg.z} * (w * bg.w);
        path.alpha = fmaxf(path.alpha, bg.w);
        path.abort = true;
        return;
      }
      V2 euv = environmentUv(c.s, path.ray.d);
      V3 emission = xyz(textureLinear(c.s.env, c.s.envW, c.s.envH, euv));
      float mis = bsdfMISWeight(c, path.scatteringPdf, envMapPdf(c.s, euv) * c.s.u->env_light_pmf);
      if (spectral) emission = spectralFilter(emission, si.spectralChannel);
      if (!(c.s.u->background_flags & MTC_BACKGROUND_COLOR)) path.alpha = 1.0f;
      path.li += path.beta * emission * mis;
      path.abort = true;
    }
  }
  depth = depth + 1;
}

// rayTrace.compute.ts:891-946 (RGB integrator, no alpha split)
static V4 integrateRgb(Ctx &c, V2 uv, const Ray &ray, Aux &aux) {
  SurfaceInteraction si;
  Material ma;
  Path path;
  path.ray = ray;
  path.alpha = c.s.u->transmissive_output_alpha_min < 1.0f ? 0.0f : 1.0f;
  path.beta = v3(1.0f);
  path.fromEye = true;
  int bounceLimit = std::max(c.s.u->bounces, 0);
  int eventLimit = std::min(bounceLimit * 3, 20);
  bool isNotTransparent = false;
  int depth = 0;
  bool sampleIgnored = false;
  for (int event = 0; event <= eventLimit; event++) {
    intersectScene(c.s, path.ray, si, depth, event != 0, c.tr);
    ma = getMaterial(c.s, si.materialIndex, si.instanceIndex, si.uv, si.uv1, si.vertexColor);
    if (c.tr) c.tr->material_fetches++;
    if (event == 0) {
      if (si.hit && (ma.materialType == 0 || ma.materialType == 2)) {
        aux.albedo = ma.transmissionWeight > 0.5f ? v3(1.0f) : ma.baseColor;
        aux.normal = dot(si.normal, si.position - cameraEye(c.s)) > 0.0f ? -si.normal : si.normal;
        si.albedoSampled = ma.transmissionWeight > 0.5f;
      }
      aux.isShadowCatcher = false;
      isNotTransparent = ma.transmissionWeight < 0.001f && ma.subsurfaceWeight < 0.001f && ma.alpha > 0.99f;
    } else {
      completeVertex(c, path, depth, si, ma, sampleIgnored);
    }
    if (isNotTransparent && event > bounceLimit) path.abort = true;
    if (path.abort || event >= eventLimit) break;
    shadeVertex(c, uv, path, depth, si, ma, aux, sampleIgnored);
    if (path.abort) break;
  }
  return {path.li.x, path.li.y, path.li.z, path.alpha};
}

// rayTrace.compute.ts:815-890: the RGB integrator of scenes with alpha
// (deterministicPrimaryAlpha).  A standard or unlit primary hit with coverage
// below 1 splits the sample: the back path continues through the surface
// first, then the front path restarts at the primary vertex with full
// coverage, and the two are mixed by the coverage.
static V4 integrateRgbAlpha(Ctx &c, V2 uv, const Ray &ray, Aux &outAux) {
  SurfaceInteraction si;
  Material ma;
  SurfaceInteraction primarySi;
  Material primaryMa;
  Aux primaryAux;
  bool primaryReady = false, query = true, split = false, front = false;
  float coverage = 1.0f;
  V4 back{0, 0, 0, 0};
  Aux backAux;
  auto freshPath = [&]() {
    Path p;
    p.ray = ray;
    p.alpha = c.s.u->transmissive_output_alpha_min < 1.0f ? 0.0f : 1.0f;
    p.beta = v3(1.0f);
    p.fromEye = true;
    return p;
  };
  Path path = freshPath();
  const int bounceLimit = std::max(c.s.u->bounces, 0);
  const int eventLimit = std::min(bounceLimit * 3, 20);
  int event = 0, depth = 0;
  bool sampleIgnored = false, isNotTransparent = false;
  for (int step = 0; step < (20 + 1) * 2 + 2; step++) {
    if (query) {
      intersectScene(c.s, path.ray, si, depth, event != 0, c.tr);
      ma = getMaterial(c.s, si.materialIndex, si.instanceIndex, si.uv, si.uv1, si.vertexColor);
      if (c.tr) c.tr->material_fetches++;
    }
    query = true;
    if (!primaryReady) {
      if (si.hit && (ma.materialType == 0 || ma.materialType == 2)) {
        outAux.albedo = ma.transmissionWeight > 0.5f ? v3(1.0f) : ma.baseColor;
        outAux.normal = dot(si.normal, si.position - cameraEye(c.s)) > 0.0f ? -si.normal : si.normal;
        si.albedoSampled = ma.transmissionWeight > 0.5f;
      }
      outAux.isShadowCatcher = false;
      primarySi = si; primaryMa = ma; primaryAux = outAux;
      primaryReady = true;
      coverage = clampf(ma.alpha, 0.0f, 1.0f);
      split = si.hit && (ma.materialType == 0 || ma.materialType == 2) && coverage < 1.0f;
      if (split) {
        path.ray.o = si.position + ray.d * (EPS * 0.02f);
        si.albedoSampled = false;
        continue;
      }
    } else if (event == 0 && !front && split) {
      if (si.hit && ma.materialType == 0) {
        outAux.albedo = ma.transmissionWeight > 0.5f ? v3(1.0f) : ma.baseColor;
        outAux.normal = dot(si.normal, si.position - cameraEye(c.s)) > 0.0f ? -si.normal : si.normal;
        si.albedoSampled = ma.transmissionWeight > 0.5f;
      }
    }
    if (event == 0) {
      isNotTransparent = ma.transmissionWeight < 0.001f && ma.subsurfaceWeight < 0.001f && ma.alpha > 0.99f;
    } else {
      completeVertex(c, path, depth, si, ma, sampleIgnored);
    }
    if (isNotTransparent && event > bounceLimit) path.abort = true;
    if (!path.abort && event < eventLimit) shadeVertex(c, uv, path, depth, si, ma, outAux, sampleIgnored);
    if (path.abort || event >= eventLimit) {
      V4 result = {path.li.x, path.li.y, path.li.z, path.alpha};
      if (!split || coverage <= 0.0f) return result;
      if (front) {
        auto mix3 = [&](V3 a, V3 b) { return a * (1.0f - coverage) + b * coverage; };
        outAux.albedo = mix3(backAux.albedo, outAux.albedo);
        V3 n = mix3(backAux.normal, outAux.normal);
        outAux.normal = dot(n, n) > 1e-12f ? normalize(n) : v3(0.0f);
        outAux.isBlank = backAux.isBlank && outAux.isBlank;
        outAux.isShadowCatcher = backAux.isShadowCatcher && outAux.isShadowCatcher;
        return {back.x * (1.0f - coverage) + result.x * coverage, back.y * (1.0f - coverage) + result.y * coverage,
                back.z * (1.0f - coverage) + result.z * coverage, back.w * (1.0f - coverage) + result.w * coverage};
      }
      back = result; backAux = outAux;
      front = true; query = false; event = 0; depth = 0; sampleIgnored = false;
      si = primarySi; ma = primaryMa; ma.alpha = 1.0f; outAux = primaryAux;
      path = freshPath();
    } else {
      event++;
    }
  }
  return {0.0f, 0.0f, 0.0f, 0.0f};
}

// rayTrace.compute.ts:947-1057: the spectral integrator (independent
// wavelength paths, shareSpectralPrefix off).  The primary hit is traced once
// and reused by the three wavelength paths (or one hero wavelength when
// dispersionWavelengths == 1); each path restarts from the primary vertex with
// the sampler state saved after the wavelength draw, refracts with a Cauchy
// IOR at its wavelength, and its radiance is filtered to its RGB channel.
// The path-prefix checkpoint of the shared-prefix spectral integrator
// (rayTrace.compute.ts:145-148 flatPrefix, spectralPrefix.wgsl.ts:52-56): the
// loop state at the fork vertex, and the sampler state (PCG words, hashed
// counter, Sobol bounce) the wavelength paths after the first restart from.
struct SpectralFlatPrefix {
  Path path;
  SurfaceInteraction si;
  Material ma;
  Aux aux;
  int depth = 0, event = 0;
  bool ignored = false, opaque = false;
  u32 s0[4] = {0, 0, 0, 0};
  u32 hashed = 0, bounce = 0;
};

// spDisperses (spectralPrefix.wgsl.ts:29-31).
static inline bool spDisperses(const Material &ma) {
  return ma.transmissionDispersionScale > 0.0f && ma.specularIor != 1.0f;
}

// The spectral integrator of rayTrace.compute.ts:947-1057.  With three
// wavelengths it shares the path prefix (the reference's default,
// WGPURayTracePass.ts:2113,2122): unless the primary surface disperses, the
// first wavelength path runs in RGB (spectral channel 0) until it reaches a
// dispersive transmissive surface past the primary vertex; there it saves
// its state and forks (spFork), and the second and third wavelength paths
// resume from that checkpoint with their own wavelength.  A path that never
// forks is the whole sample.  MTC_SCENE_SPECTRAL_INDEPENDENT turns sharing
// off: every wavelength path is spectral from the camera.
static V4 integrateSpectral(Ctx &c, V2 uv, const Ray &ray, Aux &outAux) {
  SurfaceInteraction si, primarySi;
  Material ma, primaryMa;
  bool primaryReady = false;
  Path path;
  path.ray = ray;
  const int bounceLimit = std::max(c.s.u->bounces, 0);
  const int eventLimit = std::min(bounceLimit * 3, 20);
  int depth = 0, event = 0;
  bool sampleIgnored = false, isNotTransparent = false;
  int wavelengthIndex = 0;
  const bool singleWavelength = c.s.u->dispersion_wavelengths == 1;
  bool dispersivePrimary = false;
  int heroWavelengthIndex = 0;
  float wavelengthSample = 0.0f;
  u32 savedS0[4] = {0, 0, 0, 0};
  u32 savedHashed = 0;
  Aux wavelengthAux;
  V3 color = v3(0.0f);
  float alpha = 0.0f;
  V3 guideAlbedo = v3(0.0f), guideNormal = v3(0.0f);
  bool allBlank = true;
  // spectralPrefix.wgsl.ts:13-27 state.
  const bool spEnabled = !singleWavelength && !(c.s.flags & MTC_SCENE_SPECTRAL_INDEPENDENT);
  bool spActive = false;
  int spChannel = 0, spForkCall = -1;
  float spWavelength = 0.0f;
  SpectralFlatPrefix spFlat;
  auto spFork = [&]() {  // spectralPrefix.wgsl.ts:32-36
    spActive = false;
    path.li = spectralFilter(path.li, spChannel);
    si.spectralChannel = spChannel;
    si.wavelength = spWavelength;
  };
  const int stepLimit = std::min((20 + 1) * 3, int(c.s.u->loop_unroll_guard * 16u));
  for (int step = 0; step < stepLimit; step++) {
    if (!primaryReady || (event != 0 && !path.abort)) {
      intersectScene(c.s, path.ray, si, depth, event != 0, c.tr);
      ma = getMaterial(c.s, si.materialIndex, si.instanceIndex, si.uv, si.uv1, si.vertexColor);
      if (c.tr) c.tr->material_fetches++;
    }
    if (event == 0) {
      if (!primaryReady) {
        if (si.hit && (ma.materialType == 0 || ma.materialType == 2)) {
          outAux.albedo = ma.transmissionWeight > 0.5f ? v3(1.0f) : ma.baseColor;
          outAux.normal = dot(si.normal, si.position - cameraEye(c.s)) > 0.0f ? -si.normal : si.normal;
          si.albedoSampled = ma.transmissionWeight > 0.5f;
        }
        outAux.isShadowCatcher = false;
        primarySi = si;
        primaryMa = ma;
        primaryReady = true;
        dispersivePrimary = si.hit && ma.transmissionWeight > 0.001f && ma.transmissionDispersionScale > 0.001f;
        wavelengthSample = c.smp.s1(2u);  // CAMERA_WAVELENGTH, sobol.wgsl.ts:5
        if (singleWavelength) {
          heroWavelengthIndex = std::min(int(std::floor(wavelengthSample * 3.0f)), 2);
          float w3 = wavelengthSample * 3.0f;
          wavelengthSample = w3 - std::floor(w3);
        }
        for (int k = 0; k < 4; k++) savedS0[k] = c.smp.s0[k];
        savedHashed = c.smp.hashed;
      }
      si = primarySi;
      ma = primaryMa;
      wavelengthAux = outAux;
      if (!singleWavelength) {
        for (int k = 0; k < 4; k++) c.smp.s0[k] = savedS0[k];
        c.smp.hashed = savedHashed;
        c.smp.bounce = 0;
        wavelengthAux.isBlank = false;
        wavelengthAux.isShadowCatcher = false;
      }
      si.wavelength = 0.0f;
      si.spectralChannel = 0;
      if (!singleWavelength || dispersivePrimary) {
        int channel = singleWavelength ? heroWavelengthIndex : wavelengthIndex;
        si.spectralChannel = channel + 1;
        si.wavelength = spectrumCameraWavelength(u32(channel), wavelengthSample);
        // spBegin (spectralPrefix.wgsl.ts:22-27)
        spChannel = channel + 1;
        spWavelength = si.wavelength;
        spActive = spEnabled && !spDisperses(ma);
        if (spActive) si.spectralChannel = 0;
        ma.specularIor = cauchyIor(si.wavelength, ma.specularIor, ma.transmissionDispersionScale,
                                   ma.dispersionAbbeNumber);
      }
      path = Path();
      path.ray = ray;
      path.beta = v3(1.0f);
      path.fromEye = true;
      path.alpha = c.s.u->transmissive_output_alpha_min < 1.0f ? 0.0f : 1.0f;
      depth = 0;
      sampleIgnored = false;
      isNotTransparent = ma.transmissionWeight < 0.001f && ma.subsurfaceWeight < 0.001f && ma.alpha > 0.99f;
      if (spActive && wavelengthIndex > 0 && spForkCall == 0) {
        // Resume at the first wavelength's fork vertex (:1010-1013).
        path = spFlat.path;
        si = spFlat.si;
        ma = spFlat.ma;
        wavelengthAux = spFlat.aux;
        depth = spFlat.depth;
        event = spFlat.event;
        sampleIgnored = spFlat.ignored;
        isNotTransparent = spFlat.opaque;
        for (int k = 0; k < 4; k++) c.smp.s0[k] = spFlat.s0[k];
        c.smp.hashed = spFlat.hashed;
        c.smp.bounce = spFlat.bounce;
        spFork();
      }
    }
    if (event > 0 && !path.abort) {
      if (spActive && ma.transmissionWeight > 0.001f && spDisperses(ma)) {
        // The first dispersive transmission of the RGB prefix (:1015-1019).
        spFlat.path = path;
        spFlat.si = si;
        spFlat.ma = ma;
        spFlat.aux = wavelengthAux;
        spFlat.depth = depth;
        spFlat.event = event;
        spFlat.ignored = sampleIgnored;
        spFlat.opaque = isNotTransparent;
        for (int k = 0; k < 4; k++) spFlat.s0[k] = c.smp.s0[k];
        spFlat.hashed = c.smp.hashed;
        spFlat.bounce = c.smp.bounce;
        spForkCall = 0;
        spFork();
      }
      completeVertex(c, path, depth, si, ma, sampleIgnored);
    }
    if (isNotTransparent && event > bounceLimit) path.abort = true;
    if (!path.abort && event < eventLimit) shadeVertex(c, uv, path, depth, si, ma, wavelengthAux, sampleIgnored);
    if (path.abort || event >= eventLimit) {
      if (singleWavelength) {
        outAux = wavelengthAux;
        float scale = dispersivePrimary ? 3.0f : 1.0f;
        return {path.li.x * scale, path.li.y * scale, path.li.z * scale, path.alpha};
      }
      if (spActive) {
        // No fork: the RGB path is the whole sample (:1035-1041).
        outAux.isBlank = wavelengthAux.isBlank;
        outAux.albedo = (wavelengthAux.albedo + wavelengthAux.albedo + wavelengthAux.albedo) / 3.0f;
        outAux.normal = (wavelengthAux.normal + wavelengthAux.normal + wavelengthAux.normal) / 3.0f;
        return {path.li.x, path.li.y, path.li.z, path.alpha};
      }
      color += path.li;
      alpha = std::max(alpha, path.alpha);
      guideAlbedo += wavelengthAux.albedo;
      guideNormal += wavelengthAux.normal;
      allBlank = allBlank && wavelengthAux.isBlank;
      wavelengthIndex++;
      if (wavelengthIndex >= 3) {
        outAux.albedo = guideAlbedo / 3.0f;
        outAux.normal = guideNormal / 3.0f;
        outAux.isBlank = allBlank;
        return {color.x, color.y, color.z, alpha};
      }
      event = 0;
    } else {
      event++;
    }
  }
  return {0, 0, 0, 0};
}

// rayTrace.compute.ts:1157-1263 main, for one pixel and one sample.
void tracePixel(const Scene &s, u32 x, u32 y, V4 *outColor, V4 *outNormal, V4 *outAlbedo, V4 *outCatcher,
                Traffic *tr) {
  const mtc_trace_uniform &u = *s.u;
  u32 W = u32(u.output_size[0]), H = u32(u.output_size[1]);
  if (x >= W || y >= H) return;
  u32 idx = x + y * W;
  Ctx c{s, Sampler(), BsdfContext{s.lut, (s.flags & MTC_SCENE_HAS_MEDIUM) != 0, s.feature(MTC_FEATURE_HAS_THIN_FILM)}, tr};
  V2 outputSize = {u.output_size[0], u.output_size[1]};
  V2 uv = {(float(x) + 0.5f) / outputSize.x, (float(y) + 0.5f) / outputSize.y};
  c.smp.px = x; c.smp.py = y; c.smp.width = W;
  c.smp.index = u32(outNormal[idx].w) + u.sample_sequence_offset;
  c.smp.bounce = 0; c.smp.hashed = 0;
  c.smp.seed = u.sequence_seed; c.smp.logspp = u.zsobol_log_spp;
  c.smp.pattern = int((s.flags & MTC_SCENE_PATTERN_MASK) >> MTC_SCENE_PATTERN_SHIFT);
  V2 jitter = {u.jitter[0], u.jitter[1]};
  if (c.smp.pattern == 0 || c.smp.pattern == 1) {
    V2 j = c.smp.s2(0u);
    jitter = {(j.x - 0.5f) / outputSize.x, (j.y - 0.5f) / outputSize.y};
  }
  u32 frame = c.smp.index ^ sampleHash(u.sequence_seed);
  c.smp.s0[0] = x; c.smp.s0[1] = y; c.smp.s0[2] = frame; c.smp.s0[3] = x + y;
  V2 coord = {uv.x + jitter.x, uv.y + jitter.y};
  Ray cam = initCameraRay(s, coord);
  if (s.cam->aperture_radius > 0.0f) {
    V3 eye = cameraEye(s);
    const float *vi = s.cam->view_inv;
    V3 forward = -normalize(V3{vi[8], vi[9], vi[10]});
    V3 focus = eye + cam.d * (s.cam->focus_distance / dot(cam.d, forward));
    // sampleCircle, rayTrace.compute.ts:1148-1154
    V2 ip = c.smp.s2(1u);
    V2 pp = {2.0f * ip.x - 1.0f, 2.0f * ip.y - 1.0f};
    bool greater = std::fabs(pp.x) > std::fabs(pp.y);
    float r = greater ? pp.x : pp.y;
    float theta = greater ? 0.25f * PI * pp.y / pp.x : PI * (0.5f - 0.25f * pp.x / pp.y);
    V2 lens = {s.cam->aperture_radius * r * std::cos(theta), s.cam->aperture_radius * r * std::sin(theta)};
    V4 o4 = mat4_mul4(vi, {lens.x, lens.y, 0.0f, 1.0f});
    V3 origin = {o4.x, o4.y, o4.z};
    cam = {origin, normalize(focus - origin)};
  }
  Aux aux;
  V4 li = (s.flags & MTC_SCENE_SPECTRAL) ? integrateSpectral(c, coord, cam, aux)
          : (s.flags & MTC_SCENE_HAS_ALPHA) ? integrateRgbAlpha(c, coord, cam, aux)
                                             : integrateRgb(c, coord, cam, aux);
  if (tr) tr->paths++;
  if (u.clamping > 0.0f) {
    float cl = u.clamping;
    li = {clampf(li.x, -cl, cl), clampf(li.y, -cl, cl), clampf(li.z, -cl, cl), li.w};
  }
  if (!(li.x < INF && li.x > -EPS)) li = {0, 0, 0, 1};
  outColor[idx].x += li.x; outColor[idx].y += li.y; outColor[idx].z += li.z; outColor[idx].w += li.w;
  outAlbedo[idx].x += aux.albedo.x; outAlbedo[idx].y += aux.albedo.y; outAlbedo[idx].z += aux.albedo.z;
  outAlbedo[idx].w += aux.isBlank ? 0.0f : 1.0f;
  if (u.variance_moments != 0) {
    float v = dot({li.x, li.y, li.z}, kLuminance);
    outNormal[idx].x += v * v; outNormal[idx].w += 1.0f;
  } else {
    outNormal[idx].x += aux.normal.x; outNormal[idx].y += aux.normal.y; outNormal[idx].z += aux.normal.z;
    outNormal[idx].w += 1.0f;
  }
  float lum = dot({li.x, li.y, li.z}, kLuminance);
  V4 &mom = outCatcher[size_t(idx) * 3 + 2];
  mom.x += lum;
  mom.y += lum * lum;
}

}  // namespace oracle

// ----------------------------------------------------------- test exports
// Environment and BSDF entry points for the known-answer tests.
extern "C" {

// The 4 x 61 wavelength-sampling CDFs and the spectrumCameraWavelength map.
int oracle_spectrum_cdf(float *out, unsigned capacity) {
  const auto &t = oracle::spectrumTables();
  for (unsigned i = 0; i < 244 && i < capacity; i++) out[i] = t.cdf[i];
  return 244;
}
float oracle_spectrum_camera_wavelength(unsigned channel, float u) {
  return oracle::spectrumCameraWavelength(channel, u);
}
// spectrum.ts:79-93 spectrumSample on the f32 table (distribution 0-2: RGB
// camera channels, 3: photons): the wavelength, and its pdf in *pdf.
float oracle_spectrum_sample(unsigned distribution, float u, float *pdf) {
  const float *cdf = oracle::spectrumTables().cdf + distribution * 61u;
  unsigned low = 0, high = 60;
  while (high - low > 1u) {
    unsigned middle = (low + high) / 2u;
    if (cdf[middle] <= u) low = middle; else high = middle;
  }
  float mass = cdf[low + 1] - cdf[low];
  if (pdf) *pdf = mass / 5.0f;
  return 400.0f + 5.0f * (float(low) + (u - cdf[low]) / mass);
}

// envMapPdf(uv) and sampleEnvmap(rnd) over a scene's environment:
// out = {envMapPdf(u, v), sampled pdf, envMapPdf(sampled uv), |direction|}
// (the quantities tests/gpu/environmentPdf.ts:5-10 checks).
int oracle_env_case(const mtc_scene_view *sv, const mtc_trace_uniform *u, float pu, float pv, float r0, float r1,
                    float *out) {
  oracle::Scene s;
  s.env = (const om::V4 *)sv->env_map;
  s.envDist = (const float *)sv->env_distribution;
  s.envW = sv->env_width;
  s.envH = sv->env_height;
  s.u = u;
  if (!s.env || !s.envDist) return 2;
  om::V2 uv;
  float pdf;
  om::V3 d = oracle::sampleEnvmap(s, {r0, r1}, uv, pdf);
  out[0] = oracle::envMapPdf(s, {pu, pv});
  out[1] = pdf;
  out[2] = oracle::envMapPdf(s, uv);
  out[3] = om::length(d);
  return 0;
}

// Resolves material row block `rows` (26 x vec4) with the scene feature bits
// `features`, prepares the BSDF for view direction `view` about normal +z and
// evaluates it for `light`: out = {f*cos rgb, pdf}.  sample != 0 instead draws
// a direction with rnd[3] and returns {f*cos rgb, pdf, dir xyz, transmission}.
int oracle_bsdf(const float *rows, uint32_t features, const float *view, const float *light, const float *rnd,
                int sample, const float *lut, float *out) {
  mtc_trace_uniform u{};
  u.scene_feature_flags = features;
  float ins[40] = {0};
  ins[36] = ins[37] = ins[38] = 1.0f;
  oracle::Scene s;
  s.mats = (const om::V4 *)rows;
  s.ins = (const om::V4 *)ins;
  s.u = &u;
  oracle::Material m = oracle::getMaterial(s, 0, 0, {0.0f, 0.0f}, {0.0f, 0.0f}, om::v3(1.0f));
  om::V3 v = om::normalize({view[0], view[1], view[2]});
  om::V3 n = {0.0f, 0.0f, 1.0f};
  float ndv = om::dot(v, n);
  m.inside = ndv <= 0.0f && !m.thinWalled;
  m.relativeIor = ndv > 0.0f ? 1.0f / m.specularIor : m.specularIor;
  om::V3 ff = ndv >= 0.0f ? n : -n;
  oracle::BsdfContext c{lut, false, (features & MTC_FEATURE_HAS_THIN_FILM) != 0};
  oracle::Prepared p = oracle::prepare(c, om::v3(0.0f), m, v, ff);
  om::V3 l = {light ? light[0] : 0.0f, light ? light[1] : 0.0f, light ? light[2] : 1.0f};
  bool trans = false;
  if (sample) {
    if (!oracle::sampleDirection(c, p, {rnd[0], rnd[1], rnd[2]}, l, trans)) {
      for (int k = 0; k < 8; k++) out[k] = 0.0f;
      return 1;
    }
  }
  float pdf = 0.0f;
  om::V3 f = oracle::evalPrepared(c, p, l, pdf);
  out[0] = f.x; out[1] = f.y; out[2] = f.z; out[3] = pdf;
  if (sample) { out[4] = l.x; out[5] = l.y; out[6] = l.z; out[7] = trans ? 1.0f : 0.0f; }
  return 0;
}

}  // extern "C"
