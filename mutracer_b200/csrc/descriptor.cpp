// Scene descriptor v8 ingest: the byte buffer of mt_context_commit
// (native/docs/scene-format.md, native/include/mutracer-scene.h records,
// native/include/mutracer-layout.h word offsets) decoded and validated into
// the flattened scene this library renders.
//
// Decoding follows the reference's record decoders (native/src/
// scene-records.ts: decodeMaterial :41-54, decodeGeometry :56-82,
// decodeMeshMaterials :84-91, decodeInstances :93-100, lightFromRecord
// :102-114), its camera (native/src/camera-core.ts:11-31 with Camera.ts
// getProjectionMatrix :127-155, cameraLens.ts:4-15, the vendored gl-matrix
// perspective / ortho / invert / multiply of src/math/mat4.ts), its light
// rows (wgpuSceneUniform.ts:70-152 packWgpuAnalyticLights, lightsData.ts
// :104-156 frames and areas) and selection powers (lightSampling.ts:72-107),
// generated normals (src/util/vertexNormals.ts:9-52), material emission
// (materialEmission.ts:10-22) and the environment controls of
// native/src/scene-core.ts:1696-1711.  The flattened buffers then come from
// the same producers as every other scene here: BLAS per geometry (8 bins),
// TLAS over the instances (8 bins), compact vertices, material rows, light
// sampling, environment distribution.
//
// Malformed descriptors are rejected with MT_ERROR_INVALID_ARGUMENT and a
// message naming the problem, as the reference's validator does.  Valid
// descriptors that use what this build does not render (displacement,
// anisotropy and coat-normal maps, UDIM sets, textures the atlas would
// downscale, alpha in spectral scenes, material
// graphs, IES profiles, rect-light textures, background maps and grounded
// projection, anisotropic materials in scenes with vertex tangents or UVs,
// bevel, shadow catchers, unlit materials, the remaining material
// extensions) are refused with
// MT_ERROR_UNAVAILABLE and a message naming the feature.
//
// Material textures (scene-records.ts:22-39 decodeTexture, MaterialData.ts
// :19-56, textureAtlas.ts:134-283, textureAtlasPixels.ts:9-66) become this
// library's map table: the maps in mergeTexturesFromMaterials order (slot
// by slot, material by material, one entry per texture), texels as RGBA f32
// at full size (the atlas keeps full size whenever its shelf packing fits;
// otherwise the descriptor is refused), rows flipped at packing for flip_y,
// RGBA8 as byte / 255 or, when any material texture is RGBA32F, every texel
// rounded to half precision as RGBA16F storage holds it.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <tuple>
#include <vector>

#include "mtp_api.h"
#include "scene_prep.h"

using namespace mtp;

namespace {

constexpr uint32_t NONE = 0xffffffffu;
constexpr double kPi = 3.14159265358979323846;
constexpr double kEpsilon = 2.220446049250313e-16;  // Number.EPSILON

// Record sizes in words (mutracer-layout.h).
constexpr uint32_t kHeaderWords = 32, kGeometryWords = 12, kMeshWords = 21, kMaterialWords = 24;
constexpr uint32_t kCameraWords = 32, kBatchWords = 4, kExtensionWords = 4;

struct Failure {
  int32_t status;
  std::string message;
};
[[noreturn]] void reject(const std::string &m) { throw Failure{MT_ERROR_INVALID_ARGUMENT, m}; }
[[noreturn]] void unsupported(const std::string &m) {
  throw Failure{MT_ERROR_UNAVAILABLE, m + " is not supported by this build"};
}

struct Words {
  const uint32_t *u;
  const float *f;
  uint64_t n;
  // A table of `count` records of `stride` words at `offset`: inside the
  // descriptor, after the header (even when empty).
  void table(const char *what, uint32_t offset, uint64_t count, uint32_t stride) const {
    if (offset < kHeaderWords || offset > n || uint64_t(offset) + count * stride > n)
      reject(std::string(what) + " table lies outside the descriptor");
  }
  // An optional array (offset 0 = absent) of `count` words.
  bool array(const char *what, uint32_t offset, uint64_t count) const {
    if (!offset) return false;
    if (offset < kHeaderWords || uint64_t(offset) + count > n) reject(std::string(what) + " lies outside the descriptor");
    return true;
  }
  float finite(uint64_t w, const char *what) const {
    float v = f[w];
    if (!std::isfinite(v)) reject(std::string(what) + " is not finite");
    return v;
  }
  void zero(uint64_t w, uint32_t count, const char *what) const {
    for (uint32_t i = 0; i < count; i++)
      if (u[w + i]) reject(std::string(what) + " reserved words must be zero");
  }
  // Column-major affine, invertible local-to-world matrix.
  void matrix(uint64_t w, const char *what, double out[16]) const {
    for (int i = 0; i < 16; i++) out[i] = finite(w + i, what);
    if (out[3] != 0 || out[7] != 0 || out[11] != 0 || out[15] != 1) reject(std::string(what) + " matrix is not affine");
    double inv[16];
    if (!invert4(out, inv)) reject(std::string(what) + " matrix is not invertible");
  }
};

std::string at(const char *what, uint32_t i) { return std::string(what) + " " + std::to_string(i); }

// ------------------------------------------------------------ camera
// mat4.multiply (out = a * b, column-major, summed in the vendored order).
void mul4(const double *a, const double *b, double *out) {
  double r[16];
  for (int c = 0; c < 4; c++) {
    double b0 = b[c * 4], b1 = b[c * 4 + 1], b2 = b[c * 4 + 2], b3 = b[c * 4 + 3];
    for (int k = 0; k < 4; k++) r[c * 4 + k] = b0 * a[k] + b1 * a[4 + k] + b2 * a[8 + k] + b3 * a[12 + k];
  }
  std::memcpy(out, r, sizeof(r));
}

void decodeCamera(const Words &d, uint32_t o, uint32_t width, uint32_t height, mtc_camera_uniform &cam) {
  const uint32_t projection = d.u[o];
  if (projection > 1) reject("camera projection must be 0 (perspective) or 1 (orthographic)");
  float v[13];
  for (int i = 1; i < 13; i++) v[i] = d.finite(o + i, "camera value");
  d.zero(o + 13, 3, "camera");
  double world[16];
  d.matrix(o + 16, "camera", world);
  const double fov = v[1], nearZ = v[2], farZ = v[3], zoom = v[8], fStop = v[9], focus = v[10];
  const double sensor = v[11], metersPerUnit = v[12];
  double proj[16] = {0};
  if (projection == 0) {
    if (!(fov > 0 && fov < 180)) reject("camera field of view must lie in (0, 180) degrees");
    if (!(nearZ > 0) || !(farZ > nearZ)) reject("camera clip planes need 0 < near < far");
    // Camera.getProjectionMatrix (perspective, zoomed field of view) and
    // mat4.perspectiveNO.
    const double effective = 2 * std::atan(std::tan(fov * kPi / 180 / 2) / std::max(zoom, kEpsilon));
    const double f = 1.0 / std::tan(effective / 2), aspect = double(width) / double(height);
    proj[0] = f / aspect;
    proj[5] = f;
    proj[11] = -1;
    const double nf = 1 / (nearZ - farZ);
    proj[10] = (farZ + nearZ) * nf;
    proj[14] = 2 * farZ * nearZ * nf;
  } else {
    const double l = v[4], r = v[5], b = v[6], t = v[7];
    if (!(zoom > 0) || l == r || b == t || nearZ == farZ) reject("orthographic camera needs a non-empty view volume");
    // Camera.getProjectionMatrix (orthographic, zoomed) and mat4.orthoNO.
    const double left = (l + r) / 2 - (r - l) / (2 * zoom), right = (l + r) / 2 + (r - l) / (2 * zoom);
    const double bottom = (b + t) / 2 - (t - b) / (2 * zoom), top = (b + t) / 2 + (t - b) / (2 * zoom);
    const double lr = 1 / (left - right), bt = 1 / (bottom - top), nf = 1 / (nearZ - farZ);
    proj[0] = -2 * lr;
    proj[5] = -2 * bt;
    proj[10] = 2 * nf;
    proj[12] = (left + right) * lr;
    proj[13] = (top + bottom) * bt;
    proj[14] = (farZ + nearZ) * nf;
    proj[15] = 1;
  }
  if (fStop < 0 || focus < 0 || sensor < 0 || metersPerUnit < 0) reject("camera lens values must be nonnegative");
  double inverse[16];
  if (!invert4(proj, inverse)) reject("camera projection is not invertible");
  mul4(world, inverse, inverse);
  for (int i = 0; i < 16; i++) {
    cam.view_projection_inv[i] = float(inverse[i]);
    cam.view_inv[i] = float(world[i]);
  }
  // cameraApertureRadius (cameraLens.ts:4-15).
  double radius = 0;
  if (fStop > 0 && metersPerUnit > 0) {
    const double focal = projection == 0 ? 0.5 * sensor * std::max(zoom, kEpsilon) / std::tan(fov * kPi / 360) : 0.0;
    radius = focal / (2 * fStop) / 1000 / metersPerUnit;
    if (!(std::isfinite(radius) && radius > 0)) radius = 0;
  }
  cam.aperture_radius = float(radius);
  cam.focus_distance = float(focus);
}

// ------------------------------------------------------------ lights
double luminance(const float c[3]) {
  return std::max(c[0] * 0.2126 + c[1] * 0.7152 + c[2] * 0.0722, 0.0);
}

// getRigidLightFrame (lightsData.ts:104-117).
void rigidFrame(const double *m, double x[3], double y[3], double dir[3]) {
  auto normalize = [](double *v, const double *fallback) {
    double len = std::hypot(v[0], v[1], v[2]);
    if (len > 1e-12) for (int i = 0; i < 3; i++) v[i] /= len;
    else for (int i = 0; i < 3; i++) v[i] = fallback[i];
  };
  const double fz[3] = {0, 0, 1}, fx[3] = {1, 0, 0};
  double z[3] = {m[8], m[9], m[10]};
  normalize(z, fz);
  const double projection = m[0] * z[0] + m[1] * z[1] + m[2] * z[2];
  x[0] = m[0] - projection * z[0]; x[1] = m[1] - projection * z[1]; x[2] = m[2] - projection * z[2];
  if (std::hypot(x[0], x[1], x[2]) <= 1e-12) {
    if (std::fabs(z[1]) < .99) { x[0] = z[2]; x[1] = 0; x[2] = -z[0]; }
    else { x[0] = 1; x[1] = 0; x[2] = 0; }
  }
  normalize(x, fx);
  y[0] = z[1] * x[2] - z[2] * x[1];
  y[1] = z[2] * x[0] - z[0] * x[2];
  y[2] = z[0] * x[1] - z[1] * x[0];
  for (int i = 0; i < 3; i++) dir[i] = -z[i] == 0 ? 0.0 : -z[i];  // `-z || 0` turns -0 into +0
}

LightDesc decodeLight(const Words &d, uint32_t o, uint32_t version, uint32_t index) {
  const uint32_t type = d.u[o];
  if (type > 5) reject(at("light", index) + " has an unknown type");
  float color[3];
  for (int c = 0; c < 3; c++) color[c] = d.finite(o + 1 + c, "light color");
  const float intensity = d.finite(o + 4, "light intensity"), size = d.finite(o + 5, "light size");
  const float heightOrInner = d.finite(o + 6, "light value"), spreadOrOuter = d.finite(o + 7, "light value");
  if (d.u[o + 8]) unsupported("a rect-light texture");
  if (d.u[o + 9] || d.u[o + 10]) {
    if (type != 3) reject(at("light", index) + ": only spot lights take an IES profile");
    unsupported("an IES light profile");
  }
  d.zero(o + 11, 1, "light");
  double m[16];
  d.matrix(o + 12, "light", m);
  float radius = 0, length = 0;
  uint32_t normalize = 0;
  if (version >= 6) {
    radius = d.finite(o + 28, "light radius");
    length = d.finite(o + 29, "light length");
    normalize = d.u[o + 30];
    if (normalize > 1 || d.u[o + 31] > 1) reject(at("light", index) + ": normalize and treat_as_line are 0 or 1");
  } else if (type == 4 || type == 5) {
    radius = size;
    if (type == 5) length = heightOrInner;
  }
  LightDesc L;
  L.packed = true;
  float *r = L.rows;
  double x[3], y[3], dir[3];
  rigidFrame(m, x, y, dir);
  r[0] = float(m[12]); r[1] = float(m[13]); r[2] = float(m[14]);
  const double lum = luminance(color) * double(intensity);
  auto areaRadiance = [&](double area) { return normalize ? intensity / std::max(area, 1e-8) : double(intensity); };
  double emissionScale = intensity, area = 0;
  switch (type) {
    case 0: {  // rect (MT_LIGHT_TYPE_RECT)
      if (!(size > 0) || !(heightOrInner > 0)) reject(at("light", index) + ": rect lights need positive width and height");
      r[3] = MTC_LIGHT_RECT;
      area = double(size) * double(heightOrInner);
      r[7] = float(area);
      for (int i = 0; i < 3; i++) { r[8 + i] = float(x[i] * size); r[12 + i] = float(y[i] * -double(heightOrInner)); }
      r[11] = spreadOrOuter;
      L.power = lum > 0 ? lum * kPi * std::max(area, 0.0) : 0.0;
      break;
    }
    case 1: {  // sphere
      if (size < 0) reject(at("light", index) + ": sphere radius must be nonnegative");
      r[3] = MTC_LIGHT_SPHERE;
      area = 4 * kPi * double(size) * size;
      r[7] = float(area);
      r[11] = size;
      L.power = !(lum > 0) ? 0.0 : size == 0 ? lum * 4 * kPi : lum * kPi * std::max(area, 0.0);
      break;
    }
    case 2:  // directional
      r[3] = MTC_LIGHT_DIRECTIONAL;
      for (int i = 0; i < 3; i++) r[8 + i] = float(dir[i]);
      L.power = lum > 0 ? lum * 4 * kPi : 0.0;
      break;
    case 3: {  // spot
      const double inner = heightOrInner, outer = spreadOrOuter;
      if (!(inner >= 0 && inner <= outer && outer > 0 && outer < 90))
        reject(at("light", index) + ": spot angles need 0 <= inner <= outer < 90 and outer > 0");
      if (size < 0) reject(at("light", index) + ": spot radius must be nonnegative");
      r[3] = MTC_LIGHT_SPOT;
      area = 4 * kPi * double(size) * size;
      emissionScale = size == 0 ? double(intensity) : intensity / (kPi * double(size) * size);
      r[7] = float(area);
      for (int i = 0; i < 3; i++) r[8 + i] = float(dir[i]);
      r[11] = size;
      const double cosOuter = std::cos(outer * kPi / 180), cosInner = std::cos(std::min(inner, outer) * kPi / 180);
      r[12] = float(cosOuter); r[13] = float(cosInner);
      const double shaping = 0.5 * (1 - 0.5 * (cosInner + cosOuter));
      L.power = !(lum > 0) ? 0.0
              : size == 0 ? lum * 4 * kPi * shaping
                          : luminance(color) * emissionScale * kPi * area * shaping;
      break;
    }
    case 4: {  // disk
      if (!(radius > 0)) reject(at("light", index) + ": disk lights need a positive radius");
      r[3] = MTC_LIGHT_DISK;
      area = kPi * double(radius) * radius;
      emissionScale = areaRadiance(area);
      r[7] = float(area);
      for (int i = 0; i < 3; i++) { r[8 + i] = float(x[i] * radius); r[12 + i] = float(y[i] * -double(radius)); }
      r[11] = radius;
      L.power = lum > 0 ? luminance(color) * emissionScale * kPi * area : 0.0;
      break;
    }
    default: {  // cylinder
      if (!(radius > 0) || !(length > 0)) reject(at("light", index) + ": cylinder lights need positive radius and length");
      r[3] = MTC_LIGHT_CYLINDER;
      area = 2 * kPi * double(radius) * length;
      emissionScale = areaRadiance(area);
      r[7] = float(area);
      for (int i = 0; i < 3; i++) { r[8 + i] = float(x[i] * length); r[12 + i] = float(y[i] * radius); }
      r[11] = radius;
      L.power = lum > 0 ? luminance(color) * emissionScale * kPi * area : 0.0;
      break;
    }
  }
  for (int c = 0; c < 3; c++) r[4 + c] = float(color[c] * emissionScale);
  r[15] = -1.0f;  // no texture / IES profile
  for (int i = 0; i < 3; i++) r[20 + i] = float(x[i]);
  return L;
}

// ------------------------------------------------------------ materials
struct DecodedMaterial {
  MaterialDesc desc;
  float emissionColor[3], emissionLuminance, coatColor[3], opacity;
  double emission[3];  // materialEmission in float64, before the f32 row store
  // Descriptor texture index per texture slot (MapSlot order), NONE for none.
  uint32_t slots[kMapSlots];
};

void setColor(float *dst, const float *src) { for (int c = 0; c < 3; c++) dst[c] = src[c]; }

DecodedMaterial decodeMaterial(const Words &d, uint32_t o, uint32_t version, uint32_t index, uint32_t textures) {
  DecodedMaterial m;
  MaterialDesc &md = m.desc;
  float v[14];
  for (int i = 0; i < 14; i++) v[i] = d.finite(o + i, "material value");
  // Value ranges (scene.rs material validation): unit-interval factors,
  // IOR >= 1, nonnegative colors and luminance.
  for (int k : {3, 4, 5, 11, 12, 13})
    if (!(v[k] >= 0.0f && v[k] <= 1.0f)) reject(at("material", index) + ": values out of range");
  for (int k : {0, 1, 2, 7, 8, 9, 10})
    if (v[k] < 0.0f) reject(at("material", index) + ": values out of range");
  if (v[6] < 1.0f) reject(at("material", index) + ": values out of range");
  setColor(md.baseColor, v);
  md.specularRoughness = v[3];
  md.baseMetalness = v[4];
  md.transmissionWeight = v[5];
  md.specularIor = v[6];
  setColor(m.emissionColor, v + 7);
  m.emissionLuminance = v[10];
  md.coatWeight = v[11];
  md.coatRoughness = v[12];
  m.opacity = v[13];
  if (d.u[o + 14] > 1) reject(at("material", index) + ": thin_walled is 0 or 1");
  md.thin = d.u[o + 14] != 0;
  for (int k = 15; k < 19; k++)
    if (d.u[o + k] != NONE && d.u[o + k] >= textures) reject(at("material", index) + ": texture reference out of range");
  std::fill(m.slots, m.slots + kMapSlots, NONE);
  m.slots[kMapBase] = d.u[o + 15];
  m.slots[kMapNormal] = d.u[o + 16];
  m.slots[kMapMetallicRoughness] = d.u[o + 17];
  m.slots[kMapEmissive] = d.u[o + 18];
  uint32_t alphaMode = 0, mapAlphaUsage = 0;
  if (d.u[o + 21]) {
    if (version < 8) reject(at("material", index) + ": graph_offset must be 0 before version 8");
    unsupported("a material graph");
  }
  d.zero(o + 22, 2, "material");
  const uint32_t count = d.u[o + 19], ext = d.u[o + 20];
  if (count) d.table("material extension", ext, count, kExtensionWords);
  uint64_t seen[2] = {0, 0};
  setColor(m.coatColor, md.coatColor);
  for (uint32_t e = 0; e < count; e++) {
    const uint64_t w = uint64_t(ext) + uint64_t(e) * kExtensionWords;
    const uint32_t id = d.u[w];
    if (id == 0 || id > 76) reject(at("material", index) + ": unknown extension id " + std::to_string(id));
    if (seen[id >> 6] >> (id & 63) & 1) reject(at("material", index) + ": extension id repeated");
    seen[id >> 6] |= uint64_t(1) << (id & 63);
    float f[3];
    for (int c = 0; c < 3; c++) f[c] = d.f[w + 1 + c];
    const uint32_t u0 = d.u[w + 1];
    auto scalar = [&](float &dst) {
      if (!std::isfinite(f[0]) || d.u[w + 2] || d.u[w + 3]) reject(at("material", index) + ": malformed float extension");
      dst = f[0];
    };
    auto color = [&](float *dst) {
      for (int c = 0; c < 3; c++)
        if (!std::isfinite(f[c])) reject(at("material", index) + ": malformed color extension");
      setColor(dst, f);
    };
    auto flag = [&](bool &dst) {
      if (u0 > 1 || d.u[w + 2] || d.u[w + 3]) reject(at("material", index) + ": malformed bool extension");
      dst = u0 != 0;
    };
    auto pair = [&](float *dst) {
      if (!std::isfinite(f[0]) || !std::isfinite(f[1]) || d.u[w + 3])
        reject(at("material", index) + ": malformed vec2 extension");
      dst[0] = f[0];
      dst[1] = f[1];
    };
    auto choice = [&](uint32_t variants) {
      if (u0 >= variants || d.u[w + 2] || d.u[w + 3]) reject(at("material", index) + ": invalid material enum");
      return u0;
    };
    auto texture = [&]() {
      if (d.u[w + 2] || d.u[w + 3]) reject(at("material", index) + ": malformed texture extension");
      if (u0 != NONE && u0 >= textures) reject(at("material", index) + ": texture reference out of range");
      return u0;
    };
    switch (id) {
      case 1: scalar(md.baseWeight); break;
      case 2: color(md.baseColor); break;
      case 3: scalar(md.diffuseRoughness); break;
      case 4: scalar(md.baseMetalness); break;
      case 5: scalar(md.specularWeight); break;
      case 6: color(md.specularColor); break;
      case 7: scalar(md.specularRoughness); break;
      case 8: scalar(md.specularIor); break;
      case 9: scalar(md.specularAnisotropy); break;
      case 10: scalar(md.transmissionWeight); break;
      case 11: color(md.transmissionColor); break;
      case 15: scalar(md.dispersionScale); break;
      case 16: scalar(md.abbe); break;
      case 17: scalar(md.subsurfaceWeight); break;
      case 18: color(md.subsurfaceColor); break;
      case 22: scalar(md.fuzzWeight); break;
      case 23: color(md.fuzzColor); break;
      case 24: scalar(md.fuzzRoughness); break;
      case 25: scalar(md.coatWeight); break;
      case 26: color(md.coatColor); setColor(m.coatColor, md.coatColor); break;
      case 27: scalar(md.coatRoughness); break;
      case 29: scalar(md.coatIor); break;
      case 30: scalar(md.coatDarkening); break;
      case 31: scalar(md.thinFilmWeight); break;
      case 32: scalar(md.thinFilmThickness); break;
      case 33: scalar(md.thinFilmIor); break;
      case 34: color(m.emissionColor); break;
      case 35: scalar(m.emissionLuminance); break;
      case 36: scalar(m.opacity); break;
      case 37: flag(md.thin); break;
      case 38: flag(md.doubleSided); break;
      // Texture slots (material-properties.ts ids 39-74).
      case 39: m.slots[kMapBase] = texture(); break;
      case 40: m.slots[kMapAlpha] = texture(); break;
      case 43: m.slots[kMapEmissive] = texture(); break;
      case 44: m.slots[kMapNormal] = texture(); break;
      case 46: m.slots[kMapMetallicRoughness] = texture(); break;
      case 47: m.slots[kMapRoughness] = texture(); break;
      case 48: m.slots[kMapMetalness] = texture(); break;
      case 49: m.slots[kMapTransmission] = texture(); break;
      case 50: m.slots[kMapThinFilm] = texture(); break;
      case 59: m.slots[kMapDisplacement] = texture(); break;
      case 64: m.slots[kMapCoatWeight] = texture(); break;
      case 65: m.slots[kMapCoatRoughness] = texture(); break;
      case 66: m.slots[kMapFuzzColor] = texture(); break;
      case 67: m.slots[kMapFuzzRoughness] = texture(); break;
      case 68: m.slots[kMapSpecularWeight] = texture(); break;
      case 69: m.slots[kMapSpecularColor] = texture(); break;
      case 70: m.slots[kMapAnisotropy] = texture(); break;
      case 74: m.slots[kMapCoatNormal] = texture(); break;
      case 62: scalar(md.thinFilmThicknessMinimum); break;
      case 63: md.thinFilmMapChannel = int(choice(4)); break;
      case 41: alphaMode = choice(4); break;  // auto, opaque, mask, blend
      case 42: scalar(md.alphaCutoff); break;
      case 45: pair(md.normalScale); break;
      case 54: mapAlphaUsage = choice(3); break;  // opaque, alpha, transmission
      case 55: md.uvProjection = int(choice(4)); break;  // none, spherical, cylindrical, triplanar
      case 56: pair(md.uvScale); break;  // uvProjectionScale scales the UVs of every map
      case 51: case 52: {
        bool on = false;
        flag(on);
        if (on) unsupported(id == 51 ? "a shadow-catcher material" : "an unlit material");
        break;
      }
      default: unsupported("material extension " + std::to_string(id));
    }
  }
  if (m.slots[kMapDisplacement] != NONE) unsupported("displacement maps");
  if (m.slots[kMapAnisotropy] != NONE) unsupported("anisotropy maps");
  if (m.slots[kMapCoatNormal] != NONE) unsupported("coat normal maps");
  // resolveMaterialAlphaMode (MaterialState.ts:251-264) to
  // materialAlphaModeConstants: explicit modes stay; auto masks with a
  // positive cutoff, blends with partial opacity, the base color's alpha as
  // opacity or an alpha map, and is opaque otherwise.
  md.opacity = m.opacity;
  if (alphaMode == 1) md.alphaMode = 0;
  else if (alphaMode == 2) md.alphaMode = 1;
  else if (alphaMode == 3) md.alphaMode = 2;
  else if (md.alphaCutoff > 0) md.alphaMode = 1;
  else if (m.opacity < 1 || mapAlphaUsage == 1 || m.slots[kMapAlpha] != NONE) md.alphaMode = 2;
  else md.alphaMode = 0;
  md.mapAlphaUsage = mapAlphaUsage == 1 ? 2 : mapAlphaUsage == 2 ? 3 : 0;  // mapAlphaUsageConstants
  // materialEmission (materialEmission.ts:10-22): emission crosses the coat
  // once; with a coat weight map the shader applies that passage instead.
  for (int c = 0; c < 3; c++) {
    double e = double(m.emissionColor[c]) * m.emissionLuminance;
    if (md.coatWeight > 0 && m.slots[kMapCoatWeight] == NONE) {
      const double w = std::min(double(md.coatWeight), 1.0);
      e = e * (1 + w * (std::sqrt(std::max(double(m.coatColor[c]), 0.0)) - 1));
    }
    m.emission[c] = e;
    md.emission[c] = float(e);
  }
  return m;
}

// accumulateVertexNormals (src/util/vertexNormals.ts:9-52): area-weighted face
// normals summed per vertex in f32 storage, then normalised.
std::vector<float> generateNormals(const std::vector<float> &p, const std::vector<uint32_t> &idx, uint32_t count) {
  std::vector<float> n(size_t(count) * 3, 0.0f);
  for (size_t f = 0; f + 2 < idx.size(); f += 3) {
    const uint32_t i1 = idx[f], i2 = idx[f + 1], i3 = idx[f + 2];
    float a[3], b[3], c[3], v21[3], v32[3], x[3];
    for (int k = 0; k < 3; k++) { a[k] = p[size_t(i1) * 3 + k]; b[k] = p[size_t(i2) * 3 + k]; c[k] = p[size_t(i3) * 3 + k]; }
    for (int k = 0; k < 3; k++) { v21[k] = float(double(a[k]) - b[k]); v32[k] = float(double(b[k]) - c[k]); }
    x[0] = float(double(v21[1]) * v32[2] - double(v21[2]) * v32[1]);
    x[1] = float(double(v21[2]) * v32[0] - double(v21[0]) * v32[2]);
    x[2] = float(double(v21[0]) * v32[1] - double(v21[1]) * v32[0]);
    for (uint32_t v : {i1, i2, i3})
      for (int k = 0; k < 3; k++) n[size_t(v) * 3 + k] = float(double(n[size_t(v) * 3 + k]) + x[k]);
  }
  for (size_t i = 0; i < n.size(); i += 3) {
    const double x = n[i], y = n[i + 1], z = n[i + 2];
    double len = x * x + y * y + z * z;
    if (len > 0) len = 1 / std::sqrt(len);
    n[i] = float(x * len); n[i + 1] = float(y * len); n[i + 2] = float(z * len);
  }
  return n;
}

// collectEmissiveTriangles (lightSampling.ts:237-321) for one instance: world
// corners through vec3.transformMat4 (f32 results), area 0.5 |e0 x e1| from
// f32 edges and cross product, triangles below 1e-10 area skipped.
// ------------------------------------------------------------ textures
constexpr uint64_t kTextureBudgetBytes = 3ull << 30;  // scene-configuration.ts:8 textureBudgetBytes

struct TextureRecord {
  uint32_t width, height, storage, pixels, flipY, uvChannel, wrapS, wrapT, udim;
  float transform[4];  // uv scale xy, uv offset xy
  std::tuple<uint32_t, uint32_t, uint32_t, uint32_t, uint32_t> source() const {
    return {pixels, width, height, storage, flipY};
  }
};

// float16Bits (float16.ts:1-16): nearest, ties to even, as RGBA16F storage
// holds the value; returned widened to f32.
float halfStored(double value) {
  auto roundEven = [](double v) {
    const double integer = std::floor(v), fraction = v - integer;
    return integer + ((fraction > 0.5 || (fraction == 0.5 && std::fmod(integer, 2.0) == 1.0)) ? 1.0 : 0.0);
  };
  const bool negative = value < 0 || (value == 0 && std::signbit(value));
  const double absolute = std::fabs(value);
  uint32_t bits;
  if (std::isnan(absolute)) bits = 0x7e00;
  else if (absolute >= 65520) bits = 0x7c00;
  else if (absolute < std::ldexp(1.0, -14)) bits = uint32_t(roundEven(absolute * std::ldexp(1.0, 24)));
  else {
    const int exponent = int(std::floor(std::log2(absolute)));
    bits = uint32_t((exponent + 14) * 1024 + roundEven(absolute / std::ldexp(1.0, exponent - 10)));
  }
  const int e = int(bits >> 10) & 31, mantissa = int(bits & 1023);
  float f;
  if (e == 31) f = mantissa ? NAN : INFINITY;
  else if (e == 0) f = float(std::ldexp(double(mantissa), -24));
  else f = float(std::ldexp(double(1024 + mantissa), e - 25));
  return negative ? -f : f;
}

// planTextureAtlas at full size (textureAtlas.ts:196-248 with packTextureAtlas
// :65-130): true when the shelf packing of the distinct pixel sources fits the
// atlas's page budget without scaling.
bool atlasKeepsFullSize(const std::vector<TextureRecord> &sources, uint32_t bytesPerPixel) {
  const double budget = double(kTextureBudgetBytes);
  uint32_t maxDimension = 1;
  for (const TextureRecord &t : sources) maxDimension = std::max({maxDimension, t.width, t.height});
  const double fromBudget = std::max(1.0, std::floor(std::sqrt(budget / bytesPerPixel)));
  const uint64_t pageSize = uint64_t(std::max(1.0, std::floor(std::min({double(maxDimension), 16384.0, fromBudget}))));
  const double pageBytes = double(pageSize) * double(pageSize) * bytesPerPixel;
  const size_t maxPages = size_t(std::max(1.0, std::min(256.0, std::floor(budget / pageBytes))));
  if (pageSize < maxDimension) return false;
  std::vector<size_t> order(sources.size());
  for (size_t i = 0; i < order.size(); i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
    return sources[a].height != sources[b].height ? sources[a].height > sources[b].height
                                                   : sources[a].width > sources[b].width;
  });
  struct Shelf { uint64_t height, x; };
  struct Page { uint64_t nextY; std::vector<Shelf> shelves; };
  std::vector<Page> pages;
  for (size_t i : order) {
    const uint64_t w = sources[i].width, h = sources[i].height;
    bool placed = false;
    for (size_t layer = 0; layer < pages.size() && !placed; layer++) {
      Page &page = pages[layer];
      for (Shelf &shelf : page.shelves)
        if (h <= shelf.height && shelf.x + w <= pageSize) {
          shelf.x += w;
          placed = true;
          break;
        }
      if (!placed && page.nextY + h <= pageSize) {
        page.shelves.push_back({h, w});
        page.nextY += h;
        placed = true;
      }
    }
    if (!placed) pages.push_back({h, {{h, w}}});
  }
  return pages.size() <= maxPages;
}

// The map table of `maps` (descriptor texture indices in MaterialData order):
// one record of MTC_MAP_VEC4_ROWS vec4 per map and the texels of each
// distinct pixel source (writeRawAtlasPlacement at unit scale).
void packMaterialMaps(const Words &d, const std::vector<TextureRecord> &records, const std::vector<uint32_t> &maps,
                      SceneHost &s) {
  bool floatStorage = false;
  std::vector<TextureRecord> sources;
  std::set<std::tuple<uint32_t, uint32_t, uint32_t, uint32_t, uint32_t>> seen;
  for (uint32_t t : maps) {
    const TextureRecord &r = records[t];
    if (r.udim) unsupported("UDIM texture sets");
    floatStorage |= r.storage == 1;
    if (seen.insert(r.source()).second) sources.push_back(r);
  }
  if (!atlasKeepsFullSize(sources, floatStorage ? 8 : 4)) unsupported("material textures that the atlas would downscale");
  std::map<std::tuple<uint32_t, uint32_t, uint32_t, uint32_t, uint32_t>, uint32_t> firstTexel;
  s.maps.assign(maps.size() * MTC_MAP_VEC4_ROWS * 4, 0.0f);
  for (size_t i = 0; i < maps.size(); i++) {
    const TextureRecord &r = records[maps[i]];
    auto found = firstTexel.find(r.source());
    uint32_t first;
    if (found != firstTexel.end()) {
      first = found->second;
    } else {
      first = uint32_t(s.mapTexels.size() / 4);
      firstTexel[r.source()] = first;
      s.mapTexels.resize(s.mapTexels.size() + size_t(r.width) * r.height * 4);
      float *out = &s.mapTexels[size_t(first) * 4];
      for (uint32_t y = 0; y < r.height; y++) {
        const uint32_t sy = r.flipY ? r.height - 1 - y : y;
        for (uint32_t x = 0; x < r.width; x++) {
          const uint64_t texel = uint64_t(sy) * r.width + x;
          for (int c = 0; c < 4; c++) {
            float v;
            if (r.storage == 0) {
              const uint32_t byte = (d.u[r.pixels + texel] >> (8 * c)) & 255u;
              v = floatStorage ? halfStored(double(byte) / 255.0) : float(byte) / 255.0f;
            } else {
              v = halfStored(double(d.f[r.pixels + texel * 4 + c]));
            }
            *out++ = v;
          }
        }
      }
    }
    float *row = &s.maps[i * MTC_MAP_VEC4_ROWS * 4];
    uint32_t head[3] = {r.width, r.height, first};
    std::memcpy(row, head, sizeof(head));
    for (int k = 0; k < 4; k++) row[4 + k] = r.transform[k];
    // uv channel, color linear (float sources), wrap S, wrap T (0 repeat, 1 clamp, 2 mirror)
    row[8] = float(r.uvChannel);
    row[9] = r.storage == 1 ? 1.0f : 0.0f;
    row[10] = float(r.wrapS);
    row[11] = float(r.wrapT);
  }
}

// collectEmissiveTriangles (lightSampling.ts:240-320) for one instance:
// each triangle with an emitting material (its per-vertex material, else the
// instance's) in world space.
void collectEmissive(const MeshData &md, const double *m, uint32_t instanceMaterial,
                     const std::vector<double> &samplingLuminance, SceneHost &s) {
  for (size_t t = 0; t + 2 < md.indices.size(); t += 3) {
    const uint32_t material =
        md.vertexMaterials.empty() ? instanceMaterial : uint32_t(md.vertexMaterials[md.indices[t]]);
    const double luminanceValue = samplingLuminance[material];
    if (!(luminanceValue > 1e-8)) continue;
    EmissiveTriangle tri;
    for (int c = 0; c < 3; c++) {
      const float *p = &md.positions[size_t(md.indices[t + c]) * 3];
      const double x = p[0], y = p[1], z = p[2];
      double w = m[3] * x + m[7] * y + m[11] * z + m[15];
      if (w == 0) w = 1.0;
      tri.p[c * 3] = float((m[0] * x + m[4] * y + m[8] * z + m[12]) / w);
      tri.p[c * 3 + 1] = float((m[1] * x + m[5] * y + m[9] * z + m[13]) / w);
      tri.p[c * 3 + 2] = float((m[2] * x + m[6] * y + m[10] * z + m[14]) / w);
    }
    float e0[3], e1[3], cr[3];
    for (int k = 0; k < 3; k++) {
      e0[k] = float(double(tri.p[3 + k]) - tri.p[k]);
      e1[k] = float(double(tri.p[6 + k]) - tri.p[k]);
    }
    cr[0] = float(double(e0[1]) * e1[2] - double(e0[2]) * e1[1]);
    cr[1] = float(double(e0[2]) * e1[0] - double(e0[0]) * e1[2]);
    cr[2] = float(double(e0[0]) * e1[1] - double(e0[1]) * e1[0]);
    const double area = 0.5 * std::sqrt(double(cr[0]) * cr[0] + double(cr[1]) * cr[1] + double(cr[2]) * cr[2]);
    if (!(area > 1e-10) || !std::isfinite(area)) continue;
    // collectEmissiveTriangles: uv, and uv1 ?? uv (lightSampling.ts:264, 290-299)
    const std::vector<float> &second = md.uv1s.empty() ? md.uvs : md.uv1s;
    for (int c = 0; c < 3; c++) {
      const size_t v = md.indices[t + c];
      if (!md.uvs.empty()) {
        tri.uv[c * 2] = md.uvs[v * 2];
        tri.uv[c * 2 + 1] = md.uvs[v * 2 + 1];
      }
      if (!second.empty()) {
        tri.uv1[c * 2] = second[v * 2];
        tri.uv1[c * 2 + 1] = second[v * 2 + 1];
      }
    }
    tri.area = area;
    tri.luminance = luminanceValue;
    tri.material = int32_t(material);
    s.emissive.push_back(tri);
  }
}

void decodeScene(const Words &d, SceneHost &s) {
  const uint32_t *u = d.u;
  const uint32_t version = u[0];
  if (version < 5 || version > 8) reject("unsupported scene version " + std::to_string(version) + " (5 to 8)");
  if (u[1] != d.n) reject("total_words does not match the descriptor length");
  const uint32_t width = u[2], height = u[3];
  if (width < 1 || width > 8192 || height < 1 || height > 8192 || uint64_t(width) * height > 16777216u)
    reject("output size must be 1..8192 per edge and at most 16777216 pixels");
  const uint32_t geometries = u[4], meshes = u[5], materials = u[6], lights = u[7], textures = u[8];
  if (!geometries || !meshes || !materials) reject("a scene needs at least one geometry, mesh and material");
  if (geometries > 65536 || materials > 65536 || textures > 65536) reject("more than 65536 geometries, materials or textures");
  if (lights > 1024) reject("more than 1024 analytic lights");
  if (meshes > 16777216u) reject("more than 16777216 meshes");
  const uint32_t lightWords = version < 6 ? 28 : 32, textureWords = version < 7 ? 12 : 13;
  d.table("geometry", u[9], geometries, kGeometryWords);
  d.table("mesh", u[10], meshes, kMeshWords);
  d.table("material", u[11], materials, kMaterialWords);
  d.table("light", u[12], lights, lightWords);
  d.table("texture", u[13], textures, textureWords);
  d.table("camera", u[14], 1, kCameraWords);
  d.zero(15, 1, "header");
  d.zero(28, 4, "header");
  float background[4];
  for (int c = 0; c < 4; c++) background[c] = d.finite(16 + c, "background color");
  const uint32_t envPlusOne = u[20], bgPlusOne = u[21], quality = u[22];
  if (envPlusOne > textures || bgPlusOne > textures) reject("environment or background texture index out of range");
  if (quality & ~7u) reject("quality_flags accepts only the MT_QUALITY_* bits");
  if ((quality & 4) && bgPlusOne) reject("MT_QUALITY_HIDE_BACKGROUND cannot be combined with a background map");
  if (bgPlusOne) unsupported("a background map");
  if (quality & 1) unsupported("bevel");
  if (u[23]) d.table("batch", u[23], meshes, kBatchWords);
  for (int k : {24, 25}) {
    const uint32_t count = k == 24 ? meshes : materials;
    if (!d.array("AOV id table", u[k], count)) continue;
    std::vector<uint32_t> ids(u + u[k], u + u[k] + count);
    std::sort(ids.begin(), ids.end());
    for (size_t i = 0; i < ids.size(); i++)
      if (ids[i] == NONE || (i && ids[i] == ids[i - 1])) reject("AOV ids must be unique and not UINT32_MAX");
  }
  float envSettings[4] = {1, 0, 1, 0};
  if (d.array("environment settings", u[26], 4)) {
    for (int i = 0; i < 4; i++) envSettings[i] = d.finite(u[26] + i, "environment setting");
    if (envSettings[0] < 0 || envSettings[2] < 0) reject("environment intensities must be nonnegative");
  }
  if (d.array("grounded background", u[27], 6)) {
    float g[6];
    for (int i = 0; i < 6; i++) g[i] = d.finite(u[27] + i, "grounded background value");
    if (!(g[0] > 0) || !(g[1] > g[0]) || g[5] != 0) reject("grounded background needs height > 0 and radius > height");
    unsupported("a grounded background projection");
  }

  // Texture records (the reference validator's raw-texture rules).
  std::vector<TextureRecord> textureRecords(textures);
  {
    std::set<std::tuple<uint32_t, uint32_t, uint32_t, uint32_t, uint32_t>> spans;
    uint64_t pixels = 0;
    for (uint32_t i = 0; i < textures; i++) {
      const uint32_t o = u[13] + i * textureWords;
      TextureRecord &t = textureRecords[i];
      t = {u[o], u[o + 1], u[o + 2], u[o + 3], u[o + 4], u[o + 5], u[o + 10], u[o + 11], version >= 7 ? u[o + 12] : 0u,
           {0, 0, 0, 0}};
      if (t.width == 0 || t.height == 0 || t.width > 16384 || t.height > 16384 || t.storage > 1 || t.flipY > 1 ||
          t.uvChannel > 1 || t.wrapS > 2 || t.wrapT > 2 || t.udim > 1 || (t.udim && (t.width % 10 || t.height % 10)))
        reject(at("texture", i) + ": invalid raw texture record");
      if (spans.insert(t.source()).second) pixels += uint64_t(t.width) * t.height;
      if (pixels > kTextureBudgetBytes / 4 + 4194304u) reject("textures exceed the material plus environment input budget");
      const uint64_t count = uint64_t(t.width) * t.height * (t.storage ? 4 : 1);
      if (!d.array("texture pixels", t.pixels, count)) reject(at("texture", i) + " has no pixels");
      if (t.storage)
        for (uint64_t k = 0; k < count; k++) d.finite(t.pixels + k, "texture pixel");
      for (int k = 0; k < 4; k++) t.transform[k] = d.finite(o + 6 + k, "texture UV transform");
    }
  }

  s.width = width;
  s.height = height;
  // The environment map (linear RGBA32F).
  if (envPlusOne) {
    const uint32_t o = u[13] + (envPlusOne - 1) * textureWords;
    const uint32_t w = u[o], h = u[o + 1];
    if (u[o + 2] != 1) reject("environment maps must be linear RGBA32F textures");
    if (w < 1 || h < 1 || w > 16384 || h > 16384) reject("environment texture size out of range");
    if (!d.array("environment pixels", u[o + 3], uint64_t(w) * h * 4) ) reject("environment texture has no pixels");
    s.env.width = w;
    s.env.height = h;
    s.env.image.resize(size_t(w) * h * 4);
    const double intensity = envSettings[0];
    for (size_t i = 0; i < s.env.image.size(); i++) {
      float v = d.finite(u[o + 3] + i, "environment pixel");
      // scaleEnvironment (scene-core.ts:1696-1701): RGB times the lighting intensity.
      s.env.image[i] = (i % 4 == 3 || intensity == 1) ? v : float(double(v) * intensity);
    }
    buildEnvDistribution(s.env);
  }
  // Materials.
  std::vector<MaterialDesc> mats(materials);
  std::vector<double> samplingLuminance(materials);
  std::vector<DecodedMaterial> decodedMaterials;
  for (uint32_t i = 0; i < materials; i++) {
    DecodedMaterial m = decodeMaterial(d, u[11] + i * kMaterialWords, version, i, textures);
    mats[i] = m.desc;
    decodedMaterials.push_back(m);
    // colorLuminance(materialEmission(material)) (lightSampling.ts:255-256).
    samplingLuminance[i] = std::max(m.emission[0] * 0.2126 + m.emission[1] * 0.7152 + m.emission[2] * 0.0722, 0.0);
  }
  // Geometries.
  std::vector<MeshData> meshData(geometries);
  std::vector<std::vector<uint32_t>> vertexMaterial(geometries);
  bool tangentFrames = false;
  for (uint32_t g = 0; g < geometries; g++) {
    const uint32_t o = u[9] + g * kGeometryWords;
    const uint32_t vc = u[o], ic = u[o + 1];
    if (vc > 4000000u || ic > 12000000u) reject(at("geometry", g) + " exceeds 4000000 vertices or 12000000 indices");
    if (ic % 3) reject(at("geometry", g) + ": index count is not a multiple of 3");
    if (!d.array("positions", u[o + 2], uint64_t(vc) * 3) && vc) reject(at("geometry", g) + " has no positions");
    if (!d.array("indices", u[o + 3], ic) && ic) reject(at("geometry", g) + " has no indices");
    d.zero(o + 10, 2, "geometry");
    MeshData &md = meshData[g];
    md.positions.resize(size_t(vc) * 3);
    for (size_t i = 0; i < md.positions.size(); i++) md.positions[i] = d.finite(u[o + 2] + i, "position");
    md.indices.assign(u + u[o + 3], u + u[o + 3] + ic);
    for (uint32_t i : md.indices)
      if (i >= vc) reject(at("geometry", g) + ": index past the vertex array");
    if (d.array("normals", u[o + 4], uint64_t(vc) * 3)) {
      md.normals.resize(size_t(vc) * 3);
      for (size_t i = 0; i < md.normals.size(); i++) md.normals[i] = d.finite(u[o + 4] + i, "normal");
    } else {
      md.normals = generateNormals(md.positions, md.indices, vc);
    }
    if (d.array("uvs", u[o + 5], uint64_t(vc) * 2)) {
      md.uvs.assign(d.f + u[o + 5], d.f + u[o + 5] + size_t(vc) * 2);
      tangentFrames = true;  // decodeGeometry generates tangents from UVs
    }
    if (d.array("uv1s", u[o + 6], uint64_t(vc) * 2)) md.uv1s.assign(d.f + u[o + 6], d.f + u[o + 6] + size_t(vc) * 2);
    if (d.array("vertex colors", u[o + 7], uint64_t(vc) * 3)) md.colors.assign(d.f + u[o + 7], d.f + u[o + 7] + size_t(vc) * 3);
    tangentFrames |= d.array("tangents", u[o + 8], uint64_t(vc) * 4);
    if (d.array("material indices", u[o + 9], vc)) {
      vertexMaterial[g].assign(u + u[o + 9], u + u[o + 9] + vc);
      const std::vector<uint32_t> &vm = vertexMaterial[g];
      for (size_t t = 0; t + 2 < md.indices.size(); t += 3)
        if (vm[md.indices[t]] != vm[md.indices[t + 1]] || vm[md.indices[t]] != vm[md.indices[t + 2]])
          reject(at("geometry", g) + ": all three vertices of a triangle must select the same material");
    }
  }
  // Meshes and batches -> instances.
  std::vector<Instance> instances;
  std::vector<MeshData> blasMeshes = meshData;  // one BLAS per geometry, plus per-table variants
  std::map<std::pair<uint32_t, std::vector<int32_t>>, uint32_t> blasOf;
  for (uint32_t i = 0; i < meshes; i++) {
    const uint32_t o = u[10] + i * kMeshWords;
    const uint32_t g = u[o], flags = u[o + 20];
    if (g >= geometries) reject(at("mesh", i) + ": geometry index out of range");
    if (flags & ~1u) reject(at("mesh", i) + ": only flag bit 0 (hidden) is defined");
    double world[16];
    d.matrix(o + 4, "mesh", world);
    // decodeMeshMaterials: the table, else material_index.  The instance
    // record carries the first (materialsIndices[0], bvhAccel.ts:344);
    // per-vertex material indices select table entries per triangle through
    // the triangle material plane.  A geometry used with different tables
    // gets one BLAS per table (scenePreparation.ts:246-255).
    const uint32_t tableCount = u[o + 3];
    std::vector<uint32_t> table;
    if (tableCount) {
      if (!d.array("material table", u[o + 2], tableCount)) reject(at("mesh", i) + ": material table missing");
      table.assign(u + u[o + 2], u + u[o + 2] + tableCount);
      for (uint32_t k : table)
        if (k >= materials) reject(at("mesh", i) + ": material table entry out of range");
    } else {
      table.push_back(u[o + 1]);
      if (table[0] >= materials) reject(at("mesh", i) + ": material index out of range");
    }
    const uint32_t material = table[0];
    uint32_t blas = g;
    std::vector<uint32_t> usedMaterials;
    const std::vector<uint32_t> &vm = vertexMaterial[g];
    if (vm.empty()) {
      usedMaterials.push_back(material);
    } else {
      // localMaterialIndex (materialIndices.ts:5-15): an index past the
      // mesh's materials falls back to its first (a table rejects it above).
      std::vector<int32_t> global(vm.size());
      for (size_t v = 0; v < vm.size(); v++) {
        if (tableCount && vm[v] >= tableCount)
          reject(at("mesh", i) + ": per-vertex material index past its material table");
        global[v] = int32_t(table[vm[v] < table.size() ? vm[v] : 0]);
      }
      for (size_t t = 0; t < meshData[g].indices.size(); t += 3)
        usedMaterials.push_back(uint32_t(global[meshData[g].indices[t]]));
      auto key = std::make_pair(g, global);
      auto found = blasOf.find(key);
      if (found != blasOf.end()) {
        blas = found->second;
      } else {
        if (!blasMeshes[g].vertexMaterials.empty()) {  // another table: its own BLAS
          blas = uint32_t(blasMeshes.size());
          blasMeshes.push_back(meshData[g]);
        }
        blasMeshes[blas].vertexMaterials = global;
        blasOf.emplace(std::move(key), blas);
      }
    }
    if (flags & 1) continue;                        // hidden mesh or batch
    // Vertex tangents orient anisotropic lobes (openpbr_make_basis); this
    // build shades them in the normal's own frame.
    for (uint32_t um : usedMaterials)
      if (tangentFrames && mats[um].specularAnisotropy > 0)
        unsupported("anisotropic materials in a scene with vertex tangents or UVs");
    if (meshData[g].indices.empty()) continue;      // nothing to intersect
    auto push = [&](const double *m, const float *color) {
      Instance ins;
      ins.blasIndex = blas;
      std::memcpy(ins.transform, m, sizeof(ins.transform));
      ins.material = int32_t(255 + (material << 8));
      if (color) setColor(ins.color, color);
      instances.push_back(ins);
      collectEmissive(blasMeshes[blas], m, material, samplingLuminance, s);
    };
    if (!u[23]) {
      push(world, nullptr);
      continue;
    }
    const uint32_t bo = u[23] + i * kBatchWords, count = u[bo];
    d.zero(bo + 3, 1, "batch");
    if (count == NONE || count == 0) {
      if (u[bo + 1] || u[bo + 2]) reject(at("mesh", i) + ": an ordinary or empty batch has no arrays");
      if (count == NONE) push(world, nullptr);
      continue;
    }
    if (uint64_t(count) + instances.size() > 16777216u) reject("more than 16777216 instances");
    if (!d.array("batch transforms", u[bo + 1], uint64_t(count) * 16)) reject(at("mesh", i) + ": batch transforms missing");
    const bool colors = d.array("batch colors", u[bo + 2], uint64_t(count) * 3);
    for (uint32_t k = 0; k < count; k++) {
      double local[16], composed[16];
      d.matrix(u[bo + 1] + uint64_t(k) * 16, "batch instance", local);
      mul4(world, local, composed);  // the mesh world matrix outside each local matrix (float64)
      float c[3] = {1, 1, 1};
      if (colors)
        for (int j = 0; j < 3; j++) c[j] = d.finite(u[bo + 2] + uint64_t(k) * 3 + j, "batch color");
      push(composed, c);
    }
  }
  // Material maps: MaterialData's texture list (mergeTexturesFromMaterials
  // over MATERIAL_TEXTURE_NAMES slot by slot, each over the materials in
  // order, one entry per texture).
  std::vector<uint32_t> mapTextures;
  std::vector<int32_t> mapOf(textures, -1);
  for (int slot = 0; slot < kMapSlots; slot++)
    for (uint32_t i = 0; i < materials; i++) {
      const uint32_t t = decodedMaterials[i].slots[slot];
      int32_t index = -1;
      if (t != NONE) {
        if (mapOf[t] < 0) {
          mapOf[t] = int32_t(mapTextures.size());
          mapTextures.push_back(t);
        }
        index = mapOf[t];
      }
      mats[i].maps[slot] = index;
    }
  if (mapTextures.empty()) {
    for (MeshData &md : blasMeshes) {  // nothing samples them
      md.uvs.clear();
      md.uv1s.clear();
    }
  } else {
    packMaterialMaps(d, textureRecords, mapTextures, s);
  }
  // Lights.
  std::vector<LightDesc> lightList;
  for (uint32_t i = 0; i < lights; i++) lightList.push_back(decodeLight(d, u[12] + i * lightWords, version, i));
  assembleScene(s, blasMeshes, instances, mats, lightList, 8, 8, false);
  if ((s.flags & MTC_SCENE_SPECTRAL) && (s.flags & MTC_SCENE_HAS_ALPHA))
    unsupported("alpha coverage in a dispersive (spectral) scene");
  decodeCamera(d, u[14], width, height, s.camera);
  defaultUniform(s, 6, 2, 12345, 0);
  mtc_trace_uniform &tu = s.uniform;
  tu.bevel = 0;
  tu.dispersion_wavelengths = (quality & 2) ? 3 : 1;
  // writeEnvironmentSettings (scene-core.ts:1707-1711).
  const double c = std::cos(envSettings[1]), sn = std::sin(envSettings[1]);
  const double rot[16] = {c, 0, sn == 0 ? 0 : -sn, 0, 0, 1, 0, 0, sn, 0, c, 0, 0, 0, 0, 1};
  for (int i = 0; i < 16; i++) tu.environment_rotation[i] = float(rot[i]);
  tu.background_map_transform[0] = float(std::cos(envSettings[3]));
  tu.background_map_transform[1] = float(std::sin(envSettings[3]));
  tu.background_map_transform[2] = envSettings[2];
  tu.background_map_transform[3] = 0;
  // composeScene (scene-core.ts:710-712): background color unless hidden.
  tu.background_flags = (quality & 4) ? 0 : MTC_BACKGROUND_COLOR;
  for (int k = 0; k < 4; k++) tu.background_color[k] = (quality & 4) ? 0.0f : background[k];
  s.name = "descriptor";
}

}  // namespace

namespace mtp {

// Decodes a v8 descriptor into `s`; on failure returns the status and sets
// `message`.
int32_t decodeSceneDescriptor(const uint8_t *bytes, size_t length, SceneHost &s, std::string &message) {
  if (!bytes || length % 4 || length < size_t(kHeaderWords) * 4 || length / 4 > 0xffffffffull) {
    message = "a descriptor is a whole number of 32-bit words, at least the 32-word header";
    return MT_ERROR_INVALID_ARGUMENT;
  }
  // Copy into aligned storage: the caller's bytes need not be 4-byte aligned.
  std::vector<uint32_t> words(length / 4);
  std::memcpy(words.data(), bytes, length);
  Words d{words.data(), reinterpret_cast<const float *>(words.data()), words.size()};
  try {
    decodeScene(d, s);
  } catch (const Failure &f) {
    message = f.message;
    return f.status;
  } catch (const std::exception &e) {
    message = std::string("descriptor rejected: ") + e.what();
    return MT_ERROR_INVALID_ARGUMENT;
  }
  return MT_OK;
}

}  // namespace mtp

extern "C" void *mtp_descriptor_decode(const uint8_t *bytes, size_t length, int32_t *status, char *error,
                                       size_t capacity) {
  SceneHost *s = new SceneHost();
  std::string message;
  int32_t st = decodeSceneDescriptor(bytes, length, *s, message);
  if (status) *status = st;
  if (error && capacity) {
    size_t n = std::min(capacity - 1, message.size());
    std::memcpy(error, message.data(), n);
    error[n] = 0;
  }
  if (st != MT_OK) {
    delete s;
    return nullptr;
  }
  return s;
}
