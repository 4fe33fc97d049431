// OpenPBR 1.1 layered BSDF on the device: the lobes, energy compensation,
// thin film, prepare/eval/sample of src/renderer/wgsl/chunks/openPbrBsdf.wgsl.ts
// (hasAnisotropyDirections=true, hasCoatNormals=false) and the distribution
// helpers of src/renderer/wgsl/chunks/sampling.wgsl.ts.
#pragma once
#include "dev_math.cuh"

namespace mt {

// OpenPbrResolvedMaterial, rayTraceCore.wgsl.ts:118-190.
struct Material {
  V3 baseColor; float transmissionWeight;
  V3 emission; float specularAnisotropy;
  float baseMetalness, specularIor, specularRoughness;
  float transmissionDispersionScale, dispersionAbbeNumber, thinFilmThickness, thinFilmIor, thinFilmWeight;
  int32_t mediumType; V3 mediumExtinction, mediumScattering; float mediumAnisotropy;
  float baseWeight, diffuseRoughness, specularWeight; V3 specularColor;
  float subsurfaceWeight; V3 subsurfaceColor, transmissionColor;
  float fuzzWeight; V3 fuzzColor; float fuzzRoughness;
  float coatWeight; V3 coatColor; float coatRoughness, coatAnisotropy;
  V2 anisotropyDirection; bool anisotropyDirectionEnabled; float coatAnisotropyRotation;
  V3 directionTangent, directionBitangent, geometryTangent, geometryBitangent;
  float coatIor, coatDarkening;
  float alpha; int32_t alphaMode; int32_t materialType; float bevel;
  float relativeIor; bool inside; float alphaX, alphaY; bool thinWalled;
};

struct Basis { V3 tangent, bitangent, normal; };

enum { LOBE_FUZZ = 0, LOBE_COAT = 1, LOBE_METAL = 2, LOBE_SPECULAR = 3,
       LOBE_TRANSMISSION = 4, LOBE_DIFFUSE = 5, LOBE_SUBSURFACE = 6, LOBE_COUNT = 7 };

// OpenPbrPreparedBsdf, openPbrBsdf.wgsl.ts:45-75.
struct Prepared {
  // The resolved material by reference (the WGSL copies it into the prepared
  // struct; on the GPU that copy only costs registers) plus the one field
  // prepare() overrides.
  const Material *mat;
  float relativeIor;
  Basis basis, coatBasis;
  bool directionFrames;
  V3 viewLocal, diffuseColor;
  float specularEtaTOverEtaI, refractionEtaTOverEtaI, transmissionReflectionIor,
        thinFilmExteriorIor, thinFilmBaseIor, specularAlpha, diffuseSpecularEnergyCompensation;
  V3 coatBaseScale, metalMsScale;
  float metalMsFactor, metalMsProbability;
  V3 dielectricMsReflectionScale, dielectricMsTransmissionScale;
  float dielectricMsViewLoss, dielectricMsReflectionRatio, dielectricMsProbability;
  float weights[LOBE_COUNT];
  float probabilities[LOBE_COUNT];
};

struct BsdfContext {
  const float *lut;
  bool hasMedium;
  bool hasThinFilm;
};


// Energy LUT rows, src/renderer/decodeOpenPbrEnergyLut.ts:20-33.
__device__ constexpr int LUT_METAL_ROW = 1056, LUT_METAL_AVG_ROW = 1088, LUT_DIEL_ROW = 1089,
                 LUT_DIEL_AVG_ROW = 2113, LUT_DIEL_RATIO_ROW = 2145;

// ---------------------------------------------------------- sampling.wgsl.ts
// sampling.wgsl.ts:6-22
MTD V3 ggxVisibleNormal(V3 view, V2 alpha, V2 u) {
  V3 stretch = {alpha.x, alpha.y, 1.0f};
  V3 sphericalView = normalize(stretch * view);
  float viewZ = fminf(sphericalView.z, 1.0f);
  float capSpan = 1.0f + viewZ;
  float normalZ = (1.0f - u.y) * capSpan;
  float oneMinusZ = u.y * capSpan;
  float onePlusZ = normalZ + (1.0f - viewZ);
  float radial = sqrtf(fmaxf(0.0f, onePlusZ * oneMinusZ));
  float azimuth = TWOPI * u.x;
  V3 sn = {sphericalView.x + radial * cosf(azimuth), sphericalView.y + radial * sinf(azimuth), normalZ};
  return normalize(stretch * sn);
}
// sampling.wgsl.ts:24-34
MTD float ggxNdf(V3 h, V2 alpha) {
  V3 e = {h.x / alpha.x, h.y / alpha.y, h.z};
  float den = dot(e, e);
  return 1.0f / (PI * alpha.x * alpha.y * den * den);
}
// sampling.wgsl.ts:36-45
MTD float ggxSmithG1(V3 d, V2 alpha) {
  float nc = fabsf(d.z);
  if (nc <= 1e-8f) return 0.0f;
  V2 rd = {alpha.x * d.x, alpha.y * d.y};
  float tan2 = dot2(rd, rd) / (nc * nc);
  return 2.0f / (1.0f + sqrtf(1.0f + tan2));
}
// sampling.wgsl.ts:47-50
MTD float schlickFifth(float c) {
  float k = clampf(1.0f - c, 0.0f, 1.0f);
  return powf(k, 5.0f);
}
// sampling.wgsl.ts:52-67
MTD float dielectricFresnel(float incidentCosine, float eta) {
  float ci = clampf(fabsf(incidentCosine), 0.0f, 1.0f);
  float st2 = eta * eta * fmaxf(0.0f, 1.0f - ci * ci);
  if (st2 >= 1.0f) return 1.0f;
  float ct = sqrtf(fmaxf(0.0f, 1.0f - st2));
  float perp = (ci - eta * ct) / fmaxf(ci + eta * ct, 1e-8f);
  float par = (eta * ci - ct) / fmaxf(eta * ci + ct, 1e-8f);
  return 0.5f * (perp * perp + par * par);
}
// sampling.wgsl.ts:69-92
MTD V2 concentricDisk(V2 u) {
  V2 o = {2.0f * u.x - 1.0f, 2.0f * u.y - 1.0f};
  if (o.x == 0.0f && o.y == 0.0f) return {0, 0};
  float radius, angle;
  if (fabsf(o.x) > fabsf(o.y)) { radius = o.x; angle = 0.25f * PI * (o.y / o.x); }
  else { radius = o.y; angle = 0.5f * PI - 0.25f * PI * (o.x / o.y); }
  return {radius * cosf(angle), radius * sinf(angle)};
}
MTD V3 cosineHemisphere(V2 u) {
  V2 d = concentricDisk(u);
  return {d.x, d.y, sqrtf(fmaxf(0.0f, 1.0f - dot2(d, d)))};
}
// sampling.wgsl.ts:102-111
MTD float powerHeuristic(float a, float b) {
  float scale = fmaxf(a, b);
  if (scale <= 0.0f) return 0.0f;
  float na = a / scale, nb = b / scale;
  float sa = na * na, sb = nb * nb;
  return sa / (sa + sb);
}
// sampling.wgsl.ts:113-131
MTD void orthonormalBasis(V3 n, V3 &t, V3 &b) {
  float signZ = n.z >= 0.0f ? 1.0f : -1.0f;
  float factor = -1.0f / (signZ + n.z);
  float xy = n.x * n.y * factor;
  t = {1.0f + signZ * n.x * n.x * factor, signZ * xy, -signZ * n.x};
  b = {xy, signZ + n.y * n.y * factor, -n.y};
}
// sampling.wgsl.ts:136-158
MTD float cauchyIor(float wavelength, float ior, float scale, float abbe) {
  if (wavelength == 0.0f || scale <= 0.0f) return ior;
  const float C = 656.3f, D = 587.6f, F = 486.1f;
  float inverseDifference = 1.0f / (1.0f / (F * F) - 1.0f / (C * C));
  float effectiveAbbe = fmaxf(abbe / scale, 1e-6f);
  float b = (ior - 1.0f) * inverseDifference / effectiveAbbe;
  float a = ior - b / (D * D);
  return a + b / (wavelength * wavelength);
}
// sampling.wgsl.ts:160-184
MTD V3 henyeyGreenstein(V3 forward, float g, V2 u) {
  float cosine;
  if (fabsf(g) < 0.001f) cosine = 1.0f - 2.0f * u.y;
  else {
    float ratio = (1.0f - g * g) / (1.0f + g - 2.0f * g * u.y);
    cosine = (ratio * ratio - 1.0f - g * g) / (2.0f * g);
  }
  float sine = sqrtf(fmaxf(0.0f, 1.0f - cosine * cosine));
  float az = TWOPI * u.x;
  V3 t, b;
  orthonormalBasis(forward, t, b);
  return t * (sine * cosf(az)) + b * (sine * sinf(az)) + forward * cosine;
}
// sampling.wgsl.ts:186-191
MTD float henyeyGreensteinPhase(float cosine, float g) {
  float den = 1.0f + g * g + 2.0f * g * cosine;
  return INV4PI * (1.0f - g * g) / (den * sqrtf(den));
}

// -------------------------------------------------------- openPbrBsdf.wgsl.ts
MTD float luminance(V3 c) { return dot(c, v3(0.212671f, 0.715160f, 0.072169f)); }
MTD float f0FromIor(float eta) { float v = (eta - 1.0f) / (eta + 1.0f); return v * v; }
// openPbrBsdf.wgsl.ts:86-97
MTD float applySpecularWeightToIor(float eta, float w) {
  float scaledF0 = fminf(f0FromIor(eta) * w, 0.9999f);
  float s = sqrtf(scaledF0);
  float ext = (1.0f + s) / (1.0f - s);
  return eta < 1.0f ? 1.0f / ext : ext;
}
MTD float opDielectricFresnel(float c, float rel) {
  if (fabsf(rel - 1.0f) < 1e-6f) return 0.0f;
  return dielectricFresnel(c, rel);
}
MTD float energyIorIndex(float ior) {
  if (ior < 1.0f) return 15.0f - ((1.0f / ior - 1.0f) / 1.5f) * 15.0f;
  return 16.0f + ((ior - 1.0f) / 1.5f) * 15.0f;
}
MTD float lutFetch(const BsdfContext &c, int cosIndex, int row) { return __ldg(c.lut + row * 32 + cosIndex); }
// openPbrBsdf.wgsl.ts:117-150 (row base 0) and 173-206 (ideal dielectric rows)
MTD float lutTrilinear(const BsdfContext &c, int base, float exactIor, float exactAlpha, float exactCos) {
  float ii = clampf(exactIor, 0.0f, 31.0f), ai = clampf(exactAlpha, 0.0f, 31.0f), ci = clampf(exactCos, 0.0f, 31.0f);
  int i0 = int(floorf(ii)), a0 = int(floorf(ai)), c0 = int(floorf(ci));
  int i1 = min(i0 + 1, 31), a1 = min(a0 + 1, 31), c1 = min(c0 + 1, 31);
  float im = ii - float(i0), am = ai - float(a0), cm = ci - float(c0);
  float v000 = lutFetch(c, c0, base + i0 * 32 + a0), v001 = lutFetch(c, c1, base + i0 * 32 + a0);
  float v010 = lutFetch(c, c0, base + i0 * 32 + a1), v011 = lutFetch(c, c1, base + i0 * 32 + a1);
  float v100 = lutFetch(c, c0, base + i1 * 32 + a0), v101 = lutFetch(c, c1, base + i1 * 32 + a0);
  float v110 = lutFetch(c, c0, base + i1 * 32 + a1), v111 = lutFetch(c, c1, base + i1 * 32 + a1);
  float v00 = mixf(v000, v100, im), v01 = mixf(v001, v101, im), v10 = mixf(v010, v110, im), v11 = mixf(v011, v111, im);
  return mixf(mixf(v00, v10, am), mixf(v01, v11, am), cm);
}
// openPbrBsdf.wgsl.ts:152-171, 208-247 (averages and ratio rows)
MTD float lutBilinear(const BsdfContext &c, int base, float exactIor, float exactAlpha) {
  float ii = clampf(exactIor, 0.0f, 31.0f), ai = clampf(exactAlpha, 0.0f, 31.0f);
  int i0 = int(floorf(ii)), a0 = int(floorf(ai));
  int i1 = min(i0 + 1, 31), a1 = min(a0 + 1, 31);
  float im = ii - float(i0), am = ai - float(a0);
  float v00 = lutFetch(c, a0, base + i0), v01 = lutFetch(c, a1, base + i0);
  float v10 = lutFetch(c, a0, base + i1), v11 = lutFetch(c, a1, base + i1);
  return mixf(mixf(v00, v10, im), mixf(v01, v11, im), am);
}
MTD float idealDielectricLoss(const BsdfContext &c, float ior, float alpha, float cosine) {
  return lutTrilinear(c, LUT_DIEL_ROW, energyIorIndex(ior), sqrtf(alpha) * 31.0f, cosine * 31.0f);
}
MTD float idealDielectricAverageLoss(const BsdfContext &c, float ior, float alpha) {
  return lutBilinear(c, LUT_DIEL_AVG_ROW, energyIorIndex(ior), sqrtf(alpha) * 31.0f);
}
MTD float idealDielectricReflectionRatio(const BsdfContext &c, float ior, float alpha) {
  return lutBilinear(c, LUT_DIEL_RATIO_ROW, energyIorIndex(ior), sqrtf(alpha) * 31.0f);
}
// openPbrBsdf.wgsl.ts:261-273
MTD float metalEnergyComplement(const BsdfContext &c, float alpha, float cosine) {
  float ri = clampf(sqrtf(alpha) * 31.0f, 0.0f, 31.0f);
  float ci = clampf(cosine * 31.0f, 0.0f, 31.0f);
  int r0 = int(floorf(ri)), c0 = int(floorf(ci));
  int r1 = min(r0 + 1, 31), c1 = min(c0 + 1, 31);
  return mixf(mixf(lutFetch(c, c0, LUT_METAL_ROW + r0), lutFetch(c, c1, LUT_METAL_ROW + r0), fractf(ci)),
              mixf(lutFetch(c, c0, LUT_METAL_ROW + r1), lutFetch(c, c1, LUT_METAL_ROW + r1), fractf(ci)),
              fractf(ri));
}
// openPbrBsdf.wgsl.ts:275-280
MTD float metalAverageEnergyComplement(const BsdfContext &c, float alpha) {
  float index = clampf(sqrtf(alpha) * 31.0f, 0.0f, 31.0f);
  int i0 = int(floorf(index));
  return mixf(lutFetch(c, i0, LUT_METAL_AVG_ROW), lutFetch(c, min(i0 + 1, 31), LUT_METAL_AVG_ROW), fractf(index));
}
// openPbrBsdf.wgsl.ts:282-289
MTD float extrapolateEnergyComplement(float value, float ior) {
  if (ior > 2.5f || ior < 0.4f) {
    float maxF0 = f0FromIor(2.5f);
    float progress = (f0FromIor(ior) - maxF0) / (1.0f - maxF0);
    return (1.0f - progress) * value;
  }
  return value;
}
// openPbrBsdf.wgsl.ts:291-313
MTD float opaqueEnergyComplement(const BsdfContext &c, float ior, float alpha, float cosine) {
  float v = lutTrilinear(c, 0, energyIorIndex(ior), sqrtf(alpha) * 31.0f, cosine * 31.0f);
  return extrapolateEnergyComplement(v, ior);
}
MTD float opaqueAverageEnergyComplement(const BsdfContext &c, float ior, float alpha) {
  float v = lutBilinear(c, 1024, energyIorIndex(ior), sqrtf(alpha) * 31.0f);
  return extrapolateEnergyComplement(v, ior);
}
// openPbrBsdf.wgsl.ts:315-327
MTD V3 toWorld(const Basis &b, V3 d) { return b.tangent * d.x + b.bitangent * d.y + b.normal * d.z; }
MTD V3 toLocal(const Basis &b, V3 d) { return {dot(d, b.tangent), dot(d, b.bitangent), dot(d, b.normal)}; }
// openPbrBsdf.wgsl.ts:329-347
MTD Basis makeBasis(V3 inputTangent, V3 normal, float anisotropy) {
  Basis basis;
  basis.normal = normal;
  V3 t = inputTangent, b = v3(0.0f);
  if (dot(t, t) < 0.001f || anisotropy <= 0.0f) orthonormalBasis(normal, t, b);
  else { b = normalize(cross(normal, t)); t = normalize(cross(b, normal)); }
  basis.tangent = t;
  basis.bitangent = b;
  return basis;
}
// openPbrBsdf.wgsl.ts:349-387
MTD float fresnelS(float ni, float nt, float ci, float ct) { return (ni * ci - nt * ct) / (ni * ci + nt * ct); }
MTD float fresnelP(float ni, float nt, float ci, float ct) { return (nt * ci - ni * ct) / (ni * ct + nt * ci); }
MTD float transmissionS(float ni, float nt, float ci, float ct) { return 2.0f * ni * ci / (ni * ci + nt * ct); }
MTD float transmissionP(float ni, float nt, float ci, float ct) { return 2.0f * ni * ci / (ni * ct + nt * ci); }
MTD V2 cmul(V2 a, V2 b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
MTD V2 cdiv(V2 a, V2 b) {
  float den = fmaxf(dot2(b, b), 1e-9f);
  return {(a.x * b.x + a.y * b.y) / den, (a.y * b.x - a.x * b.y) / den};
}
MTD V2 csqrt(V2 v) {
  float mag = sqrtf(dot2(v, v));
  float re = sqrtf(fmaxf(0.0f, 0.5f * (mag + v.x)));
  float im = sqrtf(fmaxf(0.0f, 0.5f * (mag - v.x)));
  return {re, v.y >= 0.0f ? im : -im};
}
// openPbrBsdf.wgsl.ts:397-425
MTD V2 complexFresnelReflection(float ci, float ni, V2 nt, bool p) {
  float si = sqrtf(fmaxf(0.0f, 1.0f - ci * ci));
  V2 ratio = cdiv({ni, 0.0f}, nt);
  V2 st = {ratio.x * si, ratio.y * si};
  V2 sq = cmul(st, st);
  V2 ct = csqrt({1.0f - sq.x, 0.0f - sq.y});
  if (cmul(nt, ct).y < 0.0f) ct = {-ct.x, -ct.y};
  V2 nic = {ni * ci, 0.0f};
  V2 ntc = cmul(nt, ct);
  if (p) {
    V2 a = {nt.x * ci, nt.y * ci};
    V2 b = {ct.x * ni, ct.y * ni};
    return cdiv({a.x - b.x, a.y - b.y}, {a.x + b.x, a.y + b.y});
  }
  return cdiv({nic.x - ntc.x, nic.y - ntc.y}, {nic.x + ntc.x, nic.y + ntc.y});
}
// openPbrBsdf.wgsl.ts:427-442
MTD float airyReflectance(float r12, float t12, float r21, float t21, V2 r23, float phase) {
  V2 rot = {cosf(phase), sinf(phase)};
  V2 rp = cmul(r23, rot);
  V2 num = {rp.x * (t12 * t21), rp.y * (t12 * t21)};
  V2 den = {1.0f - rp.x * r21, 0.0f - rp.y * r21};
  V2 q = cdiv(num, den);
  V2 total = {r12 + q.x, 0.0f + q.y};
  return dot2(total, total);
}
// openPbrBsdf.wgsl.ts:444-483 (loopUnrollGuard = 4: two polarizations)
MTD float thinFilmReflectanceChannel(float incidentCosine, float wavelength, float thickness, float ext,
                                        float film, V2 substrate) {
  float sc = clampf(fabsf(incidentCosine), 1e-5f, 1.0f);
  float fs2 = powf(ext / film, 2.0f) * (1.0f - sc * sc);
  if (fs2 >= 1.0f) return 1.0f;
  float fc = sqrtf(1.0f - fs2);
  float r12s = fresnelS(ext, film, sc, fc), r12p = fresnelP(ext, film, sc, fc);
  float t12s = transmissionS(ext, film, sc, fc), t12p = transmissionP(ext, film, sc, fc);
  float t21Scale = film * fc / fmaxf(ext * sc, 1e-9f);
  float phase = 2.0f * PI * (2.0f * film * thickness * fc) / wavelength;
  float refl = 0.0f;
  for (int pol = 0; pol < 2; pol++) {
    float r12 = pol == 1 ? r12p : r12s;
    float t12 = pol == 1 ? t12p : t12s;
    V2 r23 = complexFresnelReflection(fc, film, substrate, pol == 1);
    refl += airyReflectance(r12, t12, -r12, t12 * t21Scale, r23, phase);
  }
  return clampf(0.5f * refl, 0.0f, 1.0f);
}
// openPbrBsdf.wgsl.ts:488-498
MTD V3 metalFresnel(float cosine, V3 f0, V3 tint) {
  V3 schlick = mix3(f0, v3(1.0f), schlickFifth(cosine));
  if (tint.x == 1.0f && tint.y == 1.0f && tint.z == 1.0f) return schlick;
  const float edgeCosine = 1.0f / 7.0f;
  float edgeComplement = 1.0f - edgeCosine;
  V3 edgeFresnel = mix3(f0, v3(1.0f), schlickFifth(edgeCosine));
  float complement = 1.0f - cosine;
  float correction = cosine * schlickFifth(cosine) * complement / (edgeCosine * powf(edgeComplement, 6.0f));
  return vclamp(schlick - (edgeFresnel - tint * edgeFresnel) * correction, 0.0f, 1.0f);
}
// openPbrBsdf.wgsl.ts:500-511
MTD V2 metalComplexIor(float f0, float tint) {
  float r = clampf(f0, 0.0f, 0.99f);
  float sr = sqrtf(r);
  float minIor = (1.0f - r) / (1.0f + r);
  float maxIor = (1.0f + sr) / fmaxf(1.0f - sr, 1e-9f);
  float ior = mixf(maxIor, minIor, clampf(tint, 0.0f, 1.0f));
  float k2 = ((ior + 1.0f) * (ior + 1.0f) * r - (ior - 1.0f) * (ior - 1.0f)) / fmaxf(1.0f - r, 1e-9f);
  return {ior, sqrtf(fmaxf(k2, 0.0f))};
}
MTD float thinFilmPresence(float thickness, float weight) {
  return clampf(weight, 0.0f, 1.0f) * smoothstepf(1e-9f, 30.0f, thickness);
}
// openPbrBsdf.wgsl.ts:520-573 (EON diffuse)
MTD V3 evalDiffuse(const Material &m, V3 color, V3 view, V3 light, float comp, float &pdf) {
  pdf = 0.0f;
  if (light.z <= 0.0f) return v3(0.0f);
  float r = m.diffuseRoughness;
  const float A = 0.5f - 2.0f / (3.0f * PI);
  const float B = 2.0f / 3.0f - 28.0f / (15.0f * PI);
  float mi = light.z, mo = view.z;
  float directional = dot(light, view) - mi * mo;
  float dot_ = directional > 0.0f ? directional / fmaxf(fmaxf(mi, mo), 1e-7f) : directional;
  float ssA = 1.0f / (1.0f + A * r);
  V3 single = color * INVPI * ssA * (1.0f + r * dot_);
  float ic = 1.0f - mi, oc = 1.0f - mo;
  float ig = ic * (0.0571085289f + ic * (0.491881867f + ic * (-0.332181442f + ic * 0.0714429953f)));
  float og = oc * (0.0571085289f + oc * (0.491881867f + oc * (-0.332181442f + oc * 0.0714429953f)));
  float ia = (1.0f + r * ig) / (1.0f + A * r);
  float oa = (1.0f + r * og) / (1.0f + A * r);
  float avg = ssA * (1.0f + B * r);
  V3 msAlbedo = color * color * avg / vmax(v3(1e-7f), v3(1.0f) - color * (1.0f - avg));
  V3 multi = msAlbedo * INVPI * fmaxf(1e-7f, 1.0f - oa) * fmaxf(1e-7f, 1.0f - ia) / fmaxf(1e-7f, 1.0f - avg);
  pdf = light.z * INVPI;
  return (single + multi) * comp;
}
// openPbrBsdf.wgsl.ts:575-590
MTD float fuzzDirectionalAlbedo(float viewCosine, float roughness) {
  float x = clampf(viewCosine, 0.0f, 1.0f);
  float y = clampf(roughness, 0.01f, 1.0f);
  float scale = y * (0.0206607f + 1.58491f * y) / (0.0379424f + y * (1.32227f + y));
  float mean = y * (-0.193854f + y * (-1.14885f + y * (1.7932f - 0.95943f * y * y))) / (0.046391f + y);
  float offset = y * (0.000654023f + (-0.0207818f + 0.119681f * y) * y) / (1.26264f + y * (-1.92021f + y));
  float gaussian = expf(-0.5f * powf((x - mean) / scale, 2.0f)) / (scale * sqrtf(2.0f * PI));
  return fmaxf(gaussian + offset, 0.0f);
}
// openPbrBsdf.wgsl.ts:592-608
MTD V3 evalFuzz(const Material &m, V3 view, V3 light, float &pdf) {
  pdf = 0.0f;
  if (view.z <= 0.0f || light.z <= 0.0f) return v3(0.0f);
  float albedo = fuzzDirectionalAlbedo(view.z, m.fuzzRoughness);
  pdf = light.z * INVPI;
  return m.fuzzColor * albedo * INVPI;
}
// openPbrBsdf.wgsl.ts:610-649
MTD V3 evalMicrofacetReflection(float ax, float ay, V3 view, V3 light, V3 h, V3 fresnel, float &pdf) {
  pdf = 0.0f;
  if (light.z <= 0.0f) return v3(0.0f);
  V2 alpha = {ax, ay};
  float D = ggxNdf(h, alpha);
  float G1 = ggxSmithG1(view, alpha);
  float G = G1 * ggxSmithG1(light, alpha);
  pdf = G1 * D / (4.0f * fmaxf(view.z, 1e-8f));
  return fresnel * D * G / (4.0f * fmaxf(light.z * view.z, 1e-8f));
}
// openPbrBsdf.wgsl.ts:651-688
MTD V3 evalMicrofacetRefraction(float ax, float ay, float rel, V3 tint, V3 view, V3 light, V3 h, V3 fresnel,
                                   float &pdf) {
  pdf = 0.0f;
  if (light.z >= 0.0f) return v3(0.0f);
  float lh = dot(light, h), vh = dot(view, h);
  if (vh <= 0.0f || lh >= 0.0f) return v3(0.0f);
  V2 alpha = {ax, ay};
  float D = ggxNdf(h, alpha);
  float G1 = ggxSmithG1(view, alpha);
  float G = G1 * ggxSmithG1(light, alpha);
  float den = lh + vh * rel;
  den *= den;
  float jac = fabsf(lh) / fmaxf(den, 1e-8f);
  float rel2 = rel * rel;
  pdf = G1 * fmaxf(0.0f, vh) * D * jac / fmaxf(view.z, 1e-8f);
  return tint * (v3(1.0f) - fresnel) * D * G * fabsf(vh) * jac * rel2 / fmaxf(fabsf(light.z * view.z), 1e-8f);
}
// openPbrBsdf.wgsl.ts:690-695
MTD V3 transmissionTint(const BsdfContext &c, const Material &m) {
  if (c.hasMedium && m.mediumType > 0) return v3(1.0f);
  return m.transmissionColor;
}
MTD float thinWallFresnel(float f) { return 2.0f * f / (1.0f + f); }
MTD V3 thinWallReflectionCoefficient(V3 f, float w) {
  V3 window = f * 2.0f / (v3(1.0f) + f);
  return mix3(f, window, clampf(w, 0.0f, 1.0f));
}
// openPbrBsdf.wgsl.ts:714-730
MTD V3 finalTransmissionTint(const BsdfContext &c, const Material &m, float ci, float eta) {
  V3 tint = transmissionTint(c, m);
  if (!m.thinWalled) return tint;
  float is2 = fmaxf(0.0f, 1.0f - ci * ci);
  float ts2 = is2 / fmaxf(eta * eta, 1e-9f);
  if (ts2 >= 1.0f) return v3(0.0f);
  float tc = sqrtf(1.0f - ts2);
  float e = 1.0f / fmaxf(tc, 1e-5f);
  V3 t = vmax(tint, v3(0.0f));
  return {powf(t.x, e), powf(t.y, e), powf(t.z, e)};
}
// openPbrBsdf.wgsl.ts:732-748
MTD V3 evalSubsurfaceBoundary(float relativeIor, V3 view, V3 light, float &pdf) {
  pdf = 0.0f;
  if (view.z <= 0.0f || light.z >= 0.0f) return v3(0.0f);
  float tc = -light.z;
  float ef = dielectricFresnel(view.z, relativeIor);
  pdf = tc * INVPI;
  return v3(1.0f - ef) * INVPI;
}
// openPbrBsdf.wgsl.ts:750-769 (loopUnrollGuard = 4 covers the seven lobes)
MTD void normalizeProbabilities(Prepared &p) {
  float total = p.probabilities[0];
  for (int l = 1; l < LOBE_COUNT; l++) total += p.probabilities[l];
  if (total <= 1e-8f) { for (int l = 0; l < LOBE_COUNT; l++) p.probabilities[l] = 0.0f; return; }
  float inv = 1.0f / total;
  for (int l = 0; l < LOBE_COUNT; l++) p.probabilities[l] *= inv;
}
// openPbrBsdf.wgsl.ts:773-777
MTD float averageFresnel(float eta) {
  if (fabsf(eta - 1.0f) < 1e-6f) return 0.0f;
  if (eta > 1.0f) return (eta - 1.0f) / (4.08567f + 1.00071f * eta);
  return 0.997118f + 0.1014f * eta - 0.965241f * eta * eta - 0.130607f * eta * eta * eta;
}
// openPbrBsdf.wgsl.ts:779-784
MTD V3 metalAverageFresnel(V3 f0, V3 tint) {
  const float ec = 1.0f / 7.0f;
  V3 ef = mix3(f0, v3(1.0f), schlickFifth(ec));
  V3 b = ef * (v3(1.0f) - tint) / (ec * powf(1.0f - ec, 6.0f));
  return vclamp(f0 + (v3(1.0f) - f0) / 21.0f - b / 126.0f, 0.0f, 1.0f);
}
// openPbrBsdf.wgsl.ts:788-793
MTD V3 coatPassage(const Material &m, float cosine) {
  if (cosine <= 0.0f) return v3(1.0f);
  float rc = sqrtf(fmaxf(0.0f, 1.0f - (1.0f - cosine * cosine) / (m.coatIor * m.coatIor)));
  float e = 0.5f / fmaxf(rc, 1e-5f);
  V3 cc = vmax(m.coatColor, v3(0.0f));
  V3 pass = {powf(cc.x, e), powf(cc.y, e), powf(cc.z, e)};
  return mix3(v3(1.0f), pass, m.coatWeight);
}
// openPbrBsdf.wgsl.ts:795-803
MTD float coatEnergy(const BsdfContext &c, const Material &m, float cosine) {
  if (m.coatRoughness <= ROUGHNESS_MIN) return opDielectricFresnel(cosine, 1.0f / m.coatIor);
  return clampf(1.0f - opaqueEnergyComplement(c, m.coatIor, m.coatRoughness * m.coatRoughness, cosine), 0.0f, 1.0f);
}
// openPbrBsdf.wgsl.ts:805-823
MTD V3 coatDarkening(const Prepared &p) {
  const Material &m = *p.mat;
  float dielectric = 1.0f - m.baseMetalness;
  float opaque = dielectric * (1.0f - m.transmissionWeight) * (1.0f - m.subsurfaceWeight);
  float sss = dielectric * (1.0f - m.transmissionWeight) * m.subsurfaceWeight;
  float trans = dielectric * m.transmissionWeight;
  float opaqueSpec = averageFresnel(p.specularEtaTOverEtaI);
  float transSpec = averageFresnel(1.0f / p.transmissionReflectionIor);
  float specularity = clampf(opaque * opaqueSpec + (sss + trans) * transSpec + m.baseMetalness, 0.0f, 1.0f);
  float effRough = mixf(1.0f, m.specularRoughness, specularity);
  float ks = averageFresnel(m.coatIor);
  float kr = 1.0f - (1.0f - ks) / (m.coatIor * m.coatIor);
  float k = mixf(ks, kr, effRough);
  V3 eb = metalAverageFresnel(m.baseColor * m.baseWeight, m.specularColor) * (m.baseMetalness * m.specularWeight) +
          mix3(m.baseColor * m.baseWeight, v3(1.0f), opaqueSpec) * opaque + m.subsurfaceColor * sss + v3(trans);
  V3 delta = v3(1.0f - k) / vmax(v3(1.0f) - eb * k, v3(1e-6f));
  return mix3(v3(1.0f), delta, m.coatWeight * m.coatDarkening);
}
// openPbrBsdf.wgsl.ts:825-833
MTD V3 coatBaseScale(const BsdfContext &c, const Prepared &p, float lightCosine) {
  (void)c;
  if (p.mat->coatWeight <= 0.0f) return v3(1.0f);
  if (p.mat->inside) return coatPassage(*p.mat, -lightCosine);
  return p.coatBaseScale * coatPassage(*p.mat, lightCosine);
}
// openPbrBsdf.wgsl.ts:837-850
MTD Basis directionBasis(const Basis &fallback, V3 tangent, V3 bitangent, V2 direction) {
  V3 t = tangent - fallback.normal * dot(fallback.normal, tangent);
  if (dot(t, t) < 1e-8f) t = fallback.tangent;
  t = normalize(t);
  V3 b = cross(fallback.normal, t) * (dot(cross(fallback.normal, t), bitangent) < 0.0f ? -1.0f : 1.0f);
  t = t * direction.x + b * direction.y;
  if (dot(t, t) < 1e-8f) return fallback;
  Basis basis = fallback;
  basis.tangent = normalize(t);
  basis.bitangent = normalize(cross(basis.normal, basis.tangent));
  basis.tangent = normalize(cross(basis.bitangent, basis.normal));
  return basis;
}
MTD V2 roughnessToAlpha(float roughness, float anisotropy) {
  float alpha = roughness * roughness;
  float alphaMin = ROUGHNESS_MIN * ROUGHNESS_MIN;
  if (anisotropy == 0.0f) { float a = fmaxf(alphaMin, alpha); return {a, a}; }
  float comp = 1.0f - anisotropy;
  float alphaT = alpha * sqrtf(2.0f / (1.0f + comp * comp));
  return {fmaxf(alphaMin, alphaT), fmaxf(alphaMin, comp * alphaT)};
}

// openPbrBsdf.wgsl.ts:853-1080
MTD Prepared prepare(const BsdfContext &c, V3 tangent, const Material &material, V3 viewDirection, V3 normal) {
  Prepared p = {};
  p.mat = &material;
  p.relativeIor = material.relativeIor;
  p.basis = makeBasis(tangent, normal, fmaxf(material.specularAnisotropy, material.coatAnisotropy));
  p.coatBasis = p.basis;
  p.directionFrames = false;
  if (material.specularAnisotropy > 0.0f && material.anisotropyDirectionEnabled) {
    p.basis = directionBasis(p.basis, material.directionTangent, material.directionBitangent, material.anisotropyDirection);
    p.directionFrames = true;
  }
  if (material.coatAnisotropy > 0.0f && material.coatAnisotropyRotation != 0.0f) {
    p.coatBasis = directionBasis(p.coatBasis, material.geometryTangent, material.geometryBitangent,
                                 {cosf(material.coatAnisotropyRotation), sinf(material.coatAnisotropyRotation)});
    p.directionFrames = true;
  }
  p.viewLocal = toLocal(p.basis, viewDirection);
  p.diffuseColor = material.baseColor;
  float dielectricBase = 1.0f - material.baseMetalness;
  float opaqueDielectric = dielectricBase * (1.0f - material.transmissionWeight);
  p.weights[LOBE_FUZZ] = material.fuzzWeight;
  p.weights[LOBE_COAT] = material.coatWeight;
  if (material.inside) p.weights[LOBE_COAT] = 0.0f;
  p.weights[LOBE_METAL] = material.baseMetalness;
  p.weights[LOBE_SPECULAR] = dielectricBase;
  p.weights[LOBE_TRANSMISSION] = dielectricBase * material.transmissionWeight;
  p.weights[LOBE_DIFFUSE] = opaqueDielectric * (1.0f - material.subsurfaceWeight) * material.baseWeight;
  p.weights[LOBE_SUBSURFACE] = opaqueDielectric * material.subsurfaceWeight;

  p.specularEtaTOverEtaI = applySpecularWeightToIor(1.0f / material.relativeIor, material.specularWeight);
  p.relativeIor = 1.0f / p.specularEtaTOverEtaI;
  p.refractionEtaTOverEtaI = p.specularEtaTOverEtaI;
  p.transmissionReflectionIor = p.relativeIor;
  if (material.coatWeight > 0.0f) {
    float weightedCoatIor = 1.0f;
    if (!material.inside) weightedCoatIor = mixf(1.0f, material.coatIor, material.coatWeight);
    float weightedBaseIor = weightedCoatIor * applySpecularWeightToIor(material.specularIor / weightedCoatIor, material.specularWeight);
    float reflectionEta = weightedBaseIor / weightedCoatIor;
    if (weightedCoatIor > weightedBaseIor && weightedBaseIor >= 1.0f) reflectionEta = 1.0f / reflectionEta;
    p.specularEtaTOverEtaI = reflectionEta;
    p.transmissionReflectionIor = 1.0f / reflectionEta;
    p.refractionEtaTOverEtaI = weightedBaseIor;
    if (material.inside) {
      p.refractionEtaTOverEtaI = 1.0f / weightedBaseIor;
      p.transmissionReflectionIor = weightedBaseIor;
    }
    p.relativeIor = 1.0f / p.refractionEtaTOverEtaI;
  }
  p.thinFilmExteriorIor = 1.0f;
  p.thinFilmBaseIor = p.specularEtaTOverEtaI;
  if (material.coatWeight > 0.0f) {
    if (material.inside) { p.thinFilmExteriorIor = 1.0f / p.refractionEtaTOverEtaI; p.thinFilmBaseIor = 1.0f; }
    else { p.thinFilmExteriorIor = mixf(1.0f, material.coatIor, material.coatWeight); p.thinFilmBaseIor = p.refractionEtaTOverEtaI; }
  }
  p.specularAlpha = material.specularRoughness * material.specularRoughness;
  float viewCosine = fabsf(p.viewLocal.z);
  float sif = opDielectricFresnel(viewCosine, 1.0f / p.specularEtaTOverEtaI);
  V3 dielectricFresnelEstimate = material.specularColor *
      (material.thinWalled ? mixf(sif, thinWallFresnel(sif), material.transmissionWeight) : sif);
  V3 metalFresnelEstimate = metalFresnel(viewCosine, material.baseColor * material.baseWeight, material.specularColor) * material.specularWeight;
  float tf = opDielectricFresnel(viewCosine, p.transmissionReflectionIor);
  float transmissionFresnel = material.thinWalled ? thinWallFresnel(tf) : tf;
  V3 tint = finalTransmissionTint(c, material, viewCosine, p.refractionEtaTOverEtaI);
  float viewEC = opaqueEnergyComplement(c, p.specularEtaTOverEtaI, p.specularAlpha, viewCosine);
  float avgEC = opaqueAverageEnergyComplement(c, p.specularEtaTOverEtaI, p.specularAlpha);
  p.diffuseSpecularEnergyCompensation = viewEC / fmaxf(avgEC, 1e-12f);

  p.probabilities[LOBE_FUZZ] = p.weights[LOBE_FUZZ] * luminance(material.fuzzColor) *
                               fmaxf(fuzzDirectionalAlbedo(viewCosine, material.fuzzRoughness), 0.02f);
  p.probabilities[LOBE_COAT] = 0.0f;
  p.coatBaseScale = v3(1.0f);
  if (material.coatWeight > 0.0f && !material.inside) {
    float ce = coatEnergy(c, material, viewCosine);
    p.probabilities[LOBE_COAT] = p.weights[LOBE_COAT] * ce;
    p.coatBaseScale = coatPassage(material, viewCosine) * (1.0f - p.weights[LOBE_COAT] * ce) * coatDarkening(p);
  }
  p.probabilities[LOBE_METAL] = p.weights[LOBE_METAL] * luminance(metalFresnelEstimate);
  p.metalMsScale = v3(0.0f);
  p.metalMsFactor = 0.0f;
  p.metalMsProbability = 0.0f;
  if (material.specularRoughness >= 0.04f && p.weights[LOBE_METAL] > 0.0f) {
    V3 af = metalAverageFresnel(material.baseColor * material.baseWeight, material.specularColor);
    p.metalMsScale = af * af * material.specularWeight;
    float viewLoss = metalEnergyComplement(c, p.specularAlpha, viewCosine);
    p.metalMsFactor = viewLoss / fmaxf(metalAverageEnergyComplement(c, p.specularAlpha), 1e-12f);
    float msEstimate = p.weights[LOBE_METAL] * luminance(p.metalMsScale) * viewLoss;
    p.probabilities[LOBE_METAL] += msEstimate;
    p.metalMsProbability = msEstimate / fmaxf(p.probabilities[LOBE_METAL], 1e-12f);
  }
  p.probabilities[LOBE_SPECULAR] = p.weights[LOBE_SPECULAR] * luminance(dielectricFresnelEstimate);
  p.probabilities[LOBE_TRANSMISSION] = p.weights[LOBE_TRANSMISSION] * (1.0f - transmissionFresnel) * luminance(tint);
  p.dielectricMsReflectionScale = v3(0.0f);
  p.dielectricMsTransmissionScale = v3(0.0f);
  p.dielectricMsViewLoss = 0.0f;
  p.dielectricMsReflectionRatio = 0.0f;
  p.dielectricMsProbability = 0.0f;
  if (!material.thinWalled && material.transmissionWeight > 0.0f && p.specularAlpha >= 0.0016f &&
      p.weights[LOBE_TRANSMISSION] > 0.0f && fabsf(p.refractionEtaTOverEtaI - 1.0f) > 1e-6f) {
    float nonOpaque = p.weights[LOBE_TRANSMISSION] + p.weights[LOBE_SUBSURFACE];
    p.dielectricMsReflectionScale = (material.inside ? v3(1.0f) : material.specularColor) * nonOpaque;
    p.dielectricMsTransmissionScale = tint * p.weights[LOBE_TRANSMISSION] + v3(p.weights[LOBE_SUBSURFACE]);
    p.dielectricMsReflectionRatio = idealDielectricReflectionRatio(c, p.refractionEtaTOverEtaI, p.specularAlpha);
    p.dielectricMsViewLoss = idealDielectricLoss(c, p.refractionEtaTOverEtaI, p.specularAlpha, viewCosine);
    V3 averageScale = mix3(p.dielectricMsTransmissionScale, p.dielectricMsReflectionScale, p.dielectricMsReflectionRatio);
    float msEstimate = luminance(averageScale) * p.dielectricMsViewLoss;
    p.probabilities[LOBE_TRANSMISSION] += msEstimate;
    p.dielectricMsProbability = msEstimate / fmaxf(p.probabilities[LOBE_TRANSMISSION], 1e-12f);
  }
  p.probabilities[LOBE_DIFFUSE] = p.weights[LOBE_DIFFUSE] * luminance(p.diffuseColor) * p.diffuseSpecularEnergyCompensation;
  p.probabilities[LOBE_SUBSURFACE] = p.weights[LOBE_SUBSURFACE] * (1.0f - transmissionFresnel) *
                                     luminance(material.subsurfaceColor) * p.diffuseSpecularEnergyCompensation;
  if (material.coatWeight > 0.0f && c.hasThinFilm && material.thinFilmWeight > 0.0f) {
    float film = 0.02f * thinFilmPresence(material.thinFilmThickness, material.thinFilmWeight);
    p.probabilities[LOBE_SPECULAR] = fmaxf(p.probabilities[LOBE_SPECULAR], p.weights[LOBE_SPECULAR] * film);
    p.probabilities[LOBE_METAL] = fmaxf(p.probabilities[LOBE_METAL], p.weights[LOBE_METAL] * material.specularWeight * film);
  }
  if (material.coatWeight > 0.0f && !material.inside) {
    float bs = maxc(p.coatBaseScale);
    p.probabilities[LOBE_METAL] *= bs;
    p.probabilities[LOBE_SPECULAR] *= bs;
    p.probabilities[LOBE_TRANSMISSION] *= bs;
    p.probabilities[LOBE_DIFFUSE] *= bs;
    p.probabilities[LOBE_SUBSURFACE] *= bs;
  }
  normalizeProbabilities(p);
  return p;
}

// openPbrBsdf.wgsl.ts:1083-1091
MTD float substrateFresnel(const Prepared &p, float cosine, bool reflection) {
  if (p.mat->coatWeight <= 0.0f) return opDielectricFresnel(cosine, p.relativeIor);
  float trans = opDielectricFresnel(cosine, p.transmissionReflectionIor);
  if (!reflection) return trans;
  float opaque = opDielectricFresnel(cosine, 1.0f / p.specularEtaTOverEtaI);
  float nonOpaque = p.mat->transmissionWeight + (1.0f - p.mat->transmissionWeight) * p.mat->subsurfaceWeight;
  return mixf(opaque, trans, nonOpaque);
}

// openPbrBsdf.wgsl.ts:1092-1422 with allowedLobe = -1 (all lobes)
MTD V3 evalPrepared(const BsdfContext &c, const Prepared &p, V3 lightDirection, float &pdfOut) {
  const Material &m = *p.mat;
  V3 view = p.viewLocal;
  V3 light = toLocal(p.basis, lightDirection);
  bool reflection = light.z * view.z > 0.0f;
  V3 h = reflection ? normalize(light + view) : normalize(light + view * p.relativeIor);
  if (h.z < 0.0f) h = -h;
  V3 response = v3(0.0f);
  float pdf = 0.0f, lobePdf = 0.0f;
  float viewHalf = fabsf(dot(view, h));
  V3 thinWallHalf = h;
  float dielectricViewHalf = viewHalf;
  if (!reflection && m.thinWalled) {
    thinWallHalf = normalize(V3{light.x, light.y, -light.z} + view);
    if (thinWallHalf.z < 0.0f) thinWallHalf = -thinWallHalf;
    dielectricViewHalf = fabsf(dot(view, thinWallHalf));
  }
  bool evalDielectric = (reflection && p.weights[LOBE_SPECULAR] > 0.0f) ||
                        (!reflection && p.weights[LOBE_TRANSMISSION] > 0.0f);
  bool evalMetal = reflection && p.weights[LOBE_METAL] > 0.0f;
  V3 fresnels[2] = {v3(0.0f), v3(0.0f)};
  if (evalDielectric) fresnels[0] = v3(substrateFresnel(p, dielectricViewHalf, reflection));
  if (evalMetal) fresnels[1] = metalFresnel(viewHalf, m.baseColor * m.baseWeight, m.specularColor);
  if (c.hasThinFilm && m.thinFilmWeight > 0.0f) {
    const float wl[3] = {620.0f, 540.0f, 450.0f};
    for (int sub = 0; sub < 2; sub++) {
      if (!(sub == 1 ? evalMetal : evalDielectric)) continue;
      V3 film = v3(0.0f);
      float ic = sub == 1 ? viewHalf : dielectricViewHalf;
      for (int ch = 0; ch < 3; ch++) {
        V2 ior = {p.thinFilmBaseIor, 0.0f};
        if (sub == 1) ior = metalComplexIor(m.baseWeight * comp(m.baseColor, ch), comp(m.specularColor, ch));
        setcomp(film, ch, thinFilmReflectanceChannel(ic, wl[ch], m.thinFilmThickness, p.thinFilmExteriorIor, m.thinFilmIor, ior));
      }
      fresnels[sub] = mix3(fresnels[sub], film, thinFilmPresence(m.thinFilmThickness, m.thinFilmWeight));
    }
  }
  V3 subF = fresnels[0];
  float dsec = p.diffuseSpecularEnergyCompensation *
               opaqueEnergyComplement(c, p.specularEtaTOverEtaI, p.specularAlpha, fabsf(light.z));
  if (reflection) {
    if (p.weights[LOBE_DIFFUSE] > 0.0f) {
      response += evalDiffuse(m, p.diffuseColor, view, light, dsec, lobePdf) * p.weights[LOBE_DIFFUSE];
      pdf += p.probabilities[LOBE_DIFFUSE] * lobePdf;
    }
    if (p.weights[LOBE_SUBSURFACE] > 0.0f && m.thinWalled) {
      response += evalDiffuse(m, m.subsurfaceColor, view, light, dsec, lobePdf) * (0.5f * p.weights[LOBE_SUBSURFACE]);
      pdf += p.probabilities[LOBE_SUBSURFACE] * 0.5f * lobePdf;
    }
    if (p.weights[LOBE_SPECULAR] > 0.0f) {
      V3 df = subF;
      if (m.thinWalled) df = thinWallReflectionCoefficient(df, m.transmissionWeight);
      V3 fresnel = m.specularColor * df;
      response += evalMicrofacetReflection(m.alphaX, m.alphaY, view, light, h, fresnel, lobePdf) * p.weights[LOBE_SPECULAR];
      pdf += p.probabilities[LOBE_SPECULAR] * lobePdf;
    }
    if (p.weights[LOBE_METAL] > 0.0f) {
      V3 fresnel = fresnels[1] * m.specularWeight;
      response += evalMicrofacetReflection(m.alphaX, m.alphaY, view, light, h, fresnel, lobePdf) * p.weights[LOBE_METAL];
      if (p.metalMsFactor > 0.0f) {
        float factor = fminf(p.metalMsFactor * metalEnergyComplement(c, p.specularAlpha, light.z), 1.0f / fmaxf(light.z, 1e-8f));
        response += p.metalMsScale * (p.weights[LOBE_METAL] * factor * INVPI);
        lobePdf = mixf(lobePdf, 0.5f * INVPI, p.metalMsProbability);
      }
      pdf += p.probabilities[LOBE_METAL] * lobePdf;
    }
  } else {
    if (p.weights[LOBE_TRANSMISSION] > 0.0f) {
      if (m.thinWalled) {
        V3 mirrored = {light.x, light.y, -light.z};
        V3 window = thinWallReflectionCoefficient(subF, 1.0f);
        V3 tint = finalTransmissionTint(c, m, fabsf(view.z), p.refractionEtaTOverEtaI);
        response += evalMicrofacetReflection(m.alphaX, m.alphaY, view, mirrored, thinWallHalf, tint * (v3(1.0f) - window), lobePdf) *
                    p.weights[LOBE_TRANSMISSION];
      } else {
        response += evalMicrofacetRefraction(m.alphaX, m.alphaY, p.relativeIor, transmissionTint(c, m), view, light, h, subF, lobePdf) *
                    p.weights[LOBE_TRANSMISSION];
      }
      if (p.dielectricMsProbability > 0.0f) lobePdf *= 1.0f - p.dielectricMsProbability;
      pdf += p.probabilities[LOBE_TRANSMISSION] * lobePdf;
    }
    if (p.weights[LOBE_SUBSURFACE] > 0.0f) {
      if (m.thinWalled) {
        V3 flipped = {light.x, light.y, -light.z};
        response += evalDiffuse(m, m.subsurfaceColor, view, flipped, dsec, lobePdf) * (0.5f * p.weights[LOBE_SUBSURFACE]);
        lobePdf *= 0.5f;
      } else {
        response += evalSubsurfaceBoundary(p.relativeIor, view, light, lobePdf) * p.weights[LOBE_SUBSURFACE];
      }
      pdf += p.probabilities[LOBE_SUBSURFACE] * lobePdf;
    }
  }
  if (p.dielectricMsProbability > 0.0f) {
    float cosine = fabsf(light.z);
    if (cosine > 0.0f) {
      float ior = reflection ? p.refractionEtaTOverEtaI : 1.0f / p.refractionEtaTOverEtaI;
      float ratio = reflection ? p.dielectricMsReflectionRatio : 1.0f - p.dielectricMsReflectionRatio;
      float factors = p.dielectricMsViewLoss * idealDielectricLoss(c, ior, p.specularAlpha, cosine) /
                      fmaxf(idealDielectricAverageLoss(c, ior, p.specularAlpha), 1e-12f);
      float factor = fminf(factors * ratio, 1.0f / cosine);
      V3 scale = reflection ? p.dielectricMsReflectionScale : p.dielectricMsTransmissionScale;
      response += scale * (factor * INVPI);
      pdf += p.probabilities[LOBE_TRANSMISSION] * p.dielectricMsProbability * ratio * 0.5f * INVPI;
    }
  }
  if (m.coatWeight > 0.0f) response *= coatBaseScale(c, p, light.z);
  if (reflection && p.weights[LOBE_COAT] > 0.0f) {
    V3 coatView = view, coatLight = light, coatHalf = h;
    float coatViewHalf = viewHalf;
    if (p.directionFrames) {
      coatView = toLocal(p.coatBasis, toWorld(p.basis, view));
      coatLight = toLocal(p.coatBasis, lightDirection);
      coatHalf = normalize(coatLight + coatView);
      if (coatHalf.z < 0.0f) coatHalf = -coatHalf;
      coatViewHalf = fabsf(dot(coatView, coatHalf));
    }
    V3 coatF = v3(opDielectricFresnel(coatViewHalf, 1.0f / m.coatIor));
    V2 ca = roughnessToAlpha(m.coatRoughness, m.coatAnisotropy);
    response += evalMicrofacetReflection(ca.x, ca.y, coatView, coatLight, coatHalf, coatF, lobePdf) * p.weights[LOBE_COAT];
    pdf += p.probabilities[LOBE_COAT] * lobePdf;
  }
  if (reflection && p.weights[LOBE_FUZZ] > 0.0f) {
    float fa = fuzzDirectionalAlbedo(fabsf(view.z), m.fuzzRoughness);
    response *= vmax(v3(0.0f), v3(1.0f - p.weights[LOBE_FUZZ] * fa));
    response += evalFuzz(m, view, light, lobePdf) * p.weights[LOBE_FUZZ];
    pdf += p.probabilities[LOBE_FUZZ] * lobePdf;
  }
  pdfOut = pdf;
  return response * fabsf(light.z);
}

// openPbrBsdf.wgsl.ts:1450-1657
MTD bool sampleDirection(const BsdfContext &c, const Prepared &p, V3 rnd, V3 &lightDirection, bool &isTransmission) {
  (void)c;
  const Material &m = *p.mat;
  V3 view = p.viewLocal;
  float rx = rnd.x, ry = rnd.y, lobeSample = rnd.z;
  isTransmission = false;
  lightDirection = p.basis.normal;
  float cdf[LOBE_COUNT];
  cdf[0] = p.probabilities[0];
  for (int i = 1; i < LOBE_COUNT; i++) cdf[i] = cdf[i - 1] + p.probabilities[i];
  if (cdf[LOBE_SUBSURFACE] <= 0.0f) return false;
  V3 light;
  if (lobeSample < cdf[LOBE_FUZZ] || (lobeSample >= cdf[LOBE_TRANSMISSION] && lobeSample < cdf[LOBE_DIFFUSE])) {
    light = cosineHemisphere({rx, ry});
  } else if (lobeSample < cdf[LOBE_COAT]) {
    V3 coatView = view;
    if (p.directionFrames) coatView = toLocal(p.coatBasis, toWorld(p.basis, view));
    V3 hv = ggxVisibleNormal(coatView, roughnessToAlpha(m.coatRoughness, m.coatAnisotropy), {rx, ry});
    if (hv.z < 0.0f) hv = -hv;
    light = normalize(reflect(-coatView, hv));
    if (p.directionFrames) light = toLocal(p.basis, toWorld(p.coatBasis, light));
  } else if (lobeSample < cdf[LOBE_SPECULAR]) {
    bool isMetal = lobeSample < cdf[LOBE_METAL];
    float metalDraw = (lobeSample - cdf[LOBE_COAT]) / fmaxf(p.probabilities[LOBE_METAL], 1e-12f);
    if (isMetal && metalDraw < p.metalMsProbability) {
      float z = rx;
      float radial = sqrtf(fmaxf(0.0f, 1.0f - z * z));
      float az = TWOPI * ry;
      light = {radial * cosf(az), radial * sinf(az), z};
    } else {
      V3 hv = ggxVisibleNormal(view, {m.alphaX, m.alphaY}, {rx, ry});
      if (hv.z < 0.0f) hv = -hv;
      light = normalize(reflect(-view, hv));
    }
  } else if (lobeSample < cdf[LOBE_TRANSMISSION]) {
    isTransmission = true;
    float msDraw = (lobeSample - cdf[LOBE_SPECULAR]) / fmaxf(p.probabilities[LOBE_TRANSMISSION], 1e-12f);
    if (p.dielectricMsProbability > 0.0f && msDraw < p.dielectricMsProbability) {
      float ratio = p.dielectricMsReflectionRatio;
      bool reflectMs = rx < ratio;
      float z = reflectMs ? fminf(rx / ratio, 0.99999994f) : -fminf((rx - ratio) / (1.0f - ratio), 0.99999994f);
      float radial = sqrtf(fmaxf(0.0f, 1.0f - z * z));
      float az = TWOPI * ry;
      light = {radial * cosf(az), radial * sinf(az), z};
      isTransmission = !reflectMs;
    } else {
      V3 hv = ggxVisibleNormal(view, {m.alphaX, m.alphaY}, {rx, ry});
      if (hv.z < 0.0f) hv = -hv;
      if (m.thinWalled) {
        V3 r = normalize(reflect(-view, hv));
        light = {r.x, r.y, -r.z};
      } else {
        light = refract(-view, hv, p.relativeIor);
        if (dot(light, light) <= 1e-8f) { isTransmission = false; return false; }
        light = normalize(light);
      }
    }
  } else {
    isTransmission = true;
    if (m.thinWalled) {
      bool transmit = rx >= 0.5f;
      if (transmit) rx = (rx - 0.5f) * 2.0f; else rx *= 2.0f;
      light = cosineHemisphere({rx, ry});
      if (transmit) light.z = -light.z; else isTransmission = false;
    } else {
      light = cosineHemisphere({rx, ry});
      light.z = -light.z;
    }
  }
  lightDirection = toWorld(p.basis, light);
  if (light.z == 0.0f || ((light.z < 0.0f) != isTransmission)) return false;
  return true;
}


}  // namespace mt
