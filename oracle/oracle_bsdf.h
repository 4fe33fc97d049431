// Test infrastructure only (the checker, never the product).
//
// OpenPBR 1.1 layered BSDF of the CPU oracle, restating
// src/renderer/wgsl/chunks/openPbrBsdf.wgsl.ts (hasAnisotropyDirections=true,
// hasCoatNormals=false) and the helpers of sampling.wgsl.ts.
#pragma once
#include "oracle_core.h"

namespace oracle {

// OpenPbrResolvedMaterial, rayTraceCore.wgsl.ts:118-190.
struct Material {
  V3 baseColor{}; float transmissionWeight = 0;
  V3 emission{}; float specularAnisotropy = 0;
  float baseMetalness = 0, specularIor = 0, specularRoughness = 0;
  float transmissionDispersionScale = 0, dispersionAbbeNumber = 0, thinFilmThickness = 0,
        thinFilmIor = 0, thinFilmWeight = 0;
  i32 mediumType = 0; V3 mediumExtinction{}, mediumScattering{}; float mediumAnisotropy = 0;
  float baseWeight = 0, diffuseRoughness = 0, specularWeight = 0; V3 specularColor{};
  float subsurfaceWeight = 0; V3 subsurfaceColor{}, transmissionColor{};
  float fuzzWeight = 0; V3 fuzzColor{}; float fuzzRoughness = 0;
  float coatWeight = 0; V3 coatColor{}; float coatRoughness = 0, coatAnisotropy = 0;
  V2 anisotropyDirection{}; bool anisotropyDirectionEnabled = false; float coatAnisotropyRotation = 0;
  V3 directionTangent{}, directionBitangent{}, geometryTangent{}, geometryBitangent{};
  float coatIor = 0, coatDarkening = 0;
  float alpha = 0; i32 alphaMode = 0; i32 materialType = 0; float bevel = 0;
  float relativeIor = 0; bool inside = false; float alphaX = 0, alphaY = 0; bool thinWalled = false;
};

struct Basis { V3 tangent{}, bitangent{}, normal{}; };

enum { LOBE_FUZZ = 0, LOBE_COAT = 1, LOBE_METAL = 2, LOBE_SPECULAR = 3,
       LOBE_TRANSMISSION = 4, LOBE_DIFFUSE = 5, LOBE_SUBSURFACE = 6, LOBE_COUNT = 7 };

// OpenPbrPreparedBsdf, openPbrBsdf.wgsl.ts:45-75.
struct Prepared {
  Material material;
  Basis basis, coatBasis;
  bool directionFrames = false;
  V3 viewLocal{}, diffuseColor{};
  float specularEtaTOverEtaI = 0, refractionEtaTOverEtaI = 0, transmissionReflectionIor = 0,
        thinFilmExteriorIor = 0, thinFilmBaseIor = 0, specularAlpha = 0,
        diffuseSpecularEnergyCompensation = 0;
  V3 coatBaseScale{}, metalMsScale{};
  float metalMsFactor = 0, metalMsProbability = 0;
  V3 dielectricMsReflectionScale{}, dielectricMsTransmissionScale{};
  float dielectricMsViewLoss = 0, dielectricMsReflectionRatio = 0, dielectricMsProbability = 0;
  float weights[LOBE_COUNT] = {0, 0, 0, 0, 0, 0, 0};
  float probabilities[LOBE_COUNT] = {0, 0, 0, 0, 0, 0, 0};
};

struct BsdfContext {
  const float *lut;
  bool hasMedium;
  bool hasThinFilm;
};

float powerHeuristic(float a, float b);
void orthonormalBasis(V3 n, V3 &t, V3 &b);
V3 ggxVisibleNormal(V3 view, V2 alpha, V2 u);
V3 cosineHemisphere(V2 u);
V3 henyeyGreenstein(V3 forward, float g, V2 u);
float henyeyGreensteinPhase(float cosine, float g);
float cauchyIor(float wavelength, float ior, float dispersionScale, float abbe);
V2 roughnessToAlpha(float roughness, float anisotropy);
V3 transmissionTint(const BsdfContext &c, const Material &m);
V3 coatBaseScale(const BsdfContext &c, const Prepared &p, float lightCosine);
V3 toWorld(const Basis &b, V3 d);
Prepared prepare(const BsdfContext &c, V3 tangent, const Material &m, V3 view, V3 normal);
V3 evalPrepared(const BsdfContext &c, const Prepared &p, V3 lightDirection, float &pdf);
bool sampleDirection(const BsdfContext &c, const Prepared &p, V3 rnd, V3 &lightDirection,
                     bool &isTransmission);

}  // namespace oracle
