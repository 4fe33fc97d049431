// Test infrastructure only: the CPU oracle's scalar vector math.
//
// Every operation is written out component by component, left to right, so
// that with -ffp-contract=off each product and sum is rounded exactly as the
// WGSL source states it (no fused multiply-add).  The CUDA kernels follow the
// same order with explicit __fmul_rn/__fadd_rn wherever bit-exact hit IDs
// depend on it (traversal, slab and triangle tests).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>

namespace om {

typedef uint32_t u32;
typedef int32_t i32;

// Constants of src/renderer/wgsl/chunks/common.wgsl.ts:3-10 and
// rayTraceCore.wgsl.ts:45-46.
constexpr float PI = 3.14159265359f;
constexpr float TWOPI = 6.28318530718f;
constexpr float INVPI = 0.31830988618f;
constexpr float INVPI2 = 0.10132118364f;
constexpr float EPS = 0.0005f;
constexpr float INV4PI = 0.07957747154594766f;
constexpr float INF = 1.0e+38f;
constexpr float ROUGHNESS_MIN = 0.001f;
constexpr float RAY_MAX_DISTANCE = 9999.0f;

struct V2 { float x, y; };
struct V3 { float x, y, z; };
struct V4 { float x, y, z, w; };

inline V2 v2(float x, float y) { return {x, y}; }
inline V3 v3(float x, float y, float z) { return {x, y, z}; }
inline V3 v3(float s) { return {s, s, s}; }
inline V3 xyz(V4 a) { return {a.x, a.y, a.z}; }

inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline V3 operator/(V3 a, V3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline V3 &operator+=(V3 &a, V3 b) { a = a + b; return a; }
inline V3 &operator*=(V3 &a, V3 b) { a = a * b; return a; }
inline V3 &operator*=(V3 &a, float s) { a = a * s; return a; }
inline V3 &operator/=(V3 &a, float s) { a = a / s; return a; }

inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot2(V2 a, V2 b) { return a.x * b.x + a.y * b.y; }
inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline float length(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 normalize(V3 a) { float l = std::sqrt(dot(a, a)); return a / l; }
inline float distance(V3 a, V3 b) { return length(a - b); }
inline V3 vabs(V3 a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
// WGSL min/max on GPUs return the non-NaN operand; fminf/fmaxf do the same.
inline V3 vmin(V3 a, V3 b) { return {fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
inline V3 vmax(V3 a, V3 b) { return {fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
inline float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
inline V3 vclamp(V3 a, float lo, float hi) { return {clampf(a.x, lo, hi), clampf(a.y, lo, hi), clampf(a.z, lo, hi)}; }
inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
inline V3 mix3(V3 a, V3 b, float t) { return a * (1.0f - t) + b * t; }
inline V3 mix3(V3 a, V3 b, V3 t) { return a * (v3(1.0f) - t) + b * t; }
inline float maxc(V3 a) { return fmaxf(fmaxf(a.x, a.y), a.z); }
inline V3 reflect(V3 i, V3 n) { return i - n * (2.0f * dot(n, i)); }
// WGSL refract(e1, e2, e3).
inline V3 refract(V3 i, V3 n, float eta) {
  float ndi = dot(n, i);
  float k = 1.0f - eta * eta * (1.0f - ndi * ndi);
  if (k < 0.0f) return v3(0.0f);
  return i * eta - n * (eta * ndi + std::sqrt(k));
}
inline float fractf(float x) { return x - std::floor(x); }
inline float smoothstepf(float e0, float e1, float x) {
  float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
inline float comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
inline void setcomp(V3 &a, int i, float v) { if (i == 0) a.x = v; else if (i == 1) a.y = v; else a.z = v; }

inline float asf(u32 u) { float f; std::memcpy(&f, &u, 4); return f; }
inline u32 asu(float f) { u32 u; std::memcpy(&u, &f, 4); return u; }
inline i32 asi(float f) { i32 i; std::memcpy(&i, &f, 4); return i; }

// Column-major mat4 times (v, w): ((c0*x + c1*y) + c2*z) + c3*w per component.
inline V3 mat4_mul(const V4 *cols, V3 v, float w) {
  V3 r;
  r.x = cols[0].x * v.x + cols[1].x * v.y + cols[2].x * v.z + cols[3].x * w;
  r.y = cols[0].y * v.x + cols[1].y * v.y + cols[2].y * v.z + cols[3].y * w;
  r.z = cols[0].z * v.x + cols[1].z * v.y + cols[2].z * v.z + cols[3].z * w;
  return r;
}
inline V4 mat4_mul4(const float *m, V4 v) {
  V4 r;
  r.x = m[0] * v.x + m[4] * v.y + m[8] * v.z + m[12] * v.w;
  r.y = m[1] * v.x + m[5] * v.y + m[9] * v.z + m[13] * v.w;
  r.z = m[2] * v.x + m[6] * v.y + m[10] * v.z + m[14] * v.w;
  r.w = m[3] * v.x + m[7] * v.y + m[11] * v.z + m[15] * v.w;
  return r;
}

}  // namespace om
