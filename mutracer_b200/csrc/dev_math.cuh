// Device vector math for the sm_100a megakernel.
//
// Two flavours: ordinary float3-style helpers (the compiler may fuse
// multiply-adds; used for shading, where results are compared statistically),
// and x* helpers that round every product and sum separately with
// __fmul_rn/__fadd_rn/__fsub_rn/__fdiv_rn, in the order the WGSL source
// states them, for the traversal, slab and triangle tests whose hit IDs must
// be bit-exact.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mt {

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

#define MTD __device__ __forceinline__

MTD V2 v2(float x, float y) { return {x, y}; }
MTD V3 v3(float x, float y, float z) { return {x, y, z}; }
MTD V3 v3(float s) { return {s, s, s}; }
MTD V3 xyz(float4 a) { return {a.x, a.y, a.z}; }
MTD V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
MTD V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
MTD V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
MTD V3 operator/(V3 a, V3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
MTD V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
MTD V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
MTD V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
MTD V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
MTD V3 &operator+=(V3 &a, V3 b) { a = a + b; return a; }
MTD V3 &operator*=(V3 &a, V3 b) { a = a * b; return a; }
MTD V3 &operator*=(V3 &a, float s) { a = a * s; return a; }
MTD V3 &operator/=(V3 &a, float s) { a = a / s; return a; }
MTD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
MTD float dot2(V2 a, V2 b) { return a.x * b.x + a.y * b.y; }
MTD V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
MTD float length(V3 a) { return sqrtf(dot(a, a)); }
MTD V3 normalize(V3 a) { return a * rsqrtf(dot(a, a)); }
MTD float distance(V3 a, V3 b) { return length(a - b); }
MTD V3 vabs(V3 a) { return {fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }
MTD V3 vmin(V3 a, V3 b) { return {fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
MTD V3 vmax(V3 a, V3 b) { return {fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
MTD float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
MTD V3 vclamp(V3 a, float lo, float hi) { return {clampf(a.x, lo, hi), clampf(a.y, lo, hi), clampf(a.z, lo, hi)}; }
MTD float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
MTD V3 mix3(V3 a, V3 b, float t) { return a * (1.0f - t) + b * t; }
MTD float maxc(V3 a) { return fmaxf(fmaxf(a.x, a.y), a.z); }
MTD V3 reflect(V3 i, V3 n) { return i - n * (2.0f * dot(n, i)); }
MTD V3 refract(V3 i, V3 n, float eta) {
  float ndi = dot(n, i);
  float k = 1.0f - eta * eta * (1.0f - ndi * ndi);
  if (k < 0.0f) return v3(0.0f);
  return i * eta - n * (eta * ndi + sqrtf(k));
}
MTD float fractf(float x) { return x - floorf(x); }
MTD float smoothstepf(float e0, float e1, float x) {
  float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
MTD float comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
MTD void setcomp(V3 &a, int i, float v) { if (i == 0) a.x = v; else if (i == 1) a.y = v; else a.z = v; }

// ---- exact (unfused, round-to-nearest) helpers for bit-exact traversal ----
MTD float xm(float a, float b) { return __fmul_rn(a, b); }
MTD float xa(float a, float b) { return __fadd_rn(a, b); }
MTD float xs(float a, float b) { return __fsub_rn(a, b); }
MTD float xd(float a, float b) { return __fdiv_rn(a, b); }
MTD V3 xsub3(V3 a, V3 b) { return {xs(a.x, b.x), xs(a.y, b.y), xs(a.z, b.z)}; }
MTD V3 xmul3(V3 a, V3 b) { return {xm(a.x, b.x), xm(a.y, b.y), xm(a.z, b.z)}; }
MTD float xdot(V3 a, V3 b) { return xa(xa(xm(a.x, b.x), xm(a.y, b.y)), xm(a.z, b.z)); }
MTD V3 xcross(V3 a, V3 b) {
  return {xs(xm(a.y, b.z), xm(a.z, b.y)), xs(xm(a.z, b.x), xm(a.x, b.z)), xs(xm(a.x, b.y), xm(a.y, b.x))};
}
MTD V3 xnormalize(V3 a) {
  float l = __fsqrt_rn(xdot(a, a));
  return {xd(a.x, l), xd(a.y, l), xd(a.z, l)};
}
// Column-major mat4 (4 float4 columns) times (v, w):
// ((c0*x + c1*y) + c2*z) + c3*w, every operation rounded.
MTD V3 xmat4(float4 c0, float4 c1, float4 c2, float4 c3, V3 v, float w) {
  return {xa(xa(xa(xm(c0.x, v.x), xm(c1.x, v.y)), xm(c2.x, v.z)), xm(c3.x, w)),
          xa(xa(xa(xm(c0.y, v.x), xm(c1.y, v.y)), xm(c2.y, v.z)), xm(c3.y, w)),
          xa(xa(xa(xm(c0.z, v.x), xm(c1.z, v.y)), xm(c2.z, v.z)), xm(c3.z, w))};
}
// Shading-precision mat4 (fusion allowed).
MTD V3 mat4v(float4 c0, float4 c1, float4 c2, float4 c3, V3 v, float w) {
  return {c0.x * v.x + c1.x * v.y + c2.x * v.z + c3.x * w, c0.y * v.x + c1.y * v.y + c2.y * v.z + c3.y * w,
          c0.z * v.x + c1.z * v.y + c2.z * v.z + c3.z * w};
}

MTD float asf(uint32_t u) { return __uint_as_float(u); }
MTD uint32_t asu(float f) { return __float_as_uint(f); }
MTD int32_t asi(float f) { return __float_as_int(f); }

// Read-only 128-bit loads through the non-coherent path.
MTD float4 ld4(const float4 *p) { return __ldg(p); }

}  // namespace mt
