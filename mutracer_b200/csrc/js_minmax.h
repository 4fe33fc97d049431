// JavaScript Math.min / Math.max on IEEE values, for the BVH producers
// (src/renderer/binnedSahBvh.ts growBin and SAH sweep, bvhAccel.ts
// triangleBounds and refitTLAS, scenePreparation.ts computeBounds via
// vec3.min/max).  Unlike std::min / fminf: a NaN operand gives NaN, and -0 is
// below +0 whatever the operand order, so a reduction is independent of the
// order in which it visits its inputs.
#pragma once
#include <cmath>

#if defined(__CUDACC__)
#define MT_JS_HD __host__ __device__ __forceinline__
#else
#define MT_JS_HD inline
#endif
#if defined(__CUDA_ARCH__)
#define MT_JS_SIGNBIT(x) signbit(x)
#else
#define MT_JS_SIGNBIT(x) std::signbit(x)
#endif

template <class T>
MT_JS_HD T jsMin(T a, T b) {
  if (a != a || b != b) return a + b;  // NaN
  if (a == b) return MT_JS_SIGNBIT(a) ? a : b;
  return b < a ? b : a;
}

template <class T>
MT_JS_HD T jsMax(T a, T b) {
  if (a != a || b != b) return a + b;  // NaN
  if (a == b) return MT_JS_SIGNBIT(a) ? b : a;
  return b > a ? b : a;
}
