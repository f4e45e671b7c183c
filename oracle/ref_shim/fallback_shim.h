// fallback_shim.h -- the extra HLSL names that intersectRayLSS and
// computeLssAabb (gprt/gprt_fallbacks.slang) use, on top of hlsl_shim.h, so
// those two functions compile as C++ (oracle/Makefile extracts them).
//
// TEST INFRASTRUCTURE ONLY: pins the oracle's restatement of the sphere/LSS
// math against the reference's own code.  Never linked into the product.
#pragma once
#include "hlsl_shim.h"

static inline float3 operator*(float s, float3 a) { return float3(s * a.x, s * a.y, s * a.z); }
static inline float3 operator*(float3 a, float3 b) { return float3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline float3 operator-(float s, float3 a) { return float3(s - a.x, s - a.y, s - a.z); }
static inline float3 &operator+=(float3 &a, float3 b) {
  a = a + b;
  return a;
}
static inline float3 &operator+=(float3 &a, float s) {
  a = float3(a.x + s, a.y + s, a.z + s);
  return a;
}
static inline float dot(float3 a, float3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static inline float rcp(float v) { return 1.0f / v; }
static inline float3 abs(float3 a) { return float3(std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)); }
static inline float3 sqrt(float3 a) { return float3(std::sqrt(a.x), std::sqrt(a.y), std::sqrt(a.z)); }
static inline float sqrt(float v) { return std::sqrt(v); }
static inline float fabs(float v) { return std::fabs(v); }
static inline bool isnan(float v) { return std::isnan(v); }
static inline bool isinf(float v) { return std::isinf(v); }
