// hlsl_shim.h -- the few HLSL/GPRT device-API names that
// gprt/development/gprt_lbvh.hlsl uses, defined for the host so that file can
// be compiled unchanged (apart from the parameter qualifiers noted in
// oracle/Makefile) as C++ and run serially, one "thread" per call.
//
// TEST INFRASTRUCTURE ONLY: the result is the reference's own arithmetic,
// used to pin the oracle restatement.  Never linked into the product.
#pragma once
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>

typedef uint32_t uint;

struct int2 {
  int x, y;
  int2() : x(0), y(0) {}
  int2(int a, int b) : x(a), y(b) {}
};
struct uint2 {
  uint x, y;
};
struct uint3 {
  uint x, y, z;
  uint3() : x(0), y(0), z(0) {}
  uint3(uint a, uint b, uint c) : x(a), y(b), z(c) {}
};
struct int4 {
  int x, y, z, w;
  int4() : x(0), y(0), z(0), w(0) {}
  int4(int a, int b, int c, int d) : x(a), y(b), z(c), w(d) {}
};
struct float3 {
  float x, y, z;
  float3() : x(0), y(0), z(0) {}
  float3(float a, float b, float c) : x(a), y(b), z(c) {}
};
static inline float3 operator+(float3 a, float3 b) { return float3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline float3 operator-(float3 a, float3 b) { return float3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline float3 operator-(float3 a) { return float3(-a.x, -a.y, -a.z); }
static inline float3 operator*(float3 a, float s) { return float3(a.x * s, a.y * s, a.z * s); }
static inline float3 operator/(float3 a, float s) { return float3(a.x / s, a.y / s, a.z / s); }
static inline float3 operator/(float3 a, float3 b) { return float3(a.x / b.x, a.y / b.y, a.z / b.z); }

// HLSL min/max on floats: the non-NaN operand wins (IEEE minNum/maxNum).
static inline float min(float a, float b) { return std::fmin(a, b); }
static inline float max(float a, float b) { return std::fmax(a, b); }
static inline int min(int a, int b) { return a < b ? a : b; }
static inline int max(int a, int b) { return a > b ? a : b; }
static inline float3 min(float3 a, float3 b) { return float3(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
static inline float3 max(float3 a, float3 b) { return float3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
static inline float ceil(float v) { return std::ceil(v); }

// firstbithigh(uint): index of the highest set bit, -1 for zero.
static inline int firstbithigh(uint v) { return v ? 31 - __builtin_clz(v) : -1; }

namespace gprt {
struct Buffer {
  unsigned char *ptr;
  uint64_t bytes;
};
// Loads outside the buffer return zero (robust buffer access), which is what
// the reference's unused probe load in determine_range can reach.
template <typename T> static inline T load(Buffer b, uint64_t index) {
  T v;
  uint64_t off = index * sizeof(T);
  if (off + sizeof(T) > b.bytes) {
    std::memset(&v, 0, sizeof(T));
    return v;
  }
  std::memcpy(&v, b.ptr + off, sizeof(T));
  return v;
}
template <typename T> static inline void store(Buffer b, uint64_t index, T v) {
  uint64_t off = index * sizeof(T);
  if (off + sizeof(T) <= b.bytes) std::memcpy(b.ptr + off, &v, sizeof(T));
}
// Serial stand-ins for the CAS-loop float atomics (gprt/gprt.slang:296-352):
// store min/max, return the previous value.
static inline float atomicMin32f(Buffer b, uint64_t index, float v) {
  float old = load<float>(b, index);
  store<float>(b, index, min(old, v));
  return old;
}
static inline float atomicMax32f(Buffer b, uint64_t index, float v) {
  float old = load<float>(b, index);
  store<float>(b, index, max(old, v));
  return old;
}
}  // namespace gprt

// The LBVHData record with the field names of gprt/development/gprt_lbvh.h:28-55.
struct LBVHData {
  uint32_t numPrims;
  uint32_t numNodes;
  uint32_t numInner;
  uint32_t tmp;
  gprt::Buffer positions;
  gprt::Buffer edges;
  gprt::Buffer triangles;
  gprt::Buffer mortonCodes;
  gprt::Buffer ids;
  gprt::Buffer nodes;
  gprt::Buffer aabbs;
};

// GPRT_COMPUTE_PROGRAM(Name, (RecordType, recordName), (x,y,z)) becomes a host
// function taking the record and the dispatch thread id.
#define GPRT_SHIM_PARAM(T, n) T n
#define GPRT_COMPUTE_PROGRAM(name, rec, dims) void name(GPRT_SHIM_PARAM rec, uint3 DispatchThreadID)
