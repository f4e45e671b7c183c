// solid_shim.h -- the Slang names that the solid-cell code of
// gprt/gprt_fallbacks.slang (getVertexCount, getSolidHitKind, GetInitialRST,
// IsoIsContained, IsoToSupport, intersectPointSolid, SolidBounds) uses, so
// that code compiles as C++ (oracle/Makefile extracts it with awk and makes
// the few syntactic edits listed there).
//
// Slang semantics restated here:
//   * floating literals are single precision (the Makefile compiles with
//     -fsingle-precision-constant) and every operation is rounded once
//     (-ffp-contract=off);
//   * a float4's .xyz is its first three components; assigning a scalar to
//     a vector broadcasts it;
//   * float3x3(a, b, c) takes rows; determinant() is the cofactor expansion
//     along the first row, m00(m11 m22 - m12 m21) - m01(m10 m22 - m12 m20)
//     + m02(m10 m21 - m11 m20);
//   * rcp(x) = 1 / x;
//   * fwd_diff(f)(args, diffPair(x, dx)).getDifferential() is forward-mode
//     differentiation: f is evaluated on dual numbers (value, derivative) with
//     d(a +- b) = da +- db, d(c - a) = -da, d(a b) = da b + a db.
//
// TEST INFRASTRUCTURE ONLY: pins the oracle's restatement of the solid-cell
// math against the reference's own code.  Never linked into the product.
#pragma once
#include <cfloat>
#include <cmath>
#include <cstdint>

typedef uint32_t uint;

struct uint4 {
  uint x, y, z, w;
};

template <class S> struct V2 {
  S x, y;
  V2() = default;
  V2(S s) : x(s), y(s) {}  // scalar-to-vector broadcast, as HLSL assigns it
  V2(S a, S b) : x(a), y(b) {}
};
template <class S> struct V3 {
  S x, y, z;
  V3() = default;
  explicit V3(S s) : x(s), y(s), z(s) {}
  V3(S a, S b, S c) : x(a), y(b), z(c) {}
};
typedef V2<float> float2;
typedef V3<float> float3;

// .xyz is a member; the Makefile rewrites the code's rstw.x / .y / .z
// updates as rstw.xyz.x / .y / .z and aabbMax.yz as an explicit float2.
struct float4 {
  float3 xyz;
  float w;
  float4() = default;
  float4(float s) : xyz(s), w(s) {}
  float4(float3 a, float b) : xyz(a), w(b) {}
  float4(float2 a, float2 b) : xyz(a.x, a.y, b.x), w(b.y) {}
};

struct bool3 {
  bool x, y, z;
};

static inline float3 operator+(float3 a) { return a; }
static inline float3 operator-(float3 a) { return float3(-a.x, -a.y, -a.z); }
static inline float3 operator+(float3 a, float3 b) { return float3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline float3 operator-(float3 a, float3 b) { return float3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline float3 operator*(float3 a, float s) { return float3(a.x * s, a.y * s, a.z * s); }
static inline float3 operator-(float s, float3 a) { return float3(s - a.x, s - a.y, s - a.z); }
static inline float3 &operator+=(float3 &a, float3 b) {
  a = a + b;
  return a;
}
static inline float min(float a, float b) { return std::fmin(a, b); }
static inline float max(float a, float b) { return std::fmax(a, b); }
static inline float3 min(float3 a, float3 b) { return float3(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
static inline float3 max(float3 a, float3 b) { return float3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
static inline float abs(float v) { return std::fabs(v); }
static inline float3 abs(float3 a) { return float3(std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)); }
static inline float rcp(float v) { return 1.0f / v; }
static inline bool3 operator<(float3 a, float s) { return bool3{a.x < s, a.y < s, a.z < s}; }
static inline bool3 operator>=(float3 a, float s) { return bool3{a.x >= s, a.y >= s, a.z >= s}; }
static inline bool3 operator<=(float3 a, float s) { return bool3{a.x <= s, a.y <= s, a.z <= s}; }
static inline bool all(bool3 b) { return b.x && b.y && b.z; }

struct float3x3 {
  float3 r0, r1, r2;
  float3x3(float3 a, float3 b, float3 c) : r0(a), r1(b), r2(c) {}
};
static inline float determinant(const float3x3 &m) {
  return m.r0.x * (m.r1.y * m.r2.z - m.r1.z * m.r2.y) - m.r0.y * (m.r1.x * m.r2.z - m.r1.z * m.r2.x) +
         m.r0.z * (m.r1.x * m.r2.y - m.r1.y * m.r2.x);
}

// Dual numbers for forward-mode differentiation.
struct Dual {
  float v, d;
  Dual() = default;
  Dual(float a) : v(a), d(0.0f) {}
  Dual(float a, float b) : v(a), d(b) {}
};
static inline Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
static inline Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
static inline Dual operator-(float c, Dual a) { return Dual(c - a.v, -a.d); }
static inline Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
static inline V3<Dual> operator-(float c, V3<Dual> a) { return V3<Dual>(c - a.x, c - a.y, c - a.z); }

template <class S> struct Arr8 {
  S v[8];
  S &operator[](int i) { return v[i]; }
  const S &operator[](int i) const { return v[i]; }
};

struct DiffResult {
  Arr8<Dual> r;
  Arr8<float> getDifferential() const {
    Arr8<float> o;
    for (int i = 0; i < 8; ++i) o.v[i] = r.v[i].d;
    return o;
  }
};
static inline V3<Dual> diffPair(float3 x, float3 dx) {
  return V3<Dual>(Dual(x.x, dx.x), Dual(x.y, dx.y), Dual(x.z, dx.z));
}
#define let auto
#define fwd_diff(f) [](int n_, V3<Dual> x_) { return DiffResult{f<Dual>(n_, x_)}; }

// Hit kinds (gprt/gprt_builtins.slang:42-45).
static const uint HIT_KIND_TETRAHEDRON = 10;
static const uint HIT_KIND_HEXAHEDRON = 12;
static const uint HIT_KIND_WEDGE = 13;
static const uint HIT_KIND_PYRAMID = 14;

// SolidParameters (gprt/gprt_fallbacks.h:37-50), field names kept.
struct SolidParameters {
  float4 *vertices;
  uint4 *indices;
  uint8_t *types;
  float4 *aabbs;
  uint32_t offset;
  uint32_t count;
  uint32_t typesOffset;
  uint32_t typesStride;
  uint32_t indicesOffset;
  uint32_t indicesStride;
  uint32_t verticesOffset;
  uint32_t verticesStride;
};
struct uint3 {
  uint x, y, z;
};
#define uniform
