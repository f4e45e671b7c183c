// rtmath.cuh -- ray/box and watertight ray/triangle arithmetic shared by the
// binary and wide traversal kernels.  Every float operation is an explicit
// round-to-nearest intrinsic so nvcc cannot contract or reorder it: the
// results are bit-identical to the CPU oracle, which evaluates the same
// sequence with one IEEE rounding per operation.
//
// Methods (the reference traces through Vulkan ray-tracing hardware and has
// no software intersection code to follow):
//   * ray/triangle: Woop, Benthin, Wald 2013, "Watertight Ray/Triangle
//     Intersection", JCGT 2(1); the 2x2 edge determinants use Kahan's
//     fused-correction form, whose sign is exact, instead of a double retry;
//   * ray/box: slab test with NaN-ignoring min/max (Ize 2013, "Robust BVH Ray
//     Traversal", JCGT 2(2)), entry scaled down / exit scaled up by 2^-18;
//   * reported distance: the plane-equation t of the winning triangle in
//     double-float arithmetic (Dekker 1971 TwoSum/TwoProduct with FMA),
//     rounded once to fp32.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace gprtcu {

// Per-ray set-up of Woop et al. 2013 section 3, kept in scalars (no indexed
// arrays, so nothing spills to local memory): kz is the axis of the largest
// |d| (lowest index on ties), kx/ky follow cyclically and swap when d[kz] < 0.
struct Ray {
  float ox, oy, oz, dx, dy, dz, tmin, tmax;
  float ix, iy, iz;  // 1/d
  float Sx, Sy, Sz;
  int kx, ky, kz;
};

constexpr float kBoxLo = 1.0f - 1.0f / 262144.0f;
constexpr float kBoxHi = 1.0f + 1.0f / 262144.0f;
constexpr uint32_t kMiss = 0xFFFFFFFFu;

__device__ __forceinline__ float pick3(float x, float y, float z, int k) { return k == 0 ? x : (k == 1 ? y : z); }

__device__ __forceinline__ void ray_setup(const float4 a, const float4 b, Ray &r) {
  r.ox = a.x; r.oy = a.y; r.oz = a.z; r.tmin = a.w;
  r.dx = b.x; r.dy = b.y; r.dz = b.z; r.tmax = b.w;
  const float ax = fabsf(b.x), ay = fabsf(b.y), az = fabsf(b.z);
  const int kz = (ax >= ay) ? (ax >= az ? 0 : 2) : (ay >= az ? 1 : 2);
  int kx = kz + 1 == 3 ? 0 : kz + 1;
  int ky = kx + 1 == 3 ? 0 : kx + 1;
  const float dkz = pick3(b.x, b.y, b.z, kz);
  if (dkz < 0.0f) {
    const int t = kx;
    kx = ky;
    ky = t;
  }
  r.kx = kx; r.ky = ky; r.kz = kz;
  r.Sx = __fdiv_rn(pick3(b.x, b.y, b.z, kx), dkz);
  r.Sy = __fdiv_rn(pick3(b.x, b.y, b.z, ky), dkz);
  // correctly rounded reciprocals: the values of 1.0f / x, without a division
  r.Sz = __frcp_rn(dkz);
  r.ix = __frcp_rn(b.x);
  r.iy = __frcp_rn(b.y);
  r.iz = __frcp_rn(b.z);
}

// a*d - b*c, Kahan's algorithm (one FMA-corrected product).
__device__ __forceinline__ float det2(float a, float b, float c, float d) {
  const float w = __fmul_rn(b, c);
  const float e = __fmaf_rn(-b, c, w);
  const float f = __fmaf_rn(a, d, -w);
  return __fadd_rn(f, e);
}

// Watertight ray/triangle; on a hit inside [tmin, tmax] returns true and the
// ordering distance t = T / det.
__device__ __forceinline__ bool isect_tri(const Ray &r, const float *v0, const float *v1, const float *v2, float &t) {
  const float A0 = __fsub_rn(v0[0], r.ox), A1 = __fsub_rn(v0[1], r.oy), A2 = __fsub_rn(v0[2], r.oz);
  const float B0 = __fsub_rn(v1[0], r.ox), B1 = __fsub_rn(v1[1], r.oy), B2 = __fsub_rn(v1[2], r.oz);
  const float C0 = __fsub_rn(v2[0], r.ox), C1 = __fsub_rn(v2[1], r.oy), C2 = __fsub_rn(v2[2], r.oz);
  const float Akx = pick3(A0, A1, A2, r.kx), Aky = pick3(A0, A1, A2, r.ky), Akz = pick3(A0, A1, A2, r.kz);
  const float Bkx = pick3(B0, B1, B2, r.kx), Bky = pick3(B0, B1, B2, r.ky), Bkz = pick3(B0, B1, B2, r.kz);
  const float Ckx = pick3(C0, C1, C2, r.kx), Cky = pick3(C0, C1, C2, r.ky), Ckz = pick3(C0, C1, C2, r.kz);
  const float Ax = __fsub_rn(Akx, __fmul_rn(r.Sx, Akz)), Ay = __fsub_rn(Aky, __fmul_rn(r.Sy, Akz));
  const float Bx = __fsub_rn(Bkx, __fmul_rn(r.Sx, Bkz)), By = __fsub_rn(Bky, __fmul_rn(r.Sy, Bkz));
  const float Cx = __fsub_rn(Ckx, __fmul_rn(r.Sx, Ckz)), Cy = __fsub_rn(Cky, __fmul_rn(r.Sy, Ckz));
  const float U = det2(Cx, Cy, Bx, By);
  const float V = det2(Ax, Ay, Cx, Cy);
  const float W = det2(Bx, By, Ax, Ay);
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
  const float det = __fadd_rn(__fadd_rn(U, V), W);
  if (det == 0.0f) return false;
  const float Az = __fmul_rn(r.Sz, Akz), Bz = __fmul_rn(r.Sz, Bkz), Cz = __fmul_rn(r.Sz, Ckz);
  const float T = __fadd_rn(__fadd_rn(__fmul_rn(U, Az), __fmul_rn(V, Bz)), __fmul_rn(W, Cz));
  const float tt = __fdiv_rn(T, det);
  if (!(tt >= r.tmin && tt <= r.tmax)) return false;
  t = tt;
  return true;
}

// NaN-propagating min/max (PTX min.NaN / max.NaN): a ray parallel to an axis
// and lying in a face plane gives 0 * inf = NaN for that axis, and the
// NaN-ignoring accumulation in ray_box then drops the axis (no bound).
__device__ __forceinline__ float nan_min(float a, float b) {
  float r;
  asm("min.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ float nan_max(float a, float b) {
  float r;
  asm("max.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
}

// Slab test against box {lo.xyz, hi.xyz}; tmax is the current best distance.
// Returns the conservative entry distance in tn.
__device__ __forceinline__ bool ray_box(const Ray &r, float lox, float loy, float loz, float hix, float hiy, float hiz,
                                        float tmax, float &tn) {
  const float t0x = __fmul_rn(__fsub_rn(lox, r.ox), r.ix), t1x = __fmul_rn(__fsub_rn(hix, r.ox), r.ix);
  const float t0y = __fmul_rn(__fsub_rn(loy, r.oy), r.iy), t1y = __fmul_rn(__fsub_rn(hiy, r.oy), r.iy);
  const float t0z = __fmul_rn(__fsub_rn(loz, r.oz), r.iz), t1z = __fmul_rn(__fsub_rn(hiz, r.oz), r.iz);
  float n_ = fmaxf(fmaxf(nan_min(t0x, t1x), nan_min(t0y, t1y)), fmaxf(nan_min(t0z, t1z), r.tmin));
  float f_ = fminf(fminf(nan_max(t0x, t1x), nan_max(t0y, t1y)), fminf(nan_max(t0z, t1z), tmax));
  n_ = __fmul_rn(n_, kBoxLo);
  f_ = __fmul_rn(f_, kBoxHi);
  tn = n_;
  return n_ <= f_;
}

// ---- double-float arithmetic (pairs of fp32) ----
struct df {
  float hi, lo;
};
__device__ __forceinline__ df two_sum(float a, float b) {
  const float s = __fadd_rn(a, b);
  const float bb = __fsub_rn(s, a);
  const float e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
  return {s, e};
}
__device__ __forceinline__ df fast_two_sum(float a, float b) {
  const float s = __fadd_rn(a, b);
  return {s, __fsub_rn(b, __fsub_rn(s, a))};
}
__device__ __forceinline__ df two_prod(float a, float b) {
  const float p = __fmul_rn(a, b);
  return {p, __fmaf_rn(a, b, -p)};
}
__device__ __forceinline__ df df_add(df x, df y) {
  df s = two_sum(x.hi, y.hi);
  df t = two_sum(x.lo, y.lo);
  s.lo = __fadd_rn(s.lo, t.hi);
  s = fast_two_sum(s.hi, s.lo);
  s.lo = __fadd_rn(s.lo, t.lo);
  return fast_two_sum(s.hi, s.lo);
}
__device__ __forceinline__ df df_neg(df x) { return {-x.hi, -x.lo}; }
__device__ __forceinline__ df df_mul(df x, df y) {
  df p = two_prod(x.hi, y.hi);
  p.lo = __fadd_rn(p.lo, __fadd_rn(__fmul_rn(x.hi, y.lo), __fmul_rn(x.lo, y.hi)));
  return fast_two_sum(p.hi, p.lo);
}
__device__ __forceinline__ df df_mulf(df x, float y) {
  df p = two_prod(x.hi, y);
  p.lo = __fadd_rn(p.lo, __fmul_rn(x.lo, y));
  return fast_two_sum(p.hi, p.lo);
}
__device__ __forceinline__ float df_div_to_f(df x, df y) {
  const float q1 = __fdiv_rn(x.hi, y.hi);
  const df r = df_add(x, df_neg(df_mulf(y, q1)));
  const float q2 = __fdiv_rn(r.hi, y.hi);
  const df q = fast_two_sum(q1, q2);
  return __fadd_rn(q.hi, q.lo);
}

// Plane-equation distance of a known hit, double-float, rounded once.
__device__ __forceinline__ float refine_t(const Ray &r, const float *v0, const float *v1, const float *v2) {
  df e1[3], e2[3], w[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    e1[a] = two_sum(v1[a], -v0[a]);
    e2[a] = two_sum(v2[a], -v0[a]);
  }
  w[0] = two_sum(v0[0], -r.ox);
  w[1] = two_sum(v0[1], -r.oy);
  w[2] = two_sum(v0[2], -r.oz);
  df n0 = df_add(df_mul(e1[1], e2[2]), df_neg(df_mul(e1[2], e2[1])));
  df n1 = df_add(df_mul(e1[2], e2[0]), df_neg(df_mul(e1[0], e2[2])));
  df n2 = df_add(df_mul(e1[0], e2[1]), df_neg(df_mul(e1[1], e2[0])));
  df num = df_add(df_add(df_mul(n0, w[0]), df_mul(n1, w[1])), df_mul(n2, w[2]));
  df den = df_add(df_add(df_mulf(n0, r.dx), df_mulf(n1, r.dy)), df_mulf(n2, r.dz));
  return df_div_to_f(num, den);
}

}  // namespace gprtcu
