// ref_fallbacks.cpp -- C entry points over the reference's own
// intersectRayLSS and computeLssAabb (gprt/gprt_fallbacks.slang:45-144,
// 168-213), compiled from the reference sources by oracle/Makefile.
//
// TEST INFRASTRUCTURE ONLY: pins the oracle restatement.  The product never
// links it.
#include "fallback_shim.h"

bool intersectRayLSS(float3 rayOrigin, float3 rayDirection, float3 curveStart, float3 curveEnd, float radiusStart,
                     float radiusEnd, bool enableCapStart, bool enableCapEnd, float rayMin, float rayMax,
                     bool returnExit, float &rayParam, float &curveParam);
void computeLssAabb(float3 v0, float r0, bool endcap0, float3 v1, float r1, bool endcap1, float3 &bblo, float3 &bbhi);

extern "C" int ref_lss_intersect(const float *ray, const float *v0, const float *v1, int cap0, int cap1,
                                 int exit_test, float *t, float *u) {
  float tt = 0.0f, uu = 0.0f;
  const bool hit = intersectRayLSS(float3(ray[0], ray[1], ray[2]), float3(ray[4], ray[5], ray[6]),
                                   float3(v0[0], v0[1], v0[2]), float3(v1[0], v1[1], v1[2]), v0[3], v1[3], cap0 != 0,
                                   cap1 != 0, ray[3], ray[7], exit_test != 0, tt, uu);
  *t = tt;
  *u = uu;
  return hit ? 1 : 0;
}

extern "C" void ref_lss_aabb(const float *v0, const float *v1, int cap0, int cap1, float *lo, float *hi) {
  float3 a, b;
  computeLssAabb(float3(v0[0], v0[1], v0[2]), v0[3], cap0 != 0, float3(v1[0], v1[1], v1[2]), v1[3], cap1 != 0, a, b);
  lo[0] = a.x;
  lo[1] = a.y;
  lo[2] = a.z;
  hi[0] = b.x;
  hi[1] = b.y;
  hi[2] = b.z;
}
