// ref_solids.cpp -- C entry points over the reference's own solid-cell code
// (gprt/gprt_fallbacks.slang: getVertexCount, getSolidHitKind, SolidBounds,
// intersectPointSolid), compiled from the reference sources by
// oracle/Makefile.
//
// TEST INFRASTRUCTURE ONLY: pins the oracle restatement.  The product never
// links it.
#include "solid_shim.h"

int getVertexCount(uint32_t cellType);
uint getSolidHitKind(uint32_t cellType);
bool intersectPointSolid(float3 P, const float3 *Q, const float *W, uint32_t nodeCount, float4 &rstw);
void SolidBounds(uint3 DispatchThreadID, SolidParameters s);

extern "C" int ref_solid_vertex_count(uint32_t type) { return getVertexCount(type); }
extern "C" uint32_t ref_solid_hit_kind(uint32_t type) { return getSolidHitKind(type); }

// SolidIntersection's call (gprt/gprt_fallbacks.slang:504-566): the cell's
// vertices in index order, zero beyond its vertex count.  qw: 8 float4
// {x, y, z, density}.  Returns 1 if the point lies in the cell.
extern "C" int ref_solid_intersect(const float *p, const float *qw, uint32_t nodeCount, float *rstw) {
  float3 Q[8];
  float W[8];
  for (int i = 0; i < 8; ++i) {
    Q[i] = float3(qw[4 * i + 0], qw[4 * i + 1], qw[4 * i + 2]);
    W[i] = qw[4 * i + 3];
  }
  float4 r(0.0f);
  const bool hit = intersectPointSolid(float3(p[0], p[1], p[2]), Q, W, nodeCount, r);
  rstw[0] = r.xyz.x;
  rstw[1] = r.xyz.y;
  rstw[2] = r.xyz.z;
  rstw[3] = r.w;
  return hit ? 1 : 0;
}

// SolidBounds over `count` cells with the default strides (float4 vertices,
// eight uint32 indices and one uint8 type per cell); aabbs: two float4 per
// cell in the reference's layout.
extern "C" void ref_solid_bounds(const float *vertices, const uint32_t *indices, const uint8_t *types,
                                 uint32_t count, float *aabbs) {
  SolidParameters s;
  s.vertices = (float4 *)vertices;
  s.indices = (uint4 *)indices;
  s.types = (uint8_t *)types;
  s.aabbs = (float4 *)aabbs;
  s.offset = 0;
  s.count = count;
  s.typesOffset = 0;
  s.typesStride = 1;
  s.indicesOffset = 0;
  s.indicesStride = 32;
  s.verticesOffset = 0;
  s.verticesStride = 16;
  for (uint32_t i = 0; i < count; ++i) SolidBounds(uint3{i, 0, 0}, s);
}
