// ref_driver.cpp -- runs the reference's LBVH compute programs
// (gprt/development/gprt_lbvh.hlsl, compiled by oracle/Makefile) serially on
// the host in the order gprtLBVHBuild issues them
// (gprt/development/gprt_lbvh.h:170-195), and exposes the reference's Hilbert
// encoder (gprt/hilbert.h:179-235).
//
// TEST INFRASTRUCTURE ONLY: this produces the reference's own results for the
// golden fixtures and the pin tests.  The product never links it.
#include "hlsl_shim.h"

#include <algorithm>
#include <utility>
#include <vector>

#include "hilbert.h"

void ComputeTriangleBounds(LBVHData record, uint3 DispatchThreadID);
void ComputeTriangleMortonCodes(LBVHData record, uint3 DispatchThreadID);
void ComputePointBounds(LBVHData record, uint3 DispatchThreadID);
void ComputePointMortonCodes(LBVHData record, uint3 DispatchThreadID);
void MakeNodes(LBVHData record, uint3 DispatchThreadID);
void SplitNodes(LBVHData record, uint3 DispatchThreadID);
void BuildTriangleHierarchy(LBVHData record, uint3 DispatchThreadID);
void BuildPointHierarchy(LBVHData record, uint3 DispatchThreadID);
void ComputeEdgeBounds(LBVHData record, uint3 DispatchThreadID);
void ComputeEdgeMortonCodes(LBVHData record, uint3 DispatchThreadID);
void BuildEdgeHierarchy(LBVHData record, uint3 DispatchThreadID);

static gprt::Buffer buf(const void *p, uint64_t bytes) { return gprt::Buffer{(unsigned char *)p, bytes}; }

// gprtBufferSortPayload's semantics on the (code, id) pairs: stable ascending.
static void sort_pairs(uint32_t *codes, uint32_t *ids, uint32_t n) {
  std::vector<std::pair<uint32_t, uint32_t>> kv(n);
  for (uint32_t i = 0; i < n; ++i) kv[i] = {codes[i], ids[i]};
  std::stable_sort(kv.begin(), kv.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
  for (uint32_t i = 0; i < n; ++i) {
    codes[i] = kv[i].first;
    ids[i] = kv[i].second;
  }
}

// kind: 0 = triangles (pos float3[npos], tri uint3[n]), 1 = points (pos float3[n]),
// 2 = edges (pos float3[npos], tri uint2[n]).
// Outputs: scene[6], codes[n], ids[n], nodes int4[2n-1], aabbs float3[2(2n-1)].
extern "C" void ref_lbvh_build(int kind, const float *pos, uint32_t npos, const uint32_t *tri, uint32_t n,
                               float *scene, uint32_t *codes, uint32_t *ids, int32_t *nodes, float *aabbs) {
  LBVHData r;
  std::memset(&r, 0, sizeof(r));
  r.numPrims = n;
  r.numNodes = 2 * n - 1;
  r.numInner = n - 1;
  r.positions = buf(pos, (uint64_t)npos * 12);
  r.triangles = buf(tri, kind == 0 ? (uint64_t)n * 12 : 0);
  r.edges = buf(tri, kind == 2 ? (uint64_t)n * 8 : 0);
  r.mortonCodes = buf(codes, (uint64_t)n * 4);
  r.ids = buf(ids, (uint64_t)n * 4);
  r.nodes = buf(nodes, (uint64_t)r.numNodes * 16);
  r.aabbs = buf(aabbs, (uint64_t)r.numNodes * 24);

  // Host seeds the root box (gprt/development/gprt_lbvh.h:174-178).
  aabbs[0] = aabbs[1] = aabbs[2] = FLT_MAX;
  aabbs[3] = aabbs[4] = aabbs[5] = -FLT_MAX;
  for (uint32_t i = 0; i < n; ++i) {
    if (kind == 0) ComputeTriangleBounds(r, uint3(i, 0, 0));
    else if (kind == 2) ComputeEdgeBounds(r, uint3(i, 0, 0));
    else ComputePointBounds(r, uint3(i, 0, 0));
  }
  for (int k = 0; k < 6; ++k) scene[k] = aabbs[k];
  for (uint32_t i = 0; i < n; ++i) {
    if (kind == 0) ComputeTriangleMortonCodes(r, uint3(i, 0, 0));
    else if (kind == 2) ComputeEdgeMortonCodes(r, uint3(i, 0, 0));
    else ComputePointMortonCodes(r, uint3(i, 0, 0));
  }
  sort_pairs(codes, ids, n);
  for (uint32_t i = 0; i < r.numNodes; ++i) MakeNodes(r, uint3(i, 0, 0));
  for (uint32_t i = 0; i < r.numInner; ++i) SplitNodes(r, uint3(i, 0, 0));
  for (uint32_t i = 0; i < n; ++i) {
    if (kind == 0) BuildTriangleHierarchy(r, uint3(i, 0, 0));
    else if (kind == 2) BuildEdgeHierarchy(r, uint3(i, 0, 0));
    else BuildPointHierarchy(r, uint3(i, 0, 0));
  }
}

extern "C" uint32_t ref_hilbert3d(uint32_t x, uint32_t y, uint32_t z) {
  bitmask_t c[3] = {x, y, z};
  return (uint32_t)hilbert_c2i(3, 10, c);
}

extern "C" uint32_t ref_hilbert_encode3d(float x, float y, float z) { return hilbert_encode3D(x, y, z); }
