/*
 * oracle.h -- CPU restatement of GPRT's acceleration-structure path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: the parity tests,
 * the smoke check and the bench's CPU-baseline leg call it to produce the
 * expected results on the host.  It is never linked into, loaded by or called
 * from the product library (gprt_b200/libgprtcu.so), and no product code path
 * may fall back to it.
 *
 * Parity status per function (see the header comment of each):
 *   sort, scan            pinned by the reference tests' own host oracles
 *                         (tests/t02-bufferSort/hostCode.cpp:59,115 std::sort;
 *                          tests/t03-bufferScans/hostCode.cpp:53-58 serial sum)
 *   partition / select    pinned by the known-answer layouts of
 *                         tests/t03-bufferScans/hostCode.cpp:91-241
 *   hilbert30             pinned against gprt/hilbert.h compiled from the
 *                         reference sources (oracle/Makefile, target ref)
 *   morton30, bounds,
 *   karras, refit         pinned against gprt/development/gprt_lbvh.hlsl
 *                         compiled as C++ from the reference sources
 *                         (oracle/Makefile, target ref; golden fixtures in
 *                         tests/golden/ were generated from it)
 *   ray/triangle,
 *   ray/box, traversal,
 *   wide BVH              parity unpinned: the reference has no software
 *                         traversal (it traces through Vulkan ray-tracing
 *                         hardware, gprt/gprt.cpp:9404).  Restated from
 *                         Woop, Benthin, Wald 2013 "Watertight Ray/Triangle
 *                         Intersection" (JCGT 2(1)) and Ize 2013 "Robust BVH
 *                         Ray Traversal" (JCGT 2(2)); FP64 plane-equation t
 *                         as the accuracy reference.
 */
#ifndef GPRT_ORACLE_H
#define GPRT_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- sort ---------------- */
/* Stable ascending sort of keys (width kw = 4 or 8 bytes) carrying an optional
 * payload (vw = 0, 4 or 8 bytes).  Semantics of gprtBufferSort /
 * gprtBufferSortPayload (gprt/gprt.cpp:8821-9073): LSD radix, in place. */
void orc_sort(void *keys, int kw, void *vals, int vw, size_t n);

/* ---------------- scan ---------------- */
/* uint32 prefix sum with wraparound; returns the total (sum of all inputs mod
 * 2^32).  in may equal out.  gprt/gprt_host.h:2229-2246. */
uint32_t orc_scan_u32(const uint32_t *in, uint32_t *out, size_t n, int inclusive);

/* Partition (partition=1) or select (partition=0) of int32 by sign;
 * returns the number selected.  gprt/gprt_scan.slang:84-92,270-300;
 * tests/t03-bufferScans/hostCode.cpp:98-160,172-241. */
uint32_t orc_partition_i32(const int32_t *in, int32_t *out, size_t n, int selectPositive, int partition);

/* ---------------- space-filling codes ---------------- */
uint32_t orc_morton3d(uint32_t x, uint32_t y, uint32_t z);
uint32_t orc_hilbert3d(uint32_t x, uint32_t y, uint32_t z);

/* Scene AABB {minx,miny,minz,maxx,maxy,maxz} of indexed triangles.
 * gprt/development/gprt_lbvh.hlsl:121-129,215-226. */
void orc_tri_bounds(const float *pos, const uint32_t *tri, uint32_t n, float out[6]);
/* Morton30 (kind 0) or Hilbert30 (kind 1) of triangle centroids normalised to
 * bounds; ids[i] = i.  gprt/development/gprt_lbvh.hlsl:139-146,262-277. */
void orc_tri_codes(const float *pos, const uint32_t *tri, uint32_t n, const float bounds[6], int kind,
                   uint32_t *codes, uint32_t *ids);
/* Points (1 float3 per primitive) and edges (uint2 into pos). */
void orc_point_bounds(const float *pos, uint32_t n, float out[6]);
void orc_point_codes(const float *pos, uint32_t n, const float bounds[6], int kind, uint32_t *codes, uint32_t *ids);

/* ---------------- LBVH ---------------- */
/* Karras 2012 binary radix tree over n sorted codes.  nodes is int4[2n-1]
 * {left,right,parent,leaf}; inner [0,n-1) with root 0, leaves [n-1,2n-1).
 * Leaf fields are left at -1 (the refit fills them).
 * gprt/development/gprt_lbvh.hlsl:45-103,279-338. */
void orc_karras(const uint32_t *codes, uint32_t n, int32_t *nodes);
/* Leaf boxes from ids, then inner boxes as the union of the leaves below,
 * starting from +-1e38 exactly as MakeNodes initialises them.
 * aabbs is float[(2n-1)*6] {min.xyz,max.xyz} per node.
 * gprt/development/gprt_lbvh.hlsl:279-285,400-428. */
void orc_refit_tri(const float *pos, const uint32_t *tri, const uint32_t *ids, uint32_t n, int32_t *nodes,
                   float *aabbs);
/* Full build: bounds, codes, stable pair sort, karras, refit. */
void orc_lbvh_build_edges(const float *pos, const uint32_t *edges, uint32_t n, int kind, float scene[6],
                          uint32_t *codes, uint32_t *ids, int32_t *nodes, float *aabbs);
void orc_lbvh_build_tri(const float *pos, const uint32_t *tri, uint32_t n, int kind, float scene[6],
                        uint32_t *codes, uint32_t *ids, int32_t *nodes, float *aabbs);

void orc_lbvh_build_points(const float *pos, uint32_t n, int kind, float scene[6], uint32_t *codes,
                           uint32_t *ids, int32_t *nodes, float *aabbs);

/* ---------------- rays ---------------- */
/* Ray layout: float[8] {org.xyz, tmin, dir.xyz, tmax}.  Hit layout:
 * {uint32 primID (0xFFFFFFFF = miss), float t}. */
typedef struct {
  uint32_t prim;
  float t;
} orc_hit;

/* FP32 watertight test (Woop 2013).  Returns 1 on hit with *t = T/det.  */
int orc_isect_tri32(const float *ray, const float *v0, const float *v1, const float *v2, float *t);
/* Refined hit distance for a known hit: plane-equation t evaluated in
 * double-float (pairs of fp32) arithmetic, rounded once to fp32. */
float orc_refine_t32(const float *ray, const float *v0, const float *v1, const float *v2);
/* FP64 plane-equation t (the accuracy reference). */
double orc_t64(const float *ray, const float *v0, const float *v1, const float *v2);

/* Closest hit by exhaustive test of every triangle (small scenes). */
void orc_trace_brute(const float *pos, const uint32_t *tri, uint32_t n, const float *rays, uint64_t nrays,
                     orc_hit *hits);
/* Closest hit (anyhit=0) or any hit (anyhit=1) through the reference-layout
 * LBVH (nodes + aabbs).  OpenMP over rays.  Hit t is the refined t. */
void orc_trace_lbvh(const float *pos, const uint32_t *tri, uint32_t n, const int32_t *nodes,
                    const float *aabbs, const float *rays, uint64_t nrays, int anyhit, orc_hit *hits);
/* The watertight ray/triangle test in double precision (1 = hit, *t its
 * distance). */
int orc_isect_tri64(const float *ray, const float *v0, const float *v1, const float *v2, double *t);
/* Closest hit through the same tree with the watertight test in double
 * precision (ties to the lowest id): prim[r] and the FP64 t (INFINITY for a
 * miss).  The accuracy reference for hit ids. */
void orc_trace_lbvh64(const float *pos, const uint32_t *tri, uint32_t n, const int32_t *nodes, const float *aabbs,
                      const float *rays, uint64_t nrays, uint32_t *prim, double *t);

/* ---------------- solid cells ---------------- */
/* Vertex count and hit kind of a cell type (gprt/gprt_fallbacks.slang:289-318). */
int orc_solid_vertex_count(uint32_t type);
uint32_t orc_solid_hit_kind(uint32_t type);
/* intersectPointSolid (gprt/gprt_fallbacks.slang:409-464): qw = 8 float4
 * {x, y, z, density}, zero beyond the vertex count n; rstw = (r, s, t,
 * density).  Pinned to the reference's own function compiled from its
 * sources (oracle/_ref). */
int orc_solid_intersect(const float *p, const float *qw, uint32_t n, float *rstw);
/* SolidBounds (gprt/gprt_fallbacks.slang:467-502) with the documented
 * density range; two float4 per cell. */
void orc_solid_bounds(const float *verts, const uint32_t *idx, const uint8_t *types, uint32_t ncells, float *aabbs);
/* Point location by exhaustive search: the lowest-numbered cell whose box
 * and Newton inversion contain the point. */
void orc_solid_locate_brute(const float *verts, const uint32_t *idx, const uint8_t *types, uint32_t ncells,
                            const float *points, uint64_t npts, uint32_t *cell, uint32_t *kind, float *rstw);

/* ---------------- misc ---------------- */
int orc_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
