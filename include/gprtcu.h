/*
 * gprtcu.h -- C ABI of the B200 (sm_100a) acceleration-structure path.
 *
 * Plain pointers and sizes only.  Every device pointer is caller-owned and
 * every entry point is stream-ordered and asynchronous: it enqueues work on
 * `stream` and returns.  No entry point allocates device memory; work space
 * is passed in as `scratch` of at least the size the matching *ScratchSize()
 * query returns (256-byte aligned).  Errors detected on the host return
 * immediately; errors detected on the device (a look-back wait that ran out
 * of its iteration budget) are recorded in the scratch header and read with
 * gprtcuScratchStatus().
 *
 * Each entry point names the reference interface it replaces.  The reference
 * is GPRT (gprt/gprt_host.h), whose sort/scan calls take GPRTBuffer objects;
 * include/gprt_compat.h keeps those exact signatures on top of this ABI.
 */
#ifndef GPRTCU_H
#define GPRTCU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define GPRTCU_API __declspec(dllexport)
#else
#define GPRTCU_API __attribute__((visibility("default")))
#endif

typedef struct CUstream_st *gprtcuStream; /* a cudaStream_t; NULL = legacy default stream */

typedef enum {
  GPRTCU_OK = 0,
  GPRTCU_ERR_INVALID_ARG = 1,     /* null pointer, bad width, bad bit range, misaligned */
  GPRTCU_ERR_SIZE_MISMATCH = 2,   /* keys/values size differ (gprt/gprt.cpp:8830-8835) */
  GPRTCU_ERR_SCRATCH_TOO_SMALL = 3,
  GPRTCU_ERR_TIMEOUT = 4,         /* a device-side wait exceeded its iteration budget */
  GPRTCU_ERR_CUDA = 5,            /* a CUDA runtime call failed */
  GPRTCU_ERR_TOO_LARGE = 6        /* n beyond the documented maximum */
} gprtcuStatus;

/* Human-readable name of a status code. */
GPRTCU_API const char *gprtcuStatusString(int status);
/* Library version, major*10000 + minor*100 + patch. */
GPRTCU_API int gprtcuVersion(void);

/* Reads the device-side status word of a scratch buffer after the work that
 * used it has completed on `stream` (synchronises `stream`).  A NULL scratch
 * reads the status of the last gprtcuExclusiveSumU32NoAlloc call on the
 * current device (its fixed array's header). */
GPRTCU_API gprtcuStatus gprtcuScratchStatus(const void *scratch, gprtcuStream stream, int *deviceStatus);

/* ------------------------------------------------------------------------
 * Scan.  Replaces gprtBufferExclusiveSum (gprt/gprt_host.h:2246; host stub
 * gprt/gprt.cpp:8739-8806, intended kernel gprt/gprt_scan.slang:105-401).
 * uint32 wraparound arithmetic; in may equal out.  The total (sum of all
 * inputs mod 2^32) is written to *d_total (device pointer, may be NULL).
 * Unlike the reference there is no 2^30 cap on the aggregate
 * (gprt/gprt_host.h:2231): status words are 64-bit.
 * Maximum n: 2^40 elements.
 * ------------------------------------------------------------------------ */
GPRTCU_API size_t gprtcuScanScratchSize(uint64_t n);
GPRTCU_API gprtcuStatus gprtcuExclusiveSumU32(const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *d_total,
                                              void *scratch, size_t scratchBytes, gprtcuStream stream);
GPRTCU_API gprtcuStatus gprtcuInclusiveSumU32(const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *d_total,
                                              void *scratch, size_t scratchBytes, gprtcuStream stream);

/* Exclusive sum that allocates nothing and takes no scratch argument.  No
 * counterpart in the reference: it is for callers that cannot allocate device
 * work space -- a host application that owns the whole device-memory budget
 * and lends this library only the input and output buffers, or a foreign-
 * language binding that cannot keep a device allocation alive between calls.
 * Same results as gprtcuExclusiveSumU32.  The look-back state lives in a
 * fixed 262,400-byte array inside the library (held on every GPU that loads
 * it until the process exits), so n is limited to 2^28 elements; larger n
 * returns GPRTCU_ERR_TOO_LARGE.  The first call on a device resolves the
 * array's device address (make it before any stream capture on that device).
 * All calls share the array: calls ordered on one stream are fine, calls that
 * overlap on the GPU race and give wrong results.  A device-side timeout is
 * read with gprtcuScratchStatus(NULL, stream, &status) after the call's work
 * is done; the next call clears it. */
GPRTCU_API gprtcuStatus gprtcuExclusiveSumU32NoAlloc(const uint32_t *in, uint32_t *out, uint64_t n,
                                                     uint32_t *d_total, gprtcuStream stream);

/* Partition / select by sign.  Replaces gprtBufferPartition
 * (gprt/gprt_host.h:2295) and gprtBufferSelect (:2344); kernel modes
 * gprt/gprt_scan.slang:118-133,270-283.  Selected items (sign bit clear when
 * selectPositive, set otherwise) are compacted to the front of out in input
 * order; partition writes the rest to the back in reverse input order.
 * *d_count receives the number selected.  in and out must not alias.
 * Maximum n: 2^32 - 1 (the count is a uint32, as the reference returns). */
GPRTCU_API gprtcuStatus gprtcuPartitionI32(const int32_t *in, int32_t *out, uint64_t n, int selectPositive,
                                           uint32_t *d_count, void *scratch, size_t scratchBytes,
                                           gprtcuStream stream);
GPRTCU_API gprtcuStatus gprtcuSelectI32(const int32_t *in, int32_t *out, uint64_t n, int selectPositive,
                                        uint32_t *d_count, void *scratch, size_t scratchBytes, gprtcuStream stream);

/* ------------------------------------------------------------------------
 * Radix sort.  Replaces gprtBufferSort (gprt/gprt_host.h:2384) and
 * gprtBufferSortPayload (gprt/gprt_host.h:2416); host driver
 * gprt/gprt.cpp:8821-9073, kernels gprt/gprt_sort.slang:109-637.
 * Stable ascending sort by the key bits [beginBit, endBit), in place: the
 * result is in `keys` (and `values`) when the work completes, as in the
 * reference.  The reference sorts 64-bit keys with 64-bit payloads over all
 * 64 bits (gprt/gprt.cpp:8837,8966-8969); the 32-bit forms are what its
 * typed shims and tests/t02-bufferSort use.  Key widths 4/8 bytes, payload
 * widths 0/4/8 bytes (a 32-bit key may carry the reference's 64-bit payload,
 * gprt/gprt_sort.slang:29-36).  Maximum n: 2^32 - 1, the reference's uint32
 * key count (gprt/gprt.cpp:8837); from 2^30 keys on, the shape must have
 * 8-bit digits and tiles of at least 4096 keys (the defaults do), else
 * GPRTCU_ERR_TOO_LARGE.
 * ------------------------------------------------------------------------ */
GPRTCU_API size_t gprtcuSortScratchSize(uint64_t n, int keyBytes, int valueBytes);
GPRTCU_API gprtcuStatus gprtcuSortKeysU32(uint32_t *keys, uint64_t n, int beginBit, int endBit, void *scratch,
                                          size_t scratchBytes, gprtcuStream stream);
GPRTCU_API gprtcuStatus gprtcuSortPairsU32(uint32_t *keys, uint32_t *values, uint64_t n, int beginBit, int endBit,
                                           void *scratch, size_t scratchBytes, gprtcuStream stream);
GPRTCU_API gprtcuStatus gprtcuSortKeysU64(uint64_t *keys, uint64_t n, int beginBit, int endBit, void *scratch,
                                          size_t scratchBytes, gprtcuStream stream);
GPRTCU_API gprtcuStatus gprtcuSortPairsU64(uint64_t *keys, uint32_t *values, uint64_t n, int beginBit, int endBit,
                                           void *scratch, size_t scratchBytes, gprtcuStream stream);
GPRTCU_API gprtcuStatus gprtcuSortPairsU32U64(uint32_t *keys, uint64_t *values, uint64_t n, int beginBit, int endBit,
                                              void *scratch, size_t scratchBytes, gprtcuStream stream);
GPRTCU_API gprtcuStatus gprtcuSortPairsU64U64(uint64_t *keys, uint64_t *values, uint64_t n, int beginBit, int endBit,
                                              void *scratch, size_t scratchBytes, gprtcuStream stream);

/* Sort shapes and the autotuner (no counterpart in the reference, whose
 * FidelityFX sort is fixed at 4-bit digits and 256-thread groups).  A shape is
 * the digit width (4, 6 or 8 bits), the keys per tile (1024 .. 8192, one
 * thread block per tile) and the warps per block (4, 8 or 16); the grid holds
 * the power-of-two tiles with 1..32 keys per thread and at least one thread
 * per digit, and 6144-key tiles of 8 warps at 8-bit digits.  Each key/payload type pair has an active shape, used by the entry
 * points above (and by the LBVH builds, which sort u32/u32 or u64/u32 pairs):
 * the one installed by gprtcuSortSetConfig or gprtcuSortAutotune, else a
 * built-in default that depends on n (gprtcuSortGetConfig reports the default
 * for large n).  gprtcuSortScratchSize covers every shape, so a scratch
 * buffer stays valid when the active shape changes. */
typedef struct {
  int32_t digitBits;
  int32_t tile;
  int32_t warps;
} gprtcuSortConfig;
GPRTCU_API int gprtcuSortConfigCount(void);
GPRTCU_API gprtcuStatus gprtcuSortConfigAt(int index, gprtcuSortConfig *cfg);
GPRTCU_API gprtcuStatus gprtcuSortGetConfig(int keyBytes, int valueBytes, gprtcuSortConfig *cfg);
/* cfg = NULL restores the built-in default shape. */
GPRTCU_API gprtcuStatus gprtcuSortSetConfig(int keyBytes, int valueBytes, const gprtcuSortConfig *cfg);
/* One sort with an explicit shape (keys/values as in the typed entries). */
GPRTCU_API gprtcuStatus gprtcuSortWithConfig(void *keys, void *values, uint64_t n, int keyBytes, int valueBytes,
                                             int beginBit, int endBit, const gprtcuSortConfig *cfg, void *scratch,
                                             size_t scratchBytes, gprtcuStream stream);
/* Times every shape on n keys of [0, 2^endBit) -- a copy of sampleKeys (device
 * pointer, n keys) when given, else uniform keys from a fixed seed -- with one
 * untimed and `repeats` timed runs each (CUDA events on `stream`), installs
 * the fastest by median as the active shape for the type pair and returns it
 * in *best.  msPerConfig (optional, gprtcuSortConfigCount() floats) receives
 * each shape's median, -1 for a shape that failed.  Setup-time call: it
 * allocates and frees its own device buffers and synchronizes. */
GPRTCU_API gprtcuStatus gprtcuSortAutotune(int keyBytes, int valueBytes, uint64_t n, int endBit,
                                           const void *sampleKeys, int repeats, float *msPerConfig,
                                           gprtcuSortConfig *best, gprtcuStream stream);

/* ------------------------------------------------------------------------
 * LBVH build.  Replaces gprtTriangleLBVHCreate / gprtPointsLBVHCreate +
 * gprtLBVHBuild (gprt/development/gprt_lbvh.h:91-195; kernels
 * gprt/development/gprt_lbvh.hlsl:188-428).  The caller owns every array of
 * gprtcuLbvh; the build fills them (numPrims is set by the build):
 *   codes       uint32[n]           sorted 30-bit codes
 *   ids         uint32[n]           primitive id of leaf i (sorted order)
 *   nodes       int32[2n-1][4]      {left,right,parent,leaf}; inner nodes
 *                                   [0,n-1) with root 0, leaves [n-1,2n-1)
 *   aabbs       float[2n-1][6]      {min.xyz,max.xyz} per node     (optional)
 *   sceneBounds float[6]            scene box the codes were made in (opt.)
 *   rootBox     float[6]            box of node 0                   (opt.)
 *   bvh2        64 B x max(n-1,1)   traversal nodes: both child boxes and
 *                                   child refs (needed by the traces)
 *   leafTris    float[n][12]        leaf-order triangle vertices, w of the
 *                                   first float4 = primitive id bits (needed
 *                                   by the traces; triangles only)
 * nodes, codes, ids and aabbs are bit-identical to the reference programs'
 * output.  Either aabbs or bvh2 must be given.  codeKind: 0 Morton30
 * (gprt/development/gprt_lbvh.hlsl:25-38), 1 Hilbert30 (gprt/hilbert.h:179-235).
 * positions are float[3] per vertex (12-byte stride), triangles uint32[3].
 * Maximum n: 2^30 - 1.
 * ------------------------------------------------------------------------ */
typedef struct {
  uint32_t numPrims;
  uint32_t *codes;
  uint32_t *ids;
  int32_t *nodes;
  float *aabbs;
  float *sceneBounds;
  float *rootBox;
  void *bvh2;
  void *leafTris;
} gprtcuLbvh;

GPRTCU_API size_t gprtcuLbvhScratchSize(uint32_t n);
GPRTCU_API gprtcuStatus gprtcuLbvhBuildTriangles(const float *positions, const uint32_t *triangles,
                                                 uint32_t numTriangles, int codeKind, gprtcuLbvh *bvh, void *scratch,
                                                 size_t scratchBytes, gprtcuStream stream);
GPRTCU_API gprtcuStatus gprtcuLbvhBuildPoints(const float *positions, uint32_t numPoints, int codeKind,
                                              gprtcuLbvh *bvh, void *scratch, size_t scratchBytes,
                                              gprtcuStream stream);
/* Edge (segment) LBVH: edges uint32[n][2] index positions float[][3].  The
 * reference's build supports edges (GPRT_LBVH_EDGES; ComputeEdgeBounds,
 * ComputeEdgeMortonCodes, BuildEdgeHierarchy, gprt/development/
 * gprt_lbvh.hlsl:112-136,202-260,370-398; dispatched by gprtLBVHBuild,
 * gprt/development/gprt_lbvh.h:184-186) though its header has no create call
 * for them.  Centroid (p1 + p2) / 2.  Fills codes, ids, nodes, aabbs and
 * sceneBounds (the traversal layout is for triangles only). */
GPRTCU_API gprtcuStatus gprtcuLbvhBuildEdges(const float *positions, const uint32_t *edges, uint32_t numEdges,
                                             int codeKind, gprtcuLbvh *bvh, void *scratch, size_t scratchBytes,
                                             gprtcuStream stream);
/* Refit-only update of a triangle LBVH after its vertices moved (the
 * semantics of gprtAccelUpdate, gprt/gprt_host.h:1508-1529): topology and leaf
 * order are kept; leaf-order triangles, traversal-node boxes, reference-layout
 * boxes and rootBox are recomputed bottom-up.  triOffsets/numMeshes as for
 * gprtcuBatchBuildTriangles (NULL/1 for one mesh).  Scratch: the size of the
 * build's (gprtcuLbvhScratchSize / gprtcuBatchScratchSize). */
GPRTCU_API gprtcuStatus gprtcuLbvhRefitTriangles(const float *positions, const uint32_t *triangles,
                                                 const uint32_t *triOffsets, uint32_t numMeshes, gprtcuLbvh *bvh,
                                                 void *scratch, size_t scratchBytes, gprtcuStream stream);

/* ------------------------------------------------------------------------
 * Trace.  Software replacement for the closest-hit / any-hit semantics of
 * TraceRay (gprt/gprt_builtins.slang:105-124; RayDesc use
 * samples/s2-hitPrograms/s2-0-triangles/deviceCode.slang:52-57), whose
 * reference path is Vulkan hardware ray tracing (gprt/gprt.cpp:9404).
 * rays: float[8] per ray {org.xyz, tmin, dir.xyz, tmax} (32 B, 16-B aligned),
 * 0 <= tmin <= tmax as a Vulkan RayDesc requires (the box tests widen their
 * entry / exit distances for non-negative values; a negative tmin is not
 * supported).
 * hits: {uint32 prim (0xFFFFFFFF = miss), float t} per ray.
 * Closest hit: smallest fp32 watertight distance in [tmin, tmax], ties to the
 * lowest primitive id; the reported t is the plane-equation distance of that
 * triangle in double-float arithmetic, rounded once to fp32.
 * Any hit: some triangle hit in [tmin, tmax] (prim) or a miss.
 * ------------------------------------------------------------------------ */
typedef struct {
  uint32_t prim;
  float t;
} gprtcuHit;

/* scratch: at least gprtcuTraceScratchSize() bytes (the ray work counter and
 * the status word; a stack overflow -- impossible for trees of depth <= 64,
 * which 30-bit codes plus the index tie-break guarantee -- sets status 5). */
GPRTCU_API size_t gprtcuTraceScratchSize(void);
GPRTCU_API gprtcuStatus gprtcuTraceClosest(const gprtcuLbvh *bvh, const float *rays, uint64_t numRays,
                                           gprtcuHit *hits, void *scratch, size_t scratchBytes, gprtcuStream stream);
GPRTCU_API gprtcuStatus gprtcuTraceAny(const gprtcuLbvh *bvh, const float *rays, uint64_t numRays, gprtcuHit *hits,
                                       void *scratch, size_t scratchBytes, gprtcuStream stream);

/* ------------------------------------------------------------------------
 * Spheres and linearly swept spheres (LSS) as software-BVH primitives.  The
 * reference builds hardware AABB structures over the boxes of its
 * SphereBounds / LSSBounds programs and intersects with intersectRayLSS
 * (gprt/gprt_fallbacks.slang:45-144,168-283; gprtSphereAccelCreate /
 * gprtLSSAccelCreate, gprt/gprt_host.h).  Here: the same bounds, an LBVH over
 * them (gprtcuLbvhBuildBoxes: codes of the box centres, then as for
 * triangles; fills codes, ids, nodes, aabbs, sceneBounds, rootBox and the
 * bvh2 traversal nodes; leafTris unused), and a traversal that runs the same
 * intersection at the leaves.  Spheres: float4 {center, radius}.  LSS:
 * vertices float4 {position, radius}, indices uint32[n][2], end caps on or off
 * for the whole set.  exitTest reports the exit point instead of the entry.
 * Hits: {primitive index, t}; hitU (optional, one float per ray) receives the
 * curve parameter u (0 for spheres).  Closest hit: smallest t in the ray's
 * (tmin, tmax), ties to the lowest index.  Results are bit-identical to the
 * reference's intersectRayLSS / computeLssAabb compiled for the host.
 * ------------------------------------------------------------------------ */
GPRTCU_API gprtcuStatus gprtcuSphereBounds(const float *spheres, uint32_t n, float *aabbs, gprtcuStream stream);
GPRTCU_API gprtcuStatus gprtcuLssBounds(const float *vertices, const uint32_t *indices, uint32_t n, int endcap0,
                                        int endcap1, float *aabbs, gprtcuStream stream);
GPRTCU_API gprtcuStatus gprtcuLbvhBuildBoxes(const float *aabbs, uint32_t numBoxes, int codeKind, gprtcuLbvh *bvh,
                                             void *scratch, size_t scratchBytes, gprtcuStream stream);
GPRTCU_API gprtcuStatus gprtcuTraceSpheres(const gprtcuLbvh *bvh, const float *spheres, const float *rays,
                                           uint64_t numRays, int anyHit, int exitTest, gprtcuHit *hits, float *hitU,
                                           void *scratch, size_t scratchBytes, gprtcuStream stream);
GPRTCU_API gprtcuStatus gprtcuTraceLss(const gprtcuLbvh *bvh, const float *vertices, const uint32_t *indices,
                                       int endcap0, int endcap1, const float *rays, uint64_t numRays, int anyHit,
                                       int exitTest, gprtcuHit *hits, float *hitU, void *scratch, size_t scratchBytes,
                                       gprtcuStream stream);

/* ------------------------------------------------------------------------
 * Solid cells (volume-mesh elements) as software-BVH primitives, with point
 * location.  Replaces gprtSolidsSetVertices / SetIndices / SetTypes +
 * gprtSolidAccelCreate (gprt/gprt_host.h:552-579,1393) and TracePoint over
 * that structure (gprt/gprt_builtins.slang:80-90), whose box and point test
 * are SolidBounds and SolidIntersection (gprt/gprt_fallbacks.slang:467-566).
 * Cell types are the reference's GPRTSolidTypes (gprt/gprt_host.h:291-298):
 * 10 tetrahedron (4 vertices), 14 pyramid (5), 13 wedge (6), 12 hexahedron
 * (8), 23 tetrahedral pair (8 vertices, evaluated as a trilinear cell and
 * reported with the tetrahedron kind, as the reference does); any other code
 * is a cell with no vertices that holds no point.  Vertices are float4
 * {x, y, z, density}; each cell has up to eight uint32 vertex indices (unused
 * slots are ignored); strides are in bytes (0 selects the reference's
 * defaults: 16, 32 and 1).  The reference's buffer offsets are applied by
 * advancing the pointers.
 *   gprtcuSolidBounds: aabbs (optional) receives two float4 per cell in the
 *     reference's layout {lo.xyz, hi.x}, {hi.yz, density min, density max};
 *     boxes (optional) float[6] {lo.xyz, hi.xyz} per cell, the input of
 *     gprtcuLbvhBuildBoxes.  (The reference's program stores the last
 *     vertex's density in both density words; these are the minimum and
 *     maximum its layout documents.)
 *   gprtcuLocateSolidPoints: for each point (float4, w ignored), the
 *     lowest-numbered cell whose box holds the point (lo <= p <= hi, as a
 *     zero-length ray from the point meets it) and whose Newton inversion
 *     (intersectPointSolid) places it inside the cell; hits {cell, hit kind}
 *     (0xFFFFFFFF and 0 when none), rstw (optional) float4 (r, s, t,
 *     interpolated density) per point, zero when none.  The LBVH must be
 *     built over this set's boxes.  Results are bit-identical to the
 *     reference's SolidBounds / intersectPointSolid compiled for the host.
 * ------------------------------------------------------------------------ */
typedef struct {
  const float *vertices;    /* float4 {x, y, z, density} per vertex */
  const uint32_t *indices;  /* up to 8 vertex indices per cell */
  const uint8_t *types;     /* one cell type per cell */
  uint32_t numCells;
  uint32_t vertexStride;    /* bytes between vertices, a multiple of 16 (0: 16) */
  uint32_t indexStride;     /* bytes between cells' indices, a multiple of 4 (0: 32) */
  uint32_t typeStride;      /* bytes between types (0: 1) */
} gprtcuSolids;

typedef struct {
  uint32_t cell; /* 0xFFFFFFFF: no cell holds the point */
  uint32_t kind; /* hit kind: 10 tetrahedron, 12 hexahedron, 13 wedge, 14 pyramid */
} gprtcuSolidHit;

GPRTCU_API gprtcuStatus gprtcuSolidBounds(const gprtcuSolids *solids, float *aabbs, float *boxes,
                                          gprtcuStream stream);
GPRTCU_API gprtcuStatus gprtcuLocateSolidPoints(const gprtcuLbvh *bvh, const gprtcuSolids *solids,
                                                const float *points, uint64_t numPoints, gprtcuSolidHit *hits,
                                                float *rstw, void *scratch, size_t scratchBytes, gprtcuStream stream);

/* ------------------------------------------------------------------------
 * Two-level instancing.  Replaces gprtInstanceAccelCreate + TraceRay over an
 * instance acceleration structure (gprt/gprt_host.h:1418; instance record
 * gprt::Instance, gprt/gprt_shared.h:92-101) in software: a top-level LBVH
 * over the instances' world boxes, bottom levels = the meshes of a batched
 * LBVH (gprtcuBatchBuildTriangles; triOffsets/numMeshes as there) or of one
 * LBVH (numMeshes = 1).  The record keeps the reference's 64-byte layout;
 * `blas` (accelAddress there) is the mesh index.  geometryIndexAndFlags is
 * not used.
 *   gprtcuInstancesPrepare: per instance, worldToObject float[n][12] (the
 *     inverse transform, computed in double and rounded once) and worldBoxes
 *     float[n][6] (the mesh's rootBox mapped to world space, rounded outward;
 *     empty for a singular transform or a mesh index out of range, so such
 *     instances are never hit).  Build the top level over worldBoxes with
 *     gprtcuLbvhBuildBoxes.
 *   gprtcuTraceInstances: an instance is visible when (mask & rayMask) != 0.
 *     Closest hit: smallest t, ties to the lowest (instance, primitive); hits
 *     report mesh-local primitive ids, hitInstance (optional) the instance
 *     index.  The ray enters an instance as ((w0*x + w1*y) + w2*z) + w3 per
 *     component in float, keeping tmin/tmax (an affine map keeps the ray
 *     parameter); t is refined in that object space. */
typedef struct {
  float transform[12];            /* row-major 3x4 object-to-world */
  uint32_t customIndexAndMask;    /* instanceCustomIndex (bits 0-23) | mask (bits 24-31) */
  uint32_t geometryIndexAndFlags; /* not used */
  uint64_t blas;                  /* mesh index of the bottom-level batch */
} gprtcuInstance;
GPRTCU_API gprtcuStatus gprtcuInstancesPrepare(const gprtcuInstance *instances, uint32_t numInstances,
                                               const float *blasRootBoxes, uint32_t numMeshes, float *worldToObject,
                                               float *worldBoxes, gprtcuStream stream);
GPRTCU_API gprtcuStatus gprtcuTraceInstances(const gprtcuLbvh *tlas, const gprtcuInstance *instances,
                                             const float *worldToObject, const gprtcuLbvh *blas,
                                             const uint32_t *triOffsets, uint32_t numMeshes, const float *rays,
                                             uint64_t numRays, uint32_t rayMask, int anyHit, gprtcuHit *hits,
                                             uint32_t *hitInstance, void *scratch, size_t scratchBytes,
                                             gprtcuStream stream);

/* ------------------------------------------------------------------------
 * Batched build and trace: many meshes in one set of launches.  No
 * counterpart in the reference beyond repeated gprtLBVHBuild calls
 * (gprt/development/gprt_lbvh.h:170-195), one per mesh.
 * Meshes are consecutive triangle ranges: triOffsets (device, uint32
 * [numMeshes+1], exclusive prefix of the triangle counts, every mesh >= 1
 * triangle); `triangles` hold global vertex indices into `positions`.
 * Output arrays are the per-mesh LBVHs concatenated, each mesh's block
 * bit-identical to gprtcuLbvhBuildTriangles on that mesh alone:
 *   codes, ids (mesh-local ids), leafTris    at b = triOffsets[m]
 *   nodes, aabbs (2 n_m - 1 nodes each)       at 2b - m
 *   bvh2 (n_m - 1 nodes each)                 at b - m
 *   sceneBounds, rootBox                      float[numMeshes][6]
 * The segmented sort runs on 64-bit keys (meshID << 32 | code).
 * Trace: rays [rayOffsets[m], rayOffsets[m+1]) are traced against mesh m
 * (rayOffsets device uint32[numMeshes+1]); hits carry mesh-local ids.
 * ------------------------------------------------------------------------ */
GPRTCU_API size_t gprtcuBatchScratchSize(uint32_t numMeshes, uint32_t totalTriangles);
GPRTCU_API gprtcuStatus gprtcuBatchBuildTriangles(const float *positions, const uint32_t *triangles,
                                                  const uint32_t *triOffsets, uint32_t numMeshes,
                                                  uint32_t totalTriangles, int codeKind, gprtcuLbvh *bvh,
                                                  void *scratch, size_t scratchBytes, gprtcuStream stream);
GPRTCU_API gprtcuStatus gprtcuBatchTrace(const gprtcuLbvh *bvh, const uint32_t *triOffsets,
                                         const uint32_t *rayOffsets, uint32_t numMeshes, const float *rays,
                                         uint64_t numRays, int anyHit, gprtcuHit *hits, void *scratch,
                                         size_t scratchBytes, gprtcuStream stream);

/* ------------------------------------------------------------------------
 * 8-wide quantised BVH.  No counterpart in the reference.  Collapsed from a
 * binary LBVH (plain or batched, which needs bvh2 and leafTris): every node
 * has up to 8 children whose boxes are stored as uint8 per axis against an
 * fp32 origin and a power-of-two scale per axis (computed in FP64, floor /
 * ceil rounding), so the decoded boxes always contain the exact ones; leaf
 * triangles are copied into leaf order of the wide tree.  Traversal returns
 * the same hits as gprtcuTraceClosest / gprtcuBatchTrace.
 *   nodes     80 B x capacity (capacity >= total triangles)
 *   leafTris  float[total][12]
 *   roots     uint32[numMeshes]: root node of each mesh
 *   numNodes  optional device uint32: node count written by the build
 * triOffsets / rayOffsets: NULL (one mesh) or device uint32[numMeshes+1].
 * ------------------------------------------------------------------------ */
typedef struct {
  void *nodes;
  float *leafTris;
  uint32_t *roots;
  uint32_t *numNodes;
  uint32_t capacity;
} gprtcuWideBvh;

GPRTCU_API size_t gprtcuWideScratchSize(uint32_t numMeshes, uint32_t totalTriangles);
GPRTCU_API gprtcuStatus gprtcuWideBuild(const gprtcuLbvh *binary, const uint32_t *triOffsets, uint32_t numMeshes,
                                        gprtcuWideBvh *out, void *scratch, size_t scratchBytes, gprtcuStream stream);
GPRTCU_API gprtcuStatus gprtcuWideTrace(const gprtcuWideBvh *bvh, const uint32_t *rayOffsets, uint32_t numMeshes,
                                        const float *rays, uint64_t numRays, int anyHit, gprtcuHit *hits,
                                        void *scratch, size_t scratchBytes, gprtcuStream stream);

/* ------------------------------------------------------------------------
 * Seeded synthetic scenes on the device (benchmark and test inputs; no
 * counterpart in the reference, which has no benchmark inputs).
 * gprtcuGenSoup: n triangles; mesh m (triOffsets NULL = one mesh) inside the
 *   unit cube at offset (m mod 16, m/16 mod 16, m/256) * spacing; centroid
 *   uniform, vertices centroid + N(0, sigma^2); indices (3i, 3i+1, 3i+2).
 * gprtcuGenMixture: n triangles of a `clusters`-component Gaussian mixture
 *   (centres uniform in [0,1]^3, sigma uniform in [0.005, 0.05], equal
 *   weights, consecutive triangles in the same cluster), vertices centroid
 *   + N(0, edgeSigma^2).
 * gprtcuGenRays: rays per mesh box (meshBoxes float[numMeshes][6], NULL =
 *   the unit cube): origin uniform on the sphere of radius 2 * largest extent
 *   about the box centre, unit direction towards a uniform point in the box,
 *   tmin 0, tmax +inf.
 * ------------------------------------------------------------------------ */
GPRTCU_API gprtcuStatus gprtcuGenSoup(uint64_t n, uint64_t seed, float sigma, const uint32_t *triOffsets,
                                      uint32_t numMeshes, float spacing, float *positions, uint32_t *triangles,
                                      gprtcuStream stream);
GPRTCU_API gprtcuStatus gprtcuGenMixture(uint64_t n, uint32_t clusters, uint64_t seed, float edgeSigma,
                                         float *positions, uint32_t *triangles, gprtcuStream stream);
GPRTCU_API gprtcuStatus gprtcuGenRays(uint64_t numRays, uint64_t seed, const uint32_t *rayOffsets, uint32_t numMeshes,
                                      const float *meshBoxes, float *rays, gprtcuStream stream);

/* ------------------------------------------------------------------------
 * Test hooks (fault injection without a GPU fault).  Process-wide settings
 * read at launch time by the kernels that wait.  No counterpart in the
 * reference, whose waits happen inside the Vulkan driver.
 * gprtcuDebugSetSpinBudget: polls a look-back wait (scan, sort) or a refit's
 *   wait for its sibling makes before it records GPRTCU_ERR_TIMEOUT (0
 *   restores the default, 2^22); the mbarrier waits of the TMA-staged kernels
 *   get 16 polls for each of these.  The refit's budget is set on the current
 *   device.
 * gprtcuDebugScanSkipTile: the scan tile with this ticket never publishes its
 *   status (-1 disables), so its successors run out of budget and return.
 * gprtcuDebugScanSkipStage: in the persistent scan / partition kernel, the
 *   tile with this ticket publishes its prefix but its scan stage is never
 *   filled, so the scanner warps' wait runs out and they stop together
 *   (-1 disables).
 * gprtcuDebugSortSkipTile: in every pass of a sort, the tile with this ticket
 *   never publishes its digit counts (-1 disables); later passes see the
 *   recorded error and do nothing.
 * gprtcuDebugRefitSkipLeaf: the leaf in this sorted slot never stores its box
 *   in its parent's traversal node, so the parent's second arrival runs out of
 *   budget (-1 disables; set on the current device).
 * ------------------------------------------------------------------------ */
GPRTCU_API void gprtcuDebugSetSpinBudget(uint32_t polls);
GPRTCU_API void gprtcuDebugScanSkipTile(int64_t tile);
GPRTCU_API void gprtcuDebugScanSkipStage(int64_t tile);
GPRTCU_API void gprtcuDebugSortSkipTile(int64_t tile);
/* Kernel of the 8-bit sort passes, for tests and measurements: 0 (default)
 * the trimmed pass ranking by per-warp leader tables and five votes, 1 the
 * original pass, 2-5 the trimmed pass ranking by shared-memory OR words,
 * match.any, eight plain votes, eight predicated votes.  All give the same
 * bits. */
GPRTCU_API void gprtcuDebugSortRanking(int mode);
/* L2 prefetch distance of the 8-bit sort passes, in quarters of a resident
 * wave of CTAs (SMs x CTAs per SM): each CTA fetches into L2 the keys and
 * payloads of the tile that many tickets after its own.  Default 2; 0
 * turns it off; clamped to 0..64.  A cache hint only: results are the same
 * bits. */
GPRTCU_API void gprtcuDebugSortPrefetch(int quarterWaves);
GPRTCU_API gprtcuStatus gprtcuDebugRefitSkipLeaf(int64_t slot);
/* Scan kernel selection for tests: 0 = automatic (default: the persistent
 * re-read kernel for n >= 2^20 and the TMA-staged tile-per-CTA kernel below,
 * when in/out are 16-byte aligned; else the register-staged kernel),
 * 1 = register-staged tile per CTA, 2 = TMA-staged tile per CTA,
 * 3 = persistent re-read kernel (2 and 3 need 16-byte aligned in/out). */
GPRTCU_API void gprtcuDebugScanImpl(int impl);

#ifdef __cplusplus
}
#endif
#endif
