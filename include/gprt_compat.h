/*
 * gprt_compat.h -- drop-in replacements for GPRT's sort / scan / LBVH calls.
 *
 * Same names, argument meaning and in-place semantics as the reference's host
 * API (gprt/gprt_host.h), backed by CUDA on one B200 and by the kernels behind
 * include/gprtcu.h.  Only the subset this path needs is provided: contexts,
 * buffers (create / map / unmap / resize / pointers), gprtBufferSort,
 * gprtBufferSortPayload, gprtBufferExclusiveSum, gprtBufferPartition,
 * gprtBufferSelect, and the development LBVH helpers.
 *
 * Differences from the reference:
 *  - errors print a message and are recorded (gprtcuCompatLastError), they do
 *    not raise SIGINT (gprt/gprt.cpp:204-251);
 *  - one device per context (the reference also rejects more,
 *    gprt/gprt.cpp:5373-5374);
 *  - the untyped gprtBufferSort / gprtBufferSortPayload sort 64-bit words, as
 *    the reference's implementation does (gprt/gprt.cpp:8837,8966); the typed
 *    GPRTBufferOf<T> forms sort sizeof(T)-byte keys (4 or 8), as its header
 *    and tests/t02-bufferSort intend.
 */
#ifndef GPRT_COMPAT_H
#define GPRT_COMPAT_H

#include <stddef.h>
#include <stdint.h>

#include "gprtcu.h"

#ifdef __cplusplus
#define GPRT_IF_CPP(a) a
extern "C" {
#else
#define GPRT_IF_CPP(a)
#include <stdbool.h>
#endif

/* Opaque handles, as in gprt/gprt_host.h:104-116. */
typedef struct GPRTContext_T *GPRTContext;
typedef struct GPRTBuffer_T *GPRTBuffer;

/* gprt/gprt_host.h:992-995 */
GPRTCU_API GPRTContext gprtContextCreate(int32_t *requestedDeviceIDs GPRT_IF_CPP(= nullptr),
                                         int numDevices GPRT_IF_CPP(= 1));
GPRTCU_API void gprtContextDestroy(GPRTContext context);

/* gprt/gprt_host.h:1899,1946,1995 (size = bytes per element) */
GPRTCU_API GPRTBuffer gprtHostBufferCreate(GPRTContext context, size_t size, size_t count GPRT_IF_CPP(= 1),
                                           const void *init GPRT_IF_CPP(= nullptr),
                                           size_t alignment GPRT_IF_CPP(= 16));
GPRTCU_API GPRTBuffer gprtDeviceBufferCreate(GPRTContext context, size_t size, size_t count GPRT_IF_CPP(= 1),
                                             const void *init GPRT_IF_CPP(= nullptr),
                                             size_t alignment GPRT_IF_CPP(= 16));
GPRTCU_API GPRTBuffer gprtSharedBufferCreate(GPRTContext context, size_t size, size_t count GPRT_IF_CPP(= 1),
                                             const void *init GPRT_IF_CPP(= nullptr),
                                             size_t alignment GPRT_IF_CPP(= 16));
/* gprt/gprt_host.h:2053-2150 */
GPRTCU_API void gprtBufferDestroy(GPRTBuffer buffer);
GPRTCU_API size_t gprtBufferGetSize(GPRTBuffer buffer, int deviceID GPRT_IF_CPP(= 0));
GPRTCU_API void *gprtBufferGetHostPointer(GPRTBuffer buffer, int deviceID GPRT_IF_CPP(= 0));
GPRTCU_API void gprtBufferMap(GPRTBuffer buffer, int deviceID GPRT_IF_CPP(= 0));
GPRTCU_API void gprtBufferUnmap(GPRTBuffer buffer, int deviceID GPRT_IF_CPP(= 0));
GPRTCU_API void *gprtBufferGetDevicePointer(GPRTBuffer buffer, int deviceID GPRT_IF_CPP(= 0));
GPRTCU_API void gprtBufferResize(GPRTContext context, GPRTBuffer buffer, size_t size, size_t count,
                                 bool preserveContents, int deviceID GPRT_IF_CPP(= 0));

/* Scan family (gprt/gprt_host.h:2246,2295,2344).  Synchronous: the total /
 * the number selected is returned.  scratch may be null (temporary work
 * space) or a buffer that is grown when undersized. */
GPRTCU_API uint32_t gprtBufferExclusiveSum(GPRTContext context, GPRTBuffer input, GPRTBuffer output,
                                           GPRTBuffer scratch GPRT_IF_CPP(= 0));
GPRTCU_API uint32_t gprtBufferPartition(GPRTContext context, GPRTBuffer input, bool selectPositive,
                                        GPRTBuffer output, GPRTBuffer scratch GPRT_IF_CPP(= 0));
GPRTCU_API uint32_t gprtBufferSelect(GPRTContext context, GPRTBuffer input, bool selectPositive, GPRTBuffer output,
                                     GPRTBuffer scratch GPRT_IF_CPP(= 0));

/* Sort (gprt/gprt_host.h:2384,2416): stable ascending, in place, 64-bit words. */
GPRTCU_API void gprtBufferSort(GPRTContext context, GPRTBuffer buffer, GPRTBuffer scratch GPRT_IF_CPP(= 0));
GPRTCU_API void gprtBufferSortPayload(GPRTContext context, GPRTBuffer keys, GPRTBuffer values,
                                      GPRTBuffer scratch GPRT_IF_CPP(= 0));

/* Width-explicit sort behind the typed templates below (keyBytes 4/8,
 * valueBytes 0/4/8).  No counterpart name in the reference. */
GPRTCU_API void gprtcuCompatSort(GPRTContext context, GPRTBuffer keys, int keyBytes, GPRTBuffer values,
                                 int valueBytes, GPRTBuffer scratch);
/* Last error recorded by a compat call on this thread (0 = none); reading
 * it clears it. */
GPRTCU_API int gprtcuCompatLastError(void);
/* The stream a context enqueues on (cudaStream_t). */
GPRTCU_API gprtcuStream gprtcuCompatStream(GPRTContext context);

#ifdef __cplusplus
}  /* extern "C" */

/* ---------------- typed C++ forms (gprt/gprt_host.h:118-127,1969,2268-2439) */
template <typename T> struct _GPRTBufferOf;
template <typename T> using GPRTBufferOf = struct _GPRTBufferOf<T> *;

template <typename T>
GPRTBufferOf<T> gprtDeviceBufferCreate(GPRTContext context, size_t count = 1, const T *init = nullptr,
                                       size_t alignment = 16) {
  return (GPRTBufferOf<T>)gprtDeviceBufferCreate(context, sizeof(T), count, init, alignment);
}
template <typename T>
GPRTBufferOf<T> gprtHostBufferCreate(GPRTContext context, size_t count = 1, const T *init = nullptr,
                                     size_t alignment = 16) {
  return (GPRTBufferOf<T>)gprtHostBufferCreate(context, sizeof(T), count, init, alignment);
}
template <typename T>
GPRTBufferOf<T> gprtSharedBufferCreate(GPRTContext context, size_t count = 1, const T *init = nullptr,
                                       size_t alignment = 16) {
  return (GPRTBufferOf<T>)gprtSharedBufferCreate(context, sizeof(T), count, init, alignment);
}
template <typename T> void gprtBufferDestroy(GPRTBufferOf<T> b) { gprtBufferDestroy((GPRTBuffer)b); }
template <typename T> size_t gprtBufferGetSize(GPRTBufferOf<T> b, int d = 0) {
  return gprtBufferGetSize((GPRTBuffer)b, d) / sizeof(T);
}
template <typename T> T *gprtBufferGetHostPointer(GPRTBufferOf<T> b, int d = 0) {
  return (T *)gprtBufferGetHostPointer((GPRTBuffer)b, d);
}
template <typename T> T *gprtBufferGetDevicePointer(GPRTBufferOf<T> b, int d = 0) {
  return (T *)gprtBufferGetDevicePointer((GPRTBuffer)b, d);
}
template <typename T> void gprtBufferMap(GPRTBufferOf<T> b, int d = 0) { gprtBufferMap((GPRTBuffer)b, d); }
template <typename T> void gprtBufferUnmap(GPRTBufferOf<T> b, int d = 0) { gprtBufferUnmap((GPRTBuffer)b, d); }
template <typename T>
void gprtBufferResize(GPRTContext c, GPRTBufferOf<T> b, size_t count, bool preserve, int d = 0) {
  gprtBufferResize(c, (GPRTBuffer)b, sizeof(T), count, preserve, d);
}

template <typename T1, typename T2>
uint32_t gprtBufferExclusiveSum(GPRTContext c, GPRTBufferOf<T1> in, GPRTBufferOf<T1> out,
                                GPRTBufferOf<T2> scratch = 0) {
  return gprtBufferExclusiveSum(c, (GPRTBuffer)in, (GPRTBuffer)out, (GPRTBuffer)scratch);
}
template <typename T1, typename T2>
uint32_t gprtBufferPartition(GPRTContext c, GPRTBufferOf<T1> in, bool selectPositive, GPRTBufferOf<T1> out,
                             GPRTBufferOf<T2> scratch = 0) {
  return gprtBufferPartition(c, (GPRTBuffer)in, selectPositive, (GPRTBuffer)out, (GPRTBuffer)scratch);
}
template <typename T1, typename T2>
uint32_t gprtBufferSelect(GPRTContext c, GPRTBufferOf<T1> in, bool selectPositive, GPRTBufferOf<T1> out,
                          GPRTBufferOf<T2> scratch = 0) {
  return gprtBufferSelect(c, (GPRTBuffer)in, selectPositive, (GPRTBuffer)out, (GPRTBuffer)scratch);
}
template <typename T1, typename T2>
void gprtBufferSort(GPRTContext c, GPRTBufferOf<T1> buffer, GPRTBufferOf<T2> scratch = 0) {
  static_assert(sizeof(T1) == 4 || sizeof(T1) == 8, "keys are 32- or 64-bit");
  gprtcuCompatSort(c, (GPRTBuffer)buffer, (int)sizeof(T1), nullptr, 0, (GPRTBuffer)scratch);
}
template <typename T1, typename T2, typename T3>
void gprtBufferSortPayload(GPRTContext c, GPRTBufferOf<T1> keys, GPRTBufferOf<T2> values,
                           GPRTBufferOf<T3> scratch = 0) {
  static_assert(sizeof(T1) == 4 || sizeof(T1) == 8, "keys are 32- or 64-bit");
  static_assert(sizeof(T2) == 4 || sizeof(T2) == 8, "payloads are 32- or 64-bit");
  gprtcuCompatSort(c, (GPRTBuffer)keys, (int)sizeof(T1), (GPRTBuffer)values, (int)sizeof(T2), (GPRTBuffer)scratch);
}

/* ---------------- development LBVH (gprt/development/gprt_lbvh.h:57-210) --------
 * The reference's record keeps mortonCodes, ids, nodes (int4 {left, right,
 * parent, leaf}) and aabbs (float3 pairs); the same buffers are filled here
 * (bit-identical contents), plus the traversal layout this build adds. */
typedef enum { GPRT_LBVH_POINTS = 1, GPRT_LBVH_EDGES = 2, GPRT_LBVH_TRIANGLES = 4 } GPRTLBVHType;

struct GPRTLBVH {
  GPRTLBVHType type;
  uint32_t numPrims;
  GPRTBuffer positions, triangles;  // borrowed from the caller
  GPRTBufferOf<uint32_t> mortonCodes;
  GPRTBufferOf<uint32_t> ids;
  GPRTBuffer nodes;     // int32[2n-1][4]
  GPRTBuffer aabbs;     // float[2n-1][6]
  GPRTBuffer bvh2;      // traversal nodes (triangles only)
  GPRTBuffer leafTris;  // leaf-order triangles (triangles only)
  GPRTBuffer scratch;
};

inline GPRTLBVH gprtPointsLBVHCreate(GPRTContext context, GPRTBuffer vertices, uint32_t count) {
  GPRTLBVH l{};
  l.type = GPRT_LBVH_POINTS;
  l.numPrims = count;
  l.positions = vertices;
  l.mortonCodes = gprtDeviceBufferCreate<uint32_t>(context, count);
  l.ids = gprtDeviceBufferCreate<uint32_t>(context, count);
  l.nodes = gprtDeviceBufferCreate(context, 16, 2 * (size_t)count - 1);
  l.aabbs = gprtDeviceBufferCreate(context, 24, 2 * (size_t)count - 1);
  l.scratch = gprtDeviceBufferCreate(context, 1, gprtcuLbvhScratchSize(count));
  return l;
}
template <typename TV>
GPRTLBVH gprtPointsLBVHCreate(GPRTContext context, GPRTBufferOf<TV> vertices, uint32_t count) {
  static_assert(sizeof(TV) == 12, "vertices are three floats");
  return gprtPointsLBVHCreate(context, (GPRTBuffer)vertices, count);
}

inline GPRTLBVH gprtTriangleLBVHCreate(GPRTContext context, GPRTBuffer vertices, GPRTBuffer indices,
                                       uint32_t count) {
  GPRTLBVH l = gprtPointsLBVHCreate(context, vertices, count);
  l.type = GPRT_LBVH_TRIANGLES;
  l.triangles = indices;
  l.bvh2 = gprtDeviceBufferCreate(context, 64, count > 1 ? count - 1 : 1);
  l.leafTris = gprtDeviceBufferCreate(context, 48, count);
  return l;
}
template <typename TV, typename TI>
GPRTLBVH gprtTriangleLBVHCreate(GPRTContext context, GPRTBufferOf<TV> vertices, GPRTBufferOf<TI> indices,
                                uint32_t count) {
  static_assert(sizeof(TV) == 12 && sizeof(TI) == 12, "float3 vertices, uint3 indices");
  return gprtTriangleLBVHCreate(context, (GPRTBuffer)vertices, (GPRTBuffer)indices, count);
}

inline gprtcuLbvh gprtLBVHDescriptor(const GPRTLBVH &l) {
  gprtcuLbvh d{};
  d.numPrims = l.numPrims;
  d.codes = gprtBufferGetDevicePointer(l.mortonCodes);
  d.ids = gprtBufferGetDevicePointer(l.ids);
  d.nodes = (int32_t *)gprtBufferGetDevicePointer(l.nodes);
  d.aabbs = (float *)gprtBufferGetDevicePointer(l.aabbs);
  d.bvh2 = l.bvh2 ? gprtBufferGetDevicePointer(l.bvh2) : nullptr;
  d.leafTris = l.leafTris ? gprtBufferGetDevicePointer(l.leafTris) : nullptr;
  return d;
}

/* gprtLBVHBuild (gprt/development/gprt_lbvh.h:170-195); asynchronous on the
 * context's stream, like the reference's compute submissions. */
inline void gprtLBVHBuild(GPRTContext context, GPRTLBVH &l) {
  gprtcuLbvh d = gprtLBVHDescriptor(l);
  void *s = gprtBufferGetDevicePointer(l.scratch);
  size_t sb = gprtBufferGetSize(l.scratch);
  const float *pos = (const float *)gprtBufferGetDevicePointer(l.positions);
  if (l.type == GPRT_LBVH_TRIANGLES)
    gprtcuLbvhBuildTriangles(pos, (const uint32_t *)gprtBufferGetDevicePointer(l.triangles), l.numPrims, 0, &d, s,
                             sb, gprtcuCompatStream(context));
  else
    gprtcuLbvhBuildPoints(pos, l.numPrims, 0, &d, s, sb, gprtcuCompatStream(context));
}

inline void gprtLBVHDestroy(GPRTLBVH &l) {
  gprtBufferDestroy(l.mortonCodes);
  gprtBufferDestroy(l.ids);
  gprtBufferDestroy(l.nodes);
  gprtBufferDestroy(l.aabbs);
  if (l.bvh2) gprtBufferDestroy(l.bvh2);
  if (l.leafTris) gprtBufferDestroy(l.leafTris);
  gprtBufferDestroy(l.scratch);
  l = GPRTLBVH{};
}
#endif /* __cplusplus */

#endif
