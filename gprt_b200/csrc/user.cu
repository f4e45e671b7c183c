// user.cu -- spheres and linearly swept spheres (LSS) as software-BVH
// primitives: their bounds, and closest-hit / any-hit traversal of an LBVH
// built over those bounds (gprtcuLbvhBuildBoxes) with the reference's
// ray/LSS intersection at the leaves.
//
// The reference traces these primitives on ray-tracing hardware: an AABB
// acceleration structure over the boxes of its SphereBounds / LSSBounds
// compute programs (gprt/gprt_fallbacks.slang:215-235,263-283), with
// SphereIntersection / LSSIntersection as intersection programs (:146-166,
// 245-261), both calling intersectRayLSS (:45-144).  Here the same arithmetic
// runs in CUDA: every float operation is an explicit round-to-nearest
// intrinsic in the reference's evaluation order (dot(a, b) = (a.x*b.x +
// a.y*b.y) + a.z*b.z, rcp(x) = 1/x), so bounds, t and u are bit-identical to
// the reference's code compiled for the host.
//
// Closest hit: the smallest t in the ray's (tmin, tmax), ties to the lowest
// primitive id (the reference's hardware leaves tie order unspecified); any
// hit: the first hit found.
#include "common.cuh"
#include "lbvh.cuh"
#include "rtmath.cuh"

namespace gprtcu {

struct F3 {
  float x, y, z;
};
__device__ __forceinline__ F3 f3(float x, float y, float z) { return F3{x, y, z}; }
__device__ __forceinline__ F3 add3(F3 a, F3 b) { return f3(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)); }
__device__ __forceinline__ F3 sub3(F3 a, F3 b) { return f3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)); }
__device__ __forceinline__ float dot3(F3 a, F3 b) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}

// intersectRayLSS (gprt/gprt_fallbacks.slang:45-144).
__device__ bool lss_intersect(F3 ro, F3 d, F3 p0, F3 p1, float r0, float r1, bool cap0, bool cap1, float tmin,
                              float tmax, bool exit_test, float &t_out, float &u_out) {
  t_out = 0.0f;
  u_out = 0.0f;
  const F3 mid = f3(__fmul_rn(0.5f, __fadd_rn(p0.x, p1.x)), __fmul_rn(0.5f, __fadd_rn(p0.y, p1.y)),
                    __fmul_rn(0.5f, __fadd_rn(p0.z, p1.z)));
  const float rmid = __fmul_rn(0.5f, __fadd_rn(r0, r1));
  const float dd = dot3(d, d);
  const float inv_dd = __fdiv_rn(1.0f, dd);
  const float align = __fmul_rn(dot3(d, sub3(mid, ro)), inv_dd);
  ro = f3(__fadd_rn(ro.x, __fmul_rn(align, d.x)), __fadd_rn(ro.y, __fmul_rn(align, d.y)),
          __fadd_rn(ro.z, __fmul_rn(align, d.z)));
  const F3 off = sub3(ro, mid);
  const F3 axis = sub3(p1, p0);
  const float rdel = __fsub_rn(r1, r0);
  const float a = dd;
  const float b = dot3(axis, d);
  const float c = __fsub_rn(dot3(axis, axis), __fmul_rn(rdel, rdel));
  const float dq = dot3(d, off);
  const float e = __fadd_rn(dot3(axis, off), __fmul_rn(rmid, rdel));
  const float f = __fsub_rn(dot3(off, off), __fmul_rn(rmid, rmid));
  const float At = __fsub_rn(__fmul_rn(b, b), __fmul_rn(a, c));
  const float Bt = __fsub_rn(__fmul_rn(b, e), __fmul_rn(c, dq));
  const float Ct = __fsub_rn(__fmul_rn(e, e), __fmul_rn(c, f));
  const float disc = __fsub_rn(__fmul_rn(Bt, Bt), __fmul_rn(At, Ct));
  const bool is_sphere = axis.x == 0.0f && axis.y == 0.0f && axis.z == 0.0f && rdel == 0.0f;
  const bool use_start_sphere = !cap1;
  const bool shell_degenerate = (c <= 0.0f) && (rdel != 0.0f);
  const bool invalid = (r0 <= 0.0f && r1 <= 0.0f) || isnan(r0) || isnan(r1) || isnan(p0.x) || isnan(p1.x) ||
                       isinf(r0) || isinf(p0.x);
  if ((!is_sphere && !shell_degenerate && disc < 0.0f) || invalid) return false;
  const float sq = __fsqrt_rn(disc);
  const float inv_at = __fdiv_rn(1.0f, At);
  const float t0 = __fmul_rn(__fadd_rn(-Bt, exit_test ? -sq : sq), inv_at);
  const float inv_c = __fdiv_rn(1.0f, c);
  const float u0 = __fmul_rn(__fadd_rn(__fmul_rn(b, t0), e), inv_c);
  if (fabsf(u0) <= 0.5f && (__fmul_rn(u0, rdel) >= -rmid) && !is_sphere && !shell_degenerate) {
    const float ht = __fadd_rn(t0, align), hu = __fadd_rn(u0, 0.5f);
    if (ht <= tmin || ht >= tmax) return false;
    t_out = ht;
    u_out = hu;
    return true;
  }
  const bool start_cap = is_sphere ? use_start_sphere : (u0 < 0.0f);
  if ((start_cap && !cap0) || (!start_cap && !cap1)) return false;
  const float Bs = __fadd_rn(-dq, __fmul_rn(start_cap ? -b : b, 0.5f));
  const float BsBs = __fmul_rn(Bs, Bs);
  const float Cs = __fsub_rn(__fadd_rn(f, __fmul_rn(0.25f, c)), start_cap ? -e : e);
  const float AsCs = __fmul_rn(a, Cs);
  if (BsBs < AsCs) return false;
  const float sqc = __fsqrt_rn(__fsub_rn(BsBs, AsCs));
  const float cap_t = __fmul_rn(__fsub_rn(Bs, exit_test ? -sqc : sqc), inv_dd);
  t_out = __fadd_rn(cap_t, align);
  u_out = start_cap ? 0.0f : 1.0f;
  if (t_out <= tmin || t_out >= tmax) return false;
  return true;
}

// One end of computeLssAabb: the box of end v (radius r, cap on/off) given
// the other end's data.
__device__ __forceinline__ void lss_end_box(F3 v, float r, bool cap, F3 v0, F3 v1, float r0, float r1, F3 cme, F3 cpe,
                                            F3 &lo, F3 &hi) {
  lo = v;
  hi = v;
  if (r < 0.0f) {
    const float s = __fmul_rn(r, __fdiv_rn(1.0f, __fsub_rn(r1, r0)));
    lo = f3(__fadd_rn(lo.x, __fmul_rn(s, __fsub_rn(v0.x, v1.x))), __fadd_rn(lo.y, __fmul_rn(s, __fsub_rn(v0.y, v1.y))),
            __fadd_rn(lo.z, __fmul_rn(s, __fsub_rn(v0.z, v1.z))));
    hi = lo;
  } else if (cap) {
    lo = f3(__fadd_rn(lo.x, -r), __fadd_rn(lo.y, -r), __fadd_rn(lo.z, -r));
    hi = f3(__fadd_rn(hi.x, r), __fadd_rn(hi.y, r), __fadd_rn(hi.z, r));
  } else {
    lo = f3(__fadd_rn(lo.x, __fmul_rn(r, cme.x)), __fadd_rn(lo.y, __fmul_rn(r, cme.y)), __fadd_rn(lo.z, __fmul_rn(r, cme.z)));
    hi = f3(__fadd_rn(hi.x, __fmul_rn(r, cpe.x)), __fadd_rn(hi.y, __fmul_rn(r, cpe.y)), __fadd_rn(hi.z, __fmul_rn(r, cpe.z)));
  }
}

// computeLssAabb (gprt/gprt_fallbacks.slang:168-213).
__device__ void lss_aabb(F3 v0, float r0, bool cap0, F3 v1, float r1, bool cap1, float *out) {
  F3 cme = f3(0.f, 0.f, 0.f), cpe = f3(0.f, 0.f, 0.f);
  if (!cap0 || !cap1) {
    const float rd = __fsub_rn(r1, r0);
    const F3 n = sub3(v0, v1);
    const F3 nsq = f3(__fmul_rn(n.x, n.x), __fmul_rn(n.y, n.y), __fmul_rn(n.z, n.z));
    const float l2 = __fadd_rn(__fadd_rn(nsq.x, nsq.y), nsq.z);
    const float l2inv = __fdiv_rn(1.0f, l2);
    const F3 X = f3(__fsub_rn(1.f, __fmul_rn(nsq.x, l2inv)), __fsub_rn(1.f, __fmul_rn(nsq.y, l2inv)),
                    __fsub_rn(1.f, __fmul_rn(nsq.z, l2inv)));
    const float Y = __fsub_rn(1.f, __fmul_rn(__fmul_rn(rd, rd), l2inv));
    const F3 e = f3(__fsqrt_rn(fabsf(__fmul_rn(X.x, Y))), __fsqrt_rn(fabsf(__fmul_rn(X.y, Y))),
                    __fsqrt_rn(fabsf(__fmul_rn(X.z, Y))));
    const F3 c = f3(__fmul_rn(__fmul_rn(rd, n.x), l2inv), __fmul_rn(__fmul_rn(rd, n.y), l2inv),
                    __fmul_rn(__fmul_rn(rd, n.z), l2inv));
    cme = sub3(c, e);
    cpe = add3(c, e);
  }
  F3 lo0, hi0, lo1, hi1;
  lss_end_box(v0, r0, cap0, v0, v1, r0, r1, cme, cpe, lo0, hi0);
  lss_end_box(v1, r1, cap1, v0, v1, r0, r1, cme, cpe, lo1, hi1);
  out[0] = fminf(lo0.x, lo1.x);
  out[1] = fminf(lo0.y, lo1.y);
  out[2] = fminf(lo0.z, lo1.z);
  out[3] = fmaxf(hi0.x, hi1.x);
  out[4] = fmaxf(hi0.y, hi1.y);
  out[5] = fmaxf(hi0.z, hi1.z);
}

// SphereBounds (gprt/gprt_fallbacks.slang:263-283).
__global__ void k_sphere_bounds(const float4 *spheres, uint32_t n, float *aabbs) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 s = spheres[i];
    const float r = fmaxf(s.w, 0.0f);
    const float c[3] = {s.x, s.y, s.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      aabbs[6 * (size_t)i + k] = fminf(3.402823466e38f, __fsub_rn(c[k], r));
      aabbs[6 * (size_t)i + 3 + k] = fmaxf(-3.402823466e38f, __fadd_rn(c[k], r));
    }
  }
}

// LSSBounds (gprt/gprt_fallbacks.slang:215-235).
__global__ void k_lss_bounds(const float4 *verts, const uint2 *idx, uint32_t n, int cap0, int cap1, float *aabbs) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint2 e = idx[i];
    const float4 a = verts[e.x], b = verts[e.y];
    lss_aabb(f3(a.x, a.y, a.z), a.w, cap0 != 0, f3(b.x, b.y, b.z), b.w, cap1 != 0, aabbs + 6 * (size_t)i);
  }
}

// Primitive access: a sphere is the LSS with both ends equal and both caps on
// (SphereIntersection, gprt/gprt_fallbacks.slang:245-261).
struct SpherePrims {
  const float4 *spheres;
  __device__ __forceinline__ bool hit(const Ray &R, uint32_t id, bool exit_test, float &t, float &u) const {
    const float4 s = __ldg(spheres + id);
    const F3 c = f3(s.x, s.y, s.z);
    return lss_intersect(f3(R.ox, R.oy, R.oz), f3(R.dx, R.dy, R.dz), c, c, s.w, s.w, true, true, R.tmin, R.tmax,
                         exit_test, t, u);
  }
};
struct LssPrims {
  const float4 *verts;
  const uint2 *idx;
  bool cap0, cap1;
  __device__ __forceinline__ bool hit(const Ray &R, uint32_t id, bool exit_test, float &t, float &u) const {
    const uint2 e = __ldg(idx + id);
    const float4 a = __ldg(verts + e.x), b = __ldg(verts + e.y);
    return lss_intersect(f3(R.ox, R.oy, R.oz), f3(R.dx, R.dy, R.dz), f3(a.x, a.y, a.z), f3(b.x, b.y, b.z), a.w, b.w,
                         cap0, cap1, R.tmin, R.tmax, exit_test, t, u);
  }
};

constexpr int kUserThreads = 128;
constexpr int kUserStack = 64;

// Binary LBVH traversal (the layout of gprtcuLbvh.bvh2) with the primitive
// test at the leaves: leaf slot s holds primitive ids[s].  One lane per ray,
// 32 rays per warp taken from a global counter, warp-uniform visit loop, as
// in the triangle traversal.
template <typename PRIMS, bool ANY>
__global__ void __launch_bounds__(kUserThreads) k_trace_user(const Bvh2Node *bvh, const uint32_t *ids, uint32_t n,
                                                             const float *root_box, PRIMS prims, bool exit_test,
                                                             const float4 *rays, uint64_t nrays, Hit *hits, float *hit_u,
                                                             unsigned long long *counter, uint32_t *err) {
  const int lane = threadIdx.x & 31;
  while (true) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(counter, 32ull);
    base = __shfl_sync(FULL_MASK, base, 0);
    if (base >= nrays) break;
    const uint64_t r = base + lane;
    const bool active = r < nrays;
    Ray R;
    ray_setup(active ? __ldg(rays + 2 * r) : make_float4(0.f, 0.f, 0.f, 1.f),
              active ? __ldg(rays + 2 * r + 1) : make_float4(1.f, 0.f, 0.f, 0.f), R);
    uint32_t best = kMiss;
    float bt = R.tmax, bu = 0.0f;
    auto leaf = [&](uint32_t slot) {
      const uint32_t id = __ldg(ids + slot);
      float t, u;
      if (prims.hit(R, id, exit_test, t, u) && (best == kMiss || t < bt || (t == bt && id < best))) {
        best = id;
        bt = t;
        bu = u;
      }
    };
    bool done = !active;
    int st_node[kUserStack];
    int sp = 0;
    int node = 0;
    if (n == 1 || !active) {
      if (active) {
        float tn;
        if (ray_box(R, root_box[0], root_box[1], root_box[2], root_box[3], root_box[4], root_box[5], bt, tn)) leaf(0);
      }
      done = true;
    }
    while (__any_sync(FULL_MASK, !done)) {
      if (!done) {
        const float4 *np = reinterpret_cast<const float4 *>(bvh + node);
        const float4 f0 = __ldg(np), f1 = __ldg(np + 1), f2 = __ldg(np + 2);
        const int4 rf = __ldg(reinterpret_cast<const int4 *>(np + 3));
        float tn0, tn1;
        bool h0 = ray_box(R, f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, bt, tn0) && tn0 <= bt;
        bool h1 = ray_box(R, f1.z, f1.w, f2.x, f2.y, f2.z, f2.w, bt, tn1) && tn1 <= bt;
        if (h0 && rf.x < 0) {
          leaf((uint32_t)~rf.x);
          h0 = false;
        }
        if (h1 && rf.y < 0) {
          if (tn1 <= bt) leaf((uint32_t)~rf.y);
          h1 = false;
        }
        if (h1 && tn1 > bt) h1 = false;
        if (ANY && best != kMiss) {
          done = true;
        } else if (h0 && h1) {
          const bool first0 = tn0 <= tn1;
          if (sp < kUserStack) {
            st_node[sp++] = first0 ? rf.y : rf.x;
            node = first0 ? rf.x : rf.y;
          } else {
            atomicCAS(err, 0u, 5u);  // traversal stack overflow
            done = true;
          }
        } else if (h0) {
          node = rf.x;
        } else if (h1) {
          node = rf.y;
        } else if (sp > 0) {
          node = st_node[--sp];
        } else {
          done = true;
        }
      }
    }
    if (active) {
      Hit h;
      h.prim = best;
      h.t = best == kMiss ? __int_as_float(0x7f800000) : bt;
      hits[r] = h;
      if (hit_u) hit_u[r] = best == kMiss ? 0.0f : bu;
    }
  }
}

}  // namespace gprtcu

using namespace gprtcu;

namespace {

int user_grid(uint64_t n) {
  const uint64_t g = (n + 255) / 256, cap = (uint64_t)gprtcu_num_sms() * 16;
  return (int)(g < cap ? (g ? g : 1) : cap);
}

template <typename PRIMS>
gprtcuStatus trace_user(const gprtcuLbvh *bvh, PRIMS prims, const float *rays, uint64_t nrays, int any, int exit_test,
                        gprtcuHit *hits, float *u, void *scratch, size_t scratch_bytes, cudaStream_t stream) {
  if (!bvh || (!rays && nrays) || (!hits && nrays)) return GPRTCU_ERR_INVALID_ARG;
  if (nrays == 0) return GPRTCU_OK;
  if (bvh->numPrims == 0 || !bvh->ids || !bvh->rootBox || (bvh->numPrims > 1 && !bvh->bvh2))
    return GPRTCU_ERR_INVALID_ARG;
  if (((uintptr_t)rays & 15) || ((uintptr_t)bvh->bvh2 & 15)) return GPRTCU_ERR_INVALID_ARG;
  if (!scratch || ((uintptr_t)scratch & 255)) return GPRTCU_ERR_INVALID_ARG;
  if (scratch_bytes < sizeof(ScratchHeader)) return GPRTCU_ERR_SCRATCH_TOO_SMALL;
  ScratchHeader *hdr = (ScratchHeader *)scratch;
  unsigned long long *counter = reinterpret_cast<unsigned long long *>(&hdr->ticket[0]);
  GPRTCU_TRY(cudaMemsetAsync(scratch, 0, sizeof(ScratchHeader), stream));
  const int blocks = gprtcu_num_sms() * 8;
  const uint64_t need = (nrays + kUserThreads - 1) / kUserThreads;
  const int grid = (int)(need < (uint64_t)blocks ? need : blocks);
#define GPRTCU_UTRACE(A)                                                                                          \
  k_trace_user<PRIMS, A><<<grid, kUserThreads, 0, stream>>>((const Bvh2Node *)bvh->bvh2, bvh->ids, bvh->numPrims, \
                                                            bvh->rootBox, prims, exit_test != 0,                 \
                                                            (const float4 *)rays, nrays, (Hit *)hits, u, counter,   \
                                                            &hdr->status)
  if (any) GPRTCU_UTRACE(true);
  else GPRTCU_UTRACE(false);
#undef GPRTCU_UTRACE
  GPRTCU_TRY(cudaGetLastError());
  return GPRTCU_OK;
}

}  // namespace

extern "C" GPRTCU_API gprtcuStatus gprtcuSphereBounds(const float *spheres, uint32_t n, float *aabbs,
                                                      gprtcuStream stream) {
  if (n && (!spheres || !aabbs || ((uintptr_t)spheres & 15))) return GPRTCU_ERR_INVALID_ARG;
  if (n == 0) return GPRTCU_OK;
  k_sphere_bounds<<<user_grid(n), 256, 0, (cudaStream_t)stream>>>((const float4 *)spheres, n, aabbs);
  GPRTCU_TRY(cudaGetLastError());
  return GPRTCU_OK;
}

extern "C" GPRTCU_API gprtcuStatus gprtcuLssBounds(const float *vertices, const uint32_t *indices, uint32_t n,
                                                   int endcap0, int endcap1, float *aabbs, gprtcuStream stream) {
  if (n && (!vertices || !indices || !aabbs || ((uintptr_t)vertices & 15) || ((uintptr_t)indices & 7)))
    return GPRTCU_ERR_INVALID_ARG;
  if (n == 0) return GPRTCU_OK;
  k_lss_bounds<<<user_grid(n), 256, 0, (cudaStream_t)stream>>>((const float4 *)vertices, (const uint2 *)indices, n,
                                                               endcap0, endcap1, aabbs);
  GPRTCU_TRY(cudaGetLastError());
  return GPRTCU_OK;
}

extern "C" GPRTCU_API gprtcuStatus gprtcuTraceSpheres(const gprtcuLbvh *bvh, const float *spheres, const float *rays,
                                                      uint64_t numRays, int anyHit, int exitTest, gprtcuHit *hits,
                                                      float *hitU, void *scratch, size_t scratchBytes,
                                                      gprtcuStream stream) {
  if (!spheres || ((uintptr_t)spheres & 15)) return GPRTCU_ERR_INVALID_ARG;
  return trace_user(bvh, SpherePrims{(const float4 *)spheres}, rays, numRays, anyHit, exitTest, hits, hitU, scratch,
                    scratchBytes, (cudaStream_t)stream);
}

extern "C" GPRTCU_API gprtcuStatus gprtcuTraceLss(const gprtcuLbvh *bvh, const float *vertices,
                                                  const uint32_t *indices, int endcap0, int endcap1,
                                                  const float *rays, uint64_t numRays, int anyHit, int exitTest,
                                                  gprtcuHit *hits, float *hitU, void *scratch, size_t scratchBytes,
                                                  gprtcuStream stream) {
  if (!vertices || !indices || ((uintptr_t)vertices & 15) || ((uintptr_t)indices & 7)) return GPRTCU_ERR_INVALID_ARG;
  return trace_user(bvh, LssPrims{(const float4 *)vertices, (const uint2 *)indices, endcap0 != 0, endcap1 != 0}, rays,
                    numRays, anyHit, exitTest, hits, hitU, scratch, scratchBytes, (cudaStream_t)stream);
}
