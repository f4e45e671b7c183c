// trace.cu -- closest-hit and any-hit traversal of the binary LBVH.
//
// One thread per ray, rays handed out to persistent warps by an atomic
// counter (load balance across rays of very different cost).  Each step
// loads one 64-byte node holding both child boxes, tests both boxes,
// intersects leaf children on the spot (their triangles are stored in leaf
// order), descends into the nearer inner child and pushes the farther one on
// a per-thread stack of node indices.  A child is entered when its entry
// distance does not exceed the best hit (equal distance still enters, so a
// tie can be won by a lower primitive id).
#include "common.cuh"
#include "lbvh.cuh"
#include "rtmath.cuh"

namespace gprtcu {

constexpr int kTraceThreads = 128;
constexpr int kStack = 64;

__device__ __forceinline__ void leaf_test(const float4 *leaf, uint32_t slot, const Ray &R, uint32_t &best,
                                          uint32_t &best_slot, float &bt) {
  const float4 a = __ldg(leaf + 3 * (size_t)slot), b = __ldg(leaf + 3 * (size_t)slot + 1),
               c = __ldg(leaf + 3 * (size_t)slot + 2);
  const float v0[3] = {a.x, a.y, a.z}, v1[3] = {b.x, b.y, b.z}, v2[3] = {c.x, c.y, c.z};
  const uint32_t id = __float_as_uint(a.w);
  float t;
  if (isect_tri(R, v0, v1, v2, t)) {
    if (best == kMiss || t < bt || (t == bt && id < best)) {
      best = id;
      best_slot = slot;
      bt = t;
    }
  }
}

// Batched form: rays [ray_off[m], ray_off[m+1]) go to mesh m, whose
// primitives are [tri_off[m], tri_off[m+1]); its traversal nodes start at
// tri_off[m] - m and its leaves at tri_off[m] (mesh-local references are
// offset on the fly).  Hits report mesh-local primitive ids.
struct TraceMeshes {
  const uint32_t *tri_off;
  const uint32_t *ray_off;
  uint32_t meshes;
};

__device__ __forceinline__ uint32_t mesh_of_ray(const TraceMeshes &tm, uint64_t r) {
  uint32_t lo = 0, hi = tm.meshes;  // ray_off[lo] <= r < ray_off[hi]
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(tm.ray_off + mid) <= r) lo = mid;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ void write_hit(Hit *hits, uint64_t r, const float4 *leaf, const Ray &R, uint32_t best,
                                          uint32_t best_slot) {
  Hit h;
  h.prim = best;
  h.t = __int_as_float(0x7f800000);
  if (best != kMiss) {
    const float4 a = __ldg(leaf + 3 * (size_t)best_slot), b = __ldg(leaf + 3 * (size_t)best_slot + 1),
                 c = __ldg(leaf + 3 * (size_t)best_slot + 2);
    const float v0[3] = {a.x, a.y, a.z}, v1[3] = {b.x, b.y, b.z}, v2[3] = {c.x, c.y, c.z};
    h.t = refine_t(R, v0, v1, v2);
  }
  hits[r] = h;
}

// One mesh: one lane per ray, a warp takes 32 rays at a time from the global
// counter.  The loop over node visits is warp-uniform (a lane that has
// finished idles until the warp's last ray is done), so the lanes re-converge
// at every visit; a loop with per-lane exits lets them drift apart and run
// one at a time.  (Refilling idle lanes, as the batched form does, measured
// slower here: these rays are long -- most of them hit -- and rays that start
// at different times share less of the upper tree in L1.)
template <bool ANY>
__global__ void __launch_bounds__(kTraceThreads) k_trace_bin(const Bvh2Node *bvh, const float4 *leaf, uint32_t n,
                                                            const float4 *rays, uint64_t nrays, Hit *hits,
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
    uint32_t best = kMiss, best_slot = 0;
    float bt = R.tmax;
    bool done = !active;
    int st_node[kStack];  // inner nodes still to visit (4 B each: the hot top stays in L1)
    int sp = 0;
    int node = 0;
    if (n == 1 || !active) {
      if (active) {
        const float4 a = __ldg(leaf), b = __ldg(leaf + 1), c = __ldg(leaf + 2);
        float tn;
        if (ray_box(R, fminf(a.x, fminf(b.x, c.x)), fminf(a.y, fminf(b.y, c.y)), fminf(a.z, fminf(b.z, c.z)),
                    fmaxf(a.x, fmaxf(b.x, c.x)), fmaxf(a.y, fmaxf(b.y, c.y)), fmaxf(a.z, fmaxf(b.z, c.z)), bt, tn) &&
            tn <= bt)
          leaf_test(leaf, 0, R, best, best_slot, bt);
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
          leaf_test(leaf, (uint32_t)~rf.x, R, best, best_slot, bt);
          h0 = false;
        }
        if (h1 && rf.y < 0) {
          if (tn1 <= bt) leaf_test(leaf, (uint32_t)~rf.y, R, best, best_slot, bt);
          h1 = false;
        }
        if (h1 && tn1 > bt) h1 = false;
        if (ANY && best != kMiss) {
          done = true;
        } else if (h0 && h1) {
          const bool first0 = tn0 <= tn1;
          if (sp < kStack) {
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
    if (active) write_hit(hits, r, leaf, R, best, best_slot);
  }
}

// Many meshes: one lane per ray, the same warp-uniform loop, and lanes
// refilled as their rays finish: when at least kTraceRefill lanes of the warp
// are idle, the warp takes that many new rays from the global counter.  Rays
// of small meshes are short (most miss), so waiting for the warp's longest
// ray left most lanes idle.  Thresholds of 4, 8, 16 and 32 (no refill) idle
// lanes measured 90, 85, 81 and 111 ms on 134M rays over 16,384 meshes.
constexpr int kTraceRefill = 16;

template <bool ANY, bool BATCHED>
__global__ void __launch_bounds__(kTraceThreads, 10) k_trace_refill(const Bvh2Node *bvh_all, const float4 *leaf_all,
                                                            uint32_t n_all, TraceMeshes tm, const float4 *rays,
                                                            uint64_t nrays, Hit *hits, unsigned long long *counter,
                                                            uint32_t *err) {
  const int lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  bool active = false, drained = false;
  uint64_t r = 0;
  Ray R;
  const Bvh2Node *bvh = bvh_all;
  const float4 *leaf = leaf_all;
  uint32_t best = kMiss, best_slot = 0;
  float bt = 0.0f;
  int st_node[kStack];  // inner nodes still to visit (4 B each: the hot top stays in L1)
  int sp = 0;
  int node = 0;
  while (true) {
    const unsigned idle = __ballot_sync(FULL_MASK, !active);
    const int n_idle = __popc(idle);
    if (!drained && (n_idle >= kTraceRefill || n_idle == 32)) {
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(counter, (unsigned long long)n_idle);
      base = __shfl_sync(FULL_MASK, base, 0);
      if (base + n_idle >= nrays) drained = true;
      if (!active) {
        const uint64_t mine = base + __popc(idle & lt);
        if (mine < nrays) {
          r = mine;
          ray_setup(__ldg(rays + 2 * r), __ldg(rays + 2 * r + 1), R);
          bvh = bvh_all;
          leaf = leaf_all;
          uint32_t n = n_all;
          if (BATCHED) {
            const uint32_t m = mesh_of_ray(tm, r);
            const uint32_t b = __ldg(tm.tri_off + m);
            n = __ldg(tm.tri_off + m + 1) - b;
            bvh = bvh_all + (b - m);
            leaf = leaf_all + 3 * (size_t)b;
          }
          best = kMiss;
          best_slot = 0;
          bt = R.tmax;
          sp = 0;
          node = 0;
          if (n == 1) {
            // a one-triangle mesh has no inner node: test its leaf box and triangle
            const float4 a = __ldg(leaf), b = __ldg(leaf + 1), c = __ldg(leaf + 2);
            float tn;
            if (ray_box(R, fminf(a.x, fminf(b.x, c.x)), fminf(a.y, fminf(b.y, c.y)), fminf(a.z, fminf(b.z, c.z)),
                        fmaxf(a.x, fmaxf(b.x, c.x)), fmaxf(a.y, fmaxf(b.y, c.y)), fmaxf(a.z, fmaxf(b.z, c.z)), bt,
                        tn) &&
                tn <= bt)
              leaf_test(leaf, 0, R, best, best_slot, bt);
            write_hit(hits, r, leaf, R, best, best_slot);
          } else {
            active = true;
          }
        }
      }
    }
    if (!__any_sync(FULL_MASK, active)) {
      if (drained) break;
      continue;
    }
    if (!active) continue;

    const float4 *np = reinterpret_cast<const float4 *>(bvh + node);
    const float4 f0 = __ldg(np), f1 = __ldg(np + 1), f2 = __ldg(np + 2);
    const int4 rf = __ldg(reinterpret_cast<const int4 *>(np + 3));
    float tn0, tn1;
    bool h0 = ray_box(R, f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, bt, tn0) && tn0 <= bt;
    bool h1 = ray_box(R, f1.z, f1.w, f2.x, f2.y, f2.z, f2.w, bt, tn1) && tn1 <= bt;
    if (h0 && rf.x < 0) {
      leaf_test(leaf, (uint32_t)~rf.x, R, best, best_slot, bt);
      h0 = false;
    }
    if (h1 && rf.y < 0) {
      if (tn1 <= bt) leaf_test(leaf, (uint32_t)~rf.y, R, best, best_slot, bt);
      h1 = false;
    }
    if (h1 && tn1 > bt) h1 = false;
    bool finished = false;
    if (ANY && best != kMiss) {
      finished = true;
    } else if (h0 && h1) {
      const bool first0 = tn0 <= tn1;
      if (sp < kStack) {
        st_node[sp++] = first0 ? rf.y : rf.x;
        node = first0 ? rf.x : rf.y;
      } else {
        atomicCAS(err, 0u, 5u);  // traversal stack overflow
        finished = true;
      }
    } else if (h0) {
      node = rf.x;
    } else if (h1) {
      node = rf.y;
    } else if (sp > 0) {
      node = st_node[--sp];
    } else {
      finished = true;
    }
    if (finished) {
      write_hit(hits, r, leaf, R, best, best_slot);
      active = false;
    }
  }
}

}  // namespace gprtcu

using namespace gprtcu;

namespace {

gprtcuStatus trace_launch(const gprtcuLbvh *bvh, const uint32_t *tri_off, const uint32_t *ray_off, uint32_t meshes,
                          const float *rays, uint64_t nrays, gprtcuHit *hits, bool any, void *scratch,
                          size_t scratch_bytes, cudaStream_t stream) {
  if (!bvh || (!rays && nrays) || (!hits && nrays)) return GPRTCU_ERR_INVALID_ARG;
  if (meshes == 0 || (meshes > 1 && (!tri_off || !ray_off))) return GPRTCU_ERR_INVALID_ARG;
  if (nrays == 0) return GPRTCU_OK;
  if (bvh->numPrims == 0 || !bvh->leafTris || (bvh->numPrims > meshes && !bvh->bvh2)) return GPRTCU_ERR_INVALID_ARG;
  if (((uintptr_t)rays & 15) || ((uintptr_t)bvh->leafTris & 15) || ((uintptr_t)bvh->bvh2 & 15))
    return GPRTCU_ERR_INVALID_ARG;
  if (!scratch || ((uintptr_t)scratch & 255)) return GPRTCU_ERR_INVALID_ARG;
  if (scratch_bytes < sizeof(ScratchHeader)) return GPRTCU_ERR_SCRATCH_TOO_SMALL;
  ScratchHeader *hdr = (ScratchHeader *)scratch;
  unsigned long long *counter = reinterpret_cast<unsigned long long *>(&hdr->ticket[0]);
  GPRTCU_TRY(cudaMemsetAsync(scratch, 0, sizeof(ScratchHeader), stream));
  const int blocks = gprtcu_num_sms() * 10;  // 48 registers: 10 CTAs of 128 threads per SM
  const uint64_t need = (nrays + kTraceThreads - 1) / kTraceThreads;
  const int grid = (int)(need < (uint64_t)blocks ? need : blocks);
  const TraceMeshes tm{tri_off, ray_off, meshes};
  const Bvh2Node *nodes = (const Bvh2Node *)bvh->bvh2;
  const float4 *leaf = (const float4 *)bvh->leafTris;
  if (meshes > 1) {
#define GPRTCU_TRACE(A)                                                                                      \
  k_trace_refill<A, true><<<grid, kTraceThreads, 0, stream>>>(nodes, leaf, bvh->numPrims, tm, (const float4 *)rays, \
                                                              nrays, (Hit *)hits, counter, &hdr->status)
    if (any) GPRTCU_TRACE(true);
    else GPRTCU_TRACE(false);
#undef GPRTCU_TRACE
  } else {
#define GPRTCU_TRACE(A)                                                                                        \
  k_trace_bin<A><<<grid, kTraceThreads, 0, stream>>>(nodes, leaf, bvh->numPrims, (const float4 *)rays, nrays, \
                                                     (Hit *)hits, counter, &hdr->status)
    if (any) GPRTCU_TRACE(true);
    else GPRTCU_TRACE(false);
#undef GPRTCU_TRACE
  }
  GPRTCU_TRY(cudaGetLastError());
  return GPRTCU_OK;
}

}  // namespace

extern "C" GPRTCU_API size_t gprtcuTraceScratchSize(void) { return sizeof(ScratchHeader); }

extern "C" GPRTCU_API gprtcuStatus gprtcuTraceClosest(const gprtcuLbvh *bvh, const float *rays, uint64_t numRays,
                                                      gprtcuHit *hits, void *scratch, size_t scratchBytes,
                                                      gprtcuStream stream) {
  return trace_launch(bvh, nullptr, nullptr, 1, rays, numRays, hits, false, scratch, scratchBytes, (cudaStream_t)stream);
}

extern "C" GPRTCU_API gprtcuStatus gprtcuTraceAny(const gprtcuLbvh *bvh, const float *rays, uint64_t numRays,
                                                  gprtcuHit *hits, void *scratch, size_t scratchBytes,
                                                  gprtcuStream stream) {
  return trace_launch(bvh, nullptr, nullptr, 1, rays, numRays, hits, true, scratch, scratchBytes, (cudaStream_t)stream);
}

extern "C" GPRTCU_API gprtcuStatus gprtcuBatchTrace(const gprtcuLbvh *bvh, const uint32_t *triOffsets,
                                                    const uint32_t *rayOffsets, uint32_t numMeshes, const float *rays,
                                                    uint64_t numRays, int anyHit, gprtcuHit *hits, void *scratch,
                                                    size_t scratchBytes, gprtcuStream stream) {
  return trace_launch(bvh, triOffsets, rayOffsets, numMeshes, rays, numRays, hits, anyHit != 0, scratch, scratchBytes,
                      (cudaStream_t)stream);
}
