// inst.cu -- two-level instancing: a top-level LBVH over instances of the
// meshes of a bottom-level batch, traced in one kernel.
//
// Instance record: the reference's gprt::Instance (gprt/gprt_shared.h:92-101;
// gprtInstanceAccelCreate, gprt/gprt_host.h:1418): a row-major 3x4
// object-to-world transform, customIndex (24 bits) and mask (8 bits),
// geometryIndex and flags (not used here), and the bottom-level structure --
// here the mesh index in a batched LBVH (gprtcuBatchBuildTriangles), or 0 for
// a single-mesh LBVH.
//
// gprtcuInstancesPrepare computes, per instance, the world-to-object matrix
// (adjugate / determinant in double, fixed operation order, rounded once to
// float) and the world box of the mesh's root box (its eight corners mapped
// in double, rounded outward); the caller builds the top level over those
// boxes with gprtcuLbvhBuildBoxes.  gprtcuTraceInstances walks the top level
// with the world ray; at an instance whose mask meets the ray mask it maps
// the ray into object space (((w0*x + w1*y) + w2*z) + w3 per component, in
// float; tmin/tmax kept: an affine map keeps the ray parameter) and walks
// that mesh's binary LBVH with the same watertight test as the one-level
// traversal.  Closest hit: smallest t, ties to the lowest (instance,
// primitive); t is the refined plane-equation distance in the winning
// instance's object space.
#include "common.cuh"
#include "lbvh.cuh"
#include "rtmath.cuh"

namespace gprtcu {

struct __align__(16) InstanceRec {
  float m[12];
  uint32_t custom_mask;
  uint32_t geom_flags;
  unsigned long long blas;
};
static_assert(sizeof(InstanceRec) == 64, "64-byte instance record");

__global__ void k_instances_prepare(const InstanceRec *inst, uint32_t n, const float *root_boxes, uint32_t meshes,
                                    float *w2o, float *boxes) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const InstanceRec r = inst[i];
    const double a00 = r.m[0], a01 = r.m[1], a02 = r.m[2], t0 = r.m[3];
    const double a10 = r.m[4], a11 = r.m[5], a12 = r.m[6], t1 = r.m[7];
    const double a20 = r.m[8], a21 = r.m[9], a22 = r.m[10], t2 = r.m[11];
    const double c00 = __dsub_rn(__dmul_rn(a11, a22), __dmul_rn(a12, a21));
    const double c01 = __dsub_rn(__dmul_rn(a12, a20), __dmul_rn(a10, a22));
    const double c02 = __dsub_rn(__dmul_rn(a10, a21), __dmul_rn(a11, a20));
    const double c10 = __dsub_rn(__dmul_rn(a02, a21), __dmul_rn(a01, a22));
    const double c11 = __dsub_rn(__dmul_rn(a00, a22), __dmul_rn(a02, a20));
    const double c12 = __dsub_rn(__dmul_rn(a01, a20), __dmul_rn(a00, a21));
    const double c20 = __dsub_rn(__dmul_rn(a01, a12), __dmul_rn(a02, a11));
    const double c21 = __dsub_rn(__dmul_rn(a02, a10), __dmul_rn(a00, a12));
    const double c22 = __dsub_rn(__dmul_rn(a00, a11), __dmul_rn(a01, a10));
    const double det = __dadd_rn(__dadd_rn(__dmul_rn(a00, c00), __dmul_rn(a01, c01)), __dmul_rn(a02, c02));
    float *w = w2o + 12 * (size_t)i;
    float *bx = boxes + 6 * (size_t)i;
    const uint32_t mesh = (uint32_t)r.blas;
    if (!(det != 0.0) || !isfinite(det) || mesh >= meshes) {
      // never entered: zero matrix, empty box
      for (int k = 0; k < 12; ++k) w[k] = 0.0f;
      for (int k = 0; k < 3; ++k) {
        bx[k] = __int_as_float(0x7f800000);
        bx[3 + k] = __int_as_float(0xff800000);
      }
      continue;
    }
    const double in[9] = {__ddiv_rn(c00, det), __ddiv_rn(c10, det), __ddiv_rn(c20, det),
                          __ddiv_rn(c01, det), __ddiv_rn(c11, det), __ddiv_rn(c21, det),
                          __ddiv_rn(c02, det), __ddiv_rn(c12, det), __ddiv_rn(c22, det)};
    const double tv[3] = {t0, t1, t2};
#pragma unroll
    for (int row = 0; row < 3; ++row) {
      const double u = -__dadd_rn(__dadd_rn(__dmul_rn(in[3 * row], tv[0]), __dmul_rn(in[3 * row + 1], tv[1])),
                                  __dmul_rn(in[3 * row + 2], tv[2]));
      w[4 * row] = __double2float_rn(in[3 * row]);
      w[4 * row + 1] = __double2float_rn(in[3 * row + 1]);
      w[4 * row + 2] = __double2float_rn(in[3 * row + 2]);
      w[4 * row + 3] = __double2float_rn(u);
    }
    // world box of the mesh's root box: eight corners in double, rounded outward
    const float *rb = root_boxes + 6 * (size_t)mesh;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int c = 0; c < 8; ++c) {
      const double p[3] = {(double)rb[(c & 1) ? 3 : 0], (double)rb[(c & 2) ? 4 : 1], (double)rb[(c & 4) ? 5 : 2]};
      for (int row = 0; row < 3; ++row) {
        const double v = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn((double)r.m[4 * row], p[0]),
                                                       __dmul_rn((double)r.m[4 * row + 1], p[1])),
                                             __dmul_rn((double)r.m[4 * row + 2], p[2])),
                                   (double)r.m[4 * row + 3]);
        lo[row] = fmin(lo[row], v);
        hi[row] = fmax(hi[row], v);
      }
    }
    for (int k = 0; k < 3; ++k) {
      bx[k] = __double2float_rd(lo[k]);
      bx[3 + k] = __double2float_ru(hi[k]);
    }
  }
}

__device__ __forceinline__ void ray_to_object(const float *w, const Ray &W, Ray &O) {
  const float o[3] = {W.ox, W.oy, W.oz}, d[3] = {W.dx, W.dy, W.dz};
  float ro[3], rd[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float w0 = __ldg(w + 4 * i), w1 = __ldg(w + 4 * i + 1), w2 = __ldg(w + 4 * i + 2), w3 = __ldg(w + 4 * i + 3);
    ro[i] = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(w0, o[0]), __fmul_rn(w1, o[1])), __fmul_rn(w2, o[2])), w3);
    rd[i] = __fadd_rn(__fadd_rn(__fmul_rn(w0, d[0]), __fmul_rn(w1, d[1])), __fmul_rn(w2, d[2]));
  }
  ray_setup(make_float4(ro[0], ro[1], ro[2], W.tmin), make_float4(rd[0], rd[1], rd[2], W.tmax), O);
}

struct InstMeshes {
  const uint32_t *tri_off;  // null: one mesh of n_all triangles
  uint32_t meshes, n_all;
};

constexpr int kInstThreads = 128;
constexpr int kInstStack = 64;
constexpr int kInstRefill = 4;

// One lane per ray from a global counter, warp-uniform visit loop; lanes
// whose rays finished take new rays once kInstRefill of the 32 are idle
// (16,384 instances, 16.8M rays: 32 rays per warp without refill 147 ms,
// refill at 16 / 8 / 4 idle lanes 119.6 / 109.5 / 105.7 ms).  The top-level stack holds references (inner node >= 0, leaf
// ~slot) with their entry distances, so a popped reference behind the best hit
// is dropped; the bottom-level stack holds node indices.
template <bool ANY>
__global__ void __launch_bounds__(kInstThreads) k_trace_inst(const Bvh2Node *tnodes, const uint32_t *tids, uint32_t ninst,
                                                             const float *troot, const InstanceRec *inst,
                                                             const float *w2o, const Bvh2Node *blas_all,
                                                             const float4 *leaf_all, InstMeshes im, const float4 *rays,
                                                             uint64_t nrays, uint32_t ray_mask, Hit *hits,
                                                             uint32_t *hit_inst, unsigned long long *counter,
                                                             uint32_t *err) {
  const int lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  bool active = false, drained = false, done = true;
  uint64_t r = 0;
  Ray W, O;
  uint32_t best = kMiss, binst = kMiss, bslot = 0;
  float bt = 0.0f;
  int tref[kInstStack];
  float ttn[kInstStack];
  int tsp = 0;
  int bstack[kInstStack];
  int bsp = 0;
  int level = 0, cur = 0, bnode = 0;
  uint32_t ci = 0;  // instance being walked
  const Bvh2Node *bvh = blas_all;
  const float4 *leaf = leaf_all;
  auto tri_test = [&](uint32_t slot) {
    const float4 a = __ldg(leaf + 3 * (size_t)slot), b = __ldg(leaf + 3 * (size_t)slot + 1),
                 c = __ldg(leaf + 3 * (size_t)slot + 2);
    const float v0[3] = {a.x, a.y, a.z}, v1[3] = {b.x, b.y, b.z}, v2[3] = {c.x, c.y, c.z};
    const uint32_t id = __float_as_uint(a.w);
    float t;
    if (isect_tri(O, v0, v1, v2, t) &&
        (best == kMiss || t < bt || (t == bt && (ci < binst || (ci == binst && id < best))))) {
      best = id;
      binst = ci;
      bslot = slot;
      bt = t;
    }
  };
  auto pop_top = [&]() {
    while (tsp > 0) {
      --tsp;
      if (ttn[tsp] <= bt) {
        cur = tref[tsp];
        return;
      }
    }
    done = true;
  };
  while (true) {
    // Lanes whose rays finished take new ones once kInstRefill of the warp's
    // 32 are idle (rays differ widely in how many instances they enter).
    const unsigned idle = __ballot_sync(FULL_MASK, !active);
    const int n_idle = __popc(idle);
    if (!drained && (n_idle >= kInstRefill || n_idle == 32)) {
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(counter, (unsigned long long)n_idle);
      base = __shfl_sync(FULL_MASK, base, 0);
      if (base + n_idle >= nrays) drained = true;
      if (!active) {
        const uint64_t mine = base + __popc(idle & lt);
        if (mine < nrays) {
          r = mine;
          active = true;
          done = false;
          ray_setup(__ldg(rays + 2 * r), __ldg(rays + 2 * r + 1), W);
          O = W;
          best = kMiss;
          binst = kMiss;
          bslot = 0;
          bt = W.tmax;
          tsp = 0;
          bsp = 0;
          level = 0;
          cur = 0;
          if (ninst == 1) {
            float tn;
            cur = ~0;  // the single instance is the root leaf
            if (!ray_box(W, troot[0], troot[1], troot[2], troot[3], troot[4], troot[5], bt, tn)) done = true;
          }
        }
      }
    }
    if (!__any_sync(FULL_MASK, active)) {
      if (drained) break;
      continue;
    }
    if (active && !done) {
      if (level == 1) {
        // ---- bottom level: the instance's mesh in object space
        const float4 *np = reinterpret_cast<const float4 *>(bvh + bnode);
        const float4 f0 = __ldg(np), f1 = __ldg(np + 1), f2 = __ldg(np + 2);
        const int4 rf = __ldg(reinterpret_cast<const int4 *>(np + 3));
        float tn0, tn1;
        bool h0 = ray_box(O, f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, bt, tn0) && tn0 <= bt;
        bool h1 = ray_box(O, f1.z, f1.w, f2.x, f2.y, f2.z, f2.w, bt, tn1) && tn1 <= bt;
        if (h0 && rf.x < 0) {
          tri_test((uint32_t)~rf.x);
          h0 = false;
        }
        if (h1 && rf.y < 0) {
          if (tn1 <= bt) tri_test((uint32_t)~rf.y);
          h1 = false;
        }
        if (h1 && tn1 > bt) h1 = false;
        if (ANY && best != kMiss) {
          done = true;
        } else if (h0 && h1) {
          const bool first0 = tn0 <= tn1;
          if (bsp < kInstStack) {
            bstack[bsp++] = first0 ? rf.y : rf.x;
            bnode = first0 ? rf.x : rf.y;
          } else {
            atomicCAS(err, 0u, 5u);  // traversal stack overflow
            done = true;
          }
        } else if (h0) {
          bnode = rf.x;
        } else if (h1) {
          bnode = rf.y;
        } else if (bsp > 0) {
          bnode = bstack[--bsp];
        } else {
          level = 0;  // back to the top level
          pop_top();
        }
      } else if (cur >= 0) {
        // ---- top level, inner node
        const float4 *np = reinterpret_cast<const float4 *>(tnodes + cur);
        const float4 f0 = __ldg(np), f1 = __ldg(np + 1), f2 = __ldg(np + 2);
        const int4 rf = __ldg(reinterpret_cast<const int4 *>(np + 3));
        float tn0, tn1;
        const bool h0 = ray_box(W, f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, bt, tn0) && tn0 <= bt;
        const bool h1 = ray_box(W, f1.z, f1.w, f2.x, f2.y, f2.z, f2.w, bt, tn1) && tn1 <= bt;
        if (h0 && h1) {
          const bool first0 = tn0 <= tn1;
          if (tsp < kInstStack) {
            tref[tsp] = first0 ? rf.y : rf.x;
            ttn[tsp] = first0 ? tn1 : tn0;
            ++tsp;
            cur = first0 ? rf.x : rf.y;
          } else {
            atomicCAS(err, 0u, 5u);
            done = true;
          }
        } else if (h0) {
          cur = rf.x;
        } else if (h1) {
          cur = rf.y;
        } else {
          pop_top();
        }
      } else {
        // ---- top level, an instance: enter its mesh in object space
        ci = __ldg(tids + (uint32_t)~cur);
        const uint32_t cm = __ldg(&inst[ci].custom_mask);
        const uint32_t mesh = (uint32_t)__ldg(&inst[ci].blas);
        bool entered = false;
        if (((cm >> 24) & ray_mask) && mesh < im.meshes) {
          const float *w = w2o + 12 * (size_t)ci;
          if (__ldg(w) != 0.0f || __ldg(w + 1) != 0.0f || __ldg(w + 2) != 0.0f) {  // singular: all zero
            ray_to_object(w, W, O);
            const uint32_t b = im.tri_off ? __ldg(im.tri_off + mesh) : 0u;
            const uint32_t cnt = im.tri_off ? __ldg(im.tri_off + mesh + 1) - b : im.n_all;
            bvh = blas_all + (b - mesh);
            leaf = leaf_all + 3 * (size_t)b;
            if (cnt == 1) {
              const float4 a = __ldg(leaf), bb = __ldg(leaf + 1), c = __ldg(leaf + 2);
              float tn;
              if (ray_box(O, fminf(a.x, fminf(bb.x, c.x)), fminf(a.y, fminf(bb.y, c.y)), fminf(a.z, fminf(bb.z, c.z)),
                          fmaxf(a.x, fmaxf(bb.x, c.x)), fmaxf(a.y, fmaxf(bb.y, c.y)), fmaxf(a.z, fmaxf(bb.z, c.z)), bt,
                          tn) &&
                  tn <= bt)
                tri_test(0);
              if (ANY && best != kMiss) done = true;
            } else {
              level = 1;
              bnode = 0;
              bsp = 0;
              entered = true;
            }
          }
        }
        if (!entered && !done) pop_top();
      }
    }
    if (active && done) {
      Hit h;
      h.prim = best;
      h.t = __int_as_float(0x7f800000);
      if (best != kMiss) {
        // the winner's object-space ray again (same operations, same bits)
        ray_to_object(w2o + 12 * (size_t)binst, W, O);
        const uint32_t mesh = (uint32_t)__ldg(&inst[binst].blas);
        const uint32_t b = im.tri_off ? __ldg(im.tri_off + mesh) : 0u;
        const float4 *lf = leaf_all + 3 * (size_t)b;
        const float4 a = __ldg(lf + 3 * (size_t)bslot), bb = __ldg(lf + 3 * (size_t)bslot + 1),
                     c = __ldg(lf + 3 * (size_t)bslot + 2);
        const float v0[3] = {a.x, a.y, a.z}, v1[3] = {bb.x, bb.y, bb.z}, v2[3] = {c.x, c.y, c.z};
        h.t = refine_t(O, v0, v1, v2);
      }
      hits[r] = h;
      if (hit_inst) hit_inst[r] = binst;
      active = false;
    }
  }
}

}  // namespace gprtcu

using namespace gprtcu;

extern "C" GPRTCU_API gprtcuStatus gprtcuInstancesPrepare(const gprtcuInstance *instances, uint32_t numInstances,
                                                          const float *blasRootBoxes, uint32_t numMeshes,
                                                          float *worldToObject, float *worldBoxes,
                                                          gprtcuStream stream) {
  if (numInstances == 0) return GPRTCU_OK;
  if (!instances || !blasRootBoxes || !worldToObject || !worldBoxes || numMeshes == 0) return GPRTCU_ERR_INVALID_ARG;
  if (((uintptr_t)instances & 15)) return GPRTCU_ERR_INVALID_ARG;
  const uint64_t g = (numInstances + 255) / 256, cap = (uint64_t)gprtcu_num_sms() * 16;
  k_instances_prepare<<<(unsigned)(g < cap ? g : cap), 256, 0, (cudaStream_t)stream>>>(
      (const InstanceRec *)instances, numInstances, blasRootBoxes, numMeshes, worldToObject, worldBoxes);
  GPRTCU_TRY(cudaGetLastError());
  return GPRTCU_OK;
}

extern "C" GPRTCU_API gprtcuStatus gprtcuTraceInstances(const gprtcuLbvh *tlas, const gprtcuInstance *instances,
                                                        const float *worldToObject, const gprtcuLbvh *blas,
                                                        const uint32_t *triOffsets, uint32_t numMeshes,
                                                        const float *rays, uint64_t numRays, uint32_t rayMask,
                                                        int anyHit, gprtcuHit *hits, uint32_t *hitInstance,
                                                        void *scratch, size_t scratchBytes, gprtcuStream stream_) {
  cudaStream_t stream = (cudaStream_t)stream_;
  if (!tlas || !instances || !worldToObject || !blas || numMeshes == 0 || (numMeshes > 1 && !triOffsets))
    return GPRTCU_ERR_INVALID_ARG;
  if ((!rays || !hits) && numRays) return GPRTCU_ERR_INVALID_ARG;
  if (numRays == 0) return GPRTCU_OK;
  if (tlas->numPrims == 0 || !tlas->ids || !tlas->rootBox || (tlas->numPrims > 1 && !tlas->bvh2))
    return GPRTCU_ERR_INVALID_ARG;
  if (blas->numPrims == 0 || !blas->leafTris || (blas->numPrims > numMeshes && !blas->bvh2)) return GPRTCU_ERR_INVALID_ARG;
  if (((uintptr_t)rays & 15) || ((uintptr_t)instances & 15) || ((uintptr_t)tlas->bvh2 & 15) ||
      ((uintptr_t)blas->bvh2 & 15) || ((uintptr_t)blas->leafTris & 15))
    return GPRTCU_ERR_INVALID_ARG;
  if (!scratch || ((uintptr_t)scratch & 255)) return GPRTCU_ERR_INVALID_ARG;
  if (scratchBytes < sizeof(ScratchHeader)) return GPRTCU_ERR_SCRATCH_TOO_SMALL;
  ScratchHeader *hdr = (ScratchHeader *)scratch;
  unsigned long long *counter = reinterpret_cast<unsigned long long *>(&hdr->ticket[0]);
  GPRTCU_TRY(cudaMemsetAsync(scratch, 0, sizeof(ScratchHeader), stream));
  const int blocks = gprtcu_num_sms() * 8;
  const uint64_t need = (numRays + kInstThreads - 1) / kInstThreads;
  const int grid = (int)(need < (uint64_t)blocks ? need : blocks);
  const InstMeshes im{numMeshes > 1 ? triOffsets : nullptr, numMeshes, blas->numPrims};
#define GPRTCU_ITRACE(A)                                                                                             \
  k_trace_inst<A><<<grid, kInstThreads, 0, stream>>>(                                                              \
      (const Bvh2Node *)tlas->bvh2, tlas->ids, tlas->numPrims, tlas->rootBox, (const InstanceRec *)instances,     \
      worldToObject, (const Bvh2Node *)blas->bvh2, (const float4 *)blas->leafTris, im, (const float4 *)rays, numRays, \
      rayMask, (Hit *)hits, hitInstance, counter, &hdr->status)
  if (anyHit) GPRTCU_ITRACE(true);
  else GPRTCU_ITRACE(false);
#undef GPRTCU_ITRACE
  GPRTCU_TRY(cudaGetLastError());
  return GPRTCU_OK;
}
