// solid.cu -- solid cells (tetrahedra, pyramids, wedges, hexahedra and
// tetrahedral pairs: the linear finite elements of volume meshes) as
// software-BVH primitives: their bounds, and point location over an LBVH
// built on those bounds (gprtcuLbvhBuildBoxes).
//
// The reference builds a hardware AABB structure over the boxes of its
// SolidBounds compute program (gprt/gprt_fallbacks.slang:467-502) and answers
// TracePoint (gprt/gprt_builtins.slang:80-90: a zero-length ray from the
// point) with SolidIntersection (:504-566), which inverts the cell's
// isoparametric map by Newton's method (intersectPointSolid, :409-464).  Here
// the same arithmetic runs in CUDA with every float operation an explicit
// round-to-nearest intrinsic in the reference's evaluation order, and the
// derivatives the reference takes with forward-mode automatic differentiation
// (fwd_diff of IsoToSupport, :437-439) are carried as dual numbers with the
// same rules (d(c - a) = -da, d(a b) = da b + a db), so the containing cell,
// its (r, s, t) and its interpolated density are bit-identical to the
// reference's code compiled for the host.
//
// A point lies in a cell's box when lo <= p <= hi on every axis (a zero-length
// ray meets a box exactly then).  Of the cells whose box and Newton inversion
// contain the point, the lowest-numbered one is reported (every hit of a
// point query is at t = 0; ties go to the lowest id, as for rays).
#include "common.cuh"
#include "lbvh.cuh"

namespace gprtcu {

// Cell types (gprt/gprt_host.h:291-298) and their vertex counts and hit kinds
// (gprt/gprt_fallbacks.slang:289-318).  A tetrahedral pair has eight nodes,
// is evaluated as a trilinear cell and reports the tetrahedron kind.
__device__ __forceinline__ int solid_nodes(uint32_t type) {
  return type == 10u ? 4 : type == 14u ? 5 : type == 13u ? 6 : (type == 12u || type == 23u) ? 8 : 0;
}
__device__ __forceinline__ uint32_t solid_kind(uint32_t type) {
  return type == 23u ? 10u : (type == 10u || type == 12u || type == 13u || type == 14u) ? type : 0u;
}

// Where a cell's data lives: vertex k of the mesh at vertices + k *
// vertexStride (float4 {x, y, z, density}), cell c's vertex indices at
// indices + c * indexStride (uint32 each), its type at types + c * typeStride.
struct SolidView {
  const unsigned char *verts, *idx, *types;
  uint32_t vstride, istride, tstride, n;
  __device__ __forceinline__ uint32_t type(uint32_t c) const { return __ldg(types + (size_t)c * tstride); }
  __device__ __forceinline__ uint32_t index(uint32_t c, int i) const {
    return __ldg(reinterpret_cast<const uint32_t *>(idx + (size_t)c * istride) + i);
  }
  __device__ __forceinline__ float4 vertex(uint32_t k) const {
    return __ldg(reinterpret_cast<const float4 *>(verts + (size_t)k * vstride));
  }
};

// Dual number (value, derivative) with single-rounded operations.
struct Dl {
  float v, d;
};
__device__ __forceinline__ Dl dl_add(Dl a, Dl b) { return {__fadd_rn(a.v, b.v), __fadd_rn(a.d, b.d)}; }
__device__ __forceinline__ Dl dl_sub(Dl a, Dl b) { return {__fsub_rn(a.v, b.v), __fsub_rn(a.d, b.d)}; }
__device__ __forceinline__ Dl dl_rsub1(Dl a) { return {__fsub_rn(1.0f, a.v), -a.d}; }
__device__ __forceinline__ Dl dl_mul(Dl a, Dl b) {
  return {__fmul_rn(a.v, b.v), __fadd_rn(__fmul_rn(a.d, b.v), __fmul_rn(a.v, b.d))};
}

// IsoToSupport (gprt/gprt_fallbacks.slang:370-406): the shape functions of
// an n-node cell at (r, s, t), in the reference's operation order; with a
// seeded direction, their derivatives along it.
__device__ __forceinline__ void iso_support(int n, Dl r, Dl s, Dl t, Dl w[8]) {
#pragma unroll
  for (int i = 0; i < 8; ++i) w[i] = {0.0f, 0.0f};
  const Dl mr = dl_rsub1(r), ms = dl_rsub1(s), mt = dl_rsub1(t);
  if (n == 4) {
    w[0] = dl_rsub1(dl_add(dl_add(r, s), t));
    w[1] = r;
    w[2] = s;
    w[3] = t;
  } else if (n == 5) {
    w[0] = dl_mul(dl_mul(mr, ms), mt);
    w[1] = dl_mul(dl_mul(r, ms), mt);
    w[2] = dl_mul(dl_mul(r, s), mt);
    w[3] = dl_mul(dl_mul(mr, s), mt);
    w[4] = t;
  } else if (n == 6) {
    const Dl rs = dl_sub(mr, s);
    w[0] = dl_mul(rs, mt);
    w[1] = dl_mul(r, mt);
    w[2] = dl_mul(s, mt);
    w[3] = dl_mul(rs, t);
    w[4] = dl_mul(r, t);
    w[5] = dl_mul(s, t);
  } else if (n == 8) {
    const Dl a0 = dl_mul(mr, ms), a1 = dl_mul(r, ms), a2 = dl_mul(r, s), a3 = dl_mul(mr, s);
    w[0] = dl_mul(a0, mt);
    w[1] = dl_mul(a1, mt);
    w[2] = dl_mul(a2, mt);
    w[3] = dl_mul(a3, mt);
    w[4] = dl_mul(a0, t);
    w[5] = dl_mul(a1, t);
    w[6] = dl_mul(a2, t);
    w[7] = dl_mul(a3, t);
  }
}

// Determinant of the 3x3 matrix with rows a, b, c (cofactors of the first row).
__device__ __forceinline__ float det3(float a0, float a1, float a2, float b0, float b1, float b2, float c0, float c1,
                                      float c2) {
  const float m0 = __fsub_rn(__fmul_rn(b1, c2), __fmul_rn(b2, c1));
  const float m1 = __fsub_rn(__fmul_rn(b0, c2), __fmul_rn(b2, c0));
  const float m2 = __fsub_rn(__fmul_rn(b0, c1), __fmul_rn(b1, c0));
  return __fadd_rn(__fsub_rn(__fmul_rn(a0, m0), __fmul_rn(a1, m1)), __fmul_rn(a2, m2));
}

// intersectPointSolid (gprt/gprt_fallbacks.slang:409-464): at most five
// Newton steps from GetInitialRST (:320-325); each step uses the residual
// and Jacobian at the current (r, s, t), updates by Cramer's rule, then stops
// if that residual was below 1e-3 on every axis; a Jacobian determinant below
// 1e-20 in magnitude ends the test.  Containment per IsoIsContained
// (:327-340); the density applies the last evaluated shape functions to the
// nodal densities.  q: the cell's nodes, zero beyond n.
__device__ bool solid_intersect(float px, float py, float pz, const float4 q[8], int n, float4 &rstw) {
  float r = 0.5f, s = 0.5f, t = 0.5f;
  if (n == 4) r = s = t = 0.25f;
  if (n == 5) t = 0.2f;
  float w[8];
  bool converged = false;
  for (int it = 0; it < 5; ++it) {
    Dl dw[8];
    iso_support(n, {r, 0.0f}, {s, 0.0f}, {t, 0.0f}, dw);
    float fx = -px, fy = -py, fz = -pz;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      w[i] = dw[i].v;
      fx = __fadd_rn(fx, __fmul_rn(q[i].x, w[i]));
      fy = __fadd_rn(fy, __fmul_rn(q[i].y, w[i]));
      fz = __fadd_rn(fz, __fmul_rn(q[i].z, w[i]));
    }
    float c[3][3];
#pragma unroll
    for (int dir = 0; dir < 3; ++dir) {
      iso_support(n, {r, dir == 0 ? 1.0f : 0.0f}, {s, dir == 1 ? 1.0f : 0.0f}, {t, dir == 2 ? 1.0f : 0.0f}, dw);
      float cx = 0.0f, cy = 0.0f, cz = 0.0f;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        cx = __fadd_rn(cx, __fmul_rn(q[i].x, dw[i].d));
        cy = __fadd_rn(cy, __fmul_rn(q[i].y, dw[i].d));
        cz = __fadd_rn(cz, __fmul_rn(q[i].z, dw[i].d));
      }
      c[dir][0] = cx;
      c[dir][1] = cy;
      c[dir][2] = cz;
    }
    const float d = det3(c[0][0], c[0][1], c[0][2], c[1][0], c[1][1], c[1][2], c[2][0], c[2][1], c[2][2]);
    if (fabsf(d) < 1e-20f) return false;
    const float dinv = __fdiv_rn(1.0f, d);
    const float ur = det3(fx, fy, fz, c[1][0], c[1][1], c[1][2], c[2][0], c[2][1], c[2][2]);
    const float us = det3(c[0][0], c[0][1], c[0][2], fx, fy, fz, c[2][0], c[2][1], c[2][2]);
    const float ut = det3(c[0][0], c[0][1], c[0][2], c[1][0], c[1][1], c[1][2], fx, fy, fz);
    r = __fsub_rn(r, __fmul_rn(ur, dinv));
    s = __fsub_rn(s, __fmul_rn(us, dinv));
    t = __fsub_rn(t, __fmul_rn(ut, dinv));
    if (fabsf(fx) < 1e-3f && fabsf(fy) < 1e-3f && fabsf(fz) < 1e-3f) {
      converged = true;
      break;
    }
  }
  if (!converged) return false;
  bool in = r >= 0.0f && s >= 0.0f && t >= 0.0f && r <= 1.0f && s <= 1.0f && t <= 1.0f;
  if (n == 4) in = in && __fadd_rn(__fadd_rn(r, s), t) <= 1.0f;
  if (n == 6) in = in && __fadd_rn(r, s) <= 1.0f;
  if (!in) return false;
  float dens = 0.0f;
#pragma unroll
  for (int i = 0; i < 8; ++i) dens = __fadd_rn(dens, __fmul_rn(q[i].w, w[i]));
  rstw = make_float4(r, s, t, dens);
  return true;
}

// SolidBounds (gprt/gprt_fallbacks.slang:467-502): min / max of the cell's
// vertices and of their densities.  aabbs (optional): two float4 per cell in
// the reference's layout {lo.xyz, hi.x}, {hi.yz, density min, density max};
// boxes (optional): float[6] {lo.xyz, hi.xyz} per cell for the box LBVH.  A
// cell of unknown type has no vertices and an empty box (lo = +FLT_MAX,
// hi = -FLT_MAX), which no point lies in.
__global__ void k_solid_bounds(SolidView sv, float4 *aabbs, float *boxes) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < sv.n; c += gridDim.x * blockDim.x) {
    const int n = solid_nodes(sv.type(c));
    float lx = 3.402823466e38f, ly = 3.402823466e38f, lz = 3.402823466e38f;
    float hx = -3.402823466e38f, hy = -3.402823466e38f, hz = -3.402823466e38f;
    float dlo = 3.402823466e38f, dhi = -3.402823466e38f;
    for (int i = 0; i < n; ++i) {
      const float4 v = sv.vertex(sv.index(c, i));
      lx = fminf(lx, v.x);
      ly = fminf(ly, v.y);
      lz = fminf(lz, v.z);
      hx = fmaxf(hx, v.x);
      hy = fmaxf(hy, v.y);
      hz = fmaxf(hz, v.z);
      dlo = fminf(dlo, v.w);
      dhi = fmaxf(dhi, v.w);
    }
    if (aabbs) {
      aabbs[2 * (size_t)c] = make_float4(lx, ly, lz, hx);
      aabbs[2 * (size_t)c + 1] = make_float4(hy, hz, dlo, dhi);
    }
    if (boxes) {
      float *b = boxes + 6 * (size_t)c;
      b[0] = lx;
      b[1] = ly;
      b[2] = lz;
      b[3] = hx;
      b[4] = hy;
      b[5] = hz;
    }
  }
}

constexpr int kLocateThreads = 128;
constexpr int kLocateStack = 64;
constexpr uint32_t kNoCell = 0xFFFFFFFFu;

__device__ __forceinline__ bool point_in(float px, float py, float pz, float lx, float ly, float lz, float hx, float hy,
                                         float hz) {
  return lx <= px && px <= hx && ly <= py && py <= hy && lz <= pz && pz <= hz;
}

// Point location over the box LBVH (gprtcuLbvh.bvh2 over the cells' boxes;
// leaf slot k holds cell ids[k]).  32 points per warp, one lane per point,
// taken from a global counter.  The traversal only collects candidates: a
// leaf whose box holds the point appends (cell, lane) to the warp's queue in
// shared memory.  The Newton inversions then run from the queue with every
// lane of the warp taking one candidate, whoever's point it is, and a cell
// that holds the point lowers its owner's best cell with a shared-memory
// atomicMin.  (Running each lane's inversions where its traversal met them
// left 3.2 of 32 lanes active: lanes reach leaves at different steps, and an
// inversion is ~1,000 instructions.)  The queue is drained whenever it could
// overflow on the next step and at the end; candidates at or above the
// owner's best so far are dropped.  The winner's (r, s, t, density) is
// recomputed by its owner once at the end (the same arithmetic, so the same
// bits).  hits: {cell, kind} per point (cell 0xFFFFFFFF, kind 0 when no cell
// holds it); rstw (optional): (r, s, t, density), zero on a miss.
constexpr int kLocateQueue = 256;  // per warp; a step appends at most 64

__device__ __forceinline__ bool locate_cell(const SolidView &sv, uint32_t id, float px, float py, float pz,
                                            float4 &r) {
  const int n = solid_nodes(sv.type(id));
  float4 q[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) q[i] = i < n ? sv.vertex(sv.index(id, i)) : make_float4(0.f, 0.f, 0.f, 0.f);
  return n && solid_intersect(px, py, pz, q, n, r);
}

__global__ void __launch_bounds__(kLocateThreads) k_locate_solids(const Bvh2Node *bvh, const uint32_t *ids,
                                                                  uint32_t nleaves, const float *root_box, SolidView sv,
                                                                  const float4 *points, uint64_t npts, uint2 *hits,
                                                                  float4 *rstw_out, unsigned long long *counter,
                                                                  uint32_t *err) {
  constexpr int WARPS = kLocateThreads / 32;
  __shared__ uint32_t s_qcell[WARPS][kLocateQueue];
  __shared__ uint8_t s_qown[WARPS][kLocateQueue];
  __shared__ float4 s_pt[WARPS][32];
  __shared__ uint32_t s_best[WARPS][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  uint32_t *qcell = s_qcell[warp];
  uint8_t *qown = s_qown[warp];
  uint32_t *best = s_best[warp];
  uint32_t qn = 0;  // warp-uniform queue length
  // every lane takes one queued candidate per round
  auto drain = [&]() {
    __syncwarp();
    for (uint32_t b = 0; b < qn; b += 32) {
      const uint32_t e = b + lane;
      if (e < qn) {
        const uint32_t id = qcell[e], own = qown[e];
        if (id < *reinterpret_cast<volatile uint32_t *>(best + own)) {
          const float4 p = s_pt[warp][own];
          float4 r;
          if (locate_cell(sv, id, p.x, p.y, p.z, r)) atomicMin(best + own, id);
        }
      }
    }
    qn = 0;
    __syncwarp();
  };
  // append this lane's candidate (if want) to the warp's queue
  auto push = [&](bool want, uint32_t id) {
    const unsigned m = __ballot_sync(FULL_MASK, want);
    if (want) {
      const uint32_t at = qn + __popc(m & lt);
      qcell[at] = id;
      qown[at] = (uint8_t)lane;
    }
    qn += __popc(m);
  };
  while (true) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(counter, 32ull);
    base = __shfl_sync(FULL_MASK, base, 0);
    if (base >= npts) break;
    const uint64_t qi = base + lane;
    const bool active = qi < npts;
    const float4 p = active ? __ldg(points + qi) : make_float4(0.f, 0.f, 0.f, 0.f);
    s_pt[warp][lane] = p;
    best[lane] = kNoCell;
    __syncwarp();
    bool done = !active;
    int stack[kLocateStack];
    int sp = 0;
    int node = 0;
    if (nleaves == 1) {
      push(active && point_in(p.x, p.y, p.z, root_box[0], root_box[1], root_box[2], root_box[3], root_box[4],
                              root_box[5]),
           __ldg(ids));
      done = true;
    }
    while (__any_sync(FULL_MASK, !done)) {
      uint32_t c0 = kNoCell, c1 = kNoCell;  // leaf candidates of this step
      if (!done) {
        const float4 *np = reinterpret_cast<const float4 *>(bvh + node);
        const float4 f0 = __ldg(np), f1 = __ldg(np + 1), f2 = __ldg(np + 2);
        const int4 rf = __ldg(reinterpret_cast<const int4 *>(np + 3));
        bool h0 = point_in(p.x, p.y, p.z, f0.x, f0.y, f0.z, f0.w, f1.x, f1.y);
        bool h1 = point_in(p.x, p.y, p.z, f1.z, f1.w, f2.x, f2.y, f2.z, f2.w);
        if (h0 && rf.x < 0) {
          c0 = __ldg(ids + (uint32_t)~rf.x);
          h0 = false;
        }
        if (h1 && rf.y < 0) {
          c1 = __ldg(ids + (uint32_t)~rf.y);
          h1 = false;
        }
        if (h0 && h1) {
          if (sp < kLocateStack) {
            stack[sp++] = rf.y;
            node = rf.x;
          } else {
            atomicCAS(err, 0u, 5u);  // traversal stack overflow
            done = true;
          }
        } else if (h0) {
          node = rf.x;
        } else if (h1) {
          node = rf.y;
        } else if (sp > 0) {
          node = stack[--sp];
        } else {
          done = true;
        }
      }
      const uint32_t b = best[lane];
      push(c0 < b, c0);
      push(c1 < b, c1);
      if (qn > kLocateQueue - 64) drain();
    }
    drain();
    if (active) {
      const uint32_t id = best[lane];
      float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
      if (id != kNoCell) locate_cell(sv, id, p.x, p.y, p.z, r);
      hits[qi] = make_uint2(id, id == kNoCell ? 0u : solid_kind(sv.type(id)));
      if (rstw_out) rstw_out[qi] = r;
    }
    __syncwarp();
  }
}

}  // namespace gprtcu

using namespace gprtcu;

namespace {

bool make_view(const gprtcuSolids *s, SolidView &v) {
  if (!s) return false;
  v.n = s->numCells;
  v.vstride = s->vertexStride ? s->vertexStride : 16;
  v.istride = s->indexStride ? s->indexStride : 32;
  v.tstride = s->typeStride ? s->typeStride : 1;
  v.verts = (const unsigned char *)s->vertices;
  v.idx = (const unsigned char *)s->indices;
  v.types = (const unsigned char *)s->types;
  if (v.n == 0) return true;
  if (!v.verts || !v.idx || !v.types) return false;
  // float4 vertices (16-byte aligned, as the reference indexes them in
  // float4 units) and uint32 indices
  if (((uintptr_t)v.verts & 15) || (v.vstride & 15) || ((uintptr_t)v.idx & 3) || (v.istride & 3)) return false;
  return true;
}

}  // namespace

extern "C" GPRTCU_API gprtcuStatus gprtcuSolidBounds(const gprtcuSolids *solids, float *aabbs, float *boxes,
                                                     gprtcuStream stream) {
  SolidView v;
  if (!make_view(solids, v)) return GPRTCU_ERR_INVALID_ARG;
  if (v.n == 0) return GPRTCU_OK;
  if ((aabbs && ((uintptr_t)aabbs & 15)) || (!aabbs && !boxes)) return GPRTCU_ERR_INVALID_ARG;
  const uint64_t g = (v.n + 255) / 256, cap = (uint64_t)gprtcu_num_sms() * 16;
  k_solid_bounds<<<(unsigned)(g < cap ? g : cap), 256, 0, (cudaStream_t)stream>>>(v, (float4 *)aabbs, boxes);
  GPRTCU_TRY(cudaGetLastError());
  return GPRTCU_OK;
}

extern "C" GPRTCU_API gprtcuStatus gprtcuLocateSolidPoints(const gprtcuLbvh *bvh, const gprtcuSolids *solids,
                                                           const float *points, uint64_t numPoints,
                                                           gprtcuSolidHit *hits, float *rstw, void *scratch,
                                                           size_t scratchBytes, gprtcuStream stream_) {
  cudaStream_t stream = (cudaStream_t)stream_;
  SolidView v;
  if (!bvh || !make_view(solids, v) || (!points && numPoints) || (!hits && numPoints)) return GPRTCU_ERR_INVALID_ARG;
  if (numPoints == 0) return GPRTCU_OK;
  if (bvh->numPrims == 0 || bvh->numPrims != v.n || !bvh->ids || !bvh->rootBox || (bvh->numPrims > 1 && !bvh->bvh2))
    return GPRTCU_ERR_INVALID_ARG;
  if (((uintptr_t)points & 15) || ((uintptr_t)bvh->bvh2 & 15) || ((uintptr_t)hits & 7) || ((uintptr_t)rstw & 15))
    return GPRTCU_ERR_INVALID_ARG;
  if (!scratch || ((uintptr_t)scratch & 255)) return GPRTCU_ERR_INVALID_ARG;
  if (scratchBytes < sizeof(ScratchHeader)) return GPRTCU_ERR_SCRATCH_TOO_SMALL;
  ScratchHeader *hdr = (ScratchHeader *)scratch;
  GPRTCU_TRY(cudaMemsetAsync(scratch, 0, sizeof(ScratchHeader), stream));
  const uint64_t need = (numPoints + kLocateThreads - 1) / kLocateThreads;
  const uint64_t blocks = (uint64_t)gprtcu_num_sms() * 8;
  k_locate_solids<<<(unsigned)(need < blocks ? need : blocks), kLocateThreads, 0, stream>>>(
      (const Bvh2Node *)bvh->bvh2, bvh->ids, bvh->numPrims, bvh->rootBox, v, (const float4 *)points, numPoints,
      (uint2 *)hits, (float4 *)rstw, reinterpret_cast<unsigned long long *>(&hdr->ticket[0]), &hdr->status);
  GPRTCU_TRY(cudaGetLastError());
  return GPRTCU_OK;
}
