// lbvh.cu -- linear BVH build over indexed triangles (and points) for sm_100a.
//
// Replaces the reference's software LBVH (gprt/development/gprt_lbvh.h:170-195,
// gprt/development/gprt_lbvh.hlsl:188-428): scene bounds, 30-bit Morton (or
// Hilbert) codes of the centroids, stable (code, id) sort, Karras topology and
// bottom-up boxes.  Bit-identical results, different mechanics:
//   * bounds: block reduction, one atomic per CTA per component on
//     order-preserving integer images of the floats (the reference issues a
//     CAS loop per primitive on six global words);
//   * refit: one thread per leaf walks up and only the second child to
//     arrive at a node (atomic arrival counter) forms its union -- O(n) work
//     instead of the reference's per-leaf walk to the root with six CAS
//     atomics per ancestor.  min/max are exact, so the boxes are identical;
//   * the refit also emits the traversal layout: a 64-byte node per inner
//     node holding both child boxes and child references, and each leaf's
//     triangle gathered into leaf order (48 bytes).
#include "common.cuh"
#include "lbvh.cuh"

namespace gprtcu {

__device__ __forceinline__ uint32_t f2ord(float f) {
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t o) {
  return __uint_as_float((o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o);
}

__device__ __forceinline__ void load_tri(const float *pos, const uint32_t *tri, uint32_t id, float v[9]) {
  const uint32_t i0 = tri[3 * (size_t)id], i1 = tri[3 * (size_t)id + 1], i2 = tri[3 * (size_t)id + 2];
  const float *p0 = pos + 3 * (size_t)i0, *p1 = pos + 3 * (size_t)i1, *p2 = pos + 3 * (size_t)i2;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    v[k] = p0[k];
    v[3 + k] = p1[k];
    v[6 + k] = p2[k];
  }
}

// Centroid (p1 + p2 + p3) / 3 of a triangle (getTriangleCentroid,
// gprt/development/gprt_lbvh.hlsl:139-146), each operation rounded once.
__device__ __forceinline__ float4 tri_centroid(const float v[9]) {
  return make_float4(__fdiv_rn(__fadd_rn(__fadd_rn(v[0], v[3]), v[6]), 3.0f),
                     __fdiv_rn(__fadd_rn(__fadd_rn(v[1], v[4]), v[7]), 3.0f),
                     __fdiv_rn(__fadd_rn(__fadd_rn(v[2], v[5]), v[8]), 3.0f), 0.0f);
}

// getTriangleBounds (gprt/development/gprt_lbvh.hlsl:121-129).
__device__ __forceinline__ void tri_box(const float v[9], float b[6]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    b[k] = fminf(v[k], fminf(v[3 + k], v[6 + k]));
    b[3 + k] = fmaxf(v[k], fmaxf(v[3 + k], v[6 + k]));
  }
}

__device__ __forceinline__ uint32_t spread10(uint32_t v) {
  v &= 0x3FFu;
  v = (v | (v << 16)) & 0xFF0000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

// Hilbert index of three 10-bit coordinates with the conventions of
// gprt/hilbert.h:179-235 (hilbert_c2i, nDims=3, nBits=10), level by level.
// Each level's 3-bit cell (x in bit 0) is Gray-differenced against the level
// above, rotated by the running rotation after XOR with the entry flip; the
// rotation advances by one plus the position of the cell's lowest set bit
// among bits 0..1.  The digits are then XORed with 0b010 below the top level
// and Gray-decoded.
__device__ __forceinline__ uint32_t hilbert3d(uint32_t x, uint32_t y, uint32_t z) {
  uint32_t index = 0, rotation = 0, flip = 0, up = 0;
#pragma unroll
  for (int L = 9; L >= 0; --L) {
    const uint32_t cell = ((x >> L) & 1u) | (((y >> L) & 1u) << 1) | (((z >> L) & 1u) << 2);
    uint32_t b = flip ^ (cell ^ up);
    up = cell;
    b = ((b >> rotation) | (b << (3 - rotation))) & 7u;
    index = (index << 3) | b;
    flip = 1u << rotation;
    const uint32_t low = b & (0u - b) & 3u;
    rotation += (low == 1u) ? 1u : (low == 2u) ? 2u : 0u;
    rotation += 1u;
    if (rotation >= 3u) rotation -= 3u;
  }
  index ^= 0x04924924u;
#pragma unroll
  for (int d = 1; d < 30; d *= 2) index ^= index >> d;
  return index;
}

// Normalise, scale, clamp, truncate: gprt/development/gprt_lbvh.hlsl:268-274.
__device__ __forceinline__ uint32_t quant10(float p, float lo, float hi) {
  float v = __fdiv_rn(__fsub_rn(p, lo), __fsub_rn(hi, lo));
  v = __fmul_rn(v, 1024.0f);
  v = fmaxf(v, 0.0f);
  v = fminf(v, 1023.0f);
  return (uint32_t)v;
}

// Meshes are consecutive primitive ranges [prim_off[m], prim_off[m+1]), each
// with at least one primitive.  Mesh m's arrays sit at fixed offsets inside
// the concatenated outputs, so every mesh's block is exactly what a build of
// that mesh alone produces:
//   codes, ids, leaves' triangles     at prim base b = prim_off[m]
//   nodes, aabbs (2 n_m - 1 entries)  at node base  2b - m
//   traversal nodes (n_m - 1)         at inner base  b - m
// A plain build is the single mesh [0, n) (prim_off == nullptr).
struct MeshMap {
  const uint32_t *prim_off;
  uint32_t meshes;
  uint32_t n;
  __device__ __forceinline__ uint32_t begin(uint32_t m) const { return prim_off ? __ldg(prim_off + m) : 0u; }
  __device__ __forceinline__ uint32_t count(uint32_t m) const {
    return prim_off ? __ldg(prim_off + m + 1) - __ldg(prim_off + m) : n;
  }
  // Mesh holding global primitive i: prim_off[m] <= i < prim_off[m+1].
  __device__ __forceinline__ uint32_t mesh_of_prim(uint64_t i) const {
    if (!prim_off) return 0;
    uint32_t lo = 0, hi = meshes;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (__ldg(prim_off + mid) <= i) lo = mid;
      else hi = mid;
    }
    return lo;
  }
  // Warp-cooperative form of that lookup, for primitives or inner nodes
  // (inner node g of mesh m: (b_m - m) <= g < (b_{m+1} - m - 1)), for the 32
  // consecutive elements e0 + lane (e0 the same on every lane; all 32 lanes
  // call): the largest m with off(m) <= e0 + lane, off(m) non-decreasing.
  // The warp brackets the mesh of e0 with 32 probes a round (three rounds
  // for 16,384 meshes, against a 14-load bisection per element), then every
  // lane counts the meshes that start within its reach by bisecting the next
  // 32 offsets with shuffles (one load per lane).
  template <class Off>
  __device__ __forceinline__ uint32_t warp_mesh_of(uint64_t e0, Off off) const {
    if (!prim_off) return 0;
    const int lane = threadIdx.x & 31;
    uint32_t lo = 0, hi = meshes;  // off(lo) <= e0 < off(hi), off(meshes) taken as infinite
    while (hi - lo > 1) {
      const uint32_t p = lo + (uint32_t)(((uint64_t)(hi - lo) * (uint32_t)(lane + 1)) / 33u);
      const bool probe = p > lo && p < hi;
      const bool le = probe && off(p) <= e0;
      const unsigned pass = __ballot_sync(FULL_MASK, le), fail = __ballot_sync(FULL_MASK, probe && !le);
      if (pass) lo = __shfl_sync(FULL_MASK, p, 31 - __clz(pass));
      if (fail) hi = __shfl_sync(FULL_MASK, p, __ffs(fail) - 1);
    }
    const uint64_t e = e0 + (uint64_t)lane;
    const uint32_t j = lo + 1 + (uint32_t)lane;
    const uint64_t v = j < meshes ? off(j) : ~0ull;
    int c = 0;  // meshes after lo that start at or before e
#pragma unroll
    for (int step = 16; step > 0; step >>= 1)
      if (__shfl_sync(FULL_MASK, v, c + step - 1) <= e) c += step;
    if (c == 31 && __shfl_sync(FULL_MASK, v, 31) <= e) c = 32;
    uint32_t m = lo + (uint32_t)c;
    if (c == 32)  // 32 or more meshes start within 32 elements (empty ranges): walk on
      while (m + 1 < meshes && off(m + 1) <= e) ++m;
    return m;
  }
  __device__ __forceinline__ uint32_t warp_mesh_of_prim(uint64_t i0) const {
    return warp_mesh_of(i0, [&](uint32_t m) -> uint64_t { return __ldg(prim_off + m); });
  }
  __device__ __forceinline__ uint32_t warp_mesh_of_inner(uint64_t g0) const {
    return warp_mesh_of(g0, [&](uint32_t m) -> uint64_t { return (uint64_t)__ldg(prim_off + m) - m; });
  }
};

// Edge endpoints (getEdgeBounds / getEdgeCentroid, gprt/development/
// gprt_lbvh.hlsl:112-119,131-136): v[0..2] = p1, v[3..5] = v[6..8] = p2.
__device__ __forceinline__ void load_edge(const float *pos, const uint32_t *edge, uint32_t id, float v[9]) {
  const uint32_t i0 = edge[2 * (size_t)id], i1 = edge[2 * (size_t)id + 1];
  const float *p0 = pos + 3 * (size_t)i0, *p1 = pos + 3 * (size_t)i1;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    v[k] = p0[k];
    v[3 + k] = v[6 + k] = p1[k];
  }
}

// KIND: 0 triangles (tri = uint3 indices), 1 points, 2 edges (tri = uint2
// indices), 3 boxes (pos = float[n][6] {lo, hi}, the AABBs of user primitives).
template <int KIND>
__device__ __forceinline__ void prim_box(const float *pos, const uint32_t *tri, uint64_t id, float v[9], float b[6]) {
  if (KIND == 3) {
#pragma unroll
    for (int k = 0; k < 6; ++k) b[k] = pos[6 * (size_t)id + k];
#pragma unroll
    for (int k = 0; k < 9; ++k) v[k] = 0.0f;
  } else if (KIND == 0) {
    load_tri(pos, tri, (uint32_t)id, v);
    tri_box(v, b);
  } else if (KIND == 2) {
    load_edge(pos, tri, (uint32_t)id, v);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      b[k] = fminf(v[k], v[3 + k]);
      b[3 + k] = fmaxf(v[k], v[3 + k]);
    }
  } else {
#pragma unroll
    for (int k = 0; k < 3; ++k) v[k] = v[3 + k] = v[6 + k] = b[k] = b[3 + k] = pos[3 * (size_t)id + k];
  }
}

// Scene box of each mesh (ComputeTriangleBounds, gprt/development/
// gprt_lbvh.hlsl:215-226).  Slot words hold order-preserving integer images:
// max of f2ord for the maxima, max of ~f2ord for the minima, so one zero fill
// initialises both.  One mesh: block reduction, one atomic per CTA and
// component.  Many meshes: warp reduction when the warp's primitives share a
// mesh, per-lane atomics at mesh boundaries.
// With cent (triangles whose build writes leaf-order triangles), each
// triangle's centroid (p1 + p2 + p3) / 3 is stored there in primitive order
// for k_codes, which then reads 16 coalesced bytes instead of gathering the
// triangle again (the refit overwrites the array later).
template <int KIND, bool BATCHED>
__global__ void __launch_bounds__(256) k_bounds(const float *pos, const uint32_t *tri, MeshMap mm, uint32_t *slots,
                                                float4 *cent) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t w[6] = {0, 0, 0, 0, 0, 0};
  const uint64_t total = ((uint64_t)mm.n + 31) & ~31ull;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const bool valid = i < mm.n;
    float v[9], t[6];
    uint32_t tw[6] = {0, 0, 0, 0, 0, 0};
    if (valid) {
      prim_box<KIND>(pos, tri, i, v, t);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        tw[k] = ~f2ord(t[k]);
        tw[3 + k] = f2ord(t[3 + k]);
      }
      if (KIND == 0 && cent) cent[i] = tri_centroid(v);
    }
    if (!BATCHED) {
#pragma unroll
      for (int k = 0; k < 6; ++k) w[k] = max(w[k], tw[k]);
    } else {
      const uint32_t mw = mm.warp_mesh_of_prim(i - (uint64_t)lane);
      const uint32_t m = valid ? mw : 0xFFFFFFFFu;
      const uint32_t m0 = __shfl_sync(FULL_MASK, m, 0);
      if (__all_sync(FULL_MASK, m == m0)) {
#pragma unroll
        for (int k = 0; k < 6; ++k)
          for (int o = 16; o > 0; o >>= 1) tw[k] = max(tw[k], __shfl_xor_sync(FULL_MASK, tw[k], o));
        if (lane < 6 && m0 != 0xFFFFFFFFu) atomicMax(&slots[6 * (size_t)m0 + lane], tw[lane]);
      } else if (valid) {
#pragma unroll
        for (int k = 0; k < 6; ++k) atomicMax(&slots[6 * (size_t)m + k], tw[k]);
      }
    }
  }
  if (!BATCHED) {
#pragma unroll
    for (int k = 0; k < 6; ++k)
      for (int o = 16; o > 0; o >>= 1) w[k] = max(w[k], __shfl_xor_sync(FULL_MASK, w[k], o));
    __shared__ uint32_t s[8][6];
    if (lane == 0)
      for (int k = 0; k < 6; ++k) s[warp][k] = w[k];
    __syncthreads();
    if (threadIdx.x < 6) {
      uint32_t mx = 0;
      for (int j = 0; j < (int)(blockDim.x >> 5); ++j) mx = max(mx, s[j][threadIdx.x]);
      atomicMax(&slots[threadIdx.x], mx);
    }
  }
}

// Codes of centroids (p1 + p2 + p3) / 3 (gprt/development/gprt_lbvh.hlsl:
// 139-146, 262-277), (p1 + p2) / 2 for edges (:131-136, 245-260), or of the
// points themselves, normalised to the mesh's
// box.  One mesh: codes[i] and ids[i] = i.  Many meshes: 64-bit sort keys
// (mesh << 32 | code) and mesh-local ids.
template <int KIND, bool BATCHED>
__global__ void __launch_bounds__(256) k_codes(const float *pos, const uint32_t *tri, MeshMap mm, const uint32_t *slots,
                                               int code_kind, uint32_t *codes, uint64_t *keys, uint32_t *ids,
                                               float *scene_out, const float4 *cent) {
  const uint64_t total = ((uint64_t)mm.n + 31) & ~31ull;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t m = BATCHED ? mm.warp_mesh_of_prim(i - (threadIdx.x & 31)) : 0u;
    if (i >= mm.n) continue;
    const uint32_t *sl = slots + 6 * (size_t)m;
    float lo[3], hi[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      lo[k] = fminf(3.402823466e38f, ord2f(~sl[k]));
      hi[k] = fmaxf(-3.402823466e38f, ord2f(sl[3 + k]));
    }
    const uint32_t b = BATCHED ? mm.begin(m) : 0u;
    if (scene_out && i == b)
      for (int k = 0; k < 3; ++k) {
        scene_out[6 * (size_t)m + k] = lo[k];
        scene_out[6 * (size_t)m + 3 + k] = hi[k];
      }
    float c[3];
    if (KIND == 0) {
      float4 c4;
      if (cent) {
        c4 = cent[i];
      } else {
        float v[9];
        load_tri(pos, tri, (uint32_t)i, v);
        c4 = tri_centroid(v);
      }
      c[0] = c4.x;
      c[1] = c4.y;
      c[2] = c4.z;
    } else if (KIND == 2) {
      float v[9];
      load_edge(pos, tri, (uint32_t)i, v);
#pragma unroll
      for (int k = 0; k < 3; ++k) c[k] = __fdiv_rn(__fadd_rn(v[k], v[3 + k]), 2.0f);
    } else if (KIND == 3) {
#pragma unroll
      for (int k = 0; k < 3; ++k) c[k] = __fmul_rn(__fadd_rn(pos[6 * (size_t)i + k], pos[6 * (size_t)i + 3 + k]), 0.5f);
    } else {
#pragma unroll
      for (int k = 0; k < 3; ++k) c[k] = pos[3 * (size_t)i + k];
    }
    const uint32_t x = quant10(c[0], lo[0], hi[0]), y = quant10(c[1], lo[1], hi[1]), z = quant10(c[2], lo[2], hi[2]);
    const uint32_t code = code_kind == 0 ? (spread10(x) | (spread10(y) << 1) | (spread10(z) << 2)) : hilbert3d(x, y, z);
    if (BATCHED) {
      keys[i] = ((uint64_t)m << 32) | code;
      ids[i] = (uint32_t)(i - b);
    } else {
      codes[i] = code;
      ids[i] = (uint32_t)i;
    }
  }
}

// Karras 2012 delta with the index tie-break (gprt/development/gprt_lbvh.hlsl:45-61),
// over one mesh's sorted codes (local indices; the 64-bit batched keys carry
// the code in their low word).
template <bool BATCHED>
__device__ __forceinline__ uint32_t code_at(const uint32_t *codes, const uint64_t *keys, uint64_t j) {
  return BATCHED ? (uint32_t)__ldg(reinterpret_cast<const unsigned long long *>(keys) + j) : __ldg(codes + j);
}
template <bool BATCHED>
__device__ __forceinline__ int kdelta(const uint32_t *codes, const uint64_t *keys, uint64_t base, int64_t n, int64_t i,
                                      uint32_t ci, int64_t j, uint32_t cmask) {
  if (j < 0 || j >= n) return -1;
  const uint32_t x = (ci ^ code_at<BATCHED>(codes, keys, base + j)) & cmask;
  if (x == 0) return __clz((uint32_t)i ^ (uint32_t)j) + 32;
  return __clz(x);
}

// determine_range + SplitNodes (gprt/development/gprt_lbvh.hlsl:64-103,
// 287-338), one thread per inner node, mesh-local indices.  Writes {left,
// right, -, -1} of the node, the parent field of both children, and the child
// references of the traversal node (inner child c -> c, leaf k -> ~k).
// If the sort before it gave up on a wait (sort_status non-zero), the codes
// are not sorted and could give overlapping ranges; every code then counts as
// equal, so the index tie-break alone shapes a valid tree and nothing after it
// reads out of bounds (the build reports the sort's error).
template <bool BATCHED>
__global__ void __launch_bounds__(256, 8) k_karras(const uint32_t *codes, const uint64_t *keys, MeshMap mm, int4 *nodes,
                                                Bvh2Node *bvh, const uint32_t *sort_status) {
  const uint32_t cmask = sort_status && ld_relaxed_u32(sort_status) != 0 ? 0u : 0xFFFFFFFFu;
  const uint64_t total_inner = (uint64_t)mm.n - mm.meshes;
  const uint64_t total = (total_inner + 31) & ~31ull;
  for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < total;
       g += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t m = BATCHED ? mm.warp_mesh_of_inner(g - (threadIdx.x & 31)) : 0u;
    if (g >= total_inner) continue;
    const uint64_t b = BATCHED ? mm.begin(m) : 0;
    const int64_t N = BATCHED ? mm.count(m) : mm.n;
    const uint64_t inner_base = b - m, node_base = 2 * b - m;
    const int64_t i = (int64_t)(g - inner_base);
    const uint32_t ci = code_at<BATCHED>(codes, keys, b + i);
#define KD(j) kdelta<BATCHED>(codes, keys, b, N, i, ci, (j), cmask)
    const int d = KD(i + 1) >= KD(i - 1) ? 1 : -1;
    const int dmin = KD(i - d);
    int64_t lmax = 2;
    while (KD(i + lmax * d) > dmin) lmax *= 2;
    int64_t l = 0;
    for (int64_t t = lmax >> 1; t >= 1; t >>= 1)
      if (KD(i + (l + t) * d) > dmin) l += t;
    const int64_t j = i + l * d;
    const int dnode = KD(j);
    int64_t s = 0;
    for (int k = 1;; ++k) {
      const int64_t t = (l + ((int64_t)1 << k) - 1) >> k;
      if (KD(i + (s + t) * d) > dnode) s += t;
      if (t == 1) break;
    }
#undef KD
    const int64_t split = i + s * d + min(d, 0);
    const int64_t first = d == 1 ? i : j, last = d == 1 ? j : i;
    const int64_t left = split, right = split + 1;
    const bool lleaf = left == first, rleaf = right == last;
    const int64_t lc = lleaf ? (N - 1) + left : left;
    const int64_t rc = rleaf ? (N - 1) + right : right;
    int *nd = reinterpret_cast<int *>(&nodes[node_base + i]);
    nd[0] = (int)lc;
    nd[1] = (int)rc;
    nd[3] = -1;
    if (i == 0) nd[2] = -1;  // root; other parents are written by the parent's thread
    reinterpret_cast<int *>(&nodes[node_base + lc])[2] = (int)i;
    reinterpret_cast<int *>(&nodes[node_base + rc])[2] = (int)i;
    if (bvh) {
      // child boxes not formed yet: all-ones words, which the refit's second
      // arrival waits to see replaced (no float box bound has this pattern)
      int4 *q = reinterpret_cast<int4 *>(&bvh[inner_base + i]);
      q[0] = make_int4(-1, -1, -1, -1);
      q[1] = make_int4(-1, -1, -1, -1);
      q[2] = make_int4(-1, -1, -1, -1);
      q[3] = make_int4(lleaf ? ~(int)left : (int)lc, rleaf ? ~(int)right : (int)rc, 0, 0);
    }
  }
}

// Leaf boxes and the bottom-up union (BuildTriangleHierarchy,
// gprt/development/gprt_lbvh.hlsl:400-428, with MakeNodes' +-1e38 start
// :279-285).  One thread per leaf (no grid-stride loop: a thread's walk up
// the tree is a chain of dependent L2 round trips, so the threads must not
// queue behind each other's walks); the second arrival at a node forms it.
// With traversal nodes, a child's box goes into its slot of the parent's
// node, whose words hold all-ones until then, and the arrival count is
// relaxed: the second arrival re-reads the sibling's slot from L2 until no
// word is all-ones (a bounded wait; the writer issued its stores before its
// count).  A release/acquire count instead made every walking thread wait
// for its earlier writes to reach L2 (membar: 41 % of the stalls; 67M
// triangles: build 17.6 -> 15.5 ms without it).  Without traversal nodes the
// sibling's box is read from the reference-layout array after an
// acquire-release count.
// The sibling's box from its slot of the parent's traversal node (L2, not
// L1); false while a word still holds the all-ones "not formed" pattern.
__device__ __forceinline__ bool refit_read_box(const float2 *o2, float *sb) {
  bool ready = true;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float2 t;
    asm volatile("ld.relaxed.gpu.global.v2.f32 {%0, %1}, [%2];" : "=f"(t.x), "=f"(t.y) : "l"(o2 + k) : "memory");
    sb[2 * k] = t.x;
    sb[2 * k + 1] = t.y;
    ready &= __float_as_uint(t.x) != 0xFFFFFFFFu && __float_as_uint(t.y) != 0xFFFFFFFFu;
  }
  return ready;
}
// Test hooks (set on the current device by gprtcuDebugRefitSkipLeaf and
// gprtcuDebugSetSpinBudget): the leaf in sorted slot c_refit_skip never
// stores its box, and the polls a second arrival makes before it gives up.
__constant__ int64_t c_refit_skip = -1;
__constant__ uint32_t c_refit_budget = DEFAULT_SPIN_BUDGET;

template <int KIND, bool BATCHED>
__global__ void __launch_bounds__(256, 8) k_refit(const float *pos, const uint32_t *tri, const uint32_t *ids,
                                               const uint64_t *keys, MeshMap mm, int4 *nodes, float *aabbs,
                                               Bvh2Node *bvh, float4 *leaf_tris, uint32_t *codes_out,
                                               uint32_t *arrivals, float *root_box, const uint32_t *sort_status) {
  // 32-bit indices throughout: n < 2^30, so node indices stay below 2^31
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= mm.n) return;
  // The scratch header sits a fixed distance before the arrival counters.
  auto lbvh_header = [&]() {
    const size_t slots = ((size_t)mm.meshes * 24 + 255) & ~(size_t)255;
    return reinterpret_cast<ScratchHeader *>(reinterpret_cast<char *>(arrivals) - slots - sizeof(ScratchHeader));
  };
  // A sort that gave up on a wait leaves ids (and keys) that are not a
  // permutation: each leaf then takes its own slot's primitive, so every read
  // stays in bounds, and the build reports the sort's error.
  const uint32_t sort_err = sort_status ? ld_relaxed_u32(sort_status) : 0u;
  if (sort_err && s == 0) record_error(lbvh_header(), sort_err);
  uint32_t m = 0;
  if (BATCHED) {
    if (keys && !sort_err) {
      const uint64_t key = keys[s];  // (mesh << 32 | code), sorted
      m = (uint32_t)(key >> 32);
      if (codes_out) codes_out[s] = (uint32_t)key;
    } else {
      m = mm.mesh_of_prim(s);  // refit of an existing batch: no keys
    }
  }
  const uint32_t b = BATCHED ? mm.begin(m) : 0u;
  const int N = BATCHED ? (int)mm.count(m) : (int)mm.n;
  const uint32_t inner_base = b - m, node_base = 2 * b - m;
  const int i = (int)(s - b);
  const uint32_t id = sort_err ? (uint32_t)i : ids[s];
  const bool hooked = (int64_t)s == c_refit_skip;
  // The parent (written by the topology kernel) and its node are loaded
  // before the primitive's gather, so the two chains of dependent loads
  // overlap instead of following each other (67M triangles in 16,384 meshes:
  // batched build 16.2 -> 15.9 ms; capped at 32 registers for full occupancy,
  // 14.9 ms, and the topology kernel likewise, 14.5 ms; 32-bit indices, no
  // spills at 32 registers, 14.0 ms).  Counting the arrival before the gather
  // as well measured no faster (14.6 ms).
  const int leaf = (N - 1) + i;
  int4 *nl = &nodes[node_base + leaf];
  int p = N == 1 ? -1 : reinterpret_cast<const int *>(nl)[2];
  int4 pn = make_int4(0, 0, -1, -1);
  if (p >= 0) pn = nodes[node_base + p];
  float v[9], bx[6];
  prim_box<KIND>(pos, tri, (uint64_t)b + id, v, bx);
  if (leaf_tris) {
    leaf_tris[3 * (size_t)s + 0] = make_float4(v[0], v[1], v[2], __uint_as_float(id));
    leaf_tris[3 * (size_t)s + 1] = make_float4(v[3], v[4], v[5], 0.0f);
    leaf_tris[3 * (size_t)s + 2] = make_float4(v[6], v[7], v[8], 0.0f);
  }
  *nl = make_int4(-1, -1, p, (int)id);
  if (aabbs)
    for (int k = 0; k < 6; ++k) aabbs[6 * (size_t)(node_base + leaf) + k] = bx[k];
  int child = leaf;
  while (p >= 0) {
    const int side = pn.x == child ? 0 : 1;
    // This child's box goes into its slot of the parent's traversal node (or
    // is already in the reference-layout array); the release half of the
    // arrival count publishes it.
    // (a hooked leaf, at its first step, leaves its slot unwritten)
    const bool skip_store = hooked && child == leaf;
    if (bvh && !skip_store) {
      float2 *cb = reinterpret_cast<float2 *>(bvh[inner_base + p].box + 6 * side);
      cb[0] = make_float2(bx[0], bx[1]);
      cb[1] = make_float2(bx[2], bx[3]);
      cb[2] = make_float2(bx[4], bx[5]);
    }
    // first arrival: the sibling finishes
    if (bvh) {
      if (atomicAdd(&arrivals[inner_base + p], 1u) == 0) break;
    } else {
      if (atom_add_acq_rel_u32(&arrivals[inner_base + p], 1u) == 0) break;
    }
    // Second arrival: read the sibling's box from L2 and form the union,
    // starting from +-1e38 exactly as MakeNodes initialises inner boxes.
    // (A hooked leaf arriving second waits on its own unwritten slot, so the
    // wait below runs out whichever child arrives first.)
    const int sib = side == 0 ? pn.y : pn.x;
    const int rd = skip_store ? side : 1 - side;
    // the next parent's node, loaded while the sibling's box is read
    int4 gpn = make_int4(0, 0, -1, -1);
    if (pn.z >= 0) gpn = nodes[node_base + pn.z];
    const float *ob = bvh ? bvh[inner_base + p].box + 6 * rd : aabbs + 6 * (size_t)(node_base + sib);
    float sb[6];
    if (bvh) {
      // bounded wait for the sibling's stores; a wait that runs out records
      // GPRTCU_ERR_TIMEOUT in the scratch header
      for (uint32_t spin = 0; !refit_read_box(reinterpret_cast<const float2 *>(ob), sb); ++spin)
        if (spin == c_refit_budget) {
          record_error(lbvh_header(), GPRTCU_ERR_TIMEOUT);
          break;
        }
    } else {
#pragma unroll
      for (int k = 0; k < 6; ++k) sb[k] = __ldcg(ob + k);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      bx[k] = fminf(1e38f, fminf(bx[k], sb[k]));
      bx[3 + k] = fmaxf(-1e38f, fmaxf(bx[3 + k], sb[3 + k]));
    }
    if (aabbs)
      for (int k = 0; k < 6; ++k) aabbs[6 * (size_t)(node_base + p) + k] = bx[k];
    child = p;
    p = pn.z;
    pn = gpn;
  }
  if (p < 0 && child == 0 && root_box)
    for (int k = 0; k < 6; ++k) root_box[6 * (size_t)m + k] = bx[k];
}

}  // namespace gprtcu

using namespace gprtcu;


namespace {

int grid_for(uint64_t n, int threads, int per_sm) {
  uint64_t g = (n + threads - 1) / threads;
  uint64_t cap = (uint64_t)gprtcu_num_sms() * per_sm;
  if (g > cap) g = cap;
  return (int)(g ? g : 1);
}

struct LbvhScratch {
  size_t slots, arrivals, keys, sort, total;
};

LbvhScratch lbvh_scratch_layout(uint64_t n, uint32_t meshes) {
  LbvhScratch L;
  size_t off = sizeof(ScratchHeader);
  L.slots = off;
  off += gprtcu_align256((size_t)meshes * 6 * 4);
  L.arrivals = off;
  off += gprtcu_align256((size_t)(n > meshes ? n - meshes : 1) * 4);
  L.keys = off;
  if (meshes > 1) off += gprtcu_align256((size_t)n * 8);
  L.sort = off;
  off += meshes > 1 ? gprtcuSortScratchSize(n, 8, 4) : gprtcuSortScratchSize(n, 4, 4);
  L.total = off;
  return L;
}

int ceil_log2(uint32_t v) {
  int b = 0;
  while ((1ull << b) < v) ++b;
  return b;
}

template <int KIND, bool BATCHED>
void launch_build(const float *pos, const uint32_t *tri, MeshMap mm, int codeKind, gprtcuLbvh *out, uint32_t *slots,
                  uint64_t *keys, uint32_t *arrivals, const uint32_t *sort_status, cudaStream_t stream, int stage) {
  const int g = grid_for(mm.n, 256, 8);
  int4 *nodes = (int4 *)out->nodes;
  if (stage == 0) {
    // the centroids pass through the leaf-order triangle array, which the
    // refit overwrites afterwards
    float4 *cent = KIND == 0 ? (float4 *)out->leafTris : nullptr;
    k_bounds<KIND, BATCHED><<<g, 256, 0, stream>>>(pos, tri, mm, slots, cent);
    k_codes<KIND, BATCHED><<<g, 256, 0, stream>>>(pos, tri, mm, slots, codeKind, out->codes, keys, out->ids,
                                                  out->sceneBounds, cent);
  } else {
    if (mm.n > mm.meshes)
      k_karras<BATCHED><<<(unsigned)((mm.n - mm.meshes + 255) / 256), 256, 0, stream>>>(out->codes, keys, mm, nodes,
                                                                                         (Bvh2Node *)out->bvh2,
                                                                                         sort_status);
    // traversal nodes for triangles and user-primitive boxes; leaf-order
    // triangles for triangles only
    k_refit<KIND, BATCHED><<<(unsigned)((mm.n + 255) / 256), 256, 0, stream>>>(
        pos, tri, out->ids, keys, mm, nodes, out->aabbs, (KIND == 0 || KIND == 3) ? (Bvh2Node *)out->bvh2 : nullptr,
        KIND == 0 ? (float4 *)out->leafTris : nullptr, out->codes, arrivals, out->rootBox, sort_status);
  }
}

gprtcuStatus lbvh_build(int kind, const float *pos, const uint32_t *tri, const uint32_t *prim_off, uint32_t meshes,
                        uint32_t n, int codeKind, gprtcuLbvh *out, void *scratch, size_t scratchBytes,
                        cudaStream_t stream) {
  if (!out || !pos || ((kind == 0 || kind == 2) && !tri)) return GPRTCU_ERR_INVALID_ARG;
  if (kind >= 2 && meshes > 1) return GPRTCU_ERR_INVALID_ARG;
  if (n == 0 || meshes == 0 || meshes > n) return GPRTCU_ERR_INVALID_ARG;
  if (meshes > 1 && !prim_off) return GPRTCU_ERR_INVALID_ARG;
  if (n > (1u << 30) - 1) return GPRTCU_ERR_TOO_LARGE;
  if (!out->codes || !out->ids || !out->nodes) return GPRTCU_ERR_INVALID_ARG;
  if (n > meshes && !out->aabbs && ((kind != 0 && kind != 3) || !out->bvh2)) return GPRTCU_ERR_INVALID_ARG;
  if (out->bvh2 && ((uintptr_t)out->bvh2 & 15)) return GPRTCU_ERR_INVALID_ARG;
  if (out->leafTris && ((uintptr_t)out->leafTris & 15)) return GPRTCU_ERR_INVALID_ARG;
  if (codeKind != 0 && codeKind != 1) return GPRTCU_ERR_INVALID_ARG;
  if (!scratch || ((uintptr_t)scratch & 255)) return GPRTCU_ERR_INVALID_ARG;
  const LbvhScratch L = lbvh_scratch_layout(n, meshes);
  if (scratchBytes < L.total) return GPRTCU_ERR_SCRATCH_TOO_SMALL;
  char *s = (char *)scratch;
  out->numPrims = n;
  GPRTCU_TRY(cudaMemsetAsync(s, 0, L.keys, stream));  // header, bound slots, arrival counters
  uint32_t *slots = (uint32_t *)(s + L.slots);
  uint32_t *arrivals = (uint32_t *)(s + L.arrivals);
  uint64_t *keys = meshes > 1 ? (uint64_t *)(s + L.keys) : nullptr;
  const MeshMap mm{meshes > 1 ? prim_off : nullptr, meshes, n};
  const bool batched = meshes > 1;
  const uint32_t *sort_status = (const uint32_t *)(s + L.sort);  // the sort's own header: its error status first
  for (int stage = 0; stage < 2; ++stage) {
    if (stage == 1) {
      gprtcuStatus st = batched ? gprtcuSortPairsU64(keys, out->ids, n, 0, 32 + (ceil_log2(meshes) > 0 ? ceil_log2(meshes) : 1),
                                                     s + L.sort, scratchBytes - L.sort, (gprtcuStream)stream)
                                : gprtcuSortPairsU32(out->codes, out->ids, n, 0, 30, s + L.sort, scratchBytes - L.sort,
                                                     (gprtcuStream)stream);
      if (st != GPRTCU_OK) return st;
    }
    if (kind == 0 && batched) launch_build<0, true>(pos, tri, mm, codeKind, out, slots, keys, arrivals, sort_status, stream, stage);
    else if (kind == 0) launch_build<0, false>(pos, tri, mm, codeKind, out, slots, keys, arrivals, sort_status, stream, stage);
    else if (kind == 2) launch_build<2, false>(pos, tri, mm, codeKind, out, slots, keys, arrivals, sort_status, stream, stage);
    else if (kind == 3) launch_build<3, false>(pos, tri, mm, codeKind, out, slots, keys, arrivals, sort_status, stream, stage);
    else if (batched) launch_build<1, true>(pos, tri, mm, codeKind, out, slots, keys, arrivals, sort_status, stream, stage);
    else launch_build<1, false>(pos, tri, mm, codeKind, out, slots, keys, arrivals, sort_status, stream, stage);
    GPRTCU_TRY(cudaGetLastError());
  }
  return GPRTCU_OK;
}

}  // namespace

extern "C" GPRTCU_API size_t gprtcuLbvhScratchSize(uint32_t n) { return lbvh_scratch_layout(n, 1).total; }

extern "C" GPRTCU_API gprtcuStatus gprtcuLbvhBuildTriangles(const float *positions, const uint32_t *triangles,
                                                            uint32_t numTriangles, int codeKind, gprtcuLbvh *bvh,
                                                            void *scratch, size_t scratchBytes, gprtcuStream stream) {
  return lbvh_build(0, positions, triangles, nullptr, 1, numTriangles, codeKind, bvh, scratch, scratchBytes,
                    (cudaStream_t)stream);
}

extern "C" GPRTCU_API gprtcuStatus gprtcuLbvhBuildPoints(const float *positions, uint32_t numPoints, int codeKind,
                                                         gprtcuLbvh *bvh, void *scratch, size_t scratchBytes,
                                                         gprtcuStream stream) {
  return lbvh_build(1, positions, nullptr, nullptr, 1, numPoints, codeKind, bvh, scratch, scratchBytes,
                    (cudaStream_t)stream);
}

extern "C" GPRTCU_API gprtcuStatus gprtcuLbvhBuildEdges(const float *positions, const uint32_t *edges,
                                                        uint32_t numEdges, int codeKind, gprtcuLbvh *bvh, void *scratch,
                                                        size_t scratchBytes, gprtcuStream stream) {
  return lbvh_build(2, positions, edges, nullptr, 1, numEdges, codeKind, bvh, scratch, scratchBytes,
                    (cudaStream_t)stream);
}

extern "C" GPRTCU_API gprtcuStatus gprtcuLbvhBuildBoxes(const float *aabbs, uint32_t numBoxes, int codeKind,
                                                        gprtcuLbvh *bvh, void *scratch, size_t scratchBytes,
                                                        gprtcuStream stream) {
  return lbvh_build(3, aabbs, nullptr, nullptr, 1, numBoxes, codeKind, bvh, scratch, scratchBytes,
                    (cudaStream_t)stream);
}

// Refit of an existing triangle LBVH (one mesh, or a batch when triOffsets is
// given) after its vertices moved: the topology and the leaf order are kept,
// the leaf-order triangles, the traversal nodes' boxes and the reference-
// layout boxes are recomputed bottom-up.
extern "C" GPRTCU_API gprtcuStatus gprtcuLbvhRefitTriangles(const float *positions, const uint32_t *triangles,
                                                            const uint32_t *triOffsets, uint32_t numMeshes,
                                                            gprtcuLbvh *bvh, void *scratch, size_t scratchBytes,
                                                            gprtcuStream stream_) {
  cudaStream_t stream = (cudaStream_t)stream_;
  if (!bvh || !positions || !triangles || numMeshes == 0 || (numMeshes > 1 && !triOffsets)) return GPRTCU_ERR_INVALID_ARG;
  const uint32_t n = bvh->numPrims;
  if (n == 0 || numMeshes > n || !bvh->ids || !bvh->nodes) return GPRTCU_ERR_INVALID_ARG;
  if (n > numMeshes && !bvh->aabbs && !bvh->bvh2) return GPRTCU_ERR_INVALID_ARG;
  if (!scratch || ((uintptr_t)scratch & 255)) return GPRTCU_ERR_INVALID_ARG;
  const LbvhScratch L = lbvh_scratch_layout(n, numMeshes);
  if (scratchBytes < L.keys) return GPRTCU_ERR_SCRATCH_TOO_SMALL;
  char *s = (char *)scratch;
  GPRTCU_TRY(cudaMemsetAsync(s, 0, L.keys, stream));  // header and arrival counters
  uint32_t *arrivals = (uint32_t *)(s + L.arrivals);
  const MeshMap mm{numMeshes > 1 ? triOffsets : nullptr, numMeshes, n};
  // the traversal nodes' child boxes back to all-ones (the refit waits for them to change)
  if (bvh->bvh2 && n > numMeshes)
    GPRTCU_TRY(cudaMemset2DAsync(bvh->bvh2, sizeof(Bvh2Node), 0xFF, 12 * sizeof(float), n - numMeshes, stream));
  const unsigned grid = (unsigned)((n + 255) / 256);
  if (numMeshes > 1)
    k_refit<0, true><<<grid, 256, 0, stream>>>(positions, triangles, bvh->ids, nullptr, mm, (int4 *)bvh->nodes,
                                               bvh->aabbs, (Bvh2Node *)bvh->bvh2, (float4 *)bvh->leafTris, nullptr,
                                               arrivals, bvh->rootBox, nullptr);
  else
    k_refit<0, false><<<grid, 256, 0, stream>>>(positions, triangles, bvh->ids, nullptr, mm, (int4 *)bvh->nodes,
                                                bvh->aabbs, (Bvh2Node *)bvh->bvh2, (float4 *)bvh->leafTris, nullptr,
                                                arrivals, bvh->rootBox, nullptr);
  GPRTCU_TRY(cudaGetLastError());
  return GPRTCU_OK;
}

extern "C" GPRTCU_API size_t gprtcuBatchScratchSize(uint32_t numMeshes, uint32_t totalTriangles) {
  return lbvh_scratch_layout(totalTriangles, numMeshes).total;
}

extern "C" GPRTCU_API gprtcuStatus gprtcuBatchBuildTriangles(const float *positions, const uint32_t *triangles,
                                                             const uint32_t *triOffsets, uint32_t numMeshes,
                                                             uint32_t totalTriangles, int codeKind, gprtcuLbvh *bvh,
                                                             void *scratch, size_t scratchBytes, gprtcuStream stream) {
  return lbvh_build(0, positions, triangles, triOffsets, numMeshes, totalTriangles, codeKind, bvh, scratch,
                    scratchBytes, (cudaStream_t)stream);
}

extern "C" GPRTCU_API gprtcuStatus gprtcuDebugRefitSkipLeaf(int64_t slot) {
  GPRTCU_TRY(cudaMemcpyToSymbol(c_refit_skip, &slot, sizeof(slot)));
  return GPRTCU_OK;
}

// Called by gprtcuDebugSetSpinBudget (scan.cu): the refit's waits follow it.
gprtcuStatus gprtcu_refit_set_budget(uint32_t polls) {
  GPRTCU_TRY(cudaMemcpyToSymbol(c_refit_budget, &polls, sizeof(polls)));
  return GPRTCU_OK;
}
