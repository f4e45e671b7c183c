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

// getTriangleBounds (gprt/development/gprt_lbvh.hlsl:121-129).
__device__ __forceinline__ void tri_box(const float v[9], float b[6]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    b[k] = fminf(v[k], fminf(v[3 + k], v[6 + k]));
    b[3 + k] = fmaxf(v[k], fmaxf(v[3 + k], v[6 + k]));
  }
}

// Scene box.  Slot words hold order-preserving images: max of f2ord for the
// maxima, max of ~f2ord for the minima, so one zero fill initialises both.
template <int KIND>  // 0 triangles, 1 points
__global__ void __launch_bounds__(256) k_bounds(const float *pos, const uint32_t *tri, uint32_t n, uint32_t *slots) {
  float b[6] = {3.402823466e38f, 3.402823466e38f, 3.402823466e38f, -3.402823466e38f, -3.402823466e38f,
                -3.402823466e38f};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float t[6];
    if (KIND == 0) {
      float v[9];
      load_tri(pos, tri, i, v);
      tri_box(v, t);
    } else {
      const float *p = pos + 3 * (size_t)i;
      t[0] = t[3] = p[0];
      t[1] = t[4] = p[1];
      t[2] = t[5] = p[2];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      b[k] = fminf(b[k], t[k]);
      b[3 + k] = fmaxf(b[3 + k], t[3 + k]);
    }
  }
  uint32_t w[6];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    w[k] = ~f2ord(b[k]);
    w[3 + k] = f2ord(b[3 + k]);
  }
#pragma unroll
  for (int k = 0; k < 6; ++k)
    for (int o = 16; o > 0; o >>= 1) w[k] = max(w[k], __shfl_xor_sync(FULL_MASK, w[k], o));
  __shared__ uint32_t s[8][6];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
    for (int k = 0; k < 6; ++k) s[warp][k] = w[k];
  __syncthreads();
  if (threadIdx.x < 6) {
    uint32_t m = 0;
    for (int j = 0; j < (int)(blockDim.x >> 5); ++j) m = max(m, s[j][threadIdx.x]);
    atomicMax(&slots[threadIdx.x], m);
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

// Codes of centroids (p1 + p2 + p3) / 3 (gprt/development/gprt_lbvh.hlsl:
// 139-146, 262-277), or of the points themselves; ids[i] = i.
template <int KIND>
__global__ void __launch_bounds__(256) k_codes(const float *pos, const uint32_t *tri, uint32_t n, const uint32_t *slots,
                                               int code_kind, uint32_t *codes, uint32_t *ids, float *scene_out) {
  float lo[3], hi[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    lo[k] = fminf(3.402823466e38f, ord2f(~slots[k]));
    hi[k] = fmaxf(-3.402823466e38f, ord2f(slots[3 + k]));
  }
  if (blockIdx.x == 0 && threadIdx.x < 6 && scene_out) scene_out[threadIdx.x] = threadIdx.x < 3 ? lo[threadIdx.x] : hi[threadIdx.x - 3];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float c[3];
    if (KIND == 0) {
      float v[9];
      load_tri(pos, tri, i, v);
#pragma unroll
      for (int k = 0; k < 3; ++k) c[k] = __fdiv_rn(__fadd_rn(__fadd_rn(v[k], v[3 + k]), v[6 + k]), 3.0f);
    } else {
#pragma unroll
      for (int k = 0; k < 3; ++k) c[k] = pos[3 * (size_t)i + k];
    }
    const uint32_t x = quant10(c[0], lo[0], hi[0]), y = quant10(c[1], lo[1], hi[1]), z = quant10(c[2], lo[2], hi[2]);
    codes[i] = code_kind == 0 ? (spread10(x) | (spread10(y) << 1) | (spread10(z) << 2)) : hilbert3d(x, y, z);
    ids[i] = i;
  }
}

// Karras 2012 delta with the index tie-break (gprt/development/gprt_lbvh.hlsl:45-61).
__device__ __forceinline__ int kdelta(const uint32_t *codes, int64_t n, int64_t i, uint32_t ci, int64_t j) {
  if (j < 0 || j >= n) return -1;
  const uint32_t x = ci ^ __ldg(&codes[j]);
  if (x == 0) return __clz((uint32_t)i ^ (uint32_t)j) + 32;
  return __clz(x);
}

// determine_range + SplitNodes (gprt/development/gprt_lbvh.hlsl:64-103,
// 287-338), one thread per inner node.  Writes {left, right, -, -1} of the
// node, the parent field of both children, and the child references of the
// traversal node (inner child c -> c, leaf k -> ~k).
__global__ void __launch_bounds__(256) k_karras(const uint32_t *codes, uint32_t n, int4 *nodes, Bvh2Node *bvh) {
  const int64_t N = n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N - 1; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t ci = codes[i];
    const int d = kdelta(codes, N, i, ci, i + 1) >= kdelta(codes, N, i, ci, i - 1) ? 1 : -1;
    const int dmin = kdelta(codes, N, i, ci, i - d);
    int64_t lmax = 2;
    while (kdelta(codes, N, i, ci, i + lmax * d) > dmin) lmax *= 2;
    int64_t l = 0;
    for (int64_t t = lmax >> 1; t >= 1; t >>= 1)
      if (kdelta(codes, N, i, ci, i + (l + t) * d) > dmin) l += t;
    const int64_t j = i + l * d;
    const int dnode = kdelta(codes, N, i, ci, j);
    int64_t s = 0;
    for (int k = 1;; ++k) {
      const int64_t t = (l + ((int64_t)1 << k) - 1) >> k;
      if (kdelta(codes, N, i, ci, i + (s + t) * d) > dnode) s += t;
      if (t == 1) break;
    }
    const int64_t split = i + s * d + min(d, 0);
    const int64_t first = d == 1 ? i : j, last = d == 1 ? j : i;
    const int64_t left = split, right = split + 1;
    const bool lleaf = left == first, rleaf = right == last;
    const int64_t lc = lleaf ? (N - 1) + left : left;
    const int64_t rc = rleaf ? (N - 1) + right : right;
    int4 nd;
    nd.x = (int)lc;
    nd.y = (int)rc;
    nd.z = -1;  // overwritten by the parent's thread (root stays -1)
    nd.w = -1;
    // x, y, w of this node; z belongs to the parent's thread.
    reinterpret_cast<int *>(&nodes[i])[0] = nd.x;
    reinterpret_cast<int *>(&nodes[i])[1] = nd.y;
    reinterpret_cast<int *>(&nodes[i])[3] = -1;
    if (i == 0) reinterpret_cast<int *>(&nodes[0])[2] = -1;
    reinterpret_cast<int *>(&nodes[lc])[2] = (int)i;
    reinterpret_cast<int *>(&nodes[rc])[2] = (int)i;
    if (bvh) {
      bvh[i].ref[0] = lleaf ? ~(int)left : (int)lc;
      bvh[i].ref[1] = rleaf ? ~(int)right : (int)rc;
    }
  }
}

// Leaf boxes and the bottom-up union (BuildTriangleHierarchy,
// gprt/development/gprt_lbvh.hlsl:400-428, with MakeNodes' +-1e38 start
// :279-285).  One thread per leaf; the second arrival at a node forms it.
template <int KIND>
__global__ void __launch_bounds__(256) k_refit(const float *pos, const uint32_t *tri, const uint32_t *ids, uint32_t n,
                                               int4 *nodes, float *aabbs, Bvh2Node *bvh, float4 *leaf_tris,
                                               uint32_t *arrivals, float *root_box) {
  const int64_t N = n, inner = N - 1;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t id = ids[i];
    float v[9], b[6];
    if (KIND == 0) {
      load_tri(pos, tri, id, v);
      tri_box(v, b);
    } else {
#pragma unroll
      for (int k = 0; k < 3; ++k) v[k] = v[3 + k] = v[6 + k] = b[k] = b[3 + k] = pos[3 * (size_t)id + k];
    }
    const int64_t leaf = inner + i;
    if (leaf_tris) {
      leaf_tris[3 * i + 0] = make_float4(v[0], v[1], v[2], __uint_as_float(id));
      leaf_tris[3 * i + 1] = make_float4(v[3], v[4], v[5], 0.0f);
      leaf_tris[3 * i + 2] = make_float4(v[6], v[7], v[8], 0.0f);
    }
    int *nl = reinterpret_cast<int *>(&nodes[leaf]);
    nl[0] = -1;
    nl[1] = -1;
    nl[3] = (int)id;
    if (N == 1) nl[2] = -1;
    if (aabbs)
      for (int k = 0; k < 6; ++k) aabbs[6 * leaf + k] = b[k];
    int64_t child = leaf;
    int64_t p = N == 1 ? -1 : (int64_t)ld_relaxed_u32(reinterpret_cast<const uint32_t *>(nl + 2));
    while (p >= 0) {
      const int side = (ld_relaxed_u32(reinterpret_cast<const uint32_t *>(&nodes[p])) == (uint32_t)child) ? 0 : 1;
      // This child's box goes into its slot of the parent's traversal node
      // (or is already in the reference-layout array); publish it before
      // counting the arrival.
      if (bvh) {
        float *cb = bvh[p].box + 6 * side;
#pragma unroll
        for (int k = 0; k < 6; ++k) cb[k] = b[k];
      }
      __threadfence();
      if (atomicAdd(&arrivals[p], 1u) == 0) break;  // first arrival: the sibling finishes the node
      __threadfence();
      // Second arrival: read the sibling's box (from L2) and form the union,
      // starting from +-1e38 exactly as MakeNodes initialises inner boxes.
      float sb[6];
      const float *ob = bvh ? bvh[p].box + 6 * (1 - side)
                            : aabbs + 6 * (int64_t)(side == 0 ? nodes[p].y : nodes[p].x);
#pragma unroll
      for (int k = 0; k < 6; ++k) sb[k] = __ldcg(ob + k);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        b[k] = fminf(1e38f, fminf(b[k], sb[k]));
        b[3 + k] = fmaxf(-1e38f, fmaxf(b[3 + k], sb[3 + k]));
      }
      if (aabbs)
        for (int k = 0; k < 6; ++k) aabbs[6 * p + k] = b[k];
      child = p;
      p = (int64_t)(int)ld_relaxed_u32(reinterpret_cast<const uint32_t *>(&nodes[p]) + 2);
    }
    if (p < 0 && child == 0 && root_box) {
      for (int k = 0; k < 6; ++k) root_box[k] = b[k];
    }
  }
}

}  // namespace gprtcu

using namespace gprtcu;

namespace {

struct LbvhScratch {
  size_t slots, arrivals, sort, total;
};

LbvhScratch lbvh_scratch_layout(uint32_t n) {
  LbvhScratch L;
  size_t off = sizeof(ScratchHeader);
  L.slots = off;
  off += 256;
  L.arrivals = off;
  off += gprtcu_align256((size_t)(n > 1 ? n - 1 : 1) * 4);
  L.sort = off;
  off += gprtcuSortScratchSize(n, 4, 4);
  L.total = off;
  return L;
}

int grid_for(uint64_t n, int threads, int per_sm) {
  uint64_t g = (n + threads - 1) / threads;
  uint64_t cap = (uint64_t)gprtcu_num_sms() * per_sm;
  if (g > cap) g = cap;
  return (int)(g ? g : 1);
}

gprtcuStatus lbvh_build(int kind, const float *pos, const uint32_t *tri, uint32_t n, int codeKind, gprtcuLbvh *out,
                        void *scratch, size_t scratchBytes, cudaStream_t stream) {
  if (!out || !pos || (kind == 0 && !tri)) return GPRTCU_ERR_INVALID_ARG;
  if (n == 0) return GPRTCU_ERR_INVALID_ARG;
  if (n > (1u << 30) - 1) return GPRTCU_ERR_TOO_LARGE;
  if (!out->codes || !out->ids || !out->nodes) return GPRTCU_ERR_INVALID_ARG;
  if (n > 1 && !out->aabbs && !out->bvh2) return GPRTCU_ERR_INVALID_ARG;  // the refit needs one box store
  if (out->bvh2 && ((uintptr_t)out->bvh2 & 15)) return GPRTCU_ERR_INVALID_ARG;
  if (out->leafTris && ((uintptr_t)out->leafTris & 15)) return GPRTCU_ERR_INVALID_ARG;
  if (codeKind != 0 && codeKind != 1) return GPRTCU_ERR_INVALID_ARG;
  if (!scratch || ((uintptr_t)scratch & 255)) return GPRTCU_ERR_INVALID_ARG;
  LbvhScratch L = lbvh_scratch_layout(n);
  if (scratchBytes < L.total) return GPRTCU_ERR_SCRATCH_TOO_SMALL;
  char *s = (char *)scratch;
  out->numPrims = n;
  GPRTCU_TRY(cudaMemsetAsync(s, 0, L.sort, stream));  // header, bound slots, arrival counters
  uint32_t *slots = (uint32_t *)(s + L.slots);
  uint32_t *arrivals = (uint32_t *)(s + L.arrivals);
  int4 *nodes = (int4 *)out->nodes;
  Bvh2Node *bvh = (Bvh2Node *)out->bvh2;
  float4 *leafTris = (float4 *)out->leafTris;
  const int g = grid_for(n, 256, 8);
  if (kind == 0) {
    k_bounds<0><<<g, 256, 0, stream>>>(pos, tri, n, slots);
    k_codes<0><<<g, 256, 0, stream>>>(pos, tri, n, slots, codeKind, out->codes, out->ids, out->sceneBounds);
  } else {
    k_bounds<1><<<g, 256, 0, stream>>>(pos, tri, n, slots);
    k_codes<1><<<g, 256, 0, stream>>>(pos, tri, n, slots, codeKind, out->codes, out->ids, out->sceneBounds);
  }
  GPRTCU_TRY(cudaGetLastError());
  gprtcuStatus st = gprtcuSortPairsU32(out->codes, out->ids, n, 0, 30, s + L.sort, scratchBytes - L.sort,
                                       (gprtcuStream)stream);
  if (st != GPRTCU_OK) return st;
  if (n > 1) {
    k_karras<<<grid_for(n - 1, 256, 8), 256, 0, stream>>>(out->codes, n, nodes, bvh);
    GPRTCU_TRY(cudaGetLastError());
  }
  if (kind == 0)
    k_refit<0><<<g, 256, 0, stream>>>(pos, tri, out->ids, n, nodes, out->aabbs, bvh, leafTris, arrivals,
                                      out->rootBox);
  else
    k_refit<1><<<g, 256, 0, stream>>>(pos, tri, out->ids, n, nodes, out->aabbs, bvh, leafTris, arrivals,
                                      out->rootBox);
  GPRTCU_TRY(cudaGetLastError());
  return GPRTCU_OK;
}

}  // namespace

extern "C" GPRTCU_API size_t gprtcuLbvhScratchSize(uint32_t n) { return lbvh_scratch_layout(n).total; }

extern "C" GPRTCU_API gprtcuStatus gprtcuLbvhBuildTriangles(const float *positions, const uint32_t *triangles,
                                                            uint32_t numTriangles, int codeKind, gprtcuLbvh *bvh,
                                                            void *scratch, size_t scratchBytes, gprtcuStream stream) {
  return lbvh_build(0, positions, triangles, numTriangles, codeKind, bvh, scratch, scratchBytes, (cudaStream_t)stream);
}

extern "C" GPRTCU_API gprtcuStatus gprtcuLbvhBuildPoints(const float *positions, uint32_t numPoints, int codeKind,
                                                         gprtcuLbvh *bvh, void *scratch, size_t scratchBytes,
                                                         gprtcuStream stream) {
  return lbvh_build(1, positions, nullptr, numPoints, codeKind, bvh, scratch, scratchBytes, (cudaStream_t)stream);
}
