// wide.cu -- 8-wide BVH with 8-bit quantised child boxes, collapsed from the
// binary LBVH, and its closest-hit / any-hit traversal.  No counterpart in
// the reference (its traversal is Vulkan ray-tracing hardware); the node
// format follows the compressed-wide-BVH idea of Ylitie, Karras, Laine 2017
// ("Efficient Incoherent Ray Traversal on GPUs Through Compressed Wide
// BVHs"), written here for this build.
//
// Node (80 bytes, five 16-byte loads):
//   p.xyz      fp32 origin = min corner of the children's union box
//   e.xyz      int8 scale exponents, scale s = 2^e per axis, chosen (in FP64)
//              as the smallest power of two with 255 * s >= extent
//   imask      bit c: child slot c is an inner node
//   child_base first inner child's node index (inner children contiguous)
//   leaf_base  first leaf child's index in the wide leaf array (contiguous)
//   meta[c]    0xFF empty; else the child's rank among the inner (imask) or
//              leaf children
//   qlo/qhi    per axis, per child: floor((lo - p) / s), ceil((hi - p) / s);
//              an empty slot holds the inverted box qlo 255, qhi 0
// Decoding uses round-down (lo) and round-up (hi) FMAs, so every decoded box
// contains its exact fp32 child box; a ray therefore never misses a child the
// binary traversal would enter, and intersection is the same FP32 watertight
// test, giving the same hits.  A node is 80 bytes for up to eight children
// against 64 bytes for two in the binary layout.
#include "common.cuh"
#include "lbvh.cuh"
#include "rtmath.cuh"

namespace gprtcu {

struct __align__(16) WideNode {
  float px, py, pz;
  int8_t ex, ey, ez;
  uint8_t imask;
  uint32_t child_base;
  uint32_t leaf_base;
  uint8_t meta[8];
  uint8_t qlo[3][8];
  uint8_t qhi[3][8];
};
static_assert(sizeof(WideNode) == 80, "80-byte wide node");

struct WorkItem {
  uint32_t mesh;
  int32_t bref;  // binary inner node (mesh-local) or ~slot for a one-leaf mesh
};

// Collapse counters: the current level's items are queue[LO, HI); TAIL is
// the next free queue slot (= the number of wide nodes so far: a wide node's
// index is its queue slot), LEAF the next free wide leaf slot, TICKET the
// level kernel's CTA done-counter.
enum { C_LO = 0, C_HI = 1, C_TAIL = 2, C_LEAF = 3, C_TICKET = 4 };

// Levels a collapse runs: a binary node splits its keys at the highest
// differing bit of (30-bit code, 30-bit index), so binary and therefore wide
// depth stay below 62.
constexpr int kWideMaxLevels = 62;

__device__ __forceinline__ float box_area(const float *b) {
  const float dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
  return dx * dy + dy * dz + dz * dx;
}

// Smallest e with 255 * 2^e >= ext (FP64), clamped to the normal fp32 range.
__device__ __forceinline__ int frame_exponent(double ext) {
  if (!(ext > 0.0)) return -126;
  int k;
  frexp(ext / 255.0, &k);
  int e = k - 1;
  while (ldexp(255.0, e) < ext) ++e;
  while (e > -126 && ldexp(255.0, e - 1) >= ext) --e;
  return e < -126 ? -126 : (e > 127 ? 127 : e);
}

__global__ void k_wide_init(const uint32_t *tri_off, uint32_t meshes, uint32_t n, WorkItem *queue, uint32_t *roots,
                            uint32_t *counters) {
  for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < meshes; m += gridDim.x * blockDim.x) {
    const uint32_t cnt = tri_off ? tri_off[m + 1] - tri_off[m] : n;
    queue[m] = WorkItem{m, cnt == 1 ? ~0 : 0};
    roots[m] = m;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    counters[C_LO] = 0;
    counters[C_HI] = meshes;
    counters[C_TAIL] = meshes;
    counters[C_LEAF] = 0;
    counters[C_TICKET] = 0;
  }
}

// One level of the top-down collapse.  Every item of the level (a binary
// node that becomes a wide node) is expanded greedily -- the inner child of
// largest surface area is replaced by its two children until there are
// eight --, written as a quantised wide node at its queue slot, its leaf
// triangles copied to the wide leaf array and its inner children appended
// to the queue as the next level's items.  A warp allocates its children's
// queue slots and leaf slots with one atomic add each (prefix sums across
// the lanes); the last CTA to finish advances [LO, HI) to the items just
// appended.  The levels run as successive launches, so nothing waits on
// another thread's progress.  The eight candidate children stay in registers
// (unrolled loops, predicated updates) and quantising multiplies by the exact
// power of two 2^-e instead of dividing by 2^e: on 67M triangles in 16,384
// meshes the collapse went from 10.96 ms (local-memory arrays, FP64
// divisions) to 5.43 ms with the same nodes.  The candidates' boxes then
// moved to thread-private shared memory (72 instead of 125 registers, 7 CTAs
// per SM instead of 4): 4.8 ms.
__global__ void __launch_bounds__(128) k_wide_level(const Bvh2Node *bvh2, const float4 *leaf_tris,
                                                    const uint32_t *tri_off, WideNode *wnodes, float4 *wleaf,
                                                    WorkItem *queue, uint32_t *counters) {
  const uint32_t lo = counters[C_LO], hi = counters[C_HI];
  // an empty level appends nothing, so the next window equals this one: the
  // launch leaves the counters as they are
  if (lo == hi) return;
  const int lane = threadIdx.x & 31;
  // candidate child boxes, thread-private: [coordinate][slot][thread]
  __shared__ float s_box[6][8][128];
#define CBOX(c, k) s_box[(k)][(c)][threadIdx.x]
  const uint32_t total = hi - lo;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t i0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); i0 < total; i0 += stride) {
    const uint32_t idx = lo + i0 + lane;
    const bool valid = i0 + lane < total;
    // References and areas live in registers (every index below is a
    // compile-time slot number: unrolled loops with predicated updates), the
    // boxes in this thread's column of s_box, so nothing goes to local memory.
    int ref[8];
    float area[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      ref[c] = -1;
      area[c] = 0.0f;
    }
    int cnt = 0;
    uint32_t m = 0, b = 0;
    if (valid) {
      const WorkItem it = queue[idx];
      m = it.mesh;
      b = tri_off ? tri_off[m] : 0u;
      const Bvh2Node *mb = bvh2 + (b - m);
      if (it.bref < 0) {
        const uint32_t slot = (uint32_t)~it.bref;
        const float4 a = leaf_tris[3 * (size_t)(b + slot)], c = leaf_tris[3 * (size_t)(b + slot) + 1],
                     d = leaf_tris[3 * (size_t)(b + slot) + 2];
        ref[0] = it.bref;
        CBOX(0, 0) = fminf(a.x, fminf(c.x, d.x));
        CBOX(0, 1) = fminf(a.y, fminf(c.y, d.y));
        CBOX(0, 2) = fminf(a.z, fminf(c.z, d.z));
        CBOX(0, 3) = fmaxf(a.x, fmaxf(c.x, d.x));
        CBOX(0, 4) = fmaxf(a.y, fmaxf(c.y, d.y));
        CBOX(0, 5) = fmaxf(a.z, fmaxf(c.z, d.z));
        cnt = 1;
      } else {
        const Bvh2Node nd = mb[it.bref];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          ref[c] = nd.ref[c];
#pragma unroll
          for (int k = 0; k < 6; ++k) CBOX(c, k) = nd.box[6 * c + k];
          area[c] = box_area(nd.box + 6 * c);
        }
        cnt = 2;
        // greedy: replace the inner child of largest area (lowest slot on
        // ties) by its two children until there are eight
        while (cnt < 8) {
          int best = -1;
          float ba = -1.0f;
#pragma unroll
          for (int c = 0; c < 8; ++c)
            if (c < cnt && ref[c] >= 0 && area[c] > ba) {
              ba = area[c];
              best = c;
            }
          if (best < 0) break;
          int rb = 0;
#pragma unroll
          for (int c = 0; c < 8; ++c)
            if (c == best) rb = ref[c];
          const Bvh2Node ch = mb[rb];
          const float a0 = box_area(ch.box), a1 = box_area(ch.box + 6);
#pragma unroll
          for (int k = 0; k < 6; ++k) {
            CBOX(best, k) = ch.box[k];
            CBOX(cnt, k) = ch.box[6 + k];
          }
#pragma unroll
          for (int c = 0; c < 8; ++c) {
            if (c == best) {
              ref[c] = ch.ref[0];
              area[c] = a0;
            }
            if (c == cnt) {
              ref[c] = ch.ref[1];
              area[c] = a1;
            }
          }
          ++cnt;
        }
      }
    }
    uint32_t n_inner = 0, n_leaf = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c)
      if (c < cnt) (ref[c] >= 0 ? n_inner : n_leaf)++;
    // warp-aggregated allocation of child queue slots and leaf slots
    const uint32_t inc_i = warp_incl_scan(n_inner, lane), inc_l = warp_incl_scan(n_leaf, lane);
    const uint32_t tot_i = __shfl_sync(FULL_MASK, inc_i, 31), tot_l = __shfl_sync(FULL_MASK, inc_l, 31);
    uint32_t base_i = 0, base_l = 0;
    if (lane == 0) {
      if (tot_i) base_i = atomicAdd(&counters[C_TAIL], tot_i);
      if (tot_l) base_l = atomicAdd(&counters[C_LEAF], tot_l);
    }
    base_i = __shfl_sync(FULL_MASK, base_i, 0);
    base_l = __shfl_sync(FULL_MASK, base_l, 0);
    if (!valid) continue;
    const uint32_t child_base = base_i + inc_i - n_inner, leaf_base = base_l + inc_l - n_leaf;
    float lo3[3] = {CBOX(0, 0), CBOX(0, 1), CBOX(0, 2)}, hi3[3] = {CBOX(0, 3), CBOX(0, 4), CBOX(0, 5)};
#pragma unroll
    for (int c = 1; c < 8; ++c)
      if (c < cnt)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          lo3[k] = fminf(lo3[k], CBOX(c, k));
          hi3[k] = fmaxf(hi3[k], CBOX(c, 3 + k));
        }
    int e[3];
    double isc[3];  // 2^-e: dividing by the scale 2^e is this exact product
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      e[k] = frame_exponent((double)hi3[k] - (double)lo3[k]);
      isc[k] = ldexp(1.0, -e[k]);
    }
    uint32_t imask = 0, meta_w[2] = {0u, 0u}, qlo_w[3][2] = {{0u, 0u}, {0u, 0u}, {0u, 0u}},
             qhi_w[3][2] = {{0u, 0u}, {0u, 0u}, {0u, 0u}};
    uint32_t ri = 0, rl = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int h = c >> 2, sh = 8 * (c & 3);
      // an absent child is the inverted box (lo 255, hi 0): it fails the slab test
      uint32_t meta = 0xFF, ql[3] = {255u, 255u, 255u}, qh[3] = {0u, 0u, 0u};
      if (c < cnt) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const double l = floor(((double)CBOX(c, k) - (double)lo3[k]) * isc[k]);
          const double u = ceil(((double)CBOX(c, 3 + k) - (double)lo3[k]) * isc[k]);
          ql[k] = (uint32_t)(l < 0.0 ? 0.0 : (l > 255.0 ? 255.0 : l));
          qh[k] = (uint32_t)(u < 0.0 ? 0.0 : (u > 255.0 ? 255.0 : u));
        }
        if (ref[c] >= 0) {
          imask |= 1u << c;
          meta = ri;
          queue[child_base + ri] = WorkItem{m, ref[c]};  // the next level's item; its wide node index
          ++ri;
        } else {
          const uint32_t slot = (uint32_t)~ref[c];
          const size_t src = 3 * (size_t)(b + slot), dst = 3 * (size_t)(leaf_base + rl);
          wleaf[dst] = leaf_tris[src];
          wleaf[dst + 1] = leaf_tris[src + 1];
          wleaf[dst + 2] = leaf_tris[src + 2];
          meta = rl;
          ++rl;
        }
      }
      meta_w[h] |= meta << sh;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        qlo_w[k][h] |= ql[k] << sh;
        qhi_w[k][h] |= qh[k] << sh;
      }
    }
    // the 80-byte node as five 16-byte words (layout of WideNode)
    uint4 *op = reinterpret_cast<uint4 *>(wnodes + idx);
    op[0] = make_uint4(__float_as_uint(lo3[0]), __float_as_uint(lo3[1]), __float_as_uint(lo3[2]),
                       (uint32_t)(uint8_t)e[0] | ((uint32_t)(uint8_t)e[1] << 8) | ((uint32_t)(uint8_t)e[2] << 16) |
                           (imask << 24));
    op[1] = make_uint4(child_base, leaf_base, meta_w[0], meta_w[1]);
    op[2] = make_uint4(qlo_w[0][0], qlo_w[0][1], qlo_w[1][0], qlo_w[1][1]);
    op[3] = make_uint4(qlo_w[2][0], qlo_w[2][1], qhi_w[0][0], qhi_w[0][1]);
    op[4] = make_uint4(qhi_w[1][0], qhi_w[1][1], qhi_w[2][0], qhi_w[2][1]);
  }
#undef CBOX
  // the last CTA to finish moves the level window to the appended items
  __shared__ bool s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&counters[C_TICKET], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last && threadIdx.x == 0) {
    __threadfence();
    counters[C_LO] = hi;
    counters[C_HI] = ld_relaxed_u32(&counters[C_TAIL]);
    counters[C_TICKET] = 0;
  }
}

// ---------------------------------------------------------------------------
// traversal
// ---------------------------------------------------------------------------
constexpr int kWideThreads = 128;
constexpr int kWideStack = 64;
constexpr int kWideRefill = 8;

__device__ __forceinline__ float scale_of(int8_t e) { return __int_as_float(((int)e + 127) << 23); }
// 2^15 x the node's quantisation step (infinity past the float range: the
// axis then gives NaN and drops out of the box test, which stays conservative)
__device__ __forceinline__ float scale15_of(int8_t e) { return __int_as_float(min((int)e + 142, 255) << 23); }

// Packed pairs of fp32 (sm_100 f32x2 arithmetic; each half rounds as the
// scalar instruction would) and three-input min / max.
__device__ __forceinline__ unsigned long long pk2(float a, float b) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void up2(unsigned long long v, float &a, float &b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ unsigned long long fma2_rd(unsigned long long a, unsigned long long b, unsigned long long c) {
  unsigned long long r;
  asm("fma.rm.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
__device__ __forceinline__ unsigned long long fma2_ru(unsigned long long a, unsigned long long b, unsigned long long c) {
  unsigned long long r;
  asm("fma.rp.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
__device__ __forceinline__ unsigned long long add2_rn(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long mul2_rn(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ float max3f(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ float min3f(float a, float b, float c) {
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}

__device__ __forceinline__ void wide_leaf_test(const float4 *leaf, uint32_t i, const Ray &R, uint32_t &best,
                                               uint32_t &best_leaf, float &bt) {
  const float4 a = __ldg(leaf + 3 * (size_t)i), b = __ldg(leaf + 3 * (size_t)i + 1), c = __ldg(leaf + 3 * (size_t)i + 2);
  const float v0[3] = {a.x, a.y, a.z}, v1[3] = {b.x, b.y, b.z}, v2[3] = {c.x, c.y, c.z};
  const uint32_t id = __float_as_uint(a.w);
  float t;
  if (isect_tri(R, v0, v1, v2, t) && (best == kMiss || t < bt || (t == bt && id < best))) {
    best = id;
    best_leaf = i;
    bt = t;
  }
}

// Largest m < meshes with off[m] <= r, given off[m0] <= r: gallop upward
// from m0, then bisect.  off has meshes + 1 entries, off[meshes] > r.
__device__ __forceinline__ uint32_t mesh_from(const uint32_t *off, uint32_t meshes, uint32_t m0, uint64_t r) {
  uint32_t lo = m0, hi = m0 + 1, step = 1;
  while (hi < meshes && __ldg(off + hi) <= r) {
    lo = hi;
    step <<= 1;
    hi = lo + step;
  }
  if (hi > meshes) hi = meshes;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(off + mid) <= r) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Lane refill.  When at least kWideRefill lanes of a warp are idle (or all
// are), the warp takes that many new rays from the global counter (waiting
// for the whole warp to finish left most lanes idle behind the longest ray).
// On 16.7M rays of one 16.7M-triangle mesh and on 134M rays over 16,384
// meshes, thresholds of 4, 8, 16 and 32 (no refill) idle lanes measured
// 33.6 / 34.7 / 38.5 / 63.7 ms and 71.3 / 69.0 / 74.8 / 155.5 ms.  The
// counter only grows, so the mesh of the first new ray is at or after the
// warp's previous mesh: the 32 lanes probe the next 32 mesh offsets at once
// (one load latency instead of a serial gallop), and a lane whose ray lies
// before the end of that mesh needs no search of its own.  Called by all 32
// lanes; returns true on the lanes that took a ray (their traversal state is
// then reset by the caller).
template <bool BATCHED>
__device__ __forceinline__ bool wide_take_ray(bool &active, bool &drained, uint32_t &warp_mesh, uint64_t &r,
                                              Ray &R, uint32_t &node, const uint32_t *roots,
                                              const uint32_t *ray_off, uint32_t meshes, const float4 *rays,
                                              uint64_t nrays, unsigned long long *counter) {
  const int lane = threadIdx.x & 31;
  const unsigned idle = __ballot_sync(FULL_MASK, !active);
  const int n_idle = __popc(idle);
  if (drained || (n_idle < kWideRefill && n_idle != 32)) return false;
  unsigned long long base = 0;
  if (lane == 0) base = atomicAdd(counter, (unsigned long long)n_idle);
  base = __shfl_sync(FULL_MASK, base, 0);
  if (base + n_idle >= nrays) drained = true;
  uint64_t mesh_end = 0;  // first ray after warp_mesh
  if (BATCHED && base < nrays) {
    while (true) {
      const uint32_t j = warp_mesh + 1 + lane;
      const uint32_t v = j <= meshes ? __ldg(ray_off + j) : 0xFFFFFFFFu;
      const int k = __popc(__ballot_sync(FULL_MASK, j < meshes && v <= base));  // a prefix of the lanes
      warp_mesh += k;
      if (k < 32) {
        mesh_end = __shfl_sync(FULL_MASK, v, k);
        break;
      }
    }
  }
  if (active) return false;
  const uint64_t mine = base + __popc(idle & ((1u << lane) - 1u));
  if (mine >= nrays) return false;
  r = mine;
  active = true;
  ray_setup(__ldg(rays + 2 * r), __ldg(rays + 2 * r + 1), R);
  uint32_t m = 0;
  if (BATCHED) m = mine < mesh_end ? warp_mesh : mesh_from(ray_off, meshes, warp_mesh, r);
  node = __ldg(roots + m);
  return true;
}

// One node step: the ray is moved into the node's quantised frame once, the
// eight child boxes are tested two at a time with packed f32x2 arithmetic
// (byte decode, directed-rounding slab FMAs, the 2^-18 widening) and
// three-input min/max (68.7 -> 60.7 ms on the 134M-ray workload against the
// scalar loop).  A plane byte q is decoded by one byte permute into the float
// v = 1 + q 2^-15; with M = 2^15 x the step in t and the plane offset moved
// down (near planes) or up (far planes) by M in that direction of rounding,
// one directed-rounding FMA v M + (offset - M) gives a value never inside
// q x step + offset, without a separate bias subtraction (47.8 -> 47.2 ms).
// Absent children are inverted boxes and need no test of their own.  With
// NEAREST the nearest hit inner child is found inside the box loop (closest
// hit: entering the lowest hit slot instead measured 40.3 against 22.7 ms on
// 16.8M rays of one 16.8M-triangle mesh); without it the lowest hit inner
// slot is entered (any hit: 16.8 against 17.7 ms on the same rays).
struct WideStep {
  uint32_t hm;  // slots whose box is hit
  uint32_t imask, child_base, leaf_base, meta_lo, meta_hi;
  int ns;  // nearest hit inner slot, -1 if none
};

template <bool NEAREST>
__device__ __forceinline__ WideStep wide_node_step(const WideNode *nodes, uint32_t node, const Ray &R, float bt) {
  WideStep S;
  const uint4 *np = reinterpret_cast<const uint4 *>(nodes + node);
  const uint4 w0 = __ldg(np), w1 = __ldg(np + 1), w2 = __ldg(np + 2), w3 = __ldg(np + 3), w4 = __ldg(np + 4);
  const float px = __uint_as_float(w0.x), py = __uint_as_float(w0.y), pz = __uint_as_float(w0.z);
  const float sx = scale15_of((int8_t)(w0.w & 0xFF)), sy = scale15_of((int8_t)((w0.w >> 8) & 0xFF)),
              sz = scale15_of((int8_t)((w0.w >> 16) & 0xFF));
  S.imask = w0.w >> 24;
  S.child_base = w1.x;
  S.leaf_base = w1.y;
  S.meta_lo = w1.z;
  S.meta_hi = w1.w;
  float An[3], Af[3], Bq[3];
  uint32_t qn[3][2], qf[3][2];
  {
    const float pa[3] = {px, py, pz}, oa[3] = {R.ox, R.oy, R.oz}, ia[3] = {R.ix, R.iy, R.iz};
    const float sa[3] = {sx, sy, sz};
    const uint32_t ql[3][2] = {{w2.x, w2.y}, {w2.z, w2.w}, {w3.x, w3.y}};
    const uint32_t qh[3][2] = {{w3.z, w3.w}, {w4.x, w4.y}, {w4.z, w4.w}};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float dlo = __fsub_rd(pa[a], oa[a]), dhi = __fsub_ru(pa[a], oa[a]);
      const bool pos = !(ia[a] < 0.0f);
      An[a] = __fmul_rd(pos ? dlo : dhi, ia[a]);
      Af[a] = __fmul_ru(pos ? dhi : dlo, ia[a]);
      Bq[a] = __fmul_rn(sa[a], ia[a]);  // M: 2^15 x the step in t (exactly 2^15 x the rounded step)
      An[a] = __fsub_rd(An[a], Bq[a]);
      Af[a] = __fsub_ru(Af[a], Bq[a]);
      qn[a][0] = pos ? ql[a][0] : qh[a][0];
      qn[a][1] = pos ? ql[a][1] : qh[a][1];
      qf[a][0] = pos ? qh[a][0] : ql[a][0];
      qf[a][1] = pos ? qh[a][1] : ql[a][1];
    }
  }
  uint32_t hm = 0;
  float nt = __int_as_float(0x7f800000);
  int ns = -1;
  {
    const unsigned long long lo2 = pk2(kBoxLo, kBoxLo), hi2 = pk2(kBoxHi, kBoxHi);
    unsigned long long B2[3], N2[3], F2[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      B2[a] = pk2(Bq[a], Bq[a]);
      N2[a] = pk2(An[a], An[a]);
      F2[a] = pk2(Af[a], Af[a]);
    }
#pragma unroll
    for (int cp = 0; cp < 4; ++cp) {
      const int h = cp >> 1;
      const uint32_t s0 = 0x7604u | ((uint32_t)((2 * cp) & 3) << 4), s1 = 0x7604u | ((uint32_t)((2 * cp + 1) & 3) << 4);
      float n[2][3], f[2][3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const unsigned long long qn2 = pk2(__uint_as_float(__byte_perm(qn[a][h], 0x3F800000u, s0)),
                                           __uint_as_float(__byte_perm(qn[a][h], 0x3F800000u, s1)));
        const unsigned long long qf2 = pk2(__uint_as_float(__byte_perm(qf[a][h], 0x3F800000u, s0)),
                                           __uint_as_float(__byte_perm(qf[a][h], 0x3F800000u, s1)));
        up2(fma2_rd(qn2, B2[a], N2[a]), n[0][a], n[1][a]);
        up2(fma2_ru(qf2, B2[a], F2[a]), f[0][a], f[1][a]);
      }
      float tn[2], tf[2];
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        tn[k] = fmaxf(max3f(n[k][0], n[k][1], n[k][2]), R.tmin);
        tf[k] = min3f(f[k][0], f[k][1], f[k][2]);
      }
      up2(mul2_rn(pk2(tn[0], tn[1]), lo2), tn[0], tn[1]);
      up2(mul2_rn(pk2(tf[0], tf[1]), hi2), tf[0], tf[1]);
      // the widened exit clamped by the best distance: one compare per child
      // tests both (45.4 against 46.6 ms for two compares, exit clamped first)
      tf[0] = fminf(tf[0], bt);
      tf[1] = fminf(tf[1], bt);
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int c = 2 * cp + k;
        const bool hit = tn[k] <= tf[k];
        hm |= (uint32_t)hit << c;
        if (NEAREST && hit && ((S.imask >> c) & 1u) && tn[k] < nt) {
          nt = tn[k];
          ns = c;
        }
      }
    }
  }
  S.hm = hm;
  S.ns = NEAREST ? ns : ((hm & S.imask) ? __ffs(hm & S.imask) - 1 : -1);
  return S;
}

// The next node: the nearest hit inner child is entered and the other hit
// inner children are pushed as one entry {child_base, slot mask | inner mask
// << 8} (a popped slot's node is child_base + the inner children below it);
// with no inner child hit, the top entry's lowest slot is popped.  Returns
// false when the traversal is over (or the stack overflowed: status 5).
__device__ __forceinline__ bool wide_next(const WideStep &S, uint2 *stack, int &sp, uint32_t &node, uint32_t *err) {
  if (S.ns >= 0) {
    const uint32_t rest = S.hm & S.imask & ~(1u << S.ns);
    if (rest) {
      if (sp >= kWideStack) {
        atomicCAS(err, 0u, 5u);  // traversal stack overflow
        return false;
      }
      stack[sp++] = make_uint2(S.child_base, rest | (S.imask << 8));
    }
    node = S.child_base + (uint32_t)__popc(S.imask & ((1u << S.ns) - 1u));
    return true;
  }
  if (sp > 0) {
    uint2 &top = stack[sp - 1];
    const uint32_t c = __ffs(top.y & 0xFFu) - 1;
    top.y &= ~(1u << c);
    node = top.x + (uint32_t)__popc((top.y >> 8) & ((1u << c) - 1u));
    if ((top.y & 0xFFu) == 0) --sp;
    return true;
  }
  return false;
}

__device__ __forceinline__ uint32_t wide_leaf_meta(const WideStep &S, int c) {
  return ((c < 4 ? S.meta_lo : S.meta_hi) >> (8 * (c & 3))) & 0xFF;
}

// A finished ray's record: the primitive id and, until k_wide_refine
// replaces it by t, the leaf slot of the triangle hit.
__device__ __forceinline__ Hit wide_result(uint32_t best, uint32_t best_leaf) {
  Hit out;
  out.prim = best;
  out.t = best != kMiss ? __uint_as_float(best_leaf) : __int_as_float(0x7f800000);
  return out;
}

// t of every hit: the plane-equation distance of the hit triangle in
// double-float, rounded once.  Run after the traversal over all rays at once
// instead of by each lane as its ray finished (when few lanes of the warp ran
// it and the rest waited).  A warp reads 32 records at a time (coalesced)
// and queues the indices of the hits in shared memory; every 32 queued hits
// are refined with all lanes busy (a lane per record left ~1 in 5 busy: 2.0
// ms cold for 134M rays, 18 % of them hits).
constexpr int kRefineThreads = 256;

__global__ void __launch_bounds__(kRefineThreads) k_wide_refine(const float4 *leaf, const float4 *rays,
                                                                uint64_t nrays, Hit *hits) {
  __shared__ uint64_t s_q[kRefineThreads / 32][64];
  const int lane = threadIdx.x & 31;
  uint64_t *q = s_q[threadIdx.x >> 5];
  auto refine = [&](int count) {
    __syncwarp();
    if (lane < count) {
      const uint64_t i = q[lane];
      const uint32_t slot = __float_as_uint(hits[i].t);
      const float4 o = __ldg(rays + 2 * i), d = __ldg(rays + 2 * i + 1);
      Ray R;
      R.ox = o.x;
      R.oy = o.y;
      R.oz = o.z;
      R.dx = d.x;
      R.dy = d.y;
      R.dz = d.z;
      const float4 a = __ldg(leaf + 3 * (size_t)slot), b = __ldg(leaf + 3 * (size_t)slot + 1),
                   c = __ldg(leaf + 3 * (size_t)slot + 2);
      const float v0[3] = {a.x, a.y, a.z}, v1[3] = {b.x, b.y, b.z}, v2[3] = {c.x, c.y, c.z};
      hits[i].t = refine_t(R, v0, v1, v2);
    }
    __syncwarp();
  };
  int nq = 0;  // queued hits, the same on every lane
  const uint64_t warps = (uint64_t)gridDim.x * (kRefineThreads / 32);
  for (uint64_t base = (blockIdx.x * (uint64_t)(kRefineThreads / 32) + (threadIdx.x >> 5)) * 32; base < nrays;
       base += warps * 32) {
    const uint64_t i = base + lane;
    const bool hit = i < nrays && hits[i].prim != kMiss;
    const unsigned m = __ballot_sync(FULL_MASK, hit);
    if (hit) q[nq + __popc(m & ((1u << lane) - 1u))] = i;
    nq += __popc(m);
    if (nq >= 32) {
      refine(32);
      const uint64_t v = lane < nq - 32 ? q[32 + lane] : 0;
      __syncwarp();
      if (lane < nq - 32) q[lane] = v;
      nq -= 32;
    }
  }
  refine(nq);
}

// Any hit: one lane per ray; after a node's box loop the lanes with hit leaf
// children test those triangles together, whatever slots they are in (testing
// them inside the child loop ran each slot's test separately with few lanes
// active), and the first hit ends the ray.
template <bool BATCHED>
__global__ void __launch_bounds__(kWideThreads, 8)
    k_trace_wide_any(const WideNode *nodes, const float4 *leaf, const uint32_t *roots, const uint32_t *ray_off,
                     uint32_t meshes, const float4 *rays, uint64_t nrays, Hit *hits, unsigned long long *counter,
                     uint32_t *err) {
  bool active = false, drained = false;
  uint64_t r = 0;
  Ray R;
  uint32_t node = 0, best = kMiss, best_leaf = 0;
  float bt = 0.0f;
  uint2 stack[kWideStack];  // {child_base, mask of inner-child ranks still to visit}
  uint32_t warp_mesh = 0;  // a mesh at or below every ray this warp will still take
  int sp = 0;
  while (true) {
    if (wide_take_ray<BATCHED>(active, drained, warp_mesh, r, R, node, roots, ray_off, meshes, rays, nrays,
                               counter)) {
      best = kMiss;
      best_leaf = 0;
      bt = R.tmax;
      sp = 0;
    }
    if (!__any_sync(FULL_MASK, active)) {
      if (drained) break;
      continue;
    }
    if (!active) continue;
    const WideStep S = wide_node_step<false>(nodes, node, R, bt);
    uint32_t leaf_hit = S.hm & ~S.imask;
    while (leaf_hit) {
      const int c = __ffs(leaf_hit) - 1;
      leaf_hit &= leaf_hit - 1u;
      const uint32_t meta = wide_leaf_meta(S, c);
      if (meta != 0xFF) wide_leaf_test(leaf, S.leaf_base + meta, R, best, best_leaf, bt);
    }
    if (best != kMiss || !wide_next(S, stack, sp, node, err)) {
      hits[r] = wide_result(best, best_leaf);
      active = false;
    }
  }
}

// Order-preserving unsigned image of a distance with -0 and +0 merged:
// comparing (t_order(t) << 32 | id) as 64-bit unsigned integers compares
// (t, id) as the immediate test does (smaller t first, then the lower id).
__device__ __forceinline__ uint32_t t_order(float t) {
  const uint32_t u = t == 0.0f ? 0u : __float_as_uint(t);
  return u ^ ((uint32_t)((int32_t)u >> 31) | 0x80000000u);
}
__device__ __forceinline__ float t_from_order(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k ^ 0x80000000u) : ~k);
}

constexpr int kLeafFlush = 24;  // queued triangle tests that trigger a flush
constexpr int kLeafQueue = 256;  // per warp: one node step adds at most 8 per lane; a step that would overflow flushes first

// Closest hit: one lane per ray, and the triangle tests of the hit leaf
// children are queued per warp in shared memory as (triangle slot, lane)
// pairs instead of being run at once.  A node step hits about one leaf
// triangle per 14 lanes, so running the tests at once kept ~2 of 32 lanes
// busy for the length of a triangle test in most steps.  When kLeafFlush
// tests are queued, all 32 lanes run them (the owner's ray comes by
// shuffles and from shared memory) and fold each hit into the owner's best
// (t, id) key with one shared-memory atomicMin; the owners then take the
// key's t as their culling distance.  A lane whose traversal is over while tests of its ray are still
// queued waits for the flush, which also runs when no lane of the warp
// traverses any more, or when the waiting lanes and the idle ones add up to a
// refill.  The closest (t, id) over all tested triangles is the same in any
// order of tests, so the hits equal the immediate test's; the culling
// distance only lags.  On the 134M-ray workload flush thresholds of 8, 12,
// 16, 24, 32 and 64 tests measured 56.2 / 55.4 / 55.1 / 54.8 / 55.1 / 55.2
// ms against 57.6 ms for the immediate tests (t still refined in the
// traversal then).
template <bool BATCHED>
__global__ void __launch_bounds__(kWideThreads, 9)
    k_trace_wide_closest(const WideNode *nodes, const float4 *leaf, const uint32_t *roots, const uint32_t *ray_off,
                         uint32_t meshes, const float4 *rays, uint64_t nrays, Hit *hits,
                         unsigned long long *counter, uint32_t *err) {
  __shared__ uint32_t s_qslot[kWideThreads / 32][kLeafQueue];
  __shared__ uint8_t s_qlane[kWideThreads / 32][kLeafQueue];
  __shared__ unsigned long long s_best[kWideThreads / 32][32];
  __shared__ uint32_t s_bslot[kWideThreads / 32][32];
  // what only the flush and the final store read stays in shared memory, not
  // in registers: 56 registers let 9 CTAs share an SM (47.8 -> 46.6 ms)
  __shared__ float s_rs[kWideThreads / 32][4][32];  // Sx, Sy, Sz, tmax of each lane's ray
  __shared__ int s_rk[kWideThreads / 32][32];        // kx | ky << 2 | kz << 4
  __shared__ unsigned long long s_rid[kWideThreads / 32][32];  // ray index
  const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
  uint32_t *qslot = s_qslot[wq];
  uint8_t *qlane = s_qlane[wq];
  unsigned long long *sbest = s_best[wq];
  uint32_t *sbslot = s_bslot[wq];
  bool active = false, drained = false, done = false, pending = false;
  uint64_t r = 0;
  Ray R;
  uint32_t node = 0;
  float bt = 0.0f;
  uint2 stack[kWideStack];
  uint32_t warp_mesh = 0;
  int sp = 0, nq = 0;  // nq: queued tests, the same on every lane

  // Runs the queued tests with all lanes (warp-uniform call).
  auto flush = [&]() {
    __syncwarp();
    for (int b = 0; b < nq; b += 32) {
      const int e = b + lane;
      const uint32_t slot = e < nq ? qslot[e] : kMiss;
      const int o = e < nq ? qlane[e] : lane;
      Ray Q;
      Q.ox = __shfl_sync(FULL_MASK, R.ox, o);
      Q.oy = __shfl_sync(FULL_MASK, R.oy, o);
      Q.oz = __shfl_sync(FULL_MASK, R.oz, o);
      Q.tmin = __shfl_sync(FULL_MASK, R.tmin, o);
      Q.Sx = s_rs[wq][0][o];
      Q.Sy = s_rs[wq][1][o];
      Q.Sz = s_rs[wq][2][o];
      Q.tmax = s_rs[wq][3][o];
      const int k = s_rk[wq][o];
      Q.kx = k & 3;
      Q.ky = (k >> 2) & 3;
      Q.kz = k >> 4;
      unsigned long long key = ~0ull;
      if (slot != kMiss) {
        const float4 a = __ldg(leaf + 3 * (size_t)slot), bb = __ldg(leaf + 3 * (size_t)slot + 1),
                     c = __ldg(leaf + 3 * (size_t)slot + 2);
        const float v0[3] = {a.x, a.y, a.z}, v1[3] = {bb.x, bb.y, bb.z}, v2[3] = {c.x, c.y, c.z};
        float t;
        if (isect_tri(Q, v0, v1, v2, t)) {
          key = ((unsigned long long)t_order(t) << 32) | __float_as_uint(a.w);
          atomicMin(&sbest[o], key);
        }
      }
      __syncwarp();
      if (key != ~0ull && sbest[o] == key) sbslot[o] = slot;  // one winner per owner
      __syncwarp();
    }
    if (pending) {
      bt = t_from_order((uint32_t)(sbest[lane] >> 32));
      pending = false;
    }
    nq = 0;
  };

  while (true) {
    if (wide_take_ray<BATCHED>(active, drained, warp_mesh, r, R, node, roots, ray_off, meshes, rays, nrays,
                               counter)) {
      bt = R.tmax;
      sp = 0;
      done = false;
      sbest[lane] = ((unsigned long long)t_order(R.tmax) << 32) | kMiss;
      s_rs[wq][0][lane] = R.Sx;
      s_rs[wq][1][lane] = R.Sy;
      s_rs[wq][2][lane] = R.Sz;
      s_rs[wq][3][lane] = R.tmax;
      s_rk[wq][lane] = R.kx | (R.ky << 2) | (R.kz << 4);
      s_rid[wq][lane] = r;
    }
    if (!__any_sync(FULL_MASK, active)) {
      if (drained) break;
      continue;
    }
    uint32_t lh = 0, lbase = 0, mlo = 0, mhi = 0;
    if (active && !done) {
      const WideStep S = wide_node_step<true>(nodes, node, R, bt);
      lh = S.hm & ~S.imask;
      lbase = S.leaf_base;
      mlo = S.meta_lo;
      mhi = S.meta_hi;
      done = !wide_next(S, stack, sp, node, err);
    }
    const int cnt = __popc(lh);
    const int total = (int)__reduce_add_sync(FULL_MASK, (unsigned)cnt);
    if (total) {
      if (nq + total > kLeafQueue) flush();
      int pos;
      if (!__any_sync(FULL_MASK, cnt > 1)) {
        pos = nq + __popc(__ballot_sync(FULL_MASK, cnt) & ((1u << lane) - 1u));
      } else {
        int inc = cnt;  // inclusive prefix of the counts over the lanes
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const int v = __shfl_up_sync(FULL_MASK, inc, d);
          if (lane >= d) inc += v;
        }
        pos = nq + inc - cnt;
      }
      while (lh) {
        const int c = __ffs(lh) - 1;
        lh &= lh - 1u;
        const uint32_t meta = ((c < 4 ? mlo : mhi) >> (8 * (c & 3))) & 0xFF;
        qslot[pos] = meta == 0xFF ? kMiss : lbase + meta;
        qlane[pos] = (uint8_t)lane;
        ++pos;
      }
      if (cnt) pending = true;
      nq += total;
    }
    const unsigned waiting = __ballot_sync(FULL_MASK, done && pending);
    const unsigned running = __ballot_sync(FULL_MASK, active && !done);
    const unsigned idle = __ballot_sync(FULL_MASK, !active);
    if (nq >= kLeafFlush || (waiting && (!running || __popc(waiting) + __popc(idle) >= kWideRefill))) flush();
    if (active && done && !pending) {
      hits[s_rid[wq][lane]] = wide_result((uint32_t)sbest[lane], sbslot[lane]);
      active = false;
    }
  }
}
}  // namespace gprtcu

using namespace gprtcu;


namespace {

struct WideScratch {
  size_t counters, queue, total;
};

WideScratch wide_layout(uint32_t meshes, uint32_t n) {
  WideScratch L;
  size_t off = sizeof(ScratchHeader);
  L.counters = off;
  off += 256;
  L.queue = off;
  off += gprtcu_align256((size_t)n * sizeof(WorkItem));
  L.total = off;
  (void)meshes;
  return L;
}

}  // namespace

extern "C" GPRTCU_API size_t gprtcuWideScratchSize(uint32_t numMeshes, uint32_t totalTriangles) {
  return wide_layout(numMeshes, totalTriangles).total;
}

extern "C" GPRTCU_API gprtcuStatus gprtcuWideBuild(const gprtcuLbvh *binary, const uint32_t *triOffsets,
                                                   uint32_t numMeshes, gprtcuWideBvh *out, void *scratch,
                                                   size_t scratchBytes, gprtcuStream stream_) {
  cudaStream_t stream = (cudaStream_t)stream_;
  if (!binary || !out || numMeshes == 0) return GPRTCU_ERR_INVALID_ARG;
  const uint32_t n = binary->numPrims;
  if (n == 0 || numMeshes > n || (numMeshes > 1 && !triOffsets)) return GPRTCU_ERR_INVALID_ARG;
  if (!binary->leafTris || (n > numMeshes && !binary->bvh2)) return GPRTCU_ERR_INVALID_ARG;
  if (!out->nodes || !out->leafTris || !out->roots || out->capacity < n) return GPRTCU_ERR_INVALID_ARG;
  if (((uintptr_t)out->nodes & 15) || ((uintptr_t)out->leafTris & 15)) return GPRTCU_ERR_INVALID_ARG;
  if (!scratch || ((uintptr_t)scratch & 255)) return GPRTCU_ERR_INVALID_ARG;
  const WideScratch L = wide_layout(numMeshes, n);
  if (scratchBytes < L.total) return GPRTCU_ERR_SCRATCH_TOO_SMALL;
  char *s = (char *)scratch;
  GPRTCU_TRY(cudaMemsetAsync(s, 0, L.queue, stream));  // header, counters
  uint32_t *counters = (uint32_t *)(s + L.counters);
  WorkItem *queue = (WorkItem *)(s + L.queue);
  const uint32_t *toff = numMeshes > 1 ? triOffsets : nullptr;
  k_wide_init<<<(numMeshes + 255) / 256, 256, 0, stream>>>(toff, numMeshes, n, queue, out->roots, counters);
  GPRTCU_TRY(cudaGetLastError());
  // One launch per level; a launch whose level is empty returns at once.  The
  // grid is what fits on the GPU at once (7 CTAs of 128 threads per SM: 72
  // registers, 24 KB of shared memory): a grid-stride loop with a second wave
  // of CTAs ran the level for about twice a CTA's share (6.6 against 4.8 ms).
  static std::atomic<int> level_ctas_cache{0};  // host threads may race to fill it with the same value
  int level_ctas = level_ctas_cache.load(std::memory_order_relaxed);
  if (!level_ctas) {
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_wide_level, 128, 0) != cudaSuccess || occ < 1) occ = 1;
    level_ctas = occ;
    level_ctas_cache.store(occ, std::memory_order_relaxed);
  }
  const int grid = gprtcu_num_sms() * level_ctas;
  for (int level = 0; level < kWideMaxLevels; ++level) {
    k_wide_level<<<grid, 128, 0, stream>>>((const Bvh2Node *)binary->bvh2, (const float4 *)binary->leafTris, toff,
                                           (WideNode *)out->nodes, (float4 *)out->leafTris, queue, counters);
    GPRTCU_TRY(cudaGetLastError());
  }
  if (out->numNodes) GPRTCU_TRY(cudaMemcpyAsync(out->numNodes, counters + C_TAIL, 4, cudaMemcpyDeviceToDevice, stream));
  return GPRTCU_OK;
}

extern "C" GPRTCU_API gprtcuStatus gprtcuWideTrace(const gprtcuWideBvh *bvh, const uint32_t *rayOffsets,
                                                   uint32_t numMeshes, const float *rays, uint64_t numRays, int anyHit,
                                                   gprtcuHit *hits, void *scratch, size_t scratchBytes,
                                                   gprtcuStream stream_) {
  cudaStream_t stream = (cudaStream_t)stream_;
  if (!bvh || numMeshes == 0 || (numMeshes > 1 && !rayOffsets)) return GPRTCU_ERR_INVALID_ARG;
  if ((!rays || !hits) && numRays) return GPRTCU_ERR_INVALID_ARG;
  if (numRays == 0) return GPRTCU_OK;
  if (!bvh->nodes || !bvh->leafTris || !bvh->roots) return GPRTCU_ERR_INVALID_ARG;
  if (((uintptr_t)rays & 15) || ((uintptr_t)bvh->nodes & 15) || ((uintptr_t)bvh->leafTris & 15))
    return GPRTCU_ERR_INVALID_ARG;
  if (!scratch || ((uintptr_t)scratch & 255)) return GPRTCU_ERR_INVALID_ARG;
  if (scratchBytes < sizeof(ScratchHeader)) return GPRTCU_ERR_SCRATCH_TOO_SMALL;
  ScratchHeader *hdr = (ScratchHeader *)scratch;
  unsigned long long *counter = reinterpret_cast<unsigned long long *>(&hdr->ticket[0]);
  GPRTCU_TRY(cudaMemsetAsync(scratch, 0, sizeof(ScratchHeader), stream));
  // any hit: 64 registers, 8 CTAs of 128 threads per SM; closest hit: 56, 9
  const int blocks = gprtcu_num_sms() * (anyHit ? 8 : 9);
  const uint64_t need = (numRays + kWideThreads - 1) / kWideThreads;
  const int grid = (int)(need < (uint64_t)blocks ? need : blocks);
#define GPRTCU_WTRACE(K, B)                                                                                 \
  K<B><<<grid, kWideThreads, 0, stream>>>((const WideNode *)bvh->nodes, (const float4 *)bvh->leafTris, bvh->roots, \
                                          rayOffsets, numMeshes, (const float4 *)rays, numRays, (Hit *)hits,      \
                                          counter, &hdr->status)
  if (numMeshes > 1) {
    if (anyHit) GPRTCU_WTRACE(k_trace_wide_any, true);
    else GPRTCU_WTRACE(k_trace_wide_closest, true);
  } else {
    if (anyHit) GPRTCU_WTRACE(k_trace_wide_any, false);
    else GPRTCU_WTRACE(k_trace_wide_closest, false);
  }
#undef GPRTCU_WTRACE
  GPRTCU_TRY(cudaGetLastError());
  const uint64_t need_r = (numRays + kRefineThreads - 1) / kRefineThreads;
  const int grid_r = (int)(need_r < (uint64_t)gprtcu_num_sms() * 4 ? need_r : gprtcu_num_sms() * 4);
  k_wide_refine<<<grid_r, kRefineThreads, 0, stream>>>((const float4 *)bvh->leafTris, (const float4 *)rays,
                                                       numRays, (Hit *)hits);
  GPRTCU_TRY(cudaGetLastError());
  return GPRTCU_OK;
}
