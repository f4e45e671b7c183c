// oracle.cpp -- CPU restatement of GPRT's acceleration-structure path.
//
// TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check and the bench's
// CPU-baseline leg use this library as the checker.  The product library never
// links, loads or calls it.  Build: oracle/Makefile (g++ -O2 -fopenmp
// -ffp-contract=off; the ray math relies on every float operation being a
// separately rounded IEEE operation, exactly as the CUDA kernels issue them).
//
// Parity pins are listed per function in oracle.h.
#include "oracle.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

// ============================================================================
// sort
// ============================================================================
// gprtBufferSort / gprtBufferSortPayload (gprt/gprt.cpp:8821-9073) run a stable
// least-significant-digit radix sort in place; every pass is a stable split by
// one digit (gprt/gprt_sort.slang:353-489).  The net effect is a stable
// ascending sort, which is what the reference test checks with std::sort
// (tests/t02-bufferSort/hostCode.cpp:59,115).  Restated as std::stable_sort of
// (key, original position) so payload order within equal keys is preserved.
template <typename K, typename V>
static void sort_kv(K *keys, V *vals, size_t n) {
  std::vector<std::pair<K, V>> kv(n);
  for (size_t i = 0; i < n; ++i) kv[i] = {keys[i], vals[i]};
  std::stable_sort(kv.begin(), kv.end(), [](const std::pair<K, V> &a, const std::pair<K, V> &b) {
    return a.first < b.first;
  });
  for (size_t i = 0; i < n; ++i) {
    keys[i] = kv[i].first;
    vals[i] = kv[i].second;
  }
}

extern "C" void orc_sort(void *keys, int kw, void *vals, int vw, size_t n) {
  if (n == 0) return;
  if (vw == 0 || vals == nullptr) {
    if (kw == 4) std::sort((uint32_t *)keys, (uint32_t *)keys + n);
    else std::sort((uint64_t *)keys, (uint64_t *)keys + n);
    return;
  }
  if (kw == 4 && vw == 4) sort_kv((uint32_t *)keys, (uint32_t *)vals, n);
  else if (kw == 4 && vw == 8) sort_kv((uint32_t *)keys, (uint64_t *)vals, n);
  else if (kw == 8 && vw == 4) sort_kv((uint64_t *)keys, (uint32_t *)vals, n);
  else sort_kv((uint64_t *)keys, (uint64_t *)vals, n);
}

// ============================================================================
// scan / partition / select
// ============================================================================
// Exclusive sum as the t03 host loop computes it
// (tests/t03-bufferScans/hostCode.cpp:53-58), uint32 wraparound; inclusive is
// the same with the element added first.  The total is returned the way
// bufferScan returns state[0] (gprt/gprt_scan.slang:290-297).
extern "C" uint32_t orc_scan_u32(const uint32_t *in, uint32_t *out, size_t n, int inclusive) {
  uint32_t sum = 0;
  for (size_t i = 0; i < n; ++i) {
    uint32_t v = in[i];
    if (inclusive) {
      sum += v;
      out[i] = sum;
    } else {
      out[i] = sum;
      sum += v;
    }
  }
  return sum;
}

// Selected items (sign bit clear when selectPositive, set otherwise) go to
// out[excl[i]] (getForwardAddr, gprt/gprt_scan.slang:84-87); with partition the
// rest go to out[(n-1) - (i - excl[i])] (getReverseAddr, :89-92), i.e. to the
// back in reverse order.  Known-answer layout:
// tests/t03-bufferScans/hostCode.cpp:98-160 (partition), 172-241 (select).
extern "C" uint32_t orc_partition_i32(const int32_t *in, int32_t *out, size_t n, int selectPositive, int partition) {
  uint32_t excl = 0;
  for (size_t i = 0; i < n; ++i) {
    int32_t v = in[i];
    bool neg = ((uint32_t)v >> 31) != 0;
    bool sel = selectPositive ? !neg : neg;
    if (sel) {
      out[excl] = v;
      ++excl;
    } else if (partition) {
      out[(n - 1) - (i - excl)] = v;
    }
  }
  return excl;
}

// ============================================================================
// Morton / Hilbert
// ============================================================================
// 10-bit spread: separate_bits (gprt/development/gprt_lbvh.hlsl:25-32).
static inline uint32_t spread10(uint32_t v) {
  v &= 0x3FFu;
  v = (v | (v << 16)) & 0xFF0000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

// morton_encode3D (gprt/development/gprt_lbvh.hlsl:34-37): x in bit 0.
extern "C" uint32_t orc_morton3d(uint32_t x, uint32_t y, uint32_t z) {
  return spread10(x) | (spread10(y) << 1) | (spread10(z) << 2);
}

// 3-D, 10-bit Hilbert index with the orientation conventions of Moore's
// hilbert_c2i as used by gprt/hilbert.h:179-235 (nDims=3, nBits=10).
// Restated level by level: the coordinate bits of one level form a 3-bit cell
// (x in bit 0), each cell is Gray-differenced against the level above, rotated
// by the running rotation after XOR with the entry flip, and the rotation
// advances by one plus the position of the cell's lowest set bit among bits
// 0..1.  The concatenated digits are then XORed with 0b010 in every level
// except the top, and Gray-decoded (prefix XOR over the whole index).
extern "C" uint32_t orc_hilbert3d(uint32_t x, uint32_t y, uint32_t z) {
  uint32_t cell[10];
  for (int L = 0; L < 10; ++L) cell[L] = ((x >> L) & 1u) | (((y >> L) & 1u) << 1) | (((z >> L) & 1u) << 2);
  uint32_t g[10];
  for (int L = 0; L < 10; ++L) g[L] = cell[L] ^ (L < 9 ? cell[L + 1] : 0u);
  uint32_t index = 0, rotation = 0, flip = 0;
  for (int L = 9; L >= 0; --L) {
    uint32_t b = flip ^ g[L];
    b = ((b >> rotation) | (b << (3 - rotation))) & 7u;
    index = (index << 3) | b;
    flip = 1u << rotation;
    uint32_t low = b & (0u - b) & 3u;
    rotation += (low == 1u) ? 1u : (low == 2u) ? 2u : 0u;
    rotation += 1u;
    if (rotation >= 3u) rotation -= 3u;
  }
  index ^= 0x04924924u;  // bits 2,5,...,26
  for (int d = 1; d < 30; d *= 2) index ^= index >> d;
  return index;
}

// ============================================================================
// bounds and codes
// ============================================================================
struct f3 {
  float x, y, z;
};
static inline f3 ld3(const float *p, uint32_t i) { return {p[3 * (size_t)i], p[3 * (size_t)i + 1], p[3 * (size_t)i + 2]}; }

// getTriangleBounds (gprt/development/gprt_lbvh.hlsl:121-129): min/max of the
// three vertices, min(p1, min(p2, p3)).
static inline void tri_box(const float *pos, const uint32_t *tri, uint32_t id, float b[6]) {
  f3 p1 = ld3(pos, tri[3 * (size_t)id]), p2 = ld3(pos, tri[3 * (size_t)id + 1]), p3 = ld3(pos, tri[3 * (size_t)id + 2]);
  b[0] = std::fmin(p1.x, std::fmin(p2.x, p3.x));
  b[1] = std::fmin(p1.y, std::fmin(p2.y, p3.y));
  b[2] = std::fmin(p1.z, std::fmin(p2.z, p3.z));
  b[3] = std::fmax(p1.x, std::fmax(p2.x, p3.x));
  b[4] = std::fmax(p1.y, std::fmax(p2.y, p3.y));
  b[5] = std::fmax(p1.z, std::fmax(p2.z, p3.z));
}

// ComputeTriangleBounds (gprt/development/gprt_lbvh.hlsl:215-226): the scene
// AABB, seeded with +-FLT_MAX by the host (gprt/development/gprt_lbvh.h:174-178).
extern "C" void orc_tri_bounds(const float *pos, const uint32_t *tri, uint32_t n, float out[6]) {
  const float M = 3.402823466e38f;
  float s[6] = {M, M, M, -M, -M, -M};
  for (uint32_t i = 0; i < n; ++i) {
    float b[6];
    tri_box(pos, tri, i, b);
    for (int k = 0; k < 3; ++k) {
      s[k] = std::fmin(s[k], b[k]);
      s[3 + k] = std::fmax(s[3 + k], b[3 + k]);
    }
  }
  std::memcpy(out, s, sizeof(s));
}

extern "C" void orc_point_bounds(const float *pos, uint32_t n, float out[6]) {
  const float M = 3.402823466e38f;
  float s[6] = {M, M, M, -M, -M, -M};
  for (uint32_t i = 0; i < n; ++i) {
    f3 p = ld3(pos, i);
    float v[3] = {p.x, p.y, p.z};
    for (int k = 0; k < 3; ++k) {
      s[k] = std::fmin(s[k], v[k]);
      s[3 + k] = std::fmax(s[3 + k], v[k]);
    }
  }
  std::memcpy(out, s, sizeof(s));
}

// Normalise to the scene box, scale by 1024, clamp to [0,1023], truncate:
// gprt/development/gprt_lbvh.hlsl:268-274.  The operation order is fixed:
// (p - min), (max - min), IEEE divide, *1024, max with 0, min with 1023.
// NaN (a zero-extent axis gives 0/0) clamps to 0, as maxNum semantics give;
// an infinite extent (tests/t04-swBVH: coordinates near +-1e38) gives 0.
static inline uint32_t quant10(float p, float lo, float hi) {
  float v = (p - lo) / (hi - lo);
  v = v * 1024.0f;
  v = std::fmax(v, 0.0f);
  v = std::fmin(v, 1023.0f);
  return (uint32_t)v;
}

static inline uint32_t code_of(f3 c, const float b[6], int kind) {
  uint32_t x = quant10(c.x, b[0], b[3]), y = quant10(c.y, b[1], b[4]), z = quant10(c.z, b[2], b[5]);
  return kind == 0 ? orc_morton3d(x, y, z) : orc_hilbert3d(x, y, z);
}

// Centroid (p1 + p2 + p3) / 3 (gprt/development/gprt_lbvh.hlsl:139-146),
// evaluated left to right.
extern "C" void orc_tri_codes(const float *pos, const uint32_t *tri, uint32_t n, const float bounds[6], int kind,
                              uint32_t *codes, uint32_t *ids) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    f3 p1 = ld3(pos, tri[3 * i]), p2 = ld3(pos, tri[3 * i + 1]), p3 = ld3(pos, tri[3 * i + 2]);
    f3 c = {((p1.x + p2.x) + p3.x) / 3.0f, ((p1.y + p2.y) + p3.y) / 3.0f, ((p1.z + p2.z) + p3.z) / 3.0f};
    codes[i] = code_of(c, bounds, kind);
    ids[i] = (uint32_t)i;
  }
}

extern "C" void orc_point_codes(const float *pos, uint32_t n, const float bounds[6], int kind, uint32_t *codes,
                                uint32_t *ids) {
  for (uint32_t i = 0; i < n; ++i) {
    codes[i] = code_of(ld3(pos, i), bounds, kind);
    ids[i] = i;
  }
}

// ============================================================================
// Karras topology
// ============================================================================
static inline int clz32(uint32_t v) { return v ? __builtin_clz(v) : 32; }

// delta(i,j) (gprt/development/gprt_lbvh.hlsl:45-61): longest common prefix of
// codes i and j, extended by the index bits when the codes are equal; -1 when j
// is outside [0,n).
static inline int kdelta(const uint32_t *c, int64_t n, int64_t i, int64_t j) {
  if (j < 0 || j >= n) return -1;
  uint32_t x = c[i] ^ c[j];
  if (x == 0) return clz32((uint32_t)i ^ (uint32_t)j) + 32;
  return clz32(x);
}

// determine_range + SplitNodes (gprt/development/gprt_lbvh.hlsl:64-103,287-338).
// The split search uses t = ceil(l / 2^k) in integers.  The reference forms it
// as ceil(l / divf) in fp32 and keeps iterating with t = 1 until divf
// overflows, which lands on the same (maximal) split.
extern "C" void orc_karras(const uint32_t *codes, uint32_t n, int32_t *nodes) {
  const int64_t N = n;
  for (int64_t k = 0; k < 4 * (2 * N - 1); ++k) nodes[k] = -1;
  if (n < 2) return;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < N - 1; ++i) {
    int d = kdelta(codes, N, i, i + 1) >= kdelta(codes, N, i, i - 1) ? 1 : -1;
    int dmin = kdelta(codes, N, i, i - d);
    int64_t lmax = 2;
    while (kdelta(codes, N, i, i + lmax * d) > dmin) lmax *= 2;
    int64_t l = 0;
    for (int64_t t = lmax >> 1; t >= 1; t >>= 1)
      if (kdelta(codes, N, i, i + (l + t) * d) > dmin) l += t;
    int64_t j = i + l * d;
    int dnode = kdelta(codes, N, i, j);
    int64_t s = 0;
    for (int64_t k = 1;; ++k) {
      int64_t t = (l + ((int64_t)1 << k) - 1) >> k;
      if (kdelta(codes, N, i, i + (s + t) * d) > dnode) s += t;
      if (t == 1) break;
    }
    int64_t split = i + s * d + std::min(d, 0);
    int64_t first = d == 1 ? i : j, last = d == 1 ? j : i;
    int64_t left = split, right = split + 1;
    int64_t lc = (left == first) ? (N - 1) + left : left;
    int64_t rc = (right == last) ? (N - 1) + right : right;
    nodes[4 * i + 0] = (int32_t)lc;
    nodes[4 * i + 1] = (int32_t)rc;
    nodes[4 * lc + 2] = (int32_t)i;
    nodes[4 * rc + 2] = (int32_t)i;
  }
}

// BuildTriangleHierarchy (gprt/development/gprt_lbvh.hlsl:400-428): leaf
// n-1+i holds triangle ids[i] and its box; every inner box is the min/max of
// the leaves below it, starting from MakeNodes' +-1e38 (:279-285).  min/max
// are exact, so evaluating it bottom-up as the union of the two children gives
// the identical bits.
extern "C" void orc_refit_tri(const float *pos, const uint32_t *tri, const uint32_t *ids, uint32_t n,
                              int32_t *nodes, float *aabbs) {
  if (n == 0) return;
  const int64_t N = n, inner = N - 1;
  for (int64_t k = 0; k < 2 * N - 1; ++k) {
    for (int a = 0; a < 3; ++a) {
      aabbs[6 * k + a] = 1e38f;
      aabbs[6 * k + 3 + a] = -1e38f;
    }
  }
  for (int64_t i = 0; i < N; ++i) {
    int64_t leaf = inner + i;
    tri_box(pos, tri, ids[i], &aabbs[6 * leaf]);
    nodes[4 * leaf + 3] = (int32_t)ids[i];
  }
  // Children of inner nodes are not index-ordered, so walk up from each leaf
  // with a visit counter: the second arrival computes the union.
  std::vector<uint8_t> seen(inner > 0 ? inner : 1, 0);
  for (int64_t i = 0; i < N; ++i) {
    int64_t cur = nodes[4 * (inner + i) + 2];
    while (cur >= 0) {
      if (seen[cur]++ == 0) break;
      int64_t l = nodes[4 * cur], r = nodes[4 * cur + 1];
      float *b = &aabbs[6 * cur];
      for (int a = 0; a < 3; ++a) {
        b[a] = std::fmin(b[a], std::fmin(aabbs[6 * l + a], aabbs[6 * r + a]));
        b[3 + a] = std::fmax(b[3 + a], std::fmax(aabbs[6 * l + 3 + a], aabbs[6 * r + 3 + a]));
      }
      cur = nodes[4 * cur + 2];
    }
  }
}

// Point variant: ComputePointBounds / ComputePointMortonCodes /
// BuildPointHierarchy (gprt/development/gprt_lbvh.hlsl:188-199,228-243,340-368):
// a leaf box is the point itself.
extern "C" void orc_lbvh_build_points(const float *pos, uint32_t n, int kind, float scene[6], uint32_t *codes,
                                      uint32_t *ids, int32_t *nodes, float *aabbs) {
  orc_point_bounds(pos, n, scene);
  orc_point_codes(pos, n, scene, kind, codes, ids);
  orc_sort(codes, 4, ids, 4, n);
  orc_karras(codes, n, nodes);
  if (n == 0) return;
  // Leaf box (p, p); reuse the triangle refit with a degenerate index triple.
  std::vector<uint32_t> tri(3 * (size_t)n);
  for (uint32_t i = 0; i < n; ++i) tri[3 * i] = tri[3 * i + 1] = tri[3 * i + 2] = i;
  orc_refit_tri(pos, tri.data(), ids, n, nodes, aabbs);
}

// Edge variant: ComputeEdgeBounds / ComputeEdgeMortonCodes /
// BuildEdgeHierarchy (gprt/development/gprt_lbvh.hlsl:112-119,131-136,202-213,
// 245-260,370-398): a leaf box is the min/max of the two endpoints (the
// triangle box of the triple (p1, p2, p2) has the same bits), the code that of
// (p1 + p2) / 2.
extern "C" void orc_lbvh_build_edges(const float *pos, const uint32_t *edges, uint32_t n, int kind, float scene[6],
                                     uint32_t *codes, uint32_t *ids, int32_t *nodes, float *aabbs) {
  std::vector<uint32_t> tri(3 * (size_t)n);
  for (uint32_t i = 0; i < n; ++i) {
    tri[3 * i] = edges[2 * i];
    tri[3 * i + 1] = tri[3 * i + 2] = edges[2 * i + 1];
  }
  orc_tri_bounds(pos, tri.data(), n, scene);
  for (uint32_t i = 0; i < n; ++i) {
    f3 p1 = ld3(pos, edges[2 * i]), p2 = ld3(pos, edges[2 * i + 1]);
    f3 c = {(p1.x + p2.x) / 2.0f, (p1.y + p2.y) / 2.0f, (p1.z + p2.z) / 2.0f};
    codes[i] = code_of(c, scene, kind);
    ids[i] = i;
  }
  orc_sort(codes, 4, ids, 4, n);
  orc_karras(codes, n, nodes);
  orc_refit_tri(pos, tri.data(), ids, n, nodes, aabbs);
}

extern "C" void orc_lbvh_build_tri(const float *pos, const uint32_t *tri, uint32_t n, int kind, float scene[6],
                                   uint32_t *codes, uint32_t *ids, int32_t *nodes, float *aabbs) {
  orc_tri_bounds(pos, tri, n, scene);
  orc_tri_codes(pos, tri, n, scene, kind, codes, ids);
  orc_sort(codes, 4, ids, 4, n);
  orc_karras(codes, n, nodes);
  orc_refit_tri(pos, tri, ids, n, nodes, aabbs);
}

// ============================================================================
// ray / triangle
// ============================================================================
// Kahan's 2x2 determinant a*d - b*c with one fused correction; its sign is
// exact (relative error <= 2u, Jeannerod-Louvet-Muller 2013), which is what
// makes the edge tests below watertight without a higher-precision retry.
static inline float det2(float a, float b, float c, float d) {
  float w = b * c;
  float e = std::fma(-b, c, w);
  float f = std::fma(a, d, -w);
  return f + e;
}

struct RayPre {
  float o[3], d[3], tmin, tmax;
  int kx, ky, kz;
  float Sx, Sy, Sz;
  float inv[3];
};

// Per-ray set-up of Woop et al. 2013, section 3: kz is the axis of the
// largest |d| (lowest index on ties), kx/ky follow cyclically and swap when
// d[kz] < 0 to keep the winding.
static inline void ray_pre(const float *r, RayPre &p) {
  p.o[0] = r[0]; p.o[1] = r[1]; p.o[2] = r[2]; p.tmin = r[3];
  p.d[0] = r[4]; p.d[1] = r[5]; p.d[2] = r[6]; p.tmax = r[7];
  float ax = std::fabs(p.d[0]), ay = std::fabs(p.d[1]), az = std::fabs(p.d[2]);
  int kz = (ax >= ay) ? (ax >= az ? 0 : 2) : (ay >= az ? 1 : 2);
  int kx = kz + 1 == 3 ? 0 : kz + 1;
  int ky = kx + 1 == 3 ? 0 : kx + 1;
  if (p.d[kz] < 0.0f) std::swap(kx, ky);
  p.kx = kx; p.ky = ky; p.kz = kz;
  p.Sx = p.d[kx] / p.d[kz];
  p.Sy = p.d[ky] / p.d[kz];
  p.Sz = 1.0f / p.d[kz];
  for (int a = 0; a < 3; ++a) p.inv[a] = 1.0f / p.d[a];
}

// Watertight test, Woop et al. 2013 section 3 with the edge functions from
// det2().  Returns the hit distance t = T / det in (*t) when the ray crosses
// the triangle inside [tmin, tmax].
static inline int isect32(const RayPre &p, const float *v0, const float *v1, const float *v2, float *tout) {
  float A[3] = {v0[0] - p.o[0], v0[1] - p.o[1], v0[2] - p.o[2]};
  float B[3] = {v1[0] - p.o[0], v1[1] - p.o[1], v1[2] - p.o[2]};
  float C[3] = {v2[0] - p.o[0], v2[1] - p.o[1], v2[2] - p.o[2]};
  float Ax = A[p.kx] - p.Sx * A[p.kz], Ay = A[p.ky] - p.Sy * A[p.kz];
  float Bx = B[p.kx] - p.Sx * B[p.kz], By = B[p.ky] - p.Sy * B[p.kz];
  float Cx = C[p.kx] - p.Sx * C[p.kz], Cy = C[p.ky] - p.Sy * C[p.kz];
  float U = det2(Cx, Cy, Bx, By);  // Cx*By - Cy*Bx
  float V = det2(Ax, Ay, Cx, Cy);  // Ax*Cy - Ay*Cx
  float W = det2(Bx, By, Ax, Ay);  // Bx*Ay - By*Ax
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return 0;
  float det = (U + V) + W;
  if (det == 0.0f) return 0;
  float Az = p.Sz * A[p.kz], Bz = p.Sz * B[p.kz], Cz = p.Sz * C[p.kz];
  float T = (U * Az + V * Bz) + W * Cz;
  float t = T / det;
  if (!(t >= p.tmin && t <= p.tmax)) return 0;
  *tout = t;
  return 1;
}

extern "C" int orc_isect_tri32(const float *ray, const float *v0, const float *v1, const float *v2, float *t) {
  RayPre p;
  ray_pre(ray, p);
  return isect32(p, v0, v1, v2, t);
}

// ---- double-float (unevaluated pair of fp32) arithmetic: Dekker 1971,
// Knuth TAOCP vol. 2 4.2.2 (TwoSum), FMA-based TwoProduct. ----
struct df {
  float hi, lo;
};
static inline df two_sum(float a, float b) {
  float s = a + b;
  float bb = s - a;
  float e = (a - (s - bb)) + (b - bb);
  return {s, e};
}
static inline df fast_two_sum(float a, float b) {
  float s = a + b;
  float e = b - (s - a);
  return {s, e};
}
static inline df two_prod(float a, float b) {
  float p = a * b;
  return {p, std::fma(a, b, -p)};
}
static inline df df_add(df x, df y) {
  df s = two_sum(x.hi, y.hi);
  df t = two_sum(x.lo, y.lo);
  s.lo = s.lo + t.hi;
  s = fast_two_sum(s.hi, s.lo);
  s.lo = s.lo + t.lo;
  return fast_two_sum(s.hi, s.lo);
}
static inline df df_neg(df x) { return {-x.hi, -x.lo}; }
static inline df df_mul(df x, df y) {
  df p = two_prod(x.hi, y.hi);
  p.lo = p.lo + (x.hi * y.lo + x.lo * y.hi);
  return fast_two_sum(p.hi, p.lo);
}
static inline df df_mulf(df x, float y) {
  df p = two_prod(x.hi, y);
  p.lo = p.lo + x.lo * y;
  return fast_two_sum(p.hi, p.lo);
}
static inline float df_div_to_f(df x, df y) {
  float q1 = x.hi / y.hi;
  df r = df_add(x, df_neg(df_mulf(y, q1)));
  float q2 = r.hi / y.hi;
  df q = fast_two_sum(q1, q2);
  return q.hi + q.lo;
}

// Plane-equation distance t = ((v0 - o) . n) / (d . n), n = (v1-v0) x (v2-v0),
// evaluated in double-float and rounded once to fp32.  Used only to report the
// distance of the winning hit; which triangle wins is decided by isect32().
extern "C" float orc_refine_t32(const float *ray, const float *v0, const float *v1, const float *v2) {
  df e1[3], e2[3], w[3];
  for (int a = 0; a < 3; ++a) {
    e1[a] = two_sum(v1[a], -v0[a]);
    e2[a] = two_sum(v2[a], -v0[a]);
    w[a] = two_sum(v0[a], -ray[a]);
  }
  df n[3];
  n[0] = df_add(df_mul(e1[1], e2[2]), df_neg(df_mul(e1[2], e2[1])));
  n[1] = df_add(df_mul(e1[2], e2[0]), df_neg(df_mul(e1[0], e2[2])));
  n[2] = df_add(df_mul(e1[0], e2[1]), df_neg(df_mul(e1[1], e2[0])));
  df num = df_add(df_add(df_mul(n[0], w[0]), df_mul(n[1], w[1])), df_mul(n[2], w[2]));
  df den = df_add(df_add(df_mulf(n[0], ray[4]), df_mulf(n[1], ray[5])), df_mulf(n[2], ray[6]));
  return df_div_to_f(num, den);
}

extern "C" double orc_t64(const float *ray, const float *v0, const float *v1, const float *v2) {
  double e1[3], e2[3], w[3];
  for (int a = 0; a < 3; ++a) {
    e1[a] = (double)v1[a] - (double)v0[a];
    e2[a] = (double)v2[a] - (double)v0[a];
    w[a] = (double)v0[a] - (double)ray[a];
  }
  double n0 = e1[1] * e2[2] - e1[2] * e2[1];
  double n1 = e1[2] * e2[0] - e1[0] * e2[2];
  double n2 = e1[0] * e2[1] - e1[1] * e2[0];
  double num = n0 * w[0] + n1 * w[1] + n2 * w[2];
  double den = n0 * (double)ray[4] + n1 * (double)ray[5] + n2 * (double)ray[6];
  return num / den;
}

// ============================================================================
// ray / box and traversal
// ============================================================================
// Slab test, Ize 2013: per-axis (b - o) * (1/d); NaN slabs (0 * inf, a ray in
// a face plane) impose no bound.
// The entry is scaled down and the exit up by 2^-18 so that a triangle hit the
// watertight test reports is never pruned by a box that contains it.
static const float kBoxLo = 1.0f - 1.0f / 262144.0f;
static const float kBoxHi = 1.0f + 1.0f / 262144.0f;

// Per-axis min/max propagate NaN (a ray parallel to an axis lying in a face
// plane gives 0 * inf); the accumulation below then drops that axis, so it
// imposes no bound -- the conservative answer.
static inline float nmin(float a, float b) { return (std::isnan(a) || std::isnan(b)) ? NAN : std::fmin(a, b); }
static inline float nmax(float a, float b) { return (std::isnan(a) || std::isnan(b)) ? NAN : std::fmax(a, b); }

static inline int ray_box(const RayPre &p, const float *b, float tmax, float *tnear_out) {
  float t0x = (b[0] - p.o[0]) * p.inv[0], t1x = (b[3] - p.o[0]) * p.inv[0];
  float t0y = (b[1] - p.o[1]) * p.inv[1], t1y = (b[4] - p.o[1]) * p.inv[1];
  float t0z = (b[2] - p.o[2]) * p.inv[2], t1z = (b[5] - p.o[2]) * p.inv[2];
  float tn = std::fmax(std::fmax(nmin(t0x, t1x), nmin(t0y, t1y)), std::fmax(nmin(t0z, t1z), p.tmin));
  float tf = std::fmin(std::fmin(nmax(t0x, t1x), nmax(t0y, t1y)), std::fmin(nmax(t0z, t1z), tmax));
  tn = tn * kBoxLo;
  tf = tf * kBoxHi;
  *tnear_out = tn;
  return tn <= tf;
}

static inline void tri_verts(const float *pos, const uint32_t *tri, uint32_t id, const float *&a, const float *&b,
                             const float *&c) {
  a = pos + 3 * (size_t)tri[3 * (size_t)id];
  b = pos + 3 * (size_t)tri[3 * (size_t)id + 1];
  c = pos + 3 * (size_t)tri[3 * (size_t)id + 2];
}

extern "C" void orc_trace_brute(const float *pos, const uint32_t *tri, uint32_t n, const float *rays, uint64_t nrays,
                                orc_hit *hits) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t r = 0; r < (int64_t)nrays; ++r) {
    RayPre p;
    ray_pre(rays + 8 * r, p);
    uint32_t best = 0xFFFFFFFFu;
    float bt = 0.0f;
    for (uint32_t i = 0; i < n; ++i) {
      const float *a, *b, *c;
      tri_verts(pos, tri, i, a, b, c);
      float t;
      if (isect32(p, a, b, c, &t) && (best == 0xFFFFFFFFu || t < bt)) {
        best = i;
        bt = t;
      }
    }
    hits[r].prim = best;
    if (best != 0xFFFFFFFFu) {
      const float *a, *b, *c;
      tri_verts(pos, tri, best, a, b, c);
      hits[r].t = orc_refine_t32(rays + 8 * r, a, b, c);
    } else {
      hits[r].t = INFINITY;
    }
  }
}

// Depth-first traversal of the reference layout.  A node is entered when its
// box passes ray_box and its entry distance does not exceed the best hit so
// far (equal entry distance is entered, so that a tie can still be won by a
// lower primitive id).  Closest hit = smallest (t, primID).
extern "C" void orc_trace_lbvh(const float *pos, const uint32_t *tri, uint32_t n, const int32_t *nodes,
                               const float *aabbs, const float *rays, uint64_t nrays, int anyhit, orc_hit *hits) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t r = 0; r < (int64_t)nrays; ++r) {
    RayPre p;
    ray_pre(rays + 8 * r, p);
    uint32_t best = 0xFFFFFFFFu;
    float bt = p.tmax;
    if (n > 0) {
      int32_t stack[128];
      int sp = 0;
      stack[sp++] = 0;
      while (sp > 0) {
        int32_t node = stack[--sp];
        float tn;
        if (!ray_box(p, &aabbs[6 * (size_t)node], bt, &tn)) continue;
        if (tn > bt) continue;
        int32_t leaf = nodes[4 * (size_t)node + 3];
        if (leaf >= 0) {
          const float *a, *b, *c;
          tri_verts(pos, tri, (uint32_t)leaf, a, b, c);
          float t;
          if (isect32(p, a, b, c, &t)) {
            if (best == 0xFFFFFFFFu || t < bt || (t == bt && (uint32_t)leaf < best)) {
              best = (uint32_t)leaf;
              bt = t;
              if (anyhit) break;
            }
          }
        } else {
          stack[sp++] = nodes[4 * (size_t)node + 1];
          stack[sp++] = nodes[4 * (size_t)node + 0];
        }
      }
    }
    hits[r].prim = best;
    if (best != 0xFFFFFFFFu) {
      const float *a, *b, *c;
      tri_verts(pos, tri, best, a, b, c);
      hits[r].t = orc_refine_t32(rays + 8 * r, a, b, c);
    } else {
      hits[r].t = INFINITY;
    }
  }
}

// ---- FP64 closest hit through the same tree: the accuracy reference for
// hit ids.  The watertight test of isect32 (Woop et al. 2013, section 3)
// carried out in double precision on the float inputs, ties to the lowest
// id; boxes tested by ray_box as in orc_trace_lbvh (the 2^-18 widening also
// covers double-precision hits, which lie inside the same float boxes).  Rays
// whose FP32 and FP64 closest ids differ are the diagnostic this serves: hits
// at shared edges and near-ties that FP32 cannot separate.
struct RayPre64 {
  double o[3], d[3], tmin, tmax;
  int kx, ky, kz;
  double Sx, Sy, Sz;
};
static inline void ray_pre64(const float *r, RayPre64 &p) {
  for (int a = 0; a < 3; ++a) {
    p.o[a] = r[a];
    p.d[a] = r[4 + a];
  }
  p.tmin = r[3];
  p.tmax = r[7];
  double ax = std::fabs(p.d[0]), ay = std::fabs(p.d[1]), az = std::fabs(p.d[2]);
  int kz = (ax >= ay) ? (ax >= az ? 0 : 2) : (ay >= az ? 1 : 2);
  int kx = kz + 1 == 3 ? 0 : kz + 1;
  int ky = kx + 1 == 3 ? 0 : kx + 1;
  if (p.d[kz] < 0.0) std::swap(kx, ky);
  p.kx = kx;
  p.ky = ky;
  p.kz = kz;
  p.Sx = p.d[kx] / p.d[kz];
  p.Sy = p.d[ky] / p.d[kz];
  p.Sz = 1.0 / p.d[kz];
}
static inline int isect64(const RayPre64 &p, const float *v0, const float *v1, const float *v2, double *tout) {
  double A[3], B[3], C[3];
  for (int a = 0; a < 3; ++a) {
    A[a] = (double)v0[a] - p.o[a];
    B[a] = (double)v1[a] - p.o[a];
    C[a] = (double)v2[a] - p.o[a];
  }
  double Ax = A[p.kx] - p.Sx * A[p.kz], Ay = A[p.ky] - p.Sy * A[p.kz];
  double Bx = B[p.kx] - p.Sx * B[p.kz], By = B[p.ky] - p.Sy * B[p.kz];
  double Cx = C[p.kx] - p.Sx * C[p.kz], Cy = C[p.ky] - p.Sy * C[p.kz];
  double U = Cx * By - Cy * Bx, V = Ax * Cy - Ay * Cx, W = Bx * Ay - By * Ax;
  if ((U < 0.0 || V < 0.0 || W < 0.0) && (U > 0.0 || V > 0.0 || W > 0.0)) return 0;
  double det = (U + V) + W;
  if (det == 0.0) return 0;
  double T = (U * (p.Sz * A[p.kz]) + V * (p.Sz * B[p.kz])) + W * (p.Sz * C[p.kz]);
  double t = T / det;
  if (!(t >= p.tmin && t <= p.tmax)) return 0;
  *tout = t;
  return 1;
}

extern "C" int orc_isect_tri64(const float *ray, const float *v0, const float *v1, const float *v2, double *t) {
  RayPre64 q;
  ray_pre64(ray, q);
  return isect64(q, v0, v1, v2, t);
}

extern "C" void orc_trace_lbvh64(const float *pos, const uint32_t *tri, uint32_t n, const int32_t *nodes,
                                 const float *aabbs, const float *rays, uint64_t nrays, uint32_t *prim, double *tout) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t r = 0; r < (int64_t)nrays; ++r) {
    RayPre p;
    ray_pre(rays + 8 * r, p);
    RayPre64 q;
    ray_pre64(rays + 8 * r, q);
    uint32_t best = 0xFFFFFFFFu;
    double bt = q.tmax;
    if (n > 0) {
      int32_t stack[128];
      int sp = 0;
      stack[sp++] = 0;
      while (sp > 0) {
        int32_t node = stack[--sp];
        float tn;
        // culling distance rounded up to float, so no box holding a hit at bt is pruned
        const float btf = (float)bt < bt ? std::nextafter((float)bt, INFINITY) : (float)bt;
        if (!ray_box(p, &aabbs[6 * (size_t)node], btf, &tn)) continue;
        if ((double)tn > bt) continue;
        int32_t leaf = nodes[4 * (size_t)node + 3];
        if (leaf >= 0) {
          const float *a, *b, *c;
          tri_verts(pos, tri, (uint32_t)leaf, a, b, c);
          double t;
          if (isect64(q, a, b, c, &t) && (best == 0xFFFFFFFFu || t < bt || (t == bt && (uint32_t)leaf < best))) {
            best = (uint32_t)leaf;
            bt = t;
          }
        } else {
          stack[sp++] = nodes[4 * (size_t)node + 1];
          stack[sp++] = nodes[4 * (size_t)node + 0];
        }
      }
    }
    prim[r] = best;
    tout[r] = best != 0xFFFFFFFFu ? bt : INFINITY;
  }
}

extern "C" int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// ============================================================================
// Spheres and linearly swept spheres (LSS): the software counterparts of the
// reference's AABB primitives (gprt/gprt_fallbacks.slang).  Each float op is
// written out in the reference's evaluation order; dot(a, b) is
// (a.x*b.x + a.y*b.y) + a.z*b.z and rcp(x) is 1/x.
// ============================================================================
static inline float dot3(f3 a, f3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

// intersectRayLSS (gprt/gprt_fallbacks.slang:45-144).
static bool lss_intersect(f3 ro, f3 rd, f3 p0, f3 p1, float r0, float r1, bool cap0, bool cap1, float tmin,
                          float tmax, bool exit_test, float *t_out, float *u_out) {
  *t_out = 0.0f;
  *u_out = 0.0f;
  const f3 d = rd;
  const f3 mid = {0.5f * (p0.x + p1.x), 0.5f * (p0.y + p1.y), 0.5f * (p0.z + p1.z)};
  const float rmid = 0.5f * (r0 + r1);
  const float dd = dot3(d, d);
  const float inv_dd = 1.0f / dd;
  const float align = dot3(d, f3{mid.x - ro.x, mid.y - ro.y, mid.z - ro.z}) * inv_dd;
  ro = f3{ro.x + align * d.x, ro.y + align * d.y, ro.z + align * d.z};
  const f3 off = {ro.x - mid.x, ro.y - mid.y, ro.z - mid.z};
  const f3 axis = {p1.x - p0.x, p1.y - p0.y, p1.z - p0.z};
  const float rdel = r1 - r0;
  const float a = dd;
  const float b = dot3(axis, d);
  const float c = dot3(axis, axis) - rdel * rdel;
  const float dq = dot3(d, off);
  const float e = dot3(axis, off) + rmid * rdel;
  const float f = dot3(off, off) - rmid * rmid;
  const float At = b * b - a * c;
  const float Bt = b * e - c * dq;
  const float Ct = e * e - c * f;
  const float disc = Bt * Bt - At * Ct;
  const bool is_sphere = axis.x == 0 && axis.y == 0 && axis.z == 0 && rdel == 0;
  const bool use_start_sphere = !cap1;
  const bool shell_degenerate = (c <= 0) && (rdel != 0);
  const bool invalid = (r0 <= 0 && r1 <= 0) || std::isnan(r0) || std::isnan(r1) || std::isnan(p0.x) ||
                       std::isnan(p1.x) || std::isinf(r0) || std::isinf(p0.x);
  if ((!is_sphere && !shell_degenerate && disc < 0) || invalid) return false;
  const float sq = std::sqrt(disc);
  const float inv_at = 1.0f / At;
  const float t0 = (-Bt + (exit_test ? -sq : sq)) * inv_at;
  const float inv_c = 1.0f / c;
  const float u0 = (b * t0 + e) * inv_c;
  if (std::fabs(u0) <= 0.5f && (u0 * rdel >= -rmid) && !is_sphere && !shell_degenerate) {
    const float ht = t0 + align, hu = u0 + 0.5f;
    if (ht <= tmin || ht >= tmax) return false;
    *t_out = ht;
    *u_out = hu;
    return true;
  }
  const bool start_cap = is_sphere ? use_start_sphere : (u0 < 0.0f);
  if ((start_cap && !cap0) || (!start_cap && !cap1)) return false;
  const float Bs = -dq + (start_cap ? -b : b) * 0.5f;
  const float BsBs = Bs * Bs;
  const float Cs = f + 0.25f * c - (start_cap ? -e : e);
  const float AsCs = a * Cs;
  if (BsBs < AsCs) return false;
  const float sqc = std::sqrt(BsBs - AsCs);
  const float cap_t = (Bs - (exit_test ? -sqc : sqc)) * inv_dd;
  *t_out = cap_t + align;
  *u_out = start_cap ? 0.0f : 1.0f;
  if (*t_out <= tmin || *t_out >= tmax) return false;
  return true;
}

extern "C" int orc_lss_intersect(const float *ray, const float *v0, const float *v1, int cap0, int cap1, int exit_test,
                                 float *t, float *u) {
  return lss_intersect(f3{ray[0], ray[1], ray[2]}, f3{ray[4], ray[5], ray[6]}, f3{v0[0], v0[1], v0[2]},
                       f3{v1[0], v1[1], v1[2]}, v0[3], v1[3], cap0 != 0, cap1 != 0, ray[3], ray[7], exit_test != 0, t,
                       u)
             ? 1
             : 0;
}

// computeLssAabb (gprt/gprt_fallbacks.slang:168-213) and LSSBounds
// (:215-235): vertices float4 {xyz, radius}, indices uint2 per segment;
// aabbs [n][6] {lo.xyz, hi.xyz}.
static void lss_aabb(f3 v0, float r0, bool cap0, f3 v1, float r1, bool cap1, float *lo, float *hi) {
  f3 blo0 = v0, bhi0 = v0, blo1 = v1, bhi1 = v1;
  f3 cme = {0, 0, 0}, cpe = {0, 0, 0};
  if (!cap0 || !cap1) {
    const float rd = r1 - r0;
    const f3 n = {v0.x - v1.x, v0.y - v1.y, v0.z - v1.z};
    const f3 nsq = {n.x * n.x, n.y * n.y, n.z * n.z};
    const float l2 = (nsq.x + nsq.y) + nsq.z;
    const float l2inv = 1.0f / l2;
    const f3 X = {1.f - nsq.x * l2inv, 1.f - nsq.y * l2inv, 1.f - nsq.z * l2inv};
    const float Y = 1.f - rd * rd * l2inv;
    const f3 e = {std::sqrt(std::fabs(X.x * Y)), std::sqrt(std::fabs(X.y * Y)), std::sqrt(std::fabs(X.z * Y))};
    const f3 c = {rd * n.x * l2inv, rd * n.y * l2inv, rd * n.z * l2inv};
    cme = {c.x - e.x, c.y - e.y, c.z - e.z};
    cpe = {c.x + e.x, c.y + e.y, c.z + e.z};
  }
  if (r0 < 0.0f) {
    const float s = r0 * (1.0f / (r1 - r0));
    blo0 = {blo0.x + s * (v0.x - v1.x), blo0.y + s * (v0.y - v1.y), blo0.z + s * (v0.z - v1.z)};
    bhi0 = blo0;
  } else if (cap0) {
    blo0 = {blo0.x + -r0, blo0.y + -r0, blo0.z + -r0};
    bhi0 = {bhi0.x + r0, bhi0.y + r0, bhi0.z + r0};
  } else {
    blo0 = {blo0.x + r0 * cme.x, blo0.y + r0 * cme.y, blo0.z + r0 * cme.z};
    bhi0 = {bhi0.x + r0 * cpe.x, bhi0.y + r0 * cpe.y, bhi0.z + r0 * cpe.z};
  }
  if (r1 < 0.0f) {
    const float s = r1 * (1.0f / (r1 - r0));
    blo1 = {blo1.x + s * (v0.x - v1.x), blo1.y + s * (v0.y - v1.y), blo1.z + s * (v0.z - v1.z)};
    bhi1 = blo1;
  } else if (cap1) {
    blo1 = {blo1.x + -r1, blo1.y + -r1, blo1.z + -r1};
    bhi1 = {bhi1.x + r1, bhi1.y + r1, bhi1.z + r1};
  } else {
    blo1 = {blo1.x + r1 * cme.x, blo1.y + r1 * cme.y, blo1.z + r1 * cme.z};
    bhi1 = {bhi1.x + r1 * cpe.x, bhi1.y + r1 * cpe.y, bhi1.z + r1 * cpe.z};
  }
  lo[0] = std::fmin(blo0.x, blo1.x);
  lo[1] = std::fmin(blo0.y, blo1.y);
  lo[2] = std::fmin(blo0.z, blo1.z);
  hi[0] = std::fmax(bhi0.x, bhi1.x);
  hi[1] = std::fmax(bhi0.y, bhi1.y);
  hi[2] = std::fmax(bhi0.z, bhi1.z);
}

extern "C" void orc_lss_bounds(const float *verts, const uint32_t *idx, uint32_t n, int cap0, int cap1, float *aabbs) {
  for (uint32_t i = 0; i < n; ++i) {
    const float *a = verts + 4 * (size_t)idx[2 * i], *b = verts + 4 * (size_t)idx[2 * i + 1];
    lss_aabb(f3{a[0], a[1], a[2]}, a[3], cap0 != 0, f3{b[0], b[1], b[2]}, b[3], cap1 != 0, aabbs + 6 * (size_t)i,
             aabbs + 6 * (size_t)i + 3);
  }
}

// SphereBounds (gprt/gprt_fallbacks.slang:263-283): spheres float4 {center, radius}.
extern "C" void orc_sphere_bounds(const float *spheres, uint32_t n, float *aabbs) {
  const float M = 3.402823466e38f;
  for (uint32_t i = 0; i < n; ++i) {
    const float *s = spheres + 4 * (size_t)i;
    const float r = std::fmax(s[3], 0.0f);
    for (int k = 0; k < 3; ++k) {
      aabbs[6 * (size_t)i + k] = std::fmin(M, s[k] - r);
      aabbs[6 * (size_t)i + 3 + k] = std::fmax(-M, s[k] + r);
    }
  }
}

// Closest hit over every primitive (SphereIntersection / LSSIntersection,
// gprt/gprt_fallbacks.slang:146-166,245-261): the intersection is tested
// against the ray's own [tmin, tmax]; the closest t wins, ties to the lowest
// id.  kind 0: spheres (prims = float4 per sphere, the LSS test with both
// ends equal and both caps on); kind 1: LSS (prims = vertices, idx = uint2).
struct orc_uhit {
  uint32_t prim;
  float t;
  float u;
};
extern "C" void orc_trace_user_brute(int kind, const float *prims, const uint32_t *idx, uint32_t n, int cap0, int cap1,
                                     int exit_test, const float *rays, uint64_t nrays, orc_uhit *hits) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t r = 0; r < (int64_t)nrays; ++r) {
    const float *ray = rays + 8 * r;
    uint32_t best = 0xFFFFFFFFu;
    float bt = 0.0f, bu = 0.0f;
    for (uint32_t i = 0; i < n; ++i) {
      const float *a = kind == 0 ? prims + 4 * (size_t)i : prims + 4 * (size_t)idx[2 * i];
      const float *b = kind == 0 ? a : prims + 4 * (size_t)idx[2 * i + 1];
      const bool c0 = kind == 0 ? true : cap0 != 0, c1 = kind == 0 ? true : cap1 != 0;
      float t, u;
      if (lss_intersect(f3{ray[0], ray[1], ray[2]}, f3{ray[4], ray[5], ray[6]}, f3{a[0], a[1], a[2]},
                        f3{b[0], b[1], b[2]}, a[3], b[3], c0, c1, ray[3], ray[7], exit_test != 0, &t, &u) &&
          (best == 0xFFFFFFFFu || t < bt)) {
        best = i;
        bt = t;
        bu = u;
      }
    }
    hits[r].prim = best;
    hits[r].t = best == 0xFFFFFFFFu ? INFINITY : bt;
    hits[r].u = best == 0xFFFFFFFFu ? 0.0f : bu;
  }
}

// LBVH over given boxes [n][6] (the primitives' AABBs): centroid
// (lo + hi) * 0.5, otherwise the same codes, sort, topology and refit.
extern "C" void orc_lbvh_build_boxes(const float *boxes, uint32_t n, int kind, float scene[6], uint32_t *codes,
                                     uint32_t *ids, int32_t *nodes, float *aabbs) {
  const float M = 3.402823466e38f;
  float s[6] = {M, M, M, -M, -M, -M};
  for (uint32_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      s[k] = std::fmin(s[k], boxes[6 * (size_t)i + k]);
      s[3 + k] = std::fmax(s[3 + k], boxes[6 * (size_t)i + 3 + k]);
    }
  std::memcpy(scene, s, sizeof(s));
  for (uint32_t i = 0; i < n; ++i) {
    const float *b = boxes + 6 * (size_t)i;
    f3 c = {(b[0] + b[3]) * 0.5f, (b[1] + b[4]) * 0.5f, (b[2] + b[5]) * 0.5f};
    codes[i] = code_of(c, scene, kind);
    ids[i] = i;
  }
  orc_sort(codes, 4, ids, 4, n);
  orc_karras(codes, n, nodes);
  if (n == 0) return;
  const int64_t N = n, inner = N - 1;
  for (int64_t k = 0; k < 2 * N - 1; ++k)
    for (int a = 0; a < 3; ++a) {
      aabbs[6 * k + a] = 1e38f;
      aabbs[6 * k + 3 + a] = -1e38f;
    }
  for (int64_t i = 0; i < N; ++i) {
    std::memcpy(&aabbs[6 * (inner + i)], boxes + 6 * (size_t)ids[i], 24);
    nodes[4 * (inner + i) + 3] = (int32_t)ids[i];
  }
  std::vector<uint8_t> seen(inner > 0 ? inner : 1, 0);
  for (int64_t i = 0; i < N; ++i) {
    int64_t cur = nodes[4 * (inner + i) + 2];
    while (cur >= 0) {
      if (seen[cur]++ == 0) break;
      int64_t l = nodes[4 * cur], r = nodes[4 * cur + 1];
      float *b = &aabbs[6 * cur];
      for (int a = 0; a < 3; ++a) {
        b[a] = std::fmin(b[a], std::fmin(aabbs[6 * l + a], aabbs[6 * r + a]));
        b[3 + a] = std::fmax(b[3 + a], std::fmax(aabbs[6 * l + 3 + a], aabbs[6 * r + 3 + a]));
      }
      cur = nodes[4 * cur + 2];
    }
  }
}

// ============================================================================
// Two-level instancing: instances of the meshes of a batch, each with a
// row-major 3x4 object-to-world transform (the reference's gprt::Instance,
// gprt/gprt_shared.h:92-101: transform, customIndex:24, mask:8,
// geometryIndex:24, flags:8, accelAddress -- here the mesh index).
// ============================================================================
struct orc_instance {
  float m[12];
  uint32_t custom_mask;
  uint32_t geom_flags;
  uint64_t blas;
};
struct orc_ihit {
  uint32_t prim;
  float t;
  uint32_t inst;
};

// World-to-object matrix: the inverse of [A | t] by adjugate and determinant
// in double, in a fixed operation order, each entry rounded once to float.
// False (and zeros) when A is singular.
extern "C" int orc_instance_inverse(const float *m, float *w) {
  const double a00 = m[0], a01 = m[1], a02 = m[2], t0 = m[3];
  const double a10 = m[4], a11 = m[5], a12 = m[6], t1 = m[7];
  const double a20 = m[8], a21 = m[9], a22 = m[10], t2 = m[11];
  const double c00 = a11 * a22 - a12 * a21, c01 = a12 * a20 - a10 * a22, c02 = a10 * a21 - a11 * a20;
  const double c10 = a02 * a21 - a01 * a22, c11 = a00 * a22 - a02 * a20, c12 = a01 * a20 - a00 * a21;
  const double c20 = a01 * a12 - a02 * a11, c21 = a02 * a10 - a00 * a12, c22 = a00 * a11 - a01 * a10;
  const double det = (a00 * c00 + a01 * c01) + a02 * c02;
  if (!(det != 0.0) || !std::isfinite(det)) {
    for (int k = 0; k < 12; ++k) w[k] = 0.0f;
    return 0;
  }
  const double i00 = c00 / det, i01 = c10 / det, i02 = c20 / det;
  const double i10 = c01 / det, i11 = c11 / det, i12 = c21 / det;
  const double i20 = c02 / det, i21 = c12 / det, i22 = c22 / det;
  const double u0 = -((i00 * t0 + i01 * t1) + i02 * t2);
  const double u1 = -((i10 * t0 + i11 * t1) + i12 * t2);
  const double u2 = -((i20 * t0 + i21 * t1) + i22 * t2);
  const double r[12] = {i00, i01, i02, u0, i10, i11, i12, u1, i20, i21, i22, u2};
  for (int k = 0; k < 12; ++k) w[k] = (float)r[k];
  return 1;
}

// The ray in an instance's object space: origin and direction through the
// world-to-object matrix, each component ((w0*x + w1*y) + w2*z) (+ w3), in
// float; tmin / tmax unchanged (an affine map keeps the ray parameter).
static inline void ray_to_object(const float *w, const float *ray, float *out) {
  for (int i = 0; i < 3; ++i) {
    out[i] = ((w[4 * i] * ray[0] + w[4 * i + 1] * ray[1]) + w[4 * i + 2] * ray[2]) + w[4 * i + 3];
    out[4 + i] = (w[4 * i] * ray[4] + w[4 * i + 1] * ray[5]) + w[4 * i + 2] * ray[6];
  }
  out[3] = ray[3];
  out[7] = ray[7];
}

// Closest hit over every triangle of every visible instance ((mask & rayMask)
// != 0, non-singular transform): ties to the lowest (instance, primitive).
// Primitive ids are mesh-local; t is the refined plane-equation distance in
// the winning instance's object space.
extern "C" void orc_trace_instances_brute(const orc_instance *inst, uint32_t ninst, const float *pos,
                                          const uint32_t *tri, const uint32_t *tri_off, uint32_t meshes,
                                          const float *rays, uint64_t nrays, uint32_t ray_mask, orc_ihit *hits) {
  std::vector<float> w(12 * (size_t)ninst);
  std::vector<uint8_t> ok(ninst);
  for (uint32_t i = 0; i < ninst; ++i) ok[i] = (uint8_t)orc_instance_inverse(inst[i].m, &w[12 * (size_t)i]);
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t r = 0; r < (int64_t)nrays; ++r) {
    const float *ray = rays + 8 * r;
    uint32_t best = 0xFFFFFFFFu, binst = 0xFFFFFFFFu;
    float bt = 0.0f;
    float bro[8] = {0};
    for (uint32_t i = 0; i < ninst; ++i) {
      if (!ok[i] || !((inst[i].custom_mask >> 24) & ray_mask)) continue;
      const uint32_t m = (uint32_t)inst[i].blas;
      if (m >= meshes) continue;
      float ro[8];
      ray_to_object(&w[12 * (size_t)i], ray, ro);
      RayPre p;
      ray_pre(ro, p);
      const uint32_t b = tri_off ? tri_off[m] : 0u, e = tri_off ? tri_off[m + 1] : 0u;
      for (uint32_t k = b; k < e; ++k) {
        const float *va, *vb, *vc;
        tri_verts(pos, tri, k, va, vb, vc);
        float t;
        const uint32_t local = k - b;
        if (isect32(p, va, vb, vc, &t) &&
            (best == 0xFFFFFFFFu || t < bt || (t == bt && (i < binst || (i == binst && local < best))))) {
          best = local;
          binst = i;
          bt = t;
          std::memcpy(bro, ro, sizeof(ro));
        }
      }
    }
    hits[r].prim = best;
    hits[r].inst = binst;
    if (best != 0xFFFFFFFFu) {
      const float *va, *vb, *vc;
      tri_verts(pos, tri, tri_off[(uint32_t)inst[binst].blas] + best, va, vb, vc);
      hits[r].t = orc_refine_t32(bro, va, vb, vc);
    } else {
      hits[r].t = INFINITY;
    }
  }
}

// ============================================================================
// solid cells: bounds and point location
// ============================================================================
// Cell types and vertex counts (gprt/gprt_fallbacks.slang:289-318; the type
// codes match gprt/gprt_host.h:291-298).  A tetrahedral pair is evaluated as
// an eight-node (trilinear) cell and reports the tetrahedron hit kind.
static int solid_nodes(uint32_t type) {
  switch (type) {
    case 10: return 4;
    case 14: return 5;
    case 13: return 6;
    case 12: return 8;
    case 23: return 8;
    default: return 0;
  }
}
extern "C" uint32_t orc_solid_hit_kind(uint32_t type) {
  switch (type) {
    case 10: return 10;
    case 23: return 10;
    case 14: return 14;
    case 13: return 13;
    case 12: return 12;
    default: return 0;
  }
}
extern "C" int orc_solid_vertex_count(uint32_t type) { return solid_nodes(type); }

// Forward-mode dual number: the reference differentiates IsoToSupport with
// Slang's fwd_diff (gprt/gprt_fallbacks.slang:437-439); the derivative of
// c - a is -da and of a b is da b + a db, every operation rounded once.
struct Dl {
  float v, d;
};
static inline Dl dl_add(Dl a, Dl b) { return {a.v + b.v, a.d + b.d}; }
static inline Dl dl_sub(Dl a, Dl b) { return {a.v - b.v, a.d - b.d}; }
static inline Dl dl_rsub(float c, Dl a) { return {c - a.v, -a.d}; }
static inline Dl dl_mul(Dl a, Dl b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }

// IsoToSupport (gprt/gprt_fallbacks.slang:370-406): shape functions of the
// linear tetrahedron, pyramid, wedge and hexahedron at (r, s, t), in the
// reference's operation order; with a seed direction the derivatives too.
static void iso_support(int n, const Dl rst[3], Dl w[8]) {
  for (int i = 0; i < 8; ++i) w[i] = {0.0f, 0.0f};
  const Dl r = rst[0], s = rst[1], t = rst[2];
  const Dl mr = dl_rsub(1.0f, r), ms = dl_rsub(1.0f, s), mt = dl_rsub(1.0f, t);
  if (n == 4) {
    w[0] = dl_rsub(1.0f, dl_add(dl_add(r, s), t));
    w[1] = r;
    w[2] = s;
    w[3] = t;
  }
  if (n == 5) {
    w[0] = dl_mul(dl_mul(mr, ms), mt);
    w[1] = dl_mul(dl_mul(r, ms), mt);
    w[2] = dl_mul(dl_mul(r, s), mt);
    w[3] = dl_mul(dl_mul(mr, s), mt);
    w[4] = t;
  }
  if (n == 6) {
    const Dl rs = dl_sub(dl_rsub(1.0f, r), s);
    w[0] = dl_mul(rs, dl_rsub(1.0f, t));
    w[1] = dl_mul(r, dl_rsub(1.0f, t));
    w[2] = dl_mul(s, dl_rsub(1.0f, t));
    w[3] = dl_mul(rs, t);
    w[4] = dl_mul(r, t);
    w[5] = dl_mul(s, t);
  }
  if (n == 8) {
    w[0] = dl_mul(dl_mul(mr, ms), mt);
    w[1] = dl_mul(dl_mul(r, ms), mt);
    w[2] = dl_mul(dl_mul(r, s), mt);
    w[3] = dl_mul(dl_mul(mr, s), mt);
    w[4] = dl_mul(dl_mul(mr, ms), t);
    w[5] = dl_mul(dl_mul(r, ms), t);
    w[6] = dl_mul(dl_mul(r, s), t);
    w[7] = dl_mul(dl_mul(mr, s), t);
  }
}

// determinant of the 3x3 matrix with rows a, b, c: cofactor expansion along
// the first row.
static inline float det3(const float a[3], const float b[3], const float c[3]) {
  return a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) + a[2] * (b[0] * c[1] - b[1] * c[0]);
}

// intersectPointSolid (gprt/gprt_fallbacks.slang:409-464): Newton inversion of
// the cell's isoparametric map, at most five steps from the cell's centre
// (GetInitialRST, :320-325); the step is taken before the convergence test of
// the residual it used; containment per IsoIsContained (:327-340); the
// density is the last evaluated shape functions applied to the nodal values.
// qw: 8 float4 {x, y, z, density}, zero beyond the cell's vertex count.
extern "C" int orc_solid_intersect(const float *p, const float *qw, uint32_t n, float *rstw) {
  float rst[3] = {0.5f, 0.5f, 0.5f};
  if (n == 4) rst[0] = rst[1] = rst[2] = 0.25f;
  if (n == 5) rst[2] = 0.2f;
  rstw[0] = rst[0];
  rstw[1] = rst[1];
  rstw[2] = rst[2];
  rstw[3] = 0.0f;
  float w[8] = {0};
  bool converged = false;
  for (int it = 0; it < 5; ++it) {
    Dl x[3] = {{rst[0], 0.0f}, {rst[1], 0.0f}, {rst[2], 0.0f}}, dw[8];
    iso_support((int)n, x, dw);
    for (int i = 0; i < 8; ++i) w[i] = dw[i].v;
    float f[3] = {-p[0], -p[1], -p[2]};
    for (int i = 0; i < 8; ++i)
      for (int k = 0; k < 3; ++k) f[k] = f[k] + qw[4 * i + k] * w[i];
    float col[3][3];  // world-space derivatives along r, s, t
    for (int dir = 0; dir < 3; ++dir) {
      Dl y[3] = {{rst[0], dir == 0 ? 1.0f : 0.0f}, {rst[1], dir == 1 ? 1.0f : 0.0f}, {rst[2], dir == 2 ? 1.0f : 0.0f}};
      iso_support((int)n, y, dw);
      float c[3] = {0.0f, 0.0f, 0.0f};
      for (int i = 0; i < 8; ++i)
        for (int k = 0; k < 3; ++k) c[k] = c[k] + qw[4 * i + k] * dw[i].d;
      std::memcpy(col[dir], c, sizeof(c));
    }
    const float d = det3(col[0], col[1], col[2]);
    if (std::fabs(d) < 1e-20f) return 0;
    const float dinv = 1.0f / d;
    rst[0] = rst[0] - det3(f, col[1], col[2]) * dinv;
    rst[1] = rst[1] - det3(col[0], f, col[2]) * dinv;
    rst[2] = rst[2] - det3(col[0], col[1], f) * dinv;
    rstw[0] = rst[0];
    rstw[1] = rst[1];
    rstw[2] = rst[2];
    if (std::fabs(f[0]) < 1e-3f && std::fabs(f[1]) < 1e-3f && std::fabs(f[2]) < 1e-3f) {
      converged = true;
      break;
    }
  }
  if (!converged) return 0;
  bool in = rst[0] >= 0.0f && rst[1] >= 0.0f && rst[2] >= 0.0f && rst[0] <= 1.0f && rst[1] <= 1.0f && rst[2] <= 1.0f;
  if (n == 4) in = in && (rst[0] + rst[1] + rst[2]) <= 1.0f;
  if (n == 6) in = in && rst[0] + rst[1] <= 1.0f;
  if (!in) return 0;
  float dens = 0.0f;
  for (int i = 0; i < 8; ++i) dens = dens + qw[4 * i + 3] * w[i];
  rstw[3] = dens;
  return 1;
}

// A cell's nodes in index order (SolidIntersection's gather,
// gprt/gprt_fallbacks.slang:504-522), zero beyond its vertex count.
static int solid_gather(const float *verts, const uint32_t *idx, const uint8_t *types, uint32_t cell, float qw[32]) {
  const int n = solid_nodes(types[cell]);
  std::memset(qw, 0, 32 * sizeof(float));
  for (int i = 0; i < n; ++i) std::memcpy(qw + 4 * i, verts + 4 * (size_t)idx[8 * (size_t)cell + i], 16);
  return n;
}

// SolidBounds (gprt/gprt_fallbacks.slang:467-502): the min / max of the
// cell's vertices, and of their densities.  aabbs: two float4 per cell,
// {lo.xyz, hi.x}, {hi.yz, density min, density max}.  The reference's own
// density update assigns a scalar to its float2 (:488-489), which leaves the
// last vertex's density in both words; this follows the documented meaning
// (the minimum and maximum of the densities) instead.
extern "C" void orc_solid_bounds(const float *verts, const uint32_t *idx, const uint8_t *types, uint32_t ncells,
                                 float *aabbs) {
  for (uint32_t c = 0; c < ncells; ++c) {
    const int n = solid_nodes(types[c]);
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    float dlo = FLT_MAX, dhi = -FLT_MAX;
    for (int i = 0; i < n; ++i) {
      const float *v = verts + 4 * (size_t)idx[8 * (size_t)c + i];
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::fmin(lo[k], v[k]);
        hi[k] = std::fmax(hi[k], v[k]);
      }
      dlo = std::fmin(dlo, v[3]);
      dhi = std::fmax(dhi, v[3]);
    }
    float *o = aabbs + 8 * (size_t)c;
    o[0] = lo[0];
    o[1] = lo[1];
    o[2] = lo[2];
    o[3] = hi[0];
    o[4] = hi[1];
    o[5] = hi[2];
    o[6] = dlo;
    o[7] = dhi;
  }
}

// Point location by brute force: for every point the lowest-numbered cell
// that contains it (TracePoint, gprt/gprt_builtins.slang:80-90, traces a
// zero-length ray from the point; every accepted hit is at t = 0, so ties go
// to the lowest id as for rays), with its hit kind and (r, s, t, density).
extern "C" void orc_solid_locate_brute(const float *verts, const uint32_t *idx, const uint8_t *types, uint32_t ncells,
                                       const float *points, uint64_t npts, uint32_t *cell, uint32_t *kind,
                                       float *rstw) {
  std::vector<float> box(8 * (size_t)ncells);
  orc_solid_bounds(verts, idx, types, ncells, box.data());
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t q = 0; q < (int64_t)npts; ++q) {
    const float *p = points + 4 * q;
    cell[q] = 0xFFFFFFFFu;
    kind[q] = 0;
    float out[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (uint32_t c = 0; c < ncells; ++c) {
      const float *b = &box[8 * (size_t)c];
      if (!(b[0] <= p[0] && p[0] <= b[3] && b[1] <= p[1] && p[1] <= b[4] && b[2] <= p[2] && p[2] <= b[5])) continue;
      float qw[32], r[4];
      const int n = solid_gather(verts, idx, types, c, qw);
      if (n && orc_solid_intersect(p, qw, (uint32_t)n, r)) {
        cell[q] = c;
        kind[q] = orc_solid_hit_kind(types[c]);
        std::memcpy(out, r, sizeof(out));
        break;
      }
    }
    std::memcpy(rstw + 4 * q, out, sizeof(out));
  }
}
