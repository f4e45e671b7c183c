// gen.cu -- seeded synthetic scenes generated on the device (benchmark and
// test inputs; not part of the acceleration-structure path itself).
//
// Random numbers: SplitMix64 over (seed, stream, index) counters, so every
// value depends only on its index and the seed.  Normals by the Box-Muller
// transform.
//   soup     triangle i of mesh m: centroid uniform in mesh m's unit cube
//            (offset (m mod 16, m/16 mod 16, m/256) * spacing), vertices =
//            centroid + N(0, sigma^2) per axis; indices (3i, 3i+1, 3i+2)
//   mixture  K clusters, centre uniform in [0,1]^3, sigma uniform in
//            [0.005, 0.05]; triangle i belongs to cluster floor(i*K/n) (equal
//            weights, so consecutive triangles share a cluster); centroid =
//            centre + sigma * N(0,1)^3, vertices = centroid + N(0, edge^2)
//   rays     per mesh box (or the unit cube): origin uniform on the sphere
//            of radius 2 * (largest box extent) about the box centre,
//            direction normalised towards a uniform point in the box,
//            tmin = 0, tmax = +inf
#include "common.cuh"

namespace gprtcu {

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
__device__ __forceinline__ float u01(uint64_t seed, uint64_t stream, uint64_t i) {
  const uint64_t h = splitmix64(seed ^ splitmix64(stream * 0x632BE59BD9B4E019ull + i));
  return (float)(h >> 40) * (1.0f / 16777216.0f);  // [0, 1)
}
__device__ __forceinline__ void normal2(uint64_t seed, uint64_t stream, uint64_t i, float &a, float &b) {
  const float u = fmaxf(u01(seed, stream, 2 * i), 1e-7f), v = u01(seed, stream, 2 * i + 1);
  const float r = sqrtf(-2.0f * logf(u));
  float s, c;
  sincospif(2.0f * v, &s, &c);
  a = r * c;
  b = r * s;
}

__device__ __forceinline__ uint32_t mesh_of(const uint32_t *off, uint32_t meshes, uint64_t i) {
  if (!off) return 0;
  uint32_t lo = 0, hi = meshes;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (off[mid] <= i) lo = mid;
    else hi = mid;
  }
  return lo;
}

__global__ void k_gen_soup(uint64_t n, uint64_t seed, float sigma, const uint32_t *tri_off, uint32_t meshes,
                           float spacing, float *pos, uint32_t *tri) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t m = mesh_of(tri_off, meshes, i);
    const float ox = (float)(m % 16) * spacing, oy = (float)((m / 16) % 16) * spacing, oz = (float)(m / 256) * spacing;
    const float c[3] = {ox + u01(seed, 1, 3 * i), oy + u01(seed, 1, 3 * i + 1), oz + u01(seed, 1, 3 * i + 2)};
    float g[10];
    for (int k = 0; k < 5; ++k) normal2(seed, 2, 5 * i + k, g[2 * k], g[2 * k + 1]);
    for (int v = 0; v < 3; ++v)
      for (int k = 0; k < 3; ++k) pos[9 * i + 3 * v + k] = c[k] + sigma * g[3 * v + k];
    tri[3 * i] = (uint32_t)(3 * i);
    tri[3 * i + 1] = (uint32_t)(3 * i + 1);
    tri[3 * i + 2] = (uint32_t)(3 * i + 2);
  }
}

__global__ void k_gen_mixture(uint64_t n, uint32_t clusters, uint64_t seed, float edge, float *pos, uint32_t *tri) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = i * clusters / n;
    const float cx = u01(seed, 10, 3 * k), cy = u01(seed, 10, 3 * k + 1), cz = u01(seed, 10, 3 * k + 2);
    const float sg = 0.005f + 0.045f * u01(seed, 11, k);
    float g[12];
    for (int j = 0; j < 6; ++j) normal2(seed, 12, 6 * i + j, g[2 * j], g[2 * j + 1]);
    const float c[3] = {cx + sg * g[0], cy + sg * g[1], cz + sg * g[2]};
    for (int v = 0; v < 3; ++v)
      for (int a = 0; a < 3; ++a) pos[9 * i + 3 * v + a] = c[a] + edge * g[3 + 3 * v + a];
    tri[3 * i] = (uint32_t)(3 * i);
    tri[3 * i + 1] = (uint32_t)(3 * i + 1);
    tri[3 * i + 2] = (uint32_t)(3 * i + 2);
  }
}

__global__ void k_gen_rays(uint64_t nrays, uint64_t seed, const uint32_t *ray_off, uint32_t meshes,
                           const float *boxes, float4 *rays) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < nrays;
       r += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t m = mesh_of(ray_off, meshes, r);
    float lo[3] = {0.f, 0.f, 0.f}, hi[3] = {1.f, 1.f, 1.f};
    if (boxes)
      for (int k = 0; k < 3; ++k) {
        lo[k] = boxes[6 * (size_t)m + k];
        hi[k] = boxes[6 * (size_t)m + 3 + k];
      }
    const float ext = fmaxf(hi[0] - lo[0], fmaxf(hi[1] - lo[1], hi[2] - lo[2]));
    float ux, uy, uz, w;
    normal2(seed, 20, 2 * r, ux, uy);
    normal2(seed, 20, 2 * r + 1, uz, w);
    const float inv = rsqrtf(fmaxf(ux * ux + uy * uy + uz * uz, 1e-20f));
    const float rad = 2.0f * ext;
    const float o[3] = {0.5f * (lo[0] + hi[0]) + rad * ux * inv, 0.5f * (lo[1] + hi[1]) + rad * uy * inv,
                        0.5f * (lo[2] + hi[2]) + rad * uz * inv};
    const float t[3] = {lo[0] + (hi[0] - lo[0]) * u01(seed, 21, 3 * r), lo[1] + (hi[1] - lo[1]) * u01(seed, 21, 3 * r + 1),
                        lo[2] + (hi[2] - lo[2]) * u01(seed, 21, 3 * r + 2)};
    float d[3] = {t[0] - o[0], t[1] - o[1], t[2] - o[2]};
    const float dn = rsqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    rays[2 * r] = make_float4(o[0], o[1], o[2], 0.0f);
    rays[2 * r + 1] = make_float4(d[0] * dn, d[1] * dn, d[2] * dn, __int_as_float(0x7f800000));
  }
}

}  // namespace gprtcu

using namespace gprtcu;

static int gen_grid(uint64_t n) {
  uint64_t g = (n + 255) / 256, cap = (uint64_t)gprtcu_num_sms() * 16;
  return (int)(g < cap ? (g ? g : 1) : cap);
}

extern "C" GPRTCU_API gprtcuStatus gprtcuGenSoup(uint64_t n, uint64_t seed, float sigma, const uint32_t *triOffsets,
                                                 uint32_t numMeshes, float spacing, float *positions,
                                                 uint32_t *triangles, gprtcuStream stream) {
  if (!positions || !triangles || numMeshes == 0 || (numMeshes > 1 && !triOffsets)) return GPRTCU_ERR_INVALID_ARG;
  if (n == 0) return GPRTCU_OK;
  k_gen_soup<<<gen_grid(n), 256, 0, (cudaStream_t)stream>>>(n, seed, sigma, numMeshes > 1 ? triOffsets : nullptr,
                                                            numMeshes, spacing, positions, triangles);
  GPRTCU_TRY(cudaGetLastError());
  return GPRTCU_OK;
}

extern "C" GPRTCU_API gprtcuStatus gprtcuGenMixture(uint64_t n, uint32_t clusters, uint64_t seed, float edgeSigma,
                                                    float *positions, uint32_t *triangles, gprtcuStream stream) {
  if (!positions || !triangles || clusters == 0) return GPRTCU_ERR_INVALID_ARG;
  if (n == 0) return GPRTCU_OK;
  k_gen_mixture<<<gen_grid(n), 256, 0, (cudaStream_t)stream>>>(n, clusters, seed, edgeSigma, positions, triangles);
  GPRTCU_TRY(cudaGetLastError());
  return GPRTCU_OK;
}

extern "C" GPRTCU_API gprtcuStatus gprtcuGenRays(uint64_t numRays, uint64_t seed, const uint32_t *rayOffsets,
                                                 uint32_t numMeshes, const float *meshBoxes, float *rays,
                                                 gprtcuStream stream) {
  if (!rays || numMeshes == 0 || (numMeshes > 1 && (!rayOffsets || !meshBoxes))) return GPRTCU_ERR_INVALID_ARG;
  if ((uintptr_t)rays & 15) return GPRTCU_ERR_INVALID_ARG;
  if (numRays == 0) return GPRTCU_OK;
  k_gen_rays<<<gen_grid(numRays), 256, 0, (cudaStream_t)stream>>>(numRays, seed, numMeshes > 1 ? rayOffsets : nullptr,
                                                                  numMeshes, meshBoxes, (float4 *)rays);
  GPRTCU_TRY(cudaGetLastError());
  return GPRTCU_OK;
}
