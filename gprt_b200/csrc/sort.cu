// sort.cu -- host driver of the radix sort (kernels in sort_kernels.cuh):
// scratch layout, the per-type active shape, the C entry points and the
// autotuner that times every shape of the tuning grid on this device.
#include <algorithm>
#include <atomic>
#include <vector>

#include "sort_kernels.cuh"

using namespace gprtcu;

uint32_t gprtcu_spin_budget(void);

static int64_t g_sort_skip_tile = -1;
extern "C" GPRTCU_API void gprtcuDebugSortSkipTile(int64_t tile) { g_sort_skip_tile = tile; }
static int g_sort_ranking = 0;
extern "C" GPRTCU_API void gprtcuDebugSortRanking(int mode) { g_sort_ranking = mode; }
int gprtcu::gprtcu_sort_ranking() { return g_sort_ranking; }
// Half a resident wave ahead by default (2^28 Zipf u32 pairs 5.67 -> 5.50 ms,
// uniform 6.12 -> 5.98 ms, 2^26 segmented u64/u32 pairs 3.03 -> 2.91 ms; two
// waves or more ahead measured slower than none).
static std::atomic<int> g_sort_prefetch{2};
extern "C" GPRTCU_API void gprtcuDebugSortPrefetch(int quarterWaves) {
  g_sort_prefetch.store(quarterWaves < 0 ? 0 : (quarterWaves > 64 ? 64 : quarterWaves), std::memory_order_relaxed);
}
int gprtcu::gprtcu_sort_prefetch() { return g_sort_prefetch.load(std::memory_order_relaxed); }

namespace {

// Type pairs: 0 u32, 1 u32/u32, 2 u64, 3 u64/u32, 4 u64/u64, 5 u32/u64.
constexpr int kTypeSlots = 6;
// The reference counts keys in a uint32 (gprt/gprt.cpp:8837).
constexpr uint64_t kSortMaxN = 0xFFFFFFFFull;

int type_slot(int kw, int vw) {
  if (kw == 4 && vw == 0) return 0;
  if (kw == 4 && vw == 4) return 1;
  if (kw == 8 && vw == 0) return 2;
  if (kw == 8 && vw == 4) return 3;
  if (kw == 8 && vw == 8) return 4;
  if (kw == 4 && vw == 8) return 5;
  return -1;
}

const std::array<SortRunFn, kSortGridSize> &table_for(int slot) {
  switch (slot) {
    case 0: return kSortTableK32;
    case 1: return kSortTableK32V32;
    case 2: return kSortTableK64;
    case 3: return kSortTableK64V32;
    case 5: return kSortTableK32V64;
    default: return kSortTableK64V64;
  }
}

int grid_index(int rb, int tile, int warps) {
  for (int i = 0; i < kSortGridSize; ++i)
    if (kSortGrid[i].rb == rb && kSortGrid[i].tile == tile && kSortGrid[i].warps == warps) return i;
  return -1;
}

// Shapes used until the tuner or the caller picks others, from sweeps of the
// grid on B200 (uniform and Zipf(1.1) keys, 2^18 .. 2^28 elements): 8-bit
// digits everywhere; for 32-bit keys with 32-bit payloads 6144-key tiles of 8
// warps (73 KB of shared memory and 80 registers: three CTAs per SM; 2^28
// Zipf pairs 5.76 ms against 5.95 for 8192-key tiles, which fit two); 32-bit
// keys alone or with 64-bit payloads 8192-key tiles of 8 warps (2^28 Zipf
// keys 4.66 ms against 4.81 at 6144); 64-bit keys with 32-bit payloads
// 6144-key tiles of 8 warps (2^26 segmented (mesh, code) pairs of 44 bits:
// 3.09 ms against 3.14 at 4096 and 3.80 at 8192), other 64-bit keys
// 4096-key tiles of 8 warps; 2048-key tiles of 8 warps below 2^22 keys, where
// there are too few large tiles to fill the SMs.
int default_index(int slot, uint64_t n) {
  if (n < (1ull << 22)) return grid_index(8, 2048, 8);
  if (slot == 1 || slot == 3) return grid_index(8, 6144, 8);
  if (slot == 0 || slot == 5) return grid_index(8, 8192, 8);
  return grid_index(8, 4096, 8);
}

std::atomic<int> g_active[kTypeSlots] = {{-1}, {-1}, {-1}, {-1}, {-1}, {-1}};

int active_index(int slot, uint64_t n) {
  const int i = g_active[slot].load(std::memory_order_relaxed);
  return i >= 0 ? i : default_index(slot, n);
}

struct SortLayout {
  size_t keys_alt, vals_alt, hist, trivial, status, total;
  uint64_t tiles;
  int passes;
};

SortLayout sort_layout(uint64_t n, int kw, int vw, int begin_bit, int end_bit, const SortShape &s) {
  SortLayout L;
  L.tiles = (n + s.tile - 1) / s.tile;
  L.passes = (end_bit - begin_bit + s.rb - 1) / s.rb;
  size_t off = sizeof(SortHeader);
  L.keys_alt = off;
  off += gprtcu_align256((size_t)n * kw);
  L.vals_alt = off;
  off += gprtcu_align256((size_t)n * vw);
  L.hist = off;
  off += gprtcu_align256((size_t)SORT_MAX_PASSES * 256 * 4);
  L.trivial = off;
  off += 256;
  L.status = off;
  // look-back words: 32-bit, or 64-bit once n needs more than 30 value bits
  off += gprtcu_align256((size_t)2 * L.tiles * (1u << s.rb) * (n > (uint64_t)LB_VALUE ? 8 : 4));
  L.total = off;
  return L;
}

// Shapes that can sort n keys: all of them below 2^30; beyond, the 8-bit
// shapes with tiles of 4096 keys or more (their wide look-back words, and a
// bounded number of them).
bool shape_usable(const SortShape &s, uint64_t n) { return n <= (uint64_t)LB_VALUE || (s.rb == 8 && s.tile >= 4096); }

// Scratch that fits every usable shape of the grid, so a scratch sized once
// stays valid whatever shape the tuner installs later.
size_t scratch_any_shape(uint64_t n, int kw, int vw) {
  size_t m = 0;
  for (int i = 0; i < kSortGridSize; ++i)
    if (shape_usable(kSortGrid[i], n)) m = std::max(m, sort_layout(n, kw, vw, 0, 8 * kw, kSortGrid[i]).total);
  return m;
}

gprtcuStatus sort_dispatch(int slot, int index, void *keys, void *vals, uint64_t n, int kw, int vw, int begin_bit,
                           int end_bit, void *scratch, size_t scratch_bytes, cudaStream_t stream) {
  if (!keys && n) return GPRTCU_ERR_INVALID_ARG;
  if (vw && !vals && n) return GPRTCU_ERR_INVALID_ARG;
  if (begin_bit < 0 || end_bit > 8 * kw || begin_bit >= end_bit) return GPRTCU_ERR_INVALID_ARG;
  if (n > kSortMaxN) return GPRTCU_ERR_TOO_LARGE;
  if (!scratch || ((uintptr_t)scratch & 255)) return GPRTCU_ERR_INVALID_ARG;
  const SortShape &shape = kSortGrid[index];
  if (!shape_usable(shape, n)) return GPRTCU_ERR_TOO_LARGE;
  SortLayout L = sort_layout(n, kw, vw, begin_bit, end_bit, shape);
  if (scratch_bytes < L.total) return GPRTCU_ERR_SCRATCH_TOO_SMALL;
  char *s = (char *)scratch;
  // the header (its status word first) is valid after every call, even one
  // with nothing to sort: callers such as the LBVH build read it
  GPRTCU_TRY(cudaMemsetAsync(s, 0, sizeof(SortHeader), stream));
  if (n <= 1) return GPRTCU_OK;
  SortArgs a;
  a.keys = keys;
  a.vals = vals;
  a.keys_alt = s + L.keys_alt;
  a.vals_alt = s + L.vals_alt;
  a.n = n;
  a.tiles = L.tiles;
  a.begin_bit = begin_bit;
  a.end_bit = end_bit;
  a.passes = L.passes;
  a.hist = (uint32_t *)(s + L.hist);
  a.trivial = (uint32_t *)(s + L.trivial);
  a.hdr = (SortHeader *)s;
  a.status = (uint32_t *)(s + L.status);
  a.budget = gprtcu_spin_budget();
  a.skip_tile = g_sort_skip_tile;
  a.pf_tiles = 0;
  a.use_bulk = ((((uintptr_t)keys) | ((uintptr_t)a.keys_alt)) & 15) == 0;
  a.sms = gprtcu_num_sms();
  // Zero: histograms, trivial flags, both look-back regions.
  GPRTCU_TRY(cudaMemsetAsync(s + L.hist, 0, L.total - L.hist, stream));
  return table_for(slot)[index](a, stream);
}

gprtcuStatus sort_entry(void *keys, void *vals, uint64_t n, int kw, int vw, int begin_bit, int end_bit,
                        void *scratch, size_t scratch_bytes, gprtcuStream stream) {
  const int slot = type_slot(kw, vw);
  return sort_dispatch(slot, active_index(slot, n), keys, vals, n, kw, vw, begin_bit, end_bit, scratch, scratch_bytes,
                       (cudaStream_t)stream);
}

// Tuning input: uniform keys over [0, 2^end_bit) from a counter-based hash.
__global__ void k_tune_keys(void *keys, int kw, uint64_t n, int end_bit, uint64_t seed) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    if (end_bit < 64) z &= (1ull << end_bit) - 1ull;
    if (kw == 4) static_cast<uint32_t *>(keys)[i] = (uint32_t)z;
    else static_cast<uint64_t *>(keys)[i] = z;
  }
}

struct DeviceBuffers {
  std::vector<void *> ptrs;
  ~DeviceBuffers() {
    for (void *p : ptrs) cudaFree(p);
  }
  void *get(size_t bytes) {
    void *p = nullptr;
    if (cudaMalloc(&p, bytes ? bytes : 256) != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return p;
  }
};

}  // namespace

extern "C" GPRTCU_API size_t gprtcuSortScratchSize(uint64_t n, int keyBytes, int valueBytes) {
  if (type_slot(keyBytes, valueBytes) < 0) return 0;
  return scratch_any_shape(n, keyBytes, valueBytes);
}

extern "C" GPRTCU_API gprtcuStatus gprtcuSortKeysU32(uint32_t *keys, uint64_t n, int beginBit, int endBit,
                                                     void *scratch, size_t scratchBytes, gprtcuStream stream) {
  return sort_entry(keys, nullptr, n, 4, 0, beginBit, endBit, scratch, scratchBytes, stream);
}
extern "C" GPRTCU_API gprtcuStatus gprtcuSortPairsU32(uint32_t *keys, uint32_t *values, uint64_t n, int beginBit,
                                                      int endBit, void *scratch, size_t scratchBytes,
                                                      gprtcuStream stream) {
  return sort_entry(keys, values, n, 4, 4, beginBit, endBit, scratch, scratchBytes, stream);
}
extern "C" GPRTCU_API gprtcuStatus gprtcuSortKeysU64(uint64_t *keys, uint64_t n, int beginBit, int endBit,
                                                     void *scratch, size_t scratchBytes, gprtcuStream stream) {
  return sort_entry(keys, nullptr, n, 8, 0, beginBit, endBit, scratch, scratchBytes, stream);
}
extern "C" GPRTCU_API gprtcuStatus gprtcuSortPairsU64(uint64_t *keys, uint32_t *values, uint64_t n, int beginBit,
                                                      int endBit, void *scratch, size_t scratchBytes,
                                                      gprtcuStream stream) {
  return sort_entry(keys, values, n, 8, 4, beginBit, endBit, scratch, scratchBytes, stream);
}
extern "C" GPRTCU_API gprtcuStatus gprtcuSortPairsU32U64(uint32_t *keys, uint64_t *values, uint64_t n, int beginBit,
                                                         int endBit, void *scratch, size_t scratchBytes,
                                                         gprtcuStream stream) {
  return sort_entry(keys, values, n, 4, 8, beginBit, endBit, scratch, scratchBytes, stream);
}
extern "C" GPRTCU_API gprtcuStatus gprtcuSortPairsU64U64(uint64_t *keys, uint64_t *values, uint64_t n, int beginBit,
                                                         int endBit, void *scratch, size_t scratchBytes,
                                                         gprtcuStream stream) {
  return sort_entry(keys, values, n, 8, 8, beginBit, endBit, scratch, scratchBytes, stream);
}

extern "C" GPRTCU_API int gprtcuSortConfigCount(void) { return kSortGridSize; }

extern "C" GPRTCU_API gprtcuStatus gprtcuSortConfigAt(int index, gprtcuSortConfig *cfg) {
  if (index < 0 || index >= kSortGridSize || !cfg) return GPRTCU_ERR_INVALID_ARG;
  cfg->digitBits = kSortGrid[index].rb;
  cfg->tile = kSortGrid[index].tile;
  cfg->warps = kSortGrid[index].warps;
  return GPRTCU_OK;
}

extern "C" GPRTCU_API gprtcuStatus gprtcuSortGetConfig(int keyBytes, int valueBytes, gprtcuSortConfig *cfg) {
  const int slot = type_slot(keyBytes, valueBytes);
  if (slot < 0 || !cfg) return GPRTCU_ERR_INVALID_ARG;
  return gprtcuSortConfigAt(active_index(slot, 1ull << 28), cfg);
}

extern "C" GPRTCU_API gprtcuStatus gprtcuSortSetConfig(int keyBytes, int valueBytes, const gprtcuSortConfig *cfg) {
  const int slot = type_slot(keyBytes, valueBytes);
  if (slot < 0) return GPRTCU_ERR_INVALID_ARG;
  if (!cfg) {
    g_active[slot].store(-1);
    return GPRTCU_OK;
  }
  const int i = grid_index(cfg->digitBits, cfg->tile, cfg->warps);
  if (i < 0) return GPRTCU_ERR_INVALID_ARG;
  g_active[slot].store(i);
  return GPRTCU_OK;
}

extern "C" GPRTCU_API gprtcuStatus gprtcuSortWithConfig(void *keys, void *values, uint64_t n, int keyBytes,
                                                        int valueBytes, int beginBit, int endBit,
                                                        const gprtcuSortConfig *cfg, void *scratch,
                                                        size_t scratchBytes, gprtcuStream stream) {
  const int slot = type_slot(keyBytes, valueBytes);
  if (slot < 0 || !cfg) return GPRTCU_ERR_INVALID_ARG;
  const int i = grid_index(cfg->digitBits, cfg->tile, cfg->warps);
  if (i < 0) return GPRTCU_ERR_INVALID_ARG;
  return sort_dispatch(slot, i, keys, values, n, keyBytes, valueBytes, beginBit, endBit, scratch, scratchBytes,
                       (cudaStream_t)stream);
}

extern "C" GPRTCU_API gprtcuStatus gprtcuSortAutotune(int keyBytes, int valueBytes, uint64_t n, int endBit,
                                                      const void *sampleKeys, int repeats, float *msPerConfig,
                                                      gprtcuSortConfig *best, gprtcuStream stream) {
  const int slot = type_slot(keyBytes, valueBytes);
  if (slot < 0 || n < 2 || n > (uint64_t)LB_VALUE || endBit < 1 || endBit > 8 * keyBytes) return GPRTCU_ERR_INVALID_ARG;
  if (repeats < 1) repeats = 1;
  cudaStream_t s = (cudaStream_t)stream;
  DeviceBuffers buf;
  void *src = buf.get(n * keyBytes), *keys = buf.get(n * keyBytes);
  void *vals = valueBytes ? buf.get(n * valueBytes) : nullptr;
  const size_t sbytes = scratch_any_shape(n, keyBytes, valueBytes);
  void *scratch = buf.get(sbytes);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (!src || !keys || (valueBytes && !vals) || !scratch || cudaEventCreate(&e0) != cudaSuccess ||
      cudaEventCreate(&e1) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    return GPRTCU_ERR_CUDA;
  }
  gprtcuStatus result = GPRTCU_OK;
  if (sampleKeys) {
    if (cudaMemcpyAsync(src, sampleKeys, n * keyBytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
      result = GPRTCU_ERR_CUDA;
  } else {
    k_tune_keys<<<gprtcu_num_sms() * 4, 256, 0, s>>>(src, keyBytes, n, endBit, 0x5EEDull);
    if (cudaGetLastError() != cudaSuccess) result = GPRTCU_ERR_CUDA;
  }
  if (vals && cudaMemsetAsync(vals, 0, n * valueBytes, s) != cudaSuccess) result = GPRTCU_ERR_CUDA;
  int best_i = -1;
  float best_ms = 0.f;
  for (int i = 0; i < kSortGridSize && result == GPRTCU_OK; ++i) {
    std::vector<float> ts;
    bool ok = true;
    for (int r = 0; r <= repeats && ok; ++r) {  // first run untimed
      ok = cudaMemcpyAsync(keys, src, n * keyBytes, cudaMemcpyDeviceToDevice, s) == cudaSuccess &&
           cudaEventRecord(e0, s) == cudaSuccess &&
           sort_dispatch(slot, i, keys, vals, n, keyBytes, valueBytes, 0, endBit, scratch, sbytes, s) == GPRTCU_OK &&
           cudaEventRecord(e1, s) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess;
      int st = 0;
      ok = ok && cudaMemcpy(&st, scratch, 4, cudaMemcpyDeviceToHost) == cudaSuccess && st == 0;
      float ms = 0.f;
      if (ok && r > 0 && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) ts.push_back(ms);
    }
    if (!ok) {
      if (cudaPeekAtLastError() != cudaSuccess) result = GPRTCU_ERR_CUDA;
      if (msPerConfig) msPerConfig[i] = -1.f;
      continue;
    }
    std::sort(ts.begin(), ts.end());
    const float med = ts[ts.size() / 2];
    if (msPerConfig) msPerConfig[i] = med;
    if (best_i < 0 || med < best_ms) {
      best_i = i;
      best_ms = med;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (result != GPRTCU_OK) return result;
  if (best_i < 0) return GPRTCU_ERR_CUDA;
  g_active[slot].store(best_i);
  if (best) gprtcuSortConfigAt(best_i, best);
  return GPRTCU_OK;
}
