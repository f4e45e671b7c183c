// sort.cu -- stable LSD radix sort (keys, or key/payload pairs) for sm_100a.
//
// Replaces gprtBufferSort / gprtBufferSortPayload (gprt/gprt_host.h:2384,2416;
// host driver gprt/gprt.cpp:8821-9073; kernels gprt/gprt_sort.slang:109-637).
// Same contract: stable ascending sort, result in place in the caller's
// buffers.  The reference runs FidelityFX's reduce-then-scan with 4-bit
// digits: five dispatches per digit, 16 passes over 64-bit words.  This is a
// onesweep design instead (Adinets & Merrill 2022):
//   1. one histogram kernel reads every key once and builds the digit
//      histograms of all passes; its last CTA scans them into global digit
//      offsets and marks passes whose digit is constant (skipped);
//   2. one digit-binning kernel per pass: a tile of keys (and payloads)
//      arrives in shared memory by bulk async copy (TMA), warps rank their
//      keys with __match_any_sync against per-warp shared histograms, each
//      digit's tile count is published to a per-(tile, digit) status word
//      and a decoupled look-back over earlier tiles gives the digit's global
//      position; keys and payloads are then reordered in shared memory so the
//      scatter leaves the tile as coalesced per-digit runs.
// Traffic per pass: read + write of keys and payloads (16 B per u32/u32
// pair); plus 4 B per key for the histogram.
#include "common.cuh"

namespace gprtcu {

constexpr uint32_t LB_AGG = 1u << 30;
constexpr uint32_t LB_INC = 2u << 30;
constexpr uint32_t LB_POISON = 3u << 30;
constexpr uint32_t LB_VALUE = (1u << 30) - 1;
constexpr int SORT_MAX_PASSES = 16;

// Sort-specific part of the scratch header: per-pass "trivial" flags follow
// the ScratchHeader fields (ticket[1+p] is pass p's tile ticket, ticket[0] the
// histogram's done-counter, sel[p] which buffer holds pass p's input).
struct SortHeader {
  ScratchHeader h;
};

template <typename K> __device__ __forceinline__ uint32_t digit_of(K key, int shift, uint32_t mask) {
  return (uint32_t)(key >> shift) & mask;
}

// Lanes of the warp holding the same BITS-bit digit as this lane, among the
// lanes with valid == true (warp-level multisplit by ballots, one per digit
// bit).  Replaces __match_any_sync, whose pipe throughput made the ranking
// issue-bound on sm_100a.
template <int BITS> __device__ __forceinline__ unsigned warp_peers(uint32_t d, bool valid) {
  unsigned m = __ballot_sync(FULL_MASK, valid);
#pragma unroll
  for (int b = 0; b < BITS; ++b) {
    const bool bit = (d >> b) & 1u;
    const unsigned bb = __ballot_sync(FULL_MASK, bit);
    m &= bit ? bb : ~bb;
  }
  return valid ? m : 0u;
}

// ---------------------------------------------------------------------------
// 1. histogram of every pass's digit, one read of the keys
// ---------------------------------------------------------------------------
template <typename K, int RB>
__global__ void __launch_bounds__(512) k_sort_hist(const K *__restrict__ keys, uint64_t n, int begin_bit, int end_bit,
                                                   int passes, uint32_t *ghist, uint32_t *trivial,
                                                   ScratchHeader *hdr) {
  constexpr int RADIX = 1 << RB;
  __shared__ uint32_t sh[SORT_MAX_PASSES * RADIX > 4096 ? 4096 : SORT_MAX_PASSES * RADIX];
  __shared__ bool s_last;
  const int tid = threadIdx.x, lane = tid & 31;
  for (int i = tid; i < passes * RADIX; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  // Grid-stride over all keys; warp-aggregated shared atomics (skewed inputs
  // put a whole warp on one bin).
  const uint64_t total = (n + 31) & ~31ull;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + tid; i < total; i += stride) {
    const bool valid = i < n;
    K key = valid ? keys[i] : (K)0;
    for (int p = 0; p < passes; ++p) {
      const int shift = begin_bit + p * RB;
      const int bits = min(RB, end_bit - shift);
      const uint32_t d = valid ? digit_of(key, shift, (1u << bits) - 1u) : 0u;
      const unsigned peers = warp_peers<RB>(d, valid);
      if (valid && lane == 31 - __clz(peers)) atomicAdd(&sh[p * RADIX + d], (uint32_t)__popc(peers));
    }
  }
  __syncthreads();
  for (int i = tid; i < passes * RADIX; i += blockDim.x)
    if (sh[i]) atomicAdd(&ghist[i], sh[i]);
  __threadfence();
  __syncthreads();
  if (tid == 0) s_last = atomicAdd(&hdr->ticket[0], 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // Last CTA: exclusive scan of each pass's histogram in place, trivial-pass
  // detection, and the ping-pong selector of every pass.
  __shared__ uint32_t s_triv[SORT_MAX_PASSES];
  for (int p = tid >> 5; p < passes; p += blockDim.x >> 5) {
    uint32_t carry = 0, triv = 0;
    for (int base = 0; base < RADIX; base += 32) {
      uint32_t c = base + lane < RADIX ? ld_relaxed_u32(&ghist[p * RADIX + base + lane]) : 0u;
      if ((uint64_t)c == n) triv = 1;
      uint32_t inc = warp_incl_scan(c, lane);
      if (base + lane < RADIX) ghist[p * RADIX + base + lane] = carry + inc - c;
      carry += __shfl_sync(FULL_MASK, inc, 31);
    }
    triv = __any_sync(FULL_MASK, triv);
    if (lane == 0) s_triv[p] = triv;
  }
  __syncthreads();
  if (tid == 0) {
    uint32_t sel = 0;
    for (int p = 0; p < passes; ++p) {
      hdr->sel[p] = sel;
      trivial[p] = s_triv[p];
      if (!s_triv[p]) sel ^= 1u;
    }
    hdr->sel[passes] = sel;
  }
}

// ---------------------------------------------------------------------------
// 2. one digit-binning pass
// ---------------------------------------------------------------------------
template <typename K, typename V, int RB, int THREADS, int ITEMS> struct PassCfg {
  static constexpr int RADIX = 1 << RB;
  static constexpr int WARPS = THREADS / 32;
  static constexpr int TILE = THREADS * ITEMS;
  static constexpr int WARP_KEYS = 32 * ITEMS;
  static constexpr bool HAS_V = sizeof(V) > 1;
  static constexpr size_t KEY_BYTES = (size_t)TILE * sizeof(K);
  static constexpr size_t VAL_BYTES = HAS_V ? (size_t)TILE * sizeof(V) : 0;
  static constexpr size_t HIST_BYTES = (size_t)WARPS * RADIX * 4;
  static constexpr size_t SMEM = KEY_BYTES + VAL_BYTES + HIST_BYTES + RADIX * 8 /*goff*/ + RADIX * 4 /*tile start*/ +
                                 64 /*barriers*/;
};

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Exclusive scan of v over threads [0, RADIX) (RADIX <= 1024, multiple of 32
// or smaller than 32); every thread of the block must call it.
template <int RADIX, int THREADS>
__device__ __forceinline__ uint32_t block_excl_scan_digits(uint32_t v, uint32_t *s_tmp) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int DW = RADIX >= 32 ? RADIX / 32 : 1;
  uint32_t inc = warp_incl_scan(tid < RADIX ? v : 0u, lane);
  if (tid < RADIX && lane == 31 && DW > 1) s_tmp[warp] = inc;
  __syncthreads();
  uint32_t add = 0;
  if (DW > 1 && tid < RADIX)
    for (int w = 0; w < warp; ++w) add += s_tmp[w];
  __syncthreads();
  return add + inc - v;
}

template <typename K, typename V, int RB, int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) k_sort_pass(K *keys, K *keys_alt, V *vals, V *vals_alt, uint64_t n,
                                                       int shift, int bits, int pass, const uint32_t *goffs,
                                                       const uint32_t *trivial, ScratchHeader *hdr, uint32_t *status,
                                                       uint32_t budget, int use_bulk) {
  using C = PassCfg<K, V, RB, THREADS, ITEMS>;
  constexpr int RADIX = C::RADIX, WARPS = C::WARPS, TILE = C::TILE, WK = C::WARP_KEYS;
  if (ld_relaxed_u32(&trivial[pass])) return;  // every key has the same digit: nothing moves

  extern __shared__ __align__(128) unsigned char smem[];
  K *s_keys = reinterpret_cast<K *>(smem);
  V *s_vals = reinterpret_cast<V *>(smem + C::KEY_BYTES);
  uint32_t *s_hist = reinterpret_cast<uint32_t *>(smem + C::KEY_BYTES + C::VAL_BYTES);  // [WARPS][RADIX]
  uint64_t *s_goff = reinterpret_cast<uint64_t *>(smem + C::KEY_BYTES + C::VAL_BYTES + C::HIST_BYTES);
  uint32_t *s_tstart = reinterpret_cast<uint32_t *>(s_goff + RADIX);
  uint64_t *bars = reinterpret_cast<uint64_t *>(s_tstart + RADIX);
  __shared__ uint32_t s_tile, s_abort;
  __shared__ uint32_t s_tmp[32];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t sel = hdr->sel[pass];
  const K *src_k = sel ? keys_alt : keys;
  K *dst_k = sel ? keys : keys_alt;
  const V *src_v = sel ? vals_alt : vals;
  V *dst_v = sel ? vals : vals_alt;
  const uint32_t mask = (1u << bits) - 1u;

  if (tid == 0) {
    s_tile = atomicAdd(&hdr->ticket[1 + pass], 1u);
    s_abort = 0;
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint64_t tile_start = (uint64_t)tile * TILE;
  const uint32_t tile_n = (uint32_t)min((uint64_t)TILE, n - tile_start);
  const bool bulk = use_bulk && tile_n == TILE;
  if (tid == 0 && bulk) {
    mbar_arrive_expect_tx(&bars[0], (uint32_t)C::KEY_BYTES);
    bulk_g2s(s_keys, src_k + tile_start, (uint32_t)C::KEY_BYTES, &bars[0]);
    if (C::HAS_V) {
      mbar_arrive_expect_tx(&bars[1], (uint32_t)C::VAL_BYTES);
      bulk_g2s(s_vals, src_v + tile_start, (uint32_t)C::VAL_BYTES, &bars[1]);
    }
  }
  for (int i = tid; i < WARPS * RADIX; i += THREADS) s_hist[i] = 0;
  if (!bulk) {
    for (int i = tid; i < TILE; i += THREADS)
      if ((uint32_t)i < tile_n) s_keys[i] = src_k[tile_start + i];
  } else if (!mbar_wait(&bars[0], 0, MBAR_WAIT_BUDGET)) {
    s_abort = 1;
  }
  __syncthreads();
  if (s_abort) {
    if (tid == 0) record_error(hdr, GPRTCU_ERR_TIMEOUT);
    return;
  }

  // ---- rank: warp w owns tile positions [w*WK, (w+1)*WK), item-major.
  K k[ITEMS];
  uint32_t rank[ITEMS];
  uint32_t *wh = s_hist + warp * RADIX;
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    const uint32_t pos = warp * WK + i * 32 + lane;
    const bool valid = pos < tile_n;
    k[i] = valid ? s_keys[pos] : (K)0;
    const uint32_t d = valid ? digit_of(k[i], shift, mask) : 0u;
    const unsigned peers = warp_peers<RB>(d, valid);
    uint32_t base = 0;
    if (valid) base = wh[d];
    __syncwarp();
    if (valid && lane == 31 - __clz(peers)) wh[d] = base + __popc(peers);
    __syncwarp();
    rank[i] = base + __popc(peers & lt);
  }
  __syncthreads();

  // ---- per digit: warp-exclusive offsets, tile count, publish, look-back.
  uint32_t tcount = 0;
  if (tid < RADIX) {
    uint32_t run = 0;
#pragma unroll 4
    for (int w = 0; w < WARPS; ++w) {
      uint32_t c = s_hist[w * RADIX + tid];
      s_hist[w * RADIX + tid] = run;
      run += c;
    }
    tcount = run;
    uint32_t *st = status + (uint64_t)tile * RADIX + tid;
    st_relaxed_u32(st, (tile == 0 ? LB_INC : LB_AGG) | tcount);
  }
  const uint32_t tstart = block_excl_scan_digits<RADIX, THREADS>(tcount, s_tmp);
  if (tid < RADIX) {
    uint32_t excl = 0;
    bool ok = true;
    if (tile > 0) {
      // Eight predecessors per probe (loads issued together), nearest first:
      // the inclusive prefix of a digit can only advance one probe window per
      // L2 round trip.
      int64_t j = (int64_t)tile - 1;
      uint32_t spins = 0;
      bool done = false;
      while (!done && ok) {
        uint32_t s[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) s[c] = j - c >= 0 ? ld_relaxed_u32(status + (uint64_t)(j - c) * RADIX + tid) : LB_INC;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          if (done || !ok) break;
          uint32_t x = s[c];
          while ((x & ~LB_VALUE) == 0) {
            if (++spins > budget) {
              ok = false;
              break;
            }
            x = ld_relaxed_u32(status + (uint64_t)(j - c) * RADIX + tid);
          }
          if (!ok) break;
          const uint32_t f = x & ~LB_VALUE;
          if (f == LB_POISON) {
            ok = false;
            break;
          }
          excl += x & LB_VALUE;
          if (f == LB_INC) done = true;
        }
        j -= 8;
      }
      st_relaxed_u32(status + (uint64_t)tile * RADIX + tid, ok ? (LB_INC | (excl + tcount)) : LB_POISON);
      if (!ok) s_abort = 1;
    }
    s_tstart[tid] = tstart;
    s_goff[tid] = (uint64_t)goffs[tid] + excl - tstart;
  }
  __syncthreads();
  if (s_abort) {
    if (tid == 0) record_error(hdr, GPRTCU_ERR_TIMEOUT);
    return;
  }

  // ---- reorder keys in shared memory by (digit, rank), then scatter runs.
  uint32_t q[ITEMS];
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    const uint32_t pos = warp * WK + i * 32 + lane;
    if (pos < tile_n) {
      const uint32_t d = digit_of(k[i], shift, mask);
      q[i] = s_tstart[d] + s_hist[warp * RADIX + d] + rank[i];
      s_keys[q[i]] = k[i];
    }
  }
  __syncthreads();
  for (uint32_t p = tid; p < tile_n; p += THREADS) {
    const K key = s_keys[p];
    dst_k[s_goff[digit_of(key, shift, mask)] + p] = key;
  }
  if (C::HAS_V) {
    V v[ITEMS];
    if (bulk) {
      if (!mbar_wait(&bars[1], 0, MBAR_WAIT_BUDGET)) s_abort = 1;
    } else {
      for (int i = tid; i < TILE; i += THREADS)
        if ((uint32_t)i < tile_n) s_vals[i] = src_v[tile_start + i];
    }
    __syncthreads();
    if (s_abort) {
      if (tid == 0) record_error(hdr, GPRTCU_ERR_TIMEOUT);
      return;
    }
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      const uint32_t pos = warp * WK + i * 32 + lane;
      if (pos < tile_n) v[i] = s_vals[pos];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      const uint32_t pos = warp * WK + i * 32 + lane;
      if (pos < tile_n) s_vals[q[i]] = v[i];
    }
    __syncthreads();
    for (uint32_t p = tid; p < tile_n; p += THREADS) {
      const K key = s_keys[p];
      dst_v[s_goff[digit_of(key, shift, mask)] + p] = s_vals[p];
    }
  }
}

// Copies the sorted result back into the caller's buffers when the number of
// non-trivial passes was odd (the data then ended in the alternate buffers).
template <typename K, typename V>
__global__ void k_sort_final_copy(K *keys, const K *keys_alt, V *vals, const V *vals_alt, uint64_t n, int passes,
                                  const ScratchHeader *hdr) {
  if (hdr->sel[passes] == 0) return;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    keys[i] = keys_alt[i];
    if (sizeof(V) > 1) vals[i] = vals_alt[i];
  }
}

}  // namespace gprtcu

using namespace gprtcu;

uint32_t gprtcu_spin_budget(void);

namespace {

struct SortLayout {
  size_t keys_alt, vals_alt, hist, trivial, status, total;
  uint64_t tiles;
  int passes;
};

constexpr int kSortThreads = 512;
constexpr int kItems32 = 16;  // 8192 keys per tile for 32-bit keys
constexpr int kItems64 = 8;   // 4096 keys per tile for 64-bit keys
constexpr int kRB = 8;

SortLayout sort_layout(uint64_t n, int kw, int vw, int begin_bit, int end_bit) {
  SortLayout L;
  const int tile = kSortThreads * (kw == 4 ? kItems32 : kItems64);
  L.tiles = (n + tile - 1) / tile;
  L.passes = (end_bit - begin_bit + kRB - 1) / kRB;
  size_t off = sizeof(ScratchHeader);
  L.keys_alt = off;
  off += gprtcu_align256((size_t)n * kw);
  L.vals_alt = off;
  off += gprtcu_align256((size_t)n * vw);
  L.hist = off;
  off += gprtcu_align256((size_t)SORT_MAX_PASSES * 256 * 4);
  L.trivial = off;
  off += 256;
  L.status = off;
  off += gprtcu_align256((size_t)L.passes * L.tiles * (1u << kRB) * 4);
  L.total = off;
  return L;
}

template <typename K, typename V>
gprtcuStatus sort_impl(K *keys, V *vals, uint64_t n, int begin_bit, int end_bit, void *scratch, size_t scratch_bytes,
                       cudaStream_t stream) {
  constexpr int KW = sizeof(K), VW = sizeof(V) > 1 ? sizeof(V) : 0;
  constexpr int ITEMS = KW == 4 ? kItems32 : kItems64;
  using C = PassCfg<K, V, kRB, kSortThreads, ITEMS>;
  if (!keys && n) return GPRTCU_ERR_INVALID_ARG;
  if (VW && !vals && n) return GPRTCU_ERR_INVALID_ARG;
  if (begin_bit < 0 || end_bit > 8 * KW || begin_bit >= end_bit) return GPRTCU_ERR_INVALID_ARG;
  if (n > (uint64_t)LB_VALUE) return GPRTCU_ERR_TOO_LARGE;
  if (!scratch || ((uintptr_t)scratch & 255)) return GPRTCU_ERR_INVALID_ARG;
  SortLayout L = sort_layout(n, KW, VW, begin_bit, end_bit);
  if (scratch_bytes < L.total) return GPRTCU_ERR_SCRATCH_TOO_SMALL;
  if (n <= 1) return GPRTCU_OK;
  char *s = (char *)scratch;
  ScratchHeader *hdr = (ScratchHeader *)s;
  K *keys_alt = (K *)(s + L.keys_alt);
  V *vals_alt = (V *)(s + L.vals_alt);
  uint32_t *hist = (uint32_t *)(s + L.hist);
  uint32_t *trivial = (uint32_t *)(s + L.trivial);
  uint32_t *status = (uint32_t *)(s + L.status);
  // Zero: header, histograms, trivial flags, all passes' status words.
  GPRTCU_TRY(cudaMemsetAsync(s, 0, sizeof(ScratchHeader), stream));
  GPRTCU_TRY(cudaMemsetAsync(s + L.hist, 0, L.total - L.hist, stream));

  const int sms = gprtcu_num_sms();
  k_sort_hist<K, kRB><<<sms * 2, 512, 0, stream>>>(keys, n, begin_bit, end_bit, L.passes, hist, trivial, hdr);
  GPRTCU_TRY(cudaGetLastError());

  static bool attr = false;
  if (!attr) {
    GPRTCU_TRY(cudaFuncSetAttribute(k_sort_pass<K, V, kRB, kSortThreads, ITEMS>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM));
    attr = true;
  }
  const int use_bulk = ((((uintptr_t)keys) | ((uintptr_t)vals) | ((uintptr_t)keys_alt) | ((uintptr_t)vals_alt)) & 15) == 0;
  const uint32_t budget = gprtcu_spin_budget();
  for (int p = 0; p < L.passes; ++p) {
    const int shift = begin_bit + p * kRB;
    const int bits = end_bit - shift < kRB ? end_bit - shift : kRB;
    k_sort_pass<K, V, kRB, kSortThreads, ITEMS><<<(unsigned)L.tiles, kSortThreads, C::SMEM, stream>>>(
        keys, keys_alt, vals, vals_alt, n, shift, bits, p, hist + p * 256, trivial, hdr,
        status + (uint64_t)p * L.tiles * 256, budget, use_bulk);
    GPRTCU_TRY(cudaGetLastError());
  }
  k_sort_final_copy<K, V><<<sms * 4, 256, 0, stream>>>(keys, keys_alt, vals, vals_alt, n, L.passes, hdr);
  GPRTCU_TRY(cudaGetLastError());
  return GPRTCU_OK;
}

}  // namespace

extern "C" GPRTCU_API size_t gprtcuSortScratchSize(uint64_t n, int keyBytes, int valueBytes) {
  if ((keyBytes != 4 && keyBytes != 8) || (valueBytes != 0 && valueBytes != 4 && valueBytes != 8)) return 0;
  return sort_layout(n, keyBytes, valueBytes, 0, 8 * keyBytes).total;
}

extern "C" GPRTCU_API gprtcuStatus gprtcuSortKeysU32(uint32_t *keys, uint64_t n, int beginBit, int endBit,
                                                     void *scratch, size_t scratchBytes, gprtcuStream stream) {
  return sort_impl<uint32_t, char>(keys, nullptr, n, beginBit, endBit, scratch, scratchBytes, (cudaStream_t)stream);
}
extern "C" GPRTCU_API gprtcuStatus gprtcuSortPairsU32(uint32_t *keys, uint32_t *values, uint64_t n, int beginBit,
                                                      int endBit, void *scratch, size_t scratchBytes,
                                                      gprtcuStream stream) {
  return sort_impl<uint32_t, uint32_t>(keys, values, n, beginBit, endBit, scratch, scratchBytes, (cudaStream_t)stream);
}
extern "C" GPRTCU_API gprtcuStatus gprtcuSortKeysU64(uint64_t *keys, uint64_t n, int beginBit, int endBit,
                                                     void *scratch, size_t scratchBytes, gprtcuStream stream) {
  return sort_impl<uint64_t, char>(keys, nullptr, n, beginBit, endBit, scratch, scratchBytes, (cudaStream_t)stream);
}
extern "C" GPRTCU_API gprtcuStatus gprtcuSortPairsU64(uint64_t *keys, uint32_t *values, uint64_t n, int beginBit,
                                                      int endBit, void *scratch, size_t scratchBytes,
                                                      gprtcuStream stream) {
  return sort_impl<uint64_t, uint32_t>(keys, values, n, beginBit, endBit, scratch, scratchBytes, (cudaStream_t)stream);
}
extern "C" GPRTCU_API gprtcuStatus gprtcuSortPairsU64U64(uint64_t *keys, uint64_t *values, uint64_t n, int beginBit,
                                                         int endBit, void *scratch, size_t scratchBytes,
                                                         gprtcuStream stream) {
  return sort_impl<uint64_t, uint64_t>(keys, values, n, beginBit, endBit, scratch, scratchBytes, (cudaStream_t)stream);
}
