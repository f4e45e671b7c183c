// sort_kernels.cuh -- the radix-sort kernels, templated over the shape the
// autotuner chooses: digit width RB (4, 6 or 8 bits), warps per block and
// keys per tile.  Each sort_*.cu file instantiates the whole tuning grid for
// one key/payload type pair; sort.cu holds the host driver and the tuner.
//
// Replaces gprtBufferSort / gprtBufferSortPayload (gprt/gprt_host.h:2384,2416;
// host driver gprt/gprt.cpp:8821-9073; kernels gprt/gprt_sort.slang:109-637).
// Same contract: stable ascending sort, result in place in the caller's
// buffers.  The reference runs FidelityFX's reduce-then-scan with 4-bit
// digits: five dispatches per digit, 16 passes over 64-bit words.  This is a
// onesweep design instead (Adinets & Merrill 2022):
//   1. one histogram kernel reads every key once (16-byte loads) and builds
//      the digit histograms of all passes with shared atomics; its last CTA
//      scans them into global digit offsets and marks passes whose digit is
//      constant (skipped);
//   2. one digit-binning kernel per pass: a tile of keys and one of payloads
//      arrive in shared memory by bulk async copies (TMA); warps rank their
//      keys against per-warp shared histograms (the 8-bit pass finds a key's
//      equal-digit lanes through a per-warp leader table and five ballots),
//      each digit's tile count is published to a per-(tile, digit) status
//      word and a decoupled look-back over earlier tiles gives the digit's
//      global position; the tile-sorted order is built in shared memory so
//      the scatter leaves the tile as coalesced per-digit runs.
// Traffic per pass: read + write of keys and payloads; plus one read of the
// keys for the histograms.
#pragma once
#include <algorithm>
#include <array>
#include <type_traits>
#include <utility>

#include "common.cuh"

namespace gprtcu {

constexpr uint32_t LB_AGG = 1u << 30;
constexpr uint32_t LB_INC = 2u << 30;
constexpr uint32_t LB_POISON = 3u << 30;
constexpr uint32_t LB_VALUE = (1u << 30) - 1;
constexpr int SORT_MAX_PASSES = 16;
// Per-pass flag written by the histogram kernel: every key has the same
// digit, the pass is skipped.
constexpr uint32_t SORT_FLAG_TRIVIAL = 1u;

// The sort's scratch header: the common 256-byte header (error status first)
// followed by per-pass tile tickets and ping-pong selectors.  ticket[0] is the
// histogram kernel's done-counter, ticket[1+p] pass p's tile ticket; sel[p]
// says which buffer holds pass p's input (sel[passes]: the final result).
struct SortHeader {
  ScratchHeader h;
  uint32_t ticket[SORT_MAX_PASSES + 1];
  uint32_t sel[SORT_MAX_PASSES + 1];
  uint32_t pad[64 - 2 * (SORT_MAX_PASSES + 1)];
};
static_assert(sizeof(SortHeader) == 512, "sort header is 512 bytes");

// One point of the tuning grid.
struct SortShape {
  int rb;     // digit bits
  int tile;   // keys per tile (one CTA per tile)
  int warps;  // warps per CTA
};

// The tuning grid: digit bits {4, 6, 8} x tile {1024 .. 8192} x warps {4, 8,
// 16}, keeping shapes with 1..32 keys per thread and at least one thread per
// digit (so 8-bit digits need 8 or 16 warps); plus 6144-key tiles of 8 warps
// at 8-bit digits (the largest tile of which three CTAs share an SM with
// 32-bit keys and payloads).
inline constexpr SortShape kSortGrid[] = {
    {8, 1024, 8}, {8, 2048, 8}, {8, 4096, 8}, {8, 6144, 8}, {8, 8192, 8},     //
    {8, 1024, 16}, {8, 2048, 16}, {8, 4096, 16}, {8, 8192, 16},               //
    {6, 1024, 4}, {6, 2048, 4}, {6, 4096, 4},                                 //
    {6, 1024, 8}, {6, 2048, 8}, {6, 4096, 8}, {6, 8192, 8},                   //
    {6, 1024, 16}, {6, 2048, 16}, {6, 4096, 16}, {6, 8192, 16},               //
    {4, 1024, 4}, {4, 2048, 4}, {4, 4096, 4},                                 //
    {4, 1024, 8}, {4, 2048, 8}, {4, 4096, 8}, {4, 8192, 8},                   //
    {4, 1024, 16}, {4, 2048, 16}, {4, 4096, 16}, {4, 8192, 16},               //
};
inline constexpr int kSortGridSize = (int)(sizeof(kSortGrid) / sizeof(kSortGrid[0]));
inline constexpr int kSortMinTile = 1024;

// Everything one sort call's kernels need (device pointers into the caller's
// buffers and the scratch).
struct SortArgs {
  void *keys, *keys_alt, *vals, *vals_alt;
  uint64_t n, tiles;
  int begin_bit, end_bit, passes;
  uint32_t *hist;     // [passes][RADIX] digit counts, then global offsets
  uint32_t *trivial;  // [passes] SORT_FLAG_* bits
  SortHeader *hdr;
  uint32_t *status;   // two regions of [tiles][RADIX] look-back words
  uint32_t budget;
  int use_bulk;
  int sms;
  int64_t skip_tile;  // test hook: this tile of every pass never publishes (-1: none)
  uint32_t pf_tiles;  // 8-bit passes: a CTA prefetches into L2 the tile this far after its own (0: none)
};

using SortRunFn = gprtcuStatus (*)(const SortArgs &, cudaStream_t);

template <typename K> __device__ __forceinline__ uint32_t digit_of(K key, int shift, uint32_t mask) {
  return (uint32_t)(key >> shift) & mask;
}

// Lanes of the warp holding the same BITS-bit digit as this lane
// (warp-level multisplit by ballots, one per digit bit).  Replaces
// __match_any_sync, whose pipe throughput made the ranking issue-bound on
// sm_100a.
template <int BITS> __device__ __forceinline__ unsigned warp_peers(uint32_t d) {
  unsigned m = FULL_MASK;
#pragma unroll
  for (int b = 0; b < BITS; ++b) {
    const bool bit = (d >> b) & 1u;
    const unsigned bb = __ballot_sync(FULL_MASK, bit);
    m &= bit ? bb : ~bb;
  }
  return m;
}

// The same peers with four instructions per digit bit: a predicate from one
// AND, the vote, a select of 0 or ~0 from the predicate, and one
// three-input logic op m &= votes ^ select (the plain form above compiles to
// about six per bit).
template <int BITS> __device__ __forceinline__ unsigned warp_peers_p(uint32_t d) {
  unsigned m = FULL_MASK;
#pragma unroll
  for (int b = 0; b < BITS; ++b) {
    unsigned bb, t;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "and.b32 %1, %2, %3;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "vote.sync.ballot.b32 %0, p, 0xffffffff;\n\t"
        "selp.b32 %1, 0, -1, p;\n\t}"
        : "=r"(bb), "=&r"(t)
        : "r"(d), "r"(1u << b));
    m &= bb ^ t;
  }
  return m;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// ---------------------------------------------------------------------------
// 1. histogram of every pass's digit, one read of the keys
// ---------------------------------------------------------------------------
template <typename K, int RB>
__global__ void __launch_bounds__(512) k_sort_hist(const K *__restrict__ keys, uint64_t n, int begin_bit, int end_bit,
                                                   int passes, uint32_t *ghist, uint32_t *trivial, SortHeader *hdr) {
  constexpr int RADIX = 1 << RB;
  static_assert(SORT_MAX_PASSES * RADIX <= 4096, "histogram fits 16 KB of shared memory");
  __shared__ uint32_t sh[SORT_MAX_PASSES * RADIX];
  __shared__ bool s_last;
  __shared__ uint32_t s_triv[SORT_MAX_PASSES];
  const int tid = threadIdx.x, lane = tid & 31;
  for (int i = tid; i < passes * RADIX; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  // One shared atomic per key and pass.  The hardware merges a warp's
  // same-address adds, so skewed digits cost no more than uniform ones
  // (B200, 2^28 Zipf(1.1) keys: 0.47 ms, where aggregating each warp's equal
  // digits by ballots first was ALU-bound at 4.2 ms).
  auto count = [&](K key) {
    for (int p = 0; p < passes; ++p) {
      const int shift = begin_bit + p * RB;
      const int bits = min(RB, end_bit - shift);
      atomicAdd(&sh[p * RADIX + digit_of(key, shift, (1u << bits) - 1u)], 1u);
    }
  };
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  if ((reinterpret_cast<uintptr_t>(keys) & 15) == 0) {
    // 16-byte loads, four per thread in flight.
    constexpr int VEC = 16 / sizeof(K), UNROLL = 4;
    const uint64_t nv = n / VEC;
    const uint4 *kv = reinterpret_cast<const uint4 *>(keys);
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x * UNROLL; i0 < nv; i0 += stride * UNROLL) {
      uint4 v[UNROLL];
#pragma unroll
      for (int u = 0; u < UNROLL; ++u) {
        const uint64_t i = i0 + (uint64_t)u * blockDim.x + tid;
        v[u] = i < nv ? __ldg(kv + i) : make_uint4(0, 0, 0, 0);
      }
#pragma unroll
      for (int u = 0; u < UNROLL; ++u)
        if (i0 + (uint64_t)u * blockDim.x + tid < nv) {
          const K *kk = reinterpret_cast<const K *>(&v[u]);
#pragma unroll
          for (int e = 0; e < VEC; ++e) count(kk[e]);
        }
    }
    if (blockIdx.x == 0)
      for (uint64_t i = nv * VEC + tid; i < n; i += blockDim.x) count(keys[i]);
  } else {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + tid; i < n; i += stride) count(keys[i]);
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
    if (lane == 0) s_triv[p] = triv ? SORT_FLAG_TRIVIAL : 0u;
  }
  __syncthreads();
  if (tid == 0) {
    uint32_t sel = 0;
    for (int p = 0; p < passes; ++p) {
      hdr->sel[p] = sel;
      trivial[p] = s_triv[p];
      if (!(s_triv[p] & SORT_FLAG_TRIVIAL)) sel ^= 1u;
    }
    hdr->sel[passes] = sel;
  }
}

// ---------------------------------------------------------------------------
// 2. one digit-binning pass
// ---------------------------------------------------------------------------
template <typename K, typename V, int RB, int WARPS, int ITEMS> struct PassCfg {
  static constexpr int RADIX = 1 << RB;
  static constexpr int THREADS = WARPS * 32;
  static constexpr int TILE = THREADS * ITEMS;
  static constexpr int WARP_KEYS = 32 * ITEMS;
  static constexpr bool HAS_V = sizeof(V) > 1;
  static constexpr size_t KEY_BYTES = (size_t)TILE * sizeof(K);
  static constexpr size_t VAL_BYTES = HAS_V ? (size_t)TILE * sizeof(V) : 0;
  static constexpr size_t HIST_BYTES = (size_t)WARPS * RADIX * 4;
  static constexpr size_t SMEM = KEY_BYTES + VAL_BYTES + HIST_BYTES + RADIX * 4 /*goff*/ + RADIX * 4 /*tile start*/ +
                                 16 /*barriers*/;
  // CTAs per SM the kernel is compiled for: as many as shared memory allows,
  // up to 2048 threads, and no fewer registers than 64 per thread.
  static constexpr int SMEM_CTAS = (int)((228 * 1024) / (SMEM + 1024));
  static constexpr int THREAD_CTAS = 2048 / THREADS;
  static constexpr int REG_CTAS = 65536 / (THREADS * 64);
  static constexpr int MIN_CTAS_A = SMEM_CTAS < THREAD_CTAS ? SMEM_CTAS : THREAD_CTAS;
  static constexpr int MIN_CTAS_B = MIN_CTAS_A < REG_CTAS ? MIN_CTAS_A : REG_CTAS;
  static constexpr int MIN_CTAS = MIN_CTAS_B < 1 ? 1 : MIN_CTAS_B;
  static_assert(THREADS >= RADIX, "one thread per digit");
  static_assert(ITEMS >= 1 && ITEMS <= 32, "1..32 keys per thread");
};

// Exclusive scan of v over threads [0, RADIX) (RADIX <= THREADS); every
// thread of the block must call it.
template <int RADIX>
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

template <typename K, typename V, int RB, int WARPS, int ITEMS>
__global__ void __launch_bounds__(WARPS * 32, (PassCfg<K, V, RB, WARPS, ITEMS>::MIN_CTAS))
    k_sort_pass(const SortArgs a, int pass, int shift, int bits) {
  using C = PassCfg<K, V, RB, WARPS, ITEMS>;
  constexpr int RADIX = C::RADIX, THREADS = C::THREADS, TILE = C::TILE, WK = C::WARP_KEYS;
  const uint32_t flags = ld_relaxed_u32(&a.trivial[pass]);
  if (flags & SORT_FLAG_TRIVIAL) return;  // every key has the same digit: nothing moves
  // An earlier pass gave up on a wait: its output is not a permutation of the
  // keys, so the global digit offsets no longer bound this pass's writes.
  if (ld_relaxed_u32(&a.hdr->h.status) != 0) return;

  extern __shared__ __align__(128) unsigned char smem[];
  K *s_keys = reinterpret_cast<K *>(smem);
  V *s_vals = reinterpret_cast<V *>(smem + C::KEY_BYTES);
  uint32_t *s_hist = reinterpret_cast<uint32_t *>(smem + C::KEY_BYTES + C::VAL_BYTES);  // [WARPS][RADIX]
  uint32_t *s_goff = s_hist + WARPS * RADIX;
  uint64_t *bars = reinterpret_cast<uint64_t *>(s_goff + 2 * RADIX);
  __shared__ uint32_t s_tile, s_abort;
  __shared__ uint32_t s_tmp[32];

  SortHeader *hdr = a.hdr;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t sel = hdr->sel[pass];
  const K *src_k = static_cast<const K *>(sel ? a.keys_alt : a.keys);
  K *dst_k = static_cast<K *>(sel ? a.keys : a.keys_alt);
  const V *src_v = static_cast<const V *>(sel ? a.vals_alt : a.vals);
  V *dst_v = static_cast<V *>(sel ? a.vals : a.vals_alt);
  const uint32_t mask = (1u << bits) - 1u;
  // Look-back words: executed passes alternate between two regions (sel
  // flips with every executed pass); this pass clears its tile's words of the
  // other region for the next executed pass.
  uint32_t *status = a.status + (sel ? a.tiles * RADIX : 0);
  uint32_t *status_next = a.status + (sel ? 0 : a.tiles * RADIX);

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
  const uint32_t tile_n = (uint32_t)min((uint64_t)TILE, a.n - tile_start);
  const bool bulk = a.use_bulk && tile_n == TILE;
  if (tid == 0 && bulk) {
    mbar_arrive_expect_tx(&bars[0], (uint32_t)C::KEY_BYTES);
    bulk_g2s(s_keys, src_k + tile_start, (uint32_t)C::KEY_BYTES, &bars[0]);
    if constexpr (C::HAS_V) {
      mbar_arrive_expect_tx(&bars[1], (uint32_t)C::VAL_BYTES);
      bulk_g2s(s_vals, src_v + tile_start, (uint32_t)C::VAL_BYTES, &bars[1]);
    }
  }
  for (int i = tid; i < WARPS * RADIX; i += THREADS) s_hist[i] = 0;
  for (int i = tid; i < RADIX; i += THREADS) status_next[(uint64_t)tile * RADIX + i] = 0;
  if (!bulk) {
    // The last tile is padded with all-ones keys: they rank after every real
    // key (stable order puts them last within the top digit), so the real
    // keys fill tile-sorted slots [0, tile_n) and no loop needs a bounds test
    // before the scatter; the top digit's count leaves the padding out.
    for (int i = tid; i < TILE; i += THREADS) s_keys[i] = (uint32_t)i < tile_n ? src_k[tile_start + i] : ~(K)0;
  } else if (!mbar_wait(&bars[0], 0, mbar_budget_of(a.budget))) {
    s_abort = 1;
  }
  // On every early return, thread 0 first lets the tile's copies land, so no
  // copy writes shared memory after the CTA has released it.
  auto leave = [&]() {
    if (tid == 0) {
      record_error(&hdr->h, GPRTCU_ERR_TIMEOUT);
      if (bulk) {
        mbar_wait(&bars[0], 0, mbar_budget_of(a.budget));
        if constexpr (C::HAS_V) mbar_wait(&bars[1], 0, mbar_budget_of(a.budget));
      }
    }
  };
  __syncthreads();
  if (s_abort) {
    leave();
    return;
  }

  // ---- rank: warp w owns tile positions [w*WK, (w+1)*WK), item-major.  A
  // key's rank within its warp is the warp histogram wh[d] so far plus its
  // equal-digit lanes below it.
  K k[ITEMS];
  uint32_t rank[ITEMS];
  uint32_t *wh = s_hist + warp * RADIX;
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    k[i] = s_keys[warp * WK + i * 32 + lane];
    const uint32_t d = digit_of(k[i], shift, mask);
    const unsigned peers = warp_peers_p<RB>(d);
    const uint32_t base = wh[d];
    __syncwarp();
    if (lane == 31 - __clz(peers)) wh[d] = base + __popc(peers);
    __syncwarp();
    rank[i] = base + __popc(peers & lt);
  }
  __syncthreads();

  // ---- per digit: tile count, publish, tile-exclusive start, look-back;
  // then each warp's first slot of the digit in the tile-sorted order.
  uint32_t tcount = 0;
  // Fault injection for tests: the hooked tile never publishes its counts.
  const bool hooked = (int64_t)tile == a.skip_tile;
  if (tid < RADIX) {
#pragma unroll 4
    for (int w = 0; w < WARPS; ++w) tcount += s_hist[w * RADIX + tid];
    if ((uint32_t)tid == mask) tcount -= TILE - tile_n;  // padding of the last tile
    if (!hooked) st_relaxed_u32(status + (uint64_t)tile * RADIX + tid, (tile == 0 ? LB_INC : LB_AGG) | tcount);
  }
  const uint32_t tstart = block_excl_scan_digits<RADIX>(tcount, s_tmp);
  if (tid < RADIX) {
    uint32_t excl = 0;
    bool ok = true;
    if (hooked) {
      s_abort = 1;
    } else if (tile > 0) {
      // Eight predecessors per probe (loads issued together), nearest first:
      // the inclusive prefix of a digit can only advance one probe window per
      // L2 round trip.
      int64_t j = (int64_t)tile - 1;
      uint32_t spins = 0;
      bool done = false;
      while (!done && ok) {
        uint32_t sw[8];
#pragma unroll
        for (int c = 0; c < 8; ++c)
          sw[c] = j - c >= 0 ? ld_relaxed_u32(status + (uint64_t)(j - c) * RADIX + tid) : LB_INC;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          if (done || !ok) break;
          uint32_t x = sw[c];
          while ((x & ~LB_VALUE) == 0) {
            if (++spins > a.budget) {
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
    // global position of tile-sorted slot p of this digit = s_goff[d] + p
    // (mod 2^32; the true value is below 2^30)
    s_goff[tid] = a.hist[pass * RADIX + tid] + excl - tstart;
    uint32_t run = tstart;
#pragma unroll 4
    for (int w = 0; w < WARPS; ++w) {
      const uint32_t c = s_hist[w * RADIX + tid];
      s_hist[w * RADIX + tid] = run;
      run += c;
    }
  }
  __syncthreads();
  if (s_abort) {
    leave();
    return;
  }

  // ---- reorder keys in shared memory by (digit, rank), then scatter runs.
  uint32_t q[ITEMS];
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    q[i] = s_hist[warp * RADIX + digit_of(k[i], shift, mask)] + rank[i];
    s_keys[q[i]] = k[i];
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < ITEMS; ++j) {
    const uint32_t p = j * THREADS + tid;
    if (p < tile_n) {
      const K key = s_keys[p];
      dst_k[s_goff[digit_of(key, shift, mask)] + p] = key;
    }
  }
  if constexpr (C::HAS_V) {
    V v[ITEMS];
    if (bulk) {
      if (!mbar_wait(&bars[1], 0, mbar_budget_of(a.budget))) s_abort = 1;
    } else {
      for (int i = tid; i < TILE; i += THREADS)
        if ((uint32_t)i < tile_n) s_vals[i] = src_v[tile_start + i];
    }
    __syncthreads();
    if (s_abort) {
      leave();
      return;
    }
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) v[i] = s_vals[warp * WK + i * 32 + lane];  // padding slots: unused
    __syncthreads();
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) s_vals[q[i]] = v[i];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const uint32_t p = j * THREADS + tid;
      if (p < tile_n) dst_v[s_goff[digit_of(s_keys[p], shift, mask)] + p] = s_vals[p];
    }
  }
}

// ---------------------------------------------------------------------------
// 2b. one 8-bit digit pass with fewer instructions per key
// ---------------------------------------------------------------------------
// The pass above executes ~130 warp instructions per 32 keys on B200 (2^26
// pairs; ALU pipe 59 %, issue 59 %), about 40 of them in the eight votes of
// its ranking.  This one trims the rest: digits are one byte-permute when
// they are whole bytes (instead of a shift and a mask, four times per key),
// every lane of a digit's peers writes the warp's count (no leader
// election), no key is held in registers (the tile-sorted order is a 16-bit
// index per slot, and the scatter gathers keys and payloads from their
// untouched tiles, so payloads need no reorder round), full tiles skip bounds
// tests, and keys and payloads leave the tile in one loop.  The look-back's
// first window of loads is issued before the tile-local order is written and
// resolved after it, so its L2 round trip overlaps that work (2^28 Zipf
// pairs: 6.14 -> 5.95 ms).
//
// RANK picks how a lane finds the lanes of its row with the same digit:
//   0  leader tables (the default): every lane stores its lane number into
//      its digit's byte of a per-warp table; after the warp barrier all
//      lanes of a digit read back the same number (one of theirs), and
//      different digits read different numbers, so five votes on that
//      number replace eight on the digit (6.29 -> 6.14 ms, 2^28 Zipf pairs;
//      the same on uniform keys);
//   2  a 32-bit shared-memory OR of the lane bit into the digit's word (a
//      64-bit word carrying the count as well was 2.5x slower on Zipf keys:
//      same-word atomics serialise);
//   3  match.any;  4  eight plain votes;  5  eight predicated votes.
// All give the same bits; 2-5 stay for measurement.
template <typename K, typename V, int WARPS, int ITEMS, int RANK> struct Pass8Cfg {
  static constexpr int RADIX = 256;
  static constexpr int THREADS = WARPS * 32;
  static constexpr int TILE = THREADS * ITEMS;
  static constexpr int WARP_KEYS = 32 * ITEMS;
  static constexpr bool HAS_V = sizeof(V) > 1;
  static constexpr size_t KEY_BYTES = (size_t)TILE * sizeof(K);
  static constexpr size_t VAL_BYTES = HAS_V ? (size_t)TILE * sizeof(V) : 0;
  static constexpr size_t TBL_BYTES = (size_t)WARPS * RADIX * 4;  // per-warp counts, then first slots
  static constexpr size_t MSK_BYTES = RANK == 2 ? (size_t)WARPS * RADIX * 4 : 0;  // per-warp lane masks
  static constexpr size_t PERM_BYTES = (size_t)TILE * 2;
  static constexpr size_t LEAD_BYTES = RANK == 0 ? (size_t)WARPS * 2 * RADIX : 0;  // two leader tables per warp
  static constexpr size_t SMEM = KEY_BYTES + VAL_BYTES + TBL_BYTES + MSK_BYTES + PERM_BYTES + LEAD_BYTES +
                                 RADIX * 4 /*goff*/ + 16 /*barriers*/;
  static_assert(TILE <= 65536, "16-bit slot indices");
  static constexpr int SMEM_CTAS = (int)((228 * 1024) / (SMEM + 1024));
  static constexpr int THREAD_CTAS = 2048 / THREADS;
  static constexpr int MIN_CTAS_A = SMEM_CTAS < THREAD_CTAS ? SMEM_CTAS : THREAD_CTAS;
  static constexpr int REG_CTAS = 65536 / (THREADS * 64);
  static constexpr int MIN_CTAS_B = MIN_CTAS_A < REG_CTAS ? MIN_CTAS_A : REG_CTAS;
  static constexpr int MIN_CTAS = MIN_CTAS_B < 1 ? 1 : MIN_CTAS_B;
  static_assert(THREADS >= RADIX, "one thread per digit");
};

// Look-back words of the 8-bit pass: {flag : 2 | value : 30} for n below
// 2^30, or {flag : 2 | value : 62} (WIDE) for the larger n up to 2^32 - 1
// that the reference's uint32 key count allows.
template <bool WIDE> struct LbWord {
  using T = typename std::conditional<WIDE, uint64_t, uint32_t>::type;
  static constexpr int FB = WIDE ? 62 : 30;
  static constexpr T AGG = (T)1 << FB, INC = (T)2 << FB, POISON = (T)3 << FB, VALUE = ((T)1 << FB) - 1;
  __device__ static __forceinline__ T load(const T *p) {
    if constexpr (WIDE) return ld_relaxed_u64(p);
    else return ld_relaxed_u32(p);
  }
  __device__ static __forceinline__ void store(T *p, T v) {
    if constexpr (WIDE) st_relaxed_u64(p, v);
    else st_relaxed_u32(p, v);
  }
};


// Digit of a key: BYTE = the digit is one whole byte of the key (8 bits at a
// multiple of 8), taken by one byte-permute of the key's word that holds it.
template <bool BYTE, typename K>
__device__ __forceinline__ uint32_t digit8(K key, int shift, uint32_t mask, uint32_t sel) {
  if constexpr (BYTE) {
    const uint32_t w = sizeof(K) == 8 ? (uint32_t)((uint64_t)key >> (shift & 32)) : (uint32_t)key;
    return __byte_perm(w, 0u, sel);
  } else {
    return (uint32_t)(key >> shift) & mask;
  }
}

template <typename K, typename V, int WARPS, int ITEMS, bool BYTE, bool WIDE, int RANK>
__global__ void __launch_bounds__(WARPS * 32, (Pass8Cfg<K, V, WARPS, ITEMS, RANK>::MIN_CTAS))
    k_sort_pass8(const SortArgs a, int pass, int shift, int bits) {
  using C = Pass8Cfg<K, V, WARPS, ITEMS, RANK>;
  using LB = LbWord<WIDE>;
  using SW = typename LB::T;
  constexpr int RADIX = C::RADIX, THREADS = C::THREADS, TILE = C::TILE, WK = C::WARP_KEYS;
  SortHeader *hdr = a.hdr;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // The pass's words, this thread's digit offset and (thread 0) the tile
  // ticket are requested together, before any of them is tested: one L2
  // round trip at the start of the CTA instead of four in a row.  A ticket
  // taken by a pass that then returns is never used by anyone.
  uint32_t ticket = 0;
  if (tid == 0) ticket = atomicAdd(&hdr->ticket[1 + pass], 1u);
  const uint32_t flags = ld_relaxed_u32(&a.trivial[pass]);
  const uint32_t err0 = ld_relaxed_u32(&hdr->h.status);
  const uint32_t sel = ld_relaxed_u32(&hdr->sel[pass]);
  const uint32_t ghist = tid < RADIX ? a.hist[pass * RADIX + tid] : 0u;  // global offset of the digit
  if (flags & SORT_FLAG_TRIVIAL) return;  // every key has the same digit: nothing moves
  // An earlier pass gave up on a wait: its output is not a permutation of the
  // keys, so the global digit offsets no longer bound this pass's writes.
  if (err0 != 0) return;

  extern __shared__ __align__(128) unsigned char smem[];
  K *s_keys = reinterpret_cast<K *>(smem);
  V *s_vals = reinterpret_cast<V *>(smem + C::KEY_BYTES);
  uint32_t *s_cnt = reinterpret_cast<uint32_t *>(smem + C::KEY_BYTES + C::VAL_BYTES);  // [WARPS][RADIX]
  uint32_t *s_msk = reinterpret_cast<uint32_t *>(smem + C::KEY_BYTES + C::VAL_BYTES + C::TBL_BYTES);
  uint16_t *s_perm = reinterpret_cast<uint16_t *>(smem + C::KEY_BYTES + C::VAL_BYTES + C::TBL_BYTES + C::MSK_BYTES);
  uint8_t *s_lead = smem + C::KEY_BYTES + C::VAL_BYTES + C::TBL_BYTES + C::MSK_BYTES + C::PERM_BYTES;
  uint32_t *s_goff = reinterpret_cast<uint32_t *>(smem + C::KEY_BYTES + C::VAL_BYTES + C::TBL_BYTES + C::MSK_BYTES +
                                                  C::PERM_BYTES + C::LEAD_BYTES);
  uint64_t *bars = reinterpret_cast<uint64_t *>(s_goff + RADIX);
  __shared__ uint32_t s_tile, s_abort;
  __shared__ uint32_t s_tmp[32];

  const K *src_k = static_cast<const K *>(sel ? a.keys_alt : a.keys);
  K *dst_k = static_cast<K *>(sel ? a.keys : a.keys_alt);
  const V *src_v = static_cast<const V *>(sel ? a.vals_alt : a.vals);
  V *dst_v = static_cast<V *>(sel ? a.vals : a.vals_alt);
  const uint32_t mask = (1u << bits) - 1u;
  const uint32_t bsel = 0x4440u | (uint32_t)((shift >> 3) & 3);  // byte (shift / 8) % 4 of the word, zero above
  SW *status = reinterpret_cast<SW *>(a.status) + (sel ? a.tiles * RADIX : 0);
  SW *status_next = reinterpret_cast<SW *>(a.status) + (sel ? 0 : a.tiles * RADIX);

  if (tid == 0) {
    s_tile = ticket;
    s_abort = 0;
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
    // thread 0 knows the tile: its copies start before the block barrier
    if (a.use_bulk && ((uint64_t)ticket + 1) * TILE <= a.n) {
      const uint64_t ts = (uint64_t)ticket * TILE;
      mbar_arrive_expect_tx(&bars[0], (uint32_t)C::KEY_BYTES);
      bulk_g2s(s_keys, src_k + ts, (uint32_t)C::KEY_BYTES, &bars[0]);
      if constexpr (C::HAS_V) {
        mbar_arrive_expect_tx(&bars[1], (uint32_t)C::VAL_BYTES);
        bulk_g2s(s_vals, src_v + ts, (uint32_t)C::VAL_BYTES, &bars[1]);
      }
    }
    // The tile that a CTA starting about pf_tiles tickets later will take:
    // its keys and payloads are fetched into L2 now, so that CTA's copies
    // hit L2 instead of waiting on DRAM at its start.
    const uint64_t pt = (uint64_t)ticket + a.pf_tiles;
    if (a.pf_tiles && a.use_bulk && (pt + 1) * TILE <= a.n) {
      bulk_prefetch_l2(src_k + pt * TILE, (uint32_t)C::KEY_BYTES);
      if constexpr (C::HAS_V) bulk_prefetch_l2(src_v + pt * TILE, (uint32_t)C::VAL_BYTES);
    }
  }
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint64_t tile_start = (uint64_t)tile * TILE;
  const uint32_t tile_n = (uint32_t)min((uint64_t)TILE, a.n - tile_start);
  const bool full = tile_n == TILE;
  const bool bulk = a.use_bulk && full;
  {
    uint4 *t4 = reinterpret_cast<uint4 *>(s_cnt);  // counts and (RANK 2) masks are adjacent
    for (int i = tid; i < (int)((C::TBL_BYTES + C::MSK_BYTES) / 16); i += THREADS) t4[i] = make_uint4(0u, 0u, 0u, 0u);
  }
  for (int i = tid; i < RADIX; i += THREADS) status_next[(uint64_t)tile * RADIX + i] = 0;
  if (!bulk) {
    // The last tile is padded with all-ones keys: they rank after every real
    // key within the top digit, so the real keys fill slots [0, tile_n).
    for (int i = tid; i < TILE; i += THREADS) s_keys[i] = (uint32_t)i < tile_n ? src_k[tile_start + i] : ~(K)0;
    if constexpr (C::HAS_V)
      for (int i = tid; i < TILE; i += THREADS)
        if ((uint32_t)i < tile_n) s_vals[i] = src_v[tile_start + i];
  } else if (!mbar_wait(&bars[0], 0, mbar_budget_of(a.budget))) {
    s_abort = 1;
  }
  auto leave = [&]() {
    if (tid == 0) {
      record_error(&hdr->h, GPRTCU_ERR_TIMEOUT);
      if (bulk) {
        mbar_wait(&bars[0], 0, mbar_budget_of(a.budget));
        if constexpr (C::HAS_V) mbar_wait(&bars[1], 0, mbar_budget_of(a.budget));
      }
    }
  };
  __syncthreads();
  if (s_abort) {
    leave();
    return;
  }

  // ---- rank: warp w owns tile positions [w*WK, (w+1)*WK), row-major (row
  // i = positions w*WK + 32 i .. +31).
  uint32_t rank[ITEMS];
  uint32_t *wc = s_cnt + warp * RADIX;
  uint32_t *wm = s_msk + warp * RADIX;
  const uint32_t lanebit = 1u << lane, lt = lanebit - 1u;
  if constexpr (RANK == 0) {
    // Two leader tables alternate by row, so the next row's stores are
    // issued before this row's votes (the table they overwrite was read a
    // row earlier, before the barriers that end that row).
    uint8_t *wl = s_lead + warp * 2 * RADIX;
    uint32_t dn = digit8<BYTE>(s_keys[warp * WK + lane], shift, mask, bsel);
    wl[dn] = (uint8_t)lane;
    __syncwarp();
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      const uint32_t d = dn;
      const uint32_t ld = wl[(i & 1) * RADIX + d];
      const uint32_t base = wc[d];
      if (i + 1 < ITEMS) {
        dn = digit8<BYTE>(s_keys[warp * WK + (i + 1) * 32 + lane], shift, mask, bsel);
        wl[((i + 1) & 1) * RADIX + dn] = (uint8_t)lane;
      }
      const uint32_t peers = warp_peers_p<5>(ld);
      __syncwarp();
      wc[d] = base + __popc(peers);  // every peer stores the same count
      __syncwarp();
      rank[i] = base + __popc(peers & lt);
    }
  } else {
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
      const uint32_t d = digit8<BYTE>(s_keys[warp * WK + i * 32 + lane], shift, mask, bsel);
      uint32_t peers;
      const uint32_t base = wc[d];
      if constexpr (RANK == 2) {
        atomicOr(wm + d, lanebit);
        __syncwarp();
        peers = *reinterpret_cast<volatile uint32_t *>(wm + d);
        __syncwarp();
        wm[d] = 0u;
      } else if constexpr (RANK == 3) {
        peers = __match_any_sync(FULL_MASK, d);
        __syncwarp();
      } else if constexpr (RANK == 4) {
        peers = warp_peers<8>(d);
        __syncwarp();
      } else {
        peers = warp_peers_p<8>(d);
        __syncwarp();
      }
      wc[d] = base + __popc(peers);  // every peer stores the same count
      __syncwarp();
      rank[i] = base + __popc(peers & lt);
    }
  }
  __syncthreads();

  // ---- per digit: tile count, publish, tile-exclusive start, look-back;
  // then each warp's first slot of the digit in the tile-sorted order (kept
  // in the low half of the warp's word).
  uint32_t tcount = 0;
  const bool hooked = (int64_t)tile == a.skip_tile;  // test hook: this tile never publishes
  if (tid < RADIX) {
#pragma unroll 4
    for (int w = 0; w < WARPS; ++w) tcount += s_cnt[w * RADIX + tid];
    if ((uint32_t)tid == mask) tcount -= TILE - tile_n;  // padding of the last tile
    if (!hooked) LB::store(status + (uint64_t)tile * RADIX + tid, (tile == 0 ? LB::INC : LB::AGG) | (SW)tcount);
  }
  const uint32_t tstart = block_excl_scan_digits<RADIX>(tcount, s_tmp);

  // Look-back of this thread's digit: eight predecessors per probe (loads
  // issued together), nearest first.  excl stays below 2^32: the count of
  // keys before this tile's digit run.
  uint32_t excl = 0;
  SW sw[8];
  int64_t j = (int64_t)tile - 1;
  auto probe = [&]() {
#pragma unroll
    for (int c = 0; c < 8; ++c) sw[c] = j - c >= 0 ? LB::load(status + (uint64_t)(j - c) * RADIX + tid) : LB::INC;
  };
  // Resolves the probed window (and further ones) into excl, publishes the
  // inclusive count or the poison word; false when a wait gave up.
  auto resolve = [&]() -> bool {
    uint32_t spins = 0;
    bool done = false, ok = true;
    while (true) {
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        if (done || !ok) break;
        SW x = sw[c];
        while ((x & ~LB::VALUE) == 0) {
          if (++spins > a.budget) {
            ok = false;
            break;
          }
          x = LB::load(status + (uint64_t)(j - c) * RADIX + tid);
        }
        if (!ok) break;
        const SW f = x & ~LB::VALUE;
        if (f == LB::POISON) {
          ok = false;
          break;
        }
        excl += (uint32_t)(x & LB::VALUE);
        if (f == LB::INC) done = true;
      }
      if (done || !ok) break;
      j -= 8;
      probe();
    }
    LB::store(status + (uint64_t)tile * RADIX + tid, ok ? (LB::INC | (SW)(excl + tcount)) : LB::POISON);
    return ok;
  };
  // Each warp's first slot of the digit in the tile-sorted order.
  auto first_slots = [&]() {
    uint32_t run = tstart;
#pragma unroll 4
    for (int w = 0; w < WARPS; ++w) {
      const uint32_t c = s_cnt[w * RADIX + tid];
      s_cnt[w * RADIX + tid] = run;
      run += c;
    }
  };
  // The first probe's loads are in flight while the tile-local order is
  // written (and the predecessors have had that long to publish as well).
  if (tid < RADIX) {
    if (!hooked && tile > 0) probe();
    first_slots();
  }
  __syncthreads();
  // Tile-sorted order: slot (the warp's first slot of the digit + rank)
  // holds the key at this position.
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    const uint32_t pos = warp * WK + i * 32 + lane;
    s_perm[wc[digit8<BYTE>(s_keys[pos], shift, mask, bsel)] + rank[i]] = (uint16_t)pos;
  }
  if (tid < RADIX) {
    if (hooked) s_abort = 1;
    else if (tile > 0 && !resolve()) s_abort = 1;
    // global position of tile-sorted slot p of this digit = s_goff[d] + p
    s_goff[tid] = ghist + excl - tstart;
  }
  if constexpr (C::HAS_V)
    if (bulk && !mbar_wait(&bars[1], 0, mbar_budget_of(a.budget))) s_abort = 1;
  __syncthreads();  // order complete; payload tile landed (s_abort visible)
  if (s_abort) {
    leave();
    return;
  }

  // ---- scatter: slot p of the tile-sorted order goes to s_goff[digit] + p;
  // a digit's slots are consecutive, so each run leaves as coalesced stores.
  if (full) {
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const uint32_t p = j * THREADS + tid;
      const uint32_t src = s_perm[p];
      const K key = s_keys[src];
      const uint32_t g = s_goff[digit8<BYTE>(key, shift, mask, bsel)] + p;
      dst_k[g] = key;
      if constexpr (C::HAS_V) dst_v[g] = s_vals[src];
    }
  } else {
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
      const uint32_t p = j * THREADS + tid;
      if (p < tile_n) {
        const uint32_t src = s_perm[p];
        const K key = s_keys[src];
        const uint32_t g = s_goff[digit8<BYTE>(key, shift, mask, bsel)] + p;
        dst_k[g] = key;
        if constexpr (C::HAS_V) dst_v[g] = s_vals[src];
      }
    }
  }
}

// Copies the sorted result back into the caller's buffers when the number of
// executed passes was odd (the data then ended in the alternate buffers).
template <typename K, typename V>
__global__ void k_sort_final_copy(K *keys, const K *keys_alt, V *vals, const V *vals_alt, uint64_t n, int passes,
                                  const SortHeader *hdr) {
  if (hdr->sel[passes] == 0) return;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    keys[i] = keys_alt[i];
    if constexpr (sizeof(V) > 1) vals[i] = vals_alt[i];
  }
}

// Kernel of the 8-bit passes: 0 = k_sort_pass8 ranking by leader tables
// (default), 1 = the original k_sort_pass, 2-5 = k_sort_pass8 ranking by
// shared-memory OR words, match.any, plain votes, predicated votes; a test
// and measurement switch (sort.cu).
int gprtcu_sort_ranking();
// L2 prefetch distance of the 8-bit passes in quarters of a resident wave
// of CTAs (0: none; sort.cu).
int gprtcu_sort_prefetch();

template <typename K, typename V, int RB, int WARPS, int ITEMS>
gprtcuStatus sort_run(const SortArgs &a, cudaStream_t stream) {
  using C = PassCfg<K, V, RB, WARPS, ITEMS>;
  static_assert(C::SMEM <= 227 * 1024, "shared memory per CTA");
  K *keys = static_cast<K *>(a.keys);
  k_sort_hist<K, RB><<<a.sms * 4, 512, 0, stream>>>(keys, a.n, a.begin_bit, a.end_bit, a.passes, a.hist, a.trivial,
                                                    a.hdr);
  GPRTCU_TRY(cudaGetLastError());
  bool match = false;
  if constexpr (RB == 8) {
    using C8 = Pass8Cfg<K, V, WARPS, ITEMS, 0>;
    static_assert(Pass8Cfg<K, V, WARPS, ITEMS, 2>::SMEM <= 227 * 1024, "shared memory per CTA");
    static_assert(Pass8Cfg<K, V, WARPS, ITEMS, 0>::SMEM <= 227 * 1024, "shared memory per CTA");
    // more keys than 30-bit look-back values can count need the wide words,
    // which only the 8-bit kernel has
    const bool wide = a.n > (uint64_t)LB_VALUE;
    const int mode = gprtcu_sort_ranking();
    match = wide || mode != 1;
    if (match) {
      for (int p = 0; p < a.passes; ++p) {
        const int shift = a.begin_bit + p * RB;
        const int bits = a.end_bit - shift < RB ? a.end_bit - shift : RB;
        const bool byte = bits == 8 && (shift & 7) == 0;
        auto launch = [&](auto kernel, size_t smem) -> gprtcuStatus {
          GPRTCU_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
          SortArgs b = a;
          b.pf_tiles = (uint32_t)((uint64_t)gprtcu_sort_prefetch() * a.sms * C8::MIN_CTAS / 4);
          kernel<<<(unsigned)a.tiles, C8::THREADS, smem, stream>>>(b, p, shift, bits);
          GPRTCU_TRY(cudaGetLastError());
          return GPRTCU_OK;
        };
        // mode m runs RANK m (1 is the original pass, below); the wide
        // look-back words exist for the default ranking only
        auto go = [&](auto rank_tag) -> gprtcuStatus {
          constexpr int R = decltype(rank_tag)::value;
          constexpr size_t S = Pass8Cfg<K, V, WARPS, ITEMS, R>::SMEM;
          if constexpr (R == 0) {
            if (wide)
              return byte ? launch(k_sort_pass8<K, V, WARPS, ITEMS, true, true, 0>, S)
                          : launch(k_sort_pass8<K, V, WARPS, ITEMS, false, true, 0>, S);
          }
          return byte ? launch(k_sort_pass8<K, V, WARPS, ITEMS, true, false, R>, S)
                      : launch(k_sort_pass8<K, V, WARPS, ITEMS, false, false, R>, S);
        };
        gprtcuStatus st;
        if (wide || mode == 0) st = go(std::integral_constant<int, 0>());
        else if (mode == 2) st = go(std::integral_constant<int, 2>());
        else if (mode == 3) st = go(std::integral_constant<int, 3>());
        else if (mode == 4) st = go(std::integral_constant<int, 4>());
        else st = go(std::integral_constant<int, 5>());
        if (st != GPRTCU_OK) return st;
      }
    }
  }
  if (!match && a.n > (uint64_t)LB_VALUE) return GPRTCU_ERR_TOO_LARGE;
  if (!match) {
    GPRTCU_TRY(cudaFuncSetAttribute(k_sort_pass<K, V, RB, WARPS, ITEMS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)C::SMEM));
    for (int p = 0; p < a.passes; ++p) {
      const int shift = a.begin_bit + p * RB;
      const int bits = a.end_bit - shift < RB ? a.end_bit - shift : RB;
      k_sort_pass<K, V, RB, WARPS, ITEMS><<<(unsigned)a.tiles, C::THREADS, C::SMEM, stream>>>(a, p, shift, bits);
      GPRTCU_TRY(cudaGetLastError());
    }
  }
  k_sort_final_copy<K, V><<<a.sms * 4, 256, 0, stream>>>(keys, static_cast<const K *>(a.keys_alt),
                                                         static_cast<V *>(a.vals),
                                                         static_cast<const V *>(a.vals_alt), a.n, a.passes, a.hdr);
  GPRTCU_TRY(cudaGetLastError());
  return GPRTCU_OK;
}

template <typename K, typename V, size_t... I>
constexpr std::array<SortRunFn, sizeof...(I)> make_sort_table(std::index_sequence<I...>) {
  return {{&sort_run<K, V, kSortGrid[I].rb, kSortGrid[I].warps, kSortGrid[I].tile / (32 * kSortGrid[I].warps)>...}};
}

// One table per key/payload type pair (char = no payload), defined in the
// sort_*.cu files.
extern const std::array<SortRunFn, kSortGridSize> kSortTableK32;
extern const std::array<SortRunFn, kSortGridSize> kSortTableK32V32;
extern const std::array<SortRunFn, kSortGridSize> kSortTableK32V64;
extern const std::array<SortRunFn, kSortGridSize> kSortTableK64;
extern const std::array<SortRunFn, kSortGridSize> kSortTableK64V32;
extern const std::array<SortRunFn, kSortGridSize> kSortTableK64V64;

}  // namespace gprtcu
