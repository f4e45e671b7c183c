// scan.cu -- single-pass uint32 prefix sum with decoupled look-back.
//
// Replaces gprtBufferExclusiveSum (gprt/gprt_host.h:2246), whose host entry
// is a stub in the reference (gprt/gprt.cpp:8739-8743) and whose intended
// kernel is the chained scan of gprt/gprt_scan.slang:105-392.  Same single
// pass structure (tile ticket, tile aggregate, look-back over predecessors,
// inclusive publish), re-laid out for B200:
//   * 8192 elements per 256-thread tile, each warp owning 1024 contiguous
//     elements loaded as 8 coalesced 512-byte warp-wide 128-bit loads;
//   * 64-bit status words {flag:32 | value:32}, so the aggregate is not
//     capped at 2^30 as it is with the reference's 2-bit-flag packing
//     (gprt/gprt_scan.slang:60-63, gprt/gprt_host.h:2231);
//   * warp-wide look-back over 32 or 128 predecessors per probe, with a
//     bounded wait that poisons the chain instead of hanging;
//   * for large aligned inputs, a persistent warp-specialised kernel
//     (k_scan_reread) that publishes each tile's aggregate as soon as the
//     tile lands and reads the tile a second time, from L2, once its prefix
//     is known, so no tile holds shared memory while it waits.
// Traffic: 4 B read + 4 B written per element; HBM-bound.
#include "common.cuh"

namespace gprtcu {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_VECS = 8;                                  // uint4 per thread
constexpr int SCAN_WARP_ELEMS = SCAN_VECS * 4 * 32;           // 1024
constexpr int SCAN_TILE = SCAN_WARP_ELEMS * (SCAN_THREADS / 32);  // 8192

constexpr uint64_t ST_AGG = 1ull << 32;
constexpr uint64_t ST_INC = 2ull << 32;
constexpr uint64_t ST_POISON = 3ull << 32;

// Warp 0 of tile `tile` (>= 1) sums the aggregates of its predecessors back to
// the nearest inclusive prefix.  Returns false if the chain is poisoned or the
// wait budget ran out.
__device__ __forceinline__ bool scan_lookback(const uint64_t *status, uint64_t tile, int lane, uint32_t budget,
                                              uint32_t &excl_out) {
  uint32_t excl = 0;
  int64_t base = (int64_t)tile - 1;
  uint32_t spins = 0;
  while (true) {
    int64_t idx = base - lane;
    uint64_t s = idx >= 0 ? ld_relaxed_u64(&status[idx]) : ST_INC;
    // Wait only for the lanes up to the nearest inclusive (or poisoned)
    // predecessor: the ones beyond it are not needed.
    unsigned stopm;
    while (true) {
      unsigned ready = __ballot_sync(FULL_MASK, (s >> 32) != 0);
      stopm = __ballot_sync(FULL_MASK, (s >> 32) >= 2);
      unsigned need = stopm ? (2u << (__ffs(stopm) - 1)) - 1u : FULL_MASK;
      if ((ready & need) == need) break;
      if (++spins > budget) return false;
      if ((s >> 32) == 0) s = ld_relaxed_u64(&status[idx]);
    }
    int stop = stopm ? __ffs(stopm) - 1 : 31;
    uint32_t flag = (uint32_t)(s >> 32);
    if (__shfl_sync(FULL_MASK, flag, stop) == 3) return false;
    uint32_t v = lane <= stop ? (uint32_t)s : 0u;
    excl += warp_sum(v);
    if (stopm) break;
    base -= 32;
  }
  excl_out = excl;
  return true;
}

// Look-back over 128 predecessors per probe (4 status words per lane, lane
// l covering tiles base-4l .. base-4l-3, nearest first).  The inclusive
// prefix can only travel as fast as one probe window per L2 round trip, so a
// wide window keeps it ahead of the tile rate the HBM can feed.
__device__ __forceinline__ bool scan_lookback128(const uint64_t *status, uint64_t tile, int lane, uint32_t budget,
                                                 uint32_t &excl_out) {
  uint32_t excl = 0;
  int64_t base = (int64_t)tile - 1;
  uint32_t spins = 0;
  while (true) {
    uint64_t s[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int64_t idx = base - 4 * lane - c;
      s[c] = idx >= 0 ? ld_relaxed_u64(&status[idx]) : ST_INC;
    }
    unsigned stopm;
    int cstop;
    while (true) {
      cstop = 4;
#pragma unroll
      for (int c = 3; c >= 0; --c)
        if ((s[c] >> 32) >= 2) cstop = c;
      stopm = __ballot_sync(FULL_MASK, cstop < 4);
      const int stop_lane = stopm ? __ffs(stopm) - 1 : 32;
      const int need = lane < stop_lane ? 4 : (lane == stop_lane ? cstop + 1 : 0);
      bool ready = true;
#pragma unroll
      for (int c = 0; c < 4; ++c)
        if (c < need && (s[c] >> 32) == 0) ready = false;
      if (__all_sync(FULL_MASK, ready)) break;
      if (++spins > budget) return false;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int64_t idx = base - 4 * lane - c;
        if (c < need && (s[c] >> 32) == 0) s[c] = ld_relaxed_u64(&status[idx]);
      }
    }
    const int stop_lane = stopm ? __ffs(stopm) - 1 : 32;
    const int use = lane < stop_lane ? 4 : (lane == stop_lane ? cstop + 1 : 0);
    uint32_t v = 0;
    bool poison = false;
#pragma unroll
    for (int c = 0; c < 4; ++c)
      if (c < use) {
        v += (uint32_t)s[c];
        poison |= (s[c] >> 32) == 3;
      }
    if (__any_sync(FULL_MASK, poison)) return false;
    excl += warp_sum(v);
    if (stopm) break;
    base -= 128;
  }
  excl_out = excl;
  return true;
}

// Register-staged tile per CTA.  MODE: 0 exclusive, 1 inclusive.  VEC:
// input/output 16-byte aligned.  NC: input does not alias output (read
// through the non-coherent path).  THREADS x VECS uint4 per tile; LBW is the
// look-back window (32 or 128 predecessors per probe).
template <int MODE, bool VEC, bool NC, int THREADS, int VECS, int LBW>
__global__ void __launch_bounds__(THREADS) k_scan_u32(const uint32_t *__restrict__ in, uint32_t *out, uint64_t n,
                                                          uint64_t num_tiles, ScratchHeader *hdr, uint64_t *status,
                                                          uint32_t *d_total, uint32_t budget, int64_t skip_tile) {
  constexpr int WARP_ELEMS = VECS * 4 * 32;
  constexpr int TILE = WARP_ELEMS * (THREADS / 32);
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_warp[THREADS / 32];
  __shared__ uint32_t s_prefix;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_tile = atomicAdd(&hdr->ticket[0], 1u);
  __syncthreads();
  const uint64_t tile = s_tile;
  const uint64_t warp_start = tile * TILE + (uint64_t)warp * WARP_ELEMS;
  const bool full = VEC && (tile + 1) * TILE <= n;

  uint4 v[VECS];
  if (full) {
    const uint4 *src = reinterpret_cast<const uint4 *>(in + warp_start);
#pragma unroll
    for (int j = 0; j < VECS; ++j) v[j] = NC ? ldg_stream(src + j * 32 + lane) : ldg_coherent(src + j * 32 + lane);
  } else {
#pragma unroll
    for (int j = 0; j < VECS; ++j) {
      uint64_t e = warp_start + (uint64_t)(j * 32 + lane) * 4;
      v[j].x = e + 0 < n ? in[e + 0] : 0u;
      v[j].y = e + 1 < n ? in[e + 1] : 0u;
      v[j].z = e + 2 < n ? in[e + 2] : 0u;
      v[j].w = e + 3 < n ? in[e + 3] : 0u;
    }
  }

  // Position order inside a warp is (j, lane, component): scan each 128-
  // element row j across lanes and carry row totals forward.
  uint32_t pre[VECS];
  uint32_t carry = 0;
#pragma unroll
  for (int j = 0; j < VECS; ++j) {
    uint32_t s = v[j].x + v[j].y + v[j].z + v[j].w;
    uint32_t inc = warp_incl_scan(s, lane);
    pre[j] = carry + inc - s;
    carry += __shfl_sync(FULL_MASK, inc, 31);
  }
  if (lane == 0) s_warp[warp] = carry;
  __syncthreads();

  if (warp == 0) {
    uint32_t wt = lane < THREADS / 32 ? s_warp[lane] : 0u;
    uint32_t wi = warp_incl_scan(wt, lane);
    uint32_t agg = __shfl_sync(FULL_MASK, wi, THREADS / 32 - 1);
    if (lane < THREADS / 32) s_warp[lane] = wi - wt;
    uint32_t excl = 0;
    bool ok = true;
    if ((int64_t)tile == skip_tile) {
      // Fault injection for tests: this tile never publishes.
      ok = false;
    } else if (tile == 0) {
      if (lane == 0) st_relaxed_u64(&status[0], ST_INC | agg);
    } else {
      if (lane == 0) st_relaxed_u64(&status[tile], ST_AGG | agg);
      ok = LBW == 128 ? scan_lookback128(status, tile, lane, budget, excl)
                      : scan_lookback(status, tile, lane, budget, excl);
      if (lane == 0) st_relaxed_u64(&status[tile], ok ? (ST_INC | (uint32_t)(excl + agg)) : ST_POISON);
    }
    if (!ok && lane == 0) record_error(hdr, GPRTCU_ERR_TIMEOUT);
    if (lane == 0) {
      s_prefix = excl;
      if (tile == num_tiles - 1) {
        hdr->total = excl + agg;
        if (d_total) *d_total = excl + agg;
      }
    }
  }
  __syncthreads();

  const uint32_t base = s_prefix + s_warp[warp];
#pragma unroll
  for (int j = 0; j < VECS; ++j) {
    uint32_t p = base + pre[j];
    uint4 o;
    if (MODE == 0) {
      o.x = p;
      o.y = o.x + v[j].x;
      o.z = o.y + v[j].y;
      o.w = o.z + v[j].z;
    } else {
      o.x = p + v[j].x;
      o.y = o.x + v[j].y;
      o.z = o.y + v[j].z;
      o.w = o.z + v[j].w;
    }
    if (full) {
      stg_v4(reinterpret_cast<uint4 *>(out + warp_start) + j * 32 + lane, o);
    } else {
      uint64_t e = warp_start + (uint64_t)(j * 32 + lane) * 4;
      if (e + 0 < n) out[e + 0] = o.x;
      if (e + 1 < n) out[e + 1] = o.y;
      if (e + 2 < n) out[e + 2] = o.z;
      if (e + 3 < n) out[e + 3] = o.w;
    }
  }
}


// Tile-per-CTA scan with TMA staging (16-byte aligned in/out).  A 128-thread
// CTA owns one 8192-element tile: thread 0 takes a ticket and brings the
// whole 32 KB tile into shared memory with one bulk async copy; the four warps
// reduce it (row sums), publish the tile aggregate, warp 0 looks back, then
// the warps scan the tile row by row in shared memory and thread 0 writes it
// out with one bulk async store.  32 KB of shared memory and few registers
// per CTA let seven CTAs share an SM, so many tiles' loads are in flight while
// other tiles wait on their look-back.
constexpr int TS_THREADS = 128;
constexpr int TS_ROWS = 16;  // rows of 128 elements per warp
constexpr size_t TS_SMEM = (size_t)SCAN_TILE * 4;

// WARPS x 16 rows x 128 elements per tile.  TICKET: tile order from an atomic
// ticket (dispatch-order independent) or from blockIdx.x.
template <int MODE, int WARPS = 4, bool TICKET = true>
__global__ void __launch_bounds__(WARPS * 32) k_scan_tma(const uint32_t *in, uint32_t *out, uint64_t n,
                                                        uint64_t num_tiles, ScratchHeader *hdr, uint64_t *status,
                                                        uint32_t *d_total, uint32_t budget, int64_t skip_tile) {
  constexpr int THREADS = WARPS * 32;
  constexpr int TILE = WARPS * TS_ROWS * 128;
  constexpr uint32_t TILE_BYTES = TILE * 4;
  extern __shared__ __align__(128) unsigned char smem[];
  uint4 *buf = reinterpret_cast<uint4 *>(smem);
  __shared__ uint64_t bar;
  __shared__ uint32_t s_tile, s_abort, s_prefix;
  __shared__ uint32_t s_warp[WARPS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    s_tile = TICKET ? atomicAdd(&hdr->ticket[0], 1u) : blockIdx.x;
    s_abort = 0;
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  const uint64_t tile = s_tile;
  const uint64_t tile_start = tile * TILE;
  const bool full = tile_start + TILE <= n;
  if (full) {
    if (tid == 0) {
      mbar_arrive_expect_tx(&bar, TILE_BYTES);
      bulk_g2s(buf, in + tile_start, TILE_BYTES, &bar);
    }
    if (!mbar_wait(&bar, 0, mbar_budget_of(budget))) s_abort = 1;
  } else {
    uint32_t *sb = reinterpret_cast<uint32_t *>(buf);
    for (int i = tid; i < TILE; i += THREADS) sb[i] = tile_start + i < n ? in[tile_start + i] : 0u;
  }
  __syncthreads();
  if (s_abort) {
    if (tid == 0) {
      record_error(hdr, GPRTCU_ERR_TIMEOUT);
      // the copy must land before this CTA's shared memory is released
      mbar_wait(&bar, 0, mbar_budget_of(budget));
    }
    return;
  }
  // Warp w owns rows [w*TS_ROWS, (w+1)*TS_ROWS); row r is 32 lanes x uint4.
  uint4 *wb = buf + warp * TS_ROWS * 32;
  uint32_t part = 0;
#pragma unroll
  for (int r = 0; r < TS_ROWS; ++r) {
    const uint4 v = wb[r * 32 + lane];
    part += v.x + v.y + v.z + v.w;
  }
  part = warp_sum(part);
  if (lane == 0) s_warp[warp] = part;
  __syncthreads();
  if (warp == 0) {
    const uint32_t wt = lane < WARPS ? s_warp[lane] : 0u;
    const uint32_t wi = warp_incl_scan(wt, lane);
    const uint32_t agg = __shfl_sync(FULL_MASK, wi, WARPS - 1);
    if (lane < WARPS) s_warp[lane] = wi - wt;
    uint32_t excl = 0;
    bool ok = true;
    if ((int64_t)tile == skip_tile) {
      ok = false;  // fault injection: this tile never publishes
    } else if (tile == 0) {
      if (lane == 0) st_relaxed_u64(&status[0], ST_INC | agg);
    } else {
      if (lane == 0) st_relaxed_u64(&status[tile], ST_AGG | agg);
      ok = scan_lookback128(status, tile, lane, budget, excl);
      if (lane == 0) st_relaxed_u64(&status[tile], ok ? (ST_INC | (uint32_t)(excl + agg)) : ST_POISON);
    }
    if (!ok && lane == 0) record_error(hdr, GPRTCU_ERR_TIMEOUT);
    if (lane == 0) {
      s_prefix = excl;
      if (tile == num_tiles - 1) {
        hdr->total = excl + agg;
        if (d_total) *d_total = excl + agg;
      }
    }
  }
  __syncthreads();
  uint32_t carry = s_prefix + s_warp[warp];
#pragma unroll 4
  for (int r = 0; r < TS_ROWS; ++r) {
    const uint4 v = wb[r * 32 + lane];
    const uint32_t sum = v.x + v.y + v.z + v.w;
    const uint32_t inc = warp_incl_scan(sum, lane);
    const uint32_t p = carry + inc - sum;
    uint4 o;
    if (MODE == 0) {
      o.x = p;
      o.y = o.x + v.x;
      o.z = o.y + v.y;
      o.w = o.z + v.z;
    } else {
      o.x = p + v.x;
      o.y = o.x + v.y;
      o.z = o.y + v.z;
      o.w = o.z + v.w;
    }
    wb[r * 32 + lane] = o;
    carry += __shfl_sync(FULL_MASK, inc, 31);
  }
  if (full) {
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      bulk_s2g(out + tile_start, buf, TILE_BYTES);
      bulk_commit();
      bulk_wait_read<0>();  // shared memory must stay valid until the store has read it
    }
  } else {
    __syncthreads();
    const uint32_t *sb = reinterpret_cast<const uint32_t *>(buf);
    for (int i = tid; i < TILE; i += THREADS)
      if (tile_start + i < n) out[tile_start + i] = sb[i];
  }
}

// Persistent scan that reads each tile twice: once from HBM to publish its
// aggregate, once more (from L2) after its look-back has resolved.
//
// In the tile-per-CTA kernels a tile holds its 32 KB of shared memory from
// the moment its load is issued until its store has read it, and most of that
// time is look-back: the tile waits for the slowest load among its
// predecessors, and HBM load latency has a long tail under full load (B200,
// 2^30 elements: median 3 us, p99 9 us; look-back 8 us of a 14 us tile life).
// Shared memory per SM then caps the loads in flight below what the HBM
// needs.  Here a tile holds no shared memory while it waits:
//   warp 0   producer: takes a ticket and loads the tile into one of RS
//            "reduce" stages (bulk copy, L2 evict_last);
//   warp 1   reducer: sums the tile (one partial per scanner warp), frees the
//            stage, publishes the aggregate at once, and queues {tile,
//            partials} in one of PQ pending slots;
//   warps 2,3 look-back (even / odd pending slots): resolve the tile's
//            exclusive prefix, publish the inclusive value, then load the
//            tile again into one of SS "scan" stages (L2 evict_first) — it
//            was read microseconds ago and is still in L2;
//   warps 4..11 scanners: eight rows of 128 elements each, scanned with all
//            eight rows' shuffles interleaved, then one bulk store (L2
//            evict_first).
// HBM traffic stays 4 B read + 4 B written per element; the second read is
// L2 traffic.  Stages hand over through mbarriers: r_full/r_empty (producer
// <-> reducer), p_full/p_empty (reducer -> look-back -> scanners -> reducer),
// s_full/s_empty (look-back <-> scanners).  Progress: a tile's aggregate is
// published before its reducer can block, and every wait is on an earlier
// iteration of this CTA or on a smaller ticket, so the smallest unfinished
// tile can always advance.  Every wait is bounded; a wait that gives up
// records GPRTCU_ERR_TIMEOUT and the warp leaves its loop.
constexpr int RR_SCAN_WARPS = 8;
constexpr int RR_THREADS = (4 + RR_SCAN_WARPS) * 32;
constexpr int RR_RS = 3, RR_SS = 4, RR_PQ = 8;
// A scan stage has 64 bytes of slack past its tile: a partition stages its
// two runs shifted so that each run's shared-memory and global addresses
// agree modulo 16 bytes.
constexpr uint32_t RR_STAGE_BYTES = SCAN_TILE * 4 + 64;
constexpr size_t RR_SMEM = (size_t)RR_RS * SCAN_TILE * 4 + (size_t)RR_SS * RR_STAGE_BYTES;
constexpr uint32_t RR_END = 0xFFFFFFFFu;
struct RrPending {
  uint32_t tile, prefix, part[RR_SCAN_WARPS];
};

// MODE: 0 exclusive sum, 1 inclusive sum, 2 partition, 3 select (by the
// sign bit: want_neg selects negatives).  For 2 and 3 the tile aggregates
// are selected counts, d_total receives the total selected count, and the
// scanner warps stage each tile's selected items in order at the bottom of
// its scan stage and, for a partition, its unselected items in reverse order
// at the top, then write both groups out as runs: the 16-byte aligned middle
// of each run by one bulk copy (shared to global), the ragged ends by threads
// (the dispatch requires a 16-byte aligned output).  Bulk copies instead of
// the threads' 16-byte stores took 2^30 items from 1.85 to 1.70 ms
// (partition) and from 1.43 to 1.36 ms (select): the scanners, the pipeline's
// slowest stage, no longer copy the runs.  Taking each tile's rows, flags and
// row-count scan before the scanners' stage barrier, which then also stands
// for "every scanner holds its rows" (one named barrier fewer per tile):
// 1.70 -> 1.57 ms (partition), 1.36 -> 1.29 ms (select).
template <int MODE>
__global__ void __launch_bounds__(RR_THREADS, 1) k_scan_reread(const uint32_t *in, uint32_t *out, uint64_t n,
                                                               uint64_t ntiles, ScratchHeader *hdr, uint64_t *status,
                                                               uint32_t *d_total, uint32_t budget, int64_t skip_tile,
                                                               uint32_t want_neg, int64_t skip_stage) {
  constexpr int RS = RR_RS, SS = RR_SS, PQ = RR_PQ, SW = RR_SCAN_WARPS;
  constexpr uint32_t TILE = SCAN_TILE, TB = SCAN_TILE * 4;
  static_assert(PQ % 2 == 0, "pending slot q always belongs to look-back warp q % 2");
  static_assert(SS >= 3, "a scan stage is released one iteration late; the end marker needs two more");
  static_assert(TILE == SW * 8 * 128, "each scanner warp owns 8 rows of 128 elements");
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t r_full[RS], r_empty[RS], p_full[PQ], p_empty[PQ], s_full[SS], s_empty[SS];
  __shared__ RrPending pend[PQ];
  __shared__ uint32_t r_tile[RS], s_tile[SS];
  __shared__ volatile uint32_t s_scan_stop;  // a scanner's wait gave up: all scanners leave together
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t mb = mbar_budget_of(budget);
  unsigned char *rbuf = smem, *sbuf = smem + (size_t)RS * TB;
  if (tid == 0) {
    s_scan_stop = 0;
    for (int i = 0; i < RS; ++i) {
      mbar_init(&r_full[i], 32);
      mbar_init(&r_empty[i], 1);
    }
    for (int i = 0; i < PQ; ++i) {
      mbar_init(&p_full[i], 1);
      mbar_init(&p_empty[i], 1);
    }
    for (int i = 0; i < SS; ++i) {
      mbar_init(&s_full[i], 32);
      mbar_init(&s_empty[i], 1);
    }
    fence_mbar_init();
  }
  __syncthreads();
  // Bring tile t into a stage: bulk copy of its whole-uint4 part, plain loads
  // and zeros for the rest of a partial last tile.  All 32 lanes arrive.
  auto load_tile = [&](uint32_t *sb, uint32_t t, uint64_t *bar, uint64_t pol) {
    const uint64_t base = (uint64_t)t * TILE;
    const uint64_t r = n - base < (uint64_t)TILE ? n - base : (uint64_t)TILE;
    const uint32_t a = (uint32_t)(r & ~3ull);
    if (r < (uint64_t)TILE)
      for (uint32_t k = a + lane; k < TILE; k += 32) sb[k] = k < r ? in[base + k] : 0u;
    if (lane == 0 && a) {
      mbar_arrive_expect_tx(bar, a * 4);
      bulk_g2s_hint(sb, in + base, a * 4, bar, pol);
    } else {
      mbar_arrive(bar);
    }
  };
  if (warp == 0) {
    const uint64_t pol = l2_policy_evict_last();
    uint32_t i = 0;
    for (;; ++i) {
      const int s = i % RS;
      if (i >= RS && !mbar_wait(&r_empty[s], ((i / RS) - 1) & 1, mb)) break;
      uint32_t t = 0;
      if (lane == 0) t = atomicAdd(&hdr->ticket[0], 1u);
      t = __shfl_sync(FULL_MASK, t, 0);
      if (lane == 0) r_tile[s] = t < ntiles ? t : RR_END;
      if (t >= ntiles) {
        mbar_arrive(&r_full[s]);
        return;
      }
      load_tile(reinterpret_cast<uint32_t *>(rbuf + (size_t)s * TB), t, &r_full[s], pol);
    }
    // A wait gave up: the copies of the last RS iterations may still be in
    // flight and must land before the CTA's shared memory is released.  Only
    // this warp's own copies advance r_full, so each wait ends as soon as its
    // copy has landed (or at once, if the stage was consumed already).
    for (uint32_t j = i > (uint32_t)RS ? i - RS : 0u; j < i; ++j) mbar_wait(&r_full[j % RS], (j / RS) & 1, mb);
  } else if (warp == 1) {
    for (uint32_t i = 0;; ++i) {
      const int s = i % RS, q = i % PQ;
      if (!mbar_wait(&r_full[s], (i / RS) & 1, mb)) break;
      const uint32_t t = r_tile[s];
      if (t == RR_END) {
        for (uint32_t j = i; j < i + 2; ++j) {  // one end marker for each look-back warp
          const int qj = j % PQ;
          if (j >= PQ && !mbar_wait(&p_empty[qj], ((j / PQ) - 1) & 1, mb)) {
            if (lane == 0) record_error(hdr, GPRTCU_ERR_TIMEOUT);
            return;
          }
          if (lane == 0) {
            pend[qj].tile = RR_END;
            mbar_arrive(&p_full[qj]);
          }
        }
        return;
      }
      const uint4 *b = reinterpret_cast<const uint4 *>(rbuf + (size_t)s * TB);
      uint32_t part[SW];
      // elements of the tile (a partial last tile is zero-filled past them)
      const uint32_t tc = n - (uint64_t)t * TILE < (uint64_t)TILE ? (uint32_t)(n - (uint64_t)t * TILE) : TILE;
#pragma unroll
      for (int w = 0; w < SW; ++w) {
        uint32_t p = 0;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          const uint4 v = b[(w * 8 + r) * 32 + lane];
          if (MODE < 2)
            p += (v.x + v.y) + (v.z + v.w);
          else  // negatives; the zero fill past a partial tile counts as none
            p += ((v.x >> 31) + (v.y >> 31)) + ((v.z >> 31) + (v.w >> 31));
        }
        part[w] = p;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int w = 0; w < SW; ++w) part[w] += __shfl_xor_sync(FULL_MASK, part[w], o);
      if (MODE >= 2 && !want_neg) {  // non-negatives among each scanner's valid items
#pragma unroll
        for (int w = 0; w < SW; ++w) {
          const uint32_t lo = (uint32_t)w * 1024u;
          part[w] = (tc > lo ? (tc - lo < 1024u ? tc - lo : 1024u) : 0u) - part[w];
        }
      }
      __syncwarp();
      uint32_t agg = 0;
#pragma unroll
      for (int w = 0; w < SW; ++w) agg += part[w];
      if (lane == 0) {
        mbar_arrive(&r_empty[s]);
        if ((int64_t)t != skip_tile) st_relaxed_u64(&status[t], (t == 0 ? ST_INC : ST_AGG) | agg);
      }
      if (i >= PQ && !mbar_wait(&p_empty[q], ((i / PQ) - 1) & 1, mb)) break;
      if (lane == 0) {
        pend[q].tile = t;
#pragma unroll
        for (int w = 0; w < SW; ++w) pend[q].part[w] = part[w];
        mbar_arrive(&p_full[q]);
      }
    }
  } else if (warp < 4) {
    const uint64_t pol = l2_policy_evict_first();
    uint32_t i = warp - 2;
    bool hooked = false;
    for (;; i += 2) {
      const int q = i % PQ, ss = i % SS;
      if (!mbar_wait(&p_full[q], (i / PQ) & 1, mb)) break;
      const uint32_t t = pend[q].tile;
      uint32_t excl = 0;
      if (t != RR_END) {
        uint32_t agg = 0;
#pragma unroll
        for (int w = 0; w < SW; ++w) agg += pend[q].part[w];
        bool ok = true;
        if ((int64_t)t == skip_tile) {
          ok = false;  // fault injection: this tile never publishes
        } else if (t > 0) {
          ok = scan_lookback128(status, t, lane, budget, excl);
          if (lane == 0) st_relaxed_u64(&status[t], ok ? (ST_INC | (uint32_t)(excl + agg)) : ST_POISON);
        }
        if (!ok && lane == 0) record_error(hdr, GPRTCU_ERR_TIMEOUT);
        if (lane == 0 && t == ntiles - 1) {
          hdr->total = excl + agg;
          if (d_total) *d_total = excl + agg;
        }
      }
      if (t != RR_END && (int64_t)t == skip_stage) {
        // Fault injection for tests: the tile's prefix is published, but its
        // scan stage is never filled, so the scanners' wait on it runs out.
        hooked = true;
        break;
      }
      if (i >= SS && !mbar_wait(&s_empty[ss], ((i / SS) - 1) & 1, mb)) break;
      if (lane == 0) {
        s_tile[ss] = t;
        if (t != RR_END) pend[q].prefix = excl;
      }
      if (t == RR_END) {
        mbar_arrive(&s_full[ss]);
        return;
      }
      load_tile(reinterpret_cast<uint32_t *>(sbuf + (size_t)ss * RR_STAGE_BYTES), t, &s_full[ss], pol);
    }
    // As for the producer: this warp's own copies into its scan stages (its
    // iterations i-2 and i-4) land before the warp leaves.
    for (uint32_t back = 2; back <= 4; back += 2)
      if (i >= back) mbar_wait(&s_full[(i - back) % SS], ((i - back) / SS) & 1, mb);
    if (hooked) return;
  } else {
    const int w = warp - 4;
    const bool leader = tid == 4 * 32;
    const uint64_t pol = l2_policy_evict_first();
    int prev = -1;
    for (uint32_t i = 0;; ++i) {
      const int ss = i % SS, q = i % PQ;
      // The scanners meet at named barriers, so none may leave on its own:
      // a warp whose wait gave up raises the flag, and after this barrier
      // all of them see the same flag and the same stage.
      if (!mbar_wait(&s_full[ss], (i / SS) & 1, mb)) s_scan_stop = 1;
      // Partition / select: each scanner takes its rows, their selection
      // flags and the warp's scan of the rows' counts before the barrier
      // (the stage's tile, prefix and per-warp counts are visible once its
      // wait has succeeded), so the barrier also means that every scanner
      // holds its rows and the stage may be overwritten by the staging
      // below; no second barrier before it.  (A warp whose wait gave up
      // computes from stale words here, which nothing uses: it leaves with
      // the others after the barrier.)
      uint4 rows[8];
      uint32_t fl[8], pk[2] = {0u, 0u}, own[2] = {0u, 0u}, rowtot[2] = {0u, 0u};
      uint32_t excl = 0, tsel = 0, rowbase = 0, tc = 0;
      if constexpr (MODE >= 2) {
        const uint32_t tt = s_tile[ss];
        excl = pend[q].prefix;
#pragma unroll
        for (int k = 0; k < SW; ++k) {
          const uint32_t pc = pend[q].part[k];
          rowbase += k < w ? pc : 0u;
          tsel += pc;
        }
        const uint64_t tb = (uint64_t)tt * TILE;
        tc = tt == RR_END ? 0u : (n - tb < (uint64_t)TILE ? (uint32_t)(n - tb) : TILE);
        const uint4 *wb = reinterpret_cast<const uint4 *>(sbuf + (size_t)ss * RR_STAGE_BYTES) + w * 8 * 32;
        const uint32_t flip = want_neg ? 0u : 15u;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          rows[r] = wb[r * 32 + lane];
          const uint32_t l0 = (uint32_t)((w * 8 + r) * 128 + lane * 4);
          const uint32_t rem = tc > l0 ? tc - l0 : 0u;
          const uint32_t valid = rem >= 4 ? 15u : (1u << rem) - 1u;
          fl[r] = (((rows[r].x >> 31) | ((rows[r].y >> 31) << 1) | ((rows[r].z >> 31) << 2) |
                    ((rows[r].w >> 31) << 3)) ^ flip) & valid;
          pk[r >> 2] |= (uint32_t)__popc(fl[r]) << (8 * (r & 3));
        }
        // Inclusive warp scan of the rows' counts, four rows to a word (a
        // row's total is at most 128, so a byte holds it).
        own[0] = pk[0];
        own[1] = pk[1];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const uint32_t y = __shfl_up_sync(FULL_MASK, pk[h], o);
            if (lane >= o) pk[h] += y;
          }
        rowtot[0] = __shfl_sync(FULL_MASK, pk[0], 31);
        rowtot[1] = __shfl_sync(FULL_MASK, pk[1], 31);
      }
      // Sums: the rows, their sums and the warp scans of the sums likewise
      // come before the barrier; after it only the carry is added.
      uint32_t sum[8], inc[8];
      if constexpr (MODE < 2) {
        const uint4 *wb = reinterpret_cast<const uint4 *>(sbuf + (size_t)ss * RR_STAGE_BYTES) + w * 8 * 32;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          rows[r] = wb[r * 32 + lane];
          sum[r] = (rows[r].x + rows[r].y) + (rows[r].z + rows[r].w);
          inc[r] = sum[r];
        }
#pragma unroll
        for (int o = 1; o < 32; o <<= 1)
#pragma unroll
          for (int r = 0; r < 8; ++r) {
            const uint32_t y = __shfl_up_sync(FULL_MASK, inc[r], o);
            if (lane >= o) inc[r] += y;
          }
      }
      named_bar_sync(1, SW * 32);
      if (s_scan_stop) {
        if (leader) record_error(hdr, GPRTCU_ERR_TIMEOUT);
        break;
      }
      const uint32_t t = s_tile[ss];
      if (t == RR_END) break;
      if constexpr (MODE >= 2) {
        const uint64_t base = (uint64_t)t * TILE;
        uint32_t *sb = reinterpret_cast<uint32_t *>(sbuf + (size_t)ss * RR_STAGE_BYTES);
        // Selected rank ls goes to out[excl + ls], unselected rank lu to
        // out[top - lu].  Staged at sb[s1 + ls] and sb[u_top - lu], with the
        // shifts chosen so that shared and global indices agree modulo 4:
        // both runs then leave as 16-byte stores between ragged ends.
        const uint32_t tunsel = tc - tsel;
        const uint64_t top = (n - 1) - (base - excl);
        const uint32_t s1 = (uint32_t)(excl & 3);
        const uint32_t u_top = TILE + 7 + (uint32_t)((top - (TILE + 7)) & 3);  // <= TILE + 10; u_top == top mod 4
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          const uint32_t sh = 8 * (r & 3);
          // selected items of the tile before this lane's first in row r
          uint32_t ls = rowbase + ((pk[r >> 2] - own[r >> 2]) >> sh & 0xFFu);
          const uint32_t l0 = (uint32_t)((w * 8 + r) * 128 + lane * 4);
          const uint32_t vals[4] = {rows[r].x, rows[r].y, rows[r].z, rows[r].w};
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            const uint32_t sel = (fl[r] >> c) & 1u;
            if (MODE == 2) {
              // unselected rank is (l0 + c) - ls
              const uint32_t at = sel ? s1 + ls : u_top - (l0 + c) + ls;
              if (l0 + c < tc) sb[at] = vals[c];
            } else if (sel) {
              sb[s1 + ls] = vals[c];
            }
            ls += sel;
          }
          rowbase += rowtot[r >> 2] >> sh & 0xFFu;
        }
        fence_proxy_async_smem();
        named_bar_sync(1, SW * 32);
        const uint32_t ct = (uint32_t)(tid - 4 * 32);
        // one run: `cnt` words from sb[sidx] to out[gidx], sidx == gidx mod 4:
        // the ragged ends by threads, the 16-byte aligned middle by one bulk
        // copy that the leader issues
        auto write_run = [&](uint32_t sidx, uint64_t gidx, uint32_t cnt) {
          const uint32_t h4 = (uint32_t)((4 - (gidx & 3)) & 3);
          const uint32_t head = h4 < cnt ? h4 : cnt;
          const uint32_t mid = (cnt - head) & ~3u;
          const uint32_t tail = cnt - head - mid;
          if (ct < head) out[gidx + ct] = sb[sidx + ct];
          if (ct < tail) out[gidx + head + mid + ct] = sb[sidx + head + mid + ct];
          if (leader && mid) bulk_s2g_hint(out + gidx + head, sb + sidx + head, mid * 4, pol);
        };
        write_run(s1, excl, tsel);
        if (MODE == 2 && tunsel) write_run(u_top - (tunsel - 1), top - (tunsel - 1), tunsel);
        if (leader) {
          mbar_arrive(&p_empty[q]);
          bulk_commit();
          bulk_wait_read<1>();  // the previous tile's copies have read their stage
          if (prev >= 0) mbar_arrive(&s_empty[prev]);
        }
        prev = ss;
        continue;
      }
      uint32_t carry = pend[q].prefix;
      for (int k = 0; k < w; ++k) carry += pend[q].part[k];
      uint4 *wb = reinterpret_cast<uint4 *>(sbuf + (size_t)ss * RR_STAGE_BYTES) + w * 8 * 32;
      const uint4 *v = rows;
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const uint32_t p = carry + inc[r] - sum[r];
        uint4 o;
        if (MODE == 0) {
          o.x = p;
          o.y = o.x + v[r].x;
          o.z = o.y + v[r].y;
          o.w = o.z + v[r].z;
        } else {
          o.x = p + v[r].x;
          o.y = o.x + v[r].y;
          o.z = o.y + v[r].z;
          o.w = o.z + v[r].w;
        }
        wb[r * 32 + lane] = o;
        carry += __shfl_sync(FULL_MASK, inc[r], 31);
      }
      fence_proxy_async_smem();
      named_bar_sync(1, SW * 32);
      const uint64_t base = (uint64_t)t * TILE;
      const uint64_t r = n - base < (uint64_t)TILE ? n - base : (uint64_t)TILE;
      const uint32_t a = (uint32_t)(r & ~3ull);
      const uint32_t *sb = reinterpret_cast<const uint32_t *>(sbuf + (size_t)ss * RR_STAGE_BYTES);
      if (r < (uint64_t)TILE) {
        for (uint32_t k = a + (tid - 4 * 32); k < r; k += SW * 32) out[base + k] = sb[k];
        named_bar_sync(1, SW * 32);
      }
      if (leader) {
        mbar_arrive(&p_empty[q]);
        if (a) bulk_s2g_hint(out + base, sb, a * 4, pol);
        bulk_commit();
        bulk_wait_read<1>();  // the previous tile's store has read its stage
        if (prev >= 0) mbar_arrive(&s_empty[prev]);
      }
      prev = ss;
    }
    if (leader) bulk_wait<0>();
    return;
  }
  if (lane == 0) record_error(hdr, GPRTCU_ERR_TIMEOUT);  // a wait above gave up
}


// Partition / select by sign (gprt/gprt_scan.slang:118-133,270-283;
// known-answer layout tests/t03-bufferScans/hostCode.cpp:98-160,172-241).
// The scan runs over the 0/1 selection flags; each tile then stages its
// selected items (in order) at the bottom of a shared buffer and, for a
// partition, its unselected items (in reverse order) at the top, so both
// groups leave the tile as contiguous, coalesced runs:
//   selected   : out[excl + k]
//   unselected : out[(n-1) - (tile_start - excl) - k']   (reverse order)
template <bool PARTITION, bool VEC>
__global__ void __launch_bounds__(SCAN_THREADS) k_partition_i32(const int32_t *__restrict__ in, int32_t *__restrict__ out,
                                                               uint64_t n, uint64_t num_tiles, int select_positive,
                                                               ScratchHeader *hdr, uint64_t *status, uint32_t *d_count,
                                                               uint32_t budget) {
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_warp[SCAN_THREADS / 32];
  __shared__ uint32_t s_prefix, s_tile_sel;
  __shared__ int32_t s_buf[SCAN_TILE];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_tile = atomicAdd(&hdr->ticket[0], 1u);
  __syncthreads();
  const uint64_t tile = s_tile;
  const uint64_t tile_start = tile * SCAN_TILE;
  const uint64_t warp_start = tile_start + (uint64_t)warp * SCAN_WARP_ELEMS;
  const bool full = VEC && (tile + 1) * SCAN_TILE <= n;
  const uint32_t tile_count = (uint32_t)min((uint64_t)SCAN_TILE, n - tile_start);
  const uint32_t want_neg = select_positive ? 0u : 1u;

  int4 v[SCAN_VECS];
  uint32_t fl[SCAN_VECS];  // 4 flag bits per vector, bit c = component c selected
  if (full) {
    const uint4 *src = reinterpret_cast<const uint4 *>(in + warp_start);
#pragma unroll
    for (int j = 0; j < SCAN_VECS; ++j) {
      uint4 u = ldg_stream(src + j * 32 + lane);
      v[j] = make_int4((int)u.x, (int)u.y, (int)u.z, (int)u.w);
    }
  } else {
#pragma unroll
    for (int j = 0; j < SCAN_VECS; ++j) {
      uint64_t e = warp_start + (uint64_t)(j * 32 + lane) * 4;
      v[j].x = e + 0 < n ? in[e + 0] : 0;
      v[j].y = e + 1 < n ? in[e + 1] : 0;
      v[j].z = e + 2 < n ? in[e + 2] : 0;
      v[j].w = e + 3 < n ? in[e + 3] : 0;
    }
  }
#pragma unroll
  for (int j = 0; j < SCAN_VECS; ++j) {
    uint64_t e = warp_start + (uint64_t)(j * 32 + lane) * 4;
    uint32_t f = 0;
    f |= ((((uint32_t)v[j].x >> 31) == want_neg) && e + 0 < n) ? 1u : 0u;
    f |= ((((uint32_t)v[j].y >> 31) == want_neg) && e + 1 < n) ? 2u : 0u;
    f |= ((((uint32_t)v[j].z >> 31) == want_neg) && e + 2 < n) ? 4u : 0u;
    f |= ((((uint32_t)v[j].w >> 31) == want_neg) && e + 3 < n) ? 8u : 0u;
    fl[j] = f;
  }
  uint32_t pre[SCAN_VECS];
  uint32_t carry = 0;
#pragma unroll
  for (int j = 0; j < SCAN_VECS; ++j) {
    uint32_t s = __popc(fl[j]);
    uint32_t inc = warp_incl_scan(s, lane);
    pre[j] = carry + inc - s;
    carry += __shfl_sync(FULL_MASK, inc, 31);
  }
  if (lane == 0) s_warp[warp] = carry;
  __syncthreads();
  if (warp == 0) {
    uint32_t wt = lane < SCAN_THREADS / 32 ? s_warp[lane] : 0u;
    uint32_t wi = warp_incl_scan(wt, lane);
    uint32_t agg = __shfl_sync(FULL_MASK, wi, SCAN_THREADS / 32 - 1);
    if (lane < SCAN_THREADS / 32) s_warp[lane] = wi - wt;
    uint32_t excl = 0;
    bool ok = true;
    if (tile == 0) {
      if (lane == 0) st_relaxed_u64(&status[0], ST_INC | agg);
    } else {
      if (lane == 0) st_relaxed_u64(&status[tile], ST_AGG | agg);
      ok = scan_lookback(status, tile, lane, budget, excl);
      if (lane == 0) st_relaxed_u64(&status[tile], ok ? (ST_INC | (uint32_t)(excl + agg)) : ST_POISON);
    }
    if (!ok && lane == 0) record_error(hdr, GPRTCU_ERR_TIMEOUT);
    if (lane == 0) {
      s_prefix = excl;
      s_tile_sel = agg;
      if (tile == num_tiles - 1) {
        hdr->total = excl + agg;
        if (d_count) *d_count = excl + agg;
      }
    }
  }
  __syncthreads();
  // Stage: selected at local rank ls, unselected at SCAN_TILE-1-lu.
  const uint32_t wbase = s_warp[warp];
#pragma unroll
  for (int j = 0; j < SCAN_VECS; ++j) {
    uint32_t local0 = (uint32_t)(warp * SCAN_WARP_ELEMS + (j * 32 + lane) * 4);
    uint32_t ls = wbase + pre[j];
    int32_t vals[4] = {v[j].x, v[j].y, v[j].z, v[j].w};
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      uint32_t local = local0 + c;
      if (local >= tile_count) continue;
      if (fl[j] & (1u << c)) {
        s_buf[ls] = vals[c];
        ++ls;
      } else if (PARTITION) {
        uint32_t lu = local - ls;
        s_buf[SCAN_TILE - 1 - lu] = vals[c];
      }
    }
  }
  __syncthreads();
  const uint32_t tsel = s_tile_sel, excl = s_prefix;
  for (uint32_t p = tid; p < tsel; p += SCAN_THREADS) out[(uint64_t)excl + p] = s_buf[p];
  if (PARTITION) {
    const uint32_t tunsel = tile_count - tsel;
    // element at staging slot p has local unselected rank lu = SCAN_TILE-1-p
    const uint64_t top = (n - 1) - (tile_start - excl);
    for (uint32_t q = tid; q < tunsel; q += SCAN_THREADS) {
      uint32_t p = SCAN_TILE - tunsel + q;
      out[top - (SCAN_TILE - 1 - p)] = s_buf[p];
    }
  }
}

}  // namespace gprtcu

using namespace gprtcu;

static uint32_t g_spin_budget = DEFAULT_SPIN_BUDGET;
static int64_t g_skip_tile = -1;
static int64_t g_skip_stage = -1;
// 0: automatic; 1: register tile per CTA; 2: TMA-staged tile per CTA;
// 3: persistent re-read kernel.  1-3 are test overrides (2 and 3 need
// 16-byte aligned in/out, else 1 runs).
static int g_scan_impl = 0;
// From this size up the persistent re-read kernel is the faster one (B200:
// 2^20 elements 12 vs 16 us, 2^30 1.50 vs 2.34 ms); below it the
// tile-per-CTA kernel needs no 224 KB CTAs.
static const uint64_t kRereadMinN = 1ull << 20;
extern "C" GPRTCU_API void gprtcuDebugScanImpl(int impl) { g_scan_impl = impl; }


gprtcuStatus gprtcu_refit_set_budget(uint32_t polls);  // lbvh.cu

extern "C" GPRTCU_API void gprtcuDebugSetSpinBudget(uint32_t polls) {
  g_spin_budget = polls ? polls : DEFAULT_SPIN_BUDGET;
  gprtcu_refit_set_budget(g_spin_budget);
}
extern "C" GPRTCU_API void gprtcuDebugScanSkipTile(int64_t tile) { g_skip_tile = tile; }
extern "C" GPRTCU_API void gprtcuDebugScanSkipStage(int64_t tile) { g_skip_stage = tile; }
uint32_t gprtcu_spin_budget(void) { return g_spin_budget; }

static const uint64_t kScanMaxN = 1ull << 40;

extern "C" GPRTCU_API size_t gprtcuScanScratchSize(uint64_t n) {
  uint64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  return sizeof(ScratchHeader) + gprtcu_align256(tiles * sizeof(uint64_t));
}

// CTAs of the re-read kernel that fit on the device at once (one per SM on
// B200); 0 if it does not fit.  Sets the shared-memory attribute once per
// device (host threads may race to do so; they all store the same value, and
// a thread that finds no value yet does the set-up itself).
static int reread_ctas() {
  static std::atomic<int> cached[64];  // the CTA count + 1; 0 = not known yet
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
  const int known = cached[dev].load(std::memory_order_acquire);
  if (known > 0) return known - 1;
  {
    int occ = 0, ctas = 0;
    if (cudaFuncSetAttribute(k_scan_reread<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RR_SMEM) ==
            cudaSuccess &&
        cudaFuncSetAttribute(k_scan_reread<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RR_SMEM) ==
            cudaSuccess &&
        cudaFuncSetAttribute(k_scan_reread<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RR_SMEM) ==
            cudaSuccess &&
        cudaFuncSetAttribute(k_scan_reread<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RR_SMEM) ==
            cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_scan_reread<0>, RR_THREADS, RR_SMEM) == cudaSuccess)
      ctas = occ * gprtcu_num_sms();
    cudaGetLastError();
    cached[dev].store(ctas + 1, std::memory_order_release);
    return ctas;
  }
}

template <int THREADS, int VECS, int LBW>
static void launch_reg_scan(const uint32_t *in, uint32_t *out, uint64_t n, int inclusive, bool vec, bool nc,
                            ScratchHeader *hdr, uint64_t *status, uint32_t *d_total, uint64_t tiles,
                            cudaStream_t stream) {
  dim3 grid((unsigned)tiles), block(THREADS);
#define GPRTCU_SCAN_LAUNCH(M, V, N)                                                                              \
  k_scan_u32<M, V, N, THREADS, VECS, LBW><<<grid, block, 0, stream>>>(in, out, n, tiles, hdr, status, d_total, \
                                                                     g_spin_budget, g_skip_tile)
  if (inclusive) {
    if (vec && nc) GPRTCU_SCAN_LAUNCH(1, true, true);
    else if (vec) GPRTCU_SCAN_LAUNCH(1, true, false);
    else GPRTCU_SCAN_LAUNCH(1, false, false);
  } else {
    if (vec && nc) GPRTCU_SCAN_LAUNCH(0, true, true);
    else if (vec) GPRTCU_SCAN_LAUNCH(0, true, false);
    else GPRTCU_SCAN_LAUNCH(0, false, false);
  }
#undef GPRTCU_SCAN_LAUNCH
}

static gprtcuStatus scan_launch(const uint32_t *in, uint32_t *out, uint64_t n, int inclusive, uint32_t *d_total,
                                void *scratch, size_t scratch_bytes, cudaStream_t stream) {
  if (n > kScanMaxN) return GPRTCU_ERR_TOO_LARGE;
  if (n > 0 && (!in || !out)) return GPRTCU_ERR_INVALID_ARG;
  if (!scratch) return GPRTCU_ERR_INVALID_ARG;
  if (((uintptr_t)scratch & 255) != 0) return GPRTCU_ERR_INVALID_ARG;
  ScratchHeader *hdr = (ScratchHeader *)scratch;
  uint64_t *status = (uint64_t *)((char *)scratch + sizeof(ScratchHeader));
  const bool vec = (((uintptr_t)in | (uintptr_t)out) & 15) == 0;
  const bool nc = (const void *)in != (const void *)out;
  // Kernel choice (all on 8192-element tiles): the persistent re-read kernel
  // for large aligned buffers, the TMA-staged tile-per-CTA kernel for smaller
  // aligned ones, the register-staged kernel for any alignment.
  int impl = vec ? g_scan_impl : 1;
  if (impl == 0) impl = n >= kRereadMinN ? 3 : 2;
  const int rr_ctas = impl == 3 ? reread_ctas() : 0;
  if (impl == 3 && rr_ctas == 0) impl = 2;
  const uint64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  if (scratch_bytes < sizeof(ScratchHeader) + tiles * sizeof(uint64_t)) return GPRTCU_ERR_SCRATCH_TOO_SMALL;
  GPRTCU_TRY(cudaMemsetAsync(scratch, 0, sizeof(ScratchHeader) + tiles * sizeof(uint64_t), stream));
  if (n == 0) {
    if (d_total) GPRTCU_TRY(cudaMemsetAsync(d_total, 0, sizeof(uint32_t), stream));
    return GPRTCU_OK;
  }
  if (impl == 3) {
    const unsigned grid = (unsigned)(tiles < (uint64_t)rr_ctas ? tiles : (uint64_t)rr_ctas);
    if (inclusive)
      k_scan_reread<1><<<grid, RR_THREADS, RR_SMEM, stream>>>(in, out, n, tiles, hdr, status, d_total, g_spin_budget,
                                                             g_skip_tile, 0u, g_skip_stage);
    else
      k_scan_reread<0><<<grid, RR_THREADS, RR_SMEM, stream>>>(in, out, n, tiles, hdr, status, d_total, g_spin_budget,
                                                             g_skip_tile, 0u, g_skip_stage);
  } else if (impl == 2) {
    // TMA-staged tile-per-CTA kernel (32 KB dynamic shared memory per CTA).
    if (inclusive)
      k_scan_tma<1><<<(unsigned)tiles, TS_THREADS, TS_SMEM, stream>>>(in, out, n, tiles, hdr, status, d_total,
                                                                       g_spin_budget, g_skip_tile);
    else
      k_scan_tma<0><<<(unsigned)tiles, TS_THREADS, TS_SMEM, stream>>>(in, out, n, tiles, hdr, status, d_total,
                                                                       g_spin_budget, g_skip_tile);
  } else {
    launch_reg_scan<256, 8, 32>(in, out, n, inclusive, vec, nc, hdr, status, d_total, tiles, stream);
  }
  GPRTCU_TRY(cudaGetLastError());
  return GPRTCU_OK;
}

extern "C" GPRTCU_API gprtcuStatus gprtcuExclusiveSumU32(const uint32_t *in, uint32_t *out, uint64_t n,
                                                         uint32_t *d_total, void *scratch, size_t scratchBytes,
                                                         gprtcuStream stream) {
  return scan_launch(in, out, n, 0, d_total, scratch, scratchBytes, (cudaStream_t)stream);
}

extern "C" GPRTCU_API gprtcuStatus gprtcuInclusiveSumU32(const uint32_t *in, uint32_t *out, uint64_t n,
                                                         uint32_t *d_total, void *scratch, size_t scratchBytes,
                                                         gprtcuStream stream) {
  return scan_launch(in, out, n, 1, d_total, scratch, scratchBytes, (cudaStream_t)stream);
}

static gprtcuStatus partition_launch(const int32_t *in, int32_t *out, uint64_t n, int select_positive, int partition,
                                     uint32_t *d_count, void *scratch, size_t scratch_bytes, cudaStream_t stream) {
  if (n > 0xFFFFFFFFull) return GPRTCU_ERR_TOO_LARGE;  // the count is a uint32, as in the reference
  if (n > 0 && (!in || !out)) return GPRTCU_ERR_INVALID_ARG;
  if (n > 0 && (const void *)in == (const void *)out) return GPRTCU_ERR_INVALID_ARG;
  if (!scratch || ((uintptr_t)scratch & 255) != 0) return GPRTCU_ERR_INVALID_ARG;
  if (scratch_bytes < gprtcuScanScratchSize(n)) return GPRTCU_ERR_SCRATCH_TOO_SMALL;
  ScratchHeader *hdr = (ScratchHeader *)scratch;
  uint64_t *status = (uint64_t *)((char *)scratch + sizeof(ScratchHeader));
  uint64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  GPRTCU_TRY(cudaMemsetAsync(scratch, 0, sizeof(ScratchHeader) + tiles * sizeof(uint64_t), stream));
  if (n == 0) {
    if (d_count) GPRTCU_TRY(cudaMemsetAsync(d_count, 0, sizeof(uint32_t), stream));
    return GPRTCU_OK;
  }
  const bool vec = ((uintptr_t)in & 15) == 0;
  // Large buffers with 16-byte aligned input and output: the persistent
  // re-read kernel (as for the sums); the scan-kernel override of the test
  // hook applies here too.
  const bool rr_ok = vec && ((uintptr_t)out & 15) == 0;
  const int impl = rr_ok ? (g_scan_impl == 0 ? (n >= kRereadMinN ? 3 : 1) : g_scan_impl) : 1;
  const int rr_ctas = impl == 3 ? reread_ctas() : 0;
  if (impl == 3 && rr_ctas > 0) {
    const unsigned g = (unsigned)(tiles < (uint64_t)rr_ctas ? tiles : (uint64_t)rr_ctas);
    const uint32_t want_neg = select_positive ? 0u : 1u;
    if (partition)
      k_scan_reread<2><<<g, RR_THREADS, RR_SMEM, stream>>>((const uint32_t *)in, (uint32_t *)out, n, tiles, hdr, status,
                                                          d_count, g_spin_budget, -1, want_neg, g_skip_stage);
    else
      k_scan_reread<3><<<g, RR_THREADS, RR_SMEM, stream>>>((const uint32_t *)in, (uint32_t *)out, n, tiles, hdr, status,
                                                          d_count, g_spin_budget, -1, want_neg, g_skip_stage);
    GPRTCU_TRY(cudaGetLastError());
    return GPRTCU_OK;
  }
  dim3 grid((unsigned)tiles), block(SCAN_THREADS);
  if (partition) {
    if (vec) k_partition_i32<true, true><<<grid, block, 0, stream>>>(in, out, n, tiles, select_positive, hdr, status, d_count, g_spin_budget);
    else k_partition_i32<true, false><<<grid, block, 0, stream>>>(in, out, n, tiles, select_positive, hdr, status, d_count, g_spin_budget);
  } else {
    if (vec) k_partition_i32<false, true><<<grid, block, 0, stream>>>(in, out, n, tiles, select_positive, hdr, status, d_count, g_spin_budget);
    else k_partition_i32<false, false><<<grid, block, 0, stream>>>(in, out, n, tiles, select_positive, hdr, status, d_count, g_spin_budget);
  }
  GPRTCU_TRY(cudaGetLastError());
  return GPRTCU_OK;
}

extern "C" GPRTCU_API gprtcuStatus gprtcuPartitionI32(const int32_t *in, int32_t *out, uint64_t n, int selectPositive,
                                                      uint32_t *d_count, void *scratch, size_t scratchBytes,
                                                      gprtcuStream stream) {
  return partition_launch(in, out, n, selectPositive, 1, d_count, scratch, scratchBytes, (cudaStream_t)stream);
}

extern "C" GPRTCU_API gprtcuStatus gprtcuSelectI32(const int32_t *in, int32_t *out, uint64_t n, int selectPositive,
                                                   uint32_t *d_count, void *scratch, size_t scratchBytes,
                                                   gprtcuStream stream) {
  return partition_launch(in, out, n, selectPositive, 0, d_count, scratch, scratchBytes, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Exclusive sum that allocates nothing and takes no scratch argument.
//
// Some callers cannot allocate device memory for work space: a host
// application that owns the whole device-memory budget and lends this library
// only the input and output buffers (an engine that allocates everything up
// front and forbids allocation while a frame is in flight, for instance), or a
// foreign-language binding that has no way to keep a device allocation alive
// between calls.  For them, gprtcuExclusiveSumU32NoAlloc keeps the look-back
// state (the 256-byte header plus one 8-byte status word per 8192-element
// tile) in the fixed array below, compiled into the library.
//
// * Size limit: n <= 2^28 (268,435,456) elements, which needs 262,400 bytes;
//   larger n returns GPRTCU_ERR_TOO_LARGE.  Every GPU that loads the library
//   holds these bytes until the process exits.
// * Set-up: host code cannot use the array's name as a device address, so the
//   first call on each device (with that device current) looks the address
//   up with cudaGetSymbolAddress and caches it.  Make that first call before
//   any stream capture on the device.
// * Sharing: every call uses the same array.  Each call clears the part it
//   uses (cudaMemsetAsync, which allocates nothing) before its kernel runs,
//   so calls ordered on one stream are safe; calls whose work overlaps on the
//   GPU (different streams, no ordering between them) race on the array and
//   give wrong results.
// * Device-side errors: a look-back wait that runs out of its budget records
//   GPRTCU_ERR_TIMEOUT in the array's header, as it would in a scratch
//   buffer's.  The caller reads it with gprtcuScratchStatus(NULL, stream,
//   &status) once the call's work is done on `stream`; the next call clears it.
// * Device reset: the cached address belongs to the device's current
//   context.  It is dropped whenever a CUDA call of this entry point fails, so
//   the call after a failure resolves it again; after cudaDeviceReset, make
//   one call and ignore its result before relying on the next.
// * No cudaMalloc, cudaFree or allocating library routine is called.
// ---------------------------------------------------------------------------
static const uint64_t kNoAllocMaxN = 1ull << 28;
static const size_t kNoAllocBytes = sizeof(ScratchHeader) + ((kNoAllocMaxN + SCAN_TILE - 1) / SCAN_TILE) * 8;
static __device__ __align__(256) unsigned char g_scan_noalloc_state[kNoAllocBytes];

#include <mutex>

static std::mutex g_noalloc_mu;
static void *g_noalloc_ptrs[64] = {nullptr};

static void noalloc_forget(void) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  g_noalloc_ptrs[dev] = nullptr;
}

static void *noalloc_state_ptr(gprtcuStatus &st) {
  void **ptrs = g_noalloc_ptrs;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    st = GPRTCU_ERR_CUDA;
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!ptrs[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_scan_noalloc_state) != cudaSuccess || !p) {
      st = GPRTCU_ERR_CUDA;
      return nullptr;
    }
    ptrs[dev] = p;
  }
  st = GPRTCU_OK;
  return ptrs[dev];
}

extern "C" GPRTCU_API gprtcuStatus gprtcuExclusiveSumU32NoAlloc(const uint32_t *in, uint32_t *out, uint64_t n,
                                                                uint32_t *d_total, gprtcuStream stream) {
  if (n > kNoAllocMaxN) return GPRTCU_ERR_TOO_LARGE;
  gprtcuStatus st;
  void *state = noalloc_state_ptr(st);
  if (!state) return st;
  st = scan_launch(in, out, n, 0, d_total, state, kNoAllocBytes, (cudaStream_t)stream);
  if (st == GPRTCU_ERR_CUDA) noalloc_forget();
  return st;
}

// Device address of the fixed array on the current device (resolving it on
// first use), for gprtcuScratchStatus(NULL, ...); NULL if that fails.
void *gprtcu_noalloc_state(void) {
  gprtcuStatus st;
  return noalloc_state_ptr(st);
}
