// common.cuh -- shared device helpers for the sm_100a kernels: relaxed
// global-scope loads/stores for the look-back status words, streaming
// 128-bit loads, the scratch header, and the bounded-wait policy.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "../../include/gprtcu.h"

namespace gprtcu {

constexpr unsigned FULL_MASK = 0xFFFFFFFFu;

// Every scratch buffer starts with this 256-byte header.  The host zeroes the
// parts a call uses before launching (cudaMemsetAsync, stream-ordered).
struct ScratchHeader {
  uint32_t status;        // 0 = ok, else a gprtcuStatus written by a kernel
  uint32_t pad0;
  uint32_t ticket[16];    // tile tickets: one per pass / kernel
  uint32_t sel[16];       // sort: which ping-pong buffer holds pass p's input
  uint32_t total;         // scan: total of the last call
  uint32_t pad1[29];
};
static_assert(sizeof(ScratchHeader) == 256, "header is 256 bytes");

// Upper bound on the number of polls a look-back wait makes before it gives
// up, records GPRTCU_ERR_TIMEOUT and poisons its own status so that the tiles
// after it stop waiting too.  One poll is an L2 round trip (>= ~0.3 us), so
// this is more than a second of waiting on a predecessor that never publishes.
constexpr uint32_t DEFAULT_SPIN_BUDGET = 1u << 22;

__device__ __forceinline__ void st_relaxed_u64(uint64_t *p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t *p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u32(uint32_t *p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Atomic add with acquire-release semantics at GPU scope: the caller's earlier
// writes are visible to whoever observes this add, and writes made visible by
// the add it observes are visible to the caller's later reads.
__device__ __forceinline__ uint32_t atom_add_acq_rel_u32(uint32_t *p, uint32_t v) {
  uint32_t old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

// Streaming 128-bit load through the non-coherent path without L1 allocation
// (input read exactly once).
__device__ __forceinline__ uint4 ldg_stream(const uint4 *p) {
  uint4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}
// Coherent 128-bit load (used when input and output alias).
__device__ __forceinline__ uint4 ldg_coherent(const uint4 *p) {
  uint4 v;
  asm volatile("ld.global.v4.u32 {%0,%1,%2,%3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p));
  return v;
}
__device__ __forceinline__ void stg_v4(uint4 *p, uint4 v) {
  asm volatile("st.global.v4.u32 [%0], {%1,%2,%3,%4};" ::"l"(p), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w)
               : "memory");
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(FULL_MASK, v, o);
    if (lane >= o) v += y;
  }
  return v;
}
__device__ __forceinline__ uint32_t warp_sum(uint32_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
  return v;
}

// Record a device-side error in the scratch header (first error wins).
__device__ __forceinline__ void record_error(ScratchHeader *h, uint32_t code) { atomicCAS(&h->status, 0u, code); }

}  // namespace gprtcu

// Host-side helpers shared by the .cu files.
#define GPRTCU_TRY(expr)                                   \
  do {                                                     \
    cudaError_t _e = (expr);                               \
    if (_e != cudaSuccess) return GPRTCU_ERR_CUDA;         \
  } while (0)

static inline size_t gprtcu_align256(size_t v) { return (v + 255) & ~(size_t)255; }

// ---------------------------------------------------------------------------
// TMA bulk (non-tensor, non-multicast) copies and mbarriers.  Single-GPU only:
// every source and destination here is this GPU's own memory.
// ---------------------------------------------------------------------------
namespace gprtcu {

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
// Bounded wait on a phase of an mbarrier; false if the budget ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t budget) {
  uint32_t done = 0;
  for (uint32_t i = 0; i < budget; ++i) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
// global -> shared, completion counted on `bar` in bytes.
__device__ __forceinline__ void bulk_g2s(void *dst_smem, const void *src_gmem, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst_smem)),
      "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
// Fetches [src_gmem, src_gmem + bytes) into L2 without waiting for it (a
// hint: no completion to track; both 16-byte aligned / multiples of 16).
__device__ __forceinline__ void bulk_prefetch_l2(const void *src_gmem, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src_gmem), "r"(bytes) : "memory");
}
// shared -> global, tracked by bulk groups.
__device__ __forceinline__ void bulk_s2g(void *dst_gmem, const void *src_smem, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst_gmem), "r"(smem_addr(src_smem)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
template <int N> __device__ __forceinline__ void bulk_wait() {
  asm volatile("cp.async.bulk.wait_group %0;" ::"n"(N) : "memory");
}
// Generic-proxy shared-memory writes become visible to the async proxy.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// L2 eviction-priority policies for the cache-hinted bulk copies below.
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ void bulk_g2s_hint(void *dst_smem, const void *src_gmem, uint32_t bytes, uint64_t *bar,
                                              uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
          "r"(smem_addr(dst_smem)),
      "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
      : "memory");
}
__device__ __forceinline__ void bulk_s2g_hint(void *dst_gmem, const void *src_smem, uint32_t bytes, uint64_t policy) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group.L2::cache_hint [%0], [%1], %2, %3;" ::"l"(dst_gmem),
               "r"(smem_addr(src_smem)), "r"(bytes), "l"(policy)
               : "memory");
}
// Barrier over a subset of the CTA's warps (`threads` a multiple of 32).
__device__ __forceinline__ void named_bar_sync(int id, int threads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

// Polls an mbarrier wait makes before it gives up: 16 for every poll of the
// look-back budget the call was given (2^26 at the default 2^22), so a test
// that shortens the look-back budget shortens these waits too.  A try_wait
// poll itself suspends the thread for a while, so 2^26 polls are seconds.
__device__ __forceinline__ uint32_t mbar_budget_of(uint32_t lookback_budget) {
  return lookback_budget >= (1u << 28) ? 0xFFFFFFFFu : lookback_budget << 4;
}

}  // namespace gprtcu

// Number of SMs of the current device (cached per device id).
int gprtcu_num_sms();
