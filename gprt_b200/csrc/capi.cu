// capi.cu -- library-wide C entry points: status strings, version, and the
// read-back of a scratch buffer's device-side status word.
#include "common.cuh"

using namespace gprtcu;

extern "C" GPRTCU_API const char *gprtcuStatusString(int status) {
  switch (status) {
    case GPRTCU_OK: return "ok";
    case GPRTCU_ERR_INVALID_ARG: return "invalid argument";
    case GPRTCU_ERR_SIZE_MISMATCH: return "keys and values differ in size";
    case GPRTCU_ERR_SCRATCH_TOO_SMALL: return "scratch buffer too small";
    case GPRTCU_ERR_TIMEOUT: return "device-side wait exceeded its budget";
    case GPRTCU_ERR_CUDA: return "CUDA runtime error";
    case GPRTCU_ERR_TOO_LARGE: return "size beyond the supported maximum";
    default: return "unknown status";
  }
}

extern "C" GPRTCU_API int gprtcuVersion(void) { return 100; }

void *gprtcu_noalloc_state(void);  // scan.cu

// A null scratch reads the header of the fixed array that
// gprtcuExclusiveSumU32NoAlloc uses on the current device.
extern "C" GPRTCU_API gprtcuStatus gprtcuScratchStatus(const void *scratch, gprtcuStream stream, int *deviceStatus) {
  if (!deviceStatus) return GPRTCU_ERR_INVALID_ARG;
  if (!scratch) scratch = gprtcu_noalloc_state();
  if (!scratch) return GPRTCU_ERR_CUDA;
  uint32_t v = 0;
  GPRTCU_TRY(cudaMemcpyAsync(&v, scratch, sizeof(v), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  GPRTCU_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  *deviceStatus = (int)v;
  return GPRTCU_OK;
}

// Folds a scratch buffer's status word into *acc (first error wins), on the
// stream, without synchronising: the compat layer's asynchronous calls read
// *acc at their next synchronisation point.  acc may be mapped host memory.
__global__ void k_fold_status(const uint32_t *status, uint32_t *acc) {
  const uint32_t v = *(volatile const uint32_t *)status;
  if (v && *(volatile uint32_t *)acc == 0u) *(volatile uint32_t *)acc = v;
}

gprtcuStatus gprtcu_fold_status(const void *scratch, uint32_t *acc, cudaStream_t stream) {
  k_fold_status<<<1, 1, 0, stream>>>((const uint32_t *)scratch, acc);
  GPRTCU_TRY(cudaGetLastError());
  return GPRTCU_OK;
}

// SMs of the current device, looked up once per device (host threads may
// race to fill the cache; they all store the same value).
int gprtcu_num_sms() {
  static std::atomic<int> cached[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  int v = cached[dev].load(std::memory_order_relaxed);
  if (v == 0) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    cached[dev].store(v, std::memory_order_relaxed);
  }
  return v;
}
