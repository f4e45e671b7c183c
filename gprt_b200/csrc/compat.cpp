// compat.cpp -- GPRTContext / GPRTBuffer on CUDA and the reference-named
// sort / scan / partition / select calls (include/gprt_compat.h) on top of the
// primary C ABI (include/gprtcu.h).  Host code only.
//
// Reference behaviour kept: buffers are sized in bytes (size * count), the
// sort is in place, scratch passed in is grown when too small
// (gprt/gprt.cpp:8856-8861) and a null scratch uses temporary work space,
// ExclusiveSum / Partition / Select return the total synchronously
// (gprt/gprt_scan.slang:290-297 state[0]), a key/value size mismatch is an
// error (gprt/gprt.cpp:8830-8835).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <new>

#include "gprt_compat.h"

struct GPRTContext_T {
  int device;
  cudaStream_t stream;
  uint32_t *d_word;  // device word for totals
  uint32_t *h_word;  // pinned host words: [0] totals, [1] pending device status of asynchronous sorts
  uint32_t *h_word_dev;  // device view of h_word
};

gprtcuStatus gprtcu_fold_status(const void *scratch, uint32_t *acc, cudaStream_t stream);  // capi.cu

struct GPRTBuffer_T {
  GPRTContext ctx;
  int kind;  // 0 device, 1 host (pinned, mapped), 2 shared (managed)
  void *dptr;
  void *hptr;  // host view: staging for device buffers
  size_t bytes;
  size_t staging_bytes;
};

static thread_local int t_last_error = 0;

static void compat_error(int code, const char *what) {
  t_last_error = code;
  std::fprintf(stderr, "[gprt] error: %s (%s)\n", what, gprtcuStatusString(code));
}

extern "C" GPRTCU_API int gprtcuCompatLastError(void) {
  int e = t_last_error;
  t_last_error = 0;
  return e;
}

extern "C" GPRTCU_API gprtcuStream gprtcuCompatStream(GPRTContext context) {
  return context ? (gprtcuStream)context->stream : nullptr;
}

extern "C" GPRTCU_API GPRTContext gprtContextCreate(int32_t *requestedDeviceIDs, int numDevices) {
  if (numDevices > 1) {
    compat_error(GPRTCU_ERR_INVALID_ARG, "gprtContextCreate: one device per context");
    return nullptr;
  }
  int dev = (requestedDeviceIDs && numDevices == 1) ? requestedDeviceIDs[0] : 0;
  if (cudaSetDevice(dev) != cudaSuccess) {
    compat_error(GPRTCU_ERR_CUDA, "gprtContextCreate: cudaSetDevice");
    return nullptr;
  }
  GPRTContext c = new (std::nothrow) GPRTContext_T{dev, nullptr, nullptr, nullptr, nullptr};
  if (!c) return nullptr;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&c->d_word, 256) != cudaSuccess ||
      cudaHostAlloc((void **)&c->h_word, 256, cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer((void **)&c->h_word_dev, c->h_word, 0) != cudaSuccess) {
    compat_error(GPRTCU_ERR_CUDA, "gprtContextCreate: stream / work words");
    delete c;
    return nullptr;
  }
  std::memset(c->h_word, 0, 256);
  return c;
}

// After a synchronisation of the context's stream: reports a device-side
// error that an earlier asynchronous sort (caller scratch) recorded.
static void report_pending(GPRTContext c) {
  const uint32_t st = ((volatile uint32_t *)c->h_word)[1];
  if (st) {
    ((volatile uint32_t *)c->h_word)[1] = 0;
    compat_error((int)st, "gprtBufferSort / gprtBufferSortPayload (an earlier call on this context)");
  }
}

extern "C" GPRTCU_API void gprtContextDestroy(GPRTContext c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  report_pending(c);
  cudaFree(c->d_word);
  cudaFreeHost(c->h_word);
  cudaStreamDestroy(c->stream);
  delete c;
}

static bool alloc_storage(GPRTBuffer b, size_t bytes) {
  const size_t n = bytes ? bytes : 16;
  if (b->kind == 0) return cudaMalloc(&b->dptr, n) == cudaSuccess;
  if (b->kind == 1) {
    if (cudaHostAlloc(&b->hptr, n, cudaHostAllocMapped) != cudaSuccess) return false;
    return cudaHostGetDevicePointer(&b->dptr, b->hptr, 0) == cudaSuccess;
  }
  if (cudaMallocManaged(&b->dptr, n) != cudaSuccess) return false;
  b->hptr = b->dptr;
  return true;
}

static void free_storage(GPRTBuffer b) {
  if (b->kind == 0) {
    cudaFree(b->dptr);
    if (b->hptr) cudaFreeHost(b->hptr);
  } else if (b->kind == 1) {
    cudaFreeHost(b->hptr);
  } else {
    cudaFree(b->dptr);
  }
  b->dptr = b->hptr = nullptr;
  b->staging_bytes = 0;
}

static GPRTBuffer buffer_create(GPRTContext c, int kind, size_t size, size_t count, const void *init) {
  if (!c) {
    compat_error(GPRTCU_ERR_INVALID_ARG, "buffer create: null context");
    return nullptr;
  }
  cudaSetDevice(c->device);
  GPRTBuffer b = new (std::nothrow) GPRTBuffer_T{c, kind, nullptr, nullptr, size * count, 0};
  if (!b || !alloc_storage(b, b->bytes)) {
    compat_error(GPRTCU_ERR_CUDA, "buffer create: allocation");
    delete b;
    return nullptr;
  }
  if (init && b->bytes) {
    if (kind == 0) {
      cudaMemcpyAsync(b->dptr, init, b->bytes, cudaMemcpyHostToDevice, c->stream);
      cudaStreamSynchronize(c->stream);
    } else {
      std::memcpy(b->hptr, init, b->bytes);
    }
  }
  return b;
}

extern "C" GPRTCU_API GPRTBuffer gprtDeviceBufferCreate(GPRTContext c, size_t size, size_t count, const void *init,
                                                        size_t) {
  return buffer_create(c, 0, size, count, init);
}
extern "C" GPRTCU_API GPRTBuffer gprtHostBufferCreate(GPRTContext c, size_t size, size_t count, const void *init,
                                                      size_t) {
  return buffer_create(c, 1, size, count, init);
}
extern "C" GPRTCU_API GPRTBuffer gprtSharedBufferCreate(GPRTContext c, size_t size, size_t count, const void *init,
                                                        size_t) {
  return buffer_create(c, 2, size, count, init);
}

extern "C" GPRTCU_API void gprtBufferDestroy(GPRTBuffer b) {
  if (!b) return;
  cudaSetDevice(b->ctx->device);
  cudaStreamSynchronize(b->ctx->stream);
  free_storage(b);
  delete b;
}

extern "C" GPRTCU_API size_t gprtBufferGetSize(GPRTBuffer b, int) { return b ? b->bytes : 0; }
extern "C" GPRTCU_API void *gprtBufferGetDevicePointer(GPRTBuffer b, int) { return b ? b->dptr : nullptr; }

extern "C" GPRTCU_API void *gprtBufferGetHostPointer(GPRTBuffer b, int) {
  if (!b) return nullptr;
  if (b->kind == 0 && b->staging_bytes < b->bytes) {
    if (b->hptr) cudaFreeHost(b->hptr);
    b->hptr = nullptr;
    if (cudaMallocHost(&b->hptr, b->bytes ? b->bytes : 16) != cudaSuccess) {
      compat_error(GPRTCU_ERR_CUDA, "gprtBufferGetHostPointer: staging");
      return nullptr;
    }
    b->staging_bytes = b->bytes;
  }
  return b->hptr;
}

// Map: the host view reflects the device contents (the reference copies
// through a staging buffer and waits, gprt/gprt.cpp:841-863).
extern "C" GPRTCU_API void gprtBufferMap(GPRTBuffer b, int d) {
  if (!b) return;
  cudaSetDevice(b->ctx->device);
  cudaStreamSynchronize(b->ctx->stream);
  report_pending(b->ctx);
  if (b->kind != 0) return;
  void *h = gprtBufferGetHostPointer(b, d);
  if (h && b->bytes) cudaMemcpy(h, b->dptr, b->bytes, cudaMemcpyDeviceToHost);
}

// Unmap: host writes go back to the device.
extern "C" GPRTCU_API void gprtBufferUnmap(GPRTBuffer b, int) {
  if (!b || b->kind != 0 || !b->hptr || !b->bytes) return;
  cudaSetDevice(b->ctx->device);
  cudaMemcpyAsync(b->dptr, b->hptr, b->bytes, cudaMemcpyHostToDevice, b->ctx->stream);
  cudaStreamSynchronize(b->ctx->stream);
}

extern "C" GPRTCU_API void gprtBufferResize(GPRTContext c, GPRTBuffer b, size_t size, size_t count,
                                            bool preserveContents, int) {
  if (!b) return;
  const size_t nb = size * count;
  if (nb == b->bytes) return;
  cudaSetDevice(b->ctx->device);
  cudaStreamSynchronize(b->ctx->stream);
  GPRTBuffer_T old = *b;
  b->dptr = b->hptr = nullptr;
  b->staging_bytes = 0;
  if (!alloc_storage(b, nb)) {
    compat_error(GPRTCU_ERR_CUDA, "gprtBufferResize: allocation");
    *b = old;
    return;
  }
  if (preserveContents) {
    const size_t keep = old.bytes < nb ? old.bytes : nb;
    if (keep) cudaMemcpy(b->dptr, old.dptr, keep, cudaMemcpyDefault);
  }
  b->bytes = nb;
  free_storage(&old);
  (void)c;
}

// Work space for a call: the caller's buffer (grown when undersized) or a
// temporary allocation when none is given.
struct Work {
  void *ptr = nullptr;
  size_t bytes = 0;
  bool temp = false;
};

static bool get_work(GPRTContext c, GPRTBuffer scratch, size_t need, Work &w) {
  if (scratch) {
    if (scratch->bytes < need) gprtBufferResize(c, scratch, 1, need, false, 0);
    if (scratch->bytes < need) return false;
    w.ptr = scratch->dptr;
    w.bytes = scratch->bytes;
    // the primary ABI wants 256-byte aligned scratch; cudaMalloc gives it
    return ((uintptr_t)w.ptr & 255) == 0;
  }
  if (cudaMalloc(&w.ptr, need ? need : 256) != cudaSuccess) return false;
  w.bytes = need ? need : 256;
  w.temp = true;
  return true;
}

static void put_work(GPRTContext c, Work &w) {
  if (w.temp) {
    cudaStreamSynchronize(c->stream);
    cudaFree(w.ptr);
  }
}

static bool device_status_ok(GPRTContext c, void *scratch, const char *what) {
  int st = 0;
  if (gprtcuScratchStatus(scratch, (gprtcuStream)c->stream, &st) != GPRTCU_OK || st != 0) {
    compat_error(st ? st : GPRTCU_ERR_CUDA, what);
    return false;
  }
  return true;
}

static uint32_t scan_family(GPRTContext c, GPRTBuffer in, GPRTBuffer out, GPRTBuffer scratch, int mode,
                            bool selectPositive, const char *what) {
  if (!c || !in || !out) {
    compat_error(GPRTCU_ERR_INVALID_ARG, what);
    return (uint32_t)-1;
  }
  cudaSetDevice(c->device);
  const uint64_t n = in->bytes / 4;
  if (out->bytes < n * 4) {
    compat_error(GPRTCU_ERR_SIZE_MISMATCH, what);
    return (uint32_t)-1;
  }
  Work w;
  if (!get_work(c, scratch, gprtcuScanScratchSize(n), w)) {
    compat_error(GPRTCU_ERR_SCRATCH_TOO_SMALL, what);
    return (uint32_t)-1;
  }
  gprtcuStatus st;
  gprtcuStream s = (gprtcuStream)c->stream;
  if (mode == 0)
    st = gprtcuExclusiveSumU32((const uint32_t *)in->dptr, (uint32_t *)out->dptr, n, c->d_word, w.ptr, w.bytes, s);
  else if (mode == 1)
    st = gprtcuPartitionI32((const int32_t *)in->dptr, (int32_t *)out->dptr, n, selectPositive ? 1 : 0, c->d_word,
                            w.ptr, w.bytes, s);
  else
    st = gprtcuSelectI32((const int32_t *)in->dptr, (int32_t *)out->dptr, n, selectPositive ? 1 : 0, c->d_word,
                         w.ptr, w.bytes, s);
  uint32_t total = (uint32_t)-1;
  if (st != GPRTCU_OK) {
    compat_error(st, what);
  } else if (device_status_ok(c, w.ptr, what)) {
    cudaMemcpyAsync(c->h_word, c->d_word, 4, cudaMemcpyDeviceToHost, c->stream);
    cudaStreamSynchronize(c->stream);
    total = *c->h_word;
  }
  report_pending(c);
  put_work(c, w);
  return total;
}

extern "C" GPRTCU_API uint32_t gprtBufferExclusiveSum(GPRTContext c, GPRTBuffer in, GPRTBuffer out,
                                                      GPRTBuffer scratch) {
  return scan_family(c, in, out, scratch, 0, true, "gprtBufferExclusiveSum");
}
extern "C" GPRTCU_API uint32_t gprtBufferPartition(GPRTContext c, GPRTBuffer in, bool selectPositive, GPRTBuffer out,
                                                   GPRTBuffer scratch) {
  return scan_family(c, in, out, scratch, 1, selectPositive, "gprtBufferPartition");
}
extern "C" GPRTCU_API uint32_t gprtBufferSelect(GPRTContext c, GPRTBuffer in, bool selectPositive, GPRTBuffer out,
                                                GPRTBuffer scratch) {
  return scan_family(c, in, out, scratch, 2, selectPositive, "gprtBufferSelect");
}

extern "C" GPRTCU_API void gprtcuCompatSort(GPRTContext c, GPRTBuffer keys, int kw, GPRTBuffer values, int vw,
                                            GPRTBuffer scratch) {
  const char *what = values ? "gprtBufferSortPayload" : "gprtBufferSort";
  if (!c || !keys || (kw != 4 && kw != 8) || (values && vw != 4 && vw != 8)) {
    compat_error(GPRTCU_ERR_INVALID_ARG, what);
    return;
  }
  cudaSetDevice(c->device);
  const uint64_t n = keys->bytes / (uint64_t)kw;
  if (values && values->bytes / (uint64_t)vw != n) {
    compat_error(GPRTCU_ERR_SIZE_MISMATCH, what);
    return;
  }
  if (!values) vw = 0;
  Work w;
  if (!get_work(c, scratch, gprtcuSortScratchSize(n, kw, vw), w)) {
    compat_error(GPRTCU_ERR_SCRATCH_TOO_SMALL, what);
    return;
  }
  gprtcuStream s = (gprtcuStream)c->stream;
  void *k = keys->dptr, *v = values ? values->dptr : nullptr;
  gprtcuStatus st;
  if (kw == 4 && vw == 0) st = gprtcuSortKeysU32((uint32_t *)k, n, 0, 32, w.ptr, w.bytes, s);
  else if (kw == 4 && vw == 4) st = gprtcuSortPairsU32((uint32_t *)k, (uint32_t *)v, n, 0, 32, w.ptr, w.bytes, s);
  else if (kw == 8 && vw == 0) st = gprtcuSortKeysU64((uint64_t *)k, n, 0, 64, w.ptr, w.bytes, s);
  else if (kw == 8 && vw == 4) st = gprtcuSortPairsU64((uint64_t *)k, (uint32_t *)v, n, 0, 64, w.ptr, w.bytes, s);
  else if (kw == 8 && vw == 8) st = gprtcuSortPairsU64U64((uint64_t *)k, (uint64_t *)v, n, 0, 64, w.ptr, w.bytes, s);
  else st = gprtcuSortPairsU32U64((uint32_t *)k, (uint64_t *)v, n, 0, 32, w.ptr, w.bytes, s);
  if (st != GPRTCU_OK) compat_error(st, what);
  // asynchronous, like the reference's compute submission; temporary work
  // space is freed after the stream drains, so its status is read then
  else if (w.temp) device_status_ok(c, w.ptr, what);
  // with the caller's scratch the call stays asynchronous: the status word is
  // folded into a host word on the stream and reported at the next
  // synchronisation (gprtBufferMap, a sum / partition / select, destroy)
  else if (gprtcu_fold_status(w.ptr, c->h_word_dev + 1, c->stream) != GPRTCU_OK)
    compat_error(GPRTCU_ERR_CUDA, what);
  put_work(c, w);
}

// Untyped forms sort 64-bit words, as the reference implementation does.
extern "C" GPRTCU_API void gprtBufferSort(GPRTContext c, GPRTBuffer buffer, GPRTBuffer scratch) {
  gprtcuCompatSort(c, buffer, 8, nullptr, 0, scratch);
}
extern "C" GPRTCU_API void gprtBufferSortPayload(GPRTContext c, GPRTBuffer keys, GPRTBuffer values,
                                                 GPRTBuffer scratch) {
  if (keys && values && keys->bytes != values->bytes) {
    compat_error(GPRTCU_ERR_SIZE_MISMATCH, "gprtBufferSortPayload: keys and values differ in size");
    return;
  }
  gprtcuCompatSort(c, keys, 8, values, 8, scratch);
}
