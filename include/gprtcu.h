/*
 * gprtcu.h -- C ABI of the B200 (sm_100a) acceleration-structure path.
 *
 * Plain pointers and sizes only.  Every device pointer is caller-owned and
 * every entry point is stream-ordered and asynchronous: it enqueues work on
 * `stream` and returns.  No entry point allocates device memory; work space
 * is passed in as `scratch` of at least the size the matching *ScratchSize()
 * query returns (256-byte aligned).  Errors detected on the host return
 * immediately; errors detected on the device (a look-back wait that ran out
 * of its iteration budget) are recorded in the scratch header and read with
 * gprtcuScratchStatus().
 *
 * Each entry point names the reference interface it replaces.  The reference
 * is GPRT (gprt/gprt_host.h), whose sort/scan calls take GPRTBuffer objects;
 * include/gprt_compat.h keeps those exact signatures on top of this ABI.
 */
#ifndef GPRTCU_H
#define GPRTCU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define GPRTCU_API __declspec(dllexport)
#else
#define GPRTCU_API __attribute__((visibility("default")))
#endif

typedef struct CUstream_st *gprtcuStream; /* a cudaStream_t; NULL = legacy default stream */

typedef enum {
  GPRTCU_OK = 0,
  GPRTCU_ERR_INVALID_ARG = 1,     /* null pointer, bad width, bad bit range, misaligned */
  GPRTCU_ERR_SIZE_MISMATCH = 2,   /* keys/values size differ (gprt/gprt.cpp:8830-8835) */
  GPRTCU_ERR_SCRATCH_TOO_SMALL = 3,
  GPRTCU_ERR_TIMEOUT = 4,         /* a device-side wait exceeded its iteration budget */
  GPRTCU_ERR_CUDA = 5,            /* a CUDA runtime call failed */
  GPRTCU_ERR_TOO_LARGE = 6        /* n beyond the documented maximum */
} gprtcuStatus;

/* Human-readable name of a status code. */
GPRTCU_API const char *gprtcuStatusString(int status);
/* Library version, major*10000 + minor*100 + patch. */
GPRTCU_API int gprtcuVersion(void);

/* Reads the device-side status word of a scratch buffer after the work that
 * used it has completed on `stream` (synchronises `stream`). */
GPRTCU_API gprtcuStatus gprtcuScratchStatus(const void *scratch, gprtcuStream stream, int *deviceStatus);

/* ------------------------------------------------------------------------
 * Scan.  Replaces gprtBufferExclusiveSum (gprt/gprt_host.h:2246; host stub
 * gprt/gprt.cpp:8739-8806, intended kernel gprt/gprt_scan.slang:105-401).
 * uint32 wraparound arithmetic; in may equal out.  The total (sum of all
 * inputs mod 2^32) is written to *d_total (device pointer, may be NULL).
 * Unlike the reference there is no 2^30 cap on the aggregate
 * (gprt/gprt_host.h:2231): status words are 64-bit.
 * Maximum n: 2^40 elements.
 * ------------------------------------------------------------------------ */
GPRTCU_API size_t gprtcuScanScratchSize(uint64_t n);
GPRTCU_API gprtcuStatus gprtcuExclusiveSumU32(const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *d_total,
                                              void *scratch, size_t scratchBytes, gprtcuStream stream);
GPRTCU_API gprtcuStatus gprtcuInclusiveSumU32(const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *d_total,
                                              void *scratch, size_t scratchBytes, gprtcuStream stream);

/* Partition / select by sign.  Replaces gprtBufferPartition
 * (gprt/gprt_host.h:2295) and gprtBufferSelect (:2344); kernel modes
 * gprt/gprt_scan.slang:118-133,270-283.  Selected items (sign bit clear when
 * selectPositive, set otherwise) are compacted to the front of out in input
 * order; partition writes the rest to the back in reverse input order.
 * *d_count receives the number selected.  in and out must not alias.
 * Maximum n: 2^32 - 1 (the count is a uint32, as the reference returns). */
GPRTCU_API gprtcuStatus gprtcuPartitionI32(const int32_t *in, int32_t *out, uint64_t n, int selectPositive,
                                           uint32_t *d_count, void *scratch, size_t scratchBytes,
                                           gprtcuStream stream);
GPRTCU_API gprtcuStatus gprtcuSelectI32(const int32_t *in, int32_t *out, uint64_t n, int selectPositive,
                                        uint32_t *d_count, void *scratch, size_t scratchBytes, gprtcuStream stream);

/* ------------------------------------------------------------------------
 * Test hooks (fault injection without a GPU fault).  Process-wide settings
 * read at launch time by the look-back kernels.
 * gprtcuDebugSetSpinBudget: polls a look-back wait makes before it records
 *   GPRTCU_ERR_TIMEOUT (0 restores the default, 2^22).
 * gprtcuDebugScanSkipTile: the scan tile with this ticket never publishes its
 *   status (-1 disables), so its successors run out of budget and return.
 * ------------------------------------------------------------------------ */
GPRTCU_API void gprtcuDebugSetSpinBudget(uint32_t polls);
GPRTCU_API void gprtcuDebugScanSkipTile(int64_t tile);
/* Scan kernel selection for tests: 0 = persistent TMA-pipelined kernel when
 * in/out are 16-byte aligned (default), 1 = one tile per CTA. */
GPRTCU_API void gprtcuDebugScanImpl(int impl);

#ifdef __cplusplus
}
#endif
#endif
