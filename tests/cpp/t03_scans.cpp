// Scans through the drop-in API, on the schedule of tests/t03-bufferScans:
// 100 rounds each of N = 9973*k (k = 2..101) for the exclusive sum of all ones
// (total N, out[i] = i), the partition of x_i = i * (i odd ? 1 : -1) with
// selectPositive (selected in order at the front, the rest reversed at the
// back), and the select of the same data; a fresh context per round.
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "gprt_compat.h"

static void check(bool ok, const char *msg, uint32_t n) {
  if (!ok) {
    std::fprintf(stderr, "failed at N=%u\n", n);
    throw std::runtime_error(msg);
  }
}

int main(int argc, char **argv) {
  const int rounds = argc > 1 ? std::atoi(argv[1]) : 100;
  const uint32_t prime = 9973;
  uint32_t num = prime;
  for (int round = 0; round < rounds; ++round) {
    num += prime;
    std::vector<uint32_t> ones(num, 1);
    GPRTContext context = gprtContextCreate(nullptr, 1);
    auto data = gprtDeviceBufferCreate<uint32_t>(context, num, ones.data());
    auto out = gprtDeviceBufferCreate<uint32_t>(context, num);
    auto scratch = gprtDeviceBufferCreate<uint32_t>(context);
    uint32_t total = gprtBufferExclusiveSum(context, data, out, scratch);
    check(total == num, "exclusive sum: total", num);
    gprtBufferMap(out);
    const uint32_t *p = gprtBufferGetHostPointer(out);
    for (uint32_t i = 0; i < num; ++i) check(p[i] == i, "exclusive sum: element", num);
    gprtBufferUnmap(out);
    gprtBufferDestroy(data);
    gprtBufferDestroy(out);
    gprtBufferDestroy(scratch);
    gprtContextDestroy(context);
  }
  for (int mode = 0; mode < 2; ++mode) {
    num = prime;
    for (int round = 0; round < rounds; ++round) {
      num += prime;
      std::vector<int32_t> x(num);
      for (uint32_t i = 0; i < num; ++i) x[i] = (int32_t)i * ((i & 1) ? 1 : -1);
      GPRTContext context = gprtContextCreate(nullptr, 1);
      auto data = gprtDeviceBufferCreate<int32_t>(context, num, x.data());
      auto out = gprtDeviceBufferCreate<int32_t>(context, num);
      auto scratch = gprtDeviceBufferCreate<uint32_t>(context);
      const uint32_t total = mode == 0 ? gprtBufferPartition(context, data, true, out, scratch)
                                       : gprtBufferSelect(context, data, true, out, scratch);
      std::vector<int32_t> expect(num, 0);
      uint32_t excl = 0;
      for (uint32_t i = 0; i < num; ++i) {
        if (x[i] >= 0) expect[excl++] = x[i];
        else if (mode == 0) expect[(num - 1) - (i - excl)] = x[i];
      }
      check(total == excl, mode == 0 ? "partition: total" : "select: total", num);
      gprtBufferMap(out);
      const int32_t *p = gprtBufferGetHostPointer(out);
      const uint32_t upto = mode == 0 ? num : excl;
      for (uint32_t i = 0; i < upto; ++i) check(p[i] == expect[i], mode == 0 ? "partition: layout" : "select: layout", num);
      gprtBufferUnmap(out);
      gprtBufferDestroy(data);
      gprtBufferDestroy(out);
      gprtBufferDestroy(scratch);
      gprtContextDestroy(context);
    }
  }
  std::printf("t03 scans: ok (%d rounds)\n", rounds);
  return 0;
}
