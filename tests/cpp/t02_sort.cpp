// Sort through the drop-in API (gprt_compat.h), as tests/t02-bufferSort does
// with GPRT: keys-only (100,000,000 uint32 keys, checked against std::sort),
// key/value (keys a shuffled permutation so every key is unique, checked on
// both arrays), and the untyped 64-bit form the reference implements.
// Seeded for reproducibility (the reference seeds from std::random_device).
#include <algorithm>
#include <cstdio>
#include <numeric>
#include <random>
#include <stdexcept>
#include <vector>

#include "gprt_compat.h"

static void check(bool ok, const char *msg) {
  if (!ok) throw std::runtime_error(msg);
}

int main(int argc, char **argv) {
  const uint32_t n = argc > 1 ? (uint32_t)std::atol(argv[1]) : 100000000u;
  std::mt19937_64 rng(1234);
  {
    GPRTContext context = gprtContextCreate(nullptr, 1);
    auto data = gprtDeviceBufferCreate<uint32_t>(context, n);
    auto scratch = gprtDeviceBufferCreate<uint32_t>(context);
    std::vector<uint32_t> host(n);
    gprtBufferMap(data);
    uint32_t *ptr = gprtBufferGetHostPointer(data);
    std::uniform_int_distribution<uint32_t> dist(0, 0xFFFFFFFFu);
    for (uint32_t i = 0; i < n; ++i) host[i] = ptr[i] = dist(rng);
    gprtBufferUnmap(data);
    std::sort(host.begin(), host.end());
    gprtBufferSort(context, data, scratch);
    gprtBufferMap(data);
    ptr = gprtBufferGetHostPointer(data);
    for (uint32_t i = 0; i < n; ++i) {
      check(ptr[i] == host[i], "keys: element differs from std::sort");
      check(i == 0 || ptr[i] >= ptr[i - 1], "keys: out of order");
    }
    gprtBufferUnmap(data);
    check(gprtcuCompatLastError() == 0, "keys: error recorded");
    gprtBufferDestroy(data);
    gprtBufferDestroy(scratch);
    gprtContextDestroy(context);
  }
  {
    GPRTContext context = gprtContextCreate(nullptr, 1);
    auto keys = gprtDeviceBufferCreate<uint32_t>(context, n);
    auto values = gprtDeviceBufferCreate<uint32_t>(context, n);
    auto scratch = gprtDeviceBufferCreate<uint32_t>(context);
    std::vector<std::pair<uint32_t, uint32_t>> kv(n);
    std::uniform_int_distribution<uint32_t> dist(0, 0xFFFFFFFFu);
    for (uint32_t i = 0; i < n; ++i) kv[i] = {i, dist(rng)};
    std::shuffle(kv.begin(), kv.end(), rng);
    gprtBufferMap(keys);
    gprtBufferMap(values);
    uint32_t *kp = gprtBufferGetHostPointer(keys), *vp = gprtBufferGetHostPointer(values);
    for (uint32_t i = 0; i < n; ++i) {
      kp[i] = kv[i].first;
      vp[i] = kv[i].second;
    }
    gprtBufferUnmap(keys);
    gprtBufferUnmap(values);
    std::sort(kv.begin(), kv.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
    gprtBufferSortPayload(context, keys, values, scratch);
    gprtBufferMap(keys);
    gprtBufferMap(values);
    kp = gprtBufferGetHostPointer(keys);
    vp = gprtBufferGetHostPointer(values);
    for (uint32_t i = 0; i < n; ++i) {
      check(kp[i] == kv[i].first, "pairs: key differs");
      check(vp[i] == kv[i].second, "pairs: value differs");
    }
    gprtBufferUnmap(keys);
    gprtBufferUnmap(values);
    gprtBufferDestroy(keys);
    gprtBufferDestroy(values);
    gprtBufferDestroy(scratch);
    gprtContextDestroy(context);
  }
  {
    // 32-bit keys with the reference's 64-bit payloads (gprt/gprt_sort.slang:29-36)
    GPRTContext context = gprtContextCreate(nullptr, 1);
    const uint32_t m = n < 10000000u ? n : 10000000u;
    auto keys = gprtDeviceBufferCreate<uint32_t>(context, m);
    auto values = gprtDeviceBufferCreate<uint64_t>(context, m);
    auto scratch = gprtDeviceBufferCreate<uint32_t>(context);
    std::vector<std::pair<uint32_t, uint64_t>> kv(m);
    std::uniform_int_distribution<uint32_t> kd(0, 1023u);  // many equal keys: stability shows
    for (uint32_t i = 0; i < m; ++i) kv[i] = {kd(rng), ((uint64_t)i << 32) | (uint64_t)rng()};
    gprtBufferMap(keys);
    gprtBufferMap(values);
    uint32_t *kp = gprtBufferGetHostPointer(keys);
    uint64_t *vp = gprtBufferGetHostPointer(values);
    for (uint32_t i = 0; i < m; ++i) {
      kp[i] = kv[i].first;
      vp[i] = kv[i].second;
    }
    gprtBufferUnmap(keys);
    gprtBufferUnmap(values);
    std::stable_sort(kv.begin(), kv.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
    gprtBufferSortPayload(context, keys, values, scratch);
    gprtBufferMap(keys);
    gprtBufferMap(values);
    kp = gprtBufferGetHostPointer(keys);
    vp = gprtBufferGetHostPointer(values);
    for (uint32_t i = 0; i < m; ++i) {
      check(kp[i] == kv[i].first, "u32/u64 pairs: key differs");
      check(vp[i] == kv[i].second, "u32/u64 pairs: value differs (stability)");
    }
    gprtBufferUnmap(keys);
    gprtBufferUnmap(values);
    check(gprtcuCompatLastError() == 0, "u32/u64 pairs: error recorded");
    gprtBufferDestroy(keys);
    gprtBufferDestroy(values);
    gprtBufferDestroy(scratch);
    gprtContextDestroy(context);
  }
  {
    // untyped: 64-bit words with 64-bit payloads, stability visible through
    // repeated keys (payload = original index)
    const uint32_t m = n / 8;
    GPRTContext context = gprtContextCreate(nullptr, 1);
    std::vector<uint64_t> k(m), v(m);
    std::uniform_int_distribution<uint64_t> dist(0, 1000);
    for (uint32_t i = 0; i < m; ++i) {
      k[i] = dist(rng) << 40 | 7;
      v[i] = i;
    }
    GPRTBuffer keys = gprtDeviceBufferCreate(context, 8, m, k.data());
    GPRTBuffer values = gprtDeviceBufferCreate(context, 8, m, v.data());
    gprtBufferSortPayload(context, keys, values);  // null scratch: temporary work space
    std::vector<std::pair<uint64_t, uint64_t>> kv(m);
    for (uint32_t i = 0; i < m; ++i) kv[i] = {k[i], v[i]};
    std::stable_sort(kv.begin(), kv.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
    gprtBufferMap(keys);
    gprtBufferMap(values);
    const uint64_t *kp = (const uint64_t *)gprtBufferGetHostPointer(keys);
    const uint64_t *vp = (const uint64_t *)gprtBufferGetHostPointer(values);
    for (uint32_t i = 0; i < m; ++i) check(kp[i] == kv[i].first && vp[i] == kv[i].second, "u64 pairs: not stable-sorted");
    GPRTBuffer bad = gprtDeviceBufferCreate(context, 8, m + 1);
    gprtBufferSortPayload(context, keys, bad);
    check(gprtcuCompatLastError() == GPRTCU_ERR_SIZE_MISMATCH, "size mismatch not reported");
    gprtBufferDestroy(bad);
    gprtBufferDestroy(keys);
    gprtBufferDestroy(values);
    gprtContextDestroy(context);
  }
  std::printf("t02 sort: ok (%u keys)\n", n);
  return 0;
}
