// LBVH through the drop-in development API, as tests/t04-swBVH builds one
// over 42 points uniform in [-1e38, 1e38]^3 -- here with checks the reference
// test leaves out: every inner node's children point back to it, every leaf
// is reached once, every inner box contains its children's boxes, and the
// triangle form gives the same topology invariants.
#include <cstdio>
#include <random>
#include <stdexcept>
#include <vector>

#include "gprt_compat.h"

static void check(bool ok, const char *msg) {
  if (!ok) throw std::runtime_error(msg);
}

static void check_tree(GPRTLBVH &l) {
  const uint32_t n = l.numPrims, nn = 2 * n - 1;
  gprtBufferMap(l.nodes);
  gprtBufferMap(l.aabbs);
  const int32_t *nodes = (const int32_t *)gprtBufferGetHostPointer(l.nodes);
  const float *box = (const float *)gprtBufferGetHostPointer(l.aabbs);
  std::vector<int> parents(nn, 0);
  for (uint32_t i = 0; i + 1 < n; ++i) {
    for (int c = 0; c < 2; ++c) {
      const int ch = nodes[4 * i + c];
      check(ch >= 0 && (uint32_t)ch < nn, "child index in range");
      check(nodes[4 * ch + 2] == (int)i, "child points back to its parent");
      ++parents[ch];
      for (int k = 0; k < 3; ++k) {
        check(box[6 * i + k] <= box[6 * ch + k], "inner box contains child (min)");
        check(box[6 * i + 3 + k] >= box[6 * ch + 3 + k], "inner box contains child (max)");
      }
    }
    check(nodes[4 * i + 3] == -1, "inner nodes carry no leaf id");
  }
  for (uint32_t i = 1; i < nn; ++i) check(parents[i] == 1, "every node below the root has one parent");
  check(nodes[2] == -1, "root has no parent");
  std::vector<int> seen(n, 0);
  for (uint32_t i = n - 1; i < nn; ++i) {
    const int id = nodes[4 * i + 3];
    check(id >= 0 && (uint32_t)id < n, "leaf id in range");
    ++seen[id];
  }
  for (uint32_t i = 0; i < n; ++i) check(seen[i] == 1, "every primitive in exactly one leaf");
  gprtBufferUnmap(l.nodes);
  gprtBufferUnmap(l.aabbs);
}

int main() {
  std::mt19937 rng(42);
  {
    GPRTContext context = gprtContextCreate(nullptr, 1);
    std::uniform_real_distribution<float> dist(-1e38f, 1e38f);
    std::vector<float> pts(3 * 42);
    for (auto &v : pts) v = dist(rng);
    GPRTBuffer points = gprtDeviceBufferCreate(context, 12, 42, pts.data());
    GPRTLBVH l = gprtPointsLBVHCreate(context, points, 42);
    gprtLBVHBuild(context, l);
    check_tree(l);
    gprtLBVHDestroy(l);
    gprtBufferDestroy(points);
    gprtContextDestroy(context);
  }
  {
    GPRTContext context = gprtContextCreate(nullptr, 1);
    const uint32_t n = 100000;
    std::uniform_real_distribution<float> u(0.f, 1.f);
    std::normal_distribution<float> g(0.f, 0.002f);
    std::vector<float> pos(9 * n);
    std::vector<uint32_t> idx(3 * n);
    for (uint32_t i = 0; i < n; ++i) {
      const float c[3] = {u(rng), u(rng), u(rng)};
      for (int v = 0; v < 3; ++v) {
        for (int k = 0; k < 3; ++k) pos[9 * i + 3 * v + k] = c[k] + g(rng);
        idx[3 * i + v] = 3 * i + v;
      }
    }
    GPRTBuffer vb = gprtDeviceBufferCreate(context, 12, 3 * n, pos.data());
    GPRTBuffer ib = gprtDeviceBufferCreate(context, 12, n, idx.data());
    GPRTLBVH l = gprtTriangleLBVHCreate(context, vb, ib, n);
    gprtLBVHBuild(context, l);
    check_tree(l);
    gprtLBVHDestroy(l);
    gprtBufferDestroy(vb);
    gprtBufferDestroy(ib);
    gprtContextDestroy(context);
  }
  check(gprtcuCompatLastError() == 0, "no error recorded");
  std::printf("t04 lbvh: ok\n");
  return 0;
}
