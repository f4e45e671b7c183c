// lbvh.cuh -- device-side layouts of the LBVH traversal data.
#pragma once
#include <stdint.h>

namespace gprtcu {

// One inner node of the binary traversal layout: both child boxes and both
// child references in 64 bytes (four 16-byte loads).  box[6*c + k] is child
// c's {lo.x, lo.y, lo.z, hi.x, hi.y, hi.z}; ref[c] >= 0 is an inner node,
// ref[c] < 0 is leaf slot ~ref[c] (the leaf's position in sorted order).
struct __align__(16) Bvh2Node {
  float box[12];
  int ref[2];
  int pad[2];
};
static_assert(sizeof(Bvh2Node) == 64, "64-byte node");

// Triangle of leaf slot s: three float4 {v.xyz, w}; w of the first holds the
// primitive id bits.
struct Hit {
  uint32_t prim;
  float t;
};

}  // namespace gprtcu
