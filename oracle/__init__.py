"""ctypes bindings for the CPU oracle (oracle/oracle.cpp) and, when built,
the reference-compiled checker (oracle/_ref/libgprtref.so).

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg (and its reference arm) may import this package.  The product
(gprt_b200) never imports it, and nothing here is a fallback for the CUDA path.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libgprtref.so")

_lib = None
_ref = None

HIT_DTYPE = np.dtype([("prim", np.uint32), ("t", np.float32)])


def build(ref=None):
    """Compile the oracle, and the reference checker when ref is true or,
    with ref None, when the recipe finds the reference sources (oracle/Makefile,
    variable REF)."""
    subprocess.check_call(["make", "-s", "-C", HERE])
    if ref is None:
        ref = subprocess.call(["make", "-s", "-C", HERE, "has-ref"], stderr=subprocess.DEVNULL) == 0
    if ref:
        subprocess.check_call(["make", "-s", "-C", HERE, "ref"])


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build(ref=False)
        L = ctypes.CDLL(LIB_PATH)
        vp, u32, u64, sz, i32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t, ctypes.c_int
        L.orc_sort.argtypes = [vp, i32, vp, i32, sz]
        L.orc_scan_u32.argtypes = [vp, vp, sz, i32]
        L.orc_scan_u32.restype = u32
        L.orc_partition_i32.argtypes = [vp, vp, sz, i32, i32]
        L.orc_partition_i32.restype = u32
        L.orc_morton3d.argtypes = [u32, u32, u32]
        L.orc_morton3d.restype = u32
        L.orc_hilbert3d.argtypes = [u32, u32, u32]
        L.orc_hilbert3d.restype = u32
        L.orc_tri_bounds.argtypes = [vp, vp, u32, vp]
        L.orc_tri_codes.argtypes = [vp, vp, u32, vp, i32, vp, vp]
        L.orc_point_bounds.argtypes = [vp, u32, vp]
        L.orc_point_codes.argtypes = [vp, u32, vp, i32, vp, vp]
        L.orc_karras.argtypes = [vp, u32, vp]
        L.orc_refit_tri.argtypes = [vp, vp, vp, u32, vp, vp]
        L.orc_lbvh_build_tri.argtypes = [vp, vp, u32, i32, vp, vp, vp, vp, vp]
        L.orc_lbvh_build_points.argtypes = [vp, u32, i32, vp, vp, vp, vp, vp]
        L.orc_lbvh_build_edges.argtypes = [vp, vp, u32, i32, vp, vp, vp, vp, vp]
        L.orc_lbvh_build_boxes.argtypes = [vp, u32, i32, vp, vp, vp, vp, vp]
        L.orc_lss_intersect.argtypes = [vp, vp, vp, i32, i32, i32, vp, vp]
        L.orc_lss_intersect.restype = i32
        L.orc_lss_bounds.argtypes = [vp, vp, u32, i32, i32, vp]
        L.orc_sphere_bounds.argtypes = [vp, u32, vp]
        L.orc_trace_user_brute.argtypes = [i32, vp, vp, u32, i32, i32, i32, vp, u64, vp]
        L.orc_instance_inverse.argtypes = [vp, vp]
        L.orc_instance_inverse.restype = i32
        L.orc_trace_instances_brute.argtypes = [vp, u32, vp, vp, vp, u32, vp, u64, u32, vp]
        L.orc_isect_tri32.argtypes = [vp, vp, vp, vp, vp]
        L.orc_isect_tri32.restype = i32
        L.orc_refine_t32.argtypes = [vp, vp, vp, vp]
        L.orc_refine_t32.restype = ctypes.c_float
        L.orc_t64.argtypes = [vp, vp, vp, vp]
        L.orc_t64.restype = ctypes.c_double
        L.orc_trace_brute.argtypes = [vp, vp, u32, vp, u64, vp]
        L.orc_trace_lbvh.argtypes = [vp, vp, u32, vp, vp, vp, u64, i32, vp]
        L.orc_trace_lbvh64.argtypes = [vp, vp, u32, vp, vp, vp, u64, vp, vp]
        L.orc_isect_tri64.argtypes = [vp, vp, vp, vp, vp]
        L.orc_isect_tri64.restype = i32
        L.orc_num_threads.restype = i32
        L.orc_solid_vertex_count.argtypes = [u32]
        L.orc_solid_vertex_count.restype = i32
        L.orc_solid_hit_kind.argtypes = [u32]
        L.orc_solid_hit_kind.restype = u32
        L.orc_solid_intersect.argtypes = [vp, vp, u32, vp]
        L.orc_solid_intersect.restype = i32
        L.orc_solid_bounds.argtypes = [vp, vp, vp, u32, vp]
        L.orc_solid_locate_brute.argtypes = [vp, vp, vp, u32, vp, u64, vp, vp, vp]
        _lib = L
    return _lib


def ref_available():
    return os.path.exists(REF_PATH)


def ref():
    """The reference's own LBVH programs and Hilbert encoder, compiled from its sources."""
    global _ref
    if _ref is None:
        R = ctypes.CDLL(REF_PATH)
        vp, u32, i32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int
        R.ref_lbvh_build.argtypes = [i32, vp, u32, vp, u32, vp, vp, vp, vp, vp]
        R.ref_hilbert3d.argtypes = [u32, u32, u32]
        R.ref_hilbert3d.restype = u32
        R.ref_solid_intersect.argtypes = [vp, vp, u32, vp]
        R.ref_solid_intersect.restype = i32
        R.ref_solid_bounds.argtypes = [vp, vp, vp, u32, vp]
        R.ref_solid_vertex_count.argtypes = [u32]
        R.ref_solid_vertex_count.restype = i32
        R.ref_solid_hit_kind.argtypes = [u32]
        R.ref_solid_hit_kind.restype = u32
        _ref = R
    return _ref


# ----------------------------------------------------------------------------
# numpy-level helpers
# ----------------------------------------------------------------------------
def sort(keys, vals=None):
    """Stable ascending sort; returns new arrays."""
    k = np.ascontiguousarray(keys).copy()
    v = None if vals is None else np.ascontiguousarray(vals).copy()
    lib().orc_sort(_p(k), k.itemsize, _p(v), 0 if v is None else v.itemsize, k.size)
    return k if v is None else (k, v)


def scan(x, inclusive=False):
    x = np.ascontiguousarray(x, dtype=np.uint32)
    out = np.empty_like(x)
    total = lib().orc_scan_u32(_p(x), _p(out), x.size, 1 if inclusive else 0)
    return out, int(total)


def partition(x, select_positive=True, partition=True):
    x = np.ascontiguousarray(x, dtype=np.int32)
    out = np.zeros_like(x)
    total = lib().orc_partition_i32(_p(x), _p(out), x.size, 1 if select_positive else 0, 1 if partition else 0)
    return out, int(total)


def morton3d(x, y, z):
    return lib().orc_morton3d(int(x), int(y), int(z))


def hilbert3d(x, y, z):
    return lib().orc_hilbert3d(int(x), int(y), int(z))


def lbvh_build_tri(pos, tri, kind=0):
    """Full CPU LBVH build.  Returns dict(scene, codes, ids, nodes, aabbs)."""
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    tri = np.ascontiguousarray(tri, dtype=np.uint32)
    n = tri.shape[0]
    scene = np.zeros(6, np.float32)
    codes = np.zeros(n, np.uint32)
    ids = np.zeros(n, np.uint32)
    nn = max(2 * n - 1, 0)
    nodes = np.full((nn, 4), -1, np.int32)
    aabbs = np.zeros((nn, 6), np.float32)
    lib().orc_lbvh_build_tri(_p(pos), _p(tri), n, kind, _p(scene), _p(codes), _p(ids), _p(nodes), _p(aabbs))
    return dict(scene=scene, codes=codes, ids=ids, nodes=nodes, aabbs=aabbs)


def lbvh_build_points(pos, kind=0):
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    n = pos.shape[0]
    scene = np.zeros(6, np.float32)
    codes = np.zeros(n, np.uint32)
    ids = np.zeros(n, np.uint32)
    nn = max(2 * n - 1, 0)
    nodes = np.full((nn, 4), -1, np.int32)
    aabbs = np.zeros((nn, 6), np.float32)
    lib().orc_lbvh_build_points(_p(pos), n, kind, _p(scene), _p(codes), _p(ids), _p(nodes), _p(aabbs))
    return dict(scene=scene, codes=codes, ids=ids, nodes=nodes, aabbs=aabbs)


def lbvh_build_edges(pos, edges, kind=0):
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    edges = np.ascontiguousarray(edges, dtype=np.uint32)
    n = edges.shape[0]
    scene = np.zeros(6, np.float32)
    codes = np.zeros(n, np.uint32)
    ids = np.zeros(n, np.uint32)
    nn = max(2 * n - 1, 0)
    nodes = np.full((nn, 4), -1, np.int32)
    aabbs = np.zeros((nn, 6), np.float32)
    lib().orc_lbvh_build_edges(_p(pos), _p(edges), n, kind, _p(scene), _p(codes), _p(ids), _p(nodes), _p(aabbs))
    return dict(scene=scene, codes=codes, ids=ids, nodes=nodes, aabbs=aabbs)


def refit_tri(pos, tri, ids, nodes):
    """Bottom-up boxes of an existing topology (nodes int32 [2n-1,4] with
    parents, ids uint32 [n]) over the given vertices; returns (nodes, aabbs)."""
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    tri = np.ascontiguousarray(tri, dtype=np.uint32)
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    nodes = np.ascontiguousarray(nodes, dtype=np.int32).copy()
    aabbs = np.zeros((nodes.shape[0], 6), np.float32)
    lib().orc_refit_tri(_p(pos), _p(tri), _p(ids), ids.size, _p(nodes), _p(aabbs))
    return nodes, aabbs


def karras(codes):
    codes = np.ascontiguousarray(codes, dtype=np.uint32)
    n = codes.size
    nodes = np.full((max(2 * n - 1, 0), 4), -1, np.int32)
    lib().orc_karras(_p(codes), n, _p(nodes))
    return nodes


def ref_lbvh_build(pos, tri=None):
    """The reference's programs run serially (kind: triangles if tri is [n,3],
    edges if tri is [n,2], points if tri is None)."""
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    if tri is not None:
        tri = np.ascontiguousarray(tri, dtype=np.uint32)
        n = tri.shape[0]
        kind = 0 if tri.shape[1] == 3 else 2
    else:
        n = pos.shape[0]
        kind = 1
    scene = np.zeros(6, np.float32)
    codes = np.zeros(n, np.uint32)
    ids = np.zeros(n, np.uint32)
    nodes = np.full((2 * n - 1, 4), -1, np.int32)
    aabbs = np.zeros((2 * n - 1, 6), np.float32)
    ref().ref_lbvh_build(kind, _p(pos), pos.shape[0], _p(tri), n, _p(scene), _p(codes), _p(ids), _p(nodes),
                         _p(aabbs))
    return dict(scene=scene, codes=codes, ids=ids, nodes=nodes, aabbs=aabbs)


USER_HIT_DTYPE = np.dtype([("prim", np.uint32), ("t", np.float32), ("u", np.float32)])


def lss_intersect(ray, v0, v1, cap0=True, cap1=True, exit_test=False):
    """intersectRayLSS restated: (hit, t, u) for one ray {o, tmin, d, tmax} and
    two float4 {xyz, radius} ends."""
    a = [np.ascontiguousarray(v, dtype=np.float32) for v in (ray, v0, v1)]
    t = np.zeros(1, np.float32)
    u = np.zeros(1, np.float32)
    hit = lib().orc_lss_intersect(_p(a[0]), _p(a[1]), _p(a[2]), int(cap0), int(cap1), int(exit_test), _p(t), _p(u))
    return bool(hit), float(t[0]), float(u[0])


def ref_lss_intersect(ray, v0, v1, cap0=True, cap1=True, exit_test=False):
    """The reference's own intersectRayLSS (compiled from its sources)."""
    a = [np.ascontiguousarray(v, dtype=np.float32) for v in (ray, v0, v1)]
    t = np.zeros(1, np.float32)
    u = np.zeros(1, np.float32)
    R = ref()
    R.ref_lss_intersect.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int] * 3 + [ctypes.c_void_p] * 2
    R.ref_lss_intersect.restype = ctypes.c_int
    hit = R.ref_lss_intersect(_p(a[0]), _p(a[1]), _p(a[2]), int(cap0), int(cap1), int(exit_test), _p(t), _p(u))
    return bool(hit), t[0], u[0]


def ref_lss_aabb(v0, v1, cap0, cap1):
    """The reference's own computeLssAabb: [lo.xyz, hi.xyz]."""
    a = [np.ascontiguousarray(v, dtype=np.float32) for v in (v0, v1)]
    lo = np.zeros(3, np.float32)
    hi = np.zeros(3, np.float32)
    R = ref()
    R.ref_lss_aabb.argtypes = [ctypes.c_void_p] * 2 + [ctypes.c_int] * 2 + [ctypes.c_void_p] * 2
    R.ref_lss_aabb(_p(a[0]), _p(a[1]), int(cap0), int(cap1), _p(lo), _p(hi))
    return np.concatenate([lo, hi])


def lss_bounds(verts, idx, cap0=True, cap1=True):
    verts = np.ascontiguousarray(verts, dtype=np.float32)
    idx = np.ascontiguousarray(idx, dtype=np.uint32)
    out = np.zeros((idx.shape[0], 6), np.float32)
    lib().orc_lss_bounds(_p(verts), _p(idx), idx.shape[0], int(cap0), int(cap1), _p(out))
    return out


def sphere_bounds(spheres):
    spheres = np.ascontiguousarray(spheres, dtype=np.float32)
    out = np.zeros((spheres.shape[0], 6), np.float32)
    lib().orc_sphere_bounds(_p(spheres), spheres.shape[0], _p(out))
    return out


def trace_user_brute(kind, prims, rays, idx=None, cap0=True, cap1=True, exit_test=False):
    """Closest hit over every sphere (kind 0, prims float4[n]) or LSS (kind 1,
    prims = vertices float4[], idx uint2[n]); ties to the lowest id."""
    prims = np.ascontiguousarray(prims, dtype=np.float32)
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
    idxa = None if idx is None else np.ascontiguousarray(idx, dtype=np.uint32)
    n = prims.shape[0] if kind == 0 else idxa.shape[0]
    hits = np.zeros(rays.shape[0], USER_HIT_DTYPE)
    lib().orc_trace_user_brute(kind, _p(prims), _p(idxa), n, int(cap0), int(cap1), int(exit_test), _p(rays),
                               rays.shape[0], _p(hits))
    return hits


def lbvh_build_boxes(boxes, kind=0):
    """LBVH over primitive boxes [n][6] {lo, hi} (oracle layout dict)."""
    boxes = np.ascontiguousarray(boxes, dtype=np.float32)
    n = boxes.shape[0]
    scene = np.zeros(6, np.float32)
    codes = np.zeros(n, np.uint32)
    ids = np.zeros(n, np.uint32)
    nn = max(2 * n - 1, 0)
    nodes = np.full((nn, 4), -1, np.int32)
    aabbs = np.zeros((nn, 6), np.float32)
    lib().orc_lbvh_build_boxes(_p(boxes), n, kind, _p(scene), _p(codes), _p(ids), _p(nodes), _p(aabbs))
    return dict(scene=scene, codes=codes, ids=ids, nodes=nodes, aabbs=aabbs)


INSTANCE_DTYPE = np.dtype([("transform", np.float32, (12,)), ("custom_mask", np.uint32),
                           ("geom_flags", np.uint32), ("blas", np.uint64)])
INST_HIT_DTYPE = np.dtype([("prim", np.uint32), ("t", np.float32), ("inst", np.uint32)])


def instance_inverse(m):
    """World-to-object 3x4 matrix of a row-major object-to-world one (None if singular)."""
    m = np.ascontiguousarray(m, dtype=np.float32).reshape(12)
    w = np.zeros(12, np.float32)
    return w if lib().orc_instance_inverse(_p(m), _p(w)) else None


def trace_instances_brute(instances, pos, tri, tri_off, rays, ray_mask=0xFF):
    """Closest hit over every triangle of every visible instance; ties to the
    lowest (instance, primitive); mesh-local primitive ids."""
    inst = np.ascontiguousarray(instances, dtype=INSTANCE_DTYPE)
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    tri = np.ascontiguousarray(tri, dtype=np.uint32)
    off = np.ascontiguousarray(tri_off, dtype=np.uint32)
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
    hits = np.zeros(rays.shape[0], INST_HIT_DTYPE)
    lib().orc_trace_instances_brute(_p(inst), inst.size, _p(pos), _p(tri), _p(off), off.size - 1, _p(rays),
                                    rays.shape[0], ray_mask, _p(hits))
    return hits


def trace_brute(pos, tri, rays):
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    tri = np.ascontiguousarray(tri, dtype=np.uint32)
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
    hits = np.zeros(rays.shape[0], HIT_DTYPE)
    lib().orc_trace_brute(_p(pos), _p(tri), tri.shape[0], _p(rays), rays.shape[0], _p(hits))
    return hits


def trace_lbvh(pos, tri, bvh, rays, anyhit=False):
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    tri = np.ascontiguousarray(tri, dtype=np.uint32)
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
    nodes = np.ascontiguousarray(bvh["nodes"], dtype=np.int32)
    aabbs = np.ascontiguousarray(bvh["aabbs"], dtype=np.float32)
    hits = np.zeros(rays.shape[0], HIT_DTYPE)
    lib().orc_trace_lbvh(_p(pos), _p(tri), tri.shape[0], _p(nodes), _p(aabbs), _p(rays), rays.shape[0],
                         1 if anyhit else 0, _p(hits))
    return hits


def trace_lbvh64(pos, tri, bvh, rays):
    """Closest hit through the same tree in FP64: (prim uint32[R], t float64[R])."""
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    tri = np.ascontiguousarray(tri, dtype=np.uint32)
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
    nodes = np.ascontiguousarray(bvh["nodes"], dtype=np.int32)
    aabbs = np.ascontiguousarray(bvh["aabbs"], dtype=np.float32)
    prim = np.zeros(rays.shape[0], np.uint32)
    t = np.zeros(rays.shape[0], np.float64)
    lib().orc_trace_lbvh64(_p(pos), _p(tri), tri.shape[0], _p(nodes), _p(aabbs), _p(rays), rays.shape[0], _p(prim),
                           _p(t))
    return prim, t


def isect64(ray, v0, v1, v2):
    a = [np.ascontiguousarray(v, dtype=np.float32) for v in (ray, v0, v1, v2)]
    t = np.zeros(1, np.float64)
    hit = lib().orc_isect_tri64(*[_p(v) for v in a], _p(t))
    return bool(hit), float(t[0])


def fp64_id_diagnostic(pos, tri, bvh, rays, prim32):
    """Rays whose FP32 closest id (prim32) differs from the FP64 closest id
    through the same tree, by kind:
      fp32_edge   the FP32 test hits a triangle that the FP64 test misses
                  (a ray through a shared edge or vertex; FP64 then reports
                  a triangle behind it, or a miss);
      fp64_edge   the FP64 test hits a triangle that the FP32 test misses;
      near_ties   both precisions hit both triangles, and their FP64
                  distances agree within 1e-6 relative;
      other       anything else (none is expected)."""
    prim32 = np.asarray(prim32, dtype=np.uint32)
    p64, t64v = trace_lbvh64(pos, tri, bvh, rays)
    diff = np.nonzero(p64 != prim32)[0]
    out = {"rays": int(prim32.size), "disagreements": int(diff.size), "fp32_edge": 0, "fp64_edge": 0,
           "near_ties": 0, "other": 0}
    pos3 = np.ascontiguousarray(pos, dtype=np.float32).reshape(-1, 3)
    tri3 = np.ascontiguousarray(tri, dtype=np.uint32).reshape(-1, 3)
    rays8 = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
    for r in diff:
        a, b = int(prim32[r]), int(p64[r])
        if a != 0xFFFFFFFF and not isect64(rays8[r], *pos3[tri3[a]])[0]:
            out["fp32_edge"] += 1
        elif b != 0xFFFFFFFF and not isect32(rays8[r], *pos3[tri3[b]])[0]:
            out["fp64_edge"] += 1
        elif a != 0xFFFFFFFF and b != 0xFFFFFFFF and \
                abs(isect64(rays8[r], *pos3[tri3[a]])[1] - t64v[r]) <= 1e-6 * abs(t64v[r]):
            out["near_ties"] += 1
        else:
            out["other"] += 1
    return out


def t64(ray, v0, v1, v2):
    a = [np.ascontiguousarray(v, dtype=np.float32) for v in (ray, v0, v1, v2)]
    return lib().orc_t64(*[_p(v) for v in a])


def isect32(ray, v0, v1, v2):
    a = [np.ascontiguousarray(v, dtype=np.float32) for v in (ray, v0, v1, v2)]
    t = np.zeros(1, np.float32)
    hit = lib().orc_isect_tri32(*[_p(v) for v in a], _p(t))
    return bool(hit), float(t[0])


# ---------------------------------------------------------------- solid cells
def _qw(verts, n):
    qw = np.zeros((8, 4), np.float32)
    qw[:n] = np.asarray(verts, np.float32).reshape(-1, 4)[:n]
    return qw


def solid_intersect(p, verts, n):
    """intersectPointSolid restated: (hit, rstw[4]) for a point and a cell's
    n float4 vertices {x, y, z, density}."""
    r = np.zeros(4, np.float32)
    p = np.ascontiguousarray(p, dtype=np.float32)
    h = lib().orc_solid_intersect(_p(p), _p(_qw(verts, n)), n, _p(r))
    return bool(h), r


def ref_solid_intersect(p, verts, n):
    """The reference's own intersectPointSolid (needs oracle/_ref)."""
    r = np.zeros(4, np.float32)
    p = np.ascontiguousarray(p, dtype=np.float32)
    h = ref().ref_solid_intersect(_p(p), _p(_qw(verts, n)), n, _p(r))
    return bool(h), r


def solid_bounds(verts, idx, types):
    verts = np.ascontiguousarray(verts, dtype=np.float32)
    idx = np.ascontiguousarray(idx, dtype=np.uint32)
    types = np.ascontiguousarray(types, dtype=np.uint8)
    out = np.zeros((types.size, 8), np.float32)
    lib().orc_solid_bounds(_p(verts), _p(idx), _p(types), types.size, _p(out))
    return out


def ref_solid_bounds(verts, idx, types):
    """The reference's own SolidBounds (needs oracle/_ref)."""
    verts = np.ascontiguousarray(verts, dtype=np.float32)
    idx = np.ascontiguousarray(idx, dtype=np.uint32)
    types = np.ascontiguousarray(types, dtype=np.uint8)
    out = np.zeros((types.size, 8), np.float32)
    ref().ref_solid_bounds(_p(verts), _p(idx), _p(types), types.size, _p(out))
    return out


def solid_locate_brute(verts, idx, types, points):
    """(cell u32 [P], kind u32 [P], rstw f32 [P, 4]) by exhaustive search."""
    verts = np.ascontiguousarray(verts, dtype=np.float32)
    idx = np.ascontiguousarray(idx, dtype=np.uint32)
    types = np.ascontiguousarray(types, dtype=np.uint8)
    pts = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 4)
    cell = np.zeros(pts.shape[0], np.uint32)
    kind = np.zeros(pts.shape[0], np.uint32)
    rstw = np.zeros((pts.shape[0], 4), np.float32)
    lib().orc_solid_locate_brute(_p(verts), _p(idx), _p(types), types.size, _p(pts), pts.shape[0], _p(cell),
                                 _p(kind), _p(rstw))
    return cell, kind, rstw


def num_threads():
    return lib().orc_num_threads()
