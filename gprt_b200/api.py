"""Torch-tensor wrappers over the C ABI (include/gprtcu.h).

Every function takes CUDA tensors, enqueues on torch's current stream and
returns without synchronising unless it documents otherwise.  Scratch is
allocated by torch's caching allocator when not supplied.
"""
import ctypes

import torch

from . import GprtcuError, lib


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _check(status, where):
    if status != 0:
        raise GprtcuError(status, where)


def scratch(nbytes, device=None):
    """A 256-byte aligned device scratch buffer (torch allocations are)."""
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device or "cuda")


def scratch_status(buf):
    """Device-side status word of a scratch buffer (synchronises the stream)."""
    v = ctypes.c_int(0)
    _check(lib().gprtcuScratchStatus(_ptr(buf), _stream(), ctypes.byref(v)), "gprtcuScratchStatus")
    return v.value


def _need_cuda(*ts):
    for t in ts:
        if t is not None and not t.is_cuda:
            raise ValueError("gprt_b200 operates on CUDA tensors only (no CPU path)")


# ---------------------------------------------------------------- scan
def scan_scratch_size(n):
    return lib().gprtcuScanScratchSize(int(n))


def exclusive_sum(inp, out=None, total=None, scr=None, inclusive=False):
    """uint32 prefix sum of `inp` (int32/uint32 tensor viewed as uint32) into `out`.

    Returns (out, total_tensor) where total_tensor is a 1-element device tensor.
    """
    _need_cuda(inp)
    n = inp.numel()
    if out is None:
        out = torch.empty_like(inp)
    if total is None:
        total = torch.empty(1, dtype=torch.int32, device=inp.device)
    if scr is None:
        scr = scratch(scan_scratch_size(n), inp.device)
    f = lib().gprtcuInclusiveSumU32 if inclusive else lib().gprtcuExclusiveSumU32
    _check(f(_ptr(inp), _ptr(out), n, _ptr(total), _ptr(scr), scr.numel(), _stream()),
           "gprtcuInclusiveSumU32" if inclusive else "gprtcuExclusiveSumU32")
    return out, total


def inclusive_sum(inp, out=None, total=None, scr=None):
    return exclusive_sum(inp, out, total, scr, inclusive=True)


def partition(inp, select_positive=True, out=None, count=None, scr=None, select_only=False):
    _need_cuda(inp)
    n = inp.numel()
    if out is None:
        out = torch.zeros_like(inp)
    if count is None:
        count = torch.empty(1, dtype=torch.int32, device=inp.device)
    if scr is None:
        scr = scratch(scan_scratch_size(n), inp.device)
    f = lib().gprtcuSelectI32 if select_only else lib().gprtcuPartitionI32
    _check(f(_ptr(inp), _ptr(out), n, 1 if select_positive else 0, _ptr(count), _ptr(scr), scr.numel(), _stream()),
           "gprtcuSelectI32" if select_only else "gprtcuPartitionI32")
    return out, count


def select(inp, select_positive=True, out=None, count=None, scr=None):
    return partition(inp, select_positive, out, count, scr, select_only=True)


# ---------------------------------------------------------------- sort
_SORT_FN = {
    (4, 0): "gprtcuSortKeysU32",
    (4, 4): "gprtcuSortPairsU32",
    (4, 8): "gprtcuSortPairsU32U64",
    (8, 0): "gprtcuSortKeysU64",
    (8, 4): "gprtcuSortPairsU64",
    (8, 8): "gprtcuSortPairsU64U64",
}


def sort_scratch_size(n, key_bytes, value_bytes):
    return lib().gprtcuSortScratchSize(int(n), int(key_bytes), int(value_bytes))


def sort(keys, values=None, begin_bit=0, end_bit=None, scr=None):
    """Stable in-place radix sort of `keys` (int32/uint32 or int64/uint64
    tensors, compared as unsigned) carrying `values` (optional, 4 or 8 bytes)."""
    _need_cuda(keys, values)
    kw = keys.element_size()
    vw = 0 if values is None else values.element_size()
    if values is not None and values.numel() != keys.numel():
        raise ValueError("keys and values differ in size")
    n = keys.numel()
    if end_bit is None:
        end_bit = 8 * kw
    if scr is None:
        scr = scratch(sort_scratch_size(n, kw, vw), keys.device)
    name = _SORT_FN[(kw, vw)]
    f = getattr(lib(), name)
    if vw:
        st = f(_ptr(keys), _ptr(values), n, begin_bit, end_bit, _ptr(scr), scr.numel(), _stream())
    else:
        st = f(_ptr(keys), n, begin_bit, end_bit, _ptr(scr), scr.numel(), _stream())
    _check(st, name)
    return keys, values


class SortConfig(ctypes.Structure):
    """gprtcuSortConfig (include/gprtcu.h): digit bits, keys per tile, warps per block."""
    _fields_ = [("digitBits", ctypes.c_int32), ("tile", ctypes.c_int32), ("warps", ctypes.c_int32)]

    def tuple(self):
        return (self.digitBits, self.tile, self.warps)


def sort_configs():
    """Every shape of the sort's tuning grid as (digit bits, tile, warps)."""
    out = []
    for i in range(lib().gprtcuSortConfigCount()):
        c = SortConfig()
        _check(lib().gprtcuSortConfigAt(i, ctypes.byref(c)), "gprtcuSortConfigAt")
        out.append(c.tuple())
    return out


def sort_get_config(key_bytes, value_bytes):
    c = SortConfig()
    _check(lib().gprtcuSortGetConfig(key_bytes, value_bytes, ctypes.byref(c)), "gprtcuSortGetConfig")
    return c.tuple()


def sort_set_config(key_bytes, value_bytes, cfg):
    """Install shape `cfg` (a tuple) for the type pair; None restores the default."""
    arg = None if cfg is None else ctypes.byref(SortConfig(*cfg))
    _check(lib().gprtcuSortSetConfig(key_bytes, value_bytes, arg), "gprtcuSortSetConfig")


def sort_with_config(keys, values, cfg, begin_bit=0, end_bit=None, scr=None):
    """One sort with an explicit shape (keys/values as in sort())."""
    _need_cuda(keys, values)
    kw = keys.element_size()
    vw = 0 if values is None else values.element_size()
    n = keys.numel()
    if end_bit is None:
        end_bit = 8 * kw
    if scr is None:
        scr = scratch(sort_scratch_size(n, kw, vw), keys.device)
    _check(lib().gprtcuSortWithConfig(_ptr(keys), _ptr(values), n, kw, vw, begin_bit, end_bit,
                                      ctypes.byref(SortConfig(*cfg)), _ptr(scr), scr.numel(), _stream()),
           "gprtcuSortWithConfig")
    return keys, values


def sort_autotune(key_bytes, value_bytes, n, end_bit=None, sample=None, repeats=3):
    """Time every shape on this device, install the fastest for the type pair.
    Returns (best shape, {shape: median ms or None if it failed})."""
    if end_bit is None:
        end_bit = 8 * key_bytes
    count = lib().gprtcuSortConfigCount()
    ms = (ctypes.c_float * count)()
    best = SortConfig()
    _check(lib().gprtcuSortAutotune(key_bytes, value_bytes, int(n), end_bit, _ptr(sample), repeats, ms,
                                    ctypes.byref(best), _stream()), "gprtcuSortAutotune")
    times = {cfg: (None if ms[i] < 0 else float(ms[i])) for i, cfg in enumerate(sort_configs())}
    return best.tuple(), times


# ---------------------------------------------------------------- LBVH + trace
class LbvhDesc(ctypes.Structure):
    """gprtcuLbvh (include/gprtcu.h)."""
    _fields_ = [("numPrims", ctypes.c_uint32), ("codes", ctypes.c_void_p), ("ids", ctypes.c_void_p),
                ("nodes", ctypes.c_void_p), ("aabbs", ctypes.c_void_p), ("sceneBounds", ctypes.c_void_p),
                ("rootBox", ctypes.c_void_p), ("bvh2", ctypes.c_void_p), ("leafTris", ctypes.c_void_p)]


class Lbvh:
    """Device arrays of one LBVH (torch tensors) plus its C descriptor."""

    def __init__(self, n, device="cuda", with_aabbs=True, with_traversal=True):
        self.n = int(n)
        nn = max(2 * self.n - 1, 1)
        dev = torch.device(device)
        self.codes = torch.empty(self.n, dtype=torch.int32, device=dev)
        self.ids = torch.empty(self.n, dtype=torch.int32, device=dev)
        self.nodes = torch.empty((nn, 4), dtype=torch.int32, device=dev)
        self.aabbs = torch.empty((nn, 6), dtype=torch.float32, device=dev) if with_aabbs else None
        self.scene = torch.empty(6, dtype=torch.float32, device=dev)
        self.root = torch.empty(6, dtype=torch.float32, device=dev)
        self.bvh2 = torch.empty((max(self.n - 1, 1), 16), dtype=torch.float32, device=dev) if with_traversal else None
        self.leaf = torch.empty((self.n, 12), dtype=torch.float32, device=dev) if with_traversal else None
        self.scratch = scratch(lib().gprtcuLbvhScratchSize(self.n), dev)
        self.desc = LbvhDesc(0, _p(self.codes), _p(self.ids), _p(self.nodes), _p(self.aabbs), _p(self.scene),
                             _p(self.root), _p(self.bvh2), _p(self.leaf))

    def host(self):
        """Copy the reference-layout arrays back (numpy dict, oracle layout)."""
        import numpy as np
        torch.cuda.synchronize()
        d = dict(codes=self.codes.cpu().numpy().view(np.uint32), ids=self.ids.cpu().numpy().view(np.uint32),
                 nodes=self.nodes.cpu().numpy(), scene=self.scene.cpu().numpy())
        if self.aabbs is not None:
            d["aabbs"] = self.aabbs.cpu().numpy()
        return d


def _p(t):
    return t.data_ptr() if t is not None else None


def lbvh_build_triangles(pos, tri, bvh=None, code_kind=0):
    """Build over float32 positions [V,3] and uint32/int32 indices [N,3] (CUDA tensors)."""
    _need_cuda(pos, tri)
    n = tri.shape[0]
    if bvh is None:
        bvh = Lbvh(n, pos.device)
    st = lib().gprtcuLbvhBuildTriangles(_ptr(pos), _ptr(tri), n, code_kind, ctypes.byref(bvh.desc), _ptr(bvh.scratch),
                                        bvh.scratch.numel(), _stream())
    _check(st, "gprtcuLbvhBuildTriangles")
    return bvh


def lbvh_build_points(pos, bvh=None, code_kind=0):
    _need_cuda(pos)
    n = pos.shape[0]
    if bvh is None:
        bvh = Lbvh(n, pos.device, with_traversal=False)
    st = lib().gprtcuLbvhBuildPoints(_ptr(pos), n, code_kind, ctypes.byref(bvh.desc), _ptr(bvh.scratch),
                                     bvh.scratch.numel(), _stream())
    _check(st, "gprtcuLbvhBuildPoints")
    return bvh


def lbvh_build_edges(pos, edges, bvh=None, code_kind=0):
    """Edge LBVH over float32 positions [V,3] and uint32/int32 endpoints [N,2]."""
    _need_cuda(pos, edges)
    n = edges.shape[0]
    if bvh is None:
        bvh = Lbvh(n, pos.device, with_traversal=False)
    st = lib().gprtcuLbvhBuildEdges(_ptr(pos), _ptr(edges), n, code_kind, ctypes.byref(bvh.desc), _ptr(bvh.scratch),
                                    bvh.scratch.numel(), _stream())
    _check(st, "gprtcuLbvhBuildEdges")
    return bvh


def lbvh_refit_triangles(pos, tri, bvh, tri_off=None):
    """Refit an existing triangle LBVH (Lbvh, or BatchLbvh with its offsets) to moved vertices."""
    _need_cuda(pos, tri)
    meshes = 1 if tri_off is None else tri_off.numel() - 1
    st = lib().gprtcuLbvhRefitTriangles(_ptr(pos), _ptr(tri), _ptr(tri_off), meshes, ctypes.byref(bvh.desc),
                                        _ptr(bvh.scratch), bvh.scratch.numel(), _stream())
    _check(st, "gprtcuLbvhRefitTriangles")
    return bvh


def trace(bvh, rays, hits=None, anyhit=False, scr=None):
    """rays: float32 [R, 8] {org.xyz, tmin, dir.xyz, tmax}; returns hits int32 [R, 2] {prim, t bits}."""
    _need_cuda(rays)
    nr = rays.shape[0]
    if hits is None:
        hits = torch.empty((nr, 2), dtype=torch.int32, device=rays.device)
    if scr is None:
        scr = scratch(lib().gprtcuTraceScratchSize(), rays.device)
    f = lib().gprtcuTraceAny if anyhit else lib().gprtcuTraceClosest
    _check(f(ctypes.byref(bvh.desc), _ptr(rays), nr, _ptr(hits), _ptr(scr), scr.numel(), _stream()),
           "gprtcuTraceAny" if anyhit else "gprtcuTraceClosest")
    return hits


# ---------------------------------------------------------------- spheres / LSS
def sphere_bounds(spheres, out=None):
    """Boxes [n, 6] of spheres float32 [n, 4] {center, radius}."""
    _need_cuda(spheres)
    n = spheres.shape[0]
    if out is None:
        out = torch.empty((n, 6), dtype=torch.float32, device=spheres.device)
    _check(lib().gprtcuSphereBounds(_ptr(spheres), n, _ptr(out), _stream()), "gprtcuSphereBounds")
    return out


def lss_bounds(verts, idx, endcap0=True, endcap1=True, out=None):
    """Boxes [n, 6] of swept-sphere segments (verts float32 [V, 4], idx int32 [n, 2])."""
    _need_cuda(verts, idx)
    n = idx.shape[0]
    if out is None:
        out = torch.empty((n, 6), dtype=torch.float32, device=verts.device)
    _check(lib().gprtcuLssBounds(_ptr(verts), _ptr(idx), n, int(endcap0), int(endcap1), _ptr(out), _stream()),
           "gprtcuLssBounds")
    return out


def lbvh_build_boxes(boxes, bvh=None, code_kind=0):
    """LBVH with traversal nodes over primitive boxes [n, 6]."""
    _need_cuda(boxes)
    n = boxes.shape[0]
    if bvh is None:
        bvh = Lbvh(n, boxes.device)
    st = lib().gprtcuLbvhBuildBoxes(_ptr(boxes), n, code_kind, ctypes.byref(bvh.desc), _ptr(bvh.scratch),
                                    bvh.scratch.numel(), _stream())
    _check(st, "gprtcuLbvhBuildBoxes")
    return bvh


def trace_spheres(bvh, spheres, rays, hits=None, u=None, anyhit=False, exit_test=False, scr=None):
    _need_cuda(spheres, rays)
    nr = rays.shape[0]
    if hits is None:
        hits = torch.empty((nr, 2), dtype=torch.int32, device=rays.device)
    if scr is None:
        scr = scratch(lib().gprtcuTraceScratchSize(), rays.device)
    _check(lib().gprtcuTraceSpheres(ctypes.byref(bvh.desc), _ptr(spheres), _ptr(rays), nr, int(anyhit), int(exit_test),
                                    _ptr(hits), _ptr(u), _ptr(scr), scr.numel(), _stream()), "gprtcuTraceSpheres")
    return hits


def trace_lss(bvh, verts, idx, rays, endcap0=True, endcap1=True, hits=None, u=None, anyhit=False, exit_test=False,
              scr=None):
    _need_cuda(verts, idx, rays)
    nr = rays.shape[0]
    if hits is None:
        hits = torch.empty((nr, 2), dtype=torch.int32, device=rays.device)
    if scr is None:
        scr = scratch(lib().gprtcuTraceScratchSize(), rays.device)
    _check(lib().gprtcuTraceLss(ctypes.byref(bvh.desc), _ptr(verts), _ptr(idx), int(endcap0), int(endcap1), _ptr(rays),
                                nr, int(anyhit), int(exit_test), _ptr(hits), _ptr(u), _ptr(scr), scr.numel(),
                                _stream()), "gprtcuTraceLss")
    return hits


# ---------------------------------------------------------------- instancing
INSTANCE_DTYPE = [("transform", "<f4", (12,)), ("custom_mask", "<u4"), ("geom_flags", "<u4"), ("blas", "<u8")]


# ---------------------------------------------------------------- solid cells
class SolidsDesc(ctypes.Structure):
    """gprtcuSolids (include/gprtcu.h)."""
    _fields_ = [("vertices", ctypes.c_void_p), ("indices", ctypes.c_void_p), ("types", ctypes.c_void_p),
                ("numCells", ctypes.c_uint32), ("vertexStride", ctypes.c_uint32), ("indexStride", ctypes.c_uint32),
                ("typeStride", ctypes.c_uint32)]


class Solids:
    """A volume mesh on the device: vertices float32 [V, 4] {x, y, z, density},
    indices int32/uint32 [C, 8] (unused slots ignored), types uint8 [C]."""

    def __init__(self, vertices, indices, types):
        _need_cuda(vertices, indices, types)
        self.vertices, self.indices, self.types = vertices, indices, types
        self.n = int(types.numel())
        self.desc = SolidsDesc(_p(vertices), _p(indices), _p(types), self.n, 0, 0, 0)


def solid_bounds(solids, aabbs=None, boxes=None):
    """(aabbs float32 [C, 8] in the reference's layout, boxes float32 [C, 6])."""
    dev = solids.types.device
    if aabbs is None:
        aabbs = torch.empty((solids.n, 8), dtype=torch.float32, device=dev)
    if boxes is None:
        boxes = torch.empty((solids.n, 6), dtype=torch.float32, device=dev)
    _check(lib().gprtcuSolidBounds(ctypes.byref(solids.desc), _ptr(aabbs), _ptr(boxes), _stream()),
           "gprtcuSolidBounds")
    return aabbs, boxes


def locate_solid_points(bvh, solids, points, hits=None, rstw=None, scr=None):
    """points float32 [P, 4]; returns (hits int32 [P, 2] {cell, kind}, rstw float32 [P, 4])."""
    _need_cuda(points)
    npts = points.shape[0]
    if hits is None:
        hits = torch.empty((npts, 2), dtype=torch.int32, device=points.device)
    if rstw is None:
        rstw = torch.empty((npts, 4), dtype=torch.float32, device=points.device)
    if scr is None:
        scr = scratch(lib().gprtcuTraceScratchSize(), points.device)
    _check(lib().gprtcuLocateSolidPoints(ctypes.byref(bvh.desc), ctypes.byref(solids.desc), _ptr(points), npts,
                                         _ptr(hits), _ptr(rstw), _ptr(scr), scr.numel(), _stream()),
           "gprtcuLocateSolidPoints")
    return hits, rstw


def instances_tensor(records, device="cuda"):
    """Device copy (uint8 [n, 64]) of a numpy array of INSTANCE_DTYPE records."""
    import numpy as np
    rec = np.ascontiguousarray(records, dtype=np.dtype(INSTANCE_DTYPE))
    return torch.from_numpy(rec.view(np.uint8).reshape(-1, 64).copy()).to(device)


class Tlas:
    """Top level over instances: world-to-object matrices, world boxes and a
    box LBVH over them (see gprtcuInstancesPrepare)."""

    def __init__(self, instances, root_boxes, meshes):
        n = instances.shape[0]
        dev = instances.device
        self.instances, self.root_boxes, self.meshes = instances, root_boxes, meshes
        self.w2o = torch.empty((n, 12), dtype=torch.float32, device=dev)
        self.boxes = torch.empty((n, 6), dtype=torch.float32, device=dev)
        self.bvh = Lbvh(n, dev)
        self.build()

    def build(self):
        """Recompute matrices, world boxes and the top-level LBVH in place
        (after the instance records or the bottom-level boxes changed)."""
        n = self.instances.shape[0]
        _check(lib().gprtcuInstancesPrepare(_ptr(self.instances), n, _ptr(self.root_boxes), self.meshes,
                                            _ptr(self.w2o), _ptr(self.boxes), _stream()), "gprtcuInstancesPrepare")
        lbvh_build_boxes(self.boxes, self.bvh)


def trace_instances(tlas, blas, rays, tri_off=None, meshes=1, ray_mask=0xFF, hits=None, inst=None, anyhit=False,
                    scr=None):
    """Closest/any hit through a Tlas over the meshes of `blas` (Lbvh or BatchLbvh)."""
    _need_cuda(rays)
    nr = rays.shape[0]
    if hits is None:
        hits = torch.empty((nr, 2), dtype=torch.int32, device=rays.device)
    if inst is None:
        inst = torch.empty(nr, dtype=torch.int32, device=rays.device)
    if scr is None:
        scr = scratch(lib().gprtcuTraceScratchSize(), rays.device)
    _check(lib().gprtcuTraceInstances(ctypes.byref(tlas.bvh.desc), _ptr(tlas.instances), _ptr(tlas.w2o),
                                      ctypes.byref(blas.desc), _ptr(tri_off), meshes, _ptr(rays), nr, ray_mask,
                                      int(anyhit), _ptr(hits), _ptr(inst), _ptr(scr), scr.numel(), _stream()),
           "gprtcuTraceInstances")
    return hits, inst


def hits_numpy(hits):
    """Device hits -> numpy structured array {prim uint32, t float32}."""
    import numpy as np
    h = hits.cpu().numpy()
    out = np.zeros(h.shape[0], dtype=[("prim", np.uint32), ("t", np.float32)])
    out["prim"] = h[:, 0].view(np.uint32)
    out["t"] = h[:, 1].view(np.float32)
    return out


# ---------------------------------------------------------------- batched
class BatchLbvh:
    """Concatenated per-mesh LBVHs of a batch (see gprtcuBatchBuildTriangles)."""

    def __init__(self, tri_offsets_host, device="cuda", with_aabbs=True):
        import numpy as np
        off = np.asarray(tri_offsets_host, dtype=np.int64)
        self.meshes = int(off.size - 1)
        self.n = int(off[-1])
        dev = torch.device(device)
        self.tri_off = torch.from_numpy(off.astype(np.uint32).view(np.int32)).to(dev)
        nn = 2 * self.n - self.meshes
        ni = max(self.n - self.meshes, 1)
        self.codes = torch.empty(self.n, dtype=torch.int32, device=dev)
        self.ids = torch.empty(self.n, dtype=torch.int32, device=dev)
        self.nodes = torch.empty((nn, 4), dtype=torch.int32, device=dev)
        self.aabbs = torch.empty((nn, 6), dtype=torch.float32, device=dev) if with_aabbs else None
        self.scene = torch.empty((self.meshes, 6), dtype=torch.float32, device=dev)
        self.root = torch.empty((self.meshes, 6), dtype=torch.float32, device=dev)
        self.bvh2 = torch.empty((ni, 16), dtype=torch.float32, device=dev)
        self.leaf = torch.empty((self.n, 12), dtype=torch.float32, device=dev)
        self.scratch = scratch(lib().gprtcuBatchScratchSize(self.meshes, self.n), dev)
        self.desc = LbvhDesc(0, _p(self.codes), _p(self.ids), _p(self.nodes), _p(self.aabbs), _p(self.scene),
                             _p(self.root), _p(self.bvh2), _p(self.leaf))
        self.off_host = off

    def mesh_host(self, m):
        """Reference-layout arrays of mesh m (numpy), as a plain build of that mesh returns them."""
        import numpy as np
        torch.cuda.synchronize()
        b, e = int(self.off_host[m]), int(self.off_host[m + 1])
        nb, ne = 2 * b - m, 2 * e - (m + 1)
        d = dict(codes=self.codes[b:e].cpu().numpy().view(np.uint32), ids=self.ids[b:e].cpu().numpy().view(np.uint32),
                 nodes=self.nodes[nb:ne].cpu().numpy(), scene=self.scene[m].cpu().numpy())
        if self.aabbs is not None:
            d["aabbs"] = self.aabbs[nb:ne].cpu().numpy()
        return d


def batch_build_triangles(pos, tri, batch, code_kind=0):
    _need_cuda(pos, tri)
    st = lib().gprtcuBatchBuildTriangles(_ptr(pos), _ptr(tri), _ptr(batch.tri_off), batch.meshes, batch.n, code_kind,
                                         ctypes.byref(batch.desc), _ptr(batch.scratch), batch.scratch.numel(),
                                         _stream())
    _check(st, "gprtcuBatchBuildTriangles")
    return batch


def batch_trace(batch, rays, ray_off, hits=None, anyhit=False, scr=None):
    """rays float32 [R,8]; ray_off device int32/uint32 [meshes+1]."""
    _need_cuda(rays, ray_off)
    nr = rays.shape[0]
    if hits is None:
        hits = torch.empty((nr, 2), dtype=torch.int32, device=rays.device)
    if scr is None:
        scr = scratch(lib().gprtcuTraceScratchSize(), rays.device)
    st = lib().gprtcuBatchTrace(ctypes.byref(batch.desc), _ptr(batch.tri_off), _ptr(ray_off), batch.meshes, _ptr(rays),
                                nr, 1 if anyhit else 0, _ptr(hits), _ptr(scr), scr.numel(), _stream())
    _check(st, "gprtcuBatchTrace")
    return hits


# ---------------------------------------------------------------- wide (8-wide quantised) BVH
class WideDesc(ctypes.Structure):
    """gprtcuWideBvh (include/gprtcu.h)."""
    _fields_ = [("nodes", ctypes.c_void_p), ("leafTris", ctypes.c_void_p), ("roots", ctypes.c_void_p),
                ("numNodes", ctypes.c_void_p), ("capacity", ctypes.c_uint32)]


class WideBvh:
    def __init__(self, n, meshes=1, device="cuda"):
        dev = torch.device(device)
        self.n, self.meshes = int(n), int(meshes)
        self.nodes = torch.zeros((self.n, 20), dtype=torch.int32, device=dev)  # 80 B per node
        self.leaf = torch.empty((self.n, 12), dtype=torch.float32, device=dev)
        self.roots = torch.empty(self.meshes, dtype=torch.int32, device=dev)
        self.count = torch.zeros(1, dtype=torch.int32, device=dev)
        self.scratch = scratch(lib().gprtcuWideScratchSize(self.meshes, self.n), dev)
        self.desc = WideDesc(_p(self.nodes), _p(self.leaf), _p(self.roots), _p(self.count), self.n)


def wide_build(binary, tri_off=None, wide=None):
    """Collapse a binary Lbvh / BatchLbvh into the 8-wide quantised form."""
    meshes = getattr(binary, "meshes", 1)
    n = binary.n
    if wide is None:
        wide = WideBvh(n, meshes, binary.codes.device)
    toff = tri_off if tri_off is not None else getattr(binary, "tri_off", None)
    st = lib().gprtcuWideBuild(ctypes.byref(binary.desc), _ptr(toff) if meshes > 1 else None, meshes,
                               ctypes.byref(wide.desc), _ptr(wide.scratch), wide.scratch.numel(), _stream())
    _check(st, "gprtcuWideBuild")
    return wide


def wide_trace(wide, rays, ray_off=None, hits=None, anyhit=False, scr=None):
    _need_cuda(rays)
    nr = rays.shape[0]
    if hits is None:
        hits = torch.empty((nr, 2), dtype=torch.int32, device=rays.device)
    if scr is None:
        scr = scratch(lib().gprtcuTraceScratchSize(), rays.device)
    st = lib().gprtcuWideTrace(ctypes.byref(wide.desc), _ptr(ray_off) if wide.meshes > 1 else None, wide.meshes,
                               _ptr(rays), nr, 1 if anyhit else 0, _ptr(hits), _ptr(scr), scr.numel(), _stream())
    _check(st, "gprtcuWideTrace")
    return hits


def wide_decode(wide):
    """Host copy of the wide nodes as numpy structured fields (tests)."""
    import numpy as np
    torch.cuda.synchronize()
    cnt = int(wide.count.item())
    raw = wide.nodes[:cnt].cpu().numpy().view(np.uint8).reshape(cnt, 80)
    f = raw[:, 0:12].copy().view(np.float32).reshape(cnt, 3)
    e = raw[:, 12:15].copy().view(np.int8).astype(np.int32)
    imask = raw[:, 15].astype(np.uint32)
    cb = raw[:, 16:20].copy().view(np.uint32).ravel()
    lb = raw[:, 20:24].copy().view(np.uint32).ravel()
    meta = raw[:, 24:32]
    qlo = raw[:, 32:56].reshape(cnt, 3, 8)
    qhi = raw[:, 56:80].reshape(cnt, 3, 8)
    return dict(count=cnt, p=f, e=e, imask=imask, child_base=cb, leaf_base=lb, meta=meta, qlo=qlo, qhi=qhi,
                roots=wide.roots.cpu().numpy(), leaf=wide.leaf.cpu().numpy())


# ---------------------------------------------------------------- device scene generators
def gen_soup(n, seed=0, sigma=0.002, tri_off=None, meshes=1, spacing=2.0, device="cuda"):
    pos = torch.empty((3 * n, 3), dtype=torch.float32, device=device)
    tri = torch.empty((n, 3), dtype=torch.int32, device=device)
    _check(lib().gprtcuGenSoup(n, seed, sigma, _ptr(tri_off), meshes, spacing, _ptr(pos), _ptr(tri), _stream()),
           "gprtcuGenSoup")
    return pos, tri


def gen_mixture(n, clusters=64, seed=0, edge_sigma=0.001, device="cuda"):
    pos = torch.empty((3 * n, 3), dtype=torch.float32, device=device)
    tri = torch.empty((n, 3), dtype=torch.int32, device=device)
    _check(lib().gprtcuGenMixture(n, clusters, seed, edge_sigma, _ptr(pos), _ptr(tri), _stream()), "gprtcuGenMixture")
    return pos, tri


def gen_rays(nrays, seed=1, ray_off=None, meshes=1, boxes=None, device="cuda"):
    rays = torch.empty((nrays, 8), dtype=torch.float32, device=device)
    _check(lib().gprtcuGenRays(nrays, seed, _ptr(ray_off), meshes, _ptr(boxes), _ptr(rays), _stream()),
           "gprtcuGenRays")
    return rays
