"""Parity at the full sizes of the batched-build and quantised configurations,
through properties that do not depend on size (the oracle finishes these
sizes only on samples):

* batched build, 4,096 meshes of log-uniform size in [64, 65,536] (about 40M
  triangles), each mesh of the small-LBVH distribution in its own unit cube:
  sampled meshes' arrays bit-identical to the oracle's build of that mesh
  alone, and their hits identical to the oracle's traversal of that tree;
  batched binary and batched quantised traversal identical on every ray;
  t within 1e-6 of FP64 on a seeded 1 % of the hits;
* quantised wide BVH, 16,777,216 triangles of a 64-cluster Gaussian mixture,
  16,777,216 rays aimed at the unit cube: binary and quantised traversal
  identical on every ray (closest: ids and t bits; any hit: occlusion), ids
  of a seeded sample identical to the oracle's FP32 traversal of the same
  tree, t within 1e-6 of FP64 on a seeded 1 % of the hits.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
T_REL_TOL = 1e-6


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32) if a.dtype == np.float32 else a


def _t64_check(hits, rays, vert, tri_of_hit, frac=0.01, seed=0):
    """Largest relative error of the reported t against the FP64 plane
    distance on a seeded fraction of the hit rays; vert(tri index array)
    returns the [k, 3, 3] vertices (float64)."""
    hit = np.nonzero(hits[:, 0] != -1)[0]
    idx = np.sort(np.random.default_rng(seed).choice(hit, size=max(1, int(frac * hit.size)), replace=False))
    v = vert(tri_of_hit(idx, hits[idx, 0].astype(np.int64)))
    r = rays[idx].astype(np.float64)
    o, d = r[:, 0:3], r[:, 4:7]
    n = np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0])
    t64 = np.einsum("ij,ij->i", v[:, 0] - o, n) / np.einsum("ij,ij->i", d, n)
    t32 = hits[idx, 1].view(np.float32).astype(np.float64)
    return float((np.abs(t32 - t64) / np.abs(t64)).max()), idx.size


def test_batched_build_full_size(cuda):
    import torch
    from gprt_b200 import api
    rng = np.random.default_rng(2024)
    sizes = np.floor(np.exp(rng.uniform(np.log(64), np.log(65536), size=4096))).astype(np.int64)
    off = np.zeros(sizes.size + 1, np.int64)
    off[1:] = np.cumsum(sizes)
    n = int(off[-1])
    assert 30_000_000 < n < 50_000_000
    toff = torch.from_numpy(off.astype(np.uint32).view(np.int32)).cuda()
    pos, tri = api.gen_soup(n, seed=31, sigma=0.002, tri_off=toff, meshes=sizes.size, spacing=2.0)
    b = api.BatchLbvh(off)
    api.batch_build_triangles(pos, tri, b)
    rays = api.gen_rays(n, seed=32, ray_off=toff, meshes=sizes.size, boxes=b.scene)
    hb = api.batch_trace(b, rays, toff).cpu().numpy()
    w = api.wide_build(b)
    hw = api.wide_trace(w, rays, toff).cpu().numpy()
    assert np.array_equal(hw, hb)
    assert (hb[:, 0] != -1).sum() > n // 20
    rays_h = rays.cpu().numpy()
    pos_h = pos.cpu().numpy()
    # sampled meshes against the oracle: build arrays and hits
    sample = sorted({int(np.argmin(sizes)), int(np.argmax(sizes))} | set(rng.choice(sizes.size, 10, replace=False)))
    for m in sample:
        bgn, end = int(off[m]), int(off[m + 1])
        lp = pos_h[3 * bgn:3 * end]
        lt = np.arange(3 * (end - bgn), dtype=np.uint32).reshape(-1, 3)
        e = oracle.lbvh_build_tri(lp, lt)
        h = b.mesh_host(m)
        for k in ("scene", "codes", "ids", "nodes", "aabbs"):
            assert np.array_equal(_bits(h[k]), _bits(e[k].reshape(h[k].shape))), (m, k)
        exp = oracle.trace_lbvh(lp, lt, e, rays_h[bgn:end])
        got = hb[bgn:end]
        assert np.array_equal(got[:, 0].view(np.uint32), exp["prim"]), m
        hit = exp["prim"] != 0xFFFFFFFF
        assert np.array_equal(got[hit, 1].view(np.uint32), _bits(exp["t"][hit])), m
    worst, k = _t64_check(hb, rays_h, lambda t: pos_h.reshape(-1, 3, 3)[t].astype(np.float64),
                          lambda idx, prim: off[np.searchsorted(off, idx, side="right") - 1] + prim)
    assert k > 1000 and worst <= T_REL_TOL, worst


def test_quantised_wide_full_size(cuda):
    import torch
    from gprt_b200 import api
    n = 16_777_216
    pos, tri = api.gen_mixture(n, clusters=64, seed=41)
    rays = api.gen_rays(n, seed=42)
    b = api.lbvh_build_triangles(pos, tri)
    w = api.wide_build(b)
    hb = api.trace(b, rays).cpu().numpy()
    hw = api.wide_trace(w, rays).cpu().numpy()
    assert np.array_equal(hw, hb)
    assert (hb[:, 0] != -1).sum() > n // 4
    ab = api.trace(b, rays, anyhit=True).cpu().numpy()
    aw = api.wide_trace(w, rays, anyhit=True).cpu().numpy()
    assert np.array_equal(ab[:, 0] != -1, hb[:, 0] != -1)
    assert np.array_equal(aw[:, 0] != -1, hb[:, 0] != -1)
    pos_h, rays_h = pos.cpu().numpy(), rays.cpu().numpy()
    tri_h = tri.cpu().numpy().view(np.uint32)
    # ids of a seeded sample against the oracle's FP32 traversal of the same tree
    idx = np.sort(np.random.default_rng(43).choice(n, size=20000, replace=False))
    exp = oracle.trace_lbvh(pos_h, tri_h, b.host(), rays_h[idx])
    assert np.array_equal(hb[idx, 0].view(np.uint32), exp["prim"])
    hit = exp["prim"] != 0xFFFFFFFF
    assert np.array_equal(hb[idx[hit], 1].view(np.uint32), _bits(exp["t"][hit]))
    worst, k = _t64_check(hb, rays_h, lambda t: pos_h[tri_h[t].reshape(-1)].reshape(-1, 3, 3).astype(np.float64),
                          lambda idx_, prim: prim)
    assert k > 1000 and worst <= T_REL_TOL, worst
