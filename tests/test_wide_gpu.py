"""8-wide quantised BVH through the C ABI.

Structure: every decoded child box (exact decode in FP64 of origin + q * 2^e)
contains the exact box of what it covers, and every triangle appears in
exactly one leaf.  Traversal: hits identical (ids and t bits) to the binary
traversal and therefore to the oracle, closest and any hit, plain and
batched."""
import numpy as np
import pytest

import oracle
from gprt_b200 import scenes

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _check_structure(d, n_leaves_expected, meshes=1):
    p, e, imask, cb, lb, meta, qlo, qhi = (d[k] for k in ("p", "e", "imask", "child_base", "leaf_base", "meta",
                                                         "qlo", "qhi"))
    leaf = d["leaf"].reshape(-1, 3, 4)
    seen_leaf = np.zeros(n_leaves_expected, np.int32)
    seen_node = np.zeros(d["count"], np.int32)

    def visit(w):
        seen_node[w] += 1
        s = np.ldexp(1.0, e[w].astype(np.int64))
        lo_all = np.full(3, np.inf)
        hi_all = np.full(3, -np.inf)
        for c in range(8):
            if meta[w, c] == 0xFF:
                continue
            dlo = p[w].astype(np.float64) + qlo[w, :, c].astype(np.float64) * s
            dhi = p[w].astype(np.float64) + qhi[w, :, c].astype(np.float64) * s
            if (imask[w] >> c) & 1:
                blo, bhi = visit(int(cb[w] + meta[w, c]))
            else:
                li = int(lb[w] + meta[w, c])
                seen_leaf[li] += 1
                v = leaf[li, :, :3].astype(np.float64)
                blo, bhi = v.min(axis=0), v.max(axis=0)
            assert (dlo <= blo).all() and (dhi >= bhi).all(), (w, c)
            lo_all = np.minimum(lo_all, blo)
            hi_all = np.maximum(hi_all, bhi)
        return lo_all, hi_all

    import sys
    sys.setrecursionlimit(100000)
    for m in range(meshes):
        visit(int(d["roots"][m]))
    assert (seen_leaf == 1).all()
    assert (seen_node == 1).all()


@pytest.mark.parametrize("n", [1, 2, 3, 9, 1000, 20000])
def test_wide_structure_is_conservative_and_complete(cuda, n):
    import torch
    from gprt_b200 import api
    pos, tri = scenes.soup(n, seed=40 + n, sigma=0.01)
    b = api.lbvh_build_triangles(torch.from_numpy(pos).cuda(), torch.from_numpy(tri.view(np.int32)).cuda())
    w = api.wide_build(b)
    d = api.wide_decode(w)
    assert d["count"] <= max(n - 1, 1)
    _check_structure(d, n)
    ids = np.sort(d["leaf"][:, 3].view(np.uint32))
    assert np.array_equal(ids, np.arange(n, dtype=np.uint32))


@pytest.mark.parametrize("n,m", [(1, 2000), (2, 2000), (5000, 30000), (262144, 65536)])
@pytest.mark.parametrize("anyhit", [False, True])
def test_wide_trace_equals_binary(cuda, n, m, anyhit):
    import torch
    from gprt_b200 import api
    pos, tri = scenes.soup(n, seed=50 + n, sigma=0.002 if n > 1000 else 0.1)
    rays = scenes.rays(m, seed=51 + n)
    rt = torch.from_numpy(rays).cuda()
    b = api.lbvh_build_triangles(torch.from_numpy(pos).cuda(), torch.from_numpy(tri.view(np.int32)).cuda())
    w = api.wide_build(b)
    gb = api.hits_numpy(api.trace(b, rt, anyhit=anyhit))
    gw = api.hits_numpy(api.wide_trace(w, rt, anyhit=anyhit))
    if anyhit:
        assert np.array_equal(gw["prim"] != 0xFFFFFFFF, gb["prim"] != 0xFFFFFFFF)
        for r in np.nonzero(gw["prim"] != 0xFFFFFFFF)[0][:1000]:
            v = pos[tri[gw["prim"][r]]]
            assert oracle.isect32(rays[r], v[0], v[1], v[2])[0]
    else:
        assert np.array_equal(gw["prim"], gb["prim"])
        hit = gw["prim"] != 0xFFFFFFFF
        assert np.array_equal(_bits(gw["t"][hit]), _bits(gb["t"][hit]))
        if n <= 5000:
            exp = oracle.trace_brute(pos, tri, rays)
            assert np.array_equal(gw["prim"], exp["prim"])


def test_wide_batched_equals_batched_binary(cuda):
    import torch
    from gprt_b200 import api
    rng = np.random.default_rng(77)
    sizes = np.concatenate([[1, 2, 3], rng.integers(64, 5000, size=30)])
    pos, tri, off, rays, roff = scenes.batch(sizes, seed=6, sigma=0.01, rays_per_tri=2)
    bb = api.BatchLbvh(off)
    api.batch_build_triangles(torch.from_numpy(pos).cuda(), torch.from_numpy(tri.view(np.int32)).cuda(), bb)
    w = api.wide_build(bb)
    rt = torch.from_numpy(rays).cuda()
    ro = torch.from_numpy(roff.astype(np.uint32).view(np.int32)).cuda()
    d = api.wide_decode(w)
    _check_structure(d, int(off[-1]), meshes=len(sizes))
    for anyhit in (False, True):
        gb = api.hits_numpy(api.batch_trace(bb, rt, ro, anyhit=anyhit))
        gw = api.hits_numpy(api.wide_trace(w, rt, ro, anyhit=anyhit))
        if anyhit:
            assert np.array_equal(gw["prim"] != 0xFFFFFFFF, gb["prim"] != 0xFFFFFFFF)
        else:
            assert np.array_equal(gw["prim"], gb["prim"])
            hit = gw["prim"] != 0xFFFFFFFF
            assert hit.sum() > 1000
            assert np.array_equal(_bits(gw["t"][hit]), _bits(gb["t"][hit]))


def _axis_rays(pos, m, seed):
    """Rays with one or two zero direction components: along +-x/y/z from
    outside the unit cube, some with origin coordinates equal to vertex
    coordinates (rays in vertex / edge planes), and diagonal rays in the
    coordinate planes."""
    rng = np.random.default_rng(seed)
    r = np.zeros((m, 8), np.float32)
    r[:, 7] = np.inf
    for i in range(m):
        kind = i % 4
        a = rng.integers(0, 3)
        o = rng.random(3).astype(np.float32)
        if kind == 1:  # origin on a vertex's coordinates
            v = pos[rng.integers(0, len(pos))]
            o = v.copy()
        d = np.zeros(3, np.float32)
        if kind < 3:
            sgn = 1.0 if rng.random() < 0.5 else -1.0
            d[a] = sgn
            o[a] = -1.0 if sgn > 0 else 2.0
        else:
            b = (a + 1) % 3
            d[a], d[b] = 0.70710677, -0.70710677 if rng.random() < 0.5 else 0.70710677
            o[a] = -1.0
            o[b] = 2.0 if d[b] < 0 else -1.0
        r[i, :3], r[i, 4:7] = o, d
    return r


@pytest.mark.parametrize("anyhit", [False, True])
def test_wide_trace_axis_parallel_rays(cuda, anyhit):
    import torch
    from gprt_b200 import api
    pos, tri = scenes.soup(3000, seed=81, sigma=0.05)
    rays = _axis_rays(pos, 8000, 82)
    rt = torch.from_numpy(rays).cuda()
    b = api.lbvh_build_triangles(torch.from_numpy(pos).cuda(), torch.from_numpy(tri.view(np.int32)).cuda())
    w = api.wide_build(b)
    gb = api.hits_numpy(api.trace(b, rt, anyhit=anyhit))
    gw = api.hits_numpy(api.wide_trace(w, rt, anyhit=anyhit))
    if anyhit:
        assert np.array_equal(gw["prim"] != 0xFFFFFFFF, gb["prim"] != 0xFFFFFFFF)
    else:
        exp = oracle.trace_brute(pos, tri, rays)
        assert np.array_equal(gw["prim"], exp["prim"])
        assert np.array_equal(gw["prim"], gb["prim"])
        hit = gw["prim"] != 0xFFFFFFFF
        assert hit.sum() > 500
        assert np.array_equal(_bits(gw["t"][hit]), _bits(gb["t"][hit]))


def _layer_scene(k=16, zs=(0.25, 0.5, 0.75), dup_every=7):
    """Stacked grids of quads split into triangles sharing edges and
    vertices, with every dup_every-th triangle duplicated (coplanar copies:
    the lower id must win a tie)."""
    xs = np.linspace(0, 1, k + 1, dtype=np.float32)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    verts, tris = [], []
    for li, z in enumerate(zs):
        base = li * X.size
        verts.append(np.stack([X.ravel(), Y.ravel(), np.full(X.size, z, np.float32)], 1))
        for i in range(k):
            for j in range(k):
                a, b = i * (k + 1) + j, (i + 1) * (k + 1) + j
                c, d = (i + 1) * (k + 1) + j + 1, i * (k + 1) + j + 1
                tris += [[base + a, base + b, base + c], [base + a, base + c, base + d]]
    tris = np.array(tris, np.uint32)
    return np.concatenate(verts).astype(np.float32), np.concatenate([tris, tris[::dup_every]]), xs


def test_wide_closest_ties_and_zero_t(cuda):
    # The closest-hit kernel folds queued triangle tests into a (t, id) key:
    # ties (coplanar copies, shared vertices and edges) must still go to the
    # lowest id, and t = 0 (origin on a triangle) must count, whether the
    # triangle test returns +0 or -0.
    import torch
    from gprt_b200 import api
    verts, tris, xs = _layer_scene()
    rng = np.random.default_rng(5)
    m = 6000
    rays = np.zeros((m, 8), np.float32)
    rays[:, :3] = rng.random((m, 3))
    rays[:, 4:7] = rng.normal(size=(m, 3))
    rays[:, 7] = np.inf
    extra = []
    for x in xs[1:-1:3]:
        for y in xs[1:-1:3]:
            extra.append([x, y, 0.5, 0.0, 0.0, 0.0, -1.0, np.inf])  # starts on a layer, through a vertex: t = 0
            extra.append([x, y, 0.5, 0.0, 0.0, 0.0, 1.0, np.inf])  # the other way: t = 0 as well
            extra.append([x, y, 0.9, 0.0, 0.0, 0.0, -1.0, np.inf])  # through three layers' vertices
    rays = np.concatenate([rays, np.array(extra, np.float32)])
    rt = torch.from_numpy(rays).cuda()
    b = api.lbvh_build_triangles(torch.from_numpy(verts).cuda(), torch.from_numpy(tris.view(np.int32)).cuda())
    w = api.wide_build(b)
    gw = api.hits_numpy(api.wide_trace(w, rt))
    gb = api.hits_numpy(api.trace(b, rt))
    exp = oracle.trace_brute(verts, tris, rays)
    assert np.array_equal(gw["prim"], exp["prim"])
    assert np.array_equal(gw["prim"], gb["prim"])
    hit = gw["prim"] != 0xFFFFFFFF
    assert np.array_equal(_bits(gw["t"][hit]), _bits(gb["t"][hit]))
    assert hit.mean() > 0.4
    n_extra = len(extra)
    assert (gw["prim"][-n_extra:] != 0xFFFFFFFF).all()
    assert (gw["t"][-n_extra::3] == 0.0).all() and (gw["t"][-n_extra + 1::3] == 0.0).all()
