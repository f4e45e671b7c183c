"""LBVH build and traversal on the GPU through the C ABI.

Build: codes, ids, nodes and boxes bit-exact against the fixtures made by the
reference's own LBVH programs and against the oracle.  Trace: hit primitive
ids exact against the oracle's FP32 watertight traversal (ties to the lowest
id), hit t within 1e-6 relative of the FP64 plane-equation distance."""
import os

import numpy as np
import pytest

import oracle
from gprt_b200 import scenes

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
T_REL_TOL = 1e-6


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32) if a.dtype == np.float32 else a


def _build(torch, pos, tri, kind=0):
    from gprt_b200 import api
    p = torch.from_numpy(np.ascontiguousarray(pos, np.float32)).cuda()
    t = torch.from_numpy(np.ascontiguousarray(tri, np.uint32).view(np.int32)).cuda()
    bvh = api.lbvh_build_triangles(p, t, code_kind=kind)
    return bvh, p, t


def test_build_matches_reference_fixtures(cuda):
    import torch
    g = np.load(os.path.join(GOLD, "lbvh_ref.npz"))
    cases = sorted({k.rsplit("_", 1)[0] for k in g.files if k.endswith("_nodes") and k.startswith("tri")})
    assert len(cases) >= 8
    for c in cases:
        bvh, _, _ = _build(torch, g[c + "_pos"], g[c + "_tri"])
        h = bvh.host()
        for k in ("scene", "codes", "ids", "nodes", "aabbs"):
            exp = g[c + "_" + k].reshape(h[k].shape)
            assert np.array_equal(_bits(h[k]), _bits(exp)), (c, k)


def test_points_build_matches_reference_fixture(cuda):
    import torch
    from gprt_b200 import api
    g = np.load(os.path.join(GOLD, "lbvh_ref.npz"))
    p = torch.from_numpy(g["pts42_pos"]).cuda()
    h = api.lbvh_build_points(p).host()
    for k in ("scene", "codes", "ids", "nodes", "aabbs"):
        assert np.array_equal(_bits(h[k]), _bits(g["pts42_" + k].reshape(h[k].shape))), k
    # extent beyond FLT_MAX: every code collapses to x = 0
    pts = np.array([[-3e38, 0, 0], [3e38, 1, 1], [1e38, 0.5, 0.25], [0, 1, 0]], np.float32)
    h = api.lbvh_build_points(torch.from_numpy(pts).cuda()).host()
    e = oracle.lbvh_build_points(pts)
    for k in ("codes", "ids", "nodes"):
        assert np.array_equal(h[k], e[k].reshape(h[k].shape)), k


@pytest.mark.parametrize("n", [1, 2, 3, 5, 64, 1000, 4097, 65537, 262144])
@pytest.mark.parametrize("kind", [0, 1])
def test_build_matches_oracle(cuda, n, kind):
    import torch
    pos, tri = scenes.soup(n, seed=n + 17 * kind)
    bvh, _, _ = _build(torch, pos, tri, kind)
    h = bvh.host()
    e = oracle.lbvh_build_tri(pos, tri, kind)
    for k in ("scene", "codes", "ids", "nodes", "aabbs"):
        assert np.array_equal(_bits(h[k]), _bits(e[k].reshape(h[k].shape))), (n, kind, k)


def test_build_duplicate_codes_and_shared_vertices(cuda):
    import torch
    rng = np.random.default_rng(8)
    n = 5000
    c = (np.floor(rng.random((n, 3)) * 2) / 2).astype(np.float32)  # heavy duplicate codes
    pos = np.repeat(c, 3, axis=0) + np.float32(0)
    tri = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    h = _build(torch, pos, tri)[0].host()
    e = oracle.lbvh_build_tri(pos, tri)
    for k in ("codes", "ids", "nodes", "aabbs"):
        assert np.array_equal(_bits(h[k]), _bits(e[k].reshape(h[k].shape))), k
    grid = rng.random((300, 3), dtype=np.float32)
    tri = rng.integers(0, 300, size=(2000, 3)).astype(np.uint32)
    h = _build(torch, grid, tri)[0].host()
    e = oracle.lbvh_build_tri(grid, tri)
    for k in ("codes", "ids", "nodes", "aabbs"):
        assert np.array_equal(_bits(h[k]), _bits(e[k].reshape(h[k].shape))), k


def _check_hits(got, exp, pos, tri, rays, tol=T_REL_TOL):
    assert np.array_equal(got["prim"], exp["prim"])
    hit = got["prim"] != 0xFFFFFFFF
    assert np.array_equal(_bits(got["t"][hit]), _bits(exp["t"][hit]))  # same double-float refinement
    # accuracy against FP64 on (a sample of) the hits
    idx = np.nonzero(hit)[0]
    if idx.size > 3000:
        idx = np.random.default_rng(0).choice(idx, 3000, replace=False)
    worst = 0.0
    for r in idx:
        p = got["prim"][r]
        v = pos[tri[p]]
        t64 = oracle.t64(rays[r], v[0], v[1], v[2])
        worst = max(worst, abs(float(got["t"][r]) - t64) / abs(t64))
    assert worst <= tol, worst
    return worst


@pytest.mark.parametrize("n,m", [(1, 1000), (2, 1000), (17, 4000), (5000, 20000), (262144, 65536)])
def test_trace_closest_matches_oracle(cuda, n, m):
    import torch
    from gprt_b200 import api
    pos, tri = scenes.soup(n, seed=3 + n, sigma=0.002 if n > 1000 else 0.1)
    rays = scenes.rays(m, seed=4 + n)
    bvh, _, _ = _build(torch, pos, tri)
    got = api.hits_numpy(api.trace(bvh, torch.from_numpy(rays).cuda()))
    e = oracle.lbvh_build_tri(pos, tri)
    exp = oracle.trace_lbvh(pos, tri, e, rays)
    _check_hits(got, exp, pos, tri, rays)
    assert (got["prim"] != 0xFFFFFFFF).sum() > 0 or n < 3


def test_trace_matches_brute_force(cuda):
    import torch
    from gprt_b200 import api
    pos, tri = scenes.soup(3000, seed=21, sigma=0.02)
    rays = scenes.rays(5000, seed=22)
    bvh, _, _ = _build(torch, pos, tri)
    got = api.hits_numpy(api.trace(bvh, torch.from_numpy(rays).cuda()))
    exp = oracle.trace_brute(pos, tri, rays)
    assert np.array_equal(got["prim"], exp["prim"])
    assert (exp["prim"] != 0xFFFFFFFF).sum() > 100


def test_trace_anyhit(cuda):
    import torch
    from gprt_b200 import api
    pos, tri = scenes.soup(20000, seed=31)
    rays = scenes.rays(20000, seed=32)
    bvh, _, _ = _build(torch, pos, tri)
    rt = torch.from_numpy(rays).cuda()
    closest = api.hits_numpy(api.trace(bvh, rt))
    anyh = api.hits_numpy(api.trace(bvh, rt, anyhit=True))
    occl = anyh["prim"] != 0xFFFFFFFF
    assert np.array_equal(occl, closest["prim"] != 0xFFFFFFFF)
    for r in np.nonzero(occl)[0][:2000]:
        v = pos[tri[anyh["prim"][r]]]
        ok, t = oracle.isect32(rays[r], v[0], v[1], v[2])
        assert ok


def test_trace_edge_cases(cuda):
    import torch
    from gprt_b200 import api
    # closed grid of quads at z = 0.5 split into triangles sharing edges and
    # vertices; rays aimed exactly at shared vertices/edges must hit (no leaks)
    k = 16
    xs = np.linspace(0, 1, k + 1, dtype=np.float32)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    verts = np.stack([X.ravel(), Y.ravel(), np.full(X.size, 0.5, np.float32)], 1).astype(np.float32)
    tris = []
    for i in range(k):
        for j in range(k):
            a, b, c, d = i * (k + 1) + j, (i + 1) * (k + 1) + j, (i + 1) * (k + 1) + j + 1, i * (k + 1) + j + 1
            tris += [[a, b, c], [a, c, d]]
    tris = np.array(tris, np.uint32)
    # duplicate the first 10 triangles (coplanar duplicates: lowest id must win)
    tris = np.concatenate([tris, tris[:10]])
    rays = []
    for x in xs[1:-1]:
        for y in xs[1:-1]:
            rays.append([x, y, 2.0, 0.0, 0.0, 0.0, -1.0, np.inf])  # axis-parallel, through a vertex
            rays.append([x, (y + xs[1] / 2), 2.0, 0.0, 0.0, 0.0, -1.0, np.inf])  # through an edge
    rays.append([0.01, 0.01, 0.5, 0.0, 1.0, 0.0, 0.0, np.inf])  # in the plane: grazing
    rays.append([0.3, 0.3, 2.0, 0.0, 0.0, 0.0, -1.0, 1.0])  # tmax stops short of the plane
    rays = np.array(rays, np.float32)
    bvh, _, _ = _build(torch, verts, tris)
    got = api.hits_numpy(api.trace(bvh, torch.from_numpy(rays).cuda()))
    exp = oracle.trace_brute(verts, tris, rays)
    assert np.array_equal(got["prim"], exp["prim"])
    assert (got["prim"][:-2] != 0xFFFFFFFF).all()  # watertight: every vertex/edge ray hits
    assert got["prim"][-1] == 0xFFFFFFFF
    assert np.allclose(got["t"][:-2], 1.5, rtol=1e-6)
    # degenerate triangles never hit
    dpos = np.array([[0, 0, 0.5], [1, 1, 0.5], [2, 2, 0.5], [0, 0, 0.5], [0, 0, 0.5], [0, 0, 0.5]], np.float32)
    dtri = np.array([[0, 1, 2], [3, 4, 5]], np.uint32)
    r = np.array([[0.5, 0.5, 2, 0, 0, 0, -1, np.inf], [0, 0, 2, 0, 0, 0, -1, np.inf]], np.float32)
    bvh, _, _ = _build(torch, dpos, dtri)
    got = api.hits_numpy(api.trace(bvh, torch.from_numpy(r).cuda()))
    assert (got["prim"] == 0xFFFFFFFF).all()


def test_edge_build_matches_reference_fixtures_and_oracle(cuda):
    import torch
    from gprt_b200 import api
    g = np.load(os.path.join(GOLD, "lbvh_ref.npz"))
    cases = sorted({k.rsplit("_", 1)[0] for k in g.files if k.startswith("edge") and k.endswith("_nodes")})
    assert len(cases) >= 5
    for c in cases:
        p = torch.from_numpy(g[c + "_pos"]).cuda()
        e = torch.from_numpy(g[c + "_edges"].view(np.int32)).cuda()
        h = api.lbvh_build_edges(p, e).host()
        for k in ("scene", "codes", "ids", "nodes", "aabbs"):
            assert np.array_equal(_bits(h[k]), _bits(g[c + "_" + k].reshape(h[k].shape))), (c, k)
    rng = np.random.default_rng(31)
    for n in (5, 4097, 100000):
        pos = rng.random((n // 2 + 3, 3), dtype=np.float32)
        edges = rng.integers(0, pos.shape[0], size=(n, 2)).astype(np.uint32)
        for kind in (0, 1):
            h = api.lbvh_build_edges(torch.from_numpy(pos).cuda(), torch.from_numpy(edges.view(np.int32)).cuda(),
                                     code_kind=kind).host()
            ex = oracle.lbvh_build_edges(pos, edges, kind)
            for k in ("scene", "codes", "ids", "nodes", "aabbs"):
                assert np.array_equal(_bits(h[k]), _bits(ex[k].reshape(h[k].shape))), (n, kind, k)


@pytest.mark.parametrize("n", [2, 1000, 262144])
def test_refit_after_moving_vertices(cuda, n):
    # refit-only update: topology and leaf order kept, every box recomputed
    # bottom-up from the moved vertices (bit-exact vs the oracle's refit of the
    # same topology), and traversal stays exact against the oracle
    import torch
    from gprt_b200 import api
    pos, tri = scenes.soup(n, seed=60 + n, sigma=0.002 if n > 1000 else 0.05)
    bvh, p, t = _build(torch, pos, tri)
    before = bvh.host()
    rng = np.random.default_rng(61)
    moved = (pos + rng.normal(0.0, 0.01, pos.shape)).astype(np.float32)
    p.copy_(torch.from_numpy(moved))
    api.lbvh_refit_triangles(p, t, bvh)
    after = bvh.host()
    assert np.array_equal(after["ids"], before["ids"])
    assert np.array_equal(after["nodes"][:, :3], before["nodes"][:, :3])
    _, exp_boxes = oracle.refit_tri(moved, tri, before["ids"], before["nodes"])
    assert np.array_equal(_bits(after["aabbs"]), _bits(exp_boxes))
    rays = scenes.rays(20000, seed=62)
    got = api.hits_numpy(api.trace(bvh, torch.from_numpy(rays).cuda()))
    exp = oracle.trace_brute(moved, tri, rays)
    assert np.array_equal(got["prim"], exp["prim"])
