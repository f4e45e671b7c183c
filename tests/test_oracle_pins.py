"""The oracle against the reference: golden fixtures made by the reference's
own code (tests/golden/make_golden.py), the reference tests' known answers,
and -- where the reference sources are mounted -- the reference-compiled
checker directly.  CPU only."""
import os

import numpy as np
import pytest

import oracle

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _bits(a):
    return a.view(np.uint32) if a.dtype == np.float32 else a


@pytest.fixture(scope="module")
def lbvh_gold():
    return np.load(os.path.join(GOLD, "lbvh_ref.npz"))


def _cases(g):
    return sorted({k.rsplit("_", 1)[0] for k in g.files if k.endswith("_nodes")})


def test_lbvh_matches_reference_fixtures(lbvh_gold):
    g = lbvh_gold
    cases = _cases(g)
    assert len(cases) >= 9
    for c in cases:
        if c.startswith("pts"):
            r = oracle.lbvh_build_points(g[c + "_pos"])
        elif c.startswith("edge"):
            r = oracle.lbvh_build_edges(g[c + "_pos"], g[c + "_edges"])
        else:
            r = oracle.lbvh_build_tri(g[c + "_pos"], g[c + "_tri"])
        for k in ("scene", "codes", "ids", "nodes", "aabbs"):
            exp = g[c + "_" + k].reshape(r[k].shape)
            assert np.array_equal(_bits(r[k]), _bits(exp)), (c, k)


def test_overflowing_extent_gives_zero_codes():
    # tests/t04-swBVH draws coordinates from [-1e38, 1e38]; there the extent
    # stays finite (< FLT_MAX).  Push it past FLT_MAX: max - min = inf, every
    # normalised coordinate is 0 or inf/inf = NaN, both clamp to 0.
    pts = np.array([[-3e38, 0, 0], [3e38, 1, 1], [1e38, 0.5, 0.25], [0, 1, 0]], np.float32)
    r = oracle.lbvh_build_points(pts)
    assert np.isinf(np.float32(r["scene"][3]) - np.float32(r["scene"][0]))
    xs = [c & 0x09249249 for c in r["codes"]]  # x bits only
    assert all(x == 0 for x in xs)
    if oracle.ref_available():
        b = oracle.ref_lbvh_build(pts)
        assert np.array_equal(b["codes"], r["codes"]) and np.array_equal(b["nodes"], r["nodes"].reshape(b["nodes"].shape))


def test_hilbert_matches_reference_fixture():
    g = np.load(os.path.join(GOLD, "hilbert_ref.npz"))
    got = np.array([oracle.hilbert3d(*c) for c in g["coords"]], np.uint32)
    assert np.array_equal(got, g["codes"])


def test_morton_known_answers():
    assert oracle.morton3d(0, 0, 0) == 0
    assert oracle.morton3d(1, 0, 0) == 1
    assert oracle.morton3d(0, 1, 0) == 2
    assert oracle.morton3d(0, 0, 1) == 4
    assert oracle.morton3d(1023, 1023, 1023) == (1 << 30) - 1
    assert oracle.morton3d(1023, 0, 0) == 0x09249249


@pytest.mark.skipif(not oracle.ref_available(), reason="reference sources not compiled here")
def test_lbvh_matches_reference_compiled_random():
    rng = np.random.default_rng(5)
    for n in (5, 300, 20000):
        c = rng.random((n, 3), dtype=np.float32)
        pos = (np.repeat(c, 3, axis=0) + rng.normal(0, 0.01, (3 * n, 3))).astype(np.float32)
        tri = rng.permutation(3 * n).astype(np.uint32).reshape(n, 3)
        a = oracle.lbvh_build_tri(pos, tri)
        b = oracle.ref_lbvh_build(pos, tri)
        for k in a:
            assert np.array_equal(_bits(a[k]), _bits(b[k].reshape(a[k].shape))), (n, k)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference sources not compiled here")
def test_hilbert_matches_reference_compiled_exhaustive_slices():
    R = oracle.ref()
    L = oracle.lib()
    for x in range(0, 1024, 31):
        for y in range(0, 1024, 37):
            for z in (0, 5, 1023, (x * 7 + y) & 1023):
                assert L.orc_hilbert3d(x, y, z) == R.ref_hilbert3d(x, y, z)


def test_sort_matches_t02_oracle_fixture():
    g = np.load(os.path.join(GOLD, "sortscan.npz"))
    k, v = oracle.sort(g["keys"], np.arange(g["keys"].size, dtype=np.uint32))
    assert np.array_equal(k, g["keys_sorted"]) and np.array_equal(v, g["vals_sorted"])
    k = oracle.sort(g["keys"])
    assert np.array_equal(k, g["keys_sorted"])
    k, v = oracle.sort(g["keys64"], np.arange(g["keys64"].size, dtype=np.uint32))
    assert np.array_equal(k, g["keys64_sorted"]) and np.array_equal(v, g["vals64_sorted"])


def test_scan_matches_t03_oracle_fixture():
    g = np.load(os.path.join(GOLD, "sortscan.npz"))
    out, total = oracle.scan(g["scan_in"])
    assert np.array_equal(out, g["scan_excl"]) and total == int(g["scan_total"])
    out, _ = oracle.scan(g["big_in"])
    assert np.array_equal(out, g["big_excl"])
    inc, total2 = oracle.scan(g["scan_in"], inclusive=True)
    assert np.array_equal(inc, g["scan_excl"] + g["scan_in"]) and total2 == total


def test_scan_t03_all_ones_known_answer():
    # tests/t03-bufferScans/hostCode.cpp:38-81: all ones -> excl[i] = i, total N.
    for k in (2, 3, 17, 101):
        n = 9973 * k
        out, total = oracle.scan(np.ones(n, np.uint32))
        assert total == n and np.array_equal(out, np.arange(n, dtype=np.uint32))


def test_partition_select_t03_known_answer():
    g = np.load(os.path.join(GOLD, "sortscan.npz"))
    p, t = oracle.partition(g["t03_in"], True, True)
    assert np.array_equal(p, g["t03_partition"]) and t == int(g["t03_total"])
    s, t2 = oracle.partition(g["t03_in"], True, False)
    assert np.array_equal(s[:t2], g["t03_select"][:t2]) and t2 == t


def test_karras_structure_invariants():
    rng = np.random.default_rng(3)
    for n in (2, 3, 10, 1000):
        codes = np.sort(rng.integers(0, 1 << 30, size=n).astype(np.uint32))
        codes[n // 2:n // 2 + n // 4] = codes[n // 2]
        nodes = oracle.karras(codes)
        inner = n - 1
        parent_count = np.zeros(2 * n - 1, np.int64)
        for i in range(inner):
            l, r = nodes[i, 0], nodes[i, 1]
            assert nodes[l, 2] == i and nodes[r, 2] == i
            parent_count[l] += 1
            parent_count[r] += 1
        assert parent_count[0] == 0 and (parent_count[1:] == 1).all()
        assert nodes[0, 2] == -1


def test_edge_lbvh_matches_reference_fixtures(lbvh_gold):
    # ComputeEdgeBounds / ComputeEdgeMortonCodes / BuildEdgeHierarchy run from
    # the reference's own sources (tests/golden/make_golden.py)
    g = lbvh_gold
    cases = sorted({k.rsplit("_", 1)[0] for k in g.files if k.startswith("edge") and k.endswith("_nodes")})
    assert len(cases) >= 5
    for c in cases:
        r = oracle.lbvh_build_edges(g[c + "_pos"], g[c + "_edges"])
        for k in ("scene", "codes", "ids", "nodes", "aabbs"):
            exp = g[c + "_" + k].reshape(r[k].shape)
            assert np.array_equal(np.ascontiguousarray(r[k]).view(np.uint32),
                                  np.ascontiguousarray(exp).view(np.uint32)), (c, k)


def test_sphere_and_swept_sphere_math_matches_reference_fixture():
    # intersectRayLSS / computeLssAabb (gprt/gprt_fallbacks.slang:45-144,168-213)
    # compiled from the reference sources: hit flag, t and u bit-exact, boxes
    # bit-exact, for every combination of end caps and exit test
    g = np.load(os.path.join(GOLD, "lss_ref.npz"))
    rays, v0, v1 = g["rays"], g["v0"], g["v1"]
    total_hits = 0
    for cap0 in (0, 1):
        for cap1 in (0, 1):
            box = oracle.lss_bounds(np.concatenate([v0, v1]),
                                    np.stack([np.arange(len(v0)), len(v0) + np.arange(len(v0))], 1), cap0, cap1)
            assert np.array_equal(_bits(box), _bits(g["c%d%d_aabb" % (cap0, cap1)]))
            for ex in (0, 1):
                key = "c%d%d_x%d" % (cap0, cap1, ex)
                for i in range(len(rays)):
                    hit, t, u = oracle.lss_intersect(rays[i], v0[i], v1[i], cap0, cap1, ex)
                    assert hit == bool(g[key + "_hit"][i]), (key, i)
                    if hit:
                        total_hits += 1
                        assert np.float32(t).view(np.uint32) == g[key + "_t"][i].view(np.uint32), (key, i)
                        assert np.float32(u).view(np.uint32) == g[key + "_u"][i].view(np.uint32), (key, i)
    assert total_hits > 5000
    # SphereBounds (gprt/gprt_fallbacks.slang:263-283): center -/+ max(r, 0)
    s = np.array([[0.5, -1.0, 2.0, 0.25], [1.0, 1.0, 1.0, -3.0]], np.float32)
    assert np.array_equal(oracle.sphere_bounds(s), np.array([[0.25, -1.25, 1.75, 0.75, -0.75, 2.25],
                                                             [1, 1, 1, 1, 1, 1]], np.float32))


def test_solid_cell_math_matches_reference_fixture():
    # intersectPointSolid and SolidBounds (gprt/gprt_fallbacks.slang:409-502)
    # compiled from the reference sources: hit flag and (r, s, t, density)
    # bit-exact on every point, box words bit-exact
    g = np.load(os.path.join(GOLD, "solid_ref.npz"))
    verts, idx, types, pts = g["verts"], g["idx"], g["types"], g["points"]
    ppc = pts.shape[0] // types.size
    hits = 0
    for q in range(pts.shape[0]):
        c = q // ppc
        n = oracle.lib().orc_solid_vertex_count(int(types[c]))
        hit, r = oracle.solid_intersect(pts[q, :3], verts[idx[c, :n]], n)
        assert hit == bool(g["hit"][q]), q
        if hit:
            hits += 1
            assert np.array_equal(r.view(np.uint32), g["rstw"][q].view(np.uint32)), q
    assert hits > 1500 and hits < pts.shape[0] - 1500
    a = oracle.solid_bounds(verts, idx, types)
    assert np.array_equal(_bits(a[:, :6]), _bits(g["ref_aabbs"][:, :6]))
    # density words: the documented minimum and maximum here; the reference's
    # program leaves the last vertex's density in both (a scalar assigned to
    # its float2, gprt/gprt_fallbacks.slang:488-489)
    n = np.array([oracle.lib().orc_solid_vertex_count(int(t)) for t in types])
    dens = [verts[idx[c, :n[c]], 3] for c in range(types.size)]
    assert np.array_equal(a[:, 6], np.array([d.min() for d in dens], np.float32))
    assert np.array_equal(a[:, 7], np.array([d.max() for d in dens], np.float32))
    last = np.array([d[-1] for d in dens], np.float32)
    assert np.array_equal(g["ref_aabbs"][:, 6], last) and np.array_equal(g["ref_aabbs"][:, 7], last)


def test_solid_cell_types_match_reference():
    # vertex counts and hit kinds of every cell type code, and the restated
    # Newton inversion on fresh random cells, against the reference-compiled
    # code when the reference sources are mounted
    if not oracle.ref_available():
        pytest.skip("reference checker not built here")
    R = oracle.ref()
    for t in range(256):
        assert oracle.lib().orc_solid_vertex_count(t) == R.ref_solid_vertex_count(t), t
        assert oracle.lib().orc_solid_hit_kind(t) == R.ref_solid_hit_kind(t), t
    import sys
    sys.path.insert(0, GOLD)
    import make_golden
    verts, idx, types, pts = make_golden.solid_case_inputs(cells=300, seed=99)
    ppc = pts.shape[0] // types.size
    for q in range(pts.shape[0]):
        c = q // ppc
        n = oracle.lib().orc_solid_vertex_count(int(types[c]))
        h1, r1 = oracle.solid_intersect(pts[q, :3], verts[idx[c, :n]], n)
        h2, r2 = oracle.ref_solid_intersect(pts[q, :3], verts[idx[c, :n]], n)
        assert h1 == h2 and (not h1 or np.array_equal(r1.view(np.uint32), r2.view(np.uint32))), q


def test_fp64_traversal_matches_fp64_brute_force():
    # The FP64 closest-hit search through the tree (the accuracy reference for
    # hit ids) against an FP64 search over every triangle, on a small scene:
    # the tree must never prune a triangle that FP64 hits.
    from gprt_b200 import scenes
    pos, tri = scenes.soup(600, seed=21, sigma=0.03)
    rays = scenes.rays(1500, seed=22)
    e = oracle.lbvh_build_tri(pos, tri)
    p64, t64v = oracle.trace_lbvh64(pos, tri, e, rays)
    v = pos.reshape(-1, 3)[tri.reshape(-1)].reshape(-1, 3, 3)
    r8 = rays.reshape(-1, 8)
    for r in range(r8.shape[0]):
        best, bt = 0xFFFFFFFF, np.inf
        for i in range(v.shape[0]):
            hit, t = _isect64(r8[r], v[i])
            if hit and (t < bt or (t == bt and i < best)):
                best, bt = i, t
        assert p64[r] == best, r
        if best != 0xFFFFFFFF:
            assert t64v[r] == bt, r
    # the GPU-side FP32 ids (here the FP32 oracle's) differ from FP64 only at near ties or edges
    h32 = oracle.trace_lbvh(pos, tri, e, rays)
    d = oracle.fp64_id_diagnostic(pos, tri, e, rays, h32["prim"])
    assert d["other"] == 0, d


def _isect64(ray, v):
    """The double-precision watertight test (Woop et al. 2013, section 3) of
    the oracle's FP64 search, restated in numpy scalars."""
    o = ray[:3].astype(np.float64)
    dr = ray[4:7].astype(np.float64)
    tmin, tmax = float(ray[3]), float(ray[7])
    a = np.abs(dr)
    kz = (0 if a[0] >= a[2] else 2) if a[0] >= a[1] else (1 if a[1] >= a[2] else 2)
    kx = 0 if kz + 1 == 3 else kz + 1
    ky = 0 if kx + 1 == 3 else kx + 1
    if dr[kz] < 0.0:
        kx, ky = ky, kx
    Sx, Sy, Sz = dr[kx] / dr[kz], dr[ky] / dr[kz], 1.0 / dr[kz]
    A, B, C = (v[k].astype(np.float64) - o for k in range(3))
    Ax, Ay = A[kx] - Sx * A[kz], A[ky] - Sy * A[kz]
    Bx, By = B[kx] - Sx * B[kz], B[ky] - Sy * B[kz]
    Cx, Cy = C[kx] - Sx * C[kz], C[ky] - Sy * C[kz]
    U, V, W = Cx * By - Cy * Bx, Ax * Cy - Ay * Cx, Bx * Ay - By * Ax
    if (U < 0.0 or V < 0.0 or W < 0.0) and (U > 0.0 or V > 0.0 or W > 0.0):
        return False, 0.0
    det = (U + V) + W
    if det == 0.0:
        return False, 0.0
    T = (U * (Sz * A[kz]) + V * (Sz * B[kz])) + W * (Sz * C[kz])
    t = T / det
    if not (tmin <= t <= tmax):
        return False, 0.0
    return True, t
