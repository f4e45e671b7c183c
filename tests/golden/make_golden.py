"""Generate the golden fixtures in tests/golden/ from the reference itself.

    python tests/golden/make_golden.py      (needs the reference sources; run
                                             where they are mounted)

* lbvh_ref.npz   -- gprt/development/gprt_lbvh.hlsl compiled from the
                    reference sources (oracle/Makefile target `ref`) and run
                    serially in gprtLBVHBuild's order: scene box, Morton codes,
                    sorted (code, id) pairs, int4 nodes, float3 box pairs, for
                    seeded triangle soups, seeded edge sets and a t04-style
                    point set with coordinates in [-1e38, 1e38]
                    (tests/t04-swBVH/hostCode.cpp:47-56).
* hilbert_ref.npz -- gprt/hilbert.h hilbert_c2i(3, 10, .) on seeded and corner
                    coordinates.
* lss_ref.npz    -- intersectRayLSS and computeLssAabb of gprt/gprt_fallbacks.slang
                    compiled from the reference sources, on seeded rays, spheres
                    and swept-sphere segments, every cap / exit-test combination.
* solid_ref.npz  -- intersectPointSolid and SolidBounds of gprt/gprt_fallbacks.slang
                    compiled from the reference sources, on seeded distorted
                    tetrahedra, pyramids, wedges, hexahedra and tetrahedral
                    pairs (each cell in its own region of space) and points at
                    their vertices, edge midpoints and around their boxes.
                    `python make_golden.py solids` regenerates this file alone.
* sortscan.npz   -- the reference tests' own host oracles restated with numpy:
                    std::sort / std::sort-by-key (tests/t02-bufferSort/hostCode.cpp:59,115),
                    the serial exclusive sum (tests/t03-bufferScans/hostCode.cpp:53-58)
                    and the partition/select layouts (:98-160, :172-241), on
                    small seeded inputs.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402


def tri_soup(rng, n, sigma=0.002):
    c = rng.random((n, 3), dtype=np.float32)
    pos = (np.repeat(c, 3, axis=0) + rng.normal(0.0, sigma, (3 * n, 3))).astype(np.float32)
    tri = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    return pos, tri


def lss_case_inputs(n=4000, seed=99):
    """Seeded rays and sphere / swept-sphere segments: spheres, tapered and
    constant-radius segments, a negative start radius; rays aimed near the
    primitive so most hit."""
    r = np.random.default_rng(seed)
    rays = np.zeros((n, 8), np.float32)
    v0 = np.zeros((n, 4), np.float32)
    v1 = np.zeros((n, 4), np.float32)
    for i in range(n):
        kind = i % 4
        c0 = r.normal(size=3) * 0.5
        if kind == 0:
            c1, r0 = c0.copy(), abs(r.normal()) * 0.5 + 0.01
            r1 = r0
        else:
            c1 = c0 + r.normal(size=3) * 0.5
            r0, r1 = abs(r.normal()) * 0.3 + 0.01, abs(r.normal()) * 0.3 + 0.01
            if kind == 2:
                r1 = r0
            if kind == 3:
                r0 = -0.1 * r0
        o = r.normal(size=3)
        o = o / np.linalg.norm(o) * 3.0
        target = 0.5 * (c0 + c1) + r.normal(size=3) * 0.3
        d = target - o
        d /= np.linalg.norm(d)
        rays[i] = [*o, 0.0, *d, np.inf]
        v0[i] = [*c0, r0]
        v1[i] = [*c1, r1]
    return rays, v0, v1


def lss_cases():
    # the reference's intersectRayLSS and computeLssAabb (gprt/gprt_fallbacks.slang)
    # compiled from its sources, on every combination of caps and exit test
    rays, v0, v1 = lss_case_inputs()
    out = {"rays": rays, "v0": v0, "v1": v1}
    for cap0 in (0, 1):
        for cap1 in (0, 1):
            for ex in (0, 1):
                hit = np.zeros(len(rays), np.uint8)
                t = np.zeros(len(rays), np.float32)
                u = np.zeros(len(rays), np.float32)
                for i in range(len(rays)):
                    h, tt, uu = oracle.ref_lss_intersect(rays[i], v0[i], v1[i], cap0, cap1, ex)
                    hit[i], t[i], u[i] = h, tt, uu
                key = "c%d%d_x%d" % (cap0, cap1, ex)
                out[key + "_hit"], out[key + "_t"], out[key + "_u"] = hit, t, u
            box = np.stack([oracle.ref_lss_aabb(v0[i], v1[i], cap0, cap1) for i in range(len(rays))])
            out["c%d%d_aabb" % (cap0, cap1)] = box
    np.savez_compressed(os.path.join(HERE, "lss_ref.npz"), **out)


SOLID_BASE = {
    4: [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]],
    5: [[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0.5, 0.5, 1]],
    6: [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [0, 1, 1]],
    8: [[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]],
}
SOLID_TYPES = [(10, 4), (14, 5), (13, 6), (12, 8), (23, 8)]


def solid_case_inputs(cells=1000, pts_per_cell=8, seed=4321):
    """Distorted cells of every type, cell c in its own slab x in [16c, 16c +
    10), and points per cell: a vertex, an edge midpoint, the rest uniform in
    the cell's box grown by 10 % on each side."""
    r = np.random.default_rng(seed)
    verts = np.zeros((cells * 8, 4), np.float32)
    idx = np.full((cells, 8), 0xFFFFFFFF, np.uint32)
    types = np.zeros(cells, np.uint8)
    pts = np.zeros((cells * pts_per_cell, 4), np.float32)
    for c in range(cells):
        t, n = SOLID_TYPES[c % len(SOLID_TYPES)]
        jit = [0.0, 0.05, 0.2, 0.45][(c // len(SOLID_TYPES)) % 4]
        base = np.asarray(SOLID_BASE[n], np.float64)
        v = base * r.uniform(0.3, 3.0) + r.normal(0, jit, (n, 3))
        v = v + np.array([16.0 * c, r.uniform(-3, 3), r.uniform(-3, 3)])
        verts[8 * c:8 * c + n, :3] = v
        verts[8 * c:8 * c + n, 3] = r.uniform(-2, 2, n)
        idx[c, :n] = np.arange(8 * c, 8 * c + n)
        types[c] = t
        vv = verts[8 * c:8 * c + n, :3]
        lo, hi = vv.min(0), vv.max(0)
        for k in range(pts_per_cell):
            if k == 0:
                p = vv[r.integers(n)]
            elif k == 1:
                a, b = r.choice(n, 2, replace=False)
                p = (vv[a] + vv[b]) * np.float32(0.5)
            else:
                p = lo + (hi - lo) * r.uniform(-0.1, 1.1, 3)
            pts[pts_per_cell * c + k, :3] = p
    return verts, idx, types, pts


def solid_cases():
    """The reference's own intersectPointSolid and SolidBounds on the cases above."""
    verts, idx, types, pts = solid_case_inputs()
    ppc = pts.shape[0] // types.size
    hit = np.zeros(pts.shape[0], np.uint8)
    rstw = np.zeros((pts.shape[0], 4), np.float32)
    for q in range(pts.shape[0]):
        c = q // ppc
        n = oracle.lib().orc_solid_vertex_count(int(types[c]))
        h, r4 = oracle.ref_solid_intersect(pts[q, :3], verts[idx[c, :n]], n)
        hit[q], rstw[q] = h, r4
    aabbs = oracle.ref_solid_bounds(verts, idx, types)
    np.savez_compressed(os.path.join(HERE, "solid_ref.npz"), verts=verts, idx=idx, types=types, points=pts,
                        hit=hit, rstw=rstw, ref_aabbs=aabbs)


def main():
    oracle.build(ref=True)
    rng = np.random.default_rng(20240601)
    out = {}
    cases = []
    for n in (1, 2, 3, 7, 64, 1000, 4099):
        cases.append(("tri%d" % n,) + tri_soup(rng, n))
    # duplicate-heavy codes (equal Morton codes exercise the index tie-break)
    n = 777
    c = (np.floor(rng.random((n, 3)) * 3) / 3).astype(np.float32)
    cases.append(("tridup", np.repeat(c, 3, axis=0).astype(np.float32), np.arange(3 * n, dtype=np.uint32).reshape(n, 3)))
    # shared vertices (indexed mesh, not a soup)
    grid = rng.random((200, 3), dtype=np.float32)
    tri = rng.integers(0, 200, size=(500, 3)).astype(np.uint32)
    cases.append(("trimesh", grid, tri))
    for name, pos, tri in cases:
        r = oracle.ref_lbvh_build(pos, tri)
        out[name + "_pos"] = pos
        out[name + "_tri"] = tri
        for k, v in r.items():
            out[name + "_" + k] = v
    # t04: 42 points uniform in [-1e38, 1e38]^3 (max - min overflows to inf)
    pts = rng.uniform(-1e38, 1e38, size=(42, 3)).astype(np.float32)
    r = oracle.ref_lbvh_build(pts)
    out["pts42_pos"] = pts
    for k, v in r.items():
        out["pts42_" + k] = v
    # edges (ComputeEdgeBounds / ComputeEdgeMortonCodes / BuildEdgeHierarchy),
    # from their own generator so the cases above keep their bits
    erng = np.random.default_rng(777)
    for n in (1, 2, 3, 64, 1000):
        pos = erng.random((n + 5, 3), dtype=np.float32)
        edges = erng.integers(0, n + 5, size=(n, 2)).astype(np.uint32)
        r = oracle.ref_lbvh_build(pos, edges)
        out["edge%d_pos" % n] = pos
        out["edge%d_edges" % n] = edges
        for k, v in r.items():
            out["edge%d_%s" % (n, k)] = v
    np.savez_compressed(os.path.join(HERE, "lbvh_ref.npz"), **out)

    lss_cases()
    solid_cases()

    R = oracle.ref()
    co = rng.integers(0, 1024, size=(4096, 3)).astype(np.uint32)
    corners = np.array([[x, y, z] for x in (0, 1, 511, 512, 1023) for y in (0, 1, 511, 512, 1023)
                        for z in (0, 1, 511, 512, 1023)], np.uint32)
    co = np.concatenate([co, corners])
    h = np.array([R.ref_hilbert3d(int(a), int(b), int(c)) for a, b, c in co], np.uint32)
    np.savez_compressed(os.path.join(HERE, "hilbert_ref.npz"), coords=co, codes=h)

    # sort / scan / partition fixtures from numpy restatements of the tests' host oracles
    k = rng.integers(0, 2 ** 32, size=5000, dtype=np.uint64).astype(np.uint32)
    k[::7] = k[0]  # repeated keys so stability matters
    v = np.arange(k.size, dtype=np.uint32)
    order = np.argsort(k, kind="stable")
    k64 = rng.integers(0, 2 ** 63, size=3000, dtype=np.uint64) | (rng.integers(0, 2, size=3000, dtype=np.uint64) << np.uint64(63))
    k64[::5] = k64[1]
    o64 = np.argsort(k64, kind="stable")
    x = rng.integers(0, 256, size=9973 * 3, dtype=np.uint32)
    excl = (np.concatenate([np.zeros(1, np.uint64), np.cumsum(x.astype(np.uint64))[:-1]]) & 0xFFFFFFFF).astype(np.uint32)
    big = np.full(3000, 0xFFFFFFF0, np.uint32)  # forces uint32 wraparound
    excl_big = (np.concatenate([np.zeros(1, np.uint64), np.cumsum(big.astype(np.uint64))[:-1]]) & 0xFFFFFFFF).astype(np.uint32)
    nt = 9973 * 2
    t03 = np.array([i * (1 if (i & 1) else -1) for i in range(nt)], np.int32)
    sel = (t03 >= 0).astype(np.int64)
    ex = np.concatenate([[0], np.cumsum(sel)[:-1]])
    part = np.zeros(nt, np.int32)
    selo = np.zeros(nt, np.int32)
    for i in range(nt):
        if t03[i] >= 0:
            part[ex[i]] = t03[i]
            selo[ex[i]] = t03[i]
        else:
            part[(nt - 1) - (i - ex[i])] = t03[i]
    np.savez_compressed(os.path.join(HERE, "sortscan.npz"), keys=k, keys_sorted=k[order], vals_sorted=v[order],
                        keys64=k64, keys64_sorted=k64[o64], vals64_sorted=o64.astype(np.uint32), scan_in=x,
                        scan_excl=excl, scan_total=np.uint32(int(x.astype(np.uint64).sum()) & 0xFFFFFFFF),
                        big_in=big, big_excl=excl_big, t03_in=t03, t03_partition=part, t03_select=selo,
                        t03_total=np.uint32(sel.sum()))
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    if sys.argv[1:] == ["solids"]:
        oracle.build(ref=True)
        solid_cases()
    else:
        main()
