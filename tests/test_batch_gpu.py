"""Batched multi-mesh build and trace through the C ABI: every mesh's block of
the concatenated output is bit-identical to the oracle's (and the plain
kernel's) build of that mesh alone, and the batched trace's hits equal the
per-mesh traces."""
import numpy as np
import pytest

import oracle
from gprt_b200 import scenes

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32) if a.dtype == np.float32 else a


def _local(pos, tri, off, m):
    t = tri[off[m]:off[m + 1]]
    base = t.min()
    return pos[base:t.max() + 1], (t - base).astype(np.uint32)


@pytest.mark.parametrize("kind", [0, 1])
def test_batch_build_equals_per_mesh_builds(cuda, kind):
    import torch
    from gprt_b200 import api
    rng = np.random.default_rng(5 + kind)
    sizes = np.concatenate([[1, 2, 3, 64], rng.integers(1, 3000, size=40), [4097, 65536]])
    pos, tri, off = scenes.batch(sizes, seed=3)
    b = api.BatchLbvh(off)
    api.batch_build_triangles(torch.from_numpy(pos).cuda(), torch.from_numpy(tri.view(np.int32)).cuda(), b, kind)
    torch.cuda.synchronize()
    for m in range(len(sizes)):
        lp, lt = _local(pos, tri, off, m)
        e = oracle.lbvh_build_tri(lp, lt, kind)
        h = b.mesh_host(m)
        for k in ("scene", "codes", "ids", "nodes", "aabbs"):
            assert np.array_equal(_bits(h[k]), _bits(e[k].reshape(h[k].shape))), (m, k)


def test_batch_traversal_nodes_equal_plain_build(cuda):
    import torch
    from gprt_b200 import api
    sizes = [5, 1000, 1, 3000, 77]
    pos, tri, off = scenes.batch(sizes, seed=9)
    b = api.BatchLbvh(off)
    api.batch_build_triangles(torch.from_numpy(pos).cuda(), torch.from_numpy(tri.view(np.int32)).cuda(), b)
    torch.cuda.synchronize()
    for m, n in enumerate(sizes):
        lp, lt = _local(pos, tri, off, m)
        plain = api.lbvh_build_triangles(torch.from_numpy(lp).cuda(), torch.from_numpy(lt.view(np.int32)).cuda())
        torch.cuda.synchronize()
        if n > 1:
            got = b.bvh2[off[m] - m:off[m + 1] - m - 1].cpu().numpy()
            assert np.array_equal(_bits(got), _bits(plain.bvh2.cpu().numpy())), m
        assert np.array_equal(_bits(b.leaf[off[m]:off[m + 1]].cpu().numpy()), _bits(plain.leaf.cpu().numpy())), m


@pytest.mark.parametrize("anyhit", [False, True])
def test_batch_trace_equals_per_mesh(cuda, anyhit):
    import torch
    from gprt_b200 import api
    rng = np.random.default_rng(11)
    sizes = np.concatenate([[1, 2], rng.integers(64, 4000, size=24)])
    pos, tri, off, rays, roff = scenes.batch(sizes, seed=4, sigma=0.01, rays_per_tri=2)
    b = api.BatchLbvh(off)
    api.batch_build_triangles(torch.from_numpy(pos).cuda(), torch.from_numpy(tri.view(np.int32)).cuda(), b)
    rt = torch.from_numpy(rays).cuda()
    ro = torch.from_numpy(roff.astype(np.uint32).view(np.int32)).cuda()
    got = api.hits_numpy(api.batch_trace(b, rt, ro, anyhit=anyhit))
    nhit = 0
    for m in range(len(sizes)):
        lp, lt = _local(pos, tri, off, m)
        r = rays[roff[m]:roff[m + 1]]
        g = got[roff[m]:roff[m + 1]]
        if anyhit:
            exp = oracle.trace_lbvh(lp, lt, oracle.lbvh_build_tri(lp, lt), r)
            assert np.array_equal(g["prim"] != 0xFFFFFFFF, exp["prim"] != 0xFFFFFFFF), m
        else:
            exp = oracle.trace_lbvh(lp, lt, oracle.lbvh_build_tri(lp, lt), r)
            assert np.array_equal(g["prim"], exp["prim"]), m
            hit = g["prim"] != 0xFFFFFFFF
            assert np.array_equal(_bits(g["t"][hit]), _bits(exp["t"][hit])), m
            nhit += int(hit.sum())
    assert anyhit or nhit > 1000
