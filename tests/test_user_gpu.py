"""Spheres and linearly swept spheres (LSS) as software-BVH primitives,
through the C ABI: bounds bit-exact against the oracle (itself pinned to the
reference's SphereBounds / computeLssAabb compiled from its sources), the box
LBVH bit-exact against the oracle, and closest hits (ids, t and u bits)
identical to a brute-force search with the reference's intersectRayLSS
arithmetic, for every end-cap and exit-test combination; any hit agrees on
occlusion and reports a genuine hit."""
import numpy as np
import pytest

import oracle
from gprt_b200 import scenes

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _spheres(n, seed, rmin=0.002, rmax=0.02):
    rng = np.random.default_rng(seed)
    s = np.zeros((n, 4), np.float32)
    s[:, :3] = rng.random((n, 3), dtype=np.float32)
    s[:, 3] = rng.uniform(rmin, rmax, n).astype(np.float32)
    return s


def _strands(strands, segs, seed):
    # random-walk hair strands: vertices float4 {xyz, radius}, segments (i, i+1)
    rng = np.random.default_rng(seed)
    v = np.zeros((strands * (segs + 1), 4), np.float32)
    idx = []
    for s in range(strands):
        p = rng.random(3)
        r = rng.uniform(0.003, 0.01)
        for k in range(segs + 1):
            i = s * (segs + 1) + k
            v[i, :3] = p
            v[i, 3] = r * (1.0 - 0.5 * k / segs)
            p = p + rng.normal(0, 0.02, 3)
            if k < segs:
                idx.append((i, i + 1))
    return v, np.array(idx, np.uint32)


def _check_closest(got, u, exp):
    assert np.array_equal(got["prim"], exp["prim"])
    hit = got["prim"] != 0xFFFFFFFF
    assert np.array_equal(_bits(got["t"][hit]), _bits(exp["t"][hit]))
    assert np.array_equal(_bits(u[hit]), _bits(exp["u"][hit]))
    return int(hit.sum())


def test_sphere_and_lss_bounds_match_oracle(cuda):
    import torch
    from gprt_b200 import api
    s = _spheres(10007, 1)
    s[::97, 3] = -0.5  # negative radii clamp to 0
    got = api.sphere_bounds(torch.from_numpy(s).cuda()).cpu().numpy()
    assert np.array_equal(_bits(got), _bits(oracle.sphere_bounds(s)))
    v, idx = _strands(300, 20, 2)
    v[::13, 3] *= -0.2  # negative radius on some ends
    vt, it = torch.from_numpy(v).cuda(), torch.from_numpy(idx.view(np.int32)).cuda()
    for c0 in (False, True):
        for c1 in (False, True):
            got = api.lss_bounds(vt, it, c0, c1).cpu().numpy()
            assert np.array_equal(_bits(got), _bits(oracle.lss_bounds(v, idx, c0, c1))), (c0, c1)


@pytest.mark.parametrize("n", [1, 2, 3, 1000, 100003])
def test_box_lbvh_matches_oracle(cuda, n):
    import torch
    from gprt_b200 import api
    b = oracle.sphere_bounds(_spheres(n, 3 + n))
    for kind in (0, 1):
        h = api.lbvh_build_boxes(torch.from_numpy(b).cuda(), code_kind=kind).host()
        e = oracle.lbvh_build_boxes(b, kind)
        for k in ("scene", "codes", "ids", "nodes", "aabbs"):
            assert np.array_equal(_bits(h[k]), _bits(e[k].reshape(h[k].shape))), (n, kind, k)


@pytest.mark.parametrize("n,m", [(1, 2000), (5, 2000), (3000, 20000), (20000, 20000)])
@pytest.mark.parametrize("exit_test", [False, True])
def test_trace_spheres_matches_brute_force(cuda, n, m, exit_test):
    import torch
    from gprt_b200 import api
    s = _spheres(n, 10 + n, 0.01 if n > 100 else 0.2, 0.03 if n > 100 else 0.4)
    rays = scenes.rays(m, seed=11 + n)
    st = torch.from_numpy(s).cuda()
    bvh = api.lbvh_build_boxes(api.sphere_bounds(st))
    rt = torch.from_numpy(rays).cuda()
    u = torch.empty(m, dtype=torch.float32, device="cuda")
    got = api.hits_numpy(api.trace_spheres(bvh, st, rt, u=u, exit_test=exit_test))
    exp = oracle.trace_user_brute(0, s, rays, exit_test=exit_test)
    assert _check_closest(got, u.cpu().numpy(), exp) > 0
    anyh = api.hits_numpy(api.trace_spheres(bvh, st, rt, anyhit=True, exit_test=exit_test))
    assert np.array_equal(anyh["prim"] != 0xFFFFFFFF, exp["prim"] != 0xFFFFFFFF)
    for r in np.nonzero(anyh["prim"] != 0xFFFFFFFF)[0][:300]:
        sp = s[anyh["prim"][r]]
        assert oracle.lss_intersect(rays[r], sp, sp, True, True, exit_test)[0]


@pytest.mark.parametrize("caps", [(True, True), (False, True), (True, False), (False, False)])
@pytest.mark.parametrize("exit_test", [False, True])
def test_trace_lss_matches_brute_force(cuda, caps, exit_test):
    import torch
    from gprt_b200 import api
    v, idx = _strands(400, 16, 20)
    rays = scenes.rays(20000, seed=21)
    vt, it = torch.from_numpy(v).cuda(), torch.from_numpy(idx.view(np.int32)).cuda()
    bvh = api.lbvh_build_boxes(api.lss_bounds(vt, it, *caps))
    rt = torch.from_numpy(rays).cuda()
    u = torch.empty(len(rays), dtype=torch.float32, device="cuda")
    got = api.hits_numpy(api.trace_lss(bvh, vt, it, rt, caps[0], caps[1], u=u, exit_test=exit_test))
    exp = oracle.trace_user_brute(1, v, rays, idx, caps[0], caps[1], exit_test)
    assert _check_closest(got, u.cpu().numpy(), exp) > 100
