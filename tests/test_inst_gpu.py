"""Two-level instancing through the C ABI: world-to-object matrices
bit-identical to the oracle's (double inverse rounded once), and closest hits
(mesh-local ids, instance ids, t bits) identical to a brute-force search over
every triangle of every visible instance, with ray masks, singular
transforms, out-of-range mesh indices, one-triangle meshes and any hit."""
import numpy as np
import pytest

import oracle
from gprt_b200 import scenes

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _instances(rng, n, meshes):
    rec = np.zeros(n, oracle.INSTANCE_DTYPE)
    for i in range(n):
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        a = q * rng.uniform(0.5, 2.0, size=3)[None, :]
        m = np.zeros((3, 4))
        m[:, :3] = a
        m[:, 3] = rng.uniform(-3, 3, 3)
        rec[i]["transform"] = m.reshape(12)
        mask = [0x01, 0x02, 0x81, 0xFF][i % 4]
        rec[i]["custom_mask"] = (mask << 24) | (1000 + i)
        rec[i]["blas"] = i % meshes
    if n > 5:
        rec[3]["transform"] = np.zeros(12)          # singular: never hit
        rec[5]["blas"] = meshes + 7                  # out of range: never hit
    return rec


def _rays(rng, m):
    u = rng.normal(size=(m, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    o = 8.0 * u
    d = rng.uniform(-4, 4, (m, 3)) - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((m, 8), np.float32)
    r[:, :3], r[:, 4:7], r[:, 7] = o, d, np.inf
    return r


def _setup(torch, sizes, ninst, seed):
    from gprt_b200 import api
    rng = np.random.default_rng(seed)
    pos, tri, off = scenes.batch(sizes, seed=seed, sigma=0.05, spacing=0.0)
    bb = api.BatchLbvh(off)
    api.batch_build_triangles(torch.from_numpy(pos).cuda(), torch.from_numpy(tri.view(np.int32)).cuda(), bb)
    rec = _instances(rng, ninst, len(sizes))
    tlas = api.Tlas(api.instances_tensor(rec), bb.root, len(sizes))
    return pos, tri, off, bb, rec, tlas, rng


@pytest.mark.parametrize("sizes,ninst", [([1, 2, 300, 700, 64], 24), ([500], 1), ([3, 400], 2)])
def test_instances_match_brute_force(cuda, sizes, ninst):
    import torch
    from gprt_b200 import api
    pos, tri, off, bb, rec, tlas, rng = _setup(torch, sizes, ninst, 40 + ninst)
    w = tlas.w2o.cpu().numpy()
    for i in range(ninst):
        e = oracle.instance_inverse(rec[i]["transform"])
        if rec[i]["blas"] >= len(sizes):
            e = None
        assert np.array_equal(_bits(w[i]), _bits(np.zeros(12, np.float32) if e is None else e)), i
    rays = _rays(rng, 6000)
    rt = torch.from_numpy(rays).cuda()
    total = 0
    for ray_mask in (0xFF, 0x02, 0x80, 0x00):
        h, inst = api.trace_instances(tlas, bb, rt, bb.tri_off, len(sizes), ray_mask)
        got = api.hits_numpy(h)
        gi = inst.cpu().numpy().view(np.uint32)
        exp = oracle.trace_instances_brute(rec, pos, tri, off, rays, ray_mask)
        assert np.array_equal(got["prim"], exp["prim"]), ray_mask
        hit = exp["prim"] != 0xFFFFFFFF
        assert np.array_equal(gi[hit], exp["inst"][hit]), ray_mask
        assert np.array_equal(_bits(got["t"][hit]), _bits(exp["t"][hit])), ray_mask
        if ninst > 5:
            assert not (set(exp["inst"][hit].tolist()) & {3, 5})
        total += int(hit.sum())
        ha, _ = api.trace_instances(tlas, bb, rt, bb.tri_off, len(sizes), ray_mask, anyhit=True)
        assert np.array_equal(api.hits_numpy(ha)["prim"] != 0xFFFFFFFF, hit), ray_mask
    assert total > (1000 if ninst > 5 else 50)


def test_identical_instances_tie_to_lowest_instance(cuda):
    """Four copies of one mesh under the same transform: every hit lands on
    instance 0 with the primitive and t of a single copy; with instance 0
    masked out the winner moves to instance 1."""
    import torch
    from gprt_b200 import api
    rng = np.random.default_rng(7)
    pos, tri = scenes.soup(3000, seed=7, sigma=0.05)
    bvh = api.lbvh_build_triangles(torch.from_numpy(pos).cuda(), torch.from_numpy(tri.view(np.int32)).cuda())
    rec = np.zeros(4, oracle.INSTANCE_DTYPE)
    m = np.array([[0.0, -1.5, 0.0, 0.25], [1.5, 0.0, 0.0, -0.5], [0.0, 0.0, 1.5, 0.125]])
    for i in range(4):
        rec[i]["transform"] = m.reshape(12)
        rec[i]["custom_mask"] = ((0x01 if i == 0 else 0x03) << 24) | i
    tlas = api.Tlas(api.instances_tensor(rec), bvh.root, 1)
    rays = _rays(rng, 4000)
    tgt = rng.random((4000, 3)) @ m[:, :3].T + m[:, 3]
    d = tgt - rays[:, :3]
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rt = torch.from_numpy(rays).cuda()
    off = np.array([0, tri.shape[0]], np.int64)
    for ray_mask, first in ((0xFF, 0), (0x02, 1)):
        h, inst = api.trace_instances(tlas, bvh, rt, None, 1, ray_mask)
        got = api.hits_numpy(h)
        exp = oracle.trace_instances_brute(rec, pos, tri, off, rays, ray_mask)
        hit = exp["prim"] != 0xFFFFFFFF
        assert hit.sum() > 500
        assert np.array_equal(got["prim"], exp["prim"])
        assert np.all(inst.cpu().numpy()[hit] == first)
        assert np.all(exp["inst"][hit] == first)
        assert np.array_equal(_bits(got["t"][hit]), _bits(exp["t"][hit]))


def test_instances_reject_bad_arguments(cuda):
    import torch
    from gprt_b200 import api
    rec = np.zeros(2, oracle.INSTANCE_DTYPE)
    t = api.instances_tensor(rec)
    roots = torch.zeros(6, dtype=torch.float32, device="cuda")
    with pytest.raises(RuntimeError):
        api.Tlas(t, roots, 0)


def _cube():
    v = np.array([[x, y, z] for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)], np.float32)
    q = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    t = np.array([f for a, b, c, d in q for f in ((a, b, c), (a, c, d))], np.uint32)
    return v, t


def _quad(x0, x1, y0, y1, z):
    v = np.array([[x0, y0, z], [x1, y0, z], [x1, y1, z], [x0, y1, z]], np.float32)
    return v, np.array([[0, 1, 2], [0, 2, 3]], np.uint32)


def _batch_of(torch, meshes):
    from gprt_b200 import api
    pos, tri, off = [], [], [0]
    base = 0
    for v, t in meshes:
        pos.append(v)
        tri.append(t + base)
        base += len(v)
        off.append(off[-1] + len(t))
    pos, tri = np.concatenate(pos), np.concatenate(tri).astype(np.uint32)
    bb = api.BatchLbvh(off)
    api.batch_build_triangles(torch.from_numpy(pos).cuda(), torch.from_numpy(tri.view(np.int32)).cuda(), bb)
    return pos, tri, np.array(off, np.int64), bb


def _axis_rays(org, d):
    r = np.zeros((len(org), 8), np.float32)
    r[:, :3], r[:, 4:7], r[:, 7] = org, d, np.inf
    return r


def test_sample_transforms_place_cubes(cuda):
    """The transforms sample (samples/s3-instancing/s3-0-transforms/hostCode.cpp:19-21):
    one cube under three row-major 3x4 matrices (scale 0.5, x offsets -1.5, 0,
    1.5, translation in the last column); a ray down -z through each centre
    hits that instance's front face at t = 4.5."""
    import torch
    from gprt_b200 import api
    v, t = _cube()
    pos, tri, off, bb = _batch_of(torch, [(v, t)])
    rec = np.zeros(3, oracle.INSTANCE_DTYPE)
    for i, x in enumerate((-1.5, 0.0, 1.5)):
        rec[i]["transform"] = [0.5, 0, 0, x, 0, 0.5, 0, 0, 0, 0, 0.5, 0]
        rec[i]["custom_mask"] = (0xFF << 24) | i
    tlas = api.Tlas(api.instances_tensor(rec), bb.root, 1)
    assert np.array_equal(tlas.boxes.cpu().numpy(),
                          np.array([[x - 0.5, -0.5, -0.5, x + 0.5, 0.5, 0.5] for x in (-1.5, 0.0, 1.5)], np.float32))
    org = np.array([[x, 0.1, 5.0] for x in (-1.5, 0.0, 1.5, 0.75, 3.0)], np.float32)
    rays = _axis_rays(org, [0, 0, -1])
    h, inst = api.trace_instances(tlas, bb, torch.from_numpy(rays).cuda(), bb.tri_off, 1)
    got = api.hits_numpy(h)
    exp = oracle.trace_instances_brute(rec, pos, tri, off, rays)
    assert np.array_equal(got["prim"], exp["prim"])
    assert np.array_equal(inst.cpu().numpy()[:3], [0, 1, 2])
    assert np.array_equal(got["t"][:3], np.float32([4.5, 4.5, 4.5]))
    assert np.all(got["prim"][3:] == 0xFFFFFFFF)


def test_sample_visibility_masks(cuda):
    """The visibility-mask sample (samples/s3-instancing/s3-1-visibilityMasks):
    floor, wall and window meshes instanced at x = -6, -3, 0, 3, 6, windows
    with mask 0b11111110.  Primary rays (mask 0xFF) stop at a window; shadow
    rays (mask 0b00000001) pass through it to the wall behind."""
    import torch
    from gprt_b200 import api
    floor = _quad(-1.5, 1.5, -1.5, 1.5, 0.0)
    floor = (floor[0][:, [0, 2, 1]].copy(), floor[1])            # y = 0 plane
    wall = _quad(-1.0, 1.0, 0.0, 2.0, 1.0)
    window = _quad(-0.5, 0.5, 0.5, 1.5, 0.5)
    pos, tri, off, bb = _batch_of(torch, [floor, wall, window])
    rec = np.zeros(15, oracle.INSTANCE_DTYPE)
    for i in range(15):
        x = (-6.0, -3.0, 0.0, 3.0, 6.0)[i // 3]
        rec[i]["transform"] = [1, 0, 0, x, 0, 1, 0, 0, 0, 0, 1, 0]
        rec[i]["custom_mask"] = ((0b11111110 if i % 3 == 2 else 0xFF) << 24) | i
        rec[i]["blas"] = i % 3
    tlas = api.Tlas(api.instances_tensor(rec), bb.root, 3)
    org = np.array([[x, 1.0, -5.0] for x in (-6.0, -3.0, 0.0, 3.0, 6.0)], np.float32)
    rays = torch.from_numpy(_axis_rays(org, [0, 0, 1])).cuda()
    for mask, t_exp, which in ((0xFF, 5.5, 2), (0x01, 6.0, 1)):
        h, inst = api.trace_instances(tlas, bb, rays, bb.tri_off, 3, mask)
        got = api.hits_numpy(h)
        exp = oracle.trace_instances_brute(rec, pos, tri, off, rays.cpu().numpy(), mask)
        assert np.array_equal(got["prim"], exp["prim"])
        assert np.array_equal(inst.cpu().numpy(), exp["inst"])
        assert np.array_equal(inst.cpu().numpy(), 3 * np.arange(5) + which)
        assert np.all(got["t"] == np.float32(t_exp))
