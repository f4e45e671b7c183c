"""Solid cells on the GPU: bounds, the box LBVH over them and point location,
against the oracle (whose cell math is pinned bit for bit to the reference's
own intersectPointSolid / SolidBounds, tests/test_oracle_pins.py) and the
reference-compiled fixture directly."""
import ctypes
import os

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MISS = 0xFFFFFFFF


def _dev(a, dtype=None):
    import torch
    a = np.ascontiguousarray(a)
    if dtype is not None:
        a = a.view(dtype)
    return torch.from_numpy(a).cuda()


def _locate(verts, idx, types, pts):
    """GPU bounds + box LBVH + point location; numpy results."""
    import torch
    from gprt_b200 import api
    s = api.Solids(_dev(verts), _dev(idx, np.int32), _dev(types))
    aabbs, boxes = api.solid_bounds(s)
    bvh = api.lbvh_build_boxes(boxes)
    hits, rstw = api.locate_solid_points(bvh, s, _dev(pts))
    torch.cuda.synchronize()
    assert api.scratch_status(bvh.scratch) == 0
    h = hits.cpu().numpy().view(np.uint32)
    return aabbs.cpu().numpy(), h[:, 0], h[:, 1], rstw.cpu().numpy()


def _check_against_brute(verts, idx, types, pts):
    aabbs, cell, kind, rstw = _locate(verts, idx, types, pts)
    ea = oracle.solid_bounds(verts, idx, types)
    assert np.array_equal(aabbs.view(np.uint32), ea.view(np.uint32))
    ec, ek, er = oracle.solid_locate_brute(verts, idx, types, pts)
    assert np.array_equal(cell, ec)
    assert np.array_equal(kind, ek)
    assert np.array_equal(rstw.view(np.uint32), er.view(np.uint32))
    return cell


def test_solid_fixture_matches_reference_compiled_code(cuda):
    # each fixture cell lies in its own slab of space, so a point's answer is
    # the reference's intersectPointSolid on its own cell, or no cell
    g = np.load(os.path.join(GOLD, "solid_ref.npz"))
    verts, idx, types, pts = g["verts"], g["idx"], g["types"], g["points"]
    aabbs, cell, kind, rstw = _locate(verts, idx, types, pts)
    assert np.array_equal(aabbs[:, :6].view(np.uint32), g["ref_aabbs"][:, :6].view(np.uint32))
    ppc = pts.shape[0] // types.size
    own = np.arange(pts.shape[0]) // ppc
    hit = g["hit"].astype(bool)
    assert np.array_equal(cell, np.where(hit, own, MISS).astype(np.uint32))
    ekind = np.array([oracle.lib().orc_solid_hit_kind(int(t)) for t in types], np.uint32)[own]
    assert np.array_equal(kind, np.where(hit, ekind, 0).astype(np.uint32))
    assert np.array_equal(rstw[hit].view(np.uint32), g["rstw"][hit].view(np.uint32))
    assert not rstw[~hit].any()


@pytest.mark.parametrize("g,npts,seed", [(1, 3000, 1), (3, 5000, 2), (6, 20000, 3), (16, 20000, 4)])
def test_solid_grid_location_matches_oracle(cuda, g, npts, seed):
    from gprt_b200 import scenes
    verts, idx, types = scenes.solid_grid(g, seed=seed)
    rng = np.random.default_rng(seed + 100)
    pts = np.zeros((npts, 4), np.float32)
    pts[:, :3] = rng.uniform(-0.05, 1.05, (npts, 3))
    # some points exactly on mesh vertices
    k = min(500, verts.shape[0])
    pts[:k, :3] = verts[rng.choice(verts.shape[0], k, replace=False), :3]
    cell = _check_against_brute(verts, idx, types, pts)
    # the sampled region reaches past the mesh, and neighbouring cubes of
    # different fills meet along non-matching faces: about 3/4 of the points
    # lie in a cell
    assert (cell != MISS).mean() > 0.6


@pytest.mark.parametrize("fill", range(5))
def test_each_cell_type_alone(cuda, fill):
    from gprt_b200 import scenes
    verts, idx, types = scenes.solid_grid(5, seed=10 + fill, fills=[fill])
    rng = np.random.default_rng(fill)
    pts = np.zeros((8000, 4), np.float32)
    pts[:, :3] = rng.random((8000, 3))
    cell = _check_against_brute(verts, idx, types, pts)
    assert (cell != MISS).mean() > 0.9


def test_single_cell_and_unknown_types(cuda):
    from gprt_b200 import scenes
    verts, idx, types = scenes.solid_grid(1, seed=5, fills=[0])  # one hexahedron
    assert types.size == 1
    rng = np.random.default_rng(6)
    pts = np.zeros((2000, 4), np.float32)
    pts[:, :3] = rng.uniform(-0.2, 1.2, (2000, 3))
    _check_against_brute(verts, idx, types, pts)
    # cells of unknown type (no vertices, empty box) mixed in hold no point
    verts, idx, types = scenes.solid_grid(4, seed=7)
    types = types.copy()
    types[::3] = np.array([0, 11, 99, 255], np.uint8)[np.arange(types[::3].size) % 4]
    cell = _check_against_brute(verts, idx, types, pts)
    assert not np.isin(cell, np.nonzero(np.isin(types, [0, 11, 99, 255]))[0]).any()


def test_strides(cuda):
    # vertices interleaved with other data (32-byte stride), a tetrahedral mesh
    # with four indices per cell (16-byte stride), types every other byte
    import torch
    from gprt_b200 import api, scenes
    verts, idx, types = scenes.solid_grid(4, seed=8, fills=[3])
    rng = np.random.default_rng(9)
    pts = np.zeros((5000, 4), np.float32)
    pts[:, :3] = rng.random((5000, 3))
    ec, ek, er = oracle.solid_locate_brute(verts, idx, types, pts)
    vbig = np.zeros((verts.shape[0], 8), np.float32)
    vbig[:, :4] = verts
    vbig[:, 4:] = -7.0
    i4 = np.ascontiguousarray(idx[:, :4])
    t2 = np.zeros((types.size, 2), np.uint8)
    t2[:, 0] = types
    t2[:, 1] = 99
    dv, di, dt = _dev(vbig), _dev(i4, np.int32), _dev(t2)
    s = api.Solids(dv, di, dt)
    s.n = s.desc.numCells = types.size
    s.desc.vertexStride, s.desc.indexStride, s.desc.typeStride = 32, 16, 2
    _, boxes = api.solid_bounds(s)
    bvh = api.lbvh_build_boxes(boxes)
    hits, rstw = api.locate_solid_points(bvh, s, _dev(pts))
    torch.cuda.synchronize()
    h = hits.cpu().numpy().view(np.uint32)
    assert np.array_equal(h[:, 0], ec) and np.array_equal(h[:, 1], ek)
    assert np.array_equal(rstw.cpu().numpy().view(np.uint32), er.view(np.uint32))


def test_argument_checks(cuda):
    import torch
    import gprt_b200
    from gprt_b200 import api, scenes
    L = gprt_b200.lib()
    verts, idx, types = scenes.solid_grid(2, seed=1)
    s = api.Solids(_dev(verts), _dev(idx, np.int32), _dev(types))
    _, boxes = api.solid_bounds(s)
    bvh = api.lbvh_build_boxes(boxes)
    scr = api.scratch(L.gprtcuTraceScratchSize())
    pts = torch.zeros((4, 4), dtype=torch.float32, device="cuda")
    hits = torch.zeros((4, 2), dtype=torch.int32, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ok = L.gprtcuLocateSolidPoints(ctypes.byref(bvh.desc), ctypes.byref(s.desc), pts.data_ptr(), 0,
                                   hits.data_ptr(), None, scr.data_ptr(), scr.numel(), stream)
    assert ok == 0  # no points: nothing to do
    bad = api.SolidsDesc(s.desc.vertices, s.desc.indices, s.desc.types, s.n, 24, 0, 0)  # stride not 16-multiple
    assert L.gprtcuSolidBounds(ctypes.byref(bad), None, boxes.data_ptr(), stream) == 1
    other = api.SolidsDesc(s.desc.vertices, s.desc.indices, s.desc.types, s.n - 1, 0, 0, 0)  # not the built set
    assert L.gprtcuLocateSolidPoints(ctypes.byref(bvh.desc), ctypes.byref(other), pts.data_ptr(), 4,
                                     hits.data_ptr(), None, scr.data_ptr(), scr.numel(), stream) == 1
