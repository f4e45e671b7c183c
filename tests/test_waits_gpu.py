"""Every bounded device-side wait gives up, reports GPRTCU_ERR_TIMEOUT and
leaves the context usable -- without a GPU fault.

Each test plants the failure on the host through a test hook (a tile that
never publishes, a scan stage that is never filled, a leaf that never stores
its box), shortens the wait budget, checks the recorded status, then runs the
same call again without the hook and checks its result against the oracle."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TIMEOUT = 4
SHORT_BUDGET = 2000


@pytest.fixture
def hooks(cuda):
    import gprt_b200
    L = gprt_b200.lib()
    yield L
    L.gprtcuDebugScanSkipTile(-1)
    L.gprtcuDebugScanSkipStage(-1)
    L.gprtcuDebugSortSkipTile(-1)
    L.gprtcuDebugRefitSkipLeaf(-1)
    L.gprtcuDebugScanImpl(0)
    L.gprtcuDebugSetSpinBudget(0)


@pytest.mark.parametrize("mode", ["sum", "partition", "select"])
def test_scanners_stop_together_when_a_stage_never_fills(hooks, mode):
    # The persistent scan kernel's scanner warps meet at named barriers; when
    # their wait for a stage runs out they must all leave together, record the
    # timeout, and let the kernel end.
    import torch
    import oracle
    from gprt_b200 import api
    n = 8192 * 400 + 77  # >= 2^20: the persistent re-read kernel
    rng = np.random.default_rng(5)
    x = rng.integers(-2 ** 31, 2 ** 31, size=n, dtype=np.int64).astype(np.int32)
    d = torch.from_numpy(x).cuda()
    scr = api.scratch(api.scan_scratch_size(n))
    hooks.gprtcuDebugScanImpl(3)
    hooks.gprtcuDebugSetSpinBudget(SHORT_BUDGET)
    hooks.gprtcuDebugScanSkipStage(5)

    def run():
        if mode == "sum":
            return api.exclusive_sum(d, torch.empty_like(d), scr=scr)
        return api.partition(d, True, out=torch.zeros_like(d), scr=scr, select_only=mode == "select")

    run()
    torch.cuda.synchronize()
    assert api.scratch_status(scr) == TIMEOUT
    hooks.gprtcuDebugScanSkipStage(-1)
    hooks.gprtcuDebugSetSpinBudget(0)
    out, tot = run()
    torch.cuda.synchronize()
    assert api.scratch_status(scr) == 0
    got = out.cpu().numpy()
    if mode == "sum":
        exp, etot = oracle.scan(x.view(np.uint32))
        assert np.array_equal(got.view(np.uint32), exp) and int(tot.item()) & 0xFFFFFFFF == etot
    else:
        exp, etot = oracle.partition(x, True, mode == "partition")
        k = etot if mode == "select" else n
        assert int(tot.item()) == etot and np.array_equal(got[:k], exp[:k])


@pytest.mark.parametrize("n", [8192 * 64 + 5, 1 << 22])
def test_sort_lookback_timeout_is_reported_not_hung(hooks, n):
    # One tile of every pass never publishes its digit counts: its successors
    # run out of budget and poison the chain, later passes see the error and
    # do nothing (their digit offsets no longer bound their writes).
    import torch
    import oracle
    from gprt_b200 import api
    rng = np.random.default_rng(11)
    k = rng.integers(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)
    v = np.arange(n, dtype=np.uint32)
    dk = torch.from_numpy(k.view(np.int32)).cuda()
    dv = torch.from_numpy(v.view(np.int32)).cuda()
    scr = api.scratch(api.sort_scratch_size(n, 4, 4))
    hooks.gprtcuDebugSetSpinBudget(SHORT_BUDGET)
    hooks.gprtcuDebugSortSkipTile(3)
    api.sort(dk, dv, scr=scr)
    torch.cuda.synchronize()
    assert api.scratch_status(scr) == TIMEOUT
    hooks.gprtcuDebugSortSkipTile(-1)
    hooks.gprtcuDebugSetSpinBudget(0)
    dk.copy_(torch.from_numpy(k.view(np.int32)))
    dv.copy_(torch.from_numpy(v.view(np.int32)))
    api.sort(dk, dv, scr=scr)
    torch.cuda.synchronize()
    assert api.scratch_status(scr) == 0
    ek, ev = oracle.sort(k, v)
    assert np.array_equal(dk.cpu().numpy().view(np.uint32), ek)
    assert np.array_equal(dv.cpu().numpy().view(np.uint32), ev)


def _soup(n, seed):
    from gprt_b200 import scenes
    return scenes.soup(n, seed=seed, sigma=0.01)


def _assert_build_matches_oracle(bvh, pos, tri):
    import oracle
    h = bvh.host()
    e = oracle.lbvh_build_tri(pos, tri)
    for key in ("codes", "ids", "nodes", "aabbs"):
        assert np.array_equal(np.ascontiguousarray(h[key]).view(np.uint32),
                              np.ascontiguousarray(e[key].reshape(h[key].shape)).view(np.uint32)), key


@pytest.mark.parametrize("slot", [0, 1, 777])
def test_refit_sibling_wait_timeout_is_reported_not_hung(hooks, slot):
    # The leaf in sorted slot `slot` never stores its box: whichever child of
    # its parent arrives second waits for that box, runs out of budget and
    # records the timeout.
    import torch
    from gprt_b200 import api
    pos, tri = _soup(5000, 21)
    p = torch.from_numpy(pos).cuda()
    t = torch.from_numpy(tri.view(np.int32)).cuda()
    bvh = api.Lbvh(tri.shape[0])
    assert hooks.gprtcuDebugRefitSkipLeaf(slot) == 0
    hooks.gprtcuDebugSetSpinBudget(SHORT_BUDGET)
    api.lbvh_build_triangles(p, t, bvh)
    torch.cuda.synchronize()
    assert api.scratch_status(bvh.scratch) == TIMEOUT
    assert hooks.gprtcuDebugRefitSkipLeaf(-1) == 0
    hooks.gprtcuDebugSetSpinBudget(0)
    api.lbvh_build_triangles(p, t, bvh)
    torch.cuda.synchronize()
    assert api.scratch_status(bvh.scratch) == 0
    _assert_build_matches_oracle(bvh, pos, tri)


def test_lbvh_build_reports_its_sorts_timeout_and_stays_in_bounds(hooks):
    # The sort inside the build gives up: the build reports the sort's error
    # in its own header, and the tree it leaves is still a valid tree (every
    # code treated as equal, each leaf its own slot's triangle), so a trace
    # over it reads only in-bounds memory.
    import torch
    from gprt_b200 import api, scenes
    pos, tri = _soup(50000, 22)
    p = torch.from_numpy(pos).cuda()
    t = torch.from_numpy(tri.view(np.int32)).cuda()
    rays = torch.from_numpy(scenes.rays(4096, seed=23)).cuda()
    bvh = api.Lbvh(tri.shape[0])
    hooks.gprtcuDebugSetSpinBudget(SHORT_BUDGET)
    hooks.gprtcuDebugSortSkipTile(2)
    api.lbvh_build_triangles(p, t, bvh)
    torch.cuda.synchronize()
    assert api.scratch_status(bvh.scratch) == TIMEOUT
    hits = api.hits_numpy(api.trace(bvh, rays))
    torch.cuda.synchronize()
    ok = hits["prim"] != 0xFFFFFFFF
    assert np.all(hits["prim"][ok] < tri.shape[0])
    hooks.gprtcuDebugSortSkipTile(-1)
    hooks.gprtcuDebugSetSpinBudget(0)
    api.lbvh_build_triangles(p, t, bvh)
    torch.cuda.synchronize()
    assert api.scratch_status(bvh.scratch) == 0
    _assert_build_matches_oracle(bvh, pos, tri)


def test_compat_sort_with_caller_scratch_reports_device_error_at_map(hooks):
    # gprtBufferSort[Payload] with the caller's scratch stays asynchronous; a
    # device-side timeout is folded into a host word on the stream and
    # reported at the next synchronisation (here gprtBufferMap).
    import torch
    import oracle
    import gprt_b200
    L = ctypes.CDLL(gprt_b200.LIB_PATH)  # own handle: the signatures below stay local to this test
    vp = ctypes.c_void_p
    L.gprtContextCreate.restype = vp
    L.gprtContextCreate.argtypes = [vp, ctypes.c_int]
    L.gprtDeviceBufferCreate.restype = vp
    L.gprtDeviceBufferCreate.argtypes = [vp, ctypes.c_size_t, ctypes.c_size_t, vp, ctypes.c_size_t]
    L.gprtBufferGetHostPointer.restype = vp
    L.gprtBufferGetHostPointer.argtypes = [vp, ctypes.c_int]
    L.gprtBufferMap.argtypes = [vp, ctypes.c_int]
    L.gprtBufferDestroy.argtypes = [vp]
    L.gprtContextDestroy.argtypes = [vp]
    L.gprtcuCompatSort.argtypes = [vp, vp, ctypes.c_int, vp, ctypes.c_int, vp]
    n = 8192 * 64 + 3
    rng = np.random.default_rng(31)
    k = rng.integers(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)
    v = np.arange(n, dtype=np.uint32)
    ctx = L.gprtContextCreate(None, 0)
    assert ctx
    bufs = []
    try:
        kb = L.gprtDeviceBufferCreate(ctx, 4, n, k.ctypes.data, 16)
        vb = L.gprtDeviceBufferCreate(ctx, 4, n, v.ctypes.data, 16)
        sb = L.gprtDeviceBufferCreate(ctx, 1, 256, None, 16)  # grown by the call, as in the reference
        bufs = [kb, vb, sb]
        L.gprtcuCompatLastError()
        L.gprtcuDebugSetSpinBudget(SHORT_BUDGET)
        L.gprtcuDebugSortSkipTile(3)
        L.gprtcuCompatSort(ctx, kb, 4, vb, 4, sb)
        assert L.gprtcuCompatLastError() == 0  # asynchronous: nothing known yet
        L.gprtBufferMap(kb, 0)
        assert L.gprtcuCompatLastError() == TIMEOUT
        L.gprtcuDebugSortSkipTile(-1)
        L.gprtcuDebugSetSpinBudget(0)
        # a clean run on fresh data through the same scratch
        L.gprtBufferUnmap.argtypes = [vp, ctypes.c_int]
        for b, a in ((kb, k), (vb, v)):
            hp = L.gprtBufferGetHostPointer(b, 0)
            ctypes.memmove(hp, a.ctypes.data, a.nbytes)
            L.gprtBufferUnmap(b, 0)
        L.gprtcuCompatSort(ctx, kb, 4, vb, 4, sb)
        L.gprtBufferMap(kb, 0)
        L.gprtBufferMap(vb, 0)
        assert L.gprtcuCompatLastError() == 0
        gk = np.ctypeslib.as_array(ctypes.cast(L.gprtBufferGetHostPointer(kb, 0), ctypes.POINTER(ctypes.c_uint32)),
                                   shape=(n,)).copy()
        gv = np.ctypeslib.as_array(ctypes.cast(L.gprtBufferGetHostPointer(vb, 0), ctypes.POINTER(ctypes.c_uint32)),
                                   shape=(n,)).copy()
        ek, ev = oracle.sort(k, v)
        assert np.array_equal(gk, ek) and np.array_equal(gv, ev)
    finally:
        for b in bufs:
            L.gprtBufferDestroy(b)
        L.gprtContextDestroy(ctx)
        torch.cuda.synchronize()
