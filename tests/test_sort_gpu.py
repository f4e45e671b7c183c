"""Radix sort on the GPU through the C ABI, bit-exact against the oracle
(std::stable_sort, the semantics of tests/t02-bufferSort's std::sort check)."""
import os

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _zipf_u32(rng, n, s=1.1):
    # rank r in [1, 2^32-1] by inverse-CDF of a continuous power law, key = r-1
    u = rng.random(n)
    r = np.floor((1 - u) ** (-1.0 / (s - 1.0)))
    r = np.clip(r, 1, 2 ** 32 - 1)
    return (r - 1).astype(np.uint64).astype(np.uint32)


def _dists(rng, n, bits=32):
    top = 2 ** bits
    yield "uniform", rng.integers(0, top, size=n, dtype=np.uint64)
    yield "equal", np.full(n, 12345 % top, np.uint64)
    yield "sorted", np.sort(rng.integers(0, top, size=n, dtype=np.uint64))
    yield "reverse", np.sort(rng.integers(0, top, size=n, dtype=np.uint64))[::-1].copy()
    yield "fewdistinct", rng.choice(np.array([3, 77, 1 << (bits - 1), top - 1], np.uint64), size=n)


def _sort_gpu(torch, keys_np, vals_np=None, begin=0, end=None):
    from gprt_b200 import api
    kt = torch.from_numpy(keys_np.view(np.int32 if keys_np.itemsize == 4 else np.int64).copy()).cuda()
    vt = None
    if vals_np is not None:
        vt = torch.from_numpy(vals_np.view(np.int32 if vals_np.itemsize == 4 else np.int64).copy()).cuda()
    api.sort(kt, vt, begin, end)
    torch.cuda.synchronize()
    k = kt.cpu().numpy().view(keys_np.dtype)
    v = None if vt is None else vt.cpu().numpy().view(vals_np.dtype)
    return k, v


@pytest.mark.parametrize("n", [1, 2, 31, 32, 33, 4095, 4096, 4097, 8191, 8192, 8193, 100003, 1 << 20])
def test_sort_pairs_u32_sizes(cuda, n):
    import torch
    rng = np.random.default_rng(n)
    for name, k in _dists(rng, n):
        k = k.astype(np.uint32)
        v = np.arange(n, dtype=np.uint32)  # payload = original index: stability is visible
        gk, gv = _sort_gpu(torch, k, v)
        ek, ev = oracle.sort(k, v)
        assert np.array_equal(gk, ek), (n, name)
        assert np.array_equal(gv, ev), (n, name)


def test_sort_keys_only_and_t02_shape(cuda):
    import torch
    rng = np.random.default_rng(7)
    n = 3_000_017
    k = rng.integers(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)
    gk, _ = _sort_gpu(torch, k)
    assert np.array_equal(gk, np.sort(k))
    # t02 key/value form: keys a shuffled permutation, values random
    perm = rng.permutation(n).astype(np.uint32)
    vals = rng.integers(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)
    gk, gv = _sort_gpu(torch, perm, vals)
    order = np.argsort(perm, kind="stable")
    assert np.array_equal(gk, perm[order]) and np.array_equal(gv, vals[order])


def test_sort_zipf_pairs(cuda):
    import torch
    rng = np.random.default_rng(11)
    n = 1 << 22
    k = _zipf_u32(rng, n)
    v = np.arange(n, dtype=np.uint32)
    gk, gv = _sort_gpu(torch, k, v)
    ek, ev = oracle.sort(k, v)
    assert np.array_equal(gk, ek) and np.array_equal(gv, ev)


def test_sort_bit_ranges(cuda):
    import torch
    rng = np.random.default_rng(5)
    n = 200_001
    k = rng.integers(0, 1 << 30, size=n, dtype=np.uint64).astype(np.uint32)  # Morton-like 30-bit
    v = np.arange(n, dtype=np.uint32)
    gk, gv = _sort_gpu(torch, k, v, 0, 30)
    ek, ev = oracle.sort(k, v)
    assert np.array_equal(gk, ek) and np.array_equal(gv, ev)
    # a sub-range: stable sort by bits [8, 20) only
    gk, gv = _sort_gpu(torch, k, v, 8, 20)
    order = np.argsort((k >> 8) & 0xFFF, kind="stable")
    assert np.array_equal(gk, k[order]) and np.array_equal(gv, v[order])


@pytest.mark.parametrize("vw", [0, 4, 8])
def test_sort_u64_keys(cuda, vw):
    import torch
    rng = np.random.default_rng(100 + vw)
    for n in (1, 3, 4095, 4097, 65536 + 5, 1 << 20):
        for name, k in _dists(rng, n, 64 if n < 70000 else 63):
            v = None
            if vw == 4:
                v = np.arange(n, dtype=np.uint32)
            elif vw == 8:
                v = (np.arange(n, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15))
            gk, gv = _sort_gpu(torch, k, v)
            if v is None:
                assert np.array_equal(gk, np.sort(k)), (n, name)
            else:
                ek, ev = oracle.sort(k, v)
                assert np.array_equal(gk, ek) and np.array_equal(gv, ev), (n, name)


def test_sort_segmented_keys(cuda):
    # meshID << 32 | morton30: the batched-build key (44 significant bits).
    import torch
    rng = np.random.default_rng(9)
    n = 1_000_003
    mesh = rng.integers(0, 4096, size=n, dtype=np.uint64)
    code = rng.integers(0, 1 << 30, size=n, dtype=np.uint64)
    k = (mesh << np.uint64(32)) | code
    v = np.arange(n, dtype=np.uint32)
    gk, gv = _sort_gpu(torch, k, v, 0, 44)
    ek, ev = oracle.sort(k, v)
    assert np.array_equal(gk, ek) and np.array_equal(gv, ev)


def test_sort_golden_fixture(cuda):
    import torch
    g = np.load(os.path.join(GOLD, "sortscan.npz"))
    gk, gv = _sort_gpu(torch, g["keys"], np.arange(g["keys"].size, dtype=np.uint32))
    assert np.array_equal(gk, g["keys_sorted"]) and np.array_equal(gv, g["vals_sorted"])
    gk, gv = _sort_gpu(torch, g["keys64"], np.arange(g["keys64"].size, dtype=np.uint32))
    assert np.array_equal(gk, g["keys64_sorted"]) and np.array_equal(gv, g["vals64_sorted"])


def test_sort_host_errors(cuda):
    import torch
    import gprt_b200
    from gprt_b200 import api
    L = gprt_b200.lib()
    k = torch.zeros(100, dtype=torch.int32, device="cuda")
    scr = api.scratch(16)
    assert L.gprtcuSortKeysU32(api._ptr(k), 100, 0, 32, api._ptr(scr), scr.numel(), api._stream()) == 3
    big = api.scratch(api.sort_scratch_size(100, 4, 0))
    assert L.gprtcuSortKeysU32(api._ptr(k), 100, 0, 33, api._ptr(big), big.numel(), api._stream()) == 1
    assert L.gprtcuSortKeysU32(api._ptr(k), 100, 5, 5, api._ptr(big), big.numel(), api._stream()) == 1


_TYPES = [(4, 0), (4, 4), (4, 8), (8, 0), (8, 4), (8, 8)]


@pytest.mark.parametrize("kw,vw", _TYPES)
def test_sort_every_tuning_shape(cuda, kw, vw):
    # every shape of the tuner's grid is a correct stable sort on ragged sizes
    import torch
    from gprt_b200 import api
    rng = np.random.default_rng(kw * 10 + vw)
    kdt = np.uint32 if kw == 4 else np.uint64
    for cfg in api.sort_configs():
        for n in (cfg[1] - 1, 3 * cfg[1] + 17):
            if kw == 4:
                k = rng.integers(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)
            else:
                k = rng.integers(0, 2 ** 63, size=n, dtype=np.uint64) | (rng.integers(0, 2, size=n, dtype=np.uint64) << 63)
            k[::7] = k[0]  # repeated keys make stability visible
            v = None
            if vw:
                v = np.arange(n, dtype=np.uint32 if vw == 4 else np.uint64)
            kt = torch.from_numpy(k.view(np.int32 if kw == 4 else np.int64).copy()).cuda()
            vt = None if v is None else torch.from_numpy(v.view(np.int32 if vw == 4 else np.int64).copy()).cuda()
            api.sort_with_config(kt, vt, cfg)
            got = kt.cpu().numpy().view(kdt)
            if v is None:
                assert np.array_equal(got, np.sort(k, kind="stable")), (cfg, n)
            else:
                ek, ev = oracle.sort(k, v)
                assert np.array_equal(got, ek), (cfg, n)
                assert np.array_equal(vt.cpu().numpy().view(v.dtype), ev), (cfg, n)


def test_sort_autotune_installs_a_shape(cuda):
    import torch
    from gprt_b200 import api
    try:
        best, times = api.sort_autotune(4, 4, 1 << 20, repeats=1)
        assert best in times and times[best] is not None
        assert all(t is None or t > 0 for t in times.values())
        assert times[best] == min(t for t in times.values() if t is not None)
        assert api.sort_get_config(4, 4) == best
        # a sort through the plain entry point now runs the tuned shape
        rng = np.random.default_rng(3)
        k = rng.integers(0, 2 ** 32, size=300001, dtype=np.uint64).astype(np.uint32)
        v = np.arange(k.size, dtype=np.uint32)
        gk, gv = _sort_gpu(torch, k, v)
        ek, ev = oracle.sort(k, v)
        assert np.array_equal(gk, ek) and np.array_equal(gv, ev)
        # tuning on caller keys (a device copy is sorted, the sample is untouched)
        sample = torch.from_numpy(_zipf_u32(rng, 1 << 18).view(np.int32)).cuda()
        before = sample.clone()
        best2, _ = api.sort_autotune(4, 0, sample.numel(), sample=sample, repeats=1)
        assert torch.equal(sample, before) and api.sort_get_config(4, 0) == best2
    finally:
        api.sort_set_config(4, 4, None)
        api.sort_set_config(4, 0, None)


@pytest.mark.parametrize("kw,vw", [(4, 4), (4, 8), (8, 4)])
def test_sort_rankings_agree(cuda, kw, vw):
    # the 8-bit passes have several kernels (test switch): the trimmed pass
    # ranking by leader tables (default), the original pass, and the trimmed
    # pass ranking by shared-memory OR words, match.any, plain votes and
    # predicated votes; all must give the oracle's bits
    import torch
    import gprt_b200
    from gprt_b200 import api
    L = gprt_b200.lib()
    rng = np.random.default_rng(kw * 100 + vw)
    kdt = np.uint32 if kw == 4 else np.uint64
    try:
        for n in (8191, 65536 + 3, 1 << 21):
            for name, k in _dists(rng, n, 32 if kw == 4 else 44):
                k = k.astype(kdt)
                if name == "uniform":
                    k[::5] = k[1]
                v = rng.integers(0, 2 ** 63, size=n, dtype=np.uint64)
                v = v.astype(np.uint32) if vw == 4 else v
                ek, ev = oracle.sort(k, v)
                for mode in (0, 1, 2, 3, 4, 5):
                    L.gprtcuDebugSortRanking(mode)
                    kt = torch.from_numpy(k.view(np.int32 if kw == 4 else np.int64).copy()).cuda()
                    vt = torch.from_numpy(v.view(np.int32 if vw == 4 else np.int64).copy()).cuda()
                    api.sort(kt, vt, 0, 32 if kw == 4 else 44)
                    assert np.array_equal(kt.cpu().numpy().view(kdt), ek), (n, name, mode)
                    assert np.array_equal(vt.cpu().numpy().view(v.dtype), ev), (n, name, mode)
    finally:
        L.gprtcuDebugSortRanking(0)


@pytest.mark.parametrize("kw,vw", [(4, 4), (4, 0), (8, 4)])
def test_sort_l2_prefetch_distances_agree(cuda, kw, vw):
    # the 8-bit passes prefetch a later tile into L2 (a cache hint); every
    # distance, none included, must give the oracle's bits
    import torch
    import gprt_b200
    from gprt_b200 import api
    L = gprt_b200.lib()
    rng = np.random.default_rng(7 * kw + vw)
    kdt = np.uint32 if kw == 4 else np.uint64
    n = (1 << 22) + 5
    k = _zipf_u32(rng, n).astype(kdt) if kw == 4 else rng.integers(0, 2 ** 44, size=n, dtype=np.uint64)
    v = rng.integers(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32) if vw else None
    ek, ev = oracle.sort(k, v) if vw else (oracle.sort(k), None)
    try:
        for q in (0, 1, 2, 4, 64):
            L.gprtcuDebugSortPrefetch(q)
            kt = torch.from_numpy(k.view(np.int32 if kw == 4 else np.int64).copy()).cuda()
            vt = torch.from_numpy(v.view(np.int32).copy()).cuda() if vw else None
            api.sort(kt, vt, 0, 32 if kw == 4 else 44)
            assert np.array_equal(kt.cpu().numpy().view(kdt), ek), q
            if vw:
                assert np.array_equal(vt.cpu().numpy().view(np.uint32), ev), q
    finally:
        L.gprtcuDebugSortPrefetch(2)


def test_sort_beyond_2_30_keys(cuda):
    # n past 2^30 - 1 needs the wide look-back words; checked through
    # size-independent properties: keys ascending, the payload (original
    # index) a permutation that maps every key back to its input, equal keys
    # in input order (stability)
    import torch
    from gprt_b200 import api
    n = (1 << 30) + 4097
    g = torch.Generator(device="cuda").manual_seed(99)
    k0 = torch.randint(-2 ** 31, 2 ** 31 - 1, (n,), generator=g, dtype=torch.int32, device="cuda")
    k0[::3] = k0[7]  # many equal keys
    k = k0.clone()
    v = torch.arange(n, dtype=torch.int32, device="cuda")
    scr = api.scratch(api.sort_scratch_size(n, 4, 4))
    api.sort(k, v, 0, 32, scr)
    torch.cuda.synchronize()
    assert api.scratch_status(scr) == 0
    step = 1 << 27
    for lo in range(0, n, step):
        hi = min(n, lo + step + 1)
        ku = k[lo:hi].to(torch.int64) & 0xFFFFFFFF
        vi = v[lo:hi].to(torch.int64)
        assert bool(torch.all(ku[1:] >= ku[:-1]))
        assert bool(torch.equal(k0[vi], k[lo:hi]))
        same = ku[1:] == ku[:-1]
        assert bool(torch.all(vi[1:][same] > vi[:-1][same]))
    seen = torch.zeros(n, dtype=torch.bool, device="cuda")
    seen[v.to(torch.int64)] = True
    assert bool(seen.all())
