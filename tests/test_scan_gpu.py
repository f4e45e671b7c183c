"""Scan, partition and select on the GPU through the C ABI, bit-exact against
the oracle and the reference tests' known answers."""
import os

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _run_scan(torch, x, inclusive=False, alias=False, offset=0):
    from gprt_b200 import api
    buf = torch.zeros(x.size + offset, dtype=torch.int32, device="cuda")
    d = buf[offset:]
    d.copy_(torch.from_numpy(x.view(np.int32)))
    out = d if alias else torch.empty_like(d)
    out, total = api.exclusive_sum(d, out, inclusive=inclusive)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint32), int(total.cpu().numpy().view(np.uint32)[0])


@pytest.fixture(params=[0, 1, 2, 3], ids=["automatic", "register_staged", "tma_staged", "persistent_reread"])
def scan_impl(request, cuda):
    import gprt_b200
    gprt_b200.lib().gprtcuDebugScanImpl(request.param)
    yield request.param
    gprt_b200.lib().gprtcuDebugScanImpl(0)


@pytest.mark.parametrize("inclusive", [False, True])
def test_scan_sizes(cuda, scan_impl, inclusive):
    import torch
    rng = np.random.default_rng(0)
    sizes = [1, 2, 31, 32, 33, 1023, 1024, 1025, 4095, 8191, 8192, 8193, 16384 + 7, 100003, 1 << 20, (1 << 22) + 4]
    for n in sizes:
        x = rng.integers(0, 256, size=n, dtype=np.uint32)
        got, total = _run_scan(torch, x, inclusive)
        exp, etotal = oracle.scan(x, inclusive)
        assert np.array_equal(got, exp), n
        assert total == etotal, n


def test_scan_t03_schedule_all_ones(cuda):
    # tests/t03-bufferScans/hostCode.cpp:28-81: N = 9973*k, all ones.
    import torch
    for k in range(2, 102, 9):
        n = 9973 * k
        got, total = _run_scan(torch, np.ones(n, np.uint32))
        assert total == n
        assert np.array_equal(got, np.arange(n, dtype=np.uint32)), n


def test_scan_golden_and_wraparound(cuda):
    import torch
    g = np.load(os.path.join(GOLD, "sortscan.npz"))
    got, total = _run_scan(torch, g["scan_in"])
    assert np.array_equal(got, g["scan_excl"]) and total == int(g["scan_total"])
    got, _ = _run_scan(torch, g["big_in"])
    assert np.array_equal(got, g["big_excl"])
    # aggregate beyond 2^30 (the reference's cap) and beyond 2^32 (wraps)
    x = np.full(1 << 20, 5000, np.uint32)
    got, total = _run_scan(torch, x)
    exp, etotal = oracle.scan(x)
    assert np.array_equal(got, exp) and total == etotal


def test_scan_in_place_and_misaligned(cuda, scan_impl):
    import torch
    rng = np.random.default_rng(1)
    x = rng.integers(0, 1 << 31, size=300007, dtype=np.uint32)
    exp, etotal = oracle.scan(x)
    got, total = _run_scan(torch, x, alias=True)
    assert np.array_equal(got, exp) and total == etotal
    got, total = _run_scan(torch, x, offset=1)  # 4-byte aligned only: scalar path
    assert np.array_equal(got, exp) and total == etotal
    got, total = _run_scan(torch, x, inclusive=True, alias=True, offset=3)
    assert np.array_equal(got, oracle.scan(x, True)[0])


def test_scan_large_uniform(cuda):
    import torch
    rng = np.random.default_rng(2)
    n = (1 << 26) + 12345
    x = rng.integers(0, 256, size=n, dtype=np.uint32)
    got, total = _run_scan(torch, x)
    exp, etotal = oracle.scan(x)
    assert total == etotal
    assert np.array_equal(got, exp)


def test_scan_empty(cuda):
    import torch
    from gprt_b200 import api
    d = torch.empty(0, dtype=torch.int32, device="cuda")
    total = torch.full((1,), 77, dtype=torch.int32, device="cuda")
    api.exclusive_sum(d, torch.empty_like(d), total)
    assert int(total.item()) == 0


@pytest.mark.parametrize("select_only", [False, True])
def test_partition_select_t03(cuda, select_only, scan_impl):
    # tests/t03-bufferScans/hostCode.cpp:91-241 on the t03 schedule.
    import torch
    from gprt_b200 import api
    for k in (2, 3, 10, 57, 101):
        n = 9973 * k
        i = np.arange(n, dtype=np.int64)
        x = (i * np.where(i & 1, 1, -1)).astype(np.int32)
        d = torch.from_numpy(x).cuda()
        out, cnt = api.partition(d, True, select_only=select_only)
        exp, etot = oracle.partition(x, True, not select_only)
        got = out.cpu().numpy()
        assert int(cnt.item()) == etot
        if select_only:
            assert np.array_equal(got[:etot], exp[:etot])
        else:
            assert np.array_equal(got, exp)


def test_partition_negative_select_and_random(cuda, scan_impl):
    import torch
    from gprt_b200 import api
    rng = np.random.default_rng(4)
    for n in (1, 5, 8191, 8193, 100000, (1 << 20) + 3, 3000017):
        x = rng.integers(-2 ** 31, 2 ** 31, size=n, dtype=np.int64).astype(np.int32)
        d = torch.from_numpy(x).cuda()
        for sp in (True, False):
            out, cnt = api.partition(d, sp)
            exp, etot = oracle.partition(x, sp, True)
            assert int(cnt.item()) == etot and np.array_equal(out.cpu().numpy(), exp), (n, sp)
            out, cnt = api.partition(d, sp, select_only=True)
            exp, etot = oracle.partition(x, sp, False)
            assert int(cnt.item()) == etot and np.array_equal(out.cpu().numpy()[:etot], exp[:etot]), (n, sp)


def test_partition_edges_and_alignment(cuda):
    # One-sided inputs (every item selected: the unselected run is empty, and
    # the reverse), the int32 extremes and zeros, and buffers starting 4 bytes
    # past a 16-byte boundary (input or output), which take the tile-per-CTA
    # kernel instead of the persistent one.
    import torch
    from gprt_b200 import api
    rng = np.random.default_rng(5)
    n = (1 << 21) + 5
    cases = {
        "nonneg": rng.integers(0, 2 ** 31, size=n, dtype=np.int64).astype(np.int32),
        "neg": rng.integers(-2 ** 31, 0, size=n, dtype=np.int64).astype(np.int32),
        "extremes": rng.choice(np.array([-2 ** 31, -1, 0, 1, 2 ** 31 - 1], dtype=np.int32), size=n),
    }
    for name, x in cases.items():
        for shift_in, shift_out in ((0, 0), (1, 0), (0, 1)):
            buf = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
            buf[shift_in:shift_in + n] = torch.from_numpy(x).cuda()
            d = buf[shift_in:shift_in + n]
            for sp in (True, False):
                for sel in (False, True):
                    obuf = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
                    out = obuf[shift_out:shift_out + n]
                    _, cnt = api.partition(d, sp, out=out, select_only=sel)
                    exp, etot = oracle.partition(x, sp, not sel)
                    got = out.cpu().numpy()
                    k = etot if sel else n
                    assert int(cnt.item()) == etot and np.array_equal(got[:k], exp[:k]), (name, shift_in, shift_out, sp, sel)


def test_scan_lookback_timeout_is_reported_not_hung(cuda, scan_impl):
    # Fault injection without a GPU fault: one tile never publishes; its
    # successors exhaust a small wait budget, record TIMEOUT and return.
    import torch
    import gprt_b200
    from gprt_b200 import api
    L = gprt_b200.lib()
    n = 8192 * 40
    d = torch.ones(n, dtype=torch.int32, device="cuda")
    scr = api.scratch(api.scan_scratch_size(n))
    L.gprtcuDebugSetSpinBudget(2000)
    L.gprtcuDebugScanSkipTile(3)
    try:
        api.exclusive_sum(d, torch.empty_like(d), scr=scr)
        torch.cuda.synchronize()
        assert api.scratch_status(scr) == 4
    finally:
        L.gprtcuDebugScanSkipTile(-1)
        L.gprtcuDebugSetSpinBudget(0)
    # the context is still usable and a normal call succeeds
    out, total = api.exclusive_sum(d, torch.empty_like(d), scr=scr)
    torch.cuda.synchronize()
    assert api.scratch_status(scr) == 0 and int(total.item()) == n
