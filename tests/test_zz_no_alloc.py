"""gprtcuExclusiveSumU32NoAlloc: the exclusive sum for callers that cannot
allocate device work space (an application that owns the device-memory
budget and lends the library only its input and output buffers, or a binding
that cannot keep a device allocation alive between calls).  It must give the
same results as gprtcuExclusiveSumU32 with caller scratch, call after call,
even though every call reuses one fixed array inside the library.

This file is named to be collected last, so a run that stops at its first
failure has already run every other test; it also passes alone in a fresh
process (its first call then performs the per-device set-up)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NOALLOC_MAX_N = 1 << 28
TOO_LARGE = 6


def _call_noalloc(x, stream):
    import torch
    import gprt_b200
    out = torch.empty_like(x)
    total = torch.full((1,), -1, dtype=torch.int32, device=x.device)
    st = gprt_b200.lib().gprtcuExclusiveSumU32NoAlloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                                      x.numel(), ctypes.c_void_p(total.data_ptr()), stream)
    return st, out, total


def test_no_alloc_matches_scratch_entry_point_on_consecutive_calls(cuda):
    import torch
    from gprt_b200 import api
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(123)
    # Two calls in a row; the second is smaller, so any state the first left
    # in the shared array would show up if it were not cleared.
    for n, hi in ((3_000_017, 1 << 12), (100_003, 1 << 31)):
        x = torch.from_numpy(rng.integers(0, hi, size=n, dtype=np.uint32).view(np.int32)).cuda()
        ref_out, ref_total = api.exclusive_sum(x)  # existing entry point, caller scratch
        st, out, total = _call_noalloc(x, stream)
        assert st == 0
        torch.cuda.synchronize()
        assert torch.equal(out, ref_out), n
        assert int(total.item()) == int(ref_total.item()), n


def test_no_alloc_matches_the_oracle(cuda):
    import torch
    import oracle
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(321)
    for n in (1, 8191, 8192 * 3 + 1, (1 << 20) + 13):
        x = rng.integers(0, 256, size=n, dtype=np.uint32)
        st, out, total = _call_noalloc(torch.from_numpy(x.view(np.int32)).cuda(), stream)
        assert st == 0
        torch.cuda.synchronize()
        exp, etotal = oracle.scan(x)
        assert np.array_equal(out.cpu().numpy().view(np.uint32), exp), n
        assert int(total.item()) & 0xFFFFFFFF == etotal, n


def _noalloc_status(stream):
    import gprt_b200
    v = ctypes.c_int(-1)
    assert gprt_b200.lib().gprtcuScratchStatus(None, stream, ctypes.byref(v)) == 0
    return v.value


def test_no_alloc_reports_a_device_timeout(cuda):
    # The fixed array has no address the caller knows, so its status is read
    # with a NULL scratch.  A tile that never publishes (test hook) makes its
    # successors' waits run out; the next call clears the status again.
    import torch
    import gprt_b200
    L = gprt_b200.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    x = torch.ones(8192 * 40, dtype=torch.int32, device="cuda")
    L.gprtcuDebugSetSpinBudget(2000)
    L.gprtcuDebugScanSkipTile(3)
    try:
        st, _, _ = _call_noalloc(x, stream)
        assert st == 0
        assert _noalloc_status(stream) == 4
    finally:
        L.gprtcuDebugScanSkipTile(-1)
        L.gprtcuDebugSetSpinBudget(0)
    st, out, total = _call_noalloc(x, stream)
    assert st == 0 and _noalloc_status(stream) == 0
    assert int(total.item()) == x.numel()
    assert torch.equal(out, torch.arange(x.numel(), dtype=torch.int32, device="cuda"))


def test_no_alloc_rejects_sizes_beyond_its_fixed_array(cuda):
    import torch
    import gprt_b200
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = gprt_b200.lib().gprtcuExclusiveSumU32NoAlloc(None, None, NOALLOC_MAX_N + 1, None, stream)
    assert st == TOO_LARGE
