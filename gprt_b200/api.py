"""Torch-tensor wrappers over the C ABI (include/gprtcu.h).

Every function takes CUDA tensors, enqueues on torch's current stream and
returns without synchronising unless it documents otherwise.  Scratch is
allocated by torch's caching allocator when not supplied.
"""
import ctypes

import torch

from . import GprtcuError, lib


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _check(status, where):
    if status != 0:
        raise GprtcuError(status, where)


def scratch(nbytes, device=None):
    """A 256-byte aligned device scratch buffer (torch allocations are)."""
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device or "cuda")


def scratch_status(buf):
    """Device-side status word of a scratch buffer (synchronises the stream)."""
    v = ctypes.c_int(0)
    _check(lib().gprtcuScratchStatus(_ptr(buf), _stream(), ctypes.byref(v)), "gprtcuScratchStatus")
    return v.value


def _need_cuda(*ts):
    for t in ts:
        if t is not None and not t.is_cuda:
            raise ValueError("gprt_b200 operates on CUDA tensors only (no CPU path)")


# ---------------------------------------------------------------- scan
def scan_scratch_size(n):
    return lib().gprtcuScanScratchSize(int(n))


def exclusive_sum(inp, out=None, total=None, scr=None, inclusive=False):
    """uint32 prefix sum of `inp` (int32/uint32 tensor viewed as uint32) into `out`.

    Returns (out, total_tensor) where total_tensor is a 1-element device tensor.
    """
    _need_cuda(inp)
    n = inp.numel()
    if out is None:
        out = torch.empty_like(inp)
    if total is None:
        total = torch.empty(1, dtype=torch.int32, device=inp.device)
    if scr is None:
        scr = scratch(scan_scratch_size(n), inp.device)
    f = lib().gprtcuInclusiveSumU32 if inclusive else lib().gprtcuExclusiveSumU32
    _check(f(_ptr(inp), _ptr(out), n, _ptr(total), _ptr(scr), scr.numel(), _stream()),
           "gprtcuInclusiveSumU32" if inclusive else "gprtcuExclusiveSumU32")
    return out, total


def inclusive_sum(inp, out=None, total=None, scr=None):
    return exclusive_sum(inp, out, total, scr, inclusive=True)


def partition(inp, select_positive=True, out=None, count=None, scr=None, select_only=False):
    _need_cuda(inp)
    n = inp.numel()
    if out is None:
        out = torch.zeros_like(inp)
    if count is None:
        count = torch.empty(1, dtype=torch.int32, device=inp.device)
    if scr is None:
        scr = scratch(scan_scratch_size(n), inp.device)
    f = lib().gprtcuSelectI32 if select_only else lib().gprtcuPartitionI32
    _check(f(_ptr(inp), _ptr(out), n, 1 if select_positive else 0, _ptr(count), _ptr(scr), scr.numel(), _stream()),
           "gprtcuSelectI32" if select_only else "gprtcuPartitionI32")
    return out, count


def select(inp, select_positive=True, out=None, count=None, scr=None):
    return partition(inp, select_positive, out, count, scr, select_only=True)
