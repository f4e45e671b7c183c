"""gprt_b200 -- B200-native (sm_100a) acceleration-structure path of GPRT.

The product is the C-ABI shared library ``libgprtcu.so`` built from
``gprt_b200/csrc`` (declared in ``include/gprtcu.h`` and
``include/gprt_compat.h``).  This package loads it with ctypes and offers thin
wrappers that take torch CUDA tensors (PyTorch provides device memory and
streams; it does no compute on the path).

There is no CPU fallback: if the library is missing or no CUDA device is
present, the calls raise.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgprtcu.so")

_lib = None


class GprtcuError(RuntimeError):
    def __init__(self, status, where=""):
        self.status = status
        name = lib().gprtcuStatusString(status).decode() if _lib is not None else str(status)
        super().__init__("%s failed: %s (%d)" % (where, name, status))


def lib():
    """The loaded libgprtcu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libgprtcu.so is not built; run `python -m gprt_b200.build` "
                              "(or __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        from . import _sigs
        _sigs.declare(L)
        _lib = L
    return _lib


from . import api  # noqa: E402,F401
