"""The drop-in API (include/gprt_compat.h) exercised by C++ programs that
re-express the reference's own tests (tests/t02-bufferSort,
tests/t03-bufferScans, tests/t04-swBVH), built by __graft_entry__.build()."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
BIN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cpp", "_build")


def _run(name, *args, timeout=900):
    exe = os.path.join(BIN, name)
    if not os.path.exists(exe):
        pytest.fail("%s not built (run __graft_entry__.build())" % exe)
    r = subprocess.run([exe] + [str(a) for a in args], capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def test_t02_sort_100m_keys(cuda):
    assert "ok" in _run("t02_sort")


def test_t03_scans_schedule(cuda):
    assert "ok" in _run("t03_scans", 100)


def test_t04_lbvh(cuda):
    assert "ok" in _run("t04_lbvh")
