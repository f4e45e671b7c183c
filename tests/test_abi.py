"""The C-ABI library loads and exports every symbol the public headers declare.
CPU only: no compute call is made."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    txt = "\n".join(l for l in txt.splitlines() if not l.lstrip().startswith("#"))
    return sorted(set(re.findall(r"GPRT(?:CU)?_API\s+[^;(]*?\b(\w+)\s*\(", txt)))


def test_headers_declare_entry_points():
    names = _declared("gprtcu.h")
    assert "gprtcuExclusiveSumU32" in names and "gprtcuScanScratchSize" in names


@pytest.mark.parametrize("header", ["gprtcu.h", "gprt_compat.h"])
def test_library_exports_every_declared_symbol(header):
    if not os.path.exists(os.path.join(ROOT, "include", header)):
        pytest.skip("header not present")
    import gprt_b200
    L = gprt_b200.lib()
    missing = [n for n in _declared(header) if not hasattr(L, n)]
    assert not missing, missing


def test_ctypes_signatures_cover_header():
    from gprt_b200 import _sigs
    names = set(_declared("gprtcu.h"))
    assert names <= set(_sigs.SIGNATURES), sorted(names - set(_sigs.SIGNATURES))


def test_host_side_argument_checks_without_gpu():
    # Host-side validation returns before any CUDA call.
    import gprt_b200
    L = gprt_b200.lib()
    assert L.gprtcuExclusiveSumU32(None, None, 10, None, None, 0, None) == 1  # INVALID_ARG
    assert L.gprtcuScanScratchSize(0) == 256
    assert L.gprtcuScanScratchSize(8192) == 256 + 256
    assert L.gprtcuStatusString(4) == b"device-side wait exceeded its budget"


def test_sort_tuning_grid_host_side():
    # host-only calls: the grid, get/set of the active shape, argument checks
    import ctypes
    from gprt_b200 import api
    grid = api.sort_configs()
    assert len(grid) == len(set(grid))
    assert {g[0] for g in grid} == {4, 6, 8}
    assert {g[1] for g in grid} == {1024, 2048, 4096, 6144, 8192}
    assert {g[2] for g in grid} == {4, 8, 16}
    for rb, tile, warps in grid:
        items = tile // (32 * warps)
        assert tile % (32 * warps) == 0 and 1 <= items <= 32 and 32 * warps >= (1 << rb)
    default = api.sort_get_config(4, 4)
    assert default in grid
    api.sort_set_config(4, 4, grid[0])
    assert api.sort_get_config(4, 4) == grid[0]
    api.sort_set_config(4, 4, None)
    assert api.sort_get_config(4, 4) == default
    L = api.lib()
    bad = api.SortConfig(5, 1024, 4)
    assert L.gprtcuSortSetConfig(4, 4, ctypes.byref(bad)) == 1
    assert L.gprtcuSortSetConfig(4, 2, ctypes.byref(api.SortConfig(*grid[0]))) == 1  # no 16-bit payloads
    assert L.gprtcuSortSetConfig(4, 8, None) == 0  # u32 keys with the reference's u64 payloads
    assert L.gprtcuSortConfigAt(len(grid), ctypes.byref(bad)) == 1
    # scratch covers the largest shape: two look-back regions at 1024-key tiles, 8-bit digits
    n = 1 << 20
    assert api.sort_scratch_size(n, 4, 4) >= 8 * n + 2 * (n // 1024) * 256 * 4
