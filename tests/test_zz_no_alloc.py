"""htrip_query_all_pairs_noalloc: the allocation-free query entry point.

It serves callers that may not allocate device memory once they run (a
serving process whose pool allocator holds all of HBM, a real-time planning
loop that forbids cudaMalloc / cudaFree).  Its device scratch is a fixed
64 MiB array inside the library, shared by all calls and keeping the last
call's contents.  These tests call it through the C ABI and compare it
bit-exactly (distances are integers: tolerance 0) with the allocating
htrip_query_all_pairs on two calls in a row, the second smaller than the
first so that stale contents of the larger call would show.

This file is collected last so that a run stopping at its first failure has
run every other test already.
"""
import ctypes as C

import numpy as np
import pytest

from htrip_b200.minplus_oracle import HierarchyConfig, MinPlusOracle, load_library

from helpers import make_grid, viewpoints

_U8P = C.POINTER(C.c_uint8)
_U16P = C.POINTER(C.c_uint16)
_I32P = C.POINTER(C.c_int32)
HTRIP_ERR_UNSUPPORTED = 4


def _noalloc(lib, idx, vps, grid):
    vps = np.ascontiguousarray(vps, dtype=np.int32).reshape(-1, 2)
    obs = np.ascontiguousarray(grid, dtype=np.uint8)
    k = len(vps)
    out = np.full((k, k), 0xBEEF, dtype=np.uint16)
    st = lib.htrip_query_all_pairs_noalloc(idx.h, vps.ctypes.data_as(_I32P), k, obs.ctypes.data_as(_U8P),
                                           obs.shape[0], obs.shape[1], out.ctypes.data_as(_U16P))
    return st, out


@pytest.mark.gpu
def test_noalloc_query_matches_allocating_query_twice(gpu):
    import torch

    lib = load_library()
    grid = make_grid("street", 96, 80, 4)  # non-square, S = 128, H = 4 at b = 8
    idx = MinPlusOracle(HierarchyConfig(8, 2, 2), device=0)
    assert idx.build(grid)
    # one warm-up call: the first call on a device loads the module that
    # holds the fixed array and looks up its address
    st, _ = _noalloc(lib, idx, viewpoints(grid, 5, 9), grid)
    assert st == 0, lib.htrip_last_error().decode()
    calls = [viewpoints(grid, 60, 1, include_blocked=3), viewpoints(grid, 21, 2, include_blocked=1)]
    for vps in calls:
        want = idx.queryAllPairs(vps, grid)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(0)[0]
        st, got = _noalloc(lib, idx, vps, grid)
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info(0)[0]
        assert st == 0, lib.htrip_last_error().decode()
        assert np.array_equal(got, want)
        # read right around the call, with no allocating call in between:
        # the call took no device memory and kept none
        assert free_after == free_before


@pytest.mark.gpu
def test_noalloc_query_rejects_scratch_above_its_limit(gpu):
    lib = load_library()
    grid = make_grid("rooms", 32, 32, 1)
    idx = MinPlusOracle(HierarchyConfig(8, 2, 2), device=0)
    assert idx.build(grid)
    vps = np.repeat(viewpoints(grid, 1, 3), 4200, axis=0)  # k^2 pair matrix alone > 64 MiB
    st, _ = _noalloc(lib, idx, vps, grid)
    assert st == HTRIP_ERR_UNSUPPORTED
    assert "64" in lib.htrip_last_error().decode() or "bytes" in lib.htrip_last_error().decode()
    # the index still answers through both entry points afterwards
    small = viewpoints(grid, 9, 4)
    st, got = _noalloc(lib, idx, small, grid)
    assert st == 0
    assert np.array_equal(got, idx.queryAllPairs(small, grid))
