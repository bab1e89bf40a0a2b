"""Queries planned on the device (device-resident viewpoints, k <= 4096)
against the unmodified reference and against the host planner (host
viewpoints, batches, k > 4096): every tile shape, empty / blocked / duplicate
/ out-of-range viewpoints, H = 0, g = 4, b = 32, and once more with
HTRIP_QUERY_PLANNER=device so that host-buffer calls are planned on the
device too (tolerance 0: integer distances)."""
import os
import subprocess
import sys

import numpy as np
import pytest

from helpers import make_grid, viewpoints
from htrip_b200 import workloads as W
from oracle.ref import RefOracle, ref_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built (make -C oracle ref)")]


def _both(grid, b, g=2):
    from htrip_b200.minplus_oracle import HierarchyConfig, MinPlusOracle
    ref = RefOracle(b, g)
    ref.set_grid(grid)
    assert ref.build()
    dev = MinPlusOracle(HierarchyConfig(tile_size_b=b, group_w=g, group_h=g))
    assert dev.build(grid)
    return ref, dev


def _device_query(dev, vps, grid):
    """htrip_query_all_pairs_dev on device copies of the viewpoints and of
    their passability (as queryAllPairs decides it)."""
    import torch
    k = len(vps)
    rows, cols = grid.shape
    r, c = vps[:, 0], vps[:, 1]
    inside = (r >= 0) & (c >= 0) & (r < rows) & (c < cols)
    pf = np.zeros(k, dtype=np.uint8)
    pf[inside] = grid[r[inside], c[inside]] == W.FREE
    vd = torch.from_numpy(np.ascontiguousarray(vps, dtype=np.int32)).cuda()
    pd = torch.from_numpy(pf).cuda()
    od = torch.empty((k, k), dtype=torch.int16, device="cuda")
    torch.cuda.synchronize()
    dev.queryAllPairsDevice(vd.data_ptr(), pd.data_ptr(), k, od.data_ptr())
    dev.synchronize()
    return od.cpu().numpy().view(np.uint16)


CASES = [("maze", 64, 64, 8, 2, 1, 40), ("street", 128, 128, 16, 2, 2, 120), ("noise", 64, 64, 4, 4, 3, 60),
         ("rooms", 64, 64, 32, 2, 4, 50), ("noise", 40, 24, 8, 2, 5, 30), ("noise", 16, 16, 16, 2, 6, 25)]


@pytest.mark.parametrize("kind,rows,cols,b,g,seed,k", CASES)
def test_device_planned_query_matches_reference_and_host_planner(gpu, kind, rows, cols, b, g, seed, k):
    from htrip_b200.minplus_oracle import Batch
    grid = make_grid(kind, rows, cols, seed)
    ref, dev = _both(grid, b, g)
    vps = viewpoints(grid, k, seed, include_blocked=3)
    exp = ref.query(vps)
    np.testing.assert_array_equal(dev.queryAllPairs(vps, grid), exp)
    np.testing.assert_array_equal(_device_query(dev, vps, grid), exp)
    np.testing.assert_array_equal(_device_query(dev, vps, grid), exp)   # with the tile hint of the last call
    [via_batch] = Batch().query([(dev, vps, grid)])                     # host planner
    np.testing.assert_array_equal(via_batch, exp)


def test_edge_viewpoint_sets(gpu):
    grid = make_grid("maze", 64, 64, 11)
    ref, dev = _both(grid, 8)
    free = np.argwhere(grid == W.FREE).astype(np.int32)
    blocked = np.argwhere(grid != W.FREE).astype(np.int32)
    sets = {
        "one": free[:1],
        "two equal": np.array([free[5], free[5]], dtype=np.int32),
        "all blocked": blocked[:7],
        "out of range": np.array([[-1, 3], [3, -1], [64, 0], [0, 64], [1000, 1000]], dtype=np.int32),
        "duplicates": np.concatenate([free[:20], free[:20], free[10:15]]),
        "same leaf": free[(free[:, 0] < 8) & (free[:, 1] < 8)],
        "mixed": np.concatenate([free[::97], blocked[:3], [[-5, -5]], free[::131]]).astype(np.int32),
    }
    for name, vps in sets.items():
        exp = ref.query(vps)
        np.testing.assert_array_equal(dev.queryAllPairs(vps, grid), exp, err_msg=name)
        np.testing.assert_array_equal(_device_query(dev, vps, grid), exp, err_msg=name)


def test_every_tile_shape_through_the_device_planner(gpu):
    from htrip_b200.minplus_oracle import autotune_clear, autotune_export, autotune_import
    grid = W.maze_grid(256, 1, 5)
    ref, dev = _both(grid, 16)
    vps = W.sample_free(grid, 150, 7)
    exp = ref.query(vps)
    autotune_clear()
    dev.autotuneQuery(vps, grid, reps=2)
    key = " ".join(autotune_export().strip().split()[:4])
    for forced in range(4):
        autotune_import(f"{key} {forced}\n")
        np.testing.assert_array_equal(dev.queryAllPairs(vps, grid), exp, err_msg=f"tile shape {forced}")
        for _ in range(2):
            np.testing.assert_array_equal(_device_query(dev, vps, grid), exp, err_msg=f"tile shape {forced}")
    autotune_clear()


def test_largest_device_plan_and_first_host_plan(gpu):
    """With device-resident viewpoints k = 4096 is planned on the device and
    k = 4097 on the host; both equal the reference's BFS."""
    grid = make_grid("noise", 128, 128, 13)
    ref, dev = _both(grid, 8)
    free = np.argwhere(grid == W.FREE).astype(np.int32)
    rng = np.random.default_rng(13)
    for k in (4096, 4097):
        vps = free[rng.choice(len(free), size=k, replace=False)]
        got = dev.queryAllPairs(vps, grid)
        np.testing.assert_array_equal(got, ref.bfs(vps), err_msg=f"k={k}")
        np.testing.assert_array_equal(_device_query(dev, vps, grid), got, err_msg=f"k={k}")


def test_device_query_after_openings(gpu):
    truth = make_grid("street", 128, 128, 17)
    obs, cells = W.withheld_open(truth, 600, 17)
    ref, dev = _both(obs, 8)
    vps = viewpoints(truth, 64, 17)
    for part in np.array_split(cells, 3):
        obs[part[:, 0], part[:, 1]] = W.FREE
        ref.set_cells(part, W.FREE)
        ref.open_batch(part)
        dev.onBatchCellsOpened(part, obs)
        np.testing.assert_array_equal(_device_query(dev, vps, obs), ref.query(vps))


def test_host_buffer_calls_planned_on_the_device(gpu):
    """The tests above once more in a process where host-buffer calls are
    planned on the device as well."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, HTRIP_QUERY_PLANNER="device")
    r = subprocess.run([sys.executable, "-m", "pytest", os.path.abspath(__file__), "-q", "-x", "-p", "no:cacheprovider",
                        "-k", "not planned_on_the_device"], cwd=root, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
