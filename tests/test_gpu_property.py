"""Randomised invariants over opening streams, in the manner of the
reference's property-based test (apps/test_property_based.cpp:125-185:
seeds x steps on procedural rooms): after every opening step the all-pairs
matrix equals k x BFS on the current grid, the incremental query equals the
full one, and queryDistance equals the matrix entry for sampled pairs
(tolerance 0: integer distances)."""
import numpy as np
import pytest

from helpers import make_grid, viewpoints
from htrip_b200 import workloads as W
from oracle.ref import port_bfs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", range(6))
def test_opening_stream_invariants(gpu, seed):
    from htrip_b200.minplus_oracle import HierarchyConfig, IncrementalState, MinPlusOracle
    rng = np.random.default_rng(seed)
    truth = make_grid("rooms", 96, 96, seed)
    obs, cells = W.withheld_open(truth, 96 * 96 // 6, seed)
    b = (4, 8, 16)[seed % 3]
    dev = MinPlusOracle(HierarchyConfig(b, 2, 2))
    assert dev.build(obs)
    state = IncrementalState()
    vps = viewpoints(truth, 24, seed, include_blocked=2)
    for step, part in enumerate(np.array_split(cells, 20)):
        obs[part[:, 0], part[:, 1]] = W.FREE
        dev.onBatchCellsOpened(part, obs)
        full = dev.queryAllPairs(vps, obs)
        np.testing.assert_array_equal(full, port_bfs(obs, vps), err_msg=f"seed {seed} step {step}")
        np.testing.assert_array_equal(dev.queryAllPairsIncremental(vps, obs, state), full)
        free = [i for i in range(len(vps)) if obs[vps[i][0], vps[i][1]] == W.FREE]
        for _ in range(4):
            if len(free) < 2:
                break
            i, j = rng.choice(free, 2, replace=False)
            assert dev.queryDistance(tuple(vps[i]), tuple(vps[j]), obs) == full[i, j], (seed, step, i, j)
