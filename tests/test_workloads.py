"""Synthetic workload generators: seeded, deterministic, right shape and statistics."""
import hashlib

import numpy as np

from htrip_b200 import workloads as W


def h(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_street_grid_stats_and_determinism():
    g = W.street_grid(256, 1)
    assert g.shape == (256, 256) and g.dtype == np.uint8
    assert (g[0] == W.OBSTACLE).all() and (g[:, -1] == W.OBSTACLE).all()
    assert 0.55 < (g == W.FREE).mean() < 0.72
    assert h(g) == h(W.street_grid(256, 1))


def test_maze_is_perfect_and_connected():
    from scipy import ndimage
    g = W.maze_grid(64, 1, 3)
    free = g == W.FREE
    lab, n = ndimage.label(free, structure=[[0, 1, 0], [1, 1, 1], [0, 1, 0]])
    assert n == 1
    # a perfect maze on an n x n lattice has n*n cells and n*n - 1 passages
    assert free.sum() == 32 * 32 + 32 * 32 - 1


def test_sample_free_distinct_and_free():
    g = W.maze_grid(128, 1, 5)
    v = W.sample_free(g, 64, 9)
    assert len({(r, c) for r, c in v}) == 64
    assert (g[v[:, 0], v[:, 1]] == W.FREE).all()


def test_exploration_stream_orders_cells_by_ring():
    truth = W.street_grid(128, 4)
    obs, starts, batches = W.exploration_stream(truth, 4, 10, 64, 5, 7)
    assert len(batches) == 5 and all(len(b) == 64 for b in batches)
    cells = np.concatenate(batches)
    assert (obs[cells[:, 0], cells[:, 1]] == W.UNKNOWN).all()
    assert (truth[cells[:, 0], cells[:, 1]] == W.FREE).all()
