"""Batched calls over many maps (htrip_query_batch): one launch of the
persistent query kernel answers requests on indexes of different sizes, leaf
sides and k, and every result equals the same request made alone and the
reference's queryAllPairs / BfsOracle, bit for bit (tolerance 0)."""
import numpy as np
import pytest

from helpers import make_grid, viewpoints
from htrip_b200 import workloads as W
from oracle.ref import RefOracle, ref_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built (make -C oracle ref)")]


def _dev(b, g=2):
    from htrip_b200.minplus_oracle import HierarchyConfig, MinPlusOracle
    return MinPlusOracle(HierarchyConfig(tile_size_b=b, group_w=g, group_h=g))


MAPS = [("street", 64, 64, 8, 2, 1), ("maze", 128, 128, 16, 2, 2), ("rooms", 32, 32, 4, 2, 3),
        ("noise", 40, 24, 8, 2, 4), ("maze", 64, 64, 32, 2, 5), ("noise", 64, 64, 4, 4, 6),
        ("open", 16, 16, 16, 2, 7)]


def test_query_batch_equals_single_calls(gpu):
    from htrip_b200.minplus_oracle import Batch
    rng = np.random.default_rng(0)
    oracles, refs, grids = [], [], []
    for kind, rows, cols, b, g, seed in MAPS:
        grid = make_grid(kind, rows, cols, seed)
        dev = _dev(b, g)
        assert dev.build(grid)
        ref = RefOracle(b, g)
        ref.set_grid(grid)
        assert ref.build()
        oracles.append(dev)
        refs.append(ref)
        grids.append(grid)
    reqs, idx = [], []
    for i, (dev, grid) in enumerate(zip(oracles, grids)):
        for rep in range(2 if i % 2 == 0 else 1):   # some indexes appear twice
            k = int(rng.integers(1, 70))
            vps = viewpoints(grid, k, 100 * i + rep, include_blocked=1 + rep)
            reqs.append((dev, vps, grid))
            idx.append(i)
    reqs.append((oracles[0], np.zeros((0, 2), np.int32), grids[0]))   # empty request
    idx.append(0)
    batch = Batch()
    outs = batch.query(reqs)
    assert batch.lastKernelMs() > 0
    for (dev, vps, grid), out, i in zip(reqs, outs, idx):
        assert out.shape == (len(vps), len(vps))
        if len(vps) == 0:
            continue
        np.testing.assert_array_equal(out, dev.queryAllPairs(vps, grid))
        np.testing.assert_array_equal(out, refs[i].query(vps))
        np.testing.assert_array_equal(out, refs[i].bfs(vps))
    # the same batch again: the arena is reused and results do not change
    outs2 = batch.query(reqs)
    for a, b in zip(outs, outs2):
        np.testing.assert_array_equal(a, b)


def test_query_batch_mixed_tile_configs(gpu):
    """Requests that alone would pick different tile shapes (a crowded root
    child group vs a sparse one) share one launch with identical results."""
    from htrip_b200.minplus_oracle import Batch
    grid = W.maze_grid(256, 1, 3)
    dev = _dev(16)
    assert dev.build(grid)
    ref = RefOracle(16)
    ref.set_grid(grid)
    assert ref.build()
    dense = W.sample_free(grid[:64, :64], 200, 1)   # all viewpoints in one root child
    sparse = W.sample_free(grid, 9, 2)
    outs = Batch().query([(dev, dense, grid), (dev, sparse, grid)])
    np.testing.assert_array_equal(outs[0], ref.query(dense))
    np.testing.assert_array_equal(outs[1], ref.query(sparse))
    np.testing.assert_array_equal(outs[0], dev.queryAllPairs(dense, grid))


def test_open_batch_equals_sequential_calls(gpu):
    """htrip_open_batch over many maps (one index named twice) leaves every
    index, and its last_batch_stats, as the same calls made one by one and
    as the reference's onBatchCellsOpened."""
    from htrip_b200.minplus_oracle import Batch
    specs = [("street", 64, 64, 8, 2, 11, 40), ("maze", 128, 128, 16, 2, 12, 90),
             ("rooms", 32, 32, 4, 2, 13, 20), ("noise", 64, 64, 4, 4, 14, 50), ("maze", 64, 64, 32, 2, 15, 30)]
    batched, single, refs, grids, reqs, plan = [], [], [], [], [], []
    for kind, rows, cols, b, g, seed, m in specs:
        truth = make_grid(kind, rows, cols, seed)
        obs, cells = W.withheld_open(truth, m, seed)
        dev, one = _dev(b, g), _dev(b, g)
        assert dev.build(obs) and one.build(obs)
        ref = RefOracle(b, g)
        ref.set_grid(obs)
        assert ref.build()
        half = len(cells) // 2
        parts = [cells[:half], cells[half:]] if kind == "street" else [cells]
        batched.append(dev)
        single.append(one)
        refs.append(ref)
        grids.append(obs)
        plan.append(parts)
    stages = []   # per map: the grid as the caller holds it at each call
    for i, parts in enumerate(plan):
        grid = grids[i]
        stages.append([])
        for part in parts:
            grid[part[:, 0], part[:, 1]] = W.FREE   # the caller marks cells Free before each call
            stages[i].append(grid.copy())
            reqs.append((batched[i], part, stages[i][-1]))
    Batch().open(reqs)
    for i, parts in enumerate(plan):
        for part, grid in zip(parts, stages[i]):
            single[i].onBatchCellsOpened(part, grid)
            refs[i].set_cells(part, W.FREE)
            refs[i].open_batch(part)
        st_b, st_s = batched[i].last_batch_stats, single[i].last_batch_stats
        assert (st_b.n_touched_leaves, st_b.n_dirty_ancestors, st_b.n_pivots) == \
               (st_s.n_touched_leaves, st_s.n_dirty_ancestors, st_s.n_pivots) == refs[i].stats()
        assert batched[i].stateDigest() == single[i].stateDigest() == refs[i].digest()
        vps = viewpoints(grids[i], 20, i)
        np.testing.assert_array_equal(batched[i].queryAllPairs(vps, grids[i]), refs[i].query(vps))
